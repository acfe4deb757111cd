// Builds two of the reference's demo shapes (vulkan/src/shapes.cpp:94-117,
// :48-66) through the C++ mirror header and prints their compiled tapes in the
// reference's encoding, one hex word per line, for tests/test_cpp_mirror.py.
#include <cstdio>
#include <string>

#include "frep/csg.hpp"

using namespace frep;

static csg::Expr OrganicBalls() {
    using namespace csg;
    auto s1 = Sphere({10, 0, 0}, 8);
    s1 = TranslateX(s1, 5 * Sin(T()));
    auto s2 = Sphere({-10, 0, 0}, 10);
    auto f = Min(Min(X(), Y()), Sqrt(X() * Y()) - 40);
    return f(s1, s2, Z(), T());
}

static csg::Expr Menger(int level) {
    using namespace csg;
    if (level <= 0) return Box({0, 0, 0}, {1, 1, 1});
    auto block = ScaleXYZ(Menger(level - 1), {1 / 3.0f, 1 / 3.0f, 1});
    auto menger = Empty();
    for (int x = 0; x < 3; x++)
        for (int y = 0; y < 3; y++)
            if (!(x == 1 && y == 1)) menger = Union(menger, TranslateXYZ(block, {x / 3.0f, y / 3.0f, 0}));
    return menger;
}

static csg::Expr MengerSponge(int level) {
    using namespace csg;
    auto shape = TranslateXYZ(Menger(level), {-0.5, -0.5, -0.5});
    shape = ScaleXYZ(shape, {30, 30, 10});
    return Diff(shape, Sphere({10, 10, 0}, 10));
}

static void dump(const char* name, const csg::Expr& e) {
    csg::Tape tape(e);
    std::printf("%s %u %u %zu\n", name, tape.InstructionCount(), tape.GetSlotCount(), tape.constantPool.size());
    for (const auto& i : tape.instructions)
        std::printf("%08x\n", (unsigned)i.op | (unsigned)i.outSlot << 8 | (unsigned)i.inSlotA << 16 |
                                  (unsigned)i.inSlotB << 24);
    std::printf("eval %.9g\n", (double)tape.Eval(1.5f, -2.0f, 0.25f, 0.5f));
}

int main() {
    dump("ref_OrganicBalls", OrganicBalls());
    dump("ref_MengerSponge_2", MengerSponge(2));
    return 0;
}
