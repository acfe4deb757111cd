// A C++ host using the autotuner through the C-ABI (include/frep.h), as a
// caller replacing Voxelizer::Voxelize (vulkan/src/engine/voxelizer.cpp:
// 429-440) for a batch would.
//   autotune_host table <in.json> <out.json>   (no GPU) load a tuning file,
//       print every lookup, save it again.
//   autotune_host tune <out.json>              (GPU) tune a small batch twice
//       and print both tunings' choices, which must agree.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "frep/csg.hpp"

using namespace frep;

static void print_choices(const frep_tuning* t) {
    const uint32_t res[5] = {64, 128, 256, 512, 1024};
    const uint32_t sizes[4] = {100, 500, 2000, 9000};
    for (uint32_t r : res)
        for (uint32_t n : sizes) {
            uint32_t levels = 0, k = 0, dims[FREP_MAX_LEVELS] = {};
            check(frep_tuning_lookup(t, r, n, &levels, dims, &k));
            std::printf("%u %u %u", r, n, levels);
            for (uint32_t i = 0; i < levels; i++) std::printf(" %u", dims[i]);
            std::printf(" k%u\n", k);
        }
    uint32_t iw = 0, pw = 0;
    check(frep_tuning_warps(t, &iw, &pw));
    std::printf("warps %u %u\n", iw, pw);
}

static csg::Expr scene(int i) {
    using namespace csg;
    Expr e = Sphere({0.1f * i, 0, 0}, 0.5f);
    for (int k = 0; k < 4 + 3 * i; k++) {
        const float a = 0.37f * (float)(k + 1) + 0.11f * (float)i;
        e = Min(e, Sphere({std::sin(a), std::cos(1.3f * a), std::sin(2.1f * a)}, 0.15f + 0.01f * (float)(k % 5)));
    }
    return e;
}

int main(int argc, char** argv) {
    if (argc >= 4 && std::strcmp(argv[1], "table") == 0) {
        frep_tuning* t = nullptr;
        check(frep_tuning_create(&t));
        check(frep_tuning_load(t, argv[2], "NVIDIA B200"));
        print_choices(t);
        check(frep_tuning_save(t, argv[3], "NVIDIA B200"));
        frep_tuning_destroy(t);
        return 0;
    }
    if (argc >= 3 && std::strcmp(argv[1], "tune") == 0) {
        frep_ctx* ctx = nullptr;
        check(frep_ctx_create(0, 8ull << 30, &ctx));
        std::vector<csg::Tape> tapes;
        std::vector<const frep_tape*> ptrs;
        std::vector<uint32_t> res;
        std::vector<frep_camera> cams;
        for (int i = 0; i < 6; i++) {
            tapes.emplace_back(scene(i));
            res.push_back(i % 2 ? 128 : 64);
        }
        for (auto& t : tapes) ptrs.push_back(t.handle());
        for (int i = 0; i < 6; i++) {
            frep_camera c{};
            const float a = 0.7f * (float)i;
            c.position[0] = 4.0f * std::cos(a);
            c.position[1] = 1.0f;
            c.position[2] = 4.0f * std::sin(a);
            for (int k = 0; k < 3; k++) c.forward[k] = -c.position[k];
            c.up[1] = 1.0f;
            c.fov_deg = 60.0f;
            c.width = c.height = 128;
            cams.push_back(c);
        }
        frep_lights lights;
        check(frep_lights_default(&lights));
        const float low[3] = {-1.5f, -1.5f, -1.5f};
        frep_autotune_opts o{};
        o.per_class = 3;
        o.reps = 5;
        o.width = o.height = 128;
        o.margin = 0.10f;  // tiny scenes time in tens of microseconds: a wider margin
        for (int round = 0; round < 2; round++) {
            frep_tuning* t = nullptr;
            check(frep_tuning_create(&t));
            if (round == 1) check(frep_tuning_load(t, argv[2], "NVIDIA B200"));
            o.refine = round == 1;  // re-time every class with the saved choice as the incumbent
            check(frep_batch_autotune(ctx, ptrs.data(), res.data(), cams.data(), 6, &lights, low, 3.0f, &o, t));
            std::printf("tuning %d\n", round);
            print_choices(t);
            if (round == 0) check(frep_tuning_save(t, argv[2], "NVIDIA B200"));
            frep_tuning_destroy(t);
        }
        frep_ctx_destroy(ctx);
        return 0;
    }
    std::fprintf(stderr, "usage: autotune_host table <in> <out> | tune <out>\n");
    return 2;
}
