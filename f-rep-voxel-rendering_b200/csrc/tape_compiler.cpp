// Tape compiler (see tape_compiler.h). Each pass below names the reference
// routine whose semantics it reproduces; the data structures are this file's
// own (an index arena, hash-consing, a memoised structural order and an
// ordered free-slot set instead of shared_ptr DAGs and linear scans).
#include "tape_compiler.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <set>
#include <unordered_map>
#include <utility>

#include "frep/frep_math.h"

namespace frep {
namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;

int arity_of(uint8_t op) {
    if (op <= (uint8_t)ExprOp::CONST) return 0;
    if (op <= (uint8_t)ExprOp::SQRT) return 1;
    return 2;
}

bool is_axis(uint8_t op) { return op <= (uint8_t)ExprOp::T; }

uint32_t f2u(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// Float application of one operator with glm's min/max rule (the reference's
// csg::ApplyOperator, expression.cpp:108-149, used by constant folding).
float apply_op(uint8_t op, float a, float b) {
    switch ((ExprOp)op) {
        case ExprOp::SIN: return std::sin(a);
        case ExprOp::COS: return std::cos(a);
        case ExprOp::EXP: return std::exp(a);
        case ExprOp::NEG: return -a;
        case ExprOp::SQRT: return std::sqrt(a);
        case ExprOp::ADD: return a + b;
        case ExprOp::SUB: return a - b;
        case ExprOp::MUL: return a * b;
        case ExprOp::DIV: return a / b;
        case ExprOp::MIN: return (b < a) ? b : a;
        case ExprOp::MAX: return (a < b) ? b : a;
        default: return 0.0f;
    }
}

struct Arena {
    struct N {
        uint8_t op;
        uint32_t a, b;
        float c;
    };
    std::vector<N> nodes;

    uint32_t add(uint8_t op, uint32_t a = NONE, uint32_t b = NONE, float c = 0.0f) {
        nodes.push_back({op, a, b, c});
        return (uint32_t)nodes.size() - 1;
    }
    uint32_t konst(float c) { return add((uint8_t)ExprOp::CONST, NONE, NONE, c); }
    uint32_t neg(uint32_t a) { return add((uint8_t)ExprOp::NEG, a); }
    uint32_t bin(ExprOp op, uint32_t a, uint32_t b) { return add((uint8_t)op, a, b); }

    bool is_op(uint32_t i, ExprOp op) const { return nodes[i].op == (uint8_t)op; }
    bool is_const(uint32_t i) const { return nodes[i].op == (uint8_t)ExprOp::CONST; }
    bool is_const(uint32_t i, float v) const { return is_const(i) && nodes[i].c == v; }
    uint32_t in0(uint32_t i) const { return nodes[i].a; }
    uint32_t in1(uint32_t i) const { return nodes[i].b; }

    // Depth-first post-order from root, inputs in order, each node once
    // (csg::Expr::TopoIter, expression.cpp:298-314), iteratively.
    std::vector<uint32_t> topo(uint32_t root) const {
        std::vector<uint32_t> order;
        std::vector<uint8_t> seen(nodes.size(), 0);
        std::vector<std::pair<uint32_t, int>> stack;
        stack.push_back({root, 0});
        seen[root] = 1;
        while (!stack.empty()) {
            auto& top = stack.back();
            uint32_t n = top.first;
            int ar = arity_of(nodes[n].op);
            if (top.second < ar) {
                uint32_t child = top.second == 0 ? nodes[n].a : nodes[n].b;
                top.second++;
                if (!seen[child]) {
                    seen[child] = 1;
                    stack.push_back({child, 0});
                }
            } else {
                order.push_back(n);
                stack.pop_back();
            }
        }
        return order;
    }
};

// One constant-folding step (the reference's ConstantFoldStep,
// simplifier.cpp:31-95): all-constant inputs are evaluated; otherwise a fixed
// set of algebraic identities is applied. Recursion happens only where the
// reference recurses.
uint32_t fold_step(Arena& A, uint32_t e) {
    const uint8_t op = A.nodes[e].op;
    const int ar = arity_of(op);
    if (ar == 0) return e;
    const uint32_t i0 = A.in0(e);
    const uint32_t i1 = ar == 2 ? A.in1(e) : NONE;
    const bool c0 = A.is_const(i0), c1 = ar == 2 && A.is_const(i1);
    if (c0 && (ar == 1 || c1)) {
        return A.konst(apply_op(op, A.nodes[i0].c, ar == 2 ? A.nodes[i1].c : 0.0f));
    }
    switch ((ExprOp)op) {
        case ExprOp::ADD:
            if (A.is_const(i0, 0.0f)) return i1;
            if (A.is_const(i1, 0.0f)) return i0;
            if (A.is_op(i0, ExprOp::NEG) && A.is_op(i1, ExprOp::NEG))
                return A.neg(A.bin(ExprOp::ADD, i0, i1));
            if (A.is_op(i0, ExprOp::NEG)) return A.bin(ExprOp::SUB, i1, A.in0(i0));
            if (A.is_op(i1, ExprOp::NEG)) return A.bin(ExprOp::SUB, i0, A.in0(i1));
            break;
        case ExprOp::MUL:
            if (A.is_const(i0, 0.0f)) return A.konst(0.0f);
            if (A.is_const(i1, 0.0f)) return A.konst(0.0f);
            if (A.is_const(i0, 1.0f)) return i1;
            if (A.is_const(i1, 1.0f)) return i0;
            if (A.is_const(i0, -1.0f)) return fold_step(A, A.neg(i1));
            if (A.is_const(i1, -1.0f)) return fold_step(A, A.neg(i0));
            if (A.is_op(i0, ExprOp::NEG) || A.is_op(i1, ExprOp::NEG)) {
                uint32_t na = fold_step(A, A.neg(i0));
                uint32_t nb = fold_step(A, A.neg(i1));
                return A.bin(ExprOp::MUL, na, nb);
            }
            break;
        case ExprOp::SUB:
            if (A.is_const(i0, 0.0f)) return fold_step(A, A.neg(i1));
            if (A.is_const(i1, 0.0f)) return i0;
            if (A.is_op(i1, ExprOp::NEG)) return fold_step(A, A.bin(ExprOp::ADD, i0, A.in0(i1)));
            break;
        case ExprOp::DIV:
            if (A.is_const(i0, 0.0f)) return A.konst(0.0f);
            if (A.is_const(i1, 1.0f)) return i0;
            if (A.is_const(i1, -1.0f)) return fold_step(A, A.neg(i0));
            if (c1) return fold_step(A, A.bin(ExprOp::MUL, i0, A.konst(1.0f / A.nodes[i1].c)));
            break;
        case ExprOp::NEG:
            if (A.is_op(i0, ExprOp::NEG)) return A.in0(i0);
            if (A.is_op(i0, ExprOp::SUB)) return fold_step(A, A.bin(ExprOp::SUB, A.in1(i0), A.in0(i0)));
            break;
        default: break;
    }
    return e;
}

// Structural three-way order of two DAG nodes (the reference's
// ThreeWayCompare, simplifier.cpp:107-169), memoised on node pairs.
struct StructOrder {
    const Arena& A;
    std::unordered_map<uint64_t, int8_t> memo;
    explicit StructOrder(const Arena& arena) : A(arena) {}

    int cmp(uint32_t a, uint32_t b) {
        if (a == b) return 0;
        const auto& na = A.nodes[a];
        const auto& nb = A.nodes[b];
        if (na.op != nb.op) return na.op < nb.op ? -1 : 1;  // OpOrder == enum order
        if (na.op == (uint8_t)ExprOp::CONST) {
            if (na.c < nb.c) return -1;
            if (na.c > nb.c) return 1;
            return 0;
        }
        const int ar = arity_of(na.op);
        if (ar == 0) return 0;
        const uint64_t key = ((uint64_t)a << 32) | b;
        auto it = memo.find(key);
        if (it != memo.end()) return it->second;
        int r = cmp(na.a, nb.a);
        if (r == 0 && ar == 2) r = cmp(na.b, nb.b);
        memo.emplace(key, (int8_t)r);
        return r;
    }
};

struct KeyHash {
    size_t operator()(const std::pair<uint64_t, uint64_t>& k) const {
        return std::hash<uint64_t>()(k.first * 0x9E3779B97F4A7C15ull ^ k.second);
    }
};

}  // namespace

// Shortens the slot live ranges of constants in a wide tape, then reassigns
// slots. The reference compiler keeps a pooled constant in its slot from its
// first use to its last; in CSG tapes a handful of shared constants (0, 1,
// blend weights, repeated radii) are then live across most of the tape and
// hold ~40 % of the slots (the 256-primitive scene: 23 slots, 11 without
// them). Every slot costs each resident warp a shared-memory row on the
// device, so this pass gives a use that lies more than `dist` instructions
// after the constant's last load a CONST of its own right before it
// (~14 % more instructions, all CONSTs), and then allocates slots again in
// order: an instruction's operands that die there are freed first, the lowest
// free slot is taken, inputs x, y, z, t start in slots 0-3 and the result is
// written to slot 0. Values and their order are unchanged.
static void shorten_constant_ranges(CompiledTape* out, uint32_t dist) {
    const std::vector<uint64_t>& in = out->instrs;
    const uint32_t n = (uint32_t)in.size();
    if (n == 0) return;
    // SSA: value ids 0-3 are the inputs; an instruction of the new list at
    // position p defines value 4 + p.
    struct Ins {
        uint32_t op;
        uint32_t cbits;
        uint32_t src[2];
        uint32_t nsrc;
    };
    std::vector<Ins> outl;
    outl.reserve(n + n / 4);
    std::vector<uint32_t> slot_val(65536, 0xFFFFFFFFu);  // slot -> value held (old numbering of slots)
    for (uint32_t k = 0; k < 4; k++) slot_val[k] = k;
    std::vector<uint32_t> const_pos(n, 0);  // old index of a CONST -> position of its last load
    std::vector<int32_t> const_of_value;    // new value -> old CONST index (-1 otherwise)
    const_of_value.assign(4, -1);
    for (uint32_t i = 0; i < n; i++) {
        const uint64_t w = in[i];
        const uint32_t op = instr_op(w), o = instr_out(w);
        Ins x{op, 0u, {0u, 0u}, 0u};
        if (op == OP_CONST) {
            x.cbits = (uint32_t)(w >> 32);
        } else {
            const bool binary = op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_DIV || op == OP_MIN ||
                                op == OP_MAX;
            const uint32_t ss[2] = {instr_a(w), instr_b(w)};
            x.nsrc = binary ? 2 : 1;
            for (uint32_t k = 0; k < x.nsrc; k++) {
                uint32_t v = slot_val[ss[k]];
                const int32_t c = v < const_of_value.size() ? const_of_value[v] : -1;
                if (c >= 0 && outl.size() - const_pos[c] > dist) {
                    // reload the constant right before this use
                    Ins l{OP_CONST, (uint32_t)(in[c] >> 32), {0u, 0u}, 0u};
                    outl.push_back(l);
                    v = 4 + (uint32_t)outl.size() - 1;
                    const_of_value.push_back(c);
                    const_pos[c] = (uint32_t)outl.size() - 1;
                    slot_val[ss[k]] = v;
                    if (k == 0 && x.nsrc == 2 && ss[1] == ss[0]) slot_val[ss[1]] = v;
                }
                x.src[k] = v;
            }
        }
        outl.push_back(x);
        const uint32_t v = 4 + (uint32_t)outl.size() - 1;
        const_of_value.push_back(op == OP_CONST ? (int32_t)i : -1);
        if (op == OP_CONST) const_pos[i] = (uint32_t)outl.size() - 1;
        slot_val[o] = v;
    }
    const uint32_t result = slot_val[0];
    const uint32_t m = (uint32_t)outl.size();
    // liveness: last use position of every value (the result: past the end)
    std::vector<uint32_t> last(4 + m, 0xFFFFFFFFu);
    for (uint32_t p = 0; p < m; p++)
        for (uint32_t k = 0; k < outl[p].nsrc; k++) last[outl[p].src[k]] = p;
    last[result] = m;
    // allocation
    std::set<uint32_t> free_slots;
    std::vector<uint32_t> slot(4 + m, 0xFFFFFFFFu);
    uint32_t top = 4;
    for (uint32_t k = 0; k < 4; k++) {
        slot[k] = k;
        if (last[k] == 0xFFFFFFFFu) free_slots.insert(k);
    }
    std::vector<uint64_t> res;
    res.reserve(m);
    for (uint32_t p = 0; p < m; p++) {
        const Ins& x = outl[p];
        for (uint32_t k = 0; k < x.nsrc; k++)
            if (last[x.src[k]] == p) free_slots.insert(slot[x.src[k]]);
        uint32_t s;
        if (p + 1 == m) {
            s = 0;  // the result (slot 0 is free here: everything else is dead)
            free_slots.erase(0);
        } else if (!free_slots.empty()) {
            s = *free_slots.begin();
            free_slots.erase(free_slots.begin());
        } else {
            s = top++;
        }
        slot[4 + p] = s;
        if (last[4 + p] == 0xFFFFFFFFu) free_slots.insert(s);  // dead value (none in a compiled tape)
        if (x.op == OP_CONST) {
            float c;
            std::memcpy(&c, &x.cbits, 4);
            res.push_back(encode_const(s, c));
        } else {
            res.push_back(encode_instr(x.op, s, slot[x.src[0]], x.nsrc == 2 ? slot[x.src[1]] : 0));
        }
    }
    out->instrs.swap(res);
    out->n_slots = std::max<uint32_t>(top, 4);
}

std::string compile_tape(const DagNode* in, uint32_t n, uint32_t root, CompiledTape* out, uint32_t const_reload) {
    if (!in || n == 0 || root >= n) return "empty DAG or root out of range";
    Arena A;
    A.nodes.reserve((size_t)n * 4);
    for (uint32_t i = 0; i < n; i++) {
        const DagNode& d = in[i];
        if (d.op > (uint8_t)ExprOp::MAX) return "unknown operator at node " + std::to_string(i);
        const int ar = arity_of(d.op);
        if ((ar >= 1 && d.in0 >= i) || (ar == 2 && d.in1 >= i))
            return "DAG is not topologically ordered at node " + std::to_string(i);
        A.add(d.op, ar >= 1 ? d.in0 : NONE, ar == 2 ? d.in1 : NONE,
              d.op == (uint8_t)ExprOp::CONST ? d.constant : 0.0f);
    }

    // 1. ConstantFold (simplifier.cpp:97-104): rebuild every operator node over
    //    its folded inputs, then apply one fold step.
    uint32_t folded_root;
    {
        std::vector<uint32_t> order = A.topo(root);
        std::vector<uint32_t> map(A.nodes.size(), NONE);
        for (uint32_t e : order) {
            const auto N = A.nodes[e];
            const int ar = arity_of(N.op);
            if (ar == 0) { map[e] = e; continue; }
            uint32_t ne = A.add(N.op, map[N.a], ar == 2 ? map[N.b] : NONE);
            map[e] = fold_step(A, ne);
            if (map.size() < A.nodes.size()) map.resize(A.nodes.size(), NONE);
        }
        folded_root = map[root];
    }

    // 2. NormalForm (simplifier.cpp:172-201): rebuild operator nodes and order
    //    the operands of ADD/MUL/MIN/MAX. For two operands the reference's
    //    std::sort with "ThreeWayCompare(a, b) <= 0" swaps them exactly when
    //    cmp(second, first) <= 0.
    uint32_t nf_root;
    {
        std::vector<uint32_t> order = A.topo(folded_root);
        std::vector<uint32_t> map(A.nodes.size(), NONE);
        StructOrder so(A);
        for (uint32_t e : order) {
            const auto N = A.nodes[e];
            const int ar = arity_of(N.op);
            if (ar == 0) { map[e] = e; continue; }
            uint32_t a = map[N.a], b = ar == 2 ? map[N.b] : NONE;
            const ExprOp op = (ExprOp)N.op;
            if (op == ExprOp::ADD || op == ExprOp::MUL || op == ExprOp::MIN || op == ExprOp::MAX) {
                if (so.cmp(b, a) <= 0) std::swap(a, b);
            }
            map[e] = A.add(N.op, a, b);
            if (map.size() < A.nodes.size()) map.resize(A.nodes.size(), NONE);
        }
        nf_root = map[folded_root];
    }

    // 3. MergeDuplicates (simplifier.cpp:204-259): the first node of each
    //    structural class in TopoIter order represents it. Two constants are
    //    duplicates when they compare equal (so +0 and -0 merge, NaN never does).
    uint32_t merged_root;
    {
        std::vector<uint32_t> order = A.topo(nf_root);
        std::vector<uint32_t> map(A.nodes.size(), NONE);
        std::unordered_map<std::pair<uint64_t, uint64_t>, uint32_t, KeyHash> unique;
        for (uint32_t e : order) {
            const auto N = A.nodes[e];
            const int ar = arity_of(N.op);
            uint32_t a = ar >= 1 ? map[N.a] : NONE, b = ar == 2 ? map[N.b] : NONE;
            uint64_t k1 = (uint64_t)N.op, k2 = 0;
            if (N.op == (uint8_t)ExprOp::CONST) {
                if (N.c != N.c) return "NaN constant in the expression (the reference cannot pool it)";
                k2 = f2u(N.c == 0.0f ? 0.0f : N.c);
            } else if (ar >= 1) {
                k2 = ((uint64_t)a << 32) | (ar == 2 ? b : NONE);
            }
            auto key = std::make_pair(k1, k2);
            auto it = unique.find(key);
            if (it != unique.end()) {
                map[e] = it->second;
            } else {
                uint32_t ne = A.add(N.op, a, b, N.c);
                unique.emplace(key, ne);
                map[e] = ne;
            }
            if (map.size() < A.nodes.size()) map.resize(A.nodes.size(), NONE);
        }
        merged_root = map[nf_root];
    }
    if (is_axis(A.nodes[merged_root].op)) return "expression is a bare axis; the reference emits no instruction for it";

    // 4. TopoSort (tape.cpp:31-41).
    std::vector<uint32_t> exprs = A.topo(merged_root);
    std::unordered_map<uint32_t, uint32_t> node_idx;
    node_idx.reserve(exprs.size() * 2);
    for (uint32_t i = 0; i < exprs.size(); i++) node_idx[exprs[i]] = i;

    // 5. BuildConstantPool (tape.cpp:44-55), keyed by value equality.
    std::unordered_map<uint32_t, uint32_t> const_idx;
    std::vector<float> pool;
    for (uint32_t e : exprs) {
        if (A.is_const(e)) {
            float c = A.nodes[e].c;
            uint32_t key = f2u(c == 0.0f ? 0.0f : c);
            if (!const_idx.count(key)) {
                pool.push_back(c);
                const_idx[key] = (uint32_t)pool.size() - 1;
            }
        }
    }

    // 6. ComputeLiveliness (tape.cpp:66-79): index of the last user.
    std::vector<int64_t> live(exprs.size(), -1);
    for (uint32_t i = 0; i < exprs.size(); i++) {
        const auto& N = A.nodes[exprs[i]];
        const int ar = arity_of(N.op);
        if (ar >= 1) live[node_idx[N.a]] = std::max<int64_t>(live[node_idx[N.a]], i);
        if (ar == 2) live[node_idx[N.b]] = std::max<int64_t>(live[node_idx[N.b]], i);
    }

    // 7. BuildInstrs (tape.cpp:151-228): slots 0..3 start with X, Y, Z, T (or
    //    free when the axis is absent); inputs are released on their last use
    //    BEFORE the output takes the lowest free slot.
    std::vector<uint32_t> slot_owner(4, NONE);
    std::unordered_map<uint32_t, uint32_t> slot_of;  // node -> slot
    std::set<uint32_t> free_slots;
    for (uint32_t e : exprs) {
        uint8_t op = A.nodes[e].op;
        if (is_axis(op)) {
            slot_owner[op] = e;
            slot_of[e] = op;
        }
    }
    for (uint32_t s = 0; s < 4; s++)
        if (slot_owner[s] == NONE) free_slots.insert(s);

    auto release = [&](uint32_t node) {
        auto it = slot_of.find(node);
        if (it == slot_of.end()) return;  // already released (both inputs equal)
        slot_owner[it->second] = NONE;
        free_slots.insert(it->second);
        slot_of.erase(it);
    };
    auto acquire = [&](uint32_t node) -> uint32_t {
        uint32_t s;
        if (!free_slots.empty()) {
            s = *free_slots.begin();
            free_slots.erase(free_slots.begin());
        } else {
            s = (uint32_t)slot_owner.size();
            slot_owner.push_back(NONE);
        }
        slot_owner[s] = node;
        slot_of[node] = s;
        return s;
    };
    static const uint32_t kTapeOp[16] = {0, 0, 0, 0, OP_CONST, OP_SIN, OP_COS, OP_EXP, OP_NEG,
                                         OP_SQRT, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MIN, OP_MAX};

    out->instrs.clear();
    out->ref_instrs.clear();
    out->n_minmax = 0;
    out->uses_time = false;
    std::vector<uint32_t> ref_a;
    for (uint32_t i = 0; i < exprs.size(); i++) {
        const uint32_t e = exprs[i];
        const auto N = A.nodes[e];
        if (is_axis(N.op)) continue;
        const uint32_t top = kTapeOp[N.op];
        uint32_t sa = 0, sb = 0;
        const int ar = arity_of(N.op);
        if (ar >= 1) {
            sa = slot_of.at(N.a);
            if (ar == 2) sb = slot_of.at(N.b);
            if (live[node_idx[N.a]] == (int64_t)i) release(N.a);
            if (ar == 2 && live[node_idx[N.b]] == (int64_t)i) release(N.b);
            if (A.nodes[N.a].op == (uint8_t)ExprOp::T || (ar == 2 && A.nodes[N.b].op == (uint8_t)ExprOp::T))
                out->uses_time = true;
        }
        const uint32_t so = acquire(e);
        if (so > 0xFFFF) return "more than 65536 slots";
        if (top == OP_CONST) {
            out->instrs.push_back(encode_const(so, N.c));
            uint32_t key = f2u(N.c == 0.0f ? 0.0f : N.c);
            out->ref_instrs.push_back(OP_CONST | (so << 8) | (const_idx[key] << 16));
        } else {
            out->instrs.push_back(encode_instr(top, so, sa, sb));
            out->ref_instrs.push_back(top | (so << 8) | (sa << 16) | (sb << 24));
            if (top == OP_MIN || top == OP_MAX) out->n_minmax++;
        }
    }
    if (out->instrs.empty() || instr_out(out->instrs.back()) != 0)
        return "the result did not land in slot 0";
    out->n_slots = (uint32_t)slot_owner.size();
    out->const_pool = pool;
    out->fits_reference = out->n_slots <= 256 && pool.size() <= 256;
    if (!out->fits_reference) {
        // Beyond the reference's encoding the instruction stream is this
        // library's own: trade a few CONSTs for fewer slots.
        out->ref_instrs.clear();
        if (const_reload) shorten_constant_ranges(out, const_reload);
    }
    return "";
}

std::string import_reference_tape(const uint32_t* instrs, uint32_t n, const float* consts,
                                  uint32_t n_consts, CompiledTape* out) {
    if (!instrs || n == 0) return "empty tape";
    out->instrs.clear();
    out->ref_instrs.assign(instrs, instrs + n);
    out->const_pool.assign(consts, consts + n_consts);
    out->n_minmax = 0;
    out->uses_time = false;
    uint32_t max_slot = 3;
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t w = instrs[i];
        const uint32_t op = w & 0xFF, o = (w >> 8) & 0xFF, a = (w >> 16) & 0xFF, b = (w >> 24) & 0xFF;
        if (op >= OP_COUNT) return "unknown opcode at instruction " + std::to_string(i);
        max_slot = std::max(max_slot, o);
        if (op == OP_CONST) {
            if (a >= n_consts) return "constant index out of range at instruction " + std::to_string(i);
            out->instrs.push_back(encode_const(o, consts[a]));
            continue;
        }
        const bool binary = op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_DIV ||
                            op == OP_MIN || op == OP_MAX;
        max_slot = std::max(max_slot, a);
        if (binary) max_slot = std::max(max_slot, b);
        if (a == 3 || (binary && b == 3)) out->uses_time = true;
        out->instrs.push_back(encode_instr(op, o, a, binary ? b : 0));
        if (op == OP_MIN || op == OP_MAX) out->n_minmax++;
    }
    if (instr_out(out->instrs.back()) != 0) return "the last instruction does not write slot 0";
    out->n_slots = max_slot + 1;
    out->fits_reference = true;
    return "";
}

std::string import_wide_tape(const uint64_t* instrs, uint32_t n, CompiledTape* out) {
    if (!instrs || n == 0) return "empty tape";
    out->instrs.assign(instrs, instrs + n);
    out->ref_instrs.clear();
    out->const_pool.clear();
    out->fits_reference = false;
    out->n_minmax = 0;
    out->uses_time = false;
    uint32_t max_slot = 3;
    bool t_written = false;  // slot 3 holds T until an instruction writes it
    for (uint32_t i = 0; i < n; i++) {
        const uint64_t w = instrs[i];
        const uint32_t op = instr_op(w), o = instr_out(w);
        if (op >= OP_COUNT || (w & 0xFF00ull)) return "unknown opcode at instruction " + std::to_string(i);
        max_slot = std::max(max_slot, o);
        if (op != OP_CONST) {
            const bool binary = op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_DIV ||
                                op == OP_MIN || op == OP_MAX;
            const uint32_t a = instr_a(w), b = instr_b(w);
            max_slot = std::max(max_slot, a);
            if (binary) max_slot = std::max(max_slot, b);
            if (!t_written && (a == 3 || (binary && b == 3))) out->uses_time = true;
            if (op == OP_MIN || op == OP_MAX) out->n_minmax++;
        }
        if (o == 3) t_written = true;
    }
    if (instr_out(instrs[n - 1]) != 0) return "the last instruction does not write slot 0";
    if (max_slot > 0xFFFE) return "more than 65535 slots";
    out->n_slots = max_slot + 1;
    return "";
}

float eval_point_host(const std::vector<uint64_t>& instrs, uint32_t n_slots, float x, float y,
                      float z, float t) {
    std::vector<float> s(std::max<uint32_t>(n_slots, 4), 0.0f);
    s[0] = x;
    s[1] = y;
    s[2] = z;
    s[3] = t;
    for (uint64_t w : instrs) {
        const uint32_t op = instr_op(w), o = instr_out(w);
        if (op == OP_CONST) { s[o] = instr_const(w); continue; }
        const float a = s[instr_a(w)], b = s[instr_b(w)];
        float r = 0.0f;
        switch (op) {
            case OP_SIN: r = frep_sinf(a); break;
            case OP_COS: r = frep_cosf(a); break;
            case OP_ADD: r = a + b; break;
            case OP_SUB: r = a - b; break;
            case OP_MUL: r = a * b; break;
            case OP_DIV: r = a / b; break;
            case OP_MIN: r = (b < a) ? b : a; break;
            case OP_MAX: r = (a < b) ? b : a; break;
            case OP_EXP: r = frep_expf(a); break;
            case OP_NEG: r = -a; break;
            case OP_SQRT: r = std::sqrt(a); break;
            case OP_COPY: r = a; break;
        }
        s[o] = r;
    }
    return s[0];
}

}  // namespace frep
