// Test infrastructure: an extern "C" bridge to the REFERENCE's own CSG front end
// (vulkan/src/csg/{expression,simplifier,lib,tape}.cpp, vulkan/src/shapes.cpp and
// vulkan/src/utils/dot_graph.cpp), compiled from the reference tree by
// oracle/Makefile into oracle/_ref/libfrep_ref.so.
//
// It exists only so that tests can pin the product's tape compiler and the
// oracle's point interpreter against the reference's csg::Tape (tape.cpp:14-228)
// and csg::Tape::Eval (tape.cpp:274-302). Nothing in the product links it.
//
// Flat DAG convention (shared with the product's C-ABI, include/frep.h):
//   node i = (op, in0, in1, constant); op uses the csg::Operator numbering of
//   vulkan/include/csg/expression.h:14-22 (X=0 .. MAX=15); inputs refer to
//   earlier node indices; unused inputs are ignored.
//
// The reference asserts on 8-bit overflow (tape.cpp:223-227); this bridge is
// built with NDEBUG and reports overflow as a return code instead of aborting.
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "csg/expression.h"
#include "csg/lib.h"
#include "csg/tape.h"
#include "shapes.h"

namespace {

int arity(int op) {
    if (op <= 4) return 0;   // X Y Z T CONST
    if (op <= 9) return 1;   // SIN COS EXP NEG SQRT
    return 2;                // ADD SUB MUL DIV MIN MAX
}

csg::Expr build_expr(uint32_t n, const uint8_t* ops, const uint32_t* in0, const uint32_t* in1,
                     const float* consts, uint32_t root) {
    std::vector<csg::Expr> nodes(n);
    for (uint32_t i = 0; i < n; i++) {
        int op = ops[i];
        if (op == (int)csg::Operator::CONST) {
            nodes[i] = csg::Expr(consts[i]);
            continue;
        }
        std::vector<csg::Expr> inputs;
        if (arity(op) >= 1) inputs.push_back(nodes[in0[i]]);
        if (arity(op) >= 2) inputs.push_back(nodes[in1[i]]);
        nodes[i] = csg::Expr(std::make_shared<csg::Node>((csg::Operator)op, std::move(inputs)));
    }
    return nodes[root];
}

struct Flat {
    std::vector<uint8_t> ops;
    std::vector<uint32_t> in0, in1;
    std::vector<float> consts;
    uint32_t root = 0;
};

Flat flatten(const csg::Expr& e) {
    Flat f;
    std::unordered_map<csg::Node*, uint32_t> idx;
    e.TopoIter([&](csg::Expr x) {
        uint32_t id = (uint32_t)f.ops.size();
        idx[x.node.get()] = id;
        f.ops.push_back((uint8_t)x.node->op);
        uint32_t a = 0, b = 0;
        if (x.IsInputOp()) {
            if (x.node->inputs.size() >= 1) a = idx[x.node->inputs[0].node.get()];
            if (x.node->inputs.size() >= 2) b = idx[x.node->inputs[1].node.get()];
        }
        f.in0.push_back(a);
        f.in1.push_back(b);
        f.consts.push_back(x.IsConstantOp() ? x.node->constant : 0.0f);
    });
    f.root = idx[e.node.get()];
    return f;
}

}  // namespace

extern "C" {

// ---- tapes ---------------------------------------------------------------

// Compiles a flat DAG with csg::Tape. Returns an opaque handle, or null.
void* ref_tape_new(uint32_t n, const uint8_t* ops, const uint32_t* in0, const uint32_t* in1,
                   const float* consts, uint32_t root) {
    if (n == 0 || root >= n) return nullptr;
    csg::Expr e = build_expr(n, ops, in0, in1, consts, root);
    if (e.IsAxisOp()) return nullptr;  // the reference indexes instructions.back() of an empty tape
    return new csg::Tape(e);
}

void ref_tape_free(void* h) { delete (csg::Tape*)h; }

// counts = {instruction count, constant count, slot count}. Returns 0 when the
// tape fits the reference's 8-bit encoding, 1 when it overflowed it (the
// reference would have asserted at tape.cpp:223-227).
int ref_tape_info(void* h, uint32_t* counts) {
    auto* t = (csg::Tape*)h;
    counts[0] = (uint32_t)t->instructions.size();
    counts[1] = (uint32_t)t->constantPool.size();
    counts[2] = t->GetSlotCount();
    bool fits = counts[1] <= 256 && counts[2] <= 256 && !t->instructions.empty() &&
                t->instructions.back().outSlot == 0;
    return fits ? 0 : 1;
}

// Packed exactly as the reference uploads them (voxelizer.cpp:385-398,
// tape.comp:45-56): op | out << 8 | inA << 16 | inB << 24.
void ref_tape_instrs(void* h, uint32_t* out) {
    auto* t = (csg::Tape*)h;
    for (size_t i = 0; i < t->instructions.size(); i++) {
        const auto& in = t->instructions[i];
        out[i] = (uint32_t)in.op | ((uint32_t)in.outSlot << 8) | ((uint32_t)in.inSlotA << 16) |
                 ((uint32_t)in.inSlotB << 24);
    }
}

void ref_tape_consts(void* h, float* out) {
    auto* t = (csg::Tape*)h;
    if (!t->constantPool.empty()) std::memcpy(out, t->constantPool.data(), t->constantPool.size() * sizeof(float));
}

// csg::Tape::Eval at npts points; xyzt holds 4 floats per point.
void ref_tape_eval(void* h, const float* xyzt, uint32_t npts, float* out) {
    auto* t = (csg::Tape*)h;
    for (uint32_t i = 0; i < npts; i++)
        out[i] = t->Eval(xyzt[4 * i + 0], xyzt[4 * i + 1], xyzt[4 * i + 2], xyzt[4 * i + 3]);
}

// Recursive csg::Expr::Eval of the unsimplified DAG (expression.cpp:151-166).
void ref_dag_eval(uint32_t n, const uint8_t* ops, const uint32_t* in0, const uint32_t* in1,
                  const float* consts, uint32_t root, const float* xyzt, uint32_t npts, float* out) {
    csg::Expr e = build_expr(n, ops, in0, in1, consts, root);
    for (uint32_t i = 0; i < npts; i++)
        out[i] = e.Eval(xyzt[4 * i + 0], xyzt[4 * i + 1], xyzt[4 * i + 2], xyzt[4 * i + 3]);
}

// ---- reference demo shapes (vulkan/src/shapes.cpp) ------------------------

// Builds a named demo shape and returns an opaque csg::Expr*, or null.
void* ref_shape_new(const char* name, int level) {
    std::string s(name);
    csg::Expr e;
    if (s == "Screw") e = Screw();
    else if (s == "ElasticCube") e = ElasticCube();
    else if (s == "TangleCube") e = TangleCube();
    else if (s == "Morph") e = Morph();
    else if (s == "MengerSponge") e = MengerSponge(level);
    else if (s == "TwistedTower") e = TwistedTower(level, 0.3f, 0.8f);
    else if (s == "OrganicBalls") e = OrganicBalls();
    else return nullptr;
    return new csg::Expr(e);
}

void ref_expr_free(void* h) { delete (csg::Expr*)h; }

// Flattens an Expr in csg::Expr::TopoIter order. Call once with max_nodes = 0
// to learn the node count (the return value), then again with buffers.
uint32_t ref_expr_flatten(void* h, uint32_t max_nodes, uint8_t* ops, uint32_t* in0, uint32_t* in1,
                          float* consts, uint32_t* root) {
    Flat f = flatten(*(csg::Expr*)h);
    uint32_t n = (uint32_t)f.ops.size();
    if (max_nodes >= n) {
        std::memcpy(ops, f.ops.data(), n);
        std::memcpy(in0, f.in0.data(), n * 4);
        std::memcpy(in1, f.in1.data(), n * 4);
        std::memcpy(consts, f.consts.data(), n * 4);
        *root = f.root;
    }
    return n;
}

}  // extern "C"
