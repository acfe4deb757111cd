// frep/csg.hpp — C++ host mirror of the reference's interface for the F-rep
// voxelize + raytrace path, header-only, on top of the C-ABI in frep.h.
//
// Code written against the reference keeps its shape:
//   csg::Expr / csg::X() ... / operators / substitution e(x, y, z, t)
//                                  vulkan/include/csg/expression.h:14-118
//   csg::lib (Vector3, Sphere, Box, Union, Translate*, Scale*, Rotate*, ...)
//                                  vulkan/include/csg/lib.h:8-67
//   csg::Tape(Expr)                vulkan/include/csg/tape.h:12-83
//   VoxelStorage{gridDims, lowVertex, worldSize}.Init(ctx, shape)
//                                  vulkan/include/engine/voxel_storage.h:9-89
//   Voxelizer::Voxelize(stream, tapeTime)   vulkan/src/engine/voxelizer.cpp:429-440
//   Camera, Raytracer::Trace(stream, camera, tapeTime)
//                                  vulkan/include/engine/camera.h, raytracer.h
// Everything lives in namespace frep (`using namespace frep;` then reads
// `csg::Expr`, `csg::Sphere`, ...). Device handles replace the Vulkan ones:
// a frep_ctx for the device, a CUDA stream (void*) for the semaphores.
// Errors throw frep::Error carrying the frep_status and message.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <utility>
#include <vector>

#include "frep.h"

namespace frep {

class Error : public std::runtime_error {
public:
    Error(frep_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    frep_status status;
};

inline void check(frep_status s) {
    if (s != FREP_OK) throw Error(s, frep_last_error());
}

namespace csg {

// csg::Operator (expression.h:14-22).
enum class Operator : uint8_t { X, Y, Z, T, CONST, SIN, COS, EXP, NEG, SQRT, ADD, SUB, MUL, DIV, MIN, MAX };

class Expr;

struct Node {
    Operator op;
    std::vector<Expr> inputs;
    float constant = 0.0f;
    explicit Node(float c) : op(Operator::CONST), constant(c) {}
    Node(Operator o, std::vector<Expr>&& in) : op(o), inputs(std::move(in)) {}
};

// A handle on a DAG node, passed by value (expression.h:45-100).
class Expr {
public:
    std::shared_ptr<Node> node;

    Expr() = default;
    Expr(std::shared_ptr<Node> n) : node(std::move(n)) {}
    Expr(float c) : node(std::make_shared<Node>(c)) {}

    bool IsAxisOp() const { return node->op <= Operator::T; }
    bool IsConstantOp() const { return node->op == Operator::CONST; }
    bool IsConstantOp(float c) const { return IsConstantOp() && node->constant == c; }
    bool IsInputOp() const { return node->op >= Operator::SIN; }
    bool IsOp(Operator op) const { return node->op == op; }
    Expr operator[](size_t i) const { return node->inputs.at(i); }

    // Visits every node once, inputs before users, depth first
    // (expression.cpp:298-314), without recursion.
    void TopoIter(const std::function<void(Expr)>& f) const {
        std::unordered_set<Node*> seen;
        std::vector<std::pair<Expr, size_t>> stack;
        stack.push_back({*this, 0});
        seen.insert(node.get());
        while (!stack.empty()) {
            auto& top = stack.back();
            if (top.second < top.first.node->inputs.size()) {
                Expr child = top.first.node->inputs[top.second++];
                if (seen.insert(child.node.get()).second) stack.push_back({child, 0});
            } else {
                Expr e = top.first;
                stack.pop_back();
                f(e);
            }
        }
    }

    size_t NodeCount() const {
        size_t n = 0;
        TopoIter([&](Expr) { n++; });
        return n;
    }

    // Substitution of the axes (expression.cpp:281-295).
    Expr operator()(Expr newX, Expr newY, Expr newZ, Expr newT) const {
        std::unordered_map<Node*, Expr> mapped;
        TopoIter([&](Expr e) {
            Expr r;
            switch (e.node->op) {
                case Operator::X: r = newX; break;
                case Operator::Y: r = newY; break;
                case Operator::Z: r = newZ; break;
                case Operator::T: r = newT; break;
                case Operator::CONST: r = e; break;
                default: {
                    std::vector<Expr> in;
                    for (auto& c : e.node->inputs) in.push_back(mapped.at(c.node.get()));
                    r = Expr(std::make_shared<Node>(e.node->op, std::move(in)));
                }
            }
            mapped[e.node.get()] = r;
        });
        return mapped.at(node.get());
    }

    // The flat DAG that crosses the C-ABI (frep_dag).
    struct Flat {
        std::vector<uint8_t> ops;
        std::vector<uint32_t> in0, in1;
        std::vector<float> consts;
        uint32_t root = 0;
        frep_dag dag() const {
            return frep_dag{(uint32_t)ops.size(), ops.data(), in0.data(), in1.data(), consts.data(), root};
        }
    };
    Flat Flatten() const {
        Flat f;
        std::unordered_map<Node*, uint32_t> idx;
        TopoIter([&](Expr e) {
            idx[e.node.get()] = (uint32_t)f.ops.size();
            f.ops.push_back((uint8_t)e.node->op);
            const auto& in = e.node->inputs;
            f.in0.push_back(in.size() > 0 ? idx.at(in[0].node.get()) : 0u);
            f.in1.push_back(in.size() > 1 ? idx.at(in[1].node.get()) : 0u);
            f.consts.push_back(e.IsConstantOp() ? e.node->constant : 0.0f);
        });
        f.root = idx.at(node.get());
        return f;
    }
};

inline Expr MakeOp(Operator op, std::vector<Expr> in) { return Expr(std::make_shared<Node>(op, std::move(in))); }

inline Expr operator-(Expr e) { return MakeOp(Operator::NEG, {e}); }
inline Expr operator+(Expr a, Expr b) { return MakeOp(Operator::ADD, {a, b}); }
inline Expr operator-(Expr a, Expr b) { return MakeOp(Operator::SUB, {a, b}); }
inline Expr operator*(Expr a, Expr b) { return MakeOp(Operator::MUL, {a, b}); }
inline Expr operator/(Expr a, Expr b) { return MakeOp(Operator::DIV, {a, b}); }

inline Expr X() { return MakeOp(Operator::X, {}); }
inline Expr Y() { return MakeOp(Operator::Y, {}); }
inline Expr Z() { return MakeOp(Operator::Z, {}); }
inline Expr T() { return MakeOp(Operator::T, {}); }
inline Expr Constant(float x) { return Expr(x); }
inline Expr Sin(Expr e) { return MakeOp(Operator::SIN, {e}); }
inline Expr Cos(Expr e) { return MakeOp(Operator::COS, {e}); }
inline Expr Exp(Expr e) { return MakeOp(Operator::EXP, {e}); }
inline Expr Sqrt(Expr e) { return MakeOp(Operator::SQRT, {e}); }
inline Expr Min(Expr a, Expr b) { return MakeOp(Operator::MIN, {a, b}); }
inline Expr Max(Expr a, Expr b) { return MakeOp(Operator::MAX, {a, b}); }

// ---- lib.h ---------------------------------------------------------------------
struct Vector3 {
    Expr x, y, z;
    Vector3(Expr x_, Expr y_, Expr z_) : x(x_), y(y_), z(z_) {}
};
inline Vector3 operator+(Vector3 a, Vector3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vector3 operator-(Vector3 a, Vector3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vector3 operator*(Vector3 a, Vector3 b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline Vector3 operator/(Vector3 a, Vector3 b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
inline Vector3 operator-(Vector3 v) { return {-v.x, -v.y, -v.z}; }
inline Vector3 operator*(Vector3 v, Expr e) { return {v.x * e, v.y * e, v.z * e}; }
inline Vector3 operator*(Expr e, Vector3 v) { return {e * v.x, e * v.y, e * v.z}; }
inline Vector3 operator/(Vector3 v, Expr e) { return {v.x / e, v.y / e, v.z / e}; }

inline Expr Empty() { return Expr(1.0f); }
inline Vector3 Axes() { return {X(), Y(), Z()}; }
inline Expr Pi() { return Expr(3.14159265358979323846f); }
inline Expr Square(Expr x) { return x * x; }
inline Expr Abs(Expr x) { return Sqrt(Square(x)); }
inline Expr Pow(Expr x, uint32_t p) {
    if (p == 0) return Constant(1.0f);
    if (p == 1) return x;
    return p % 2 == 0 ? Square(Pow(x, p / 2)) : Square(Pow(x, p / 2)) * x;
}
inline Expr Dot(Vector3 a, Vector3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline Expr Norm(Vector3 a) { return Sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline Expr Norm2(Vector3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
inline Expr Dist(Vector3 a, Vector3 b) { return Norm(b - a); }
inline Expr Dist2(Vector3 a, Vector3 b) { return Norm2(b - a); }
inline Expr Union(Expr a, Expr b) { return Min(a, b); }
inline Expr Intersect(Expr a, Expr b) { return Max(a, b); }
inline Expr Complement(Expr a) { return -a; }
inline Expr Diff(Expr a, Expr b) { return Intersect(a, Complement(b)); }
inline Expr Sphere(Vector3 center, Expr radius) { return Dist2(Axes(), center) - Square(radius); }
inline Expr Box(Vector3 lo, Vector3 size) {
    Expr a = Square(X() - (lo.x + size.x / 2)) - Square(size.x / 2);
    Expr b = Square(Y() - (lo.y + size.y / 2)) - Square(size.y / 2);
    Expr c = Square(Z() - (lo.z + size.z / 2)) - Square(size.z / 2);
    return Intersect(a, Intersect(b, c));
}
inline Expr TranslateX(Expr a, Expr dx) { return a(X() - dx, Y(), Z(), T()); }
inline Expr TranslateY(Expr a, Expr dy) { return a(X(), Y() - dy, Z(), T()); }
inline Expr TranslateZ(Expr a, Expr dz) { return a(X(), Y(), Z() - dz, T()); }
inline Expr TranslateXYZ(Expr a, Vector3 d) { return a(X() - d.x, Y() - d.y, Z() - d.z, T()); }
inline Expr ScaleX(Expr a, Expr s) { return a(X() / s, Y(), Z(), T()); }
inline Expr ScaleY(Expr a, Expr s) { return a(X(), Y() / s, Z(), T()); }
inline Expr ScaleZ(Expr a, Expr s) { return a(X(), Y(), Z() / s, T()); }
inline Expr ScaleXYZ(Expr a, Expr s) { return a(X() / s, Y() / s, Z() / s, T()); }
inline Expr ScaleXYZ(Expr a, Vector3 s) { return a(X() / s.x, Y() / s.y, Z() / s.z, T()); }
inline Expr RotateX(Expr a, Expr angle) {
    Expr c = Cos(-angle), s = Sin(-angle);
    return a(X(), c * Y() - s * Z(), s * Y() + c * Z(), T());
}
inline Expr RotateY(Expr a, Expr angle) {
    Expr c = Cos(-angle), s = Sin(-angle);
    return a(c * X() + s * Z(), Y(), -s * X() + c * Z(), T());
}
inline Expr RotateZ(Expr a, Expr angle) {
    Expr c = Cos(-angle), s = Sin(-angle);
    return a(c * X() - s * Y(), s * X() + c * Y(), Z(), T());
}

// ---- Tape (tape.h:12-83) ---------------------------------------------------------
class Tape {
public:
    struct Instr {  // the reference's 4-byte instruction (tape.h:33-39)
        uint8_t op, outSlot, inSlotA, inSlotB;
    };
    std::vector<Instr> instructions;   // filled when the tape fits 8 bits
    std::vector<float> constantPool;

    Tape() = default;
    explicit Tape(const Expr& e) {
        Expr::Flat f = e.Flatten();
        frep_dag d = f.dag();
        frep_tape* t = nullptr;
        check(frep_tape_compile(&d, &t));
        handle_.reset(t, frep_tape_destroy);
        load();
    }
    uint32_t GetSlotCount() const { return info_.n_slots; }
    uint32_t InstructionCount() const { return info_.n_instr; }
    float Eval(float x, float y, float z, float t) const {
        float in[4] = {x, y, z, t}, out = 0.0f;
        check(frep_tape_eval(handle_.get(), in, 1, &out));
        return out;
    }
    const frep_tape* handle() const { return handle_.get(); }
    const frep_tape_info& info() const { return info_; }

private:
    std::shared_ptr<frep_tape> handle_;
    frep_tape_info info_{};
    void load() {
        check(frep_tape_get_info(handle_.get(), &info_));
        if (!info_.fits_reference) return;
        std::vector<uint32_t> words(info_.n_instr);
        constantPool.resize(info_.n_consts);
        std::vector<float> consts(info_.n_consts ? info_.n_consts : 1);
        check(frep_tape_get_reference(handle_.get(), words.data(), consts.data()));
        constantPool.assign(consts.begin(), consts.begin() + info_.n_consts);
        for (uint32_t w : words)
            instructions.push_back({(uint8_t)w, (uint8_t)(w >> 8), (uint8_t)(w >> 16), (uint8_t)(w >> 24)});
    }
};

}  // namespace csg

// ---- VoxelStorage / Voxelizer / Raytracer ------------------------------------------

// VoxelStorage (voxel_storage.h:9-89): fill gridDims, lowVertex, worldSize, then
// Init(ctx, shape) compiles the tape and creates the device tree.
class VoxelStorage {
public:
    std::vector<uint32_t> gridDims;
    float lowVertex[3] = {0, 0, 0};
    float worldSize = 1.0f;
    uint32_t gridLevels = 0;
    uint32_t fineGridDim = 0;
    std::vector<uint32_t> interiorNodeCount;
    csg::Tape tape;
    frep_voxelize_opts opts{FREP_ROUND_OUTWARD, 1, 0, 0, 0, 0};

    void Init(frep_ctx* ctx, const csg::Expr& shape) {
        gridLevels = (uint32_t)gridDims.size();
        fineGridDim = 1;
        for (uint32_t d : gridDims) fineGridDim *= d;
        interiorNodeCount.assign(gridLevels, 0);
        tape = csg::Tape(shape);
        frep_grid g{};
        g.levels = gridLevels;
        for (uint32_t i = 0; i < gridLevels && i < FREP_MAX_LEVELS; i++) g.dims[i] = gridDims[i];
        for (int k = 0; k < 3; k++) g.low_vertex[k] = lowVertex[k];
        g.world_size = worldSize;
        frep_tree* t = nullptr;
        check(frep_tree_create(ctx, &g, &opts, &t));
        tree_.reset(t, frep_tree_destroy);
        ctx_ = ctx;
    }
    frep_tree* tree() const { return tree_.get(); }
    frep_ctx* ctx() const { return ctx_; }
    // Reads the header back (interiorNodeCount, voxelizer.cpp:326-328).
    frep_tree_info Sync() {
        frep_tree_info info{};
        check(frep_tree_sync(tree_.get(), &info));
        for (uint32_t i = 0; i < gridLevels; i++) interiorNodeCount[i] = info.node_count[i];
        return info;
    }

private:
    std::shared_ptr<frep_tree> tree_;
    frep_ctx* ctx_ = nullptr;
};

class Voxelizer {
public:
    void Init(frep_ctx* ctx, VoxelStorage* voxels) {
        ctx_ = ctx;
        voxels_ = voxels;
    }
    // Enqueues every level pass on `stream` (no host round trip per level).
    void Voxelize(void* stream, float tapeTime) {
        check(frep_voxelize(ctx_, voxels_->tree(), voxels_->tape.handle(), tapeTime, stream));
    }
    // The same tree, copying from `prev` (the previous frame's storage, same
    // grid) every subtree that does not depend on the time
    // (frep_voxelize_reuse).
    void Voxelize(void* stream, float tapeTime, const VoxelStorage& prev) {
        check(frep_voxelize_reuse(ctx_, voxels_->tree(), prev.tree(), voxels_->tape.handle(), tapeTime, stream));
    }

private:
    frep_ctx* ctx_ = nullptr;
    VoxelStorage* voxels_ = nullptr;
};

// SceneBuilder (scene_builder.h:9-61): the reference builds a compactified
// tree on the CPU and uploads it; here BuildScene compacts the voxelized tree
// on the device (frep_tree_compact: empty children dropped and all-leaf
// children turned into leaf cells when `prune`, every level in depth-first
// preorder, no per-node child lists). Export / Import move it through host
// memory (e.g. a file) as one position-independent blob.
class SceneBuilder {
public:
    void Init(frep_ctx* ctx, VoxelStorage* voxels) {
        ctx_ = ctx;
        voxels_ = voxels;
    }
    void BuildScene(bool prune = true, void* stream = nullptr) {
        frep_compact* c = nullptr;
        check(frep_tree_compact(ctx_, voxels_->tree(), prune ? FREP_COMPACT_PRUNE : FREP_COMPACT_LAYOUT, stream, &c));
        compact_.reset(c, frep_compact_destroy);
    }
    std::vector<uint8_t> Export() const {
        uint64_t size = 0;
        check(frep_compact_export(compact_.get(), nullptr, 0, &size));
        std::vector<uint8_t> blob(size);
        check(frep_compact_export(compact_.get(), blob.data(), blob.size(), &size));
        return blob;
    }
    void Import(frep_ctx* ctx, const std::vector<uint8_t>& blob) {
        frep_compact* c = nullptr;
        check(frep_compact_import(ctx, blob.data(), blob.size(), &c));
        ctx_ = ctx;
        compact_.reset(c, frep_compact_destroy);
    }
    frep_compact_info Info() const {
        frep_compact_info info{};
        check(frep_compact_get_info(compact_.get(), &info));
        return info;
    }
    frep_compact* compact() const { return compact_.get(); }

private:
    frep_ctx* ctx_ = nullptr;
    VoxelStorage* voxels_ = nullptr;
    std::shared_ptr<frep_compact> compact_;
};

// Camera (camera.h:6-41); the library normalises forward / initialUp.
struct Camera {
    float position[3] = {0, 0, 40};
    float forward[3] = {0, 0, -1};
    float initialUp[3] = {0, 1, 0};
    float fovDeg = 45.0f;
    bool orthographic = false;
    float orthoWidth = 2.0f;
};

class Raytracer {
public:
    void Init(frep_ctx* ctx, VoxelStorage* voxels) {
        ctx_ = ctx;
        voxels_ = voxels;
        check(frep_lights_default(&lights_));
    }
    void SetBackgroundColor(float r, float g, float b) {
        lights_.background[0] = r;
        lights_.background[1] = g;
        lights_.background[2] = b;
        lights_.background[3] = 1.0f;
    }
    frep_lights& Lights() { return lights_; }
    // Renders into a device rgba8 buffer of width*height*4 bytes.
    void Trace(void* stream, const Camera& cam, float tapeTime, uint32_t width, uint32_t height,
               uint8_t* device_rgba8, frep_hit* device_hits = nullptr) {
        const frep_camera c = MakeCamera(cam, width, height);
        frep_image img{device_rgba8, device_hits};
        check(frep_render(ctx_, voxels_->tree(), &c, &lights_, tapeTime, &img, stream));
    }
    // The same frame from a compact tree (frep_render_compact).
    void Trace(void* stream, const SceneBuilder& scene, const Camera& cam, float tapeTime, uint32_t width,
               uint32_t height, uint8_t* device_rgba8, frep_hit* device_hits = nullptr) {
        const frep_camera c = MakeCamera(cam, width, height);
        frep_image img{device_rgba8, device_hits};
        check(frep_render_compact(ctx_, scene.compact(), &c, &lights_, tapeTime, &img, stream));
    }

private:
    static frep_camera MakeCamera(const Camera& cam, uint32_t width, uint32_t height) {
        frep_camera c{};
        for (int k = 0; k < 3; k++) {
            c.position[k] = cam.position[k];
            c.forward[k] = cam.forward[k];
            c.up[k] = cam.initialUp[k];
        }
        c.fov_deg = cam.fovDeg;
        c.ortho_width = cam.orthoWidth;
        c.projection = cam.orthographic ? FREP_ORTHOGRAPHIC : FREP_PERSPECTIVE;
        c.width = width;
        c.height = height;
        return c;
    }

    frep_ctx* ctx_ = nullptr;
    VoxelStorage* voxels_ = nullptr;
    frep_lights lights_{};
};

}  // namespace frep
