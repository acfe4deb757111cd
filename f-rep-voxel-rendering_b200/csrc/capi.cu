// C-ABI of the library (include/frep.h): tapes, device contexts, trees,
// voxelization and rendering. Host code only; kernels live in voxelizer.cu and
// raytracer.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "capi_internal.h"

namespace frep {
namespace detail {

thread_local std::string g_error;

frep_status fail(frep_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return s;
}

frep_status cuda_fail(cudaError_t e, const char* what) {
    return fail(FREP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

}  // namespace detail
}  // namespace frep

using frep::detail::align_up;
using frep::detail::cuda_fail;
using frep::detail::fail;
using frep::detail::g_error;

extern "C" {

const char* frep_last_error(void) { return g_error.c_str(); }
const char* frep_version(void) { return "frep-b200 0.1 (sm_100a)"; }

// ---- tapes -------------------------------------------------------------------

frep_status frep_tape_compile(const frep_dag* dag, frep_tape** out) { return frep_tape_compile_opts(dag, nullptr, out); }

frep_status frep_tape_compile_opts(const frep_dag* dag, const frep_tape_opts* opts, frep_tape** out) {
    if (!dag || !out || !dag->ops || !dag->in0 || !dag->in1 || !dag->consts)
        return fail(FREP_ERR_INVALID_ARG, "frep_tape_compile: null argument");
    const uint32_t reload = !opts || opts->const_reload_distance == 0 ? 8u
                            : opts->const_reload_distance == 0xFFFFFFFFu ? 0u : opts->const_reload_distance;
    std::vector<frep::DagNode> nodes(dag->n_nodes);
    for (uint32_t i = 0; i < dag->n_nodes; i++)
        nodes[i] = {dag->ops[i], dag->in0[i], dag->in1[i], dag->consts[i]};
    auto* t = new frep_tape();
    std::string err = frep::compile_tape(nodes.data(), dag->n_nodes, dag->root, &t->ct, reload);
    if (!err.empty()) {
        delete t;
        return fail(FREP_ERR_COMPILE, "frep_tape_compile: %s", err.c_str());
    }
    t->build_record();
    *out = t;
    return FREP_OK;
}

frep_status frep_tape_from_reference(const uint32_t* instrs, uint32_t n_instr, const float* consts,
                                     uint32_t n_consts, frep_tape** out) {
    if (!instrs || !out || (n_consts && !consts))
        return fail(FREP_ERR_INVALID_ARG, "frep_tape_from_reference: null argument");
    auto* t = new frep_tape();
    std::string err = frep::import_reference_tape(instrs, n_instr, consts, n_consts, &t->ct);
    if (!err.empty()) {
        delete t;
        return fail(FREP_ERR_INVALID_ARG, "frep_tape_from_reference: %s", err.c_str());
    }
    t->build_record();
    *out = t;
    return FREP_OK;
}

frep_status frep_tape_from_wide(const uint64_t* instrs, uint32_t n_instr, frep_tape** out) {
    if (!instrs || !out) return fail(FREP_ERR_INVALID_ARG, "frep_tape_from_wide: null argument");
    auto* t = new frep_tape();
    std::string err = frep::import_wide_tape(instrs, n_instr, &t->ct);
    if (!err.empty()) {
        delete t;
        return fail(FREP_ERR_INVALID_ARG, "frep_tape_from_wide: %s", err.c_str());
    }
    t->build_record();
    *out = t;
    return FREP_OK;
}

frep_status frep_tape_get_info(const frep_tape* tape, frep_tape_info* info) {
    if (!tape || !info) return fail(FREP_ERR_INVALID_ARG, "frep_tape_get_info: null argument");
    info->n_instr = (uint32_t)tape->ct.instrs.size();
    info->n_slots = tape->ct.n_slots;
    info->n_consts = (uint32_t)tape->ct.const_pool.size();
    info->n_minmax = tape->ct.n_minmax;
    info->fits_reference = tape->ct.fits_reference ? 1u : 0u;
    info->uses_time = tape->ct.uses_time ? 1u : 0u;
    return FREP_OK;
}

frep_status frep_tape_get_instrs(const frep_tape* tape, uint64_t* out, uint32_t cap) {
    if (!tape || !out) return fail(FREP_ERR_INVALID_ARG, "frep_tape_get_instrs: null argument");
    if (cap < tape->ct.instrs.size()) return fail(FREP_ERR_INVALID_ARG, "frep_tape_get_instrs: capacity too small");
    std::memcpy(out, tape->ct.instrs.data(), tape->ct.instrs.size() * 8);
    return FREP_OK;
}

frep_status frep_tape_get_reference(const frep_tape* tape, uint32_t* instrs, float* consts) {
    if (!tape || !instrs || !consts) return fail(FREP_ERR_INVALID_ARG, "frep_tape_get_reference: null argument");
    if (!tape->ct.fits_reference)
        return fail(FREP_ERR_UNSUPPORTED, "tape has %u slots / %zu constants; the 8-bit encoding holds 256",
                    tape->ct.n_slots, tape->ct.const_pool.size());
    std::memcpy(instrs, tape->ct.ref_instrs.data(), tape->ct.ref_instrs.size() * 4);
    if (!tape->ct.const_pool.empty())
        std::memcpy(consts, tape->ct.const_pool.data(), tape->ct.const_pool.size() * 4);
    return FREP_OK;
}

frep_status frep_tape_eval(const frep_tape* tape, const float* xyzt, uint32_t n, float* out) {
    if (!tape || (n && (!xyzt || !out))) return fail(FREP_ERR_INVALID_ARG, "frep_tape_eval: null argument");
    for (uint32_t i = 0; i < n; i++)
        out[i] = frep::eval_point_host(tape->ct.instrs, tape->ct.n_slots, xyzt[4 * i], xyzt[4 * i + 1],
                                       xyzt[4 * i + 2], xyzt[4 * i + 3]);
    return FREP_OK;
}

void frep_tape_destroy(frep_tape* tape) { delete tape; }

// ---- context -----------------------------------------------------------------

frep_status frep_ctx_create(int device, uint64_t hbm_budget_bytes, frep_ctx** out) {
    if (!out) return fail(FREP_ERR_INVALID_ARG, "frep_ctx_create: null argument");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) return fail(FREP_ERR_CUDA, "frep_ctx_create: no CUDA device (%s)", cudaGetErrorString(e));
    if (device < 0 || device >= n) return fail(FREP_ERR_INVALID_ARG, "frep_ctx_create: device %d of %d", device, n);
    FREP_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    FREP_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) return fail(FREP_ERR_UNSUPPORTED, "frep_ctx_create: device is sm_%d%d; this build is sm_100a", prop.major, prop.minor);
    size_t free_b = 0, total_b = 0;
    FREP_CUDA(cudaMemGetInfo(&free_b, &total_b));
    auto* c = new frep_ctx();
    c->device = device;
    c->budget = hbm_budget_bytes ? hbm_budget_bytes : (uint64_t)(free_b * 0.9);
    c->sm_count = prop.multiProcessorCount;
    *out = c;
    return FREP_OK;
}

void frep_ctx_destroy(frep_ctx* ctx) { delete ctx; }

frep_status frep_ctx_memory(const frep_ctx* ctx, uint64_t* used, uint64_t* budget) {
    if (!ctx) return fail(FREP_ERR_INVALID_ARG, "frep_ctx_memory: null argument");
    if (used) *used = ctx->used;
    if (budget) *budget = ctx->budget;
    return FREP_OK;
}

// ---- trees -------------------------------------------------------------------

static frep_status validate_grid(const frep_grid* g) {
    if (g->levels == 0 || g->levels > FREP_MAX_LEVELS)
        return fail(FREP_ERR_INVALID_ARG, "grid: levels must be 1..8 (got %u)", g->levels);
    for (uint32_t l = 0; l < g->levels; l++) {
        const uint32_t d = g->dims[l];
        // Masks are whole 32-bit words and a warp owns one word (voxelizer.cpp:270 asserts dim^3 % 64).
        if (d < 4 || d > 32 || d % 4 != 0)
            return fail(FREP_ERR_INVALID_ARG, "grid: dims[%u] = %u must be a multiple of 4 in 4..32", l, d);
    }
    if (!(g->world_size > 0.0f)) return fail(FREP_ERR_INVALID_ARG, "grid: world_size must be > 0");
    return FREP_OK;
}

}  // extern "C"

namespace frep {
namespace dev {

// Writes a tree's static header and its self pointer (trees in caller
// memory). The header travels as a kernel parameter: a cudaMemcpyAsync from
// pageable host memory may wait for the stream's earlier work.
__global__ void tree_header_write_kernel(const TreeHeader h, TreeHeader* dst, TreeHeader** self) {
    *dst = h;
    *self = dst;
}

}  // namespace dev

namespace detail {

uint64_t tree_external_bytes(uint64_t node_words, uint64_t tape_words) {
    return align_up(sizeof(dev::TreeHeader), 256) + 256 + align_up(node_words * 4, 256) + tape_words * 8;
}

// Creates a tree; with `ext` its header, work prefix and pools are carved
// from that caller-owned device memory (the serving loop's arena) instead of
// cudaMalloc'd, the device header is written later (write_tree_header, on
// the stream that first uses the tree), and nothing is charged to the
// context's budget.
frep_status tree_create_impl(frep_ctx* ctx, const frep_grid* grid, const frep_voxelize_opts* opts, uint8_t* ext,
                             uint64_t ext_bytes, cudaStream_t stream, frep_tree** out) {
    if (!ctx || !grid || !out) return fail(FREP_ERR_INVALID_ARG, "frep_tree_create: null argument");
    frep_status s = validate_grid(grid);
    if (s != FREP_OK) return s;
    FREP_CUDA(cudaSetDevice(ctx->device));
    auto* t = new frep_tree();
    t->external = ext != nullptr;
    t->ctx = ctx;
    t->grid = *grid;
    if (opts) t->opts = *opts;
    else { t->opts.rounding = FREP_ROUND_OUTWARD; t->opts.shorten = 1; }
    if (t->opts.rounding > FREP_ROUND_HYBRID) {
        delete t;
        return fail(FREP_ERR_INVALID_ARG, "opts.rounding must be FREP_ROUND_NEAREST, _OUTWARD or _HYBRID");
    }
    {
        const uint32_t dl = grid->dims[grid->levels - 1];
        const uint32_t k = t->opts.point_cells_per_lane;
        if (k != 0 && k != 2 && k != 4 && k != 8) {
            delete t;
            return fail(FREP_ERR_INVALID_ARG, "opts.point_cells_per_lane must be 0, 2, 4 or 8");
        }
        if (k && (dl * dl * dl / 32) % k != 0) {
            delete t;
            return fail(FREP_ERR_INVALID_ARG, "opts.point_cells_per_lane = %u does not divide the last level's %u mask "
                        "words (4 and 8 need a last-level dim that is a multiple of 8)",
                        k, dl * dl * dl / 32);
        }
        t->point_k = k ? (int)k : frep::point_k_for(dl);
        // Alone, a tree takes 8 cells per lane where its nodes allow (the
        // 2048^3 scene's last-level pass: 17.2 ms with 4, 15.9 ms with 8);
        // batches group their last-level passes by 4 or 2.
        t->plain_k = k ? (int)k : ((dl * dl * dl / 32) % 8 == 0 ? 8 : t->point_k);
    }
    // Cell sizes by successive division (voxelizer.cpp:209-216).
    float cs = grid->world_size;
    uint64_t dense_nodes = 1, dense_words = 0;
    for (uint32_t l = 0; l < grid->levels; l++) {
        cs /= (float)grid->dims[l];
        t->cell_size[l] = cs;
        t->node_size[l] = frep::dev::node_words(grid->dims[l], l == grid->levels - 1);
        dense_words += dense_nodes * t->node_size[l];
        const uint64_t d3 = (uint64_t)grid->dims[l] * grid->dims[l] * grid->dims[l];
        dense_nodes = std::min<uint64_t>(dense_nodes * d3, 1ull << 40);
        dense_words = std::min<uint64_t>(dense_words, 1ull << 44);
    }
    const uint64_t avail = ext ? ext_bytes : (ctx->budget > ctx->used ? ctx->budget - ctx->used : 0);
    if (ext && (!t->opts.node_words || !t->opts.tape_words)) {
        delete t;
        return fail(FREP_ERR_INVALID_ARG, "tree in caller memory: pool sizes must be given");
    }
    t->node_cap = t->opts.node_words ? t->opts.node_words : std::min<uint64_t>(dense_words, avail / 4 / 4);
    t->tape_cap = t->opts.tape_words ? t->opts.tape_words : avail / 4 / 8;
    t->tape_cap = std::min<uint64_t>(t->tape_cap, 0xFFFFFFF0ull);  // tape indices are u32
    const uint64_t bytes = ext ? tree_external_bytes(t->node_cap, t->tape_cap)
                               : t->node_cap * 4 + t->tape_cap * 8 + sizeof(frep::dev::TreeHeader);
    if (t->node_cap < t->node_size[0] || bytes > avail) {
        delete t;
        return fail(FREP_ERR_OOM, "frep_tree_create: %llu bytes requested, %llu left in the budget",
                    (unsigned long long)bytes, (unsigned long long)avail);
    }
    cudaError_t e = cudaSuccess;
    if (ext) {
        t->hdr = reinterpret_cast<frep::dev::TreeHeader*>(ext);
        t->d_small = reinterpret_cast<unsigned long long*>(ext + align_up(sizeof(frep::dev::TreeHeader), 256));
        t->nodes = reinterpret_cast<uint32_t*>(reinterpret_cast<uint8_t*>(t->d_small) + 256);
        t->tapes = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(t->nodes) + align_up(t->node_cap * 4, 256));
    } else {
        e = cudaMalloc(&t->hdr, sizeof(frep::dev::TreeHeader));
        if (e == cudaSuccess) e = cudaMalloc(&t->d_small, 64);
        if (e == cudaSuccess) e = cudaMalloc(&t->nodes, t->node_cap * 4);
        if (e == cudaSuccess) e = cudaMalloc(&t->tapes, t->tape_cap * 8);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->upload_done, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (!ext) {
            cudaFree(t->hdr);
            cudaFree(t->d_small);
            cudaFree(t->nodes);
            cudaFree(t->tapes);
        }
        delete t;
        return fail(FREP_ERR_OOM, "frep_tree_create: cudaMalloc failed (%s)", cudaGetErrorString(e));
    }
    // The header's static part: where the pools are and the grid.
    frep::dev::TreeHeader h{};
    h.nodes = t->nodes;
    h.tapes = t->tapes;
    h.node_cap = t->node_cap;
    h.tape_cap = t->tape_cap;
    h.levels = grid->levels;
    h.shorten = t->opts.shorten;
    h.share_tapes = t->opts.separate_tapes ? 0u : 1u;
    for (uint32_t l = 0; l < grid->levels; l++) {
        h.dims[l] = grid->dims[l];
        h.node_size[l] = t->node_size[l];
        h.cell_size[l] = t->cell_size[l];
    }
    for (int k = 0; k < 3; k++) h.low[k] = grid->low_vertex[k];
    h.point_k = (uint32_t)t->point_k;
    t->d_self = reinterpret_cast<frep::dev::TreeHeader**>(t->d_small);
    t->d_prefix = t->d_small + 1;
    t->d_cursor = t->d_small + 3;
    cudaError_t ce = cudaSuccess;
    if (ext) {  // written later by write_tree_header
        t->pending_hdr = h;
        t->hdr_pending = true;
    } else {
        ce = cudaMemcpy(t->hdr, &h, sizeof(h), cudaMemcpyHostToDevice);
        if (ce == cudaSuccess) ce = cudaMemcpy(t->d_self, &t->hdr, sizeof(void*), cudaMemcpyHostToDevice);
    }
    if (ce != cudaSuccess) {
        if (!ext) {
            cudaFree(t->hdr);
            cudaFree(t->d_small);
            cudaFree(t->nodes);
            cudaFree(t->tapes);
        }
        cudaEventDestroy(t->upload_done);
        delete t;
        return cuda_fail(ce, "frep_tree_create: header upload");
    }
    if (ext) {
        t->stream = stream;
    } else {
        t->bytes = bytes;
        ctx->used += bytes;
    }
    *out = t;
    return FREP_OK;
}

frep_status write_tree_header(frep_tree* t, cudaStream_t stream) {
    if (!t->hdr_pending) return FREP_OK;
    frep::dev::tree_header_write_kernel<<<1, 1, 0, stream>>>(t->pending_hdr, t->hdr, t->d_self);
    FREP_CUDA(cudaGetLastError());
    t->hdr_pending = false;
    return FREP_OK;
}

}  // namespace detail
}  // namespace frep

extern "C" {

frep_status frep_tree_create(frep_ctx* ctx, const frep_grid* grid, const frep_voxelize_opts* opts,
                             frep_tree** out) {
    return frep::detail::tree_create_impl(ctx, grid, opts, nullptr, 0, nullptr, out);
}

void frep_tree_destroy(frep_tree* t) {
    if (!t) return;
    cudaSetDevice(t->ctx->device);
    if (!t->external) {
        // (a tree in caller memory is released in stream order by its owner)
        if (t->stream) cudaStreamSynchronize(t->stream);
        else cudaDeviceSynchronize();
        cudaFree(t->hdr);
        cudaFree(t->d_small);
        cudaFree(t->nodes);
        cudaFree(t->tapes);
    }
    cudaFree(t->keep);
    cudaFree(t->reuse_src);
    if (t->staging) cudaFreeHost(t->staging);
    if (t->upload_done) cudaEventDestroy(t->upload_done);
    for (auto& e : t->ev)
        if (e) cudaEventDestroy(e);
    t->ctx->used -= std::min(t->ctx->used, t->bytes);
    delete t;
}

}  // extern "C"

namespace {

// Plans the level passes of `tree` for `tape` (cached on the tree).
frep_status ensure_plan(frep_tree* tree, const frep_tape* tape, const char* who) {
    const uint32_t n_slots = std::max<uint32_t>(tape->ct.n_slots, 4);
    if (tree->plan_valid && tree->plan_slots == n_slots && tree->plan_mm == tape->ct.n_minmax &&
        tree->plan_round == tree->opts.rounding)
        return FREP_OK;
    const int k = tree->plain_k;
    cudaError_t e = frep::plan_levels(n_slots, tape->ct.n_minmax, k, (int)tree->opts.rounding, &tree->plan);
    if (e == cudaErrorInvalidValue)
        return fail(FREP_ERR_UNSUPPORTED, "%s: %u slots / %u min-max ops exceed shared memory", who, n_slots,
                    tape->ct.n_minmax);
    if (e != cudaSuccess) return cuda_fail(e, "plan_levels");
    tree->plan_valid = true;
    tree->plan_slots = n_slots;
    tree->plan_mm = tape->ct.n_minmax;
    tree->plan_round = tree->opts.rounding;
    return FREP_OK;
}

// Enqueues init + every level pass of one tree whose root tape is already at
// word 0 of its pool. `plan` may narrow the grid (the static-scratch path).
// With `prev`, nodes whose time-free tape equals prev's at the same place are
// copied from it (reuse.cu): a match pass fixes every node's source before its
// level pass, and a copy pass follows it.
frep_status enqueue_tree_levels(frep_tree* tree, const frep_tape* tape, float tape_time, uint32_t* keep,
                                frep::WarpScratch ws, const frep::LevelPlan& plan, cudaStream_t stream,
                                const frep_tree* prev = nullptr) {
    cudaError_t e = frep::launch_tree_init(tree->d_self, 1, nullptr, tape_time, stream);
    if (e != cudaSuccess) return cuda_fail(e, "tree_init_kernel");
    if (prev) {
        e = frep::launch_reuse_match(tree->hdr, prev->hdr, tree->reuse_src, tree->reuse_list, 0, stream);
        if (e != cudaSuccess) return cuda_fail(e, "reuse_match_kernel");
    }
    const frep_grid& g = tree->grid;
    if (tree->profile) FREP_CUDA(cudaEventRecord(tree->ev[0], stream));
    frep::LevelLaunch a{};
    a.trees = tree->d_self;
    a.prefix = tree->d_prefix;
    a.cursor = tree->d_cursor;
    a.n_trees = 1;
    a.keep_scratch = keep;
    a.keep_stride = ws.stride;
    a.mm_ofs = ws.mm_ofs;
    a.item_ofs = ws.item_ofs;
    a.item_cap = ws.item_cap;
    a.n_slots = std::max<uint32_t>(tape->ct.n_slots, 4);
    a.mm_cap = std::max<uint32_t>(tape->ct.n_minmax, 1);
    a.eval_list = prev ? tree->reuse_list : nullptr;
    a.any_point_k = 1;
    for (uint32_t l = 0; l < g.levels; l++) {
        const bool point = l == g.levels - 1;
        a.level = l;
        // Level 0 of one tree is one node: too few items to fill the GPU with
        // two cells per lane, so it keeps one (latency, not issue, bounds it).
        const int ki = l == 0 ? 1 : plan.interval_ki;
        e = frep::launch_level_scan(a, point, point ? plan.point_k : ki, stream);
        if (e != cudaSuccess) return cuda_fail(e, "level_scan_kernel");
        e = frep::launch_level(a, plan, (int)tree->opts.rounding, point, stream, ki);
        if (e != cudaSuccess) return cuda_fail(e, "level kernel");
        if (prev) {
            if (!point) {  // before the copies add children of their own
                e = frep::launch_reuse_match(tree->hdr, prev->hdr, tree->reuse_src, tree->reuse_list, l + 1,
                                             stream);
                if (e != cudaSuccess) return cuda_fail(e, "reuse_match_kernel");
            }
            e = frep::launch_reuse_copy(tree->hdr, prev->hdr, tree->reuse_src, l, stream);
            if (e != cudaSuccess) return cuda_fail(e, "reuse_copy_kernel");
        }
        if (tree->profile) FREP_CUDA(cudaEventRecord(tree->ev[l + 1], stream));
    }
    tree->voxelized = true;
    tree->reuse_last = prev != nullptr;
    return FREP_OK;
}

}  // namespace

extern "C" {

}  // extern "C"

namespace {

// Pools and grid that make a tree's subtrees interchangeable with prev's.
frep_status check_reuse(const frep_tree* tree, const frep_tree* prev) {
    if (prev == tree) return fail(FREP_ERR_INVALID_ARG, "frep_voxelize_reuse: prev is the tree being voxelized");
    if (prev->ctx != tree->ctx) return fail(FREP_ERR_INVALID_ARG, "frep_voxelize_reuse: prev belongs to another context");
    if (!prev->voxelized) return fail(FREP_ERR_INVALID_ARG, "frep_voxelize_reuse: prev has not been voxelized");
    const frep_grid &a = tree->grid, &b = prev->grid;
    bool same = a.levels == b.levels && a.world_size == b.world_size && tree->point_k == prev->point_k;
    for (int k = 0; k < 3; k++) same = same && a.low_vertex[k] == b.low_vertex[k];
    for (uint32_t l = 0; same && l < a.levels; l++) same = a.dims[l] == b.dims[l];
    if (!same) return fail(FREP_ERR_INVALID_ARG, "frep_voxelize_reuse: prev has another grid");
    if (tree->opts.rounding != prev->opts.rounding || tree->opts.shorten != prev->opts.shorten)
        return fail(FREP_ERR_INVALID_ARG, "frep_voxelize_reuse: prev was built with other rounding / shortening");
    return FREP_OK;
}

frep_status voxelize_impl(frep_ctx* ctx, frep_tree* tree, const frep_tree* prev, const frep_tape* tape,
                          float tape_time, void* stream_ptr) {
    if (!ctx || !tree || !tape) return fail(FREP_ERR_INVALID_ARG, "frep_voxelize: null argument");
    if (tree->ctx != ctx) return fail(FREP_ERR_INVALID_ARG, "frep_voxelize: tree belongs to another context");
    if (prev) {
        frep_status rs = check_reuse(tree, prev);
        if (rs != FREP_OK) return rs;
    }
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    FREP_CUDA(cudaSetDevice(ctx->device));
    const uint32_t n = (uint32_t)tape->ct.instrs.size();
    const uint32_t n_slots = std::max<uint32_t>(tape->ct.n_slots, 4);
    const uint64_t root_words = tape->record.size();
    if (root_words > tree->tape_cap)
        return fail(FREP_ERR_CAPACITY, "frep_voxelize: root tape (%llu words) exceeds the tape pool", (unsigned long long)root_words);

    frep_status pst = ensure_plan(tree, tape, "frep_voxelize");
    if (pst != FREP_OK) return pst;
    // Per-warp scratch: a keep mask per instruction, a choice-mask pair per
    // MIN/MAX, and room for item tapes (item-level pruning) when that room is
    // at most a quarter of the tree's own pools and the context's budget
    // holds it; else the passes run without item pruning (the same trees).
    // Each tree keeps its scratch between voxelizations, so the bound keeps
    // many small resident trees from each holding item room.
    const uint64_t warps = (uint64_t)tree->plan.blocks * tree->plan.warps_per_block;
    frep::WarpScratch ws = frep::warp_scratch(n, tape->ct.n_minmax, (uint32_t)tree->plan.interval_ki,
                                              tree->opts.rounding != FREP_ROUND_HYBRID);
    if (ws.item_cap) {
        const uint64_t item_bytes = warps * ws.item_cap * 8;
        const uint64_t pool_bytes = tree->node_cap * 4 + tree->tape_cap * 8;
        const bool fits = warps * ws.stride <= tree->keep_words ||
                          ctx->used - std::min<uint64_t>(ctx->used, tree->keep_words * 4) + warps * ws.stride * 4 <=
                              ctx->budget;
        if (item_bytes * 4 > pool_bytes || !fits)
            ws = frep::warp_scratch(n, tape->ct.n_minmax, (uint32_t)tree->plan.interval_ki, false);
    }
    const uint64_t keep_words = warps * ws.stride;
    if (keep_words > tree->keep_words) {
        if (tree->keep) {
            cudaStreamSynchronize(tree->stream);
            cudaFree(tree->keep);
            tree->ctx->used -= std::min<uint64_t>(tree->ctx->used, tree->keep_words * 4);
            tree->bytes -= tree->keep_words * 4;
        }
        tree->keep = nullptr;
        tree->keep_words = 0;
        if (ctx->used + keep_words * 4 > ctx->budget)
            return fail(FREP_ERR_OOM, "frep_voxelize: scratch of %llu bytes exceeds the budget", (unsigned long long)keep_words * 4);
        FREP_CUDA(cudaMalloc(&tree->keep, keep_words * 4));
        tree->keep_words = keep_words;
        tree->bytes += keep_words * 4;
        ctx->used += keep_words * 4;
    }
    if (prev && !tree->reuse_src) {  // one entry per possible node (nodes are >= 8 words), twice
        const uint64_t words = tree->node_cap / 8 + 1;
        if (ctx->used + words * 8 > ctx->budget)
            return fail(FREP_ERR_OOM, "frep_voxelize_reuse: side arrays of %llu bytes exceed the budget",
                        (unsigned long long)words * 8);
        FREP_CUDA(cudaMalloc(&tree->reuse_src, words * 8));
        tree->reuse_list = tree->reuse_src + words;
        tree->reuse_words = words;
        tree->bytes += words * 8;
        ctx->used += words * 8;
    }
    // Root tape upload through pinned staging (reused once the previous copy is done).
    if (root_words > tree->staging_words) {
        if (tree->staging) {
            cudaEventSynchronize(tree->upload_done);
            cudaFreeHost(tree->staging);
        }
        FREP_CUDA(cudaMallocHost(&tree->staging, root_words * 8));
        tree->staging_words = root_words;
    } else {
        FREP_CUDA(cudaEventSynchronize(tree->upload_done));
    }
    std::memcpy(tree->staging, tape->record.data(), root_words * 8);
    FREP_CUDA(cudaMemcpyAsync(tree->tapes, tree->staging, root_words * 8, cudaMemcpyHostToDevice, stream));
    FREP_CUDA(cudaEventRecord(tree->upload_done, stream));

    tree->n_slots = n_slots;
    tree->mm_cap = tape->ct.n_minmax;
    tree->root_n = n;
    tree->root_words = (uint32_t)root_words;
    tree->stream = stream;

    return enqueue_tree_levels(tree, tape, tape_time, tree->keep, ws, tree->plan, stream, prev);
}

}  // namespace

extern "C" {

frep_status frep_voxelize(frep_ctx* ctx, frep_tree* tree, const frep_tape* tape, float tape_time,
                          void* stream_ptr) {
    return voxelize_impl(ctx, tree, nullptr, tape, tape_time, stream_ptr);
}

frep_status frep_voxelize_reuse(frep_ctx* ctx, frep_tree* tree, const frep_tree* prev, const frep_tape* tape,
                                float tape_time, void* stream_ptr) {
    if (!prev) return fail(FREP_ERR_INVALID_ARG, "frep_voxelize_reuse: null prev");
    return voxelize_impl(ctx, tree, prev, tape, tape_time, stream_ptr);
}

frep_status frep_tree_sync(frep_tree* tree, frep_tree_info* info) {
    if (!tree) return fail(FREP_ERR_INVALID_ARG, "frep_tree_sync: null argument");
    FREP_CUDA(cudaSetDevice(tree->ctx->device));
    FREP_CUDA(cudaStreamSynchronize(tree->stream));
    frep::dev::TreeHeader h;
    FREP_CUDA(cudaMemcpy(&h, tree->hdr, sizeof(h), cudaMemcpyDeviceToHost));
    frep_tree_info local;
    frep_tree_info& I = info ? *info : local;
    std::memset(&I, 0, sizeof(I));
    const frep_grid& g = tree->grid;
    I.levels = g.levels;
    uint64_t end = 0;
    for (uint32_t l = 0; l < g.levels; l++) {
        I.dims[l] = g.dims[l];
        I.node_size[l] = tree->node_size[l];
        I.node_offset[l] = h.node_ofs[l];
        const uint64_t cap = tree->node_cap > h.node_ofs[l] ? (tree->node_cap - h.node_ofs[l]) / tree->node_size[l] : 0;
        I.node_count[l] = (uint32_t)std::min<uint64_t>(h.node_count[l], cap);
        I.tape_size_sum[l] = h.tape_size_sum[l];
        I.tape_size_max[l] = h.tape_size_max[l];
        end = h.node_ofs[l] + (uint64_t)I.node_count[l] * tree->node_size[l];
    }
    I.node_words_used = end;
    I.node_words_cap = tree->node_cap;
    I.tape_words_used = std::min<uint64_t>(h.tape_top, tree->tape_cap);
    I.tape_words_cap = tree->tape_cap;
    I.overflow = h.overflow;
    I.root_tape_words = tree->root_words;
    if (h.overflow)
        return fail(FREP_ERR_CAPACITY, "tree pools overflowed (flags %u: 1 = nodes, 2 = tapes)", h.overflow);
    return FREP_OK;
}

frep_status frep_tree_set_profiling(frep_tree* tree, int enable) {
    if (!tree) return fail(FREP_ERR_INVALID_ARG, "frep_tree_set_profiling: null argument");
    FREP_CUDA(cudaSetDevice(tree->ctx->device));
    if (enable && !tree->ev[0])
        for (auto& e : tree->ev) FREP_CUDA(cudaEventCreate(&e));
    tree->profile = enable != 0;
    return FREP_OK;
}

frep_status frep_tree_timings(frep_tree* tree, float ms[FREP_MAX_LEVELS]) {
    if (!tree || !ms) return fail(FREP_ERR_INVALID_ARG, "frep_tree_timings: null argument");
    if (!tree->profile || !tree->voxelized) return fail(FREP_ERR_INVALID_ARG, "frep_tree_timings: profiling is off");
    for (uint32_t l = 0; l < FREP_MAX_LEVELS; l++) ms[l] = 0.0f;
    FREP_CUDA(cudaEventSynchronize(tree->ev[tree->grid.levels]));
    for (uint32_t l = 0; l < tree->grid.levels; l++)
        FREP_CUDA(cudaEventElapsedTime(&ms[l], tree->ev[l], tree->ev[l + 1]));
    return FREP_OK;
}

frep_status frep_tree_work(frep_tree* tree, uint64_t* cell_instr) {
    if (!tree || !cell_instr) return fail(FREP_ERR_INVALID_ARG, "frep_tree_work: null argument");
    FREP_CUDA(cudaStreamSynchronize(tree->stream));
    frep::dev::TreeHeader h;
    FREP_CUDA(cudaMemcpy(&h, tree->hdr, sizeof(h), cudaMemcpyDeviceToHost));
    for (int l = 0; l < FREP_MAX_LEVELS; l++) cell_instr[l] = h.cell_instr[l];
    return FREP_OK;
}

frep_status frep_tree_fp32_ops(frep_tree* tree, uint64_t* ops) {
    if (!tree || !ops) return fail(FREP_ERR_INVALID_ARG, "frep_tree_fp32_ops: null argument");
    if (!tree->voxelized) return fail(FREP_ERR_INVALID_ARG, "frep_tree_fp32_ops: the tree has not been voxelized");
    FREP_CUDA(cudaSetDevice(tree->ctx->device));
    const frep_grid& g = tree->grid;
    FREP_CUDA(cudaMemsetAsync(&tree->hdr->fp32_ops[0], 0, sizeof(tree->hdr->fp32_ops), tree->stream));
    for (uint32_t l = 0; l < g.levels; l++) {
        cudaError_t e = frep::launch_count_ops(tree->hdr, tree->nodes, tree->tapes, tree->node_cap, l,
                                               tree->node_size[l], g.dims[l] * g.dims[l] * g.dims[l],
                                               l == g.levels - 1, tree->reuse_last ? tree->reuse_src : nullptr,
                                               tree->stream);
        if (e != cudaSuccess) return cuda_fail(e, "count_ops_kernel");
    }
    FREP_CUDA(cudaStreamSynchronize(tree->stream));
    frep::dev::TreeHeader h;
    FREP_CUDA(cudaMemcpy(&h, tree->hdr, sizeof(h), cudaMemcpyDeviceToHost));
    for (int l = 0; l < FREP_MAX_LEVELS; l++) ops[l] = h.fp32_ops[l];
    return FREP_OK;
}

frep_status frep_tree_copy_nodes(frep_tree* tree, uint32_t* dst, uint64_t n_words) {
    if (!tree || !dst) return fail(FREP_ERR_INVALID_ARG, "frep_tree_copy_nodes: null argument");
    if (n_words > tree->node_cap) return fail(FREP_ERR_INVALID_ARG, "frep_tree_copy_nodes: beyond the pool");
    FREP_CUDA(cudaStreamSynchronize(tree->stream));
    FREP_CUDA(cudaMemcpy(dst, tree->nodes, n_words * 4, cudaMemcpyDeviceToHost));
    return FREP_OK;
}

frep_status frep_tree_copy_tapes(frep_tree* tree, uint64_t* dst, uint64_t n_words) {
    if (!tree || !dst) return fail(FREP_ERR_INVALID_ARG, "frep_tree_copy_tapes: null argument");
    if (n_words > tree->tape_cap) return fail(FREP_ERR_INVALID_ARG, "frep_tree_copy_tapes: beyond the pool");
    FREP_CUDA(cudaStreamSynchronize(tree->stream));
    FREP_CUDA(cudaMemcpy(dst, tree->tapes, n_words * 8, cudaMemcpyDeviceToHost));
    return FREP_OK;
}

// ---- rendering ---------------------------------------------------------------

frep_status frep_lights_default(frep_lights* L) {
    if (!L) return fail(FREP_ERR_INVALID_ARG, "frep_lights_default: null argument");
    std::memset(L, 0, sizeof(*L));
    // raytracer.cpp:183-192 (directions normalised at render time)
    L->count = 2;
    L->direction[0][0] = -1.0f; L->direction[0][1] = -1.0f; L->direction[0][2] = -0.2f;
    L->color[0][0] = 1.0f;
    L->direction[1][0] = 1.0f; L->direction[1][1] = -1.0f; L->direction[1][2] = -0.2f;
    L->color[1][2] = 2.0f;
    L->ambient[0] = L->ambient[1] = L->ambient[2] = 0.2f;  // main.comp:136
    L->ambient[3] = 1.0f;
    L->background[3] = 1.0f;  // glm::vec4(black, 1)
    L->shadow_mask = 0;
    return FREP_OK;
}

namespace {
struct H3 {
    float x, y, z;
};
H3 cross3(H3 a, H3 b) { return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y}; }
float dot3(H3 a, H3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
H3 normalize3(H3 v) {
    const float inv = 1.0f / std::sqrt(dot3(v, v));
    return {v.x * inv, v.y * inv, v.z * inv};
}
}  // namespace

}  // extern "C"

namespace frep {
namespace detail {

frep_status fill_render_args(const frep_tree* tree, const frep_camera* cam, const frep_lights* lights,
                             float tape_time, const frep_image* out, RenderArgs* args) {
    if (!tree || !cam || !lights || !out) return fail(FREP_ERR_INVALID_ARG, "frep_render: null argument");
    if (!tree->voxelized) return fail(FREP_ERR_INVALID_ARG, "frep_render: the tree has not been voxelized");
    frep_status st = fill_view_args(cam, lights, tape_time, out, args);
    if (st != FREP_OK) return st;
    RenderArgs& a = *args;
    a.hdr = tree->hdr;
    a.nodes = tree->nodes;
    a.tapes = tree->tapes;
    a.levels = tree->grid.levels;
    for (uint32_t l = 0; l < a.levels; l++) {
        a.dims[l] = tree->grid.dims[l];
        a.node_size[l] = tree->node_size[l];
        a.cell_size[l] = tree->cell_size[l];
    }
    for (int k = 0; k < 3; k++) a.low[k] = tree->grid.low_vertex[k];
    a.world_size = tree->grid.world_size;
    a.n_slots = tree->n_slots;
    return FREP_OK;
}

frep_status fill_view_args(const frep_camera* cam, const frep_lights* lights, float tape_time,
                           const frep_image* out, RenderArgs* args) {
    if (!cam || !lights || !out) return fail(FREP_ERR_INVALID_ARG, "frep_render: null argument");
    if (cam->width == 0 || cam->height == 0 || cam->projection > 1)
        return fail(FREP_ERR_INVALID_ARG, "frep_render: bad camera");
    if (lights->count > FREP_MAX_LIGHTS) return fail(FREP_ERR_INVALID_ARG, "frep_render: too many lights");
    if (((uintptr_t)out->rgba8 & 3) || ((uintptr_t)out->hits & 3))
        return fail(FREP_ERR_INVALID_ARG, "frep_render: output buffers must be 4-byte aligned");
    RenderArgs& a = *args;
    a = RenderArgs{};
    a.tape_time = tape_time;
    // Camera::Init, Right(), Up() (camera.cpp:8-27); raytracer.cpp:177-181.
    const H3 fwd = normalize3({cam->forward[0], cam->forward[1], cam->forward[2]});
    const H3 up0 = normalize3({cam->up[0], cam->up[1], cam->up[2]});
    const H3 right = normalize3(cross3(fwd, up0));
    const H3 up = cross3(right, fwd);
    for (int k = 0; k < 3; k++) a.pos[k] = cam->position[k];
    a.fwd[0] = fwd.x; a.fwd[1] = fwd.y; a.fwd[2] = fwd.z;
    a.right[0] = right.x; a.right[1] = right.y; a.right[2] = right.z;
    a.up[0] = up.x; a.up[1] = up.y; a.up[2] = up.z;
    a.sws_x = 2.0f * std::tan((cam->fov_deg * 0.01745329251994329577f) / 2.0f);
    const float aspect = (float)cam->height / (float)cam->width;
    a.sws_y = a.sws_x * aspect;
    a.half_w = cam->ortho_width / 2.0f;
    a.half_h = (cam->ortho_width * aspect) / 2.0f;
    a.projection = cam->projection;
    a.width = cam->width;
    a.height = cam->height;
    a.jitter = cam->jitter;
    a.jitter_seed = cam->jitter_seed;
    a.n_lights = lights->count;
    for (uint32_t i = 0; i < lights->count; i++) {
        const H3 d = normalize3({lights->direction[i][0], lights->direction[i][1], lights->direction[i][2]});
        a.light_dir[i][0] = d.x; a.light_dir[i][1] = d.y; a.light_dir[i][2] = d.z;
        for (int c = 0; c < 4; c++) a.light_color[i][c] = lights->color[i][c];
    }
    for (int c = 0; c < 4; c++) {
        a.ambient[c] = lights->ambient[c];
        a.background[c] = lights->background[c];
    }
    a.shadow_mask = lights->shadow_mask;
    a.rgba8 = out->rgba8;
    a.hits = out->hits;
    return FREP_OK;
}

}  // namespace detail
}  // namespace frep

extern "C" {

frep_status frep_render(frep_ctx* ctx, const frep_tree* tree, const frep_camera* cam,
                        const frep_lights* lights, float tape_time, const frep_image* out,
                        void* stream_ptr) {
    if (!ctx || !tree) return fail(FREP_ERR_INVALID_ARG, "frep_render: null argument");
    FREP_CUDA(cudaSetDevice(ctx->device));
    frep::RenderArgs a{};
    frep_status st = frep::detail::fill_render_args(tree, cam, lights, tape_time, out, &a);
    if (st != FREP_OK) return st;
    cudaError_t e = frep::launch_render(a, (cudaStream_t)stream_ptr);
    if (e == cudaErrorInvalidValue) return fail(FREP_ERR_UNSUPPORTED, "frep_render: more than 1024 slots");
    if (e != cudaSuccess) return cuda_fail(e, "render_kernel");
    return FREP_OK;
}

frep_status frep_resolve_layers(const uint8_t* layers, uint32_t n_layers, uint32_t width, uint32_t height,
                                uint8_t* out, void* stream_ptr) {
    if (!layers || !out || n_layers == 0) return fail(FREP_ERR_INVALID_ARG, "frep_resolve_layers: bad arguments");
    if (((uintptr_t)layers & 3) || ((uintptr_t)out & 3))
        return fail(FREP_ERR_INVALID_ARG, "frep_resolve_layers: buffers must be 4-byte aligned");
    if (n_layers > (1u << 22)) return fail(FREP_ERR_INVALID_ARG, "frep_resolve_layers: too many layers");
    cudaError_t e = frep::launch_resolve_layers(layers, n_layers, width * height, out, (cudaStream_t)stream_ptr);
    if (e != cudaSuccess) return cuda_fail(e, "resolve_layers_kernel");
    return FREP_OK;
}

frep_status frep_render_temporal(frep_ctx* ctx, const frep_tree* tree, const frep_camera* cam,
                                 const frep_lights* lights, float tape_time, uint32_t n_samples, uint8_t* layers,
                                 uint8_t* rgba8, void* stream_ptr) {
    if (!ctx || !tree || !cam || !layers || !rgba8 || n_samples == 0)
        return fail(FREP_ERR_INVALID_ARG, "frep_render_temporal: bad arguments");
    FREP_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = (cudaStream_t)stream_ptr;
    const size_t frame = (size_t)cam->width * cam->height * 4;
    for (uint32_t i = 0; i < n_samples; i++) {
        frep_camera c = *cam;
        c.jitter = 1;
        c.jitter_seed = cam->jitter_seed + (float)i;
        frep_image img{layers + i * frame, nullptr};
        frep::RenderArgs a{};
        frep_status st = frep::detail::fill_render_args(tree, &c, lights, tape_time, &img, &a);
        if (st != FREP_OK) return st;
        cudaError_t e = frep::launch_render(a, s);
        if (e == cudaErrorInvalidValue) return fail(FREP_ERR_UNSUPPORTED, "frep_render_temporal: more than 1024 slots");
        if (e != cudaSuccess) return cuda_fail(e, "render_kernel");
    }
    return frep_resolve_layers(layers, n_samples, cam->width, cam->height, rgba8, stream_ptr);
}

}  // extern "C"

// ---- voxelization without allocation -------------------------------------------
//
// Some callers cannot allocate device memory at the moment they voxelize: a
// renderer running under a fixed memory budget that was reserved up front, a
// real-time frame loop that must not hit cudaMalloc's implicit device
// synchronisation, or a host application that hands every buffer to this
// library from its own allocator. frep_voxelize allocates the interval pass's
// per-warp scratch (and a pinned staging buffer) on first use; the entry point
// below instead takes that scratch from a fixed array in device memory that
// exists from the moment the library is loaded, and copies the root tape
// straight from the tape object, so it makes no allocation at all.
namespace {

// 8 MiB of interval-pass scratch (per resident warp: a 32-bit lane mask per
// tape instruction and a pair per MIN/MAX). Every GPU that loads the library
// holds it until exit.
constexpr uint64_t kStaticScratchWords = 2ull << 20;
static __device__ __align__(256) uint32_t g_static_scratch[kStaticScratchWords];

std::mutex g_static_mutex;
uint32_t* g_static_scratch_addr[256] = {};  // device address, per device ordinal

// Looks up the array's device address once per device (the device must be
// current): in host code the symbol is only a stand-in for the device array.
frep_status static_scratch_for(int device, uint32_t** out) {
    std::lock_guard<std::mutex> lock(g_static_mutex);
    if (device < 0 || device >= 256) return fail(FREP_ERR_INVALID_ARG, "device ordinal %d out of range", device);
    if (!g_static_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(static scratch)");
        g_static_scratch_addr[device] = static_cast<uint32_t*>(p);
    }
    *out = g_static_scratch_addr[device];
    return FREP_OK;
}

}  // namespace

extern "C" frep_status frep_voxelize_static_scratch(frep_ctx* ctx, frep_tree* tree, const frep_tape* tape,
                                                    float tape_time, void* stream_ptr) {
    if (!ctx || !tree || !tape) return fail(FREP_ERR_INVALID_ARG, "frep_voxelize_static_scratch: null argument");
    if (tree->ctx != ctx)
        return fail(FREP_ERR_INVALID_ARG, "frep_voxelize_static_scratch: tree belongs to another context");
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    FREP_CUDA(cudaSetDevice(ctx->device));
    uint32_t* scratch = nullptr;
    frep_status st = static_scratch_for(ctx->device, &scratch);
    if (st != FREP_OK) return st;

    const uint32_t n = (uint32_t)tape->ct.instrs.size();
    const uint32_t n_slots = std::max<uint32_t>(tape->ct.n_slots, 4);
    const uint64_t root_words = tape->record.size();
    if (root_words > tree->tape_cap)
        return fail(FREP_ERR_CAPACITY, "frep_voxelize_static_scratch: root tape (%llu words) exceeds the tape pool",
                    (unsigned long long)root_words);
    frep_status pst = ensure_plan(tree, tape, "frep_voxelize_static_scratch");
    if (pst != FREP_OK) return pst;
    // Each resident warp owns ws.stride words of the array (a keep mask per
    // instruction, a choice-mask pair per MIN/MAX); launch only as many blocks
    // as fit, and refuse tapes too long for even one block.
    const frep::WarpScratch ws = frep::warp_scratch(n, tape->ct.n_minmax, (uint32_t)tree->plan.interval_ki);
    const uint64_t per_block = (uint64_t)tree->plan.warps_per_block * ws.stride;
    if (per_block > kStaticScratchWords)
        return fail(FREP_ERR_UNSUPPORTED,
                    "frep_voxelize_static_scratch: a root tape of %u instructions (%u MIN/MAX) needs %llu scratch "
                    "words per block; the static scratch holds %llu",
                    n, tape->ct.n_minmax, (unsigned long long)per_block, (unsigned long long)kStaticScratchWords);
    frep::LevelPlan plan = tree->plan;
    plan.blocks = (int)std::min<uint64_t>((uint64_t)plan.blocks, kStaticScratchWords / per_block);

    // The root tape goes straight from the tape object (pageable host memory).
    FREP_CUDA(cudaMemcpyAsync(tree->tapes, tape->record.data(), root_words * 8, cudaMemcpyHostToDevice, stream));
    tree->n_slots = n_slots;
    tree->mm_cap = tape->ct.n_minmax;
    tree->root_n = n;
    tree->root_words = (uint32_t)root_words;
    tree->stream = stream;

    return enqueue_tree_levels(tree, tape, tape_time, scratch, ws, plan, stream);
}
