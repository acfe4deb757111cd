// Batched voxelize + render (frep_batch_*): many trees in one launch per level
// pass and one launch for all frames, optionally replayed as a CUDA graph.
//
// The reference voxelizes one scene at a time with a host fence per level
// (vulkan/src/engine/voxelizer.cpp:295-329). Here a set of trees shares every
// launch: the scan kernel lays all trees' work items end to end and the level
// kernels' warps take items from any tree (work stealing through one device
// cursor), so small and large scenes fill the GPU together.
//
// Each call stages its inputs (root tapes, tape times, the tree tables, frame
// arguments) in one upload area and copies it to the device with one
// cudaMemcpyAsync. Four upload areas rotate, so the host prepares the next
// calls while earlier ones still run on the device; it waits only for the
// call four back (a serving loop makes two calls per step). The tree
// set can change between calls (frep_batch_set_trees), which is what a serving
// loop needs; frep_batch_run can capture the whole sequence into a CUDA graph
// (one per upload area) and replay it while the batch keeps its shape.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <vector>

#include "capi_internal.h"

using frep::detail::align_up;
using frep::detail::cuda_fail;
using frep::detail::fail;

namespace {

constexpr int kAreas = 4;  // upload areas in rotation

struct UploadArea {
    uint8_t* h = nullptr;  // pinned
    uint8_t* d = nullptr;
    size_t bytes = 0;
    cudaEvent_t done = nullptr;  // after the last work that reads `d`
    bool pending = false;        // `done` has been recorded since the last wait
    cudaGraphExec_t graph = nullptr;
    std::vector<uint64_t> graph_key;
};

}  // namespace

struct frep_batch {
    frep_ctx* ctx = nullptr;
    std::vector<frep_tree*> trees;
    int rounding = 0;
    // device work prefix (capacity + 1 entries) and cursor
    unsigned long long* d_prefix = nullptr;
    unsigned long long* d_cursor = nullptr;
    uint32_t prefix_cap = 0;
    UploadArea area[kAreas];
    int next_area = 0;
    // interval-pass scratch (keep masks + choice masks per warp)
    uint32_t* keep = nullptr;
    uint64_t keep_words = 0;
    uint64_t bytes = 0;
    // plans: interval passes + point passes with 4 and 2 cells per lane
    frep::LevelPlan plan4{}, plan2{};
    uint32_t plan_slots = 0, plan_mm = 0;
    bool plan_valid = false;
    int interval_warps = 0, point_warps = 0;  // tuning hints (0 = automatic)
    // profiling (plain launches only): ev[0] before the root copy, ev[1] after
    // it, ev[2 + 3 l + kind] after level l's pass of that kind (0 interval,
    // 1 point with 4 cells per lane, 2 point with 2); rev around the frames
    bool profile = false;
    bool profiled = false, render_profiled = false;
    uint32_t profiled_levels = 0;
    cudaEvent_t ev[2 + 3 * FREP_MAX_LEVELS] = {};
    cudaEvent_t rev[2] = {};
    // pinned halves of upload areas that grew, freed at destruction
    std::vector<void*> retired_host;
    // host time of the last voxelize call, ms: plans + prefix + scratch
    // (growing them waits for the device), the upload area (waiting for its
    // previous use, growing it), staging + launches
    double host_ms[3] = {};
    // what the last call enqueued
    uint64_t last_upload = 0;
    uint32_t last_launches = 0;
    cudaStream_t capture_stream = nullptr;
};

namespace {

// One upload area: [tape times][root offsets][tree table][level-pass order]
// [frame arguments][root tapes].
struct Layout {
    size_t times = 0, offsets = 0, tree_ptrs = 0, order = 0, frames = 0, roots = 0, total = 0;
    std::vector<unsigned long long> root_ofs;  // n + 1, in words, relative to `roots`
};

Layout make_layout(uint32_t n, uint32_t nf, const frep_tape* const* tapes) {
    Layout L;
    L.times = 0;
    L.offsets = align_up(sizeof(float) * n, 16);
    L.tree_ptrs = L.offsets + align_up(sizeof(unsigned long long) * (n + 1), 16);
    L.order = L.tree_ptrs + align_up(sizeof(void*) * n, 16);
    L.frames = L.order + align_up(sizeof(void*) * n, 16);
    L.roots = L.frames + align_up(sizeof(frep::RenderArgs) * nf, 16);
    L.root_ofs.assign(n + 1, 0);
    unsigned long long w = 0;
    for (uint32_t i = 0; i < n && tapes; i++) {
        L.root_ofs[i] = w;
        w += tapes[i]->record.size();
    }
    L.root_ofs[n] = w;
    L.total = L.roots + w * 8;
    return L;
}

// Takes the next upload area, waiting until the call that used it last is
// done with it on the device, and grows it to `bytes`. Growing waits for
// nothing else: the device half is released and allocated in stream order
// (cudaFreeAsync / cudaMallocAsync on `s`; its last use is complete), and the
// pinned host half is kept until the batch is destroyed (freeing pinned
// memory waits for the whole device: in a serving loop that stalled a step's
// enqueue behind the step before it, up to half a second).
frep_status acquire_area(frep_batch* b, size_t bytes, int* which, cudaStream_t s) {
    const int i = b->next_area;
    UploadArea& A = b->area[i];
    if (A.pending) {
        FREP_CUDA(cudaEventSynchronize(A.done));
        A.pending = false;
    }
    if (bytes > A.bytes) {
        const size_t prev = A.bytes;
        if (A.graph) {
            cudaGraphExecDestroy(A.graph);
            A.graph = nullptr;
            A.graph_key.clear();
        }
        if (A.h) b->retired_host.push_back(A.h);
        A.h = nullptr;
        uint8_t* old_d = A.d;
        A.d = nullptr;
        b->ctx->used -= std::min<uint64_t>(b->ctx->used, A.bytes);
        b->bytes -= std::min<uint64_t>(b->bytes, A.bytes);
        A.bytes = 0;
        if (old_d) FREP_CUDA(cudaFreeAsync(old_d, s));
        // (each growth costs allocations and a new graph capture: at least twofold)
        const size_t cap = align_up(std::max(bytes + bytes / 4, 2 * prev), 4096);
        if (b->ctx->used + cap > b->ctx->budget) return fail(FREP_ERR_OOM, "frep_batch: upload area exceeds the budget");
        FREP_CUDA(cudaMallocHost(&A.h, cap));
        FREP_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&A.d), cap, s));
        A.bytes = cap;
        b->bytes += cap;
        b->ctx->used += cap;
    }
    if (!A.done) FREP_CUDA(cudaEventCreateWithFlags(&A.done, cudaEventDisableTiming));
    b->next_area = (i + 1) % kAreas;
    *which = i;
    return FREP_OK;
}

frep_status release_area(frep_batch* b, int i, cudaStream_t s) {
    FREP_CUDA(cudaEventRecord(b->area[i].done, s));
    b->area[i].pending = true;
    return FREP_OK;
}

frep_status ensure_prefix(frep_batch* b, uint32_t n) {
    if (n <= b->prefix_cap && b->d_prefix) return FREP_OK;
    if (b->d_prefix) {
        cudaDeviceSynchronize();
        cudaFree(b->d_prefix);
        b->d_prefix = nullptr;
    }
    // Growing waits for the device: start at 512 trees (a serving step's
    // default maximum) and double, so that a changing tree set rarely grows it.
    const uint32_t cap = std::max<uint32_t>(n, std::max<uint32_t>(512, 2 * b->prefix_cap));
    FREP_CUDA(cudaMalloc(&b->d_prefix, sizeof(unsigned long long) * (cap + 2)));
    b->d_cursor = b->d_prefix + cap + 1;
    b->prefix_cap = cap;
    return FREP_OK;
}

frep_status ensure_keep(frep_batch* b, uint64_t words) {
    if (words <= b->keep_words) return FREP_OK;
    // Growing waits for the device: take half again as much as before when
    // that fits the budget, so that steps with ever longer tapes grow it
    // rarely.
    const uint64_t grown = b->keep_words + b->keep_words / 2;
    const uint64_t freed = b->keep_words * 4;
    if (grown > words && b->ctx->used - std::min(b->ctx->used, freed) + grown * 4 <= b->ctx->budget) words = grown;
    if (b->keep) {
        cudaDeviceSynchronize();
        cudaFree(b->keep);
        b->ctx->used -= std::min<uint64_t>(b->ctx->used, b->keep_words * 4);
        b->bytes -= b->keep_words * 4;
        b->keep = nullptr;
        b->keep_words = 0;
    }
    if (b->ctx->used + words * 4 > b->ctx->budget) return fail(FREP_ERR_OOM, "frep_batch: scratch exceeds the budget");
    FREP_CUDA(cudaMalloc(&b->keep, words * 4));
    b->keep_words = words;
    b->bytes += words * 4;
    b->ctx->used += words * 4;
    return FREP_OK;
}

// What the level sequence needs to know about the batch's tapes.
struct TapeStats {
    uint32_t slots = 4, mm = 1, longest = 1, max_levels = 0;
    bool any_k4 = false, any_k2 = false;
};

frep_status check_tapes(const frep_batch* b, const frep_tape* const* tapes, TapeStats* st) {
    if (!tapes) return fail(FREP_ERR_INVALID_ARG, "frep_batch: null tapes");
    for (uint32_t i = 0; i < b->trees.size(); i++) {
        const frep_tape* t = tapes[i];
        const frep_tree* tr = b->trees[i];
        if (!t) return fail(FREP_ERR_INVALID_ARG, "frep_batch: tape %u is null", i);
        if (t->record.size() > tr->tape_cap)
            return fail(FREP_ERR_CAPACITY, "frep_batch: root tape %u (%zu words) exceeds its tree's tape pool", i,
                        t->record.size());
        st->slots = std::max<uint32_t>(st->slots, t->ct.n_slots);
        st->mm = std::max<uint32_t>(st->mm, t->ct.n_minmax);
        st->longest = std::max<uint32_t>(st->longest, (uint32_t)t->ct.instrs.size());
        st->max_levels = std::max<uint32_t>(st->max_levels, tr->grid.levels);
        (tr->point_k == 4 ? st->any_k4 : st->any_k2) = true;
    }
    return FREP_OK;
}

frep_status ensure_plans(frep_batch* b, const TapeStats& st) {
    if (b->plan_valid && b->plan_slots == st.slots && b->plan_mm == st.mm) return FREP_OK;
    cudaError_t e = frep::plan_levels(st.slots, st.mm, 4, b->rounding, &b->plan4, b->interval_warps, b->point_warps);
    if (e == cudaSuccess)
        e = frep::plan_levels(st.slots, st.mm, 2, b->rounding, &b->plan2, b->interval_warps, b->point_warps);
    if (e == cudaErrorInvalidValue)
        return fail(FREP_ERR_UNSUPPORTED, "frep_batch: %u slots / %u min-max ops exceed shared memory", st.slots, st.mm);
    if (e != cudaSuccess) return cuda_fail(e, "plan_levels");
    b->plan_valid = true;
    b->plan_slots = st.slots;
    b->plan_mm = st.mm;
    return FREP_OK;
}

frep::WarpScratch batch_scratch(const frep_batch* b, const TapeStats& st);

// Plans, work prefix and scratch for voxelizing the current tree set.
frep_status prepare_voxelize(frep_batch* b, const frep_tape* const* tapes, TapeStats* st) {
    frep_status r = check_tapes(b, tapes, st);
    if (r == FREP_OK) r = ensure_plans(b, *st);
    if (r == FREP_OK) r = ensure_prefix(b, (uint32_t)b->trees.size());
    if (r == FREP_OK)
        r = ensure_keep(b, (uint64_t)std::max(b->plan4.blocks * b->plan4.warps_per_block,
                                              b->plan2.blocks * b->plan2.warps_per_block) *
                               batch_scratch(b, *st).stride);
    return r;
}

// Cells per lane of the level-0 interval pass: those of the other interval
// passes (two where the plan's shared memory holds them). With two, the
// passes run the jump-table loop (interval_dispatch.cuh); on a 128-scene
// batch level 0 took 11.6 ms with two and 18.6 ms with one (with the earlier
// C++ loop for both widths, two had been slower: 16.5 against 10.1 ms).
// A set so small that its root items at one cell per lane all run at once
// on the persistent grid (a serving step of a few trees) takes one: each
// item is then shorter, and the pass lasts about one item.
int level0_cells(const frep_batch* b) {
    if (b->plan4.interval_ki < 2) return 1;
    uint64_t items1 = 0;  // root items at one cell per lane
    for (const frep_tree* t : b->trees) {
        if (t->grid.levels < 2) continue;
        const uint64_t d = t->grid.dims[0];
        items1 += d * d * d / 32;
    }
    const uint64_t warps = (uint64_t)b->plan4.blocks * (uint64_t)b->plan4.warps_per_block;
    return items1 <= warps ? 1 : 2;
}

// The interval passes' per-warp scratch for the current set.
frep::WarpScratch batch_scratch(const frep_batch* b, const TapeStats& st) {
    return frep::warp_scratch(st.longest, st.mm, (uint32_t)b->plan4.interval_ki, b->rounding != 2);
}

// Enqueues the voxelization of every tree of the set: root copy + header
// reset, then for each level index one interval pass and up to two point
// passes, each a single launch over the whole set. The level passes walk the
// trees longest root tape first (the staged order): warps take the costliest
// items first and the cheap ones fill the tail.
frep_status enqueue_voxelize(frep_batch* b, const uint8_t* d_area, const TapeStats& st, const Layout& L,
                             cudaStream_t s, bool prof) {
    const uint32_t n = (uint32_t)b->trees.size();
    if (prof) FREP_CUDA(cudaEventRecord(b->ev[0], s));
    auto* const* tree_tab = reinterpret_cast<frep::dev::TreeHeader* const*>(d_area + L.tree_ptrs);
    cudaError_t e = frep::launch_tree_init_staged(tree_tab, n, reinterpret_cast<const uint64_t*>(d_area + L.roots),
                                                  reinterpret_cast<const unsigned long long*>(d_area + L.offsets),
                                                  reinterpret_cast<const float*>(d_area + L.times), s);
    if (e != cudaSuccess) return cuda_fail(e, "tree_init_staged_kernel");
    if (prof) FREP_CUDA(cudaEventRecord(b->ev[1], s));
    frep::LevelLaunch a{};
    a.trees = reinterpret_cast<frep::dev::TreeHeader* const*>(d_area + L.order);
    a.prefix = b->d_prefix;
    a.cursor = b->d_cursor;
    a.n_trees = n;
    a.keep_scratch = b->keep;
    const frep::WarpScratch ws = batch_scratch(b, st);
    a.keep_stride = ws.stride;
    a.mm_ofs = ws.mm_ofs;
    a.item_ofs = ws.item_ofs;
    a.item_cap = ws.item_cap;
    a.n_slots = st.slots;
    a.mm_cap = st.mm;
    const int ki0 = level0_cells(b);
    for (uint32_t l = 0; l < st.max_levels; l++) {
        a.level = l;
        const int ki = l == 0 ? ki0 : b->plan4.interval_ki;
        e = frep::launch_level_scan(a, false, ki, s);
        if (e == cudaSuccess) e = frep::launch_level(a, b->plan4, b->rounding, false, s, ki);
        if (e != cudaSuccess) return cuda_fail(e, "batched interval pass");
        if (prof) FREP_CUDA(cudaEventRecord(b->ev[2 + 3 * l], s));
        if (st.any_k4) {
            e = frep::launch_level_scan(a, true, 4, s);
            if (e == cudaSuccess) e = frep::launch_level(a, b->plan4, b->rounding, true, s);
            if (e != cudaSuccess) return cuda_fail(e, "batched point pass");
        }
        if (prof) FREP_CUDA(cudaEventRecord(b->ev[3 + 3 * l], s));
        if (st.any_k2) {
            e = frep::launch_level_scan(a, true, 2, s);
            if (e == cudaSuccess) e = frep::launch_level(a, b->plan2, b->rounding, true, s);
            if (e != cudaSuccess) return cuda_fail(e, "batched point pass");
        }
        if (prof) FREP_CUDA(cudaEventRecord(b->ev[4 + 3 * l], s));
    }
    if (prof) {
        b->profiled = true;
        b->profiled_levels = st.max_levels;
    }
    b->last_launches = 1 + 2 * st.max_levels * (1u + (st.any_k4 ? 1u : 0u) + (st.any_k2 ? 1u : 0u));
    b->last_upload = L.total;
    return FREP_OK;
}

void mark_voxelized(frep_batch* b, const frep_tape* const* tapes, cudaStream_t s) {
    for (uint32_t i = 0; i < b->trees.size(); i++) {
        frep_tree* t = b->trees[i];
        t->voxelized = true;
        t->reuse_last = false;
        t->stream = s;
        t->n_slots = std::max<uint32_t>(tapes[i]->ct.n_slots, 4);
        t->mm_cap = tapes[i]->ct.n_minmax;
        t->root_n = (uint32_t)tapes[i]->ct.instrs.size();
        t->root_words = (uint32_t)tapes[i]->record.size();
    }
}

// Host part of a voxelization's upload: tape times, root offsets, the tree
// table (set order), the level-pass order (by descending root tape length),
// the root tapes.
void stage_inputs(const frep_batch* b, uint8_t* h, const frep_tape* const* tapes, const float* tape_times,
                  const Layout& L) {
    const uint32_t n = (uint32_t)b->trees.size();
    float* times = reinterpret_cast<float*>(h + L.times);
    for (uint32_t i = 0; i < n; i++) times[i] = tape_times ? tape_times[i] : 0.0f;
    std::memcpy(h + L.offsets, L.root_ofs.data(), sizeof(unsigned long long) * (n + 1));
    auto** tab = reinterpret_cast<frep::dev::TreeHeader**>(h + L.tree_ptrs);
    for (uint32_t i = 0; i < n; i++) tab[i] = b->trees[i]->hdr;
    std::vector<uint32_t> idx(n);
    for (uint32_t i = 0; i < n; i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
        return tapes[x]->ct.instrs.size() > tapes[y]->ct.instrs.size();
    });
    auto** order = reinterpret_cast<frep::dev::TreeHeader**>(h + L.order);
    for (uint32_t i = 0; i < n; i++) order[i] = b->trees[idx[i]]->hdr;
    uint64_t* roots = reinterpret_cast<uint64_t*>(h + L.roots);
    for (uint32_t i = 0; i < n; i++)
        std::memcpy(roots + L.root_ofs[i], tapes[i]->record.data(), tapes[i]->record.size() * 8);
}

struct FrameDims {
    uint32_t max_w = 0, max_h = 0, max_slots = 4;
};

frep_status stage_frames(uint8_t* h, const frep_tree* const* frame_trees, uint32_t nf, const frep_camera* cams,
                         const frep_lights* lights, const float* tape_times, const frep_image* images,
                         const Layout& L, FrameDims* fd) {
    frep::RenderArgs* frames = reinterpret_cast<frep::RenderArgs*>(h + L.frames);
    for (uint32_t i = 0; i < nf; i++) {
        frep_status st = frep::detail::fill_render_args(frame_trees[i], &cams[i], lights,
                                                        tape_times ? tape_times[i] : 0.0f, &images[i], &frames[i]);
        if (st != FREP_OK) return st;
        fd->max_w = std::max(fd->max_w, cams[i].width);
        fd->max_h = std::max(fd->max_h, cams[i].height);
        fd->max_slots = std::max(fd->max_slots, frames[i].n_slots);
    }
    return FREP_OK;
}

frep_status enqueue_frames(frep_batch* b, const uint8_t* d_area, const Layout& L, uint32_t nf, const FrameDims& fd,
                           cudaStream_t s, bool prof) {
    if (prof) FREP_CUDA(cudaEventRecord(b->rev[0], s));
    cudaError_t e = frep::launch_render_batch(reinterpret_cast<const frep::RenderArgs*>(d_area + L.frames), nf,
                                              fd.max_w, fd.max_h, fd.max_slots, s);
    if (e == cudaErrorInvalidValue) return fail(FREP_ERR_UNSUPPORTED, "frep_batch: too many frames or slots");
    if (e != cudaSuccess) return cuda_fail(e, "render_batch_kernel");
    if (prof) {
        FREP_CUDA(cudaEventRecord(b->rev[1], s));
        b->render_profiled = true;
    }
    return FREP_OK;
}

frep_status check_trees(frep_ctx* ctx, frep_tree* const* trees, uint32_t n, int* rounding) {
    if (!trees || n == 0) return fail(FREP_ERR_INVALID_ARG, "frep_batch: empty tree set");
    for (uint32_t i = 0; i < n; i++) {
        if (!trees[i] || trees[i]->ctx != ctx)
            return fail(FREP_ERR_INVALID_ARG, "frep_batch: tree %u is null or from another context", i);
        if (i == 0) *rounding = (int)trees[0]->opts.rounding;
        if ((int)trees[i]->opts.rounding != *rounding)
            return fail(FREP_ERR_INVALID_ARG, "frep_batch: all trees of a batch use the same rounding");
        // the batch runs its last-level passes with 4 and 2 cells per lane
        if (trees[i]->point_k == 8)
            return fail(FREP_ERR_UNSUPPORTED, "frep_batch: tree %u uses 8 cells per lane in its last level", i);
    }
    return FREP_OK;
}

}  // namespace

namespace frep {
namespace detail {
void batch_host_ms(const frep_batch* b, double out[3]) {
    for (int i = 0; i < 3; i++) out[i] = b ? b->host_ms[i] : 0.0;
}
}  // namespace detail
}  // namespace frep

extern "C" {

frep_status frep_batch_create(frep_ctx* ctx, frep_tree* const* trees, uint32_t n, frep_batch** out) {
    if (!ctx || !out) return fail(FREP_ERR_INVALID_ARG, "frep_batch_create: bad arguments");
    int rounding = 0;
    frep_status r = check_trees(ctx, trees, n, &rounding);
    if (r != FREP_OK) return r;
    FREP_CUDA(cudaSetDevice(ctx->device));
    auto* b = new frep_batch();
    b->ctx = ctx;
    b->trees.assign(trees, trees + n);
    b->rounding = rounding;
    cudaError_t e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return cuda_fail(e, "frep_batch_create");
    }
    r = ensure_prefix(b, n);
    if (r != FREP_OK) {
        cudaStreamDestroy(b->capture_stream);
        delete b;
        return r;
    }
    *out = b;
    return FREP_OK;
}

void frep_batch_destroy(frep_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    cudaDeviceSynchronize();
    for (UploadArea& A : b->area) {
        if (A.graph) cudaGraphExecDestroy(A.graph);
        if (A.h) cudaFreeHost(A.h);
        if (A.d) cudaFree(A.d);
        if (A.done) cudaEventDestroy(A.done);
    }
    for (void* h : b->retired_host) cudaFreeHost(h);
    cudaFree(b->d_prefix);
    cudaFree(b->keep);
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : b->rev)
        if (e) cudaEventDestroy(e);
    b->ctx->used -= std::min<uint64_t>(b->ctx->used, b->bytes);
    delete b;
}

frep_status frep_batch_set_trees(frep_batch* b, frep_tree* const* trees, uint32_t n) {
    if (!b) return fail(FREP_ERR_INVALID_ARG, "frep_batch_set_trees: null batch");
    int rounding = 0;
    frep_status r = check_trees(b->ctx, trees, n, &rounding);
    if (r != FREP_OK) return r;
    if (rounding != b->rounding) {
        b->rounding = rounding;
        b->plan_valid = false;
    }
    b->trees.assign(trees, trees + n);
    return FREP_OK;
}

frep_status frep_batch_voxelize(frep_batch* b, const frep_tape* const* tapes, const float* tape_times,
                                void* stream_ptr) {
    if (!b) return fail(FREP_ERR_INVALID_ARG, "frep_batch_voxelize: null batch");
    FREP_CUDA(cudaSetDevice(b->ctx->device));
    cudaStream_t s = (cudaStream_t)stream_ptr;
    TapeStats st;
    const auto t0 = std::chrono::steady_clock::now();
    frep_status r = prepare_voxelize(b, tapes, &st);
    if (r != FREP_OK) return r;
    const auto t1 = std::chrono::steady_clock::now();
    const Layout L = make_layout((uint32_t)b->trees.size(), 0, tapes);
    int ai = 0;
    r = acquire_area(b, L.total, &ai, s);
    if (r != FREP_OK) return r;
    const auto t2 = std::chrono::steady_clock::now();
    UploadArea& A = b->area[ai];
    stage_inputs(b, A.h, tapes, tape_times, L);
    FREP_CUDA(cudaMemcpyAsync(A.d, A.h, L.total, cudaMemcpyHostToDevice, s));
    r = enqueue_voxelize(b, A.d, st, L, s, b->profile);
    if (r != FREP_OK) return r;
    mark_voxelized(b, tapes, s);
    r = release_area(b, ai, s);
    const auto t3 = std::chrono::steady_clock::now();
    auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point c) {
        return std::chrono::duration<double, std::milli>(c - a).count();
    };
    b->host_ms[0] = ms(t0, t1);
    b->host_ms[1] = ms(t1, t2);
    b->host_ms[2] = ms(t2, t3);
    return r;
}

frep_status frep_batch_render_frames(frep_batch* b, const frep_tree* const* frame_trees, uint32_t n_frames,
                                     const frep_camera* cameras, const frep_lights* lights, const float* tape_times,
                                     const frep_image* images, void* stream_ptr) {
    if (!b || !frame_trees || !cameras || !lights || !images)
        return fail(FREP_ERR_INVALID_ARG, "frep_batch_render_frames: null argument");
    if (n_frames == 0) return FREP_OK;
    for (uint32_t i = 0; i < n_frames; i++)
        if (!frame_trees[i] || frame_trees[i]->ctx != b->ctx)
            return fail(FREP_ERR_INVALID_ARG, "frep_batch_render_frames: tree of frame %u is null or foreign", i);
    FREP_CUDA(cudaSetDevice(b->ctx->device));
    cudaStream_t s = (cudaStream_t)stream_ptr;
    const Layout L = make_layout(0, n_frames, nullptr);
    int ai = 0;
    frep_status r = acquire_area(b, L.total, &ai, s);
    if (r != FREP_OK) return r;
    UploadArea& A = b->area[ai];
    FrameDims fd;
    r = stage_frames(A.h, frame_trees, n_frames, cameras, lights, tape_times, images, L, &fd);
    if (r != FREP_OK) return r;
    FREP_CUDA(cudaMemcpyAsync(A.d + L.frames, A.h + L.frames, L.roots - L.frames, cudaMemcpyHostToDevice, s));
    r = enqueue_frames(b, A.d, L, n_frames, fd, s, b->profile);
    if (r != FREP_OK) return r;
    return release_area(b, ai, s);
}

frep_status frep_batch_render(frep_batch* b, const frep_camera* cameras, const frep_lights* lights,
                              const float* tape_times, const frep_image* images, void* stream_ptr) {
    if (!b) return fail(FREP_ERR_INVALID_ARG, "frep_batch_render: null batch");
    std::vector<const frep_tree*> ft(b->trees.begin(), b->trees.end());
    return frep_batch_render_frames(b, ft.data(), (uint32_t)ft.size(), cameras, lights, tape_times, images,
                                    stream_ptr);
}

frep_status frep_batch_run(frep_batch* b, const frep_tape* const* tapes, const float* tape_times,
                           const frep_camera* cameras, const frep_lights* lights, const frep_image* images,
                           int use_graph, void* stream_ptr) {
    if (!b || !cameras || !lights || !images) return fail(FREP_ERR_INVALID_ARG, "frep_batch_run: null argument");
    if (!use_graph) {
        frep_status r = frep_batch_voxelize(b, tapes, tape_times, stream_ptr);
        return r != FREP_OK ? r : frep_batch_render(b, cameras, lights, tape_times, images, stream_ptr);
    }
    FREP_CUDA(cudaSetDevice(b->ctx->device));
    cudaStream_t s = (cudaStream_t)stream_ptr;
    const uint32_t n = (uint32_t)b->trees.size();
    TapeStats st;
    frep_status r = prepare_voxelize(b, tapes, &st);
    if (r != FREP_OK) return r;
    const Layout L = make_layout(n, n, tapes);
    int ai = 0;
    r = acquire_area(b, L.total, &ai, s);
    if (r != FREP_OK) return r;
    UploadArea& A = b->area[ai];
    // Fill the whole upload area (the graph's copy node reads it when it
    // runs). The frame arguments describe the trees as this run leaves them.
    mark_voxelized(b, tapes, s);
    stage_inputs(b, A.h, tapes, tape_times, L);
    std::vector<const frep_tree*> ft(b->trees.begin(), b->trees.end());
    FrameDims fd;
    r = stage_frames(A.h, ft.data(), n, cameras, lights, tape_times, images, L, &fd);
    if (r != FREP_OK) return r;
    // The area's graph stays valid while the batch keeps its shape.
    std::vector<uint64_t> key = {L.total, n, st.slots, st.mm, st.longest, st.max_levels, st.any_k4, st.any_k2,
                                 fd.max_w, fd.max_h, fd.max_slots, (uint64_t)b->plan4.blocks,
                                 (uint64_t)b->plan4.warps_per_block, (uint64_t)b->plan4.point_warps_per_block,
                                 (uint64_t)b->plan2.point_warps_per_block, (uint64_t)b->plan4.interval_ki,
                                 (uint64_t)level0_cells(b), (uint64_t)(uintptr_t)b->keep,
                                 (uint64_t)(uintptr_t)b->d_prefix, (uint64_t)(uintptr_t)A.d};
    for (uint32_t i = 0; i < n; i++) key.push_back(L.root_ofs[i]);
    if (!A.graph || key != A.graph_key) {
        if (A.graph) {
            cudaGraphExecDestroy(A.graph);
            A.graph = nullptr;
        }
        cudaStream_t cs = b->capture_stream;
        FREP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        cudaError_t ce = cudaMemcpyAsync(A.d, A.h, L.total, cudaMemcpyHostToDevice, cs);
        frep_status vr = ce == cudaSuccess ? enqueue_voxelize(b, A.d, st, L, cs, false) : cuda_fail(ce, "upload");
        if (vr == FREP_OK) vr = enqueue_frames(b, A.d, L, n, fd, cs, false);
        cudaGraph_t g = nullptr;
        cudaError_t ee = cudaStreamEndCapture(cs, &g);
        if (vr != FREP_OK) {
            if (g) cudaGraphDestroy(g);
            return vr;
        }
        if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
        ce = cudaGraphInstantiate(&A.graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
        A.graph_key = key;
    } else {
        b->last_upload = L.total;
    }
    FREP_CUDA(cudaGraphLaunch(A.graph, s));
    return release_area(b, ai, s);
}

frep_status frep_batch_get_info(const frep_batch* b, frep_batch_info* info) {
    if (!b || !info) return fail(FREP_ERR_INVALID_ARG, "frep_batch_get_info: null argument");
    info->n_trees = (uint32_t)b->trees.size();
    info->voxelize_launches = b->last_launches;
    info->upload_bytes = b->last_upload;
    info->device_bytes = b->bytes;
    info->interval_warps_per_block = b->plan_valid ? (uint32_t)b->plan4.warps_per_block : 0;
    info->point_warps_per_block = b->plan_valid ? (uint32_t)b->plan4.point_warps_per_block : 0;
    info->root_cells_per_lane = b->plan_valid ? (uint32_t)level0_cells(b) : 0;
    return FREP_OK;
}

frep_status frep_batch_set_tuning(frep_batch* b, uint32_t interval_warps_per_block, uint32_t point_warps_per_block) {
    if (!b) return fail(FREP_ERR_INVALID_ARG, "frep_batch_set_tuning: null batch");
    auto ok = [](uint32_t w) { return w == 0 || w == 1 || w == 4; };
    if (!ok(interval_warps_per_block) || !ok(point_warps_per_block))
        return fail(FREP_ERR_INVALID_ARG, "frep_batch_set_tuning: warps per block must be 0, 1 or 4");
    b->interval_warps = (int)interval_warps_per_block;
    b->point_warps = (int)point_warps_per_block;
    b->plan_valid = false;
    return FREP_OK;
}

frep_status frep_batch_set_profiling(frep_batch* b, int enable) {
    if (!b) return fail(FREP_ERR_INVALID_ARG, "frep_batch_set_profiling: null batch");
    FREP_CUDA(cudaSetDevice(b->ctx->device));
    if (enable && !b->ev[0]) {
        for (cudaEvent_t& e : b->ev) FREP_CUDA(cudaEventCreate(&e));
        for (cudaEvent_t& e : b->rev) FREP_CUDA(cudaEventCreate(&e));
    }
    b->profile = enable != 0;
    b->profiled = b->render_profiled = false;
    return FREP_OK;
}

frep_status frep_batch_timings(frep_batch* b, float ms[3 * FREP_MAX_LEVELS + 2]) {
    if (!b || !ms) return fail(FREP_ERR_INVALID_ARG, "frep_batch_timings: null argument");
    if (!b->profile || !b->profiled)
        return fail(FREP_ERR_INVALID_ARG, "frep_batch_timings: no profiled frep_batch_voxelize since profiling was enabled");
    FREP_CUDA(cudaSetDevice(b->ctx->device));
    for (int i = 0; i < 3 * FREP_MAX_LEVELS + 2; i++) ms[i] = 0.0f;
    const uint32_t last = 1 + 3 * b->profiled_levels;
    FREP_CUDA(cudaEventSynchronize(b->ev[last]));
    FREP_CUDA(cudaEventElapsedTime(&ms[3 * FREP_MAX_LEVELS], b->ev[0], b->ev[1]));
    for (uint32_t g = 0; g < 3 * b->profiled_levels; g++)
        FREP_CUDA(cudaEventElapsedTime(&ms[g], b->ev[1 + g], b->ev[2 + g]));
    if (b->render_profiled) {
        FREP_CUDA(cudaEventSynchronize(b->rev[1]));
        FREP_CUDA(cudaEventElapsedTime(&ms[3 * FREP_MAX_LEVELS + 1], b->rev[0], b->rev[1]));
    }
    return FREP_OK;
}

}  // extern "C"
