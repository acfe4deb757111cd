// Batched voxelize + render (frep_batch_*): many trees in one launch per level
// pass and one launch for all frames, optionally replayed as a CUDA graph.
//
// The reference voxelizes one scene at a time with a host fence per level
// (vulkan/src/engine/voxelizer.cpp:295-329). Here a fixed set of trees shares
// every launch: the scan kernel lays all trees' work items end to end and the
// level kernels' warps take items from any tree (work stealing through one
// device cursor), so small and large scenes fill the GPU together. The whole
// sequence — one staged upload (root tapes, tape times, frame arguments), the
// root copy + header reset, the level passes and the frames — is captured once
// into a CUDA graph and replayed while the batch's shape stays the same.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "capi_internal.h"

using frep::detail::align_up;
using frep::detail::cuda_fail;
using frep::detail::fail;

struct frep_batch {
    frep_ctx* ctx = nullptr;
    std::vector<frep_tree*> trees;
    uint32_t n = 0;
    int rounding = 0;
    // device: [n header pointers][prefix n+1][cursor]
    void* d_meta = nullptr;
    frep::dev::TreeHeader** d_trees = nullptr;
    unsigned long long* d_prefix = nullptr;
    unsigned long long* d_cursor = nullptr;
    // one upload area: [tape times][root offsets][frame arguments][root tapes]
    size_t stage_bytes = 0;
    uint8_t* h_stage = nullptr;  // pinned
    uint8_t* d_stage = nullptr;
    cudaEvent_t upload_done = nullptr;
    // keep-mask scratch for the interval passes
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
    // what the last voxelization enqueued
    uint64_t last_upload = 0;
    uint32_t last_launches = 0;
    // graph replay
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<uint64_t> graph_key;
};

namespace {

// The upload area: [tape times][root offsets][level-pass tree order][frame
// arguments][root tapes]. Everything before the root tapes depends only on
// the batch size.
struct Layout {
    size_t times = 0, offsets = 0, order = 0, frames = 0, roots = 0, total = 0;
    std::vector<unsigned long long> root_ofs;  // n + 1, in words, relative to `roots`
};

Layout base_layout(uint32_t n) {
    Layout L;
    L.times = 0;
    L.offsets = align_up(sizeof(float) * n, 16);
    L.order = L.offsets + align_up(sizeof(unsigned long long) * (n + 1), 16);
    L.frames = L.order + align_up(sizeof(void*) * n, 16);
    L.roots = L.frames + align_up(sizeof(frep::RenderArgs) * n, 16);
    L.total = L.roots;
    return L;
}

Layout make_layout(const frep_batch* b, const frep_tape* const* tapes) {
    Layout L = base_layout(b->n);
    L.root_ofs.resize(b->n + 1);
    unsigned long long w = 0;
    for (uint32_t i = 0; i < b->n; i++) {
        L.root_ofs[i] = w;
        w += tapes[i]->record.size();
    }
    L.root_ofs[b->n] = w;
    L.total = L.roots + w * 8;
    return L;
}

frep_status ensure_stage(frep_batch* b, size_t bytes) {
    if (bytes <= b->stage_bytes) {
        FREP_CUDA(cudaEventSynchronize(b->upload_done));
        return FREP_OK;
    }
    if (b->h_stage) {
        cudaEventSynchronize(b->upload_done);
        cudaFreeHost(b->h_stage);
        cudaFree(b->d_stage);
        b->ctx->used -= std::min<uint64_t>(b->ctx->used, b->stage_bytes);
        b->bytes -= b->stage_bytes;
        b->h_stage = nullptr;
        b->d_stage = nullptr;
        b->stage_bytes = 0;
    }
    const size_t cap = align_up(bytes + bytes / 4, 4096);
    if (b->ctx->used + cap > b->ctx->budget) return fail(FREP_ERR_OOM, "frep_batch: upload area exceeds the budget");
    FREP_CUDA(cudaMallocHost(&b->h_stage, cap));
    FREP_CUDA(cudaMalloc(&b->d_stage, cap));
    b->stage_bytes = cap;
    b->bytes += cap;
    b->ctx->used += cap;
    return FREP_OK;
}

frep_status ensure_keep(frep_batch* b, uint64_t words) {
    if (words <= b->keep_words) return FREP_OK;
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

frep_status check_tapes(frep_batch* b, const frep_tape* const* tapes, TapeStats* st) {
    if (!tapes) return fail(FREP_ERR_INVALID_ARG, "frep_batch: null tapes");
    for (uint32_t i = 0; i < b->n; i++) {
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
        const int k = tr->point_k;
        (k == 4 ? st->any_k4 : st->any_k2) = true;
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

// Enqueues the voxelization of every tree: root copy + header reset, then for
// each level index one interval pass and up to two point passes, each a single
// launch over the whole batch.
frep_status enqueue_voxelize(frep_batch* b, const TapeStats& st, const Layout& L, cudaStream_t s, bool prof) {
    if (prof) FREP_CUDA(cudaEventRecord(b->ev[0], s));
    const uint64_t* staged_roots = reinterpret_cast<const uint64_t*>(b->d_stage + L.roots);
    const unsigned long long* offsets = reinterpret_cast<const unsigned long long*>(b->d_stage + L.offsets);
    const float* times = reinterpret_cast<const float*>(b->d_stage + L.times);
    cudaError_t e = frep::launch_tree_init_staged(b->d_trees, b->n, staged_roots, offsets, times, s);
    if (e != cudaSuccess) return cuda_fail(e, "tree_init_staged_kernel");
    if (prof) FREP_CUDA(cudaEventRecord(b->ev[1], s));
    frep::LevelLaunch a{};
    // The level passes walk the trees longest root tape first (staged order):
    // warps take the costliest items first and the cheap ones fill the tail.
    a.trees = reinterpret_cast<frep::dev::TreeHeader* const*>(b->d_stage + L.order);
    a.prefix = b->d_prefix;
    a.cursor = b->d_cursor;
    a.n_trees = b->n;
    a.keep_scratch = b->keep;
    const frep::WarpScratch ws = frep::warp_scratch(st.longest, st.mm);
    a.keep_stride = ws.stride;
    a.mm_ofs = ws.mm_ofs;
    a.n_slots = st.slots;
    a.mm_cap = st.mm;
    for (uint32_t l = 0; l < st.max_levels; l++) {
        a.level = l;
        // interval passes of every tree that has a level below l
        e = frep::launch_level_scan(a, false, 4, s);
        if (e == cudaSuccess) e = frep::launch_level(a, b->plan4, b->rounding, false, s);
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
    for (uint32_t i = 0; i < b->n; i++) {
        frep_tree* t = b->trees[i];
        t->voxelized = true;
        t->stream = s;
        t->n_slots = std::max<uint32_t>(tapes[i]->ct.n_slots, 4);
        t->mm_cap = tapes[i]->ct.n_minmax;
        t->root_n = (uint32_t)tapes[i]->ct.instrs.size();
        t->root_words = (uint32_t)tapes[i]->record.size();
    }
}

// Writes the host part of the upload area: tape times, root offsets, the
// level-pass order (headers by descending root tape length), roots.
void stage_inputs(frep_batch* b, const frep_tape* const* tapes, const float* tape_times, const Layout& L) {
    float* times = reinterpret_cast<float*>(b->h_stage + L.times);
    for (uint32_t i = 0; i < b->n; i++) times[i] = tape_times ? tape_times[i] : 0.0f;
    std::memcpy(b->h_stage + L.offsets, L.root_ofs.data(), sizeof(unsigned long long) * (b->n + 1));
    std::vector<uint32_t> idx(b->n);
    for (uint32_t i = 0; i < b->n; i++) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) {
        return tapes[x]->ct.instrs.size() > tapes[y]->ct.instrs.size();
    });
    auto** order = reinterpret_cast<frep::dev::TreeHeader**>(b->h_stage + L.order);
    for (uint32_t i = 0; i < b->n; i++) order[i] = b->trees[idx[i]]->hdr;
    uint64_t* roots = reinterpret_cast<uint64_t*>(b->h_stage + L.roots);
    for (uint32_t i = 0; i < b->n; i++)
        std::memcpy(roots + L.root_ofs[i], tapes[i]->record.data(), tapes[i]->record.size() * 8);
}

frep_status stage_frames(frep_batch* b, const frep_camera* cams, const frep_lights* lights, const float* tape_times,
                         const frep_image* images, const Layout& L, uint32_t* max_w, uint32_t* max_h,
                         uint32_t* max_slots) {
    frep::RenderArgs* frames = reinterpret_cast<frep::RenderArgs*>(b->h_stage + L.frames);
    *max_w = *max_h = 0;
    *max_slots = 4;
    for (uint32_t i = 0; i < b->n; i++) {
        frep_status st = frep::detail::fill_render_args(b->trees[i], &cams[i], lights,
                                                        tape_times ? tape_times[i] : 0.0f, &images[i], &frames[i]);
        if (st != FREP_OK) return st;
        *max_w = std::max(*max_w, cams[i].width);
        *max_h = std::max(*max_h, cams[i].height);
        *max_slots = std::max(*max_slots, frames[i].n_slots);
    }
    return FREP_OK;
}

}  // namespace

extern "C" {

frep_status frep_batch_create(frep_ctx* ctx, frep_tree* const* trees, uint32_t n, frep_batch** out) {
    if (!ctx || !trees || !out || n == 0) return fail(FREP_ERR_INVALID_ARG, "frep_batch_create: bad arguments");
    FREP_CUDA(cudaSetDevice(ctx->device));
    auto* b = new frep_batch();
    b->ctx = ctx;
    b->n = n;
    b->trees.assign(trees, trees + n);
    b->rounding = (int)trees[0]->opts.rounding;
    for (uint32_t i = 0; i < n; i++) {
        if (!trees[i] || trees[i]->ctx != ctx) {
            delete b;
            return fail(FREP_ERR_INVALID_ARG, "frep_batch_create: tree %u is null or from another context", i);
        }
        if ((int)trees[i]->opts.rounding != b->rounding) {
            delete b;
            return fail(FREP_ERR_INVALID_ARG, "frep_batch_create: all trees of a batch use the same rounding");
        }
    }
    const size_t meta = align_up(sizeof(void*) * n, 16) + sizeof(unsigned long long) * (n + 2);
    cudaError_t e = cudaMalloc(&b->d_meta, meta);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->upload_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->capture_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cudaFree(b->d_meta);
        delete b;
        return cuda_fail(e, "frep_batch_create");
    }
    b->d_trees = static_cast<frep::dev::TreeHeader**>(b->d_meta);
    b->d_prefix = reinterpret_cast<unsigned long long*>(static_cast<uint8_t*>(b->d_meta) + align_up(sizeof(void*) * n, 16));
    b->d_cursor = b->d_prefix + n + 1;
    std::vector<frep::dev::TreeHeader*> h(n);
    for (uint32_t i = 0; i < n; i++) h[i] = trees[i]->hdr;
    e = cudaMemcpy(b->d_trees, h.data(), sizeof(void*) * n, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaFree(b->d_meta);
        delete b;
        return cuda_fail(e, "frep_batch_create: tree table upload");
    }
    *out = b;
    return FREP_OK;
}

void frep_batch_destroy(frep_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    cudaDeviceSynchronize();
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->d_meta);
    cudaFree(b->keep);
    cudaFree(b->d_stage);
    if (b->h_stage) cudaFreeHost(b->h_stage);
    if (b->upload_done) cudaEventDestroy(b->upload_done);
    if (b->capture_stream) cudaStreamDestroy(b->capture_stream);
    for (cudaEvent_t e : b->ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : b->rev)
        if (e) cudaEventDestroy(e);
    b->ctx->used -= std::min<uint64_t>(b->ctx->used, b->bytes);
    delete b;
}

frep_status frep_batch_voxelize(frep_batch* b, const frep_tape* const* tapes, const float* tape_times,
                                void* stream_ptr) {
    if (!b) return fail(FREP_ERR_INVALID_ARG, "frep_batch_voxelize: null batch");
    FREP_CUDA(cudaSetDevice(b->ctx->device));
    cudaStream_t s = (cudaStream_t)stream_ptr;
    TapeStats st;
    frep_status r = check_tapes(b, tapes, &st);
    if (r == FREP_OK) r = ensure_plans(b, st);
    const Layout L = make_layout(b, tapes);
    if (r == FREP_OK) r = ensure_stage(b, L.total);
    if (r == FREP_OK) r = ensure_keep(b, (uint64_t)std::max(b->plan4.blocks * b->plan4.warps_per_block,
                                                           b->plan2.blocks * b->plan2.warps_per_block) *
                                             frep::warp_scratch(st.longest, st.mm).stride);
    if (r != FREP_OK) return r;
    stage_inputs(b, tapes, tape_times, L);
    FREP_CUDA(cudaMemcpyAsync(b->d_stage, b->h_stage, L.frames, cudaMemcpyHostToDevice, s));  // times..order
    FREP_CUDA(cudaMemcpyAsync(b->d_stage + L.roots, b->h_stage + L.roots, L.total - L.roots,
                              cudaMemcpyHostToDevice, s));
    FREP_CUDA(cudaEventRecord(b->upload_done, s));
    r = enqueue_voxelize(b, st, L, s, b->profile);
    if (r != FREP_OK) return r;
    mark_voxelized(b, tapes, s);
    return FREP_OK;
}

frep_status frep_batch_render(frep_batch* b, const frep_camera* cameras, const frep_lights* lights,
                              const float* tape_times, const frep_image* images, void* stream_ptr) {
    if (!b || !cameras || !lights || !images) return fail(FREP_ERR_INVALID_ARG, "frep_batch_render: null argument");
    FREP_CUDA(cudaSetDevice(b->ctx->device));
    cudaStream_t s = (cudaStream_t)stream_ptr;
    // Frame arguments go to the upload area's frame block; make sure it is large
    // enough even before the first voxelization.
    const Layout L = base_layout(b->n);
    frep_status r = ensure_stage(b, std::max<size_t>(L.roots, b->stage_bytes));
    if (r != FREP_OK) return r;
    uint32_t mw, mh, ms;
    r = stage_frames(b, cameras, lights, tape_times, images, L, &mw, &mh, &ms);
    if (r != FREP_OK) return r;
    FREP_CUDA(cudaMemcpyAsync(b->d_stage + L.frames, b->h_stage + L.frames, L.roots - L.frames,
                              cudaMemcpyHostToDevice, s));
    FREP_CUDA(cudaEventRecord(b->upload_done, s));
    if (b->profile) FREP_CUDA(cudaEventRecord(b->rev[0], s));
    cudaError_t e = frep::launch_render_batch(reinterpret_cast<const frep::RenderArgs*>(b->d_stage + L.frames), b->n,
                                              mw, mh, ms, s);
    if (e == cudaErrorInvalidValue) return fail(FREP_ERR_UNSUPPORTED, "frep_batch_render: too many frames or slots");
    if (e != cudaSuccess) return cuda_fail(e, "render_batch_kernel");
    if (b->profile) {
        FREP_CUDA(cudaEventRecord(b->rev[1], s));
        b->render_profiled = true;
    }
    return FREP_OK;
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
    TapeStats st;
    frep_status r = check_tapes(b, tapes, &st);
    if (r == FREP_OK) r = ensure_plans(b, st);
    const Layout L = make_layout(b, tapes);
    if (r == FREP_OK) r = ensure_stage(b, L.total);
    if (r == FREP_OK) r = ensure_keep(b, (uint64_t)std::max(b->plan4.blocks * b->plan4.warps_per_block,
                                                           b->plan2.blocks * b->plan2.warps_per_block) *
                                             frep::warp_scratch(st.longest, st.mm).stride);
    if (r != FREP_OK) return r;
    // Fill the whole upload area (the graph's memcpy node reads it when it runs).
    // The frame arguments describe the trees as this run leaves them.
    mark_voxelized(b, tapes, s);
    stage_inputs(b, tapes, tape_times, L);
    uint32_t mw, mh, ms;
    r = stage_frames(b, cameras, lights, tape_times, images, L, &mw, &mh, &ms);
    if (r != FREP_OK) return r;
    // The graph stays valid while the batch keeps its shape.
    std::vector<uint64_t> key = {L.total, st.slots, st.mm, st.longest, st.max_levels, mw, mh, ms,
                                 (uint64_t)b->plan4.blocks, (uint64_t)b->plan4.warps_per_block,
                                 (uint64_t)b->plan4.point_warps_per_block, (uint64_t)b->plan2.point_warps_per_block,
                                 (uint64_t)(uintptr_t)b->keep, (uint64_t)(uintptr_t)b->d_stage};
    for (uint32_t i = 0; i < b->n; i++) key.push_back(L.root_ofs[i]);
    if (!b->graph || key != b->graph_key) {
        if (b->graph) {
            cudaGraphExecDestroy(b->graph);
            b->graph = nullptr;
        }
        cudaStream_t cs = b->capture_stream;
        FREP_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        cudaError_t ce = cudaMemcpyAsync(b->d_stage, b->h_stage, L.total, cudaMemcpyHostToDevice, cs);
        frep_status vr = ce == cudaSuccess ? enqueue_voxelize(b, st, L, cs, false) : cuda_fail(ce, "upload");
        if (vr == FREP_OK) {
            ce = frep::launch_render_batch(reinterpret_cast<const frep::RenderArgs*>(b->d_stage + L.frames), b->n,
                                           mw, mh, ms, cs);
            if (ce != cudaSuccess) vr = cuda_fail(ce, "render_batch_kernel");
        }
        cudaGraph_t g = nullptr;
        cudaError_t ee = cudaStreamEndCapture(cs, &g);
        if (vr != FREP_OK) {
            if (g) cudaGraphDestroy(g);
            return vr;
        }
        if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
        ce = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaGraphInstantiate");
        b->graph_key = key;
    }
    FREP_CUDA(cudaGraphLaunch(b->graph, s));
    FREP_CUDA(cudaEventRecord(b->upload_done, s));
    return FREP_OK;
}

frep_status frep_batch_get_info(const frep_batch* b, frep_batch_info* info) {
    if (!b || !info) return fail(FREP_ERR_INVALID_ARG, "frep_batch_get_info: null argument");
    info->n_trees = b->n;
    info->voxelize_launches = b->last_launches;
    info->upload_bytes = b->last_upload;
    info->device_bytes = b->bytes;
    info->interval_warps_per_block = b->plan_valid ? (uint32_t)b->plan4.warps_per_block : 0;
    info->point_warps_per_block = b->plan_valid ? (uint32_t)b->plan4.point_warps_per_block : 0;
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
