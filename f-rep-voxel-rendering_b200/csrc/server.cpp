// Serving loop (frep_server_*): continuous batching of voxelize + render
// requests over resident trees, admission by an HBM budget, LRU eviction.
//
// Threads: callers submit from any thread; a scheduler thread forms steps and
// enqueues them on the server's stream; a completion thread waits for each
// step's event in order, checks the voxelized trees' pool use (read back in
// the step itself) and publishes the results.
//
// Everything a step does on the device is ordered on one stream, so memory
// handed back by an eviction, and the frame area, can be reused by the next
// step at once: the device finishes the earlier step before it starts the
// later one. The host only has to keep its own bookkeeping straight.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <thread>
#include <unordered_map>
#include <vector>

#include "arena.h"
#include "capi_internal.h"

using frep::detail::align_up;
using frep::detail::cuda_fail;
using frep::detail::fail;
using frep::serving::Arena;
using frep::serving::LruOrder;

namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t).count();
}

struct Scene {
    uint64_t id = 0;  // index in frep_server::scenes
    frep_tape tape;
    frep_grid grid{};
    frep_voxelize_opts opts{};
    uint64_t node_words = 0, tape_words = 0;  // pool request for the next admission
    frep_tree* tree = nullptr;
    uint64_t arena_off = 0, arena_bytes = 0;
    bool valid = false;      // the tree holds the scene at `time` (as of the last enqueued step)
    float time = 0.0f;
    uint64_t gen = 0;        // voxelizations enqueued so far
    uint64_t bad_gen = ~0ull;  // a voxelization that overflowed
    uint64_t last_used = 0;  // LRU tick
    uint64_t step = 0;       // last step that referenced the tree
    bool rebuild = false;    // pools grew after an overflow: recreate the tree
};

struct Request {
    frep_request req{};
    Clock::time_point submit;
    int32_t state = FREP_REQ_QUEUED;
    int32_t status = FREP_OK;
    uint32_t voxelized = 0;
    uint32_t retries = 0;
    uint64_t gen = 0;  // the scene's voxelization this request rendered
    double latency_ms = 0.0;
};

struct Step {
    uint64_t id = 0;
    std::vector<uint64_t> requests;
    std::vector<uint64_t> vox_scenes;
    std::vector<uint64_t> vox_gens;
    cudaEvent_t done = nullptr;
    int ring = 0;  // usage buffer slot
};

constexpr int kRing = 8;  // usage read-back buffers (> max_inflight + 1)

}  // namespace

struct frep_server {
    frep_ctx* ctx = nullptr;
    frep_server_config cfg{};
    frep_lights lights{};
    cudaStream_t stream = nullptr;
    frep_batch* batch = nullptr;
    uint8_t* arena_mem = nullptr;
    Arena arena;
    uint8_t* d_frames = nullptr;
    uint64_t frames_bytes = 0;
    // usage read-back: per ring slot, tree header table (pinned + device) and results
    frep::dev::TreeHeader** h_tab[kRing] = {};
    frep::dev::TreeHeader** d_tab[kRing] = {};
    unsigned long long* h_use[kRing] = {};
    unsigned long long* d_use[kRing] = {};
    uint32_t ring_cap = 0;
    int ring_next = 0;

    std::mutex mu;
    std::condition_variable cv_work;   // scheduler: new requests or a finished step
    std::condition_variable cv_done;   // waiters: a request finished
    std::condition_variable cv_steps;  // completion thread: a new step
    std::deque<uint64_t> pending;
    std::unordered_map<uint64_t, Request> requests;
    std::vector<std::unique_ptr<Scene>> scenes;
    // resident scenes (a tree in the arena) by (last_used, id): the eviction
    // order, found in O(log n) however many scenes are registered
    LruOrder lru;
    std::deque<Step> inflight;
    uint64_t next_request = 1, next_step = 1, tick = 0;
    bool stop = false;
    frep_status fatal = FREP_OK;
    std::thread scheduler, completer;

    // statistics
    uint64_t submitted = 0, completed = 0, failed = 0, voxelized = 0, rerendered = 0, evictions = 0, steps = 0;
    uint64_t max_step_evictions = 0;  // most evictions one step's planning made
    double max_plan_ms = 0.0;         // longest planning of one step (the lock held)
    double max_enqueue_ms = 0.0;      // longest host time to enqueue one step
    double slow_ms = 0.0;             // FREP_SERVER_SLOW_MS: log steps slower to enqueue (0 = off)
    std::vector<double> latencies;
    bool window_open = false;
    Clock::time_point window_start, window_end;
};

namespace {

// Pool estimate for a scene without given sizes: generous for the first
// voxelization; refitted from the measured use afterwards.
void estimate_pools(Scene& S) {
    const uint64_t n = S.tape.ct.instrs.size();
    uint64_t nodes = 1, words = 0;
    for (uint32_t l = 0; l < S.grid.levels; l++) {
        const uint64_t d3 = (uint64_t)S.grid.dims[l] * S.grid.dims[l] * S.grid.dims[l];
        words += nodes * frep::dev::node_words(S.grid.dims[l], l + 1 == S.grid.levels);
        nodes = std::min<uint64_t>(nodes * d3, 1ull << 40);
    }
    S.node_words = S.opts.node_words ? S.opts.node_words : std::min<uint64_t>(words, 16ull << 20);
    S.tape_words = S.opts.tape_words ? S.opts.tape_words : std::max<uint64_t>(64 * n, 4ull << 20);
    // at least the root node and the root tape
    S.node_words = std::max<uint64_t>(S.node_words, frep::dev::node_words(S.grid.dims[0], S.grid.levels == 1) + 64);
    S.tape_words = std::max<uint64_t>(S.tape_words, S.tape.record.size() + 64);
}

// Releases the scene's tree; returns the size of the free arena block that
// now holds its memory.
uint64_t drop_tree(frep_server* sv, Scene& S) {
    sv->lru.erase({S.last_used, S.id});
    frep_tree_destroy(S.tree);
    const uint64_t merged = sv->arena.release(S.arena_off, S.arena_bytes);
    S.tree = nullptr;
    S.valid = false;
    return merged;
}

uint64_t evict(frep_server* sv, Scene& S) {
    sv->evictions++;
    return drop_tree(sv, S);
}

// Marks a scene used by the step being formed (its place in the LRU order).
void touch(frep_server* sv, Scene& S) {
    if (S.tree) sv->lru.erase({S.last_used, S.id});
    S.last_used = sv->tick;
    if (S.tree) sv->lru.insert({S.last_used, S.id});
}

// Places the scene's tree in the arena, evicting least recently used trees
// that the step being formed does not use. false: it does not fit.
bool admit(frep_server* sv, Scene& S, uint64_t step) {
    const uint64_t bytes = frep::detail::tree_external_bytes(S.node_words, S.tape_words);
    if (bytes > sv->arena.capacity()) return false;
    uint64_t off = 0;
    // Evict least recently used trees (not those of the step being formed)
    // until a free block holds the new one.
    const bool placed = frep::serving::place_evicting(
        sv->arena, sv->lru, bytes, [&](uint64_t id) { return sv->scenes[id]->step == step; },
        [&](uint64_t id) { return evict(sv, *sv->scenes[id]); }, &off);
    if (!placed) return false;
    frep_voxelize_opts o = S.opts;
    o.node_words = S.node_words;
    o.tape_words = S.tape_words;
    frep_status st = frep::detail::tree_create_impl(sv->ctx, &S.grid, &o, sv->arena_mem + off, bytes, sv->stream,
                                                    &S.tree);
    if (st != FREP_OK) {
        sv->arena.release(off, bytes);
        S.tree = nullptr;
        return false;
    }
    S.arena_off = off;
    S.arena_bytes = bytes;
    S.valid = false;
    sv->lru.insert({S.last_used, S.id});
    return true;
}

// Grows the frame area in stream order: the old area is released after the
// steps already enqueued on the server's stream (cudaFreeAsync) and the new
// one allocated on that stream, so a growth waits for no step (a cudaFree here
// waited for the whole device: up to 280 ms at 2000 requests/s). The first
// area holds max_batch frames of the step's largest frame (at most 1 GB), so
// that later steps of that frame size never grow it (a growth in the middle
// of a serving run still took 288 ms to allocate at 2000 requests/s).
frep_status ensure_frames(frep_server* sv, uint64_t bytes, uint64_t largest_frame) {
    if (bytes <= sv->frames_bytes) return FREP_OK;
    const uint64_t prev = sv->frames_bytes;
    if (sv->d_frames) FREP_CUDA(cudaFreeAsync(sv->d_frames, sv->stream));
    sv->d_frames = nullptr;
    sv->frames_bytes = 0;
    // at least double, and at least max_batch of the largest frame (up to 1 GB)
    const uint64_t presize = std::min<uint64_t>((uint64_t)sv->cfg.max_batch * largest_frame, 1ull << 30);
    const uint64_t cap = align_up(std::max<uint64_t>(std::max<uint64_t>(bytes + bytes / 4, 2 * prev), presize),
                                  1 << 20);
    FREP_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&sv->d_frames), cap, sv->stream));
    sv->frames_bytes = cap;
    return FREP_OK;
}

frep_status ensure_ring(frep_server* sv, uint32_t n) {
    if (n <= sv->ring_cap) return FREP_OK;
    FREP_CUDA(cudaStreamSynchronize(sv->stream));
    const uint32_t cap = std::max<uint32_t>(n, std::max<uint32_t>(sv->cfg.max_batch, 2 * sv->ring_cap));
    for (int i = 0; i < kRing; i++) {
        cudaFreeHost(sv->h_tab[i]);
        cudaFree(sv->d_tab[i]);
        cudaFreeHost(sv->h_use[i]);
        cudaFree(sv->d_use[i]);
        FREP_CUDA(cudaMallocHost(&sv->h_tab[i], sizeof(void*) * cap));
        FREP_CUDA(cudaMalloc(&sv->d_tab[i], sizeof(void*) * cap));
        FREP_CUDA(cudaMallocHost(&sv->h_use[i], sizeof(unsigned long long) * 3 * cap));
        FREP_CUDA(cudaMalloc(&sv->d_use[i], sizeof(unsigned long long) * 3 * cap));
    }
    sv->ring_cap = cap;
    return FREP_OK;
}

void finish_request(frep_server* sv, Request& R, int32_t state, int32_t status, Clock::time_point now) {
    R.state = state;
    R.status = status;
    R.latency_ms = std::chrono::duration<double, std::milli>(now - R.submit).count();
    if (state == FREP_REQ_DONE) {
        sv->completed++;
        (R.voxelized ? sv->voxelized : sv->rerendered)++;
        sv->latencies.push_back(R.latency_ms);
        sv->window_end = now;
    } else {
        sv->failed++;
    }
}

// What one step enqueues, gathered under the lock so that the enqueue itself
// runs without it (Request objects may move when the request map grows; the
// Scene objects and their trees do not, and only the scheduler thread
// creates or destroys trees).
struct StepPlan {
    Step step;
    std::vector<const frep_tape*> vtapes;
    std::vector<frep_tree*> vtrees;
    std::vector<float> vtimes;
    std::vector<const frep_tree*> ftrees;
    std::vector<frep_camera> cams;
    std::vector<float> ftimes;
    std::vector<uint8_t*> dst;
};

// Chooses the step's requests from the pending queue and places their trees
// (lock held). Returns false when nothing could be scheduled.
bool plan_step(frep_server* sv, StepPlan* P) {
    const uint64_t step_id = sv->next_step;
    sv->tick++;
    Step& st = P->step;
    st.id = step_id;
    std::unordered_map<uint64_t, float> vox_time;
    std::deque<uint64_t> deferred;
    const uint32_t max_batch = sv->cfg.max_batch;
    while (!sv->pending.empty() && st.requests.size() < max_batch) {
        const uint64_t rid = sv->pending.front();
        sv->pending.pop_front();
        Request& R = sv->requests[rid];
        Scene& S = *sv->scenes[R.req.scene];
        if (S.rebuild && S.tree && S.step != step_id) {
            // an overflowed voxelization: rebuild at the grown size
            drop_tree(sv, S);
            S.rebuild = false;
        }
        const float t = R.req.tape_time;
        const bool tdep = S.tape.ct.uses_time;
        auto same = [&](float a) { return !tdep || a == t; };
        auto it = vox_time.find(R.req.scene);
        if (it != vox_time.end()) {  // voxelized in this step
            if (!same(it->second)) {
                deferred.push_back(rid);
                continue;
            }
            R.voxelized = 0;
        } else if (S.tree && S.valid && same(S.time)) {  // resident: re-render only
            R.voxelized = 0;
        } else if (S.step == step_id) {
            // Re-rendered earlier in this step at another time: a voxelization
            // now would run before those frames (a step voxelizes first).
            deferred.push_back(rid);
            continue;
        } else {
            if (!S.tree && !admit(sv, S, step_id)) {
                if (frep::detail::tree_external_bytes(S.node_words, S.tape_words) > sv->arena.capacity()) {
                    finish_request(sv, R, FREP_REQ_FAILED, FREP_ERR_OOM, Clock::now());
                    sv->cv_done.notify_all();
                } else {
                    deferred.push_back(rid);
                }
                continue;
            }
            vox_time[R.req.scene] = t;
            S.valid = true;
            S.time = t;
            S.gen++;
            P->vtapes.push_back(&S.tape);
            P->vtrees.push_back(S.tree);
            P->vtimes.push_back(t);
            st.vox_scenes.push_back(R.req.scene);
            st.vox_gens.push_back(S.gen);
            R.voxelized = 1;
        }
        S.step = step_id;
        touch(sv, S);
        R.gen = S.gen;
        R.state = FREP_REQ_RUNNING;
        st.requests.push_back(rid);
        P->ftrees.push_back(S.tree);
        P->cams.push_back(R.req.camera);
        P->ftimes.push_back(t);
        P->dst.push_back(R.req.rgba8);
    }
    while (!deferred.empty()) {
        sv->pending.push_front(deferred.back());
        deferred.pop_back();
    }
    if (st.requests.empty()) return false;
    sv->next_step++;
    st.ring = sv->ring_next;
    sv->ring_next = (sv->ring_next + 1) % kRing;
    return true;
}

// Enqueues a planned step on the server's stream (no lock held; only the
// scheduler thread runs this and it owns the batch, frame area and ring).
frep_status enqueue_step(frep_server* sv, StepPlan& P) {
    frep_status r = FREP_OK;
    cudaStream_t s = sv->stream;
    Step& st = P.step;
    // phase marks for the slow-step log (FREP_SERVER_SLOW_MS)
    Clock::time_point mark[6];
    double vox_ms[3] = {};
    mark[0] = Clock::now();
    // headers of the trees admitted while the step was planned (under the
    // lock, where nothing is enqueued: a launch can wait for queue space)
    for (frep_tree* t : P.vtrees)
        if (r == FREP_OK) r = frep::detail::write_tree_header(t, s);
    mark[1] = Clock::now();
    if (r == FREP_OK && !P.vtrees.empty()) {
        if (!sv->batch) {
            r = frep_batch_create(sv->ctx, P.vtrees.data(), (uint32_t)P.vtrees.size(), &sv->batch);
            if (r == FREP_OK && (sv->cfg.interval_warps_per_block || sv->cfg.point_warps_per_block))
                r = frep_batch_set_tuning(sv->batch, sv->cfg.interval_warps_per_block, sv->cfg.point_warps_per_block);
        } else {
            r = frep_batch_set_trees(sv->batch, P.vtrees.data(), (uint32_t)P.vtrees.size());
        }
        if (r == FREP_OK) r = frep_batch_voxelize(sv->batch, P.vtapes.data(), P.vtimes.data(), s);
        frep::detail::batch_host_ms(sv->batch, vox_ms);
    }
    mark[2] = Clock::now();
    const uint32_t nf = (uint32_t)P.cams.size();
    std::vector<frep_image> imgs(nf);
    std::vector<uint64_t> ofs(nf);
    uint64_t total = 0, largest = 0;
    for (uint32_t i = 0; i < nf; i++) {
        ofs[i] = total;
        const uint64_t fb = align_up((uint64_t)P.cams[i].width * P.cams[i].height * 4, 256);
        total += fb;
        largest = std::max(largest, fb);
    }
    if (r == FREP_OK) r = ensure_frames(sv, total, largest);
    mark[3] = Clock::now();
    if (r == FREP_OK && !sv->batch) r = fail(FREP_ERR_INVALID_ARG, "frep_server: no voxelized tree to render");
    if (r == FREP_OK) {
        for (uint32_t i = 0; i < nf; i++) {
            imgs[i].rgba8 = sv->d_frames + ofs[i];
            imgs[i].hits = nullptr;
        }
        r = frep_batch_render_frames(sv->batch, P.ftrees.data(), nf, P.cams.data(), &sv->lights, P.ftimes.data(),
                                     imgs.data(), s);
    }
    mark[4] = Clock::now();
    // pool use of the voxelized trees, read back in the step
    if (r == FREP_OK) r = ensure_ring(sv, (uint32_t)P.vtrees.size());
    if (r == FREP_OK && !P.vtrees.empty()) {
        for (size_t i = 0; i < P.vtrees.size(); i++) sv->h_tab[st.ring][i] = P.vtrees[i]->hdr;
        cudaError_t e = cudaMemcpyAsync(sv->d_tab[st.ring], sv->h_tab[st.ring], sizeof(void*) * P.vtrees.size(),
                                        cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = frep::launch_gather_usage(sv->d_tab[st.ring], (uint32_t)P.vtrees.size(), sv->d_use[st.ring], s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(sv->h_use[st.ring], sv->d_use[st.ring],
                                sizeof(unsigned long long) * 3 * P.vtrees.size(), cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) r = cuda_fail(e, "frep_server: pool use read-back");
    }
    for (uint32_t i = 0; i < nf && r == FREP_OK; i++) {
        cudaError_t e = cudaMemcpyAsync(P.dst[i], sv->d_frames + ofs[i], (size_t)P.cams[i].width * P.cams[i].height * 4,
                                        cudaMemcpyDeviceToHost, s);
        if (e != cudaSuccess) r = cuda_fail(e, "frep_server: image copy");
    }
    if (r == FREP_OK) {
        cudaError_t e = cudaEventCreateWithFlags(&st.done, cudaEventDisableTiming | cudaEventBlockingSync);
        if (e == cudaSuccess) e = cudaEventRecord(st.done, s);
        if (e != cudaSuccess) r = cuda_fail(e, "frep_server: step event");
    }
    mark[5] = Clock::now();
    if (sv->slow_ms > 0.0) {
        auto d = [&](int a, int b) { return std::chrono::duration<double, std::milli>(mark[b] - mark[a]).count(); };
        if (d(0, 5) >= sv->slow_ms)
            std::fprintf(stderr,
                         "frep_server: step %llu enqueued in %.1f ms: headers %.1f, voxelize %.1f (plans/scratch %.1f, "
                         "upload area %.1f, staging/launches %.1f), frame area %.1f, render %.1f, read-backs %.1f; "
                         "%zu trees, %u frames\n",
                         (unsigned long long)st.id, d(0, 5), d(0, 1), d(1, 2), vox_ms[0], vox_ms[1], vox_ms[2],
                         d(2, 3), d(3, 4), d(4, 5), P.vtrees.size(), nf);
    }
    return r;
}

void scheduler_main(frep_server* sv) {
    cudaSetDevice(sv->ctx->device);
    std::unique_lock<std::mutex> lock(sv->mu);
    while (true) {
        sv->cv_work.wait(lock, [&] {
            return sv->stop || (!sv->pending.empty() && sv->inflight.size() < sv->cfg.max_inflight);
        });
        if (sv->stop) break;
        StepPlan P;
        const auto plan_start = Clock::now();
        const uint64_t ev_before = sv->evictions;
        const bool planned = plan_step(sv, &P);
        sv->max_plan_ms = std::max(sv->max_plan_ms, ms_since(plan_start));
        sv->max_step_evictions = std::max(sv->max_step_evictions, sv->evictions - ev_before);
        if (!planned) {
            // Nothing could be placed, although every tree outside the step
            // being formed may be evicted: the arena is exhausted for good.
            const auto now = Clock::now();
            while (!sv->pending.empty()) {
                finish_request(sv, sv->requests[sv->pending.front()], FREP_REQ_FAILED, FREP_ERR_OOM, now);
                sv->pending.pop_front();
            }
            sv->cv_done.notify_all();
            continue;
        }
        lock.unlock();
        const auto enqueue_start = Clock::now();
        const frep_status r = enqueue_step(sv, P);
        const double enqueue_ms = ms_since(enqueue_start);
        lock.lock();
        sv->max_enqueue_ms = std::max(sv->max_enqueue_ms, enqueue_ms);
        Step& st = P.step;
        if (r != FREP_OK) {
            // The step could not be enqueued: fail its requests, invalidate what it touched.
            const auto now = Clock::now();
            for (uint64_t rid : st.requests) finish_request(sv, sv->requests[rid], FREP_REQ_FAILED, r, now);
            for (uint64_t sc : st.vox_scenes) sv->scenes[sc]->valid = false;
            if (st.done) cudaEventDestroy(st.done);
            sv->cv_done.notify_all();
            continue;
        }
        sv->steps++;
        sv->inflight.push_back(std::move(st));
        sv->cv_steps.notify_all();
    }
}

void completer_main(frep_server* sv) {
    cudaSetDevice(sv->ctx->device);
    std::unique_lock<std::mutex> lock(sv->mu);
    // the previous step's event, destroyed outside the lock (a CUDA call
    // under the lock could make submits wait behind the driver)
    cudaEvent_t spent = nullptr;
    while (true) {
        sv->cv_steps.wait(lock, [&] { return sv->stop || !sv->inflight.empty(); });
        if (sv->inflight.empty()) {
            if (sv->stop) break;
            continue;
        }
        const cudaEvent_t ev = sv->inflight.front().done;
        lock.unlock();
        if (spent) cudaEventDestroy(spent);
        spent = nullptr;
        const cudaError_t e = cudaEventSynchronize(ev);
        const auto now = Clock::now();
        lock.lock();
        Step st = std::move(sv->inflight.front());
        sv->inflight.pop_front();
        spent = st.done;
        // Overflowed voxelizations: grow the scene's pools and run its
        // requests again (the tree is rebuilt at the new size).
        std::unordered_map<uint64_t, bool> overflowed;
        for (size_t i = 0; i < st.vox_scenes.size() && e == cudaSuccess; i++) {
            Scene& S = *sv->scenes[st.vox_scenes[i]];
            const unsigned long long* u = sv->h_use[st.ring] + 3 * i;
            if (u[0]) {
                if (u[0] & 1u) S.node_words *= 2;
                if (u[0] & 2u) S.tape_words *= 2;
                S.bad_gen = st.vox_gens[i];
                if (S.gen == st.vox_gens[i]) {
                    // The scheduler rebuilds the tree at the new size when the
                    // scene is next requested (steps already enqueued that use
                    // it run first: one stream).
                    S.valid = false;
                    S.rebuild = true;
                }
            } else if (!S.opts.node_words) {
                // refit: what this voxelization used, plus headroom
                S.node_words = std::max<uint64_t>(u[1] + u[1] / 8 + 4096, 4096);
                S.tape_words = std::max<uint64_t>(u[2] + u[2] / 8 + 4096, S.tape.record.size() + 4096);
            }
        }
        std::deque<uint64_t> retry;
        for (uint64_t rid : st.requests) {
            Request& R = sv->requests[rid];
            Scene& S = *sv->scenes[R.req.scene];
            if (e != cudaSuccess) {
                finish_request(sv, R, FREP_REQ_FAILED, FREP_ERR_CUDA, now);
            } else if (S.bad_gen == R.gen) {
                if (++R.retries > 4) {
                    finish_request(sv, R, FREP_REQ_FAILED, FREP_ERR_CAPACITY, now);
                } else {
                    R.state = FREP_REQ_QUEUED;
                    retry.push_back(rid);
                }
            } else {
                finish_request(sv, R, FREP_REQ_DONE, FREP_OK, now);
            }
        }
        while (!retry.empty()) {
            sv->pending.push_front(retry.back());
            retry.pop_back();
        }
        if (e != cudaSuccess && sv->fatal == FREP_OK) sv->fatal = cuda_fail(e, "frep_server: step");
        sv->cv_done.notify_all();
        sv->cv_work.notify_all();
    }
    lock.unlock();
    if (spent) cudaEventDestroy(spent);
}

}  // namespace

extern "C" {

frep_status frep_server_create(frep_ctx* ctx, const frep_server_config* config, const frep_lights* lights,
                               frep_server** out) {
    if (!ctx || !out) return fail(FREP_ERR_INVALID_ARG, "frep_server_create: null argument");
    FREP_CUDA(cudaSetDevice(ctx->device));
    auto sv = std::make_unique<frep_server>();
    sv->ctx = ctx;
    if (const char* v = std::getenv("FREP_SERVER_SLOW_MS")) sv->slow_ms = std::atof(v);
    if (config) sv->cfg = *config;
    if (!sv->cfg.max_batch) sv->cfg.max_batch = 512;
    if (!sv->cfg.max_inflight) sv->cfg.max_inflight = 2;
    sv->cfg.max_inflight = std::min<uint32_t>(sv->cfg.max_inflight, kRing - 2);
    if (sv->cfg.max_batch > 65535) return fail(FREP_ERR_INVALID_ARG, "frep_server_create: max_batch above 65535");
    if (lights) sv->lights = *lights;
    else frep_lights_default(&sv->lights);
    const uint64_t left = ctx->budget > ctx->used ? ctx->budget - ctx->used : 0;
    uint64_t arena = sv->cfg.hbm_budget ? sv->cfg.hbm_budget : left / 5 * 4;
    arena = align_up(arena, 4096);
    if (arena == 0 || arena > left) return fail(FREP_ERR_OOM, "frep_server_create: arena of %llu bytes exceeds the budget",
                                                (unsigned long long)arena);
    sv->cfg.hbm_budget = arena;
    cudaError_t e = cudaMalloc(&sv->arena_mem, arena);
    if (e != cudaSuccess) return fail(FREP_ERR_OOM, "frep_server_create: cudaMalloc(%llu) failed (%s)",
                                      (unsigned long long)arena, cudaGetErrorString(e));
    sv->arena.reset(arena);
    ctx->used += arena;
    e = cudaStreamCreateWithFlags(&sv->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        cudaFree(sv->arena_mem);
        ctx->used -= arena;
        return cuda_fail(e, "frep_server_create: stream");
    }
    frep_server* raw = sv.release();
    raw->scheduler = std::thread(scheduler_main, raw);
    raw->completer = std::thread(completer_main, raw);
    *out = raw;
    return FREP_OK;
}

void frep_server_destroy(frep_server* sv) {
    if (!sv) return;
    {
        std::unique_lock<std::mutex> lock(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    sv->cv_steps.notify_all();
    if (sv->scheduler.joinable()) sv->scheduler.join();
    // the completion thread drains the steps already on the device
    {
        std::unique_lock<std::mutex> lock(sv->mu);
        sv->cv_steps.notify_all();
    }
    if (sv->completer.joinable()) sv->completer.join();
    cudaSetDevice(sv->ctx->device);
    cudaStreamSynchronize(sv->stream);
    for (auto& S : sv->scenes)
        if (S->tree) frep_tree_destroy(S->tree);
    if (sv->batch) frep_batch_destroy(sv->batch);
    for (int i = 0; i < kRing; i++) {
        cudaFreeHost(sv->h_tab[i]);
        cudaFree(sv->d_tab[i]);
        cudaFreeHost(sv->h_use[i]);
        cudaFree(sv->d_use[i]);
    }
    cudaFree(sv->d_frames);
    cudaFree(sv->arena_mem);
    sv->ctx->used -= std::min<uint64_t>(sv->ctx->used, sv->cfg.hbm_budget);
    cudaStreamDestroy(sv->stream);
    delete sv;
}

frep_status frep_server_add_scene(frep_server* sv, const frep_tape* tape, const frep_grid* grid,
                                  const frep_voxelize_opts* opts, uint64_t* scene) {
    if (!sv || !tape || !grid || !scene) return fail(FREP_ERR_INVALID_ARG, "frep_server_add_scene: null argument");
    if (grid->levels == 0 || grid->levels > FREP_MAX_LEVELS)
        return fail(FREP_ERR_INVALID_ARG, "frep_server_add_scene: bad grid");
    for (uint32_t l = 0; l < grid->levels; l++)
        if (grid->dims[l] < 4 || grid->dims[l] > 32 || grid->dims[l] % 4)
            return fail(FREP_ERR_INVALID_ARG, "frep_server_add_scene: dims[%u] = %u", l, grid->dims[l]);
    if (opts && opts->point_cells_per_lane != 0 && opts->point_cells_per_lane != 2 && opts->point_cells_per_lane != 4)
        return fail(FREP_ERR_INVALID_ARG, "frep_server_add_scene: point_cells_per_lane must be 0, 2 or 4");
    auto S = std::make_unique<Scene>();
    S->tape = *tape;
    S->grid = *grid;
    if (opts) S->opts = *opts;
    else { S->opts.rounding = FREP_ROUND_OUTWARD; S->opts.shorten = 1; }
    estimate_pools(*S);
    std::lock_guard<std::mutex> lock(sv->mu);
    *scene = sv->scenes.size();
    S->id = *scene;
    sv->scenes.push_back(std::move(S));
    return FREP_OK;
}

frep_status frep_server_submit(frep_server* sv, const frep_request* req, uint64_t* request_id) {
    if (!sv || !req || !request_id || !req->rgba8) return fail(FREP_ERR_INVALID_ARG, "frep_server_submit: null argument");
    if (req->camera.width == 0 || req->camera.height == 0 || req->camera.projection > 1)
        return fail(FREP_ERR_INVALID_ARG, "frep_server_submit: bad camera");
    const auto submitted_at = Clock::now();  // latency includes any wait for the lock
    std::lock_guard<std::mutex> lock(sv->mu);
    if (sv->fatal != FREP_OK) return fail(sv->fatal, "frep_server: a step failed on the device");
    if (req->scene >= sv->scenes.size()) return fail(FREP_ERR_INVALID_ARG, "frep_server_submit: unknown scene");
    const uint64_t id = sv->next_request++;
    Request& R = sv->requests[id];
    R.req = *req;
    R.submit = submitted_at;
    if (!sv->window_open) {
        sv->window_open = true;
        sv->window_start = R.submit;
    }
    sv->submitted++;
    sv->pending.push_back(id);
    *request_id = id;
    sv->cv_work.notify_all();
    return FREP_OK;
}

static void fill_status(const Request& R, frep_request_status* out) {
    out->state = R.state;
    out->status = R.status;
    out->voxelized = R.voxelized;
    out->retries = R.retries;
    out->latency_ms = R.latency_ms;
}

frep_status frep_server_poll(frep_server* sv, uint64_t request_id, frep_request_status* status) {
    if (!sv || !status) return fail(FREP_ERR_INVALID_ARG, "frep_server_poll: null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->requests.find(request_id);
    if (it == sv->requests.end()) return fail(FREP_ERR_INVALID_ARG, "frep_server_poll: unknown request");
    fill_status(it->second, status);
    return FREP_OK;
}

frep_status frep_server_wait(frep_server* sv, uint64_t request_id, uint32_t timeout_ms,
                             frep_request_status* status) {
    if (!sv) return fail(FREP_ERR_INVALID_ARG, "frep_server_wait: null server");
    std::unique_lock<std::mutex> lock(sv->mu);
    auto it = sv->requests.find(request_id);
    if (it == sv->requests.end()) return fail(FREP_ERR_INVALID_ARG, "frep_server_wait: unknown request");
    const bool ok = sv->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] {
        return it->second.state == FREP_REQ_DONE || it->second.state == FREP_REQ_FAILED;
    });
    if (status) fill_status(it->second, status);
    if (!ok) return fail(FREP_ERR_TIMEOUT, "frep_server_wait: request %llu not finished after %u ms",
                         (unsigned long long)request_id, timeout_ms);
    return FREP_OK;
}

frep_status frep_server_release(frep_server* sv, uint64_t request_id) {
    if (!sv) return fail(FREP_ERR_INVALID_ARG, "frep_server_release: null server");
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->requests.find(request_id);
    if (it == sv->requests.end()) return fail(FREP_ERR_INVALID_ARG, "frep_server_release: unknown request");
    if (it->second.state != FREP_REQ_DONE && it->second.state != FREP_REQ_FAILED)
        return fail(FREP_ERR_INVALID_ARG, "frep_server_release: request %llu is not finished",
                    (unsigned long long)request_id);
    sv->requests.erase(it);
    return FREP_OK;
}

frep_status frep_server_drain(frep_server* sv, uint32_t timeout_ms) {
    if (!sv) return fail(FREP_ERR_INVALID_ARG, "frep_server_drain: null server");
    std::unique_lock<std::mutex> lock(sv->mu);
    const bool ok = sv->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] {
        return sv->completed + sv->failed == sv->submitted;
    });
    if (!ok) return fail(FREP_ERR_TIMEOUT, "frep_server_drain: %llu of %llu requests unfinished after %u ms",
                         (unsigned long long)(sv->submitted - sv->completed - sv->failed),
                         (unsigned long long)sv->submitted, timeout_ms);
    return sv->fatal;
}

frep_status frep_server_get_stats(frep_server* sv, int reset, frep_server_stats* out) {
    if (!sv || !out) return fail(FREP_ERR_INVALID_ARG, "frep_server_get_stats: null argument");
    std::lock_guard<std::mutex> lock(sv->mu);
    std::memset(out, 0, sizeof(*out));
    out->submitted = sv->submitted;
    out->completed = sv->completed;
    out->failed = sv->failed;
    out->voxelized = sv->voxelized;
    out->rerendered = sv->rerendered;
    out->evictions = sv->evictions;
    out->steps = sv->steps;
    out->resident_trees = sv->lru.size();
    out->resident_bytes = sv->arena.used();
    out->arena_bytes = sv->arena.capacity();
    std::vector<double> l = sv->latencies;
    if (!l.empty()) {
        auto pct = [&](double q) {
            const size_t k = std::min(l.size() - 1, (size_t)(q * (double)(l.size() - 1) + 0.5));
            std::nth_element(l.begin(), l.begin() + k, l.end());
            return l[k];
        };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        double sum = 0.0, mx = 0.0;
        for (double v : sv->latencies) {
            sum += v;
            mx = std::max(mx, v);
        }
        out->mean_ms = sum / (double)sv->latencies.size();
        out->max_ms = mx;
        const double span = std::chrono::duration<double>(sv->window_end - sv->window_start).count();
        out->scenes_per_s = span > 0.0 ? (double)sv->latencies.size() / span : 0.0;
    }
    out->max_plan_ms = sv->max_plan_ms;
    out->max_enqueue_ms = sv->max_enqueue_ms;
    out->max_step_evictions = sv->max_step_evictions;
    if (reset) {
        sv->latencies.clear();
        sv->window_open = false;
        sv->max_plan_ms = 0.0;
        sv->max_enqueue_ms = 0.0;
        sv->max_step_evictions = 0;
    }
    return FREP_OK;
}

}  // extern "C"
