// Internal definitions shared by the C-ABI translation units (capi.cu,
// batch.cu): the opaque handle structs and error helpers.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "frep.h"
#include "kernels.h"
#include "tape_compiler.h"

namespace frep {
namespace detail {

frep_status fail(frep_status s, const char* fmt, ...);
frep_status cuda_fail(cudaError_t e, const char* what);
inline uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

}  // namespace detail
}  // namespace frep

struct frep_tree;
namespace frep {
namespace detail {
// Trees whose header and pools are carved from caller-owned device memory.
// With such memory the device header is not written here: the tree keeps it
// (hdr_pending) until write_tree_header enqueues it on a stream, so that a
// caller holding a lock creates trees without touching the device.
uint64_t tree_external_bytes(uint64_t node_words, uint64_t tape_words);
frep_status tree_create_impl(frep_ctx* ctx, const frep_grid* grid, const frep_voxelize_opts* opts, uint8_t* ext,
                             uint64_t ext_bytes, cudaStream_t stream, frep_tree** out);
// Enqueues the pending header write of a tree in caller memory (no-op when
// already written); the tree is usable on `stream` afterwards.
frep_status write_tree_header(frep_tree* tree, cudaStream_t stream);
// Camera basis, lights and tree description for one frame (frep_render).
frep_status fill_render_args(const frep_tree* tree, const frep_camera* cam, const frep_lights* lights,
                             float tape_time, const frep_image* out, RenderArgs* args);
// The frame part alone (camera basis, lights, outputs): resets *args first.
frep_status fill_view_args(const frep_camera* cam, const frep_lights* lights, float tape_time,
                           const frep_image* out, RenderArgs* args);
// Host time of a batch's last frep_batch_voxelize, ms: plans, prefix and
// scratch; the upload area; staging and launches.
void batch_host_ms(const frep_batch* b, double out[3]);
}  // namespace detail
}  // namespace frep

#define FREP_CUDA(call)                                                   \
    do {                                                                  \
        cudaError_t e_ = (call);                                          \
        if (e_ != cudaSuccess) return frep::detail::cuda_fail(e_, #call); \
    } while (0)

struct frep_tape {
    frep::CompiledTape ct;
    std::vector<uint64_t> record;  // [n_instr][instrs...] padded to 16 words
    void build_record() {
        record.assign(frep::detail::align_up(1 + ct.instrs.size(), frep::dev::TAPE_ALIGN_WORDS), 0);
        record[0] = ct.instrs.size();
        std::memcpy(&record[1], ct.instrs.data(), ct.instrs.size() * 8);
    }
};

struct frep_ctx {
    int device = 0;
    uint64_t budget = 0;
    uint64_t used = 0;
    int sm_count = 0;
};

struct frep_tree {
    frep_ctx* ctx = nullptr;
    frep_grid grid{};
    frep_voxelize_opts opts{};
    int point_k = 4;  // cells per lane of the last-level pass in batches (its batch kind, 4 or 2)
    int plain_k = 4;  // cells per lane of its own last-level passes (frep_voxelize and variants)
    bool external = false;  // header and pools live in caller-owned memory
    bool hdr_pending = false;              // external: header not yet written to the device
    frep::dev::TreeHeader pending_hdr{};   //   (write_tree_header)
    float cell_size[FREP_MAX_LEVELS] = {};
    uint32_t node_size[FREP_MAX_LEVELS] = {};
    frep::dev::TreeHeader* hdr = nullptr;
    // A batch of one, for the level launches: d_self[0] = hdr, the work prefix
    // (2 entries) and the work cursor, in one small device allocation.
    unsigned long long* d_small = nullptr;
    frep::dev::TreeHeader** d_self = nullptr;
    unsigned long long* d_prefix = nullptr;
    unsigned long long* d_cursor = nullptr;
    uint32_t* nodes = nullptr;
    uint64_t* tapes = nullptr;
    uint64_t node_cap = 0, tape_cap = 0;
    uint32_t* keep = nullptr;
    uint64_t keep_words = 0;
    uint64_t bytes = 0;
    // staging for the root tape upload
    uint64_t* staging = nullptr;
    uint64_t staging_words = 0;
    cudaEvent_t upload_done = nullptr;
    // the root tape of the last voxelization
    uint32_t n_slots = 4, mm_cap = 0, root_n = 0, root_words = 0;
    bool plan_valid = false;
    uint32_t plan_slots = 0, plan_mm = 0, plan_round = 0;
    frep::LevelPlan plan{};
    cudaStream_t stream = nullptr;
    bool voxelized = false;
    bool profile = false;
    // reuse of a previous tree (frep_voxelize_reuse), allocated on first use:
    // reuse_src one u32 per node (reuse_slot), reuse_list the nodes of a level
    // to evaluate (reuse_words entries each); reuse_last: the last
    // voxelization copied the nodes whose entry is set
    uint32_t* reuse_src = nullptr;
    uint32_t* reuse_list = nullptr;
    uint64_t reuse_words = 0;
    bool reuse_last = false;
    cudaEvent_t ev[FREP_MAX_LEVELS + 1] = {};
};

