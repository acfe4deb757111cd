// Host-side launch interface of the CUDA kernels (voxelizer.cu, raytracer.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace frep {
namespace dev {
struct TreeHeader;
}

// Arguments of one level pass (voxelizer/main.comp's ParamsBuffer, made
// per-launch and device-resident where the reference read it back on the host).
struct LevelArgs {
    dev::TreeHeader* hdr;
    uint32_t* nodes;
    unsigned long long node_cap;     // u32 words
    uint64_t* tapes;
    unsigned long long tape_cap;     // u64 words
    uint32_t* keep_scratch;          // per-warp keep ballots (global scratch)
    uint32_t keep_stride;            // u32 words per warp (>= longest tape)
    uint32_t level, levels;
    uint32_t dim, dim_next;
    uint32_t node_size, node_size_next;
    float cell_size;
    float low[3];
    float tape_time;
    uint32_t n_slots;                // slot-file entries per lane
    uint32_t mm_cap;                 // MIN/MAX choice entries per warp
    uint32_t shorten;
    uint32_t smem_per_warp;          // bytes
};

// Launch geometry of the level passes for one (slot count, MIN/MAX count).
struct LevelPlan {
    int warps_per_block;
    int blocks;                      // persistent grid
    uint32_t smem_per_warp;
    int point_k;                     // cells per lane in the point pass
    int point_warps_per_block;
    int point_blocks;
    uint32_t point_smem_per_warp;
};

cudaError_t plan_levels(uint32_t n_slots, uint32_t mm_cap, uint32_t last_dim, int rounding,
                        LevelPlan* plan);
cudaError_t launch_tree_init(dev::TreeHeader* hdr, uint32_t* nodes, uint32_t root_n_instr,
                             uint32_t root_words, cudaStream_t stream);
cudaError_t launch_level(const LevelArgs& a, const LevelPlan& plan, int rounding, bool last,
                         cudaStream_t stream);

// Op-weighted work of every node of `level` (interval or point weights),
// added to the header's fp32_ops[level].
cudaError_t launch_count_ops(dev::TreeHeader* hdr, const uint32_t* nodes, const uint64_t* tapes,
                             unsigned long long node_cap, uint32_t level, uint32_t node_size,
                             uint32_t cells, bool point, cudaStream_t stream);

struct RenderArgs {
    const dev::TreeHeader* hdr;
    const uint32_t* nodes;
    const uint64_t* tapes;
    uint32_t levels;
    uint32_t dims[8];
    uint32_t node_size[8];
    float cell_size[8];
    float low[3];
    float world_size;
    float tape_time;
    float pos[3], fwd[3], right[3], up[3];
    float sws_x, sws_y, half_w, half_h;
    uint32_t projection, width, height, jitter;
    float jitter_seed;
    uint32_t n_lights;
    float light_dir[8][3];
    float light_color[8][4];
    float ambient[4];
    float background[4];
    uint32_t shadow_mask;
    uint32_t n_slots;
    uint8_t* rgba8;
    void* hits;                      // frep_hit*
};

cudaError_t launch_render(const RenderArgs& a, cudaStream_t stream);

}  // namespace frep
