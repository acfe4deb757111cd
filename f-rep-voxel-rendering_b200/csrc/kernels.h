// Host-side launch interface of the CUDA kernels (voxelizer.cu, raytracer.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace frep {
namespace dev {
struct TreeHeader;
}

// One level launch over a batch of trees (a single tree is a batch of one).
// The scan kernel fills `prefix` (work items before each tree, for the trees
// this launch serves) and resets `cursor`; the level kernel then hands out
// items of every tree from that one cursor.
struct LevelLaunch {
    dev::TreeHeader* const* trees;     // device array of n_trees header pointers
    unsigned long long* prefix;        // device, n_trees + 1 entries
    unsigned long long* cursor;        // device work cursor
    uint32_t n_trees;
    uint32_t level;
    uint32_t* keep_scratch;            // per-warp global scratch of the interval pass:
    uint32_t keep_stride;              //   u32 words per warp: keep masks [mm_ofs words,
    uint32_t mm_ofs;                   //   >= longest tape] then MIN/MAX choice masks
    uint32_t n_slots;                  // slot-file rows per lane (max over the batch)
    uint32_t mm_cap;                   // MIN/MAX choice entries per warp (max over the batch)
    uint32_t smem_per_warp;            // bytes (set by launch_level from the plan)
    const uint32_t* eval_list;         // one-tree launches that copy subtrees from a previous
                                       //   tree: the nodes to evaluate (reuse_eval[level] of
                                       //   them, listed by reuse_match_kernel); null = all
    uint32_t any_point_k;              // 1: a one-tree launch, whose last level runs with the
                                       //   launch's cells per lane whatever the tree's batch
                                       //   kind (TreeHeader::point_k); 0: only trees of that kind
    uint32_t item_ofs;                 // per-warp scratch, u32 words: where the item tapes start
    uint32_t item_cap;                 //   and how many u64 words they may take (0 = no item
                                       //   pruning in the interval passes)
};

// Per-warp global scratch of the interval pass, in u32 words: one keep mask per
// instruction of the longest tape, then a pair of choice masks per MIN/MAX,
// then (with item pruning) the work items' pruned tapes, u64 words.
struct WarpScratch {
    uint32_t stride;    // words per warp
    uint32_t mm_ofs;    // where the choice masks start
    uint32_t item_ofs;  // where the item tapes start
    uint32_t item_cap;  // u64 words of item tapes (0 = no item pruning)
};
// At most this many u64 words of item tapes per warp (256 KB; a multiple of
// 16 and at most 2^19, so that an item tape's offset / 16 packs into 15
// bits): a group of up to 32 items of one node stores the pruned tapes that
// fit, the others run on the node's tape. (On the 128-scene batch, 1 MB per
// warp executed exactly the same instructions.)
constexpr uint32_t kItemTapeWords = 32768;
// ki: cells per lane of the interval pass (a keep mask and a choice-mask pair
// per group of 32 cells). items: room for item tapes.
inline WarpScratch warp_scratch(uint32_t longest, uint32_t mm_cap, uint32_t ki, bool items = false) {
    const uint32_t k = (ki * (longest ? longest : 1u) + 31u) / 32u * 32u;
    const uint32_t m = (2u * ki * (mm_cap ? mm_cap : 1u) + 31u) / 32u * 32u;
    const uint64_t want = 32ull * (longest ? longest : 1u);
    const uint32_t ic = items ? (uint32_t)(want < kItemTapeWords ? (want + 15u) / 16u * 16u : kItemTapeWords) : 0u;
    return WarpScratch{k + m + 2u * ic, k, k + m, ic};
}



// Launch geometry of the level passes for one (slot count, MIN/MAX count).
struct LevelPlan {
    int warps_per_block;
    int blocks;                        // persistent grid
    uint32_t smem_per_warp;
    int interval_ki;                   // cells per lane in the interval passes (1 or 2)
    int point_k;                       // cells per lane in the point pass
    int point_warps_per_block;
    int point_blocks;
    uint32_t point_smem_per_warp;
};

// Cells per lane the point pass uses for a last level of this dim.
int point_k_for(uint32_t dim);
// interval_warps / point_warps: warps (tapes) per block, 0 = chosen from the
// shared memory a warp needs, 1 or 4 = that many where shared memory allows.
// interval_ki: cells per lane of the interval passes, 1 or 2 (0 = default).
cudaError_t plan_levels(uint32_t n_slots, uint32_t mm_cap, int point_k, int rounding, LevelPlan* plan,
                        int interval_warps = 0, int point_warps = 0, int interval_ki = 0);

// Resets the headers of n trees (tape time from `tape_times`, or `tape_time`
// when it is null) and writes their root nodes. Each tree's root tape must
// already be at word 0 of its tape pool.
cudaError_t launch_tree_init(dev::TreeHeader* const* trees, uint32_t n, const float* tape_times, float tape_time,
                             cudaStream_t stream);
// Same for a batch whose root tapes are staged in one device buffer: tree i's
// record is words [offsets[i], offsets[i+1]) of `staged`; it is copied to
// word 0 of the tree's pool first. tape_times has n entries.
cudaError_t launch_tree_init_staged(dev::TreeHeader* const* trees, uint32_t n, const uint64_t* staged,
                                    const unsigned long long* offsets, const float* tape_times,
                                    cudaStream_t stream);
// Work prefix of `level` over the batch, for interval (point = false) or
// point passes with `point_k` cells per lane.
// out[3i..3i+2] = overflow flags, node words used, tape words used of tree i.
cudaError_t launch_gather_usage(dev::TreeHeader* const* trees, uint32_t n, unsigned long long* out,
                                cudaStream_t stream);
cudaError_t launch_level_scan(const LevelLaunch& a, bool point, int point_k, cudaStream_t stream);
cudaError_t launch_level(const LevelLaunch& a, const LevelPlan& plan, int rounding, bool point,
                         cudaStream_t stream, int interval_ki = 0);

// Reuse of a previous tree (reuse.cu), one tree per launch; src is the tree's
// side array (one u32 per node, indexed by reuse_slot).
// match: entries of the nodes of `level` present now (previous node id or ~0);
// the nodes left to evaluate are appended to `list` (count: reuse_eval[level]).
// copy: the nodes of `level` with an entry are copied from `prev`, with their
// children (entries set to the previous children).
cudaError_t launch_reuse_match(dev::TreeHeader* hdr, const dev::TreeHeader* prev, uint32_t* src, uint32_t* list,
                               uint32_t level, cudaStream_t stream);
cudaError_t launch_reuse_copy(dev::TreeHeader* hdr, const dev::TreeHeader* prev, uint32_t* src, uint32_t level,
                              cudaStream_t stream);

// Op-weighted work of every node of `level` (interval or point weights),
// added to the header's fp32_ops[level].
// Nodes with a `skip` entry other than ~0 (copied, not evaluated) are left out.
cudaError_t launch_count_ops(dev::TreeHeader* hdr, const uint32_t* nodes, const uint64_t* tapes,
                             unsigned long long node_cap, uint32_t level, uint32_t node_size,
                             uint32_t cells, bool point, const uint32_t* skip, cudaStream_t stream);

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
    uint32_t compact;                // 1: nodes are in the compact layout (compact.cu), whose
    unsigned long long node_ofs[8];  //   level offsets (u32 words) are given here; 0: the
                                     //   reference's layout, offsets from hdr
};

cudaError_t launch_render(const RenderArgs& a, cudaStream_t stream);
// out[p] = rounded mean of the n layers' rgb at pixel p, alpha 255 (layers:
// n consecutive rgba8 images of `pixels` pixels).
cudaError_t launch_resolve_layers(const uint8_t* layers, uint32_t n, uint32_t pixels, uint8_t* out,
                                  cudaStream_t stream);
// Renders n frames in one launch: args is a device array of n RenderArgs,
// max_w / max_h bound every frame's size.
cudaError_t launch_render_batch(const RenderArgs* args, uint32_t n, uint32_t max_w, uint32_t max_h,
                                uint32_t max_slots, cudaStream_t stream);

}  // namespace frep
