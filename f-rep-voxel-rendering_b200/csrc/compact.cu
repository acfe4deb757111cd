// Compact trees: frep_tree_compact, frep_render_compact, export / import.
//
// Replaces SceneBuilder's compaction and layout (vulkan/src/engine/
// scene_builder.cpp: BuildNode :91-156, HasAllLeafChildren :79-89,
// CountInteriorNodes :158-168, LayoutNode :199-238). The reference builds
// that tree on the CPU by point-sampling every finest voxel and recursing per
// node; here the voxelizer's tree is compacted on the device, level by level:
//
//   1. (prune) compact_status_kernel, last level to root: per source node,
//      EMPTY (no leaf or interior cell after its children are compacted),
//      FULL (every cell a leaf) or KEPT — BuildNode's rules.
//   2. root to last level, with the nodes of level l already in preorder
//      (order[r] = source node of compact node r; the root is node 0):
//        compact_node_kernel     — masks after compaction, per-word interior
//                                  prefix counts, children per node, tape marks;
//        scan (3 kernels)        — children before each node = its base;
//        compact_children_kernel — the preorder of level l+1: the children of
//                                  node r, in cell order, at base[r] + k.
//      Children of consecutive nodes are consecutive, which is LayoutNode's
//      depth-first numbering restricted to one level.
//   3. tapes: every 16-word slot of the source pool that holds a used record
//      gets its record size, a scan gives the new offsets, the records are
//      copied once each (shared tapes stay shared) and node tape indices are
//      remapped.
// Every kernel takes its element count from the device header (no host
// round trip between levels); the call synchronizes once at the end to size
// the result exactly.
#include <cmath>
#include <memory>

#include "capi_internal.h"

using frep::detail::align_up;
using frep::detail::cuda_fail;
using frep::detail::fail;

struct frep_compact {
    frep_ctx* ctx = nullptr;
    frep_grid grid{};
    uint32_t mode = 0;
    uint32_t n_slots = 4;
    float cell_size[FREP_MAX_LEVELS] = {};
    uint32_t node_size[FREP_MAX_LEVELS] = {};
    uint32_t node_count[FREP_MAX_LEVELS] = {};
    uint64_t node_ofs[FREP_MAX_LEVELS] = {};
    uint64_t node_words = 0, tape_words = 0;
    uint32_t* nodes = nullptr;
    uint64_t* tapes = nullptr;
    uint64_t bytes = 0;
};

namespace frep {
namespace dev {

constexpr uint8_t ST_EMPTY = 0, ST_KEPT = 1, ST_FULL = 2;
constexpr unsigned FULL_MASK = 0xFFFFFFFFu;

// Words of a compact record: [tape, leaf[W], interior[W], prefix[W], base],
// last level [tape, leaf[W]].
__host__ __device__ inline uint32_t compact_words(uint32_t dim, bool last) {
    const uint32_t W = dim * dim * dim / 32;
    return last ? 1 + W : 2 + 3 * W;
}

struct CompactHeader {
    uint32_t count[MAX_LEVELS];             // compact nodes per level
    unsigned long long ofs[MAX_LEVELS];     // first word of each level
    uint32_t tape_slots;                    // 16-word slots of the source tape pool
    uint32_t tape_words;                    // words of the compact tape pool
};

// One level of the source tree (reference layout; counts read after its sync).
struct SrcLevel {
    const uint32_t* nodes;                  // first record of the level
    uint32_t size;                          // words per record
    uint32_t count;
    uint32_t dim;
    uint32_t last;
};

// BuildNode's rule for the interior cells of one mask word (list32: the
// child-list entries of its 32 cells): a FULL child becomes a leaf cell, an
// EMPTY child is dropped.
__device__ __forceinline__ void apply_child_status(const uint32_t* __restrict__ list32,
                                                   const uint8_t* __restrict__ child_st, uint32_t& leaf,
                                                   uint32_t& inter) {
    uint32_t bits = inter;
    while (bits) {
        const uint32_t b = __ffs(bits) - 1;
        bits &= bits - 1;
        const uint8_t cs = child_st[list32[b]];
        if (cs == ST_FULL) {
            leaf |= 1u << b;
            inter &= ~(1u << b);
        } else if (cs == ST_EMPTY) {
            inter &= ~(1u << b);
        }
    }
}

// A warp per source node of one level.
__global__ void __launch_bounds__(256) compact_status_kernel(SrcLevel S, const uint8_t* __restrict__ child_st,
                                                             uint8_t* __restrict__ st) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t c3 = S.dim * S.dim * S.dim, W = c3 >> 5;
    for (uint32_t node = warp; node < S.count; node += nwarps) {
        const uint32_t* r = S.nodes + (size_t)node * S.size;
        bool any = false, full = true;
        for (uint32_t w = lane; w < W; w += 32) {
            uint32_t leaf = __ldg(&r[4 + w]);
            uint32_t inter = 0;
            if (!S.last) {
                inter = __ldg(&r[4 + W + w]);
                apply_child_status(r + 4 + c3 / 16 + w * 32, child_st, leaf, inter);
            }
            any = any || (leaf | inter) != 0;
            full = full && leaf == 0xFFFFFFFFu;
        }
        any = __any_sync(FULL_MASK, any);
        full = __all_sync(FULL_MASK, full);
        if (lane == 0) st[node] = !any ? ST_EMPTY : (full ? ST_FULL : ST_KEPT);
    }
}

// A warp per compact node r of `level` (preorder): writes its record but the
// base, its child count, and marks its tape's slot.
__global__ void __launch_bounds__(256) compact_node_kernel(SrcLevel S, uint32_t level, uint32_t prune,
                                                           const uint8_t* __restrict__ child_st,
                                                           const uint32_t* __restrict__ order,
                                                           const CompactHeader* __restrict__ H,
                                                           uint32_t* __restrict__ dnodes, uint32_t dsize,
                                                           uint32_t* __restrict__ cnt,
                                                           uint32_t* __restrict__ tape_mark) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t c3 = S.dim * S.dim * S.dim, W = c3 >> 5;
    const uint32_t n = H->count[level];
    const unsigned long long lofs = H->ofs[level];
    for (uint32_t r = warp; r < n; r += nwarps) {
        const uint32_t src = order ? order[r] : 0u;
        const uint32_t* s = S.nodes + (size_t)src * S.size;
        uint32_t* d = dnodes + lofs + (size_t)r * dsize;
        if (lane == 0) {
            const uint32_t t = s[0];
            d[0] = t;
            tape_mark[t >> 4] = 1u;
        }
        uint32_t carry = 0;
        for (uint32_t c = 0; c < W; c += 32) {
            const uint32_t w = c + lane;
            uint32_t leaf = 0, inter = 0;
            if (w < W) {
                leaf = s[4 + w];
                if (!S.last) {
                    inter = s[4 + W + w];
                    if (prune) apply_child_status(s + 4 + c3 / 16 + w * 32, child_st, leaf, inter);
                }
                d[1 + w] = leaf;
            }
            if (!S.last) {
                const uint32_t pc = __popc(inter);
                uint32_t incl = pc;
#pragma unroll
                for (int k = 1; k < 32; k <<= 1) {
                    const uint32_t v = __shfl_up_sync(FULL_MASK, incl, k);
                    if (lane >= (uint32_t)k) incl += v;
                }
                if (w < W) {
                    d[1 + W + w] = inter;
                    d[1 + 2 * W + w] = carry + incl - pc;
                }
                carry += __shfl_sync(FULL_MASK, incl, 31);
            }
        }
        if (!S.last && lane == 0) cnt[r] = carry;
    }
}

// ofs[level + 1] = ofs[level] + count[level] * size (count[level + 1] is the
// scan's total).
__global__ void compact_ofs_kernel(CompactHeader* H, uint32_t level, uint32_t size) {
    H->ofs[level + 1] = H->ofs[level] + (unsigned long long)H->count[level] * size;
}

// A warp per compact node r of `level`: its base, and the preorder of level
// + 1 (next_order[base + k] = source node of its k-th child in cell order).
__global__ void __launch_bounds__(256) compact_children_kernel(SrcLevel S, uint32_t level,
                                                               const uint32_t* __restrict__ order,
                                                               const CompactHeader* __restrict__ H,
                                                               uint32_t* __restrict__ dnodes, uint32_t dsize,
                                                               const uint32_t* __restrict__ base,
                                                               uint32_t* __restrict__ next_order) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t c3 = S.dim * S.dim * S.dim, W = c3 >> 5;
    const uint32_t n = H->count[level];
    const unsigned long long lofs = H->ofs[level];
    for (uint32_t r = warp; r < n; r += nwarps) {
        const uint32_t src = order ? order[r] : 0u;
        const uint32_t* list = S.nodes + (size_t)src * S.size + 4 + c3 / 16;
        uint32_t* d = dnodes + lofs + (size_t)r * dsize;
        const uint32_t b = base[r];
        if (lane == 0) d[1 + 3 * W] = b;
        for (uint32_t w = lane; w < W; w += 32) {
            uint32_t bits = d[1 + W + w];
            uint32_t k = b + d[1 + 2 * W + w];
            while (bits) {
                const uint32_t bit = __ffs(bits) - 1;
                bits &= bits - 1;
                next_order[k++] = list[w * 32 + bit];
            }
        }
    }
}

// Marked slots get the size of the record they start (16-word multiples).
__global__ void tape_size_kernel(const uint64_t* __restrict__ tapes, uint32_t* __restrict__ mark,
                                 const CompactHeader* __restrict__ H) {
    const uint32_t n = H->tape_slots;
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x)
        if (mark[s]) {
            const uint32_t len = (uint32_t)tapes[(size_t)s * TAPE_ALIGN_WORDS];
            mark[s] = (1u + len + TAPE_ALIGN_WORDS - 1) / TAPE_ALIGN_WORDS * TAPE_ALIGN_WORDS;
        }
}

// A warp per slot: copies each used record to its new offset.
__global__ void __launch_bounds__(256) tape_copy_kernel(const uint64_t* __restrict__ src,
                                                        const uint32_t* __restrict__ size,
                                                        const uint32_t* __restrict__ newofs,
                                                        const CompactHeader* __restrict__ H,
                                                        uint64_t* __restrict__ dst) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const uint32_t n = H->tape_slots;
    for (uint32_t s = warp; s < n; s += nwarps) {
        const uint32_t words = size[s];
        if (!words) continue;
        const uint64_t* a = src + (size_t)s * TAPE_ALIGN_WORDS;
        uint64_t* b = dst + newofs[s];
        for (uint32_t i = lane; i < words; i += 32) b[i] = a[i];
    }
}

__global__ void tape_remap_kernel(const CompactHeader* __restrict__ H, uint32_t level, uint32_t* __restrict__ dnodes,
                                  uint32_t dsize, const uint32_t* __restrict__ newofs) {
    const uint32_t n = H->count[level];
    const unsigned long long lofs = H->ofs[level];
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        uint32_t* d = dnodes + lofs + (size_t)r * dsize;
        d[0] = newofs[d[0] >> 4];
    }
}

// ---- exclusive scan of u32 values, element count read on the device --------
constexpr uint32_t SCAN_THREADS = 1024;
constexpr uint32_t SCAN_BLOCKS = 296;  // <= SCAN_THREADS: the partials fit one block

// Exclusive scan of one value per thread of the block (a multiple of 32
// threads, at most 1024); *total gets the block's sum. Every thread of the
// block must call it.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_ofs[32];
    __shared__ uint32_t block_total;
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t incl = v;
#pragma unroll
    for (int k = 1; k < 32; k <<= 1) {
        const uint32_t u = __shfl_up_sync(FULL_MASK, incl, k);
        if (lane >= (uint32_t)k) incl += u;
    }
    if (lane == 31) warp_ofs[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        const uint32_t ws = lane < (blockDim.x >> 5) ? warp_ofs[lane] : 0u;
        uint32_t wi = ws;
#pragma unroll
        for (int k = 1; k < 32; k <<= 1) {
            const uint32_t u = __shfl_up_sync(FULL_MASK, wi, k);
            if (lane >= (uint32_t)k) wi += u;
        }
        warp_ofs[lane] = wi - ws;
        if (lane == 31) block_total = wi;
    }
    __syncthreads();
    const uint32_t excl = warp_ofs[wid] + incl - v;
    *total = block_total;
    __syncthreads();  // the next call rewrites warp_ofs / block_total
    return excl;
}

__device__ __forceinline__ void scan_range(uint32_t n, unsigned long long& b, unsigned long long& e) {
    const unsigned long long chunk = ((unsigned long long)n + gridDim.x - 1) / gridDim.x;
    b = min((unsigned long long)blockIdx.x * chunk, (unsigned long long)n);
    e = min(b + chunk, (unsigned long long)n);
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_reduce_kernel(const uint32_t* __restrict__ in,
                                                                   const uint32_t* __restrict__ d_n,
                                                                   uint32_t* __restrict__ partials) {
    unsigned long long b, e;
    scan_range(*d_n, b, e);
    uint32_t s = 0;
    for (unsigned long long i = b + threadIdx.x; i < e; i += blockDim.x) s += in[i];
    uint32_t total;
    block_excl_scan(s, &total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_top_kernel(uint32_t* __restrict__ partials, uint32_t n,
                                                                uint32_t* __restrict__ total_out) {
    const uint32_t v = threadIdx.x < n ? partials[threadIdx.x] : 0u;
    uint32_t total;
    const uint32_t excl = block_excl_scan(v, &total);
    if (threadIdx.x < n) partials[threadIdx.x] = excl;
    if (threadIdx.x == 0 && total_out) *total_out = total;
}

__global__ void __launch_bounds__(SCAN_THREADS) scan_down_kernel(const uint32_t* in, const uint32_t* __restrict__ d_n,
                                                                 const uint32_t* __restrict__ partials,
                                                                 uint32_t* out) {
    unsigned long long b, e;
    scan_range(*d_n, b, e);
    uint32_t carry = partials[blockIdx.x];
    for (unsigned long long t = b; t < e; t += blockDim.x) {
        const unsigned long long i = t + threadIdx.x;
        const uint32_t v = i < e ? in[i] : 0u;
        uint32_t total;
        const uint32_t excl = block_excl_scan(v, &total);
        if (i < e) out[i] = carry + excl;
        carry += total;
    }
}

}  // namespace dev
}  // namespace frep

namespace {

using frep::dev::CompactHeader;
using frep::dev::SrcLevel;

// out[i] = in[0] + ... + in[i-1] for i < *d_n; *total_out = the sum.
cudaError_t scan_u32(const uint32_t* in, uint32_t* out, const uint32_t* d_n, uint32_t* partials, uint32_t* total_out,
                     cudaStream_t stream) {
    using namespace frep::dev;
    scan_reduce_kernel<<<SCAN_BLOCKS, SCAN_THREADS, 0, stream>>>(in, d_n, partials);
    scan_top_kernel<<<1, SCAN_THREADS, 0, stream>>>(partials, SCAN_BLOCKS, total_out);
    scan_down_kernel<<<SCAN_BLOCKS, SCAN_THREADS, 0, stream>>>(in, d_n, partials, out);
    return cudaGetLastError();
}

uint32_t warp_grid(uint64_t warps, int sm_count) {
    const uint64_t blocks = (warps + 7) / 8;  // 8 warps per 256-thread block
    return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)sm_count * 16));
}

void compact_geometry(frep_compact* c) {
    float cs = c->grid.world_size;
    for (uint32_t l = 0; l < c->grid.levels; l++) {  // voxelizer.cpp:209-216
        cs /= (float)c->grid.dims[l];
        c->cell_size[l] = cs;
        c->node_size[l] = frep::dev::compact_words(c->grid.dims[l], l == c->grid.levels - 1);
    }
}

// RAII for the temporary device buffers of one compaction.
struct DevBufs {
    std::vector<void*> ptrs;
    ~DevBufs() {
        for (void* p : ptrs) cudaFree(p);
    }
    // Hands a buffer over to the caller (no longer freed here).
    void* take(void* p) {
        ptrs.erase(std::remove(ptrs.begin(), ptrs.end(), p), ptrs.end());
        return p;
    }
    template <typename T>
    cudaError_t alloc(T** p, uint64_t count) {
        *p = nullptr;
        cudaError_t e = cudaMalloc((void**)p, std::max<uint64_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
};

// Carves 256-byte-aligned pieces from one block (base null: sizes only).
struct Carve {
    uint8_t* base = nullptr;
    uint64_t at = 0;
    template <typename T>
    T* take(uint64_t count) {
        T* p = reinterpret_cast<T*>(base + at);
        at += align_up(std::max<uint64_t>(count, 1) * sizeof(T), 256);
        return p;
    }
};

bool valid_dims(uint32_t levels, const uint32_t* dims) {
    if (levels == 0 || levels > FREP_MAX_LEVELS) return false;
    for (uint32_t l = 0; l < levels; l++)
        if (dims[l] < 4 || dims[l] > 32 || dims[l] % 4 != 0) return false;
    return true;
}

constexpr char kMagic[8] = {'F', 'R', 'E', 'P', 'C', 'T', '0', '1'};
static_assert(sizeof(frep_compact_header) == 120, "blob header layout");

uint64_t blob_nodes_at() { return align_up(sizeof(frep_compact_header), 8); }
uint64_t blob_tapes_at(uint64_t node_words) { return blob_nodes_at() + align_up(node_words * 4, 8); }

}  // namespace

extern "C" {

frep_status frep_tree_compact(frep_ctx* ctx, frep_tree* tree, uint32_t mode, void* stream_ptr, frep_compact** out) {
    if (!ctx || !tree || !out) return fail(FREP_ERR_INVALID_ARG, "frep_tree_compact: null argument");
    if (tree->ctx != ctx) return fail(FREP_ERR_INVALID_ARG, "frep_tree_compact: tree belongs to another context");
    if (mode > FREP_COMPACT_PRUNE) return fail(FREP_ERR_INVALID_ARG, "frep_tree_compact: mode must be 0 or 1");
    if (!tree->voxelized) return fail(FREP_ERR_INVALID_ARG, "frep_tree_compact: the tree has not been voxelized");
    frep_tree_info info;
    frep_status st = frep_tree_sync(tree, &info);  // waits for the voxelization; refuses overflowed pools
    if (st != FREP_OK) return st;
    cudaStream_t stream = (cudaStream_t)stream_ptr;
    const uint32_t L = tree->grid.levels;
    const int sms = ctx->sm_count;

    auto* c = new frep_compact();
    std::unique_ptr<frep_compact> guard(c);
    c->ctx = ctx;
    c->grid = tree->grid;
    c->mode = mode;
    c->n_slots = tree->n_slots;
    compact_geometry(c);

    uint64_t node_bound = 0, max_count = 0, sum_count = 0;
    SrcLevel S[FREP_MAX_LEVELS];
    for (uint32_t l = 0; l < L; l++) {
        S[l].nodes = tree->nodes + info.node_offset[l];
        S[l].size = tree->node_size[l];
        S[l].count = info.node_count[l];
        S[l].dim = tree->grid.dims[l];
        S[l].last = l == L - 1;
        node_bound += (uint64_t)info.node_count[l] * c->node_size[l];
        max_count = std::max<uint64_t>(max_count, info.node_count[l]);
        sum_count += info.node_count[l];
    }
    const uint64_t tape_top = info.tape_words_used;
    const uint32_t slots = (uint32_t)((tape_top + frep::dev::TAPE_ALIGN_WORDS - 1) / frep::dev::TAPE_ALIGN_WORDS);
    // Working buffers (the result's upper bounds, preorder, counts, statuses,
    // tape slots) plus room for an exactly sized copy of the result.
    const uint64_t scratch =
        2 * (node_bound * 4 + tape_top * 8) + max_count * 16 + sum_count + (uint64_t)slots * 8;
    if (ctx->used + scratch > ctx->budget)
        return fail(FREP_ERR_OOM, "frep_tree_compact: %llu bytes of working memory exceed the budget",
                    (unsigned long long)scratch);

    FREP_CUDA(cudaSetDevice(ctx->device));
    DevBufs tmp;
    uint32_t *dnodes, *order0, *order1, *cnt, *base, *mark, *newofs, *partials;
    uint64_t* dtapes;
    uint8_t* status;
    CompactHeader* H;
    // The result's two buffers (kept when already exact) and one block for
    // everything else: few allocations, few synchronizing frees.
    Carve cv;
    for (int pass = 0; pass < 2; pass++) {
        cv.at = 0;
        order0 = cv.take<uint32_t>(max_count);
        order1 = cv.take<uint32_t>(max_count);
        cnt = cv.take<uint32_t>(max_count);
        base = cv.take<uint32_t>(max_count);
        status = cv.take<uint8_t>(mode ? sum_count : 1);
        mark = cv.take<uint32_t>(slots);
        newofs = cv.take<uint32_t>(slots);
        partials = cv.take<uint32_t>(frep::dev::SCAN_BLOCKS);
        H = cv.take<CompactHeader>(1);
        if (pass == 0) {
            uint8_t* block = nullptr;
            cudaError_t be = tmp.alloc(&block, cv.at);
            if (be != cudaSuccess) {
                cudaGetLastError();
                return fail(FREP_ERR_OOM, "frep_tree_compact: cudaMalloc failed (%s)", cudaGetErrorString(be));
            }
            cv.base = block;
        }
    }
    cudaError_t e = tmp.alloc(&dnodes, node_bound);
    if (e == cudaSuccess) e = tmp.alloc(&dtapes, tape_top);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(FREP_ERR_OOM, "frep_tree_compact: cudaMalloc failed (%s)", cudaGetErrorString(e));
    }
    CompactHeader h0{};
    h0.count[0] = 1;
    h0.tape_slots = slots;
    FREP_CUDA(cudaMemcpyAsync(H, &h0, sizeof(h0), cudaMemcpyHostToDevice, stream));
    FREP_CUDA(cudaMemsetAsync(mark, 0, (size_t)std::max<uint32_t>(slots, 1) * 4, stream));

    // 1. BuildNode's statuses, last level first.
    uint8_t* st_of[FREP_MAX_LEVELS] = {};
    if (mode == FREP_COMPACT_PRUNE) {
        uint64_t at = 0;
        for (uint32_t l = 0; l < L; l++) {
            st_of[l] = status + at;
            at += info.node_count[l];
        }
        for (int l = (int)L - 1; l >= 0; l--) {
            if (!S[l].count) continue;
            frep::dev::compact_status_kernel<<<warp_grid(S[l].count, sms), 256, 0, stream>>>(
                S[l], l + 1 < (int)L ? st_of[l + 1] : nullptr, st_of[l]);
        }
        FREP_CUDA(cudaGetLastError());
    }
    // 2. Levels in preorder, root first.
    uint32_t* order_l = nullptr;  // level 0: the root alone
    uint32_t* order_next = order0;
    for (uint32_t l = 0; l < L; l++) {
        const uint32_t warps = std::max<uint32_t>(S[l].count, 1);
        frep::dev::compact_node_kernel<<<warp_grid(warps, sms), 256, 0, stream>>>(
            S[l], l, mode, l + 1 < L ? st_of[l + 1] : nullptr, order_l, H, dnodes, c->node_size[l], cnt, mark);
        FREP_CUDA(cudaGetLastError());
        if (l + 1 == L) break;
        e = scan_u32(cnt, base, &H->count[l], partials, &H->count[l + 1], stream);
        if (e != cudaSuccess) return cuda_fail(e, "compaction scan");
        frep::dev::compact_ofs_kernel<<<1, 1, 0, stream>>>(H, l, c->node_size[l]);
        frep::dev::compact_children_kernel<<<warp_grid(warps, sms), 256, 0, stream>>>(
            S[l], l, order_l, H, dnodes, c->node_size[l], base, order_next);
        FREP_CUDA(cudaGetLastError());
        order_l = order_next;
        order_next = order_next == order0 ? order1 : order0;
    }
    // 3. Tapes: sizes of the used records, new offsets, copies, remapped indices.
    const uint32_t tblocks = std::max<uint32_t>(1, std::min<uint32_t>((slots + 255) / 256, sms * 16));
    frep::dev::tape_size_kernel<<<tblocks, 256, 0, stream>>>(tree->tapes, mark, H);
    e = scan_u32(mark, newofs, &H->tape_slots, partials, &H->tape_words, stream);
    if (e != cudaSuccess) return cuda_fail(e, "compaction scan");
    frep::dev::tape_copy_kernel<<<warp_grid(slots, sms), 256, 0, stream>>>(tree->tapes, mark, newofs, H, dtapes);
    for (uint32_t l = 0; l < L; l++) {
        const uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>((S[l].count + 255) / 256, sms * 16));
        frep::dev::tape_remap_kernel<<<blocks, 256, 0, stream>>>(H, l, dnodes, c->node_size[l], newofs);
    }
    FREP_CUDA(cudaGetLastError());
    CompactHeader hh;
    FREP_CUDA(cudaMemcpyAsync(&hh, H, sizeof(hh), cudaMemcpyDeviceToHost, stream));
    FREP_CUDA(cudaStreamSynchronize(stream));

    for (uint32_t l = 0; l < L; l++) {
        c->node_count[l] = hh.count[l];
        c->node_ofs[l] = hh.ofs[l];
    }
    c->node_words = hh.ofs[L - 1] + (uint64_t)hh.count[L - 1] * c->node_size[L - 1];
    c->tape_words = hh.tape_words;
    if (c->node_words > node_bound || c->tape_words > tape_top)
        return fail(FREP_ERR_CUDA, "frep_tree_compact: inconsistent sizes (%llu > %llu node words)",
                    (unsigned long long)c->node_words, (unsigned long long)node_bound);
    // The result, sized exactly: a working buffer that is already exact is
    // kept, a larger one is copied into an exact one (and released on return).
    e = cudaSuccess;
    if (c->node_words == node_bound) c->nodes = (uint32_t*)tmp.take(dnodes);
    else e = cudaMalloc(&c->nodes, std::max<uint64_t>(c->node_words, 1) * 4);
    if (e == cudaSuccess) {
        if (c->tape_words == tape_top) c->tapes = (uint64_t*)tmp.take(dtapes);
        else e = cudaMalloc(&c->tapes, std::max<uint64_t>(c->tape_words, 1) * 8);
    }
    if (e == cudaSuccess && c->nodes != dnodes)
        e = cudaMemcpyAsync(c->nodes, dnodes, c->node_words * 4, cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess && c->tapes != dtapes)
        e = cudaMemcpyAsync(c->tapes, dtapes, c->tape_words * 8, cudaMemcpyDeviceToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(c->nodes);
        cudaFree(c->tapes);
        return fail(FREP_ERR_OOM, "frep_tree_compact: result allocation or copy failed (%s)", cudaGetErrorString(e));
    }
    c->bytes = c->node_words * 4 + c->tape_words * 8;
    ctx->used += c->bytes;
    *out = guard.release();
    return FREP_OK;
}

frep_status frep_compact_get_info(const frep_compact* c, frep_compact_info* info) {
    if (!c || !info) return fail(FREP_ERR_INVALID_ARG, "frep_compact_get_info: null argument");
    std::memset(info, 0, sizeof(*info));
    info->levels = c->grid.levels;
    info->mode = c->mode;
    info->n_slots = c->n_slots;
    for (uint32_t l = 0; l < c->grid.levels; l++) {
        info->dims[l] = c->grid.dims[l];
        info->node_count[l] = c->node_count[l];
        info->node_offset[l] = c->node_ofs[l];
        info->node_size[l] = c->node_size[l];
    }
    info->node_words = c->node_words;
    info->tape_words = c->tape_words;
    info->device_bytes = c->bytes;
    return FREP_OK;
}

void frep_compact_destroy(frep_compact* c) {
    if (!c) return;
    cudaSetDevice(c->ctx->device);
    cudaDeviceSynchronize();  // renders of it may still be in flight on any stream
    cudaFree(c->nodes);
    cudaFree(c->tapes);
    c->ctx->used -= std::min(c->ctx->used, c->bytes);
    delete c;
}

frep_status frep_render_compact(frep_ctx* ctx, const frep_compact* c, const frep_camera* cam,
                                const frep_lights* lights, float tape_time, const frep_image* out, void* stream_ptr) {
    if (!ctx || !c) return fail(FREP_ERR_INVALID_ARG, "frep_render_compact: null argument");
    if (c->ctx != ctx) return fail(FREP_ERR_INVALID_ARG, "frep_render_compact: tree belongs to another context");
    FREP_CUDA(cudaSetDevice(ctx->device));
    frep::RenderArgs a{};
    frep_status st = frep::detail::fill_view_args(cam, lights, tape_time, out, &a);
    if (st != FREP_OK) return st;
    a.compact = 1;
    a.hdr = nullptr;
    a.nodes = c->nodes;
    a.tapes = c->tapes;
    a.levels = c->grid.levels;
    for (uint32_t l = 0; l < a.levels; l++) {
        a.dims[l] = c->grid.dims[l];
        a.node_size[l] = c->node_size[l];
        a.cell_size[l] = c->cell_size[l];
        a.node_ofs[l] = c->node_ofs[l];
    }
    for (int k = 0; k < 3; k++) a.low[k] = c->grid.low_vertex[k];
    a.world_size = c->grid.world_size;
    a.n_slots = c->n_slots;
    cudaError_t e = frep::launch_render(a, (cudaStream_t)stream_ptr);
    if (e == cudaErrorInvalidValue) return fail(FREP_ERR_UNSUPPORTED, "frep_render_compact: more than 1024 slots");
    if (e != cudaSuccess) return cuda_fail(e, "render_kernel (compact)");
    return FREP_OK;
}

frep_status frep_compact_export(const frep_compact* c, void* dst, uint64_t cap, uint64_t* size) {
    if (!c || !size) return fail(FREP_ERR_INVALID_ARG, "frep_compact_export: null argument");
    const uint64_t total = blob_tapes_at(c->node_words) + c->tape_words * 8;
    *size = total;
    if (!dst) return FREP_OK;
    if (cap < total) return fail(FREP_ERR_INVALID_ARG, "frep_compact_export: %llu bytes needed, %llu given",
                                 (unsigned long long)total, (unsigned long long)cap);
    frep_compact_header h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kMagic, 8);
    h.version = 1;
    h.levels = c->grid.levels;
    for (uint32_t l = 0; l < c->grid.levels; l++) {
        h.dims[l] = c->grid.dims[l];
        h.node_count[l] = c->node_count[l];
    }
    for (int k = 0; k < 3; k++) h.low_vertex[k] = c->grid.low_vertex[k];
    h.world_size = c->grid.world_size;
    h.mode = c->mode;
    h.n_slots = c->n_slots;
    h.node_words = c->node_words;
    h.tape_words = c->tape_words;
    uint8_t* p = (uint8_t*)dst;
    std::memcpy(p, &h, sizeof(h));
    std::memset(p + sizeof(h), 0, blob_tapes_at(c->node_words) - sizeof(h));
    FREP_CUDA(cudaSetDevice(c->ctx->device));
    FREP_CUDA(cudaMemcpy(p + blob_nodes_at(), c->nodes, c->node_words * 4, cudaMemcpyDeviceToHost));
    FREP_CUDA(cudaMemcpy(p + blob_tapes_at(c->node_words), c->tapes, c->tape_words * 8, cudaMemcpyDeviceToHost));
    return FREP_OK;
}

frep_status frep_compact_check(const void* blob, uint64_t size) {
    if (!blob) return fail(FREP_ERR_INVALID_ARG, "compact blob: null pointer");
    if (size < sizeof(frep_compact_header)) return fail(FREP_ERR_INVALID_ARG, "compact blob: shorter than its header");
    frep_compact_header h;
    std::memcpy(&h, blob, sizeof(h));
    if (std::memcmp(h.magic, kMagic, 8) != 0) return fail(FREP_ERR_INVALID_ARG, "compact blob: bad magic");
    if (h.version != 1) return fail(FREP_ERR_INVALID_ARG, "compact blob: version %u (1 expected)", h.version);
    if (!valid_dims(h.levels, h.dims)) return fail(FREP_ERR_INVALID_ARG, "compact blob: bad levels or dims");
    for (uint32_t l = h.levels; l < FREP_MAX_LEVELS; l++)
        if (h.dims[l] || h.node_count[l]) return fail(FREP_ERR_INVALID_ARG, "compact blob: entries beyond the levels");
    if (h.mode > FREP_COMPACT_PRUNE) return fail(FREP_ERR_INVALID_ARG, "compact blob: mode %u", h.mode);
    if (h.n_slots < 4 || h.n_slots > 1024) return fail(FREP_ERR_INVALID_ARG, "compact blob: n_slots %u", h.n_slots);
    if (!std::isfinite(h.world_size) || !(h.world_size > 0.0f) || !std::isfinite(h.low_vertex[0]) ||
        !std::isfinite(h.low_vertex[1]) || !std::isfinite(h.low_vertex[2]))
        return fail(FREP_ERR_INVALID_ARG, "compact blob: bad grid placement");
    if (h.node_count[0] != 1) return fail(FREP_ERR_INVALID_ARG, "compact blob: %u root nodes", h.node_count[0]);
    uint64_t ofs[FREP_MAX_LEVELS], words = 0;
    uint32_t nsize[FREP_MAX_LEVELS];
    for (uint32_t l = 0; l < h.levels; l++) {
        nsize[l] = frep::dev::compact_words(h.dims[l], l + 1 == h.levels);
        ofs[l] = words;
        words += (uint64_t)h.node_count[l] * nsize[l];  // < 2^32 * 2^17: no overflow
    }
    if (words != h.node_words) return fail(FREP_ERR_INVALID_ARG, "compact blob: node_words does not match the counts");
    if (h.tape_words == 0 || h.tape_words > 0xFFFFFFF0ull)
        return fail(FREP_ERR_INVALID_ARG, "compact blob: tape_words %llu", (unsigned long long)h.tape_words);
    if (size != blob_tapes_at(h.node_words) + h.tape_words * 8)
        return fail(FREP_ERR_INVALID_ARG, "compact blob: %llu bytes, %llu expected", (unsigned long long)size,
                    (unsigned long long)(blob_tapes_at(h.node_words) + h.tape_words * 8));
    const uint8_t* p = (const uint8_t*)blob;
    const uint32_t* nodes = (const uint32_t*)(p + blob_nodes_at());
    const uint64_t* tapes = (const uint64_t*)(p + blob_tapes_at(h.node_words));
    std::vector<uint8_t> seen(h.tape_words, 0);  // 1: a record checked at this index
    for (uint32_t l = 0; l < h.levels; l++) {
        const uint32_t W = h.dims[l] * h.dims[l] * h.dims[l] / 32;
        const bool last = l + 1 == h.levels;
        uint64_t next_base = 0;
        for (uint32_t r = 0; r < h.node_count[l]; r++) {
            const uint32_t* d = nodes + ofs[l] + (uint64_t)r * nsize[l];
            const uint32_t t = d[0];
            if (t >= h.tape_words)
                return fail(FREP_ERR_INVALID_ARG, "compact blob: level %u node %u tape %u out of range", l, r, t);
            if (!seen[t]) {
                const uint64_t n = tapes[t] & 0xFFFFFFFFull;
                if (t + 1 + n > h.tape_words)
                    return fail(FREP_ERR_INVALID_ARG, "compact blob: level %u node %u tape record overruns the pool", l, r);
                for (uint64_t i = 0; i < n; i++) {
                    const uint64_t w = tapes[t + 1 + i];
                    const uint32_t op = (uint32_t)(w & 0xFF), o = (uint32_t)((w >> 16) & 0xFFFF),
                                   a = (uint32_t)((w >> 32) & 0xFFFF), b = (uint32_t)(w >> 48);
                    if (op > 12 || o >= h.n_slots || (op != 0 && (a >= h.n_slots || b >= h.n_slots)))
                        return fail(FREP_ERR_INVALID_ARG, "compact blob: tape at %u instruction %llu is invalid", t,
                                    (unsigned long long)i);
                }
                seen[t] = 1;
            }
            if (last) continue;
            uint32_t run = 0;
            for (uint32_t w = 0; w < W; w++) {
                const uint32_t leaf = d[1 + w], inter = d[1 + W + w];
                if (leaf & inter) return fail(FREP_ERR_INVALID_ARG, "compact blob: level %u node %u cell both leaf and interior", l, r);
                if (d[1 + 2 * W + w] != run)
                    return fail(FREP_ERR_INVALID_ARG, "compact blob: level %u node %u prefix word %u is wrong", l, r, w);
                run += (uint32_t)__builtin_popcount(inter);
            }
            if (d[1 + 3 * W] != next_base)
                return fail(FREP_ERR_INVALID_ARG, "compact blob: level %u node %u children not in preorder", l, r);
            next_base += run;
        }
        if (!last && next_base != h.node_count[l + 1])
            return fail(FREP_ERR_INVALID_ARG, "compact blob: level %u references %llu children, level %u has %u", l,
                        (unsigned long long)next_base, l + 1, h.node_count[l + 1]);
    }
    return FREP_OK;
}

frep_status frep_compact_import(frep_ctx* ctx, const void* blob, uint64_t size, frep_compact** out) {
    if (!ctx || !out) return fail(FREP_ERR_INVALID_ARG, "frep_compact_import: null argument");
    frep_status st = frep_compact_check(blob, size);
    if (st != FREP_OK) return st;
    frep_compact_header h;
    std::memcpy(&h, blob, sizeof(h));
    const uint64_t bytes = h.node_words * 4 + h.tape_words * 8;
    if (ctx->used + bytes > ctx->budget)
        return fail(FREP_ERR_OOM, "frep_compact_import: %llu bytes exceed the budget", (unsigned long long)bytes);
    FREP_CUDA(cudaSetDevice(ctx->device));
    auto* c = new frep_compact();
    c->ctx = ctx;
    c->grid.levels = h.levels;
    for (uint32_t l = 0; l < h.levels; l++) c->grid.dims[l] = h.dims[l];
    for (int k = 0; k < 3; k++) c->grid.low_vertex[k] = h.low_vertex[k];
    c->grid.world_size = h.world_size;
    c->mode = h.mode;
    c->n_slots = h.n_slots;
    compact_geometry(c);
    uint64_t ofs = 0;
    for (uint32_t l = 0; l < h.levels; l++) {
        c->node_count[l] = h.node_count[l];
        c->node_ofs[l] = ofs;
        ofs += (uint64_t)h.node_count[l] * c->node_size[l];
    }
    c->node_words = h.node_words;
    c->tape_words = h.tape_words;
    const uint8_t* p = (const uint8_t*)blob;
    cudaError_t e = cudaMalloc(&c->nodes, std::max<uint64_t>(h.node_words, 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc(&c->tapes, h.tape_words * 8);
    if (e == cudaSuccess) e = cudaMemcpy(c->nodes, p + blob_nodes_at(), h.node_words * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(c->tapes, p + blob_tapes_at(h.node_words), h.tape_words * 8, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        cudaGetLastError();
        cudaFree(c->nodes);
        cudaFree(c->tapes);
        delete c;
        return fail(FREP_ERR_OOM, "frep_compact_import: device upload failed (%s)", cudaGetErrorString(e));
    }
    c->bytes = bytes;
    ctx->used += bytes;
    *out = c;
    return FREP_OK;
}

}  // extern "C"
