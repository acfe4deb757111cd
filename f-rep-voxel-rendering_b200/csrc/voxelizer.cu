// Level passes of the sparse-tree voxelizer (sm_100a).
//
// Replaces vulkan/shaders/voxelizer/main.comp + tape/interval.comp +
// tape/shorten.comp + tape/point.comp and the host level loop of
// vulkan/src/engine/voxelizer.cpp:295-329, :429-440.
//
// Work decomposition: one WARP owns one work item = (node, a run of cells that
// forms whole words of the node's masks, in bit-index order z + dim*y + dim^2*x).
// All lanes follow the same tape, so the opcode stream is warp-uniform:
//   * the tape is staged through shared memory 128 instructions at a time, each
//     instruction decoded once into {op, row offset A, row offset B, row offset
//     out} (one coalesced load per chunk, the next chunk prefetched into
//     registers while the current one executes);
//   * the slot file lives in shared memory as rows of [slot][lane] values
//     (float2 intervals, or K floats per lane for the point pass);
//   * MIN/MAX choices are kept as two 32-bit lane masks per MIN/MAX instruction;
//   * shortening runs the reference's backward liveness on TRANSPOSED bitsets:
//     live[slot] holds one bit per lane, so the pass is warp-uniform scalar code;
//   * leaf / interior mask words are written whole from ballots (no atomics);
//   * children are claimed with one warp-aggregated atomic per item, tapes with
//     one more; shortened tapes are written by the whole warp, 32 instructions
//     per coalesced store.
// Items are fetched in chunks from a device counter, so a level pass needs no
// host round trip: the node count of level l is read on the device. One launch
// serves a whole batch of trees: a scan kernel lays the trees' items end to end
// and a warp resolves each item to its tree (binary search, cached per warp),
// so idle warps steal work from any scene of the batch.
#include "device_common.cuh"
#include "kernels.h"

namespace frep {
namespace dev {

constexpr uint32_t STAGE = 128;  // instructions staged per warp

// ---- shared-memory access by 32-bit address ----------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint4 lds_u4(uint32_t a) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0,%1,%2,%3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ float2 lds_f2(uint32_t a) {
    float2 v;
    asm volatile("ld.shared.v2.f32 {%0,%1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(a));
    return v;
}
__device__ __forceinline__ void sts_f2(uint32_t a, float2 v) {
    asm volatile("st.shared.v2.f32 [%0], {%1,%2};" ::"r"(a), "f"(v.x), "f"(v.y) : "memory");
}
__device__ __forceinline__ float4 lds_f4(uint32_t a) {
    float4 v;
    asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
    return v;
}
__device__ __forceinline__ void sts_f4(uint32_t a, float4 v) {
    asm volatile("st.shared.v4.f32 [%0], {%1,%2,%3,%4};" ::"r"(a), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w)
                 : "memory");
}

// Decoded instruction as staged for execution (16 bytes):
//   x: opcode (bits 0-3) | F_FWD_A | F_FWD_B (point passes only)
//   y: byte offset of the A slot row (CONST: the constant's bits)
//   z: byte offset of the B slot row (slot 0 for unary opcodes)
//   w: byte offset of the output slot row
// A row holds 32 lanes x row_bytes. F_FWD_A / F_FWD_B: the operand is the
// previous instruction's output, so the point interpreter takes it from the
// register holding that result instead of loading the slot row.
constexpr uint32_t F_FWD_A = 1u << 4, F_FWD_B = 1u << 5;

__device__ __forceinline__ uint4 decode(uint64_t w, uint32_t prev_out, uint32_t row_bytes) {
    const uint32_t op = w_op(w);
    const uint32_t stride = 32u * row_bytes;
    if (op == OP_CONST) return make_uint4(op, (uint32_t)(w >> 32), 0u, w_out(w) * stride);
    const bool bin = is_binary(op);
    const uint32_t fa = w_a(w) == prev_out ? F_FWD_A : 0u;
    const uint32_t fb = bin && w_b(w) == prev_out ? F_FWD_B : 0u;
    return make_uint4(op | fa | fb, w_a(w) * stride, bin ? w_b(w) * stride : 0u, w_out(w) * stride);
}

// Dispatch of the interval interpreter: opcodes are tested in the order of
// their frequency in CSG tapes (CONST ~26 %, SUB ~25 %, MUL ~25 %, ADD ~11 %,
// MIN/MAX ~10 %, the rest ~2 %), so a typical instruction costs two or three
// uniform compare-and-branch pairs; the rare opcodes share one switch. (This
// measured ~20 % faster than one switch case per opcode and forwarding
// combination; the point interpreter keeps that switch, below.)

// Fetches the next chunk of work items for this warp. Returns the first item
// of the chunk in *first and its size; 0 when the level is exhausted.
__device__ __forceinline__ uint32_t fetch_items(unsigned long long* cursor, unsigned long long total,
                                                uint32_t chunk, unsigned long long* first) {
    unsigned long long f = 0;
    if ((threadIdx.x & 31) == 0) f = atomicAdd(cursor, (unsigned long long)chunk);
    f = __shfl_sync(0xFFFFFFFFu, f, 0);
    *first = f;
    if (f >= total) return 0;
    return (uint32_t)min((unsigned long long)chunk, total - f);
}

// Chunk size: enough items per fetch to keep counter traffic low, few enough
// that every warp gets work.
__device__ __forceinline__ uint32_t chunk_for(unsigned long long total, uint32_t grid_warps) {
    unsigned long long c = total / ((unsigned long long)grid_warps * 8ull);
    return (uint32_t)max(1ull, min(c, 32ull));
}

// Largest tree index i with prefix[i] <= item (prefix[0] = 0 <= item < prefix[n]).
__device__ __forceinline__ uint32_t find_tree(const unsigned long long* prefix, uint32_t n, unsigned long long item) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldcg(&prefix[mid]) <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

__host__ __device__ inline int point_k_of(uint32_t dim) { return (dim * dim * dim / 32) % 4 == 0 ? 4 : 2; }

// log2(dim) for a power-of-two node dim, else NOT_POW2: lets the per-item
// and per-cell index arithmetic use shifts instead of integer division for
// dims 4, 8, 16 and 32 (the usual ones).
constexpr uint32_t NOT_POW2 = 0xFFu;
__device__ __forceinline__ uint32_t dim_shift(uint32_t dim) {
    return (dim & (dim - 1)) == 0 ? (uint32_t)(__ffs(dim) - 1) : NOT_POW2;
}

// Node and mask-word group of a work item: `local` counts the tree's items of
// this pass, `groups` items per node (dim^3 / 32 / cells-per-lane, a power of
// two exactly when dim is, with gsh its log2).
__device__ __forceinline__ void split_item(unsigned long long local, uint32_t groups, uint32_t gsh, uint32_t* node,
                                           uint32_t* grp) {
    if (gsh != NOT_POW2) {
        *grp = (uint32_t)local & (groups - 1);
        *node = (uint32_t)(local >> gsh);
    } else if (local < (1ull << 32)) {
        const uint32_t l = (uint32_t)local;
        *grp = l % groups;
        *node = l / groups;
    } else {
        *grp = (uint32_t)(local % groups);
        *node = (uint32_t)(local / groups);
    }
}

// Cell coordinates inside a node from the bit index z + dim*y + dim^2*x
// (utils.comp:6).
__device__ __forceinline__ void cell_xyz(uint32_t cell, uint32_t dim, uint32_t sh, uint32_t* cx, uint32_t* cy,
                                         uint32_t* cz) {
    if (sh != NOT_POW2) {
        *cz = cell & (dim - 1);
        *cy = (cell >> sh) & (dim - 1);
        *cx = cell >> (2 * sh);
    } else {
        *cz = cell % dim;
        *cy = (cell / dim) % dim;
        *cx = cell / (dim * dim);
    }
}

// Work items of the interval passes are bricks: KI = 2 cells per lane take a
// 4x4x4 brick of the node, KI = 1 a 2x4x4 one (x extent XS = 2 * KI), bricks
// numbered z fastest. Lane l's h-th cell is brick cell i = 32h + l with
// z = i & 3, y = (i >> 2) & 3, x = i >> 4: each 32-cell group is eight rows
// of four cells along z (lanes 4r .. 4r + 3), and a row's four bits lie in
// one mask word (dim is a multiple of 4, so a row starts on a 4-bit
// boundary). A compact brick keeps the intervals of the item-level prepass
// narrow, where a run of whole mask words would be a rod through the node.
template <int KI>
__device__ __forceinline__ void brick_origin(uint32_t grp, uint32_t dim, uint32_t sh, uint32_t* bx, uint32_t* by,
                                             uint32_t* bz) {
    constexpr uint32_t XS = 2 * KI;
    if (sh != NOT_POW2) {
        const uint32_t bs = sh - 2;  // log2(bricks along y and z)
        *bz = (grp & ((1u << bs) - 1u)) * 4u;
        *by = ((grp >> bs) & ((1u << bs) - 1u)) * 4u;
        *bx = (grp >> (2 * bs)) * XS;
    } else {
        const uint32_t nb = dim / 4u;
        *bz = grp % nb * 4u;
        *by = grp / nb % nb * 4u;
        *bx = grp / (nb * nb) * XS;
    }
}
template <int KI>
__device__ __forceinline__ uint32_t brick_cell(uint32_t bx, uint32_t by, uint32_t bz, uint32_t i, uint32_t dim,
                                               uint32_t* cx, uint32_t* cy, uint32_t* cz) {
    *cx = bx + (i >> 4);
    *cy = by + ((i >> 2) & 3u);
    *cz = bz + (i & 3u);
    return (*cx * dim + *cy) * dim + *cz;
}

// ORs a 32-cell brick group's leaf and interior ballots into the node's mask
// words: the first lane of each row of four issues one atomic per mask with
// the row's four bits. The node's mask words start at zero (written when the
// node was created).
__device__ __forceinline__ void or_group_masks(uint32_t* leaf_words, uint32_t* interior_words, uint32_t cell,
                                               uint32_t leaf_w, uint32_t interior_w, uint32_t lane) {
    if ((lane & 3u) == 0u) {
        const uint32_t w = cell >> 5, s = cell & 31u;
        const uint32_t lf = (leaf_w >> lane) & 0xFu, in = (interior_w >> lane) & 0xFu;
        if (lf) atomicOr(&leaf_words[w], lf << s);
        if (in) atomicOr(&interior_words[w], in << s);
    }
}

// What a level pass needs of one tree, read from its header when a warp
// moves on to that tree.
struct LevelTree {
    TreeHeader* H;
    uint32_t* nodes;
    uint64_t* tapes;
    unsigned long long tape_cap, ofs_l, ofs_next, child_cap;
    uint32_t dim, dim_sh, node_size, node_size_next, shorten, share;
    uint32_t next_mask_words;  // mask words a new child needs zeroed (its level is an interval level), else 0
    float cs, lx, ly, lz, tt;
};

__device__ __forceinline__ LevelTree load_tree(TreeHeader* H, uint32_t L, bool point) {
    LevelTree t;
    t.H = H;
    t.nodes = H->nodes;
    t.tapes = H->tapes;
    t.tape_cap = H->tape_cap;
    t.dim = H->dims[L];
    t.dim_sh = dim_shift(t.dim);
    t.node_size = H->node_size[L];
    t.ofs_l = H->node_ofs[L];
    t.shorten = H->shorten;
    t.share = H->share_tapes;
    t.cs = H->cell_size[L];
    t.lx = H->low[0];
    t.ly = H->low[1];
    t.lz = H->low[2];
    t.tt = H->tape_time;
    if (!point) {
        t.node_size_next = H->node_size[L + 1];
        t.ofs_next = H->node_ofs[L + 1];  // written by the scan kernel
        const unsigned long long cap = H->node_cap;
        t.child_cap = cap > t.ofs_next ? (cap - t.ofs_next) / t.node_size_next : 0ull;
        const uint32_t dn = H->dims[L + 1];
        t.next_mask_words = L + 2 < H->levels ? dn * dn * dn / 16u : 0u;
    } else {
        t.node_size_next = 1;
        t.ofs_next = 0;
        t.child_cap = 0;
        t.next_mask_words = 0;
    }
    return t;
}

// Stages the prefetched chunk `pre` (lane l of group q holds instruction
// q*32 + l of the chunk), decoded, into stage[]: only the 32-entry groups that
// hold the chunk's m instructions (short leaf tapes need one or two). FWD:
// mark operands forwarded from the previous instruction (never for the first
// instruction of a chunk). Entries past the tape's end decode to a CONST that
// is never executed; the interpreter reads one entry past the last one (not
// executing it), which may be left from an earlier tape or be stage[STAGE].
template <bool FWD>
__device__ __forceinline__ void stage_chunk(uint4* stage, const uint64_t (&pre)[STAGE / 32], uint32_t row_bytes,
                                            uint32_t lane, uint32_t m) {
    uint32_t prev_group_last = 0xFFFFFFFFu;
#pragma unroll
    for (int q = 0; q < (int)(STAGE / 32); q++) {
        if ((uint32_t)q * 32u >= m) break;
        uint32_t prev = 0xFFFFFFFFu;
        if constexpr (FWD) {
            const uint32_t out = w_out(pre[q]);
            prev = __shfl_up_sync(0xFFFFFFFFu, out, 1);
            if (lane == 0) prev = prev_group_last;
            prev_group_last = __shfl_sync(0xFFFFFFFFu, out, 31);
        }
        stage[q * 32 + lane] = decode(pre[q], prev, row_bytes);
    }
}
__device__ __forceinline__ void prefetch_chunk(uint64_t (&pre)[STAGE / 32], const uint64_t* tape, uint32_t base,
                                               uint32_t n, uint32_t lane) {
#pragma unroll
    for (int q = 0; q < (int)(STAGE / 32); q++) {
        const uint32_t i = base + q * 32 + lane;
        pre[q] = i < n ? __ldcg(&tape[i]) : 0ull;
    }
}

// KI intervals per lane (one per cell): slot rows of 8 * KI bytes per lane.
template <int KI>
struct IVK {
    float2 v[KI];
};
template <int KI>
__device__ __forceinline__ IVK<KI> lds_iv(uint32_t a) {
    IVK<KI> r;
    if constexpr (KI == 1) {
        r.v[0] = lds_f2(a);
    } else {
        const float4 t = lds_f4(a);
        r.v[0] = make_float2(t.x, t.y);
        r.v[1] = make_float2(t.z, t.w);
    }
    return r;
}
template <int KI>
__device__ __forceinline__ void sts_iv(uint32_t a, const IVK<KI>& r) {
    if constexpr (KI == 1) sts_f2(a, r.v[0]);
    else sts_f4(a, make_float4(r.v[0].x, r.v[0].y, r.v[1].x, r.v[1].y));
}

// One interval instruction (any opcode but CONST) on KI cells per lane,
// dispatched by frequency. MIN/MAX also record each cell's choice
// (interval.comp:140-155) as two ballots per group of 32 cells: bit 0 = the
// first operand may be the result, bit 1 = the second.
template <int ROUND, int KI>
__device__ __forceinline__ IVK<KI> iv_exec(const uint4 d, uint32_t lane_base, uint32_t lane, uint2* mmb,
                                           uint32_t& mm, uint32_t mm_cap) {
    const uint32_t op = d.x;
    const IVK<KI> a = lds_iv<KI>(lane_base + d.y);
    const IVK<KI> b = lds_iv<KI>(lane_base + d.z);
    IVK<KI> r;
    if (op == OP_SUB) {
#pragma unroll
        for (int h = 0; h < KI; h++)
            r.v[h] = ROUND ? make_float2(__fsub_rd(a.v[h].x, b.v[h].y), __fsub_ru(a.v[h].y, b.v[h].x))
                           : make_float2(__fsub_rn(a.v[h].x, b.v[h].y), __fsub_rn(a.v[h].y, b.v[h].x));
        return r;
    }
    if (op == OP_MUL) {
#pragma unroll
        for (int h = 0; h < KI; h++) r.v[h] = iv_mul<ROUND>(a.v[h], b.v[h]);
        return r;
    }
    if (op == OP_ADD) {
#pragma unroll
        for (int h = 0; h < KI; h++)
            r.v[h] = ROUND ? make_float2(__fadd_rd(a.v[h].x, b.v[h].x), __fadd_ru(a.v[h].y, b.v[h].y))
                           : make_float2(__fadd_rn(a.v[h].x, b.v[h].x), __fadd_rn(a.v[h].y, b.v[h].y));
        return r;
    }
    if (op == OP_MIN || op == OP_MAX) {
        const bool mx = op == OP_MAX;
        uint2 ch[KI];
#pragma unroll
        for (int h = 0; h < KI; h++) {
            const bool first_low = a.v[h].y < b.v[h].x, second_low = b.v[h].y < a.v[h].x;
            const uint32_t c =
                first_low ? (mx ? MM_SECOND : MM_FIRST) : (second_low ? (mx ? MM_FIRST : MM_SECOND) : MM_BOTH);
            ch[h] = make_uint2(__ballot_sync(0xFFFFFFFFu, c & 1u), __ballot_sync(0xFFFFFFFFu, c & 2u));
            r.v[h] = mx ? make_float2(max_sel(a.v[h].x, b.v[h].x), max_sel(a.v[h].y, b.v[h].y))
                        : make_float2(min_sel(a.v[h].x, b.v[h].x), min_sel(a.v[h].y, b.v[h].y));
        }
        if (lane == 0 && mm < mm_cap) {
            if constexpr (KI == 1) mmb[mm] = ch[0];
            else reinterpret_cast<uint4*>(mmb)[mm] = make_uint4(ch[0].x, ch[0].y, ch[1].x, ch[1].y);
        }
        mm++;
        return r;
    }
#pragma unroll
    for (int h = 0; h < KI; h++) r.v[h] = iv_apply<ROUND>(op, 0ull, a.v[h], b.v[h]);
    return r;
}

// 32 x 32 bit-matrix transpose across a warp: lane j holds row j (bit c =
// entry (j, c)); lane c gets column c (bit j = entry (j, c)). Five butterfly
// steps, each swapping the off-diagonal s-blocks with lane ^ s.
__device__ __forceinline__ uint32_t transpose32(uint32_t x, uint32_t lane) {
    const uint32_t masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int i = 0; i < 5; i++) {
        const uint32_t sh = 16u >> i, m = masks[i];
        const uint32_t t = __shfl_xor_sync(0xFFFFFFFFu, x, sh);
        x = (lane & sh) ? ((x & ~m) | ((t & ~m) >> sh)) : ((x & m) | ((t & m) << sh));
    }
    return x;
}

// Backward liveness walk of one item's cells over a tape of at most 32 * S
// slots (shorten.comp:148-186). The live sets are kept transposed and spread
// over the lanes: lane l holds, per cell group h (32 cells) and q < S, the
// 32-bit mask of the group's cells for which slot 32 q + l is live. From the
// last instruction down, an instruction's keep mask is the mask of its output
// slot (one shuffle, the same in every lane); the output then dies and the
// inputs its choice uses (both for arithmetic, the chosen ones for MIN/MAX,
// none for CONST) become live for the cells that kept it: three predicated
// lane updates, whatever the number of cells.
//
// Per 32-instruction chunk the keep masks go to keep[]; each cell's kept
// count and grouping signature (kept positions and MIN/MAX rewrites) come
// from the chunk's masks transposed to one word per cell.
//
// A chunk is walked in one of two ways, chosen from how many of the previous
// chunk's instructions were live somewhere (the top chunk as if all were):
// below half, each step jumps (one ballot) straight to the next instruction
// whose output is live in some cell; otherwise every instruction is visited.
// Long tapes of which each cell keeps a few percent (the root level) skip
// most instructions.
template <int KI, int S>
__device__ __forceinline__ void walk_lanes(const uint64_t* tape, uint32_t n, int mm, const uint2* mmb,
                                           uint32_t* keep, const uint32_t (&ok_w)[KI], uint32_t lane,
                                           uint32_t (&kept)[KI], uint32_t (&sig)[KI]) {
    uint32_t lv[S][KI];
#pragma unroll
    for (int q = 0; q < S; q++)
#pragma unroll
        for (int h = 0; h < KI; h++) lv[q][h] = (q == 0 && lane == 0) ? ok_w[h] : 0u;  // slot 0: the result
    bool plain = true;  // (the top chunk: mostly live)
    int mm_top = mm;    // MIN/MAX instructions before the current chunk's end
    for (int hi = (int)n; hi > 0; hi -= 32) {
        const int lo = max(0, hi - 32);
        const int m = hi - lo;
        // lane j holds instruction lo + j (packed: out | a << 6 | b << 12 | op
        // << 18) and, for a MIN/MAX, its choices
        const uint64_t mine = (int)lane < m ? __ldcg(&tape[lo + lane]) : 0ull;
        const uint32_t pk = (w_out(mine) & 63u) | (w_a(mine) & 63u) << 6 | (w_b(mine) & 63u) << 12 |
                            w_op(mine) << 18;
        const bool ism = (int)lane < m && is_mm(w_op(mine));
        const uint32_t mball = __ballot_sync(0xFFFFFFFFu, ism);
        const int mbase = mm_top - __popc(mball);
        uint2 cb[KI];
#pragma unroll
        for (int h = 0; h < KI; h++)
            cb[h] = ism ? mmb[(mbase + __popc(mball & lanemask_lt())) * KI + h] : make_uint2(0u, 0u);
        uint32_t my_keep[KI], my_f[KI], my_s[KI];  // this lane's instruction: keep / chosen-input masks
#pragma unroll
        for (int h = 0; h < KI; h++) my_keep[h] = my_f[h] = my_s[h] = 0u;
        int live = 0;  // instructions of this chunk live in some cell
        int j = m - 1;
        while (j >= 0) {
            if (!plain) {
                uint32_t u0 = 0, u1 = 0;
#pragma unroll
                for (int h = 0; h < KI; h++) {
                    u0 |= lv[0][h];
                    if constexpr (S == 2) u1 |= lv[S - 1][h];
                }
                const uint64_t U = (uint64_t)__ballot_sync(0xFFFFFFFFu, u0 != 0u) |
                                   (S == 2 ? (uint64_t)__ballot_sync(0xFFFFFFFFu, u1 != 0u) << 32 : 0ull);
                const uint32_t cand = __ballot_sync(0xFFFFFFFFu, (int)lane <= j && ((U >> (pk & 63u)) & 1ull));
                if (!cand) break;
                j = 31 - __clz(cand);
            }
            const uint32_t q = __shfl_sync(0xFFFFFFFFu, pk, j);
            const uint32_t o = q & 63u, a = (q >> 6) & 63u, b = (q >> 12) & 63u, op = q >> 18;
            uint32_t k[KI], anyk = 0;
#pragma unroll
            for (int h = 0; h < KI; h++) {
                const uint32_t src = (S == 2 && o >= 32u) ? lv[S - 1][h] : lv[0][h];
                k[h] = __shfl_sync(0xFFFFFFFFu, src, o & 31u);
                anyk |= k[h];
            }
            if (anyk) {
                const bool arith = op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_DIV;
                const bool mmop = is_mm(op);
                const bool at_o = lane == (o & 31u), at_a = lane == (a & 31u), at_b = lane == (b & 31u);
                live++;
#pragma unroll
                for (int h = 0; h < KI; h++) {
                    uint32_t f, sc;
                    if (mmop) {
                        f = __shfl_sync(0xFFFFFFFFu, cb[h].x, j);
                        sc = __shfl_sync(0xFFFFFFFFu, cb[h].y, j);
                    } else {
                        f = op != OP_CONST ? ~0u : 0u;
                        sc = arith ? ~0u : 0u;
                    }
                    f &= k[h];
                    sc &= k[h];
                    // clear the output slot, then set the inputs the choice uses
                    if (at_o) {
                        if (S == 1 || o < 32u) lv[0][h] = 0u;
                        else lv[S - 1][h] = 0u;
                    }
                    if (at_a) {
                        if (S == 1 || a < 32u) lv[0][h] |= f;
                        else lv[S - 1][h] |= f;
                    }
                    if (at_b) {
                        if (S == 1 || b < 32u) lv[0][h] |= sc;
                        else lv[S - 1][h] |= sc;
                    }
                    if ((int)lane == j) {
                        my_keep[h] = k[h];
                        if (mmop) {
                            my_f[h] = f;
                            my_s[h] = sc;
                        }
                    }
                }
            }
            j--;
        }
        plain = 2 * live >= m;  // the next chunk's mode, from this one's liveness
        if ((int)lane < m) {
            if constexpr (KI == 1) keep[lo + lane] = my_keep[0];
            else reinterpret_cast<uint2*>(keep)[lo + lane] = make_uint2(my_keep[0], my_keep[1]);
        }
        // per cell: the chunk's kept instructions and MIN/MAX rewrites
#pragma unroll
        for (int h = 0; h < KI; h++) {
            if (!__any_sync(0xFFFFFFFFu, my_keep[h] != 0u)) continue;
            const uint32_t kc = transpose32(my_keep[h], lane);
            kept[h] += __popc(kc);
            uint32_t fc = 0, sc = 0;
            if (__any_sync(0xFFFFFFFFu, (my_f[h] | my_s[h]) != 0u)) {
                fc = transpose32(my_f[h], lane);
                sc = transpose32(my_s[h], lane);
            }
            sig[h] = sig[h] * 0x9E3779B1u + (kc ^ (uint32_t)lo) * 0x85EBCA6Bu + fc * 0xC2B2AE35u + sc * 0x27D4EB2Fu;
        }
        mm_top = mbase;
    }
}

// The forward loop's common opcodes as inline PTX with a jump table.
#include "interval_dispatch.cuh"

// ---- item-level pruning (this library's addition) ----------------------------------
//
// Before the cells of a work item are evaluated, the node's tape is evaluated
// once over the item's bounding box and shortened there, like a cell's tape;
// the cells then run that shorter tape. This is exact: for algebraic tapes
// (no SIN/COS/EXP, whose rounding is not monotone) whose every interval over
// the item box is finite, each formula of interval.comp:8-111 is monotone in
// its operands' bounds in both roundings, so every cell's interval lies inside
// the item's; a MIN/MAX decided over the item box is decided the same way in
// every cell and an instruction dead for the item is dead for every cell. A
// cell's child tape, the node tape shortened by the cell's choices, is then
// the item tape shortened by the same choices, word for word. An item box
// that is empty (low > 0) or inside (high < 0) makes every cell of the item
// empty or a leaf without evaluating them.
//
// Up to 32 consecutive items of one node are prepared together, one per lane
// (the same forward pass and backward walk as cells, one box per lane, in the
// first 256 bytes of each slot row: lane_base = row base + 8 * lane); each
// item's tape goes to the warp's item scratch, on a 16-word boundary, while
// it fits. Returns per lane (one item) a packed plan: bits 0-1 the mode, 0 =
// run the node's tape, 1 = run the item tape, 2 = every cell empty, 3 = every
// cell a leaf; bits 2-16 the item tape's offset in the scratch / 16, bits
// 17-31 its length (item tapes of 2^15 words or more are not stored; the
// scratch holds at most kItemTapeWords <= 2^19 words).
struct ItemNode {  // the node of a group of items, and its tree's frame
    uint32_t dim, dim_sh, ncx, ncy, ncz;
    float cs, lx, ly, lz, tt;
};
template <int ROUND, int KI>
__device__ __noinline__ uint32_t prepare_items(const uint64_t* tape, uint32_t n, const ItemNode T, uint32_t grp,
                                               uint32_t g, uint32_t lane_base, uint4* stage, uint32_t* keep,
                                               uint2* mmb, uint64_t* items, uint32_t mm_cap, uint32_t n_slots,
                                               uint32_t item_cap) {
    constexpr uint32_t ROWB = 8 * KI;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t dim = T.dim, ncx = T.ncx, ncy = T.ncy, ncz = T.ncz;
    const bool valid = lane < g;
    // the item is a brick (brick_origin): its cells' bounding box
    uint32_t x0, y0, z0;
    brick_origin<KI>(grp + (valid ? lane : 0u), dim, T.dim_sh, &x0, &y0, &z0);
    const uint32_t x1 = x0 + 2u * KI - 1u, y1 = y0 + 3u, z1 = z0 + 3u;
    // the cells' own box formula (voxelizer/main.comp:113-126), so the item box
    // contains each of them exactly
    const float cs = T.cs;
    const uint32_t glo[3] = {ncx * dim + x0, ncy * dim + y0, ncz * dim + z0};
    const uint32_t ghi[3] = {ncx * dim + x1, ncy * dim + y1, ncz * dim + z1};
    const float low[3] = {T.lx, T.ly, T.lz};
#pragma unroll
    for (int k = 0; k < 3; k++) {
        IVK<1> b;
        b.v[0] = make_float2(__fadd_rn(low[k], __fmul_rn((float)glo[k], cs)),
                             __fadd_rn(__fadd_rn(low[k], __fmul_rn((float)ghi[k], cs)), cs));
        sts_iv<1>(lane_base + k * 32 * ROWB, b);
    }
    {
        IVK<1> b;
        b.v[0] = make_float2(T.tt, T.tt);
        sts_iv<1>(lane_base + 3 * 32 * ROWB, b);
    }
    uint32_t mm = 0;
    bool fin = true, trans = false;
    IVK<1> r;
    uint64_t pre[STAGE / 32];
    prefetch_chunk(pre, tape, 0, n, lane);
    for (uint32_t base = 0; base < n; base += STAGE) {
        const uint32_t m = min(STAGE, n - base);
        __syncwarp();
        stage_chunk<false>(stage, pre, ROWB, lane, m);
        prefetch_chunk(pre, tape, base + STAGE, n, lane);
        __syncwarp();
        const uint32_t sbase = smem_addr(stage);
        for (uint32_t j = 0; j < m; j++) {
            const uint4 d = lds_u4(sbase + j * 16);
            if (d.x == OP_CONST) {
                const float c = __uint_as_float(d.y);
                r.v[0] = make_float2(c, c);
            } else {
                trans |= d.x == OP_SIN || d.x == OP_COS || d.x == OP_EXP;
                r = iv_exec<ROUND, 1>(d, lane_base, lane, mmb, mm, mm_cap);
            }
            fin &= fabsf(r.v[0].x) <= 3.40282347e38f && fabsf(r.v[0].y) <= 3.40282347e38f;
            sts_iv<1>(lane_base + d.w, r);
        }
    }
    __syncwarp();
    if (trans || mm > mm_cap) return 0u;  // the whole group runs the node's tape
    const IVK<1> res = lds_iv<1>(lane_base);
    const bool empty = res.v[0].x > 0.0f, full = !empty && res.v[0].y < 0.0f;
    uint32_t plan = 0;
    if (valid && fin && empty) plan = 2;
    if (valid && fin && full) plan = 3;
    const uint32_t cand = __ballot_sync(0xFFFFFFFFu, valid && fin && !empty && !full);
    if (!cand || n_slots > 64) return plan;
    uint32_t ok_w[1] = {cand}, kept[1] = {0}, sig[1] = {0};
    if (n_slots <= 32) walk_lanes<1, 1>(tape, n, (int)mm, mmb, keep, ok_w, lane, kept, sig);
    else walk_lanes<1, 2>(tape, n, (int)mm, mmb, keep, ok_w, lane, kept, sig);
    __syncwarp();
    // the items whose tape is shorter, in lane order, while the scratch holds them
    const bool want = ((cand >> lane) & 1u) && kept[0] < n && kept[0] < 32768u;
    const uint32_t mine = want ? (kept[0] + 15u) & ~15u : 0u;
    uint32_t incl = mine;
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if ((int)lane >= o) incl += v;
    }
    const bool fits = want && incl <= item_cap;
    const uint32_t wmask = __ballot_sync(0xFFFFFFFFu, fits);
    const uint32_t my_off = incl - mine;
    if (fits) plan = 1u | (my_off >> 4) << 2 | kept[0] << 17;
    if (!wmask) return plan;
    // copy: chunk-outer, one ballot + one coalesced store per item tape that
    // keeps some instruction of the chunk; a MIN/MAX decided for the item
    // becomes a COPY of the chosen operand (shorten.comp:148-186)
    uint32_t run = 0, mm_run = 0;
    for (uint32_t b = 0; b < n; b += 32) {
        const uint32_t idx = b + lane;
        const bool v = idx < n;
        const uint64_t w = v ? __ldcg(&tape[idx]) : 0ull;
        const uint32_t km = v ? keep[idx] : 0u;
        const bool ism = v && is_mm(w_op(w));
        const uint32_t mball = __ballot_sync(0xFFFFFFFFu, ism);
        const uint2 cb = ism ? mmb[mm_run + __popc(mball & lanemask_lt())] : make_uint2(0u, 0u);
        uint32_t pending = wmask & __reduce_or_sync(0xFFFFFFFFu, km);
        while (pending) {
            const int sel = __ffs(pending) - 1;
            pending &= pending - 1;
            const bool kb = (km >> sel) & 1u;
            uint64_t wo = w;
            if (kb && ism) {
                const uint32_t c = ((cb.x >> sel) & 1u) | (((cb.y >> sel) & 1u) << 1);
                if (c == MM_FIRST) wo = (w & ~0xFFull) | OP_COPY;
                else if (c == MM_SECOND) wo = (w & ~0xFFull & ~(0xFFFFull << 32)) | OP_COPY | ((uint64_t)w_b(w) << 32);
            }
            const uint32_t kball = __ballot_sync(0xFFFFFFFFu, kb);
            const uint32_t dst = __shfl_sync(0xFFFFFFFFu, my_off, sel);
            const uint32_t rr = __shfl_sync(0xFFFFFFFFu, run, sel);
            if (kb) items[dst + rr + __popc(kball & lanemask_lt())] = wo;
            if ((int)lane == sel) run += __popc(kball);
        }
        mm_run += __popc(mball);
    }
    __syncwarp();
    return plan;
}

// ---- interval level pass -------------------------------------------------------
//
// A work item is KI whole mask words of a node (32 * KI cells); lane l
// evaluates cells grp*32*KI + h*32 + l, h < KI, so one decoded instruction
// drives 32 * KI interval evaluations and the backward liveness walk covers
// 32 * KI cells per step.
//
// Per-warp shared memory: slots [n_slots][32 lanes][KI] float2 | stage
// [STAGE] uint4 | live [n_slots][KI] u32. Per-warp global scratch: keep masks
// (KI words per instruction) | choice masks (KI uint2 per MIN/MAX): they grow
// with the tape, and in shared memory they would cap the resident warps for
// every tree of a batch at what its longest tape allows.
template <int ROUND, int WARPS, int KI>
// At least 16 warps per SM (4 blocks of 4 or 16 of 1): up to 128 registers.
// Shared memory already limits a batch's plan to about 16 resident warps, and
// a cap of 96 registers spills inside the forward pass: on a 128-scene batch
// the level-1 pass measured 35.0 ms with the cap and 26.7 ms without.
__global__ void __launch_bounds__(WARPS * 32, WARPS == 4 ? 4 : 16)
interval_level_kernel(LevelLaunch p) {
    extern __shared__ __align__(16) unsigned char smem[];
    static_assert(ROUND != 2 || KI == 1, "the hybrid affine mode runs one cell per lane");
    // bytes per lane per slot: KI intervals; the hybrid mode's 8 floats (lo, hi,
    // c, x | y, z, e, 0) as two conflict-free half rows of 16 bytes per lane
    constexpr uint32_t ROWB = ROUND == 2 ? 32 : 8 * KI;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* wbase = smem + (size_t)warp * p.smem_per_warp;
    const uint32_t lane_base = smem_addr(wbase) + lane * (ROUND == 2 ? 16u : ROWB);
    uint4* stage = reinterpret_cast<uint4*>(wbase + (size_t)p.n_slots * 32 * ROWB);
    uint32_t* live = reinterpret_cast<uint32_t*>(wbase + (size_t)p.n_slots * 32 * ROWB + (STAGE + 1) * 16);
    if (lane == 0) stage[STAGE] = make_uint4(0u, 0u, 0u, 0u);  // sentinel past a full chunk

    const uint32_t L = p.level;
    const unsigned long long total = __ldcg(&p.prefix[p.n_trees]);
    const uint32_t chunk = chunk_for(total, gridDim.x * WARPS);
    uint32_t* keep = p.keep_scratch + (size_t)(blockIdx.x * WARPS + warp) * p.keep_stride;
    uint2* mmb = reinterpret_cast<uint2*>(keep + p.mm_ofs);

    // The tree of the current item, and its statistics so far (flushed to its
    // header when the warp moves to another tree: stats_buf, main.comp:146-147).
    LevelTree T{};
    unsigned long long t_lo = 0, t_hi = 0;
    bool have_tree = false;
    unsigned long long stat_sum = 0, stat_work = 0;
    uint32_t stat_max = 0;
    auto flush = [&]() {
        unsigned long long ssum = stat_sum;
        uint32_t smax = stat_max;
        for (int off = 16; off > 0; off >>= 1) {
            ssum += __shfl_down_sync(0xFFFFFFFFu, ssum, off);
            smax = max(smax, __shfl_down_sync(0xFFFFFFFFu, smax, off));
        }
        if (lane == 0) {
            if (ssum) atomicAdd(&T.H->tape_size_sum[L + 1], ssum);
            if (smax) atomicMax(&T.H->tape_size_max[L + 1], smax);
            if (stat_work) atomicAdd(&T.H->cell_instr[L], stat_work);
        }
        stat_sum = 0;
        stat_max = 0;
        stat_work = 0;
    };

    // item pruning: the prepared group of items (one node, lanes = items)
    // (not at level 0: with bricks, a batch's root level pruned per brick, a
    // dozen bricks per fetch, took 74.7 ms against 43.0 ms without)
    uint64_t* items = nullptr;
    if constexpr (ROUND < 2)
        if (p.item_cap && L > 0) items = reinterpret_cast<uint64_t*>(keep + p.item_ofs);
    // (the items pg_first .. pg_first + pg_g - 1, consecutive in this warp's
    // fetches; this lane's plan is item pg_first + lane's)
    unsigned long long pg_first = 0;
    uint32_t pg_g = 0, p_plan = 0;

    unsigned long long first;
    uint32_t got;
    while ((got = fetch_items(p.cursor, total, chunk, &first)) != 0) {
        for (uint32_t it = 0; it < got; it++) {
            const unsigned long long item = first + it;
            if (!have_tree || item >= t_hi) {
                if (have_tree) flush();
                const uint32_t ti = find_tree(p.prefix, p.n_trees, item);
                t_lo = __ldcg(&p.prefix[ti]);
                t_hi = __ldcg(&p.prefix[ti + 1]);
                T = load_tree(p.trees[ti], L, false);
                have_tree = true;
            }
            const uint32_t dim = T.dim;
            const uint32_t words = dim * dim * dim / 32;  // mask words per node
            const uint32_t groups = words / KI;           // items per node
            uint32_t node, grp;
            split_item(item - t_lo, groups, T.dim_sh == NOT_POW2 ? NOT_POW2 : 3 * T.dim_sh - 5 - (KI == 2),
                       &node, &grp);
            if (p.eval_list) node = __ldcg(&p.eval_list[node]);  // the others are copies
            uint32_t* rec = T.nodes + T.ofs_l + (size_t)node * T.node_size;
            const uint32_t tape_idx = rec[0];
            const uint32_t ncx = rec[1], ncy = rec[2], ncz = rec[3];
            const uint64_t* tape = T.tapes + tape_idx + 1;
            const uint32_t n_node = (uint32_t)__ldcg(&T.tapes[tape_idx]);
            uint32_t n = n_node;  // length of the tape the cells run (the item's, when pruned)
            const float cs = T.cs;
            // the item's brick: this lane's cells, their bit indices in the node
            uint32_t cell[KI], gx[KI], gy[KI], gz[KI];
            {
                uint32_t ox, oy, oz;
                brick_origin<KI>(grp, dim, T.dim_sh, &ox, &oy, &oz);
#pragma unroll
                for (int h = 0; h < KI; h++) {
                    uint32_t cx, cy, cz;
                    cell[h] = brick_cell<KI>(ox, oy, oz, h * 32u + lane, dim, &cx, &cy, &cz);
                    gx[h] = ncx * dim + cx;
                    gy[h] = ncy * dim + cy;
                    gz[h] = ncz * dim + cz;
                }
            }

            if constexpr (ROUND < 2) {
                if (items && 32u * KI < dim * dim * dim) {
                    if (item - pg_first >= pg_g) {
                        // the rest of this node's items in the fetched chunk, up to 32
                        const uint32_t g = min(min(32u, groups - grp), got - it);
                        p_plan = prepare_items<ROUND, KI>(
                            tape, n_node, ItemNode{dim, T.dim_sh, ncx, ncy, ncz, cs, T.lx, T.ly, T.lz, T.tt}, grp, g,
                            smem_addr(wbase) + lane * 8u, stage, keep, mmb, items, p.mm_cap, p.n_slots,
                            p.item_cap);
                        pg_first = item;
                        pg_g = g;
                    }
                    const uint32_t plan = __shfl_sync(0xFFFFFFFFu, p_plan, (int)(item - pg_first));
                    const uint32_t mode = plan & 3u;
                    if (mode == 1) {
                        tape = items + ((plan >> 2) & 0x7FFFu) * 16u;
                        n = plan >> 17;
                    } else if (mode >= 2) {  // every cell empty (2) or a leaf (3): no evaluation
#pragma unroll
                        for (int h = 0; h < KI; h++) {
                            rec[4 + 2 * words + cell[h]] = 0xFFFFFFFFu;
                            if (mode == 3) or_group_masks(rec + 4, rec + 4 + words, cell[h], 0xFFFFFFFFu, 0u, lane);
                        }
                        stat_work += 32ull * KI * n_node;
                        continue;
                    }
                }
            }

            IVK<KI> bx, by, bz, bt;
#pragma unroll
            for (int h = 0; h < KI; h++) {
                // voxelizer/main.comp:113-116, :124-126
                const float lox = __fadd_rn(T.lx, __fmul_rn((float)gx[h], cs));
                const float loy = __fadd_rn(T.ly, __fmul_rn((float)gy[h], cs));
                const float loz = __fadd_rn(T.lz, __fmul_rn((float)gz[h], cs));
                bx.v[h] = make_float2(lox, __fadd_rn(lox, cs));
                by.v[h] = make_float2(loy, __fadd_rn(loy, cs));
                bz.v[h] = make_float2(loz, __fadd_rn(loz, cs));
                bt.v[h] = make_float2(T.tt, T.tt);
            }
            uint32_t mm = 0;
            IVK<KI> r;
            uint64_t pre[STAGE / 32];
            prefetch_chunk(pre, tape, 0, n, lane);
            if constexpr (ROUND == 2) {
                // ---- forward pass, hybrid affine mode (device_common.cuh) ----
                const float2 ax[3] = {bx.v[0], by.v[0], bz.v[0]};
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const Af f = af_axis(ax[k].x, ax[k].y, k);
                    sts_f4(lane_base + k * 32 * ROWB, make_float4(ax[k].x, ax[k].y, f.c, f.x));
                    sts_f4(lane_base + k * 32 * ROWB + 512, make_float4(f.y, f.z, f.e, 0.0f));
                }
                sts_f4(lane_base + 3 * 32 * ROWB, make_float4(T.tt, T.tt, T.tt, 0.0f));
                sts_f4(lane_base + 3 * 32 * ROWB + 512, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
                for (uint32_t base = 0; base < n; base += STAGE) {
                    const uint32_t m = min(STAGE, n - base);
                    __syncwarp();
                    stage_chunk<false>(stage, pre, ROWB, lane, m);
                    prefetch_chunk(pre, tape, base + STAGE, n, lane);
                    __syncwarp();
                    const uint32_t sbase = smem_addr(stage);
                    for (uint32_t j = 0; j < m; j++) {
                        const uint4 d = lds_u4(sbase + j * 16);
                        float2 v;
                        Af f;
                        if (d.x == OP_CONST) {
                            const float c = __uint_as_float(d.y);
                            v = make_float2(c, c);
                            f = Af{c, 0.0f, 0.0f, 0.0f, 0.0f};
                        } else {
                            const float4 a0 = lds_f4(lane_base + d.y), a1 = lds_f4(lane_base + d.y + 512);
                            const float4 b0 = lds_f4(lane_base + d.z), b1 = lds_f4(lane_base + d.z + 512);
                            const float2 a = make_float2(a0.x, a0.y), b = make_float2(b0.x, b0.y);
                            const Af fa{a0.z, a0.w, a1.x, a1.y, a1.z}, fb{b0.z, b0.w, b1.x, b1.y, b1.z};
                            uint32_t c = 0;
                            if (is_mm(d.x)) {
                                c = mm_choice(d.x, a, b);
                                const uint2 ch = make_uint2(__ballot_sync(0xFFFFFFFFu, c & 1u),
                                                            __ballot_sync(0xFFFFFFFFu, c & 2u));
                                if (lane == 0 && mm < p.mm_cap) mmb[mm] = ch;
                                mm++;
                            }
                            v = hy_apply(d.x, 0ull, a, b, fa, fb, d.x == OP_MUL && d.y == d.z, c, &f);
                        }
                        sts_f4(lane_base + d.w, make_float4(v.x, v.y, f.c, f.x));
                        sts_f4(lane_base + d.w + 512, make_float4(f.y, f.z, f.e, 0.0f));
                    }
                }
            } else {
            sts_iv<KI>(lane_base + 0 * 32 * ROWB, bx);
            sts_iv<KI>(lane_base + 1 * 32 * ROWB, by);
            sts_iv<KI>(lane_base + 2 * 32 * ROWB, bz);
            sts_iv<KI>(lane_base + 3 * 32 * ROWB, bt);

            // ---- forward interval pass (interval.comp:121-160) ----
            // With two cells per lane the jump-table loop (interval_dispatch.cuh)
            // runs every opcode but DIV / SIN / COS / EXP, which it hands back
            // to iv_exec here.
            for (uint32_t base = 0; base < n; base += STAGE) {
                const uint32_t m = min(STAGE, n - base);
                __syncwarp();
                stage_chunk<false>(stage, pre, ROWB, lane, m);
                prefetch_chunk(pre, tape, base + STAGE, n, lane);
                __syncwarp();
                const uint32_t sbase = smem_addr(stage);
                if constexpr (KI == 2) {
                    uint32_t j = 0;
                    while (true) {
                        IvRun run;
                        if constexpr (ROUND == 0) run = iv_run_0_2(sbase, j, m, lane_base, mmb, mm, p.mm_cap);
                        else run = iv_run_1_2(sbase, j, m, lane_base, mmb, mm, p.mm_cap);
                        j = run.j;
                        mm = run.mm;
                        if (j >= m) break;
                        const uint4 d = lds_u4(sbase + j * 16);
                        r = iv_exec<ROUND, KI>(d, lane_base, lane, mmb, mm, p.mm_cap);
                        sts_iv<KI>(lane_base + d.w, r);
                        j++;
                    }
                } else {
                    // The decode word of j+1 is read one instruction early.
                    uint4 dn = lds_u4(sbase);
                    for (uint32_t j = 0; j < m; j++) {
                        const uint4 d = dn;
                        dn = lds_u4(sbase + (j + 1) * 16);
                        if (d.x == OP_CONST) {
                            const float c = __uint_as_float(d.y);
#pragma unroll
                            for (int h = 0; h < KI; h++) r.v[h] = make_float2(c, c);
                        } else {
                            r = iv_exec<ROUND, KI>(d, lane_base, lane, mmb, mm, p.mm_cap);
                        }
                        sts_iv<KI>(lane_base + d.w, r);
                    }
                }
            }
            }
            __syncwarp();
            // the reference's work: every cell evaluates its node's tape
            stat_work += 32ull * KI * n_node;

            // ---- classification (voxelizer/main.comp:88-108) ----
            const IVK<KI> res = lds_iv<KI>(lane_base);
            uint32_t leaf_w[KI], amb_w[KI], ok_w[KI];
            bool ok[KI];
            unsigned long long my_child[KI];
            uint32_t n_amb = 0;
#pragma unroll
            for (int h = 0; h < KI; h++) {
                const bool empty = res.v[h].x > 0.0f;
                const bool leaf = !empty && res.v[h].y < 0.0f;
                const bool amb = !empty && !leaf;
                leaf_w[h] = __ballot_sync(0xFFFFFFFFu, leaf);
                amb_w[h] = __ballot_sync(0xFFFFFFFFu, amb);
                n_amb += __popc(amb_w[h]);
            }

            // ---- child allocation (main.comp:138-148), warp-aggregated ----
            unsigned long long child_base = 0;
            if (n_amb) {
                if (lane == 0) child_base = atomicAdd(&T.H->node_count[L + 1], n_amb);
                child_base = __shfl_sync(0xFFFFFFFFu, child_base, 0);
                // The children (ids child_base .. child_base + n_amb - 1, those
                // below child_cap are created) of an interval level get their
                // mask words zeroed here: their own pass ORs bricks into them.
                if (T.next_mask_words) {
                    const unsigned long long c_end = min(child_base + n_amb, T.child_cap);
                    const uint32_t made = c_end > child_base ? (uint32_t)(c_end - child_base) : 0u;
                    const uint32_t mw = T.next_mask_words;
                    for (uint32_t k = lane; k < made * mw; k += 32) {
                        const uint32_t c = k / mw;
                        T.nodes[T.ofs_next + (child_base + c) * T.node_size_next + 4 + (k - c * mw)] = 0u;
                    }
                }
            }
            bool any_ok = false, lost = false;
#pragma unroll
            for (int h = 0; h < KI; h++) {
                my_child[h] = child_base + __popc(amb_w[h] & lanemask_lt());
                child_base += __popc(amb_w[h]);
                const bool amb = (amb_w[h] >> lane) & 1u;
                ok[h] = amb && my_child[h] < T.child_cap;
                ok_w[h] = __ballot_sync(0xFFFFFFFFu, ok[h]);
                any_ok |= ok_w[h] != 0u;
                lost |= ok_w[h] != amb_w[h];
            }
            if (lost && lane == 0) atomicOr(&T.H->overflow, 1u);

            uint32_t child_tape[KI], child_len[KI];
#pragma unroll
            for (int h = 0; h < KI; h++) {
                child_tape[h] = tape_idx;
                child_len[h] = n_node;
            }
            if (any_ok && T.shorten) {
                // ---- backward liveness (shorten.comp:148-186) ----
                uint32_t kept[KI];
                // sig: a cheap summary of this cell's output tape (the kept
                // instruction positions and the MIN/MAX rewrites), to group
                // cells whose tapes may be identical (verified exactly below)
                uint32_t sig[KI];
#pragma unroll
                for (int h = 0; h < KI; h++) {
                    kept[h] = 0;
                    sig[h] = 0;
                }
                if (p.n_slots <= 32) {
                    // live sets spread over the lanes' registers: no shared
                    // memory on the walk's path
                    walk_lanes<KI, 1>(tape, n, (int)mm, mmb, keep, ok_w, lane, kept, sig);
                } else if (p.n_slots <= 64) {
                    walk_lanes<KI, 2>(tape, n, (int)mm, mmb, keep, ok_w, lane, kept, sig);
                } else {
                    // wider slot files: transposed bitsets, live[s][h] bit l =
                    // slot s is live for cell grp*32*KI + h*32 + l. The
                    // kept-mask of an instruction is live[out]; then live[out] =
                    // 0 and the inputs its choice uses become live for the cells
                    // that kept it.
                    for (uint32_t s = lane; s < p.n_slots * KI; s += 32) live[s] = 0u;
                    __syncwarp();
                    if (lane == 0) {
#pragma unroll
                        for (int h = 0; h < KI; h++) live[h] = ok_w[h];
                    }
                    __syncwarp();
                    int mmi = (int)mm - 1;
                    for (int hi = (int)n; hi > 0; hi -= 32) {
                        const int lo = max(0, hi - 32);
                        const int m = hi - lo;
                        // lane j holds instruction lo + j; walked from the top down
                        const uint64_t mine = (int)lane < m ? __ldcg(&tape[lo + lane]) : 0ull;
                        uint32_t my_keep[KI];
#pragma unroll
                        for (int h = 0; h < KI; h++) my_keep[h] = 0;
                        for (int j = m - 1; j >= 0; j--) {
                            const uint64_t w = __shfl_sync(0xFFFFFFFFu, mine, j);
                            const uint32_t op = w_op(w), o = w_out(w);
                            uint32_t k[KI];
                            if constexpr (KI == 1) {
                                k[0] = live[o];
                            } else {
                                const uint2 kk = *reinterpret_cast<const uint2*>(&live[o * 2]);
                                k[0] = kk.x;
                                k[1] = kk.y;
                            }
                            bool any = false;
#pragma unroll
                            for (int h = 0; h < KI; h++) any |= k[h] != 0u;
                            if (any) {
                                uint32_t first_m[KI], second_m[KI];
                                if (op == OP_CONST) {
#pragma unroll
                                    for (int h = 0; h < KI; h++) first_m[h] = second_m[h] = 0u;
                                } else if (op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_DIV) {
#pragma unroll
                                    for (int h = 0; h < KI; h++) first_m[h] = second_m[h] = ~0u;
                                } else if (is_mm(op)) {
#pragma unroll
                                    for (int h = 0; h < KI; h++) {
                                        const uint2 cb = mmb[mmi * KI + h];
                                        first_m[h] = cb.x;
                                        second_m[h] = cb.y;
                                    }
                                } else {
#pragma unroll
                                    for (int h = 0; h < KI; h++) {
                                        first_m[h] = ~0u;
                                        second_m[h] = 0u;
                                    }
                                }
                                __syncwarp();
                                if (lane == 0) {
                                    const uint32_t ia = w_a(w), ib = w_b(w);
#pragma unroll
                                    for (int h = 0; h < KI; h++) {
                                        live[o * KI + h] = 0u;
                                        const uint32_t fa = k[h] & first_m[h], sb = k[h] & second_m[h];
                                        if (fa) live[ia * KI + h] |= fa;
                                        if (sb) live[ib * KI + h] |= sb;
                                    }
                                }
                                __syncwarp();
#pragma unroll
                                for (int h = 0; h < KI; h++) {
                                    const uint32_t kb = (k[h] >> lane) & 1u;
                                    kept[h] += kb;
                                    const uint32_t code = kb + ((first_m[h] >> lane) & kb) + ((second_m[h] >> lane) & kb) * 2u;
                                    sig[h] += code * (uint32_t)(lo + j + 1) * 0x9E3779B1u;
                                }
                            }
                            if ((int)lane == j) {
#pragma unroll
                                for (int h = 0; h < KI; h++) my_keep[h] = k[h];
                            }
                            if (is_mm(op)) mmi--;
                        }
                        if ((int)lane < m) {
                            if constexpr (KI == 1) keep[lo + lane] = my_keep[0];
                            else reinterpret_cast<uint2*>(keep)[lo + lane] = make_uint2(my_keep[0], my_keep[1]);
                        }
                    }
                }
                __syncwarp();

                // ---- one tape per distinct output (this library's addition) ----
                // Cells of a 32-cell group whose shortened tapes are identical
                // share one copy: neighbouring cells usually keep the same
                // primitives, and the pool then holds ~3x fewer tape words. A
                // cell's leader is the lowest lane with the same signature and
                // length; the grouping is then verified exactly (keep bits and
                // MIN/MAX rewrites column by column), so a signature collision
                // only costs a copy. Contents per cell are unchanged.
                bool do_short[KI];
                uint32_t leader[KI], lead_w[KI], group[KI];
#pragma unroll
                for (int h = 0; h < KI; h++) {
                    // "not shorter -> reuse" (:188-191), against the node's tape
                    do_short[h] = ok[h] && kept[h] < n_node;
                    const unsigned long long key = do_short[h] && T.share
                                                       ? ((unsigned long long)sig[h] << 32 | kept[h]) * 2ull + 1ull
                                                       : 2ull * (lane + 1);
                    group[h] = __match_any_sync(0xFFFFFFFFu, key);
                    leader[h] = __ffs(group[h]) - 1;
                }
                {
                    // leaders whose group has followers
                    uint32_t lwf[KI], any_fol = 0;
#pragma unroll
                    for (int h = 0; h < KI; h++) {
                        lwf[h] = __ballot_sync(0xFFFFFFFFu, do_short[h] && leader[h] == lane && __popc(group[h]) > 1);
                        any_fol |= lwf[h];
                    }
                    if (any_fol) {
                        uint32_t bad[KI];
#pragma unroll
                        for (int h = 0; h < KI; h++) bad[h] = 0;
                        uint32_t mm_v = 0;
                        for (uint32_t b = 0; b < n; b += 32) {
                            const uint32_t idx = b + lane;
                            const bool valid = idx < n;
                            const uint64_t w = valid ? __ldcg(&tape[idx]) : 0ull;
                            const bool ism = valid && is_mm(w_op(w));
                            const uint32_t mball = __ballot_sync(0xFFFFFFFFu, ism);
#pragma unroll
                            for (int h = 0; h < KI; h++) {
                                const uint32_t km = valid ? keep[(size_t)idx * KI + h] : 0u;
                                uint2 cb = make_uint2(0u, 0u);
                                if (ism) cb = mmb[(mm_v + __popc(mball & lanemask_lt())) * KI + h];
                                // lane `lane` holds instruction idx: within each group,
                                // every member's keep bit (and, where kept, its MIN/MAX
                                // choice bits) must equal the leader's; groups that keep
                                // nothing of this chunk agree on it
                                const uint32_t anyk = __reduce_or_sync(0xFFFFFFFFu, km);
                                uint32_t pend = __ballot_sync(0xFFFFFFFFu, ((lwf[h] >> lane) & 1u) && (group[h] & anyk)),
                                         d = 0;
                                while (pend) {
                                    const int ld = __ffs(pend) - 1;
                                    pend &= pend - 1;
                                    const uint32_t M = __shfl_sync(0xFFFFFFFFu, group[h], ld);
                                    uint32_t diff = (km & M) ^ (((km >> ld) & 1u) ? M : 0u);
                                    if (ism)
                                        diff |= ((cb.x & M) ^ (((cb.x >> ld) & 1u) ? M : 0u) |
                                                 (cb.y & M) ^ (((cb.y >> ld) & 1u) ? M : 0u)) & km;
                                    d |= diff;
                                }
                                bad[h] |= __reduce_or_sync(0xFFFFFFFFu, d);
                            }
                            mm_v += __popc(mball);
                        }
#pragma unroll
                        for (int h = 0; h < KI; h++)
                            if ((bad[h] >> lane) & 1u) leader[h] = lane;
                    }
                }

                // ---- claim output tapes (shorten.comp:136-142), one atomic per warp ----
                uint32_t tw[KI], lane_words = 0;
#pragma unroll
                for (int h = 0; h < KI; h++) {
                    lead_w[h] = __ballot_sync(0xFFFFFFFFu, do_short[h] && leader[h] == lane);
                    tw[h] = ((lead_w[h] >> lane) & 1u)
                                ? (1 + kept[h] + TAPE_ALIGN_WORDS - 1) / TAPE_ALIGN_WORDS * TAPE_ALIGN_WORDS
                                : 0;
                    lane_words += tw[h];
                }
                uint32_t incl = lane_words;
                for (int off = 1; off < 32; off <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
                    if ((int)lane >= off) incl += v;
                }
                const uint32_t total_words = __shfl_sync(0xFFFFFFFFu, incl, 31);
                unsigned long long tbase = 0;
                if (total_words) {
                    if (lane == 0) tbase = atomicAdd(&T.H->tape_top, (unsigned long long)total_words);
                    tbase = __shfl_sync(0xFFFFFFFFu, tbase, 0);
                }
                unsigned long long my_tape[KI];
                bool tape_ok[KI];
                uint32_t short_w[KI], any_short = 0;
                unsigned long long at = tbase + (incl - lane_words);
#pragma unroll
                for (int h = 0; h < KI; h++) {
                    my_tape[h] = at;
                    at += tw[h];
                    const bool lead = (lead_w[h] >> lane) & 1u;
                    tape_ok[h] = lead && my_tape[h] + tw[h] <= T.tape_cap;
                    if (lead && !tape_ok[h]) atomicOr(&T.H->overflow, 2u);
                    short_w[h] = __ballot_sync(0xFFFFFFFFu, tape_ok[h]);  // leaders whose tape is written
                    any_short |= short_w[h];
                    // followers take their leader's tape
                    const unsigned long long lt = __shfl_sync(0xFFFFFFFFu, my_tape[h], (int)leader[h]);
                    if (do_short[h] && !lead) {
                        my_tape[h] = lt;
                        tape_ok[h] = (short_w[h] >> leader[h]) & 1u;
                    }
                }

                // ---- copy of the shortened tapes (shorten.comp:193-221) ----
                // Chunk-outer: lane j holds instruction base + j, its keep masks
                // and (for MIN/MAX) its choice masks; each output tape then takes
                // one ballot + one coalesced store per chunk.
                if (any_short) {
                    uint32_t run[KI];  // lane L: instructions written so far to its own tapes
#pragma unroll
                    for (int h = 0; h < KI; h++) {
                        if ((short_w[h] >> lane) & 1u) T.tapes[my_tape[h]] = (uint64_t)kept[h];
                        run[h] = 0;
                    }
                    uint32_t mm_run = 0;
                    for (uint32_t b = 0; b < n; b += 32) {
                        const uint32_t idx = b + lane;
                        const bool valid = idx < n;
                        const uint64_t w = valid ? __ldcg(&tape[idx]) : 0ull;
                        uint32_t kmask[KI];
                        if constexpr (KI == 1) {
                            kmask[0] = valid ? keep[idx] : 0u;
                        } else {
                            const uint2 kk = valid ? reinterpret_cast<const uint2*>(keep)[idx] : make_uint2(0u, 0u);
                            kmask[0] = kk.x;
                            kmask[1] = kk.y;
                        }
                        const bool ism = valid && is_mm(w_op(w));
                        const uint32_t mball = __ballot_sync(0xFFFFFFFFu, ism);
                        uint2 cb[KI];
#pragma unroll
                        for (int h = 0; h < KI; h++) {
                            cb[h] = make_uint2(0u, 0u);
                            if (ism) cb[h] = mmb[(mm_run + __popc(mball & lanemask_lt())) * KI + h];
                        }
#pragma unroll
                        for (int h = 0; h < KI; h++) {
                            // only the tapes that keep some instruction of this chunk
                            uint32_t pending = short_w[h] & __reduce_or_sync(0xFFFFFFFFu, kmask[h]);
                            while (pending) {
                                const int sel = __ffs(pending) - 1;
                                pending &= pending - 1;
                                const bool kb = (kmask[h] >> sel) & 1u;
                                uint64_t wo = w;
                                if (kb && ism) {
                                    const uint32_t c = ((cb[h].x >> sel) & 1u) | (((cb[h].y >> sel) & 1u) << 1);
                                    if (c == MM_FIRST) {
                                        wo = (w & ~0xFFull) | OP_COPY;
                                    } else if (c == MM_SECOND) {  // COPY of B; the B field is kept
                                        wo = (w & ~0xFFull & ~(0xFFFFull << 32)) | OP_COPY | ((uint64_t)w_b(w) << 32);
                                    }
                                }
                                const uint32_t kball = __ballot_sync(0xFFFFFFFFu, kb);
                                const unsigned long long dst = __shfl_sync(0xFFFFFFFFu, my_tape[h], sel);
                                const uint32_t rr = __shfl_sync(0xFFFFFFFFu, run[h], sel);
                                if (kb) T.tapes[dst + 1 + rr + __popc(kball & lanemask_lt())] = wo;
                                if ((int)lane == sel) run[h] += __popc(kball);
                            }
                        }
                        mm_run += __popc(mball);
                    }
                }
#pragma unroll
                for (int h = 0; h < KI; h++) {
                    if (tape_ok[h]) {
                        child_tape[h] = (uint32_t)my_tape[h];
                        child_len[h] = kept[h];
                    }
                }
            }

            // ---- node records: masks, child list, children ----
#pragma unroll
            for (int h = 0; h < KI; h++) {
                if (ok[h]) {
                    uint32_t* crec = T.nodes + T.ofs_next + (size_t)my_child[h] * T.node_size_next;
                    crec[0] = child_tape[h];
                    crec[1] = gx[h];
                    crec[2] = gy[h];
                    crec[3] = gz[h];
                    stat_sum += child_len[h];
                    stat_max = max(stat_max, child_len[h]);
                }
                rec[4 + 2 * words + cell[h]] = ok[h] ? (uint32_t)my_child[h] : 0xFFFFFFFFu;
                or_group_masks(rec + 4, rec + 4 + words, cell[h], leaf_w[h], ok_w[h], lane);
            }
        }
    }

    if (have_tree) flush();
}

// ---- point level pass (the last level) ---------------------------------------------
//
// The leaf bit is the sign of the point value at the cell's low corner
// (voxelize_point, main.comp:74-83; tape_eval_point, point.comp:2-63).
// Each lane evaluates K cells at once (cells grp*32K + k*32 + lane; K = 4, or
// 2 for nodes too small for 4, or 8 on request), so one decoded instruction
// drives 32*K evaluations and a lane's slot row is one K-float vector (two
// for K = 8). A tape that fits one
// staged chunk stays staged across consecutive items of the same node.
template <int K>
struct alignas(4 * K) FK {
    float v[K];
};

// K = 8: a slot row is two halves of 32 lanes x 16 bytes ([slot][half][lane]),
// so that each 16-byte access of the warp stays conflict-free.
constexpr uint32_t K8_HALF = 32 * 16;

template <int K>
__device__ __forceinline__ FK<K> lds_k(uint32_t a) {
    FK<K> r;
    if constexpr (K == 8) {
        const float4 v = lds_f4(a), w = lds_f4(a + K8_HALF);
        r.v[0] = v.x; r.v[1] = v.y; r.v[2] = v.z; r.v[3] = v.w;
        r.v[4] = w.x; r.v[5] = w.y; r.v[6] = w.z; r.v[7] = w.w;
    } else if constexpr (K == 4) {
        const float4 v = lds_f4(a);
        r.v[0] = v.x; r.v[1] = v.y; r.v[2] = v.z; r.v[3] = v.w;
    } else {
        const float2 v = lds_f2(a);
        r.v[0] = v.x; r.v[1] = v.y;
    }
    return r;
}
template <int K>
__device__ __forceinline__ void sts_k(uint32_t a, const FK<K>& r) {
    if constexpr (K == 8) {
        sts_f4(a, make_float4(r.v[0], r.v[1], r.v[2], r.v[3]));
        sts_f4(a + K8_HALF, make_float4(r.v[4], r.v[5], r.v[6], r.v[7]));
    } else if constexpr (K == 4) sts_f4(a, make_float4(r.v[0], r.v[1], r.v[2], r.v[3]));
    else sts_f2(a, make_float2(r.v[0], r.v[1]));
}

// Case generators for the point interpreter's switch: one case per (opcode,
// forwarding) combination, each straight-line code with its operand sources
// fixed. (On the point pass, with four cells per lane and vector slot rows,
// this measured faster than testing the frequent combinations first.)
#define FREP_CASES_BINARY(X, OPC) \
    X(OPC, false, false)          \
    X(OPC, true, false)           \
    X(OPC, false, true)           \
    X(OPC, true, true)
#define FREP_CASES_UNARY(X, OPC) \
    X(OPC, false, false)         \
    X(OPC, true, false)
#define FREP_ALL_CASES(X)               \
    FREP_CASES_BINARY(X, OP_MUL)        \
    FREP_CASES_BINARY(X, OP_SUB)        \
    FREP_CASES_BINARY(X, OP_ADD)        \
    FREP_CASES_BINARY(X, OP_MAX)        \
    FREP_CASES_BINARY(X, OP_MIN)        \
    FREP_CASES_BINARY(X, OP_DIV)        \
    FREP_CASES_UNARY(X, OP_COPY)        \
    FREP_CASES_UNARY(X, OP_SQRT)        \
    FREP_CASES_UNARY(X, OP_NEG)         \
    FREP_CASES_UNARY(X, OP_SIN)         \
    FREP_CASES_UNARY(X, OP_COS)         \
    FREP_CASES_UNARY(X, OP_EXP)

// One point instruction with its operand sources fixed at compile time.
// r: in = the previous instruction's result, out = this one's.
template <int K, uint32_t OP, bool FA, bool FB>
__device__ __forceinline__ void pt_exec(const uint4 d, FK<K>& r, uint32_t lane_base) {
    const FK<K> a = FA ? r : lds_k<K>(lane_base + d.y);
    FK<K> b;
    if constexpr (is_binary(OP)) b = FB ? r : lds_k<K>(lane_base + d.z);
#pragma unroll
    for (int k = 0; k < K; k++) {
        float v;
        if constexpr (OP == OP_MUL) v = __fmul_rn(a.v[k], b.v[k]);
        else if constexpr (OP == OP_SUB) v = __fsub_rn(a.v[k], b.v[k]);
        else if constexpr (OP == OP_ADD) v = __fadd_rn(a.v[k], b.v[k]);
        else if constexpr (OP == OP_MAX) v = max_sel(a.v[k], b.v[k]);
        else if constexpr (OP == OP_MIN) v = min_sel(a.v[k], b.v[k]);
        else if constexpr (OP == OP_COPY) v = a.v[k];
        else if constexpr (OP == OP_NEG) v = -a.v[k];
        else if constexpr (OP == OP_SQRT) v = __fsqrt_rn(a.v[k]);
        else if constexpr (OP == OP_DIV) v = __fdiv_rn(a.v[k], b.v[k]);
        else if constexpr (OP == OP_SIN) v = frep_sinf(a.v[k]);
        else if constexpr (OP == OP_COS) v = frep_cosf(a.v[k]);
        else v = frep_expf(a.v[k]);  // OP_EXP
        r.v[k] = v;
    }
}

// (inside namespace frep::dev: the generated loop uses FK<K>)
#include "point_dispatch.cuh"

template <int WARPS, int K>
__global__ void __launch_bounds__(WARPS * 32)
point_level_kernel(LevelLaunch p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* wbase = smem + (size_t)warp * p.smem_per_warp;
    constexpr uint32_t ROW = 4 * K;  // bytes per lane per slot
    const uint32_t lane_base = smem_addr(wbase) + lane * (K == 8 ? 16u : ROW);
    uint4* stage = reinterpret_cast<uint4*>(wbase + (size_t)p.n_slots * 32 * ROW);
    if (lane == 0) stage[STAGE] = make_uint4(0u, 0u, 0u, 0u);  // sentinel past a full chunk

    const uint32_t L = p.level;
    const unsigned long long total = __ldcg(&p.prefix[p.n_trees]);
    const uint32_t chunk = chunk_for(total, gridDim.x * WARPS);
    unsigned long long stat_work = 0;
    uint32_t staged_tape = 0xFFFFFFFFu;  // tape whose whole body is in `stage`
    const uint64_t* staged_pool = nullptr;
    LevelTree T{};
    unsigned long long t_lo = 0, t_hi = 0;
    bool have_tree = false;

    unsigned long long first;
    uint32_t got;
    while ((got = fetch_items(p.cursor, total, chunk, &first)) != 0) {
        for (uint32_t it = 0; it < got; it++) {
            const unsigned long long item = first + it;
            if (!have_tree || item >= t_hi) {
                if (have_tree && lane == 0 && stat_work) atomicAdd(&T.H->cell_instr[L], stat_work);
                stat_work = 0;
                const uint32_t ti = find_tree(p.prefix, p.n_trees, item);
                t_lo = __ldcg(&p.prefix[ti]);
                t_hi = __ldcg(&p.prefix[ti + 1]);
                T = load_tree(p.trees[ti], L, true);
                have_tree = true;
            }
            const uint32_t dim = T.dim;
            const uint32_t words = dim * dim * dim / 32;      // mask words per node
            const uint32_t groups = words / K;                // items per node
            const float cs = T.cs;
            constexpr uint32_t LOG2K = K == 8 ? 3 : (K == 4 ? 2 : 1);
            uint32_t node, grp;
            split_item(item - t_lo, groups, T.dim_sh == NOT_POW2 ? NOT_POW2 : 3 * T.dim_sh - 5 - LOG2K, &node,
                       &grp);
            if (p.eval_list) node = __ldcg(&p.eval_list[node]);  // the others are copies
            uint32_t* rec = T.nodes + T.ofs_l + (size_t)node * T.node_size;
            const uint32_t tape_idx = rec[0];
            const uint64_t* tape = T.tapes + tape_idx + 1;
            const uint32_t n = (uint32_t)__ldcg(&T.tapes[tape_idx]);
            const uint32_t ncx = rec[1], ncy = rec[2], ncz = rec[3];
            FK<K> px, py, pz, pt;
#pragma unroll
            for (int k = 0; k < K; k++) {
                const uint32_t cell = grp * 32 * K + k * 32 + lane;
                uint32_t cx, cy, cz;
                cell_xyz(cell, dim, T.dim_sh, &cx, &cy, &cz);
                px.v[k] = __fadd_rn(T.lx, __fmul_rn((float)(ncx * dim + cx), cs));
                py.v[k] = __fadd_rn(T.ly, __fmul_rn((float)(ncy * dim + cy), cs));
                pz.v[k] = __fadd_rn(T.lz, __fmul_rn((float)(ncz * dim + cz), cs));
                pt.v[k] = T.tt;
            }
            sts_k<K>(lane_base + 0 * 32 * ROW, px);
            sts_k<K>(lane_base + 1 * 32 * ROW, py);
            sts_k<K>(lane_base + 2 * 32 * ROW, pz);
            sts_k<K>(lane_base + 3 * 32 * ROW, pt);
            const bool resident = n <= STAGE && staged_tape == tape_idx && staged_pool == T.tapes;
            FK<K> r;
#pragma unroll
            for (int k = 0; k < K; k++) r.v[k] = 0.0f;
            uint64_t pre[STAGE / 32];
            if (!resident) prefetch_chunk(pre, tape, 0, n, lane);
            for (uint32_t base = 0; base < n; base += STAGE) {
                const uint32_t m = min(STAGE, n - base);
                if (!resident) {
                    __syncwarp();
                    stage_chunk<true>(stage, pre, ROW, lane, m);
                    prefetch_chunk(pre, tape, base + STAGE, n, lane);
                    __syncwarp();
                }
                const uint32_t sbase = smem_addr(stage);
                if constexpr (K == 2 || K == 4 || K == 8) {
                    // the jump-table loop (point_dispatch.cuh); SIN / COS / EXP here
                    uint32_t j = 0;
                    while (true) {
                        PtRun<K> run;
                        if constexpr (K == 2) run = pt_run_2(sbase, j, m, lane_base, r);
                        else if constexpr (K == 4) run = pt_run_4(sbase, j, m, lane_base, r);
                        else run = pt_run_8(sbase, j, m, lane_base, r);
                        j = run.j;
                        r = run.r;
                        if (j >= m) break;
                        const uint4 d = lds_u4(sbase + j * 16);
                        switch (d.x) {
#define FREP_PT_CASE(OPC, FA, FB)                         \
    case OPC | (FA ? F_FWD_A : 0u) | (FB ? F_FWD_B : 0u): \
        pt_exec<K, OPC, FA, FB>(d, r, lane_base);         \
        break;
                            FREP_CASES_UNARY(FREP_PT_CASE, OP_SIN)
                            FREP_CASES_UNARY(FREP_PT_CASE, OP_COS)
                            FREP_CASES_UNARY(FREP_PT_CASE, OP_EXP)
#undef FREP_PT_CASE
                            default: break;
                        }
                        sts_k<K>(lane_base + d.w, r);
                        j++;
                    }
                } else {
                // The decode word of j+1 is read one instruction early.
                uint4 dn = lds_u4(sbase);
                for (uint32_t j = 0; j < m; j++) {
                    const uint4 d = dn;
                    dn = lds_u4(sbase + (j + 1) * 16);
                    switch (d.x) {
                        case OP_CONST:
#pragma unroll
                            for (int k = 0; k < K; k++) r.v[k] = __uint_as_float(d.y);
                            break;
#define FREP_PT_CASE(OPC, FA, FB)                         \
    case OPC | (FA ? F_FWD_A : 0u) | (FB ? F_FWD_B : 0u): \
        pt_exec<K, OPC, FA, FB>(d, r, lane_base);         \
        break;
                        FREP_ALL_CASES(FREP_PT_CASE)
#undef FREP_PT_CASE
                        default: break;
                    }
                    sts_k<K>(lane_base + d.w, r);
                }
                }
            }
            staged_tape = n <= STAGE ? tape_idx : 0xFFFFFFFFu;
            staged_pool = T.tapes;
            __syncwarp();
            stat_work += 32ull * K * n;
            const FK<K> d = lds_k<K>(lane_base);
#pragma unroll
            for (int k = 0; k < K; k++) {
                const uint32_t leaf_w = __ballot_sync(0xFFFFFFFFu, d.v[k] < 0.0f);
                if (lane == 0) {
                    rec[4 + grp * K + k] = leaf_w;
                    rec[4 + words + grp * K + k] = 0u;  // the unused second mask word range
                }
            }
        }
    }
    if (have_tree && lane == 0 && stat_work) atomicAdd(&T.H->cell_instr[L], stat_work);
}

// Lays the batch's items for `level` end to end: prefix[i] = items of trees
// before i that this launch serves (interval passes: trees for which `level`
// is not the last; point passes: trees for which it is, with a last-level node
// size that takes `k` cells per lane). An item is k mask words of a node (k
// cells per lane). Interval passes also fix where each tree's next level
// starts (node_ofs[level + 1]). One block.
__device__ __forceinline__ unsigned long long level_items(TreeHeader* H, uint32_t L, int point, int k,
                                                          bool write_ofs, bool reuse, bool any_k) {
    if (L >= H->levels) return 0;
    const bool last = L == H->levels - 1;
    if ((point != 0) != last) return 0;
    const uint32_t dim = H->dims[L];
    const uint32_t words = dim * dim * dim / 32;
    if (point && !any_k && H->point_k != (uint32_t)k) return 0;
    const uint32_t count = level_count(H, L, H->node_cap, H->node_size[L]);
    if (!point && write_ofs) H->node_ofs[L + 1] = H->node_ofs[L] + (unsigned long long)count * H->node_size[L];
    // with reuse, only the listed nodes are evaluated
    const uint32_t evaluated = reuse ? min(count, H->reuse_eval[L]) : count;
    return (unsigned long long)evaluated * (words / (uint32_t)k);  // k: cells per lane of the pass
}

__global__ void __launch_bounds__(1024)
level_scan_kernel(TreeHeader* const* trees, uint32_t n, uint32_t L, int point, int point_k,
                  unsigned long long* prefix, unsigned long long* cursor, int reuse, int any_k) {
    __shared__ unsigned long long part[1024];
    const uint32_t t = threadIdx.x, T = blockDim.x;
    const uint32_t per = (n + T - 1) / T;
    const uint32_t b = min(n, t * per), e = min(n, b + per);
    unsigned long long sum = 0;
    for (uint32_t i = b; i < e; i++) sum += level_items(trees[i], L, point, point_k, true, reuse != 0, any_k != 0);
    part[t] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < T; off <<= 1) {  // inclusive scan
        const unsigned long long v = t >= off ? part[t - off] : 0ull;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    unsigned long long run = part[t] - sum;
    for (uint32_t i = b; i < e; i++) {
        prefix[i] = run;
        run += level_items(trees[i], L, point, point_k, false, reuse != 0, any_k != 0);
    }
    if (t == T - 1) prefix[n] = part[t];
    if (t == 0) *cursor = 0ull;
}

// A root at an interval level (more than one level) starts with zeroed mask
// words: the level pass ORs its bricks into them.
__device__ __forceinline__ void zero_root_masks(TreeHeader* H, uint32_t t, uint32_t nt) {
    if (H->levels < 2) return;
    const uint32_t d = H->dims[0];
    const uint32_t mw = d * d * d / 16u;
    for (uint32_t w = t; w < mw; w += nt) H->nodes[4 + w] = 0u;
}

// Resets the headers and writes the root nodes (Voxelizer::Voxelize sets
// interiorNodeCount[0] = 1 and relies on a zeroed root, voxelizer.cpp:432-435).
// One block per tree; each tree's root tape is already at word 0 of its pool.
__global__ void tree_init_kernel(TreeHeader* const* trees, uint32_t n, const float* tape_times, float tape_time) {
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        TreeHeader* H = trees[i];
        const uint32_t t = threadIdx.x;
        const uint32_t root_n = (uint32_t)H->tapes[0];
        if (t < MAX_LEVELS) {
            H->node_count[t] = t == 0 ? 1u : 0u;
            H->node_ofs[t] = 0;
            H->tape_size_sum[t] = t == 0 ? root_n : 0;
            H->tape_size_max[t] = t == 0 ? root_n : 0;
            H->cell_instr[t] = 0;
            H->fp32_ops[t] = 0;
            H->reuse_eval[t] = 0;
        }
        if (t == 0) {
            H->tape_top = (1 + (unsigned long long)root_n + TAPE_ALIGN_WORDS - 1) / TAPE_ALIGN_WORDS * TAPE_ALIGN_WORDS;
            H->overflow = 0;
            H->status = 0;
            H->tape_time = tape_times ? tape_times[i] : tape_time;
            uint32_t* root = H->nodes;
            root[0] = 0;  // root tape at word 0 of the tape pool
            root[1] = 0;
            root[2] = 0;
            root[3] = 0;
        }
        zero_root_masks(H, t, blockDim.x);
    }
}

// Batch variant of tree_init_kernel: block i first copies tree i's root tape
// record from the staged upload (words offsets[i] .. offsets[i+1] of `staged`)
// to word 0 of its tape pool, then resets its header like tree_init_kernel.
__global__ void tree_init_staged_kernel(TreeHeader* const* trees, uint32_t n, const uint64_t* staged,
                                        const unsigned long long* offsets, const float* tape_times) {
    for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        TreeHeader* H = trees[i];
        uint64_t* pool = H->tapes;
        const unsigned long long b = offsets[i], e = offsets[i + 1];
        for (unsigned long long w = b + threadIdx.x; w < e; w += blockDim.x) pool[w - b] = staged[w];
        __syncthreads();
        const uint32_t t = threadIdx.x;
        const uint32_t root_n = (uint32_t)pool[0];
        if (t < MAX_LEVELS) {
            H->node_count[t] = t == 0 ? 1u : 0u;
            H->node_ofs[t] = 0;
            H->tape_size_sum[t] = t == 0 ? root_n : 0;
            H->tape_size_max[t] = t == 0 ? root_n : 0;
            H->cell_instr[t] = 0;
            H->fp32_ops[t] = 0;
            H->reuse_eval[t] = 0;
        }
        if (t == 0) {
            H->tape_top = e - b;
            H->overflow = 0;
            H->status = 0;
            H->tape_time = tape_times[i];
            uint32_t* root = H->nodes;
            root[0] = 0;
            root[1] = 0;
            root[2] = 0;
            root[3] = 0;
        }
        zero_root_masks(H, t, blockDim.x);
        __syncthreads();
    }
}

// Pool use of n trees after a voxelization, for a host that must not read
// the headers synchronously: out[3i] = overflow flags, out[3i+1] = node words
// used, out[3i+2] = tape words used.
__global__ void gather_usage_kernel(TreeHeader* const* trees, uint32_t n, unsigned long long* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const TreeHeader* H = trees[i];
    const uint32_t last = H->levels - 1;
    const uint32_t count = level_count(H, last, H->node_cap, H->node_size[last]);
    out[3 * i] = H->overflow;
    out[3 * i + 1] = H->node_ofs[last] + (unsigned long long)count * H->node_size[last];
    out[3 * i + 2] = min(H->tape_top, H->tape_cap);
}

// Work accounting (run on demand, outside the level passes): for every node of
// `level`, the op-weighted FP32 work of evaluating its tape on all its cells,
// with the interval weights (interior levels) or the point weights (last level).
__global__ void count_ops_kernel(TreeHeader* H, const uint32_t* nodes, const uint64_t* tapes,
                                 unsigned long long node_cap, uint32_t level, uint32_t node_size,
                                 uint32_t cells, int point, const uint32_t* skip) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t count = level_count(H, level, node_cap, node_size);
    const unsigned long long ofs = H->node_ofs[level];
    const uint8_t* wt = point ? kPointOps : kIntervalOps;
    unsigned long long sum = 0;
    for (uint32_t node = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); node < count;
         node += gridDim.x * (blockDim.x / 32)) {
        if (skip && skip[reuse_slot(ofs, node, node_size)] != 0xFFFFFFFFu) continue;
        const uint32_t tidx = nodes[ofs + (size_t)node * node_size];
        const uint32_t n = (uint32_t)tapes[tidx];
        uint32_t s = 0;
        for (uint32_t i = lane; i < n; i += 32) s += wt[w_op(tapes[tidx + 1 + i]) & 15];
        sum += (unsigned long long)s * cells;
    }
    for (int off = 16; off > 0; off >>= 1) sum += __shfl_down_sync(0xFFFFFFFFu, sum, off);
    if (lane == 0 && sum) atomicAdd(&H->fp32_ops[level], sum);
}

}  // namespace dev

namespace {

// The kernel's dynamic shared memory limit is raised to the device's opt-in
// maximum, never to this plan's size: plans are cached per tree and per batch,
// and a smaller limit set by a later plan would make an earlier plan's
// launches fail. The limit does not change occupancy; the launch's size does.
template <typename Kern>
cudaError_t occupancy(Kern kernel, int threads, size_t smem, int* blocks) {
    int dev = 0, sms = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (smem > (size_t)optin) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    *blocks = per_sm * sms;
    return cudaSuccess;
}

}  // namespace

// Cells per lane of the point pass: a node of dim^3 cells is dim^3 / (32 K)
// items, so K must divide the node's dim^3 / 32 mask words. With dim a
// multiple of 4 that count is even; it is a multiple of 4 when dim is a
// multiple of 8.
int point_k_for(uint32_t dim) { return dev::point_k_of(dim); }

template <int K>
static cudaError_t plan_point(uint32_t n_slots, LevelPlan* plan, int warps_hint) {
    const uint32_t pt = (uint32_t)(n_slots * 32 * 4 * K + (dev::STAGE + 1) * 16 + 15) / 16 * 16;
    plan->point_smem_per_warp = pt;
    plan->point_warps_per_block = 4ull * pt <= (warps_hint == 4 ? 227u : 200u) * 1024 && warps_hint != 1 ? 4 : 1;
    if (pt > 227 * 1024) return cudaErrorInvalidValue;
    if (plan->point_warps_per_block == 4)
        return occupancy(dev::point_level_kernel<4, K>, 128, 4 * pt, &plan->point_blocks);
    return occupancy(dev::point_level_kernel<1, K>, 32, pt, &plan->point_blocks);
}

template <int KI>
static cudaError_t plan_interval(bool four, int rounding, uint32_t iv, LevelPlan* plan) {
    if (rounding == 2)
        return four ? occupancy(dev::interval_level_kernel<2, 4, 1>, 128, 4 * iv, &plan->blocks)
                    : occupancy(dev::interval_level_kernel<2, 1, 1>, 32, iv, &plan->blocks);
    if (four)
        return rounding ? occupancy(dev::interval_level_kernel<1, 4, KI>, 128, 4 * iv, &plan->blocks)
                        : occupancy(dev::interval_level_kernel<0, 4, KI>, 128, 4 * iv, &plan->blocks);
    return rounding ? occupancy(dev::interval_level_kernel<1, 1, KI>, 32, iv, &plan->blocks)
                    : occupancy(dev::interval_level_kernel<0, 1, KI>, 32, iv, &plan->blocks);
}

cudaError_t plan_levels(uint32_t n_slots, uint32_t mm_cap, int point_k, int rounding, LevelPlan* plan,
                        int interval_warps, int point_warps, int interval_ki) {
    (void)mm_cap;  // the choice masks live in global scratch
    // Two cells per lane halve the dispatch work per cell but double a warp's
    // slot rows: by default only while 16 warps still fit in an SM's shared
    // memory (up to ~23 slots). Measured: the 23-slot 2048^3 scene's level-1
    // pass 8.8 ms with two vs 9.5 ms with one; the 28-slot batch (13 warps
    // with two) 106 vs 90 ms.
    const auto iv_bytes = [&](uint32_t k) {
        return (n_slots * 256 * k + (dev::STAGE + 1) * 16 + n_slots * 4 * k + 15) / 16 * 16;
    };
    // The hybrid affine mode: one cell per lane, 32-byte slot rows (four
    // times an interval's).
    const int ki = rounding == 2 ? 1
                                 : (interval_ki == 1 || interval_ki == 2 ? interval_ki
                                                                         : (16 * iv_bytes(2) <= 227 * 1024 ? 2 : 1));
    plan->interval_ki = ki;
    const uint32_t iv = rounding == 2 ? iv_bytes(4) : iv_bytes((uint32_t)ki);
    plan->smem_per_warp = iv;
    // Four warps (four tapes) per block when they fit in shared memory, else
    // one; a hint of 1 or 4 overrides the choice where shared memory allows.
    const bool four = 4ull * iv <= (interval_warps == 4 ? 227u : 200u) * 1024 && interval_warps != 1;
    plan->warps_per_block = four ? 4 : 1;
    if (!four && iv > 227 * 1024) return cudaErrorInvalidValue;
    // Both cell widths may run with this plan's shared memory (a level-0 pass
    // takes one cell per lane): raise both kernels' limits, then size the grid
    // for the planned width.
    cudaError_t e = ki == 2 ? plan_interval<1>(four, rounding, iv, plan) : plan_interval<2>(four, rounding, iv, plan);
    if (e == cudaSuccess)
        e = ki == 2 ? plan_interval<2>(four, rounding, iv, plan) : plan_interval<1>(four, rounding, iv, plan);
    if (e != cudaSuccess) return e;
    plan->point_k = point_k;
    if (point_k == 8) return plan_point<8>(n_slots, plan, point_warps);
    return point_k == 4 ? plan_point<4>(n_slots, plan, point_warps) : plan_point<2>(n_slots, plan, point_warps);
}

cudaError_t launch_tree_init(dev::TreeHeader* const* trees, uint32_t n, const float* tape_times, float tape_time,
                             cudaStream_t stream) {
    const uint32_t blocks = n < 4096 ? n : 4096;
    dev::tree_init_kernel<<<blocks, 32, 0, stream>>>(trees, n, tape_times, tape_time);
    return cudaGetLastError();
}

cudaError_t launch_tree_init_staged(dev::TreeHeader* const* trees, uint32_t n, const uint64_t* staged,
                                    const unsigned long long* offsets, const float* tape_times,
                                    cudaStream_t stream) {
    const uint32_t blocks = n < 4096 ? n : 4096;
    dev::tree_init_staged_kernel<<<blocks, 256, 0, stream>>>(trees, n, staged, offsets, tape_times);
    return cudaGetLastError();
}

cudaError_t launch_level_scan(const LevelLaunch& a, bool point, int point_k, cudaStream_t stream) {
    dev::level_scan_kernel<<<1, 1024, 0, stream>>>(a.trees, a.n_trees, a.level, point ? 1 : 0, point_k, a.prefix,
                                                   a.cursor, a.eval_list ? 1 : 0, a.any_point_k ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_level(const LevelLaunch& a, const LevelPlan& plan, int rounding, bool point,
                         cudaStream_t stream, int interval_ki) {
    if (point) {
        LevelLaunch b = a;
        b.smem_per_warp = plan.point_smem_per_warp;
        const int w4 = plan.point_warps_per_block == 4;
        const size_t smem = (size_t)plan.point_warps_per_block * plan.point_smem_per_warp;
        if (plan.point_k == 8) {
            if (w4) dev::point_level_kernel<4, 8><<<plan.point_blocks, 128, smem, stream>>>(b);
            else dev::point_level_kernel<1, 8><<<plan.point_blocks, 32, smem, stream>>>(b);
        } else if (plan.point_k == 4) {
            if (w4) dev::point_level_kernel<4, 4><<<plan.point_blocks, 128, smem, stream>>>(b);
            else dev::point_level_kernel<1, 4><<<plan.point_blocks, 32, smem, stream>>>(b);
        } else {
            if (w4) dev::point_level_kernel<4, 2><<<plan.point_blocks, 128, smem, stream>>>(b);
            else dev::point_level_kernel<1, 2><<<plan.point_blocks, 32, smem, stream>>>(b);
        }
        return cudaGetLastError();
    }
    LevelLaunch b = a;
    b.smem_per_warp = plan.smem_per_warp;
    const int w = plan.warps_per_block;
    const size_t smem = (size_t)w * plan.smem_per_warp;
    const int tpb = 32 * w;
#define FREP_IV_LAUNCH(R, W, KI) dev::interval_level_kernel<R, W, KI><<<plan.blocks, tpb, smem, stream>>>(b)
    if (rounding == 2) {
        if (w == 4) FREP_IV_LAUNCH(2, 4, 1);
        else FREP_IV_LAUNCH(2, 1, 1);
    } else if ((interval_ki ? interval_ki : plan.interval_ki) == 2) {
        if (w == 4) {
            if (rounding) FREP_IV_LAUNCH(1, 4, 2);
            else FREP_IV_LAUNCH(0, 4, 2);
        } else {
            if (rounding) FREP_IV_LAUNCH(1, 1, 2);
            else FREP_IV_LAUNCH(0, 1, 2);
        }
    } else {
        if (w == 4) {
            if (rounding) FREP_IV_LAUNCH(1, 4, 1);
            else FREP_IV_LAUNCH(0, 4, 1);
        } else {
            if (rounding) FREP_IV_LAUNCH(1, 1, 1);
            else FREP_IV_LAUNCH(0, 1, 1);
        }
    }
#undef FREP_IV_LAUNCH
    return cudaGetLastError();
}

cudaError_t launch_gather_usage(dev::TreeHeader* const* trees, uint32_t n, unsigned long long* out,
                                cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    dev::gather_usage_kernel<<<(n + 127) / 128, 128, 0, stream>>>(trees, n, out);
    return cudaGetLastError();
}

cudaError_t launch_count_ops(dev::TreeHeader* hdr, const uint32_t* nodes, const uint64_t* tapes,
                             unsigned long long node_cap, uint32_t level, uint32_t node_size,
                             uint32_t cells, bool point, const uint32_t* skip, cudaStream_t stream) {
    dev::count_ops_kernel<<<1184, 256, 0, stream>>>(hdr, nodes, tapes, node_cap, level, node_size, cells,
                                                    point ? 1 : 0, skip);
    return cudaGetLastError();
}

}  // namespace frep
