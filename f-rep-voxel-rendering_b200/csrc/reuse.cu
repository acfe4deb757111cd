// Re-voxelization with reuse of the previous frame's tree (animated scenes).
//
// The reference re-voxelizes the whole tree every frame when the shape
// depends on time (application.cpp:68-79: Voxelize(sem, Timer::s_time)); the
// time input is tape slot 3, [T, T] (interval.comp:128, point.comp:6). A
// node's subtree is a function of its tape, its coordinates and the grid
// alone when that tape never reads slot 3's initial value; shortening only
// drops instructions, so every tape below such a node is time-free as well.
// Such a subtree is copied from the previous tree when that tree has a node at
// the same level and coordinates with a bit-identical tape, instead of being
// evaluated again. The result is the tree a full voxelization would build
// (the same nodes, masks and tape contents; node ids, as always, differ).
//
// Per level L of the new tree (one tree per launch):
//   reuse_match_kernel  every node of L created by an evaluated parent: find
//                       the previous tree's node at the same coordinates (a
//                       descent from its root) and compare tapes; the side
//                       array entry becomes that node's id, or ~0;
//                       nodes left to evaluate are listed for the level pass;
//   level pass          evaluates the listed nodes (entry ~0);
//   reuse_copy_kernel   the nodes whose entry is set: masks from the previous
//                       node; each interior cell gets a new child whose tape is
//                       copied (tapes shared within a 32-cell group stay
//                       shared) and whose entry is the previous child, so the
//                       next level copies it in turn.
#include <cstdint>

#include "device_common.cuh"
#include "kernels.h"

namespace frep {
namespace dev {

namespace {

constexpr uint32_t NONE = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t lanemask_lt_r() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// The previous tree's node of level L at coordinates (gx, gy, gz) (in cells of
// level L-1), by descent from its root; NONE if that cell is not interior
// there. Warp-uniform.
__device__ uint32_t prev_node_at(const TreeHeader* P, uint32_t L, uint32_t gx, uint32_t gy, uint32_t gz) {
    uint32_t pn = 0;
    for (uint32_t k = 0; k < L; k++) {
        uint32_t span = 1;  // cells of level L-1 per cell of level k
        for (uint32_t j = k + 1; j < L; j++) span *= P->dims[j];
        const uint32_t dim = P->dims[k];
        const uint32_t cx = (gx / span) % dim, cy = (gy / span) % dim, cz = (gz / span) % dim;
        const uint32_t cell = (cx * dim + cy) * dim + cz;
        const uint32_t words = dim * dim * dim / 32;
        if (pn >= level_count(P, k, P->node_cap, P->node_size[k])) return NONE;
        const uint32_t* rec = P->nodes + P->node_ofs[k] + (size_t)pn * P->node_size[k];
        if (!((__ldcg(&rec[4 + words + (cell >> 5)]) >> (cell & 31)) & 1u)) return NONE;
        pn = __ldcg(&rec[4 + 2 * words + cell]);
    }
    if (pn >= level_count(P, L, P->node_cap, P->node_size[L])) return NONE;
    return pn;
}

// True when the tapes at a (pool A) and b (pool B) are identical and never
// read slot 3 (the time) before writing it. Warp-uniform.
__device__ bool same_time_free_tape(const uint64_t* A, uint32_t a, const uint64_t* B, uint32_t b, uint32_t lane) {
    const uint64_t ha = __ldcg(&A[a]), hb = __ldcg(&B[b]);
    if (ha != hb) return false;
    const uint32_t n = (uint32_t)ha;
    bool time_live = true;  // slot 3 still holds the time
    for (uint32_t base = 0; base < n; base += 32) {
        const uint32_t i = base + lane;
        const bool valid = i < n;
        const uint64_t wa = valid ? __ldcg(&A[a + 1 + i]) : 0ull;
        const uint64_t wb = valid ? __ldcg(&B[b + 1 + i]) : 0ull;
        if (__any_sync(0xFFFFFFFFu, wa != wb)) return false;
        if (time_live) {
            const uint32_t op = w_op(wa);
            const bool reads = valid && op != OP_CONST && (w_a(wa) == 3u || (is_binary(op) && w_b(wa) == 3u));
            const uint32_t writes = __ballot_sync(0xFFFFFFFFu, valid && w_out(wa) == 3u);
            uint32_t rd = __ballot_sync(0xFFFFFFFFu, reads);
            if (writes) {
                const uint32_t first = __ffs(writes) - 1;  // reads up to and including it see the time
                rd &= first == 31 ? 0xFFFFFFFFu : (2u << first) - 1u;
                time_live = false;
            }
            if (rd) return false;
        }
    }
    return true;
}

}  // namespace

// Side-array entries of every node of level L present now (children of
// evaluated parents; the root for L = 0).
__global__ void __launch_bounds__(128) reuse_match_kernel(TreeHeader* H, const TreeHeader* P, uint32_t* src,
                                                          uint32_t* list, uint32_t L) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t count = level_count(H, L, H->node_cap, H->node_size[L]);
    const unsigned long long ofs = H->node_ofs[L];
    const uint32_t size = H->node_size[L];
    const bool prev_ok = P->overflow == 0u && P->levels == H->levels;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t node = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); node < count; node += warps) {
        const uint32_t* rec = H->nodes + ofs + (size_t)node * size;
        uint32_t from = NONE;
        if (prev_ok) {
            const uint32_t tidx = rec[0], gx = rec[1], gy = rec[2], gz = rec[3];
            const uint32_t pn = prev_node_at(P, L, gx, gy, gz);
            if (pn != NONE) {
                const uint32_t* prec = P->nodes + P->node_ofs[L] + (size_t)pn * P->node_size[L];
                if (__ldcg(&prec[1]) == gx && __ldcg(&prec[2]) == gy && __ldcg(&prec[3]) == gz &&
                    same_time_free_tape(H->tapes, tidx, P->tapes, __ldcg(&prec[0]), lane))
                    from = pn;
            }
        }
        if (lane == 0) {
            src[reuse_slot(ofs, node, size)] = from;
            if (from == NONE) list[atomicAdd(&H->reuse_eval[L], 1u)] = node;  // to evaluate
        }
    }
}

// Copies the nodes of level L whose entry is set from the previous tree:
// masks, and (below the last level) new children with copied tapes, whose
// entries are set to the previous children. Last level: a warp per node (its
// leaf words). Above: a warp per 32-cell group of a node (one leaf word, one
// interior word, 32 child slots), so that a level of few large nodes still
// spreads over the whole GPU.
__global__ void __launch_bounds__(128) reuse_copy_kernel(TreeHeader* H, const TreeHeader* P, uint32_t* src,
                                                         uint32_t L) {
    const uint32_t lane = threadIdx.x & 31;
    const bool last = L == H->levels - 1;
    const uint32_t count = level_count(H, L, H->node_cap, H->node_size[L]);
    const unsigned long long ofs = H->node_ofs[L];
    const uint32_t size = H->node_size[L];
    const uint32_t dim = H->dims[L];
    const uint32_t words = dim * dim * dim / 32;
    const unsigned long long pofs = P->node_ofs[L];
    const uint32_t psize = P->node_size[L];
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    const uint32_t warp0 = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (last) {
        for (uint32_t node = warp0; node < count; node += warps) {
            const uint32_t from = __ldcg(&src[reuse_slot(ofs, node, size)]);
            if (from == NONE) continue;
            uint32_t* rec = H->nodes + ofs + (size_t)node * size;
            const uint32_t* prec = P->nodes + pofs + (size_t)from * psize;
            for (uint32_t w = lane; w < 2 * words; w += 32) rec[4 + w] = __ldcg(&prec[4 + w]);
        }
        return;
    }
    const unsigned long long ofs_next = H->node_ofs[L + 1];
    const uint32_t size_next = H->node_size[L + 1];
    const unsigned long long child_cap = H->node_cap > ofs_next ? (H->node_cap - ofs_next) / size_next : 0ull;
    const unsigned long long pofs_next = P->node_ofs[L + 1];
    const uint32_t psize_next = P->node_size[L + 1];
    const uint32_t pcount_next = level_count(P, L + 1, P->node_cap, P->node_size[L + 1]);
    unsigned long long stat_sum = 0;
    uint32_t stat_max = 0;
    const unsigned long long items = (unsigned long long)count * words;
    for (unsigned long long item = warp0; item < items; item += warps) {
        const uint32_t node = (uint32_t)(item / words), grp = (uint32_t)(item % words);
        const uint32_t from = __ldcg(&src[reuse_slot(ofs, node, size)]);
        if (from == NONE) continue;
        uint32_t* rec = H->nodes + ofs + (size_t)node * size;
        const uint32_t* prec = P->nodes + pofs + (size_t)from * psize;
        const uint32_t own_tape = rec[0];
        const uint32_t prev_own = __ldcg(&prec[0]);
        const uint32_t own_len = (uint32_t)__ldcg(&H->tapes[own_tape]);
        const uint32_t cell = grp * 32 + lane;
        const uint32_t inter_w = __ldcg(&prec[4 + words + grp]);
        const bool inter = (inter_w >> lane) & 1u;
        const uint32_t pch = inter ? __ldcg(&prec[4 + 2 * words + cell]) : NONE;
        const bool have = inter && pch < pcount_next;
        const uint32_t amb_w = __ballot_sync(0xFFFFFFFFu, have);
        unsigned long long base = 0;
        if (amb_w) {
            if (lane == 0) base = atomicAdd(&H->node_count[L + 1], (uint32_t)__popc(amb_w));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
        }
        const unsigned long long mine = base + __popc(amb_w & lanemask_lt_r());
        const bool ok = have && mine < child_cap;
        const uint32_t ok_w = __ballot_sync(0xFFFFFFFFu, ok);
        if (lane == 0) {
            rec[4 + grp] = __ldcg(&prec[4 + grp]);  // leaf word
            rec[4 + words + grp] = ok_w;
            // a child that did not fit (or a previous child id out of range)
            if (ok_w != inter_w) atomicOr(&H->overflow, 1u);
        }
        rec[4 + 2 * words + cell] = ok ? (uint32_t)mine : NONE;
        if (!ok_w) continue;

        // the child's tape: its parent's own (not shortened), or a copy of the
        // previous child's, one copy per distinct tape of the group
        const uint32_t* pcrec = P->nodes + pofs_next + (size_t)(ok ? pch : 0u) * psize_next;
        const uint32_t ptape = ok ? __ldcg(&pcrec[0]) : 0u;
        const bool need = ok && ptape != prev_own;
        const uint32_t plen = need ? (uint32_t)__ldcg(&P->tapes[ptape]) : own_len;
        const unsigned long long key = need ? (unsigned long long)ptape : (1ull << 32) + lane;
        const uint32_t groupm = __match_any_sync(0xFFFFFFFFu, key);
        const uint32_t leader = __ffs(groupm) - 1;
        const bool lead = need && leader == lane;
        const uint32_t tw = lead ? (1u + plen + TAPE_ALIGN_WORDS - 1) / TAPE_ALIGN_WORDS * TAPE_ALIGN_WORDS : 0u;
        uint32_t incl = tw;
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
            if ((int)lane >= off) incl += v;
        }
        const uint32_t total = __shfl_sync(0xFFFFFFFFu, incl, 31);
        unsigned long long tbase = 0;
        if (total) {
            if (lane == 0) tbase = atomicAdd(&H->tape_top, (unsigned long long)total);
            tbase = __shfl_sync(0xFFFFFFFFu, tbase, 0);
        }
        const unsigned long long my_t = tbase + (incl - tw);
        const bool t_ok = lead && my_t + tw <= H->tape_cap;
        if (lead && !t_ok) atomicOr(&H->overflow, 2u);
        const uint32_t written = __ballot_sync(0xFFFFFFFFu, t_ok);
        uint32_t pending = written;
        while (pending) {  // copy the leaders' records, one per pass, coalesced
            const int sel = __ffs(pending) - 1;
            pending &= pending - 1;
            const unsigned long long d = __shfl_sync(0xFFFFFFFFu, my_t, sel);
            const uint32_t s = __shfl_sync(0xFFFFFFFFu, ptape, sel);
            const uint32_t nw = 1u + __shfl_sync(0xFFFFFFFFu, plen, sel);
            for (uint32_t w = lane; w < nw; w += 32) H->tapes[d + w] = __ldcg(&P->tapes[s + w]);
        }
        const unsigned long long lt = __shfl_sync(0xFFFFFFFFu, my_t, leader);
        if (ok) {
            const bool copied = need && ((written >> leader) & 1u);
            uint32_t* crec = H->nodes + ofs_next + mine * size_next;
            crec[0] = copied ? (uint32_t)lt : own_tape;
            crec[1] = __ldcg(&pcrec[1]);
            crec[2] = __ldcg(&pcrec[2]);
            crec[3] = __ldcg(&pcrec[3]);
            src[reuse_slot(ofs_next, (uint32_t)mine, size_next)] = pch;
            const uint32_t len = copied ? plen : own_len;
            stat_sum += len;
            stat_max = max(stat_max, len);
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        stat_sum += __shfl_down_sync(0xFFFFFFFFu, stat_sum, off);
        stat_max = max(stat_max, __shfl_down_sync(0xFFFFFFFFu, stat_max, off));
    }
    if (lane == 0) {
        if (stat_sum) atomicAdd(&H->tape_size_sum[L + 1], stat_sum);
        if (stat_max) atomicMax(&H->tape_size_max[L + 1], stat_max);
    }
}

}  // namespace dev

static uint32_t reuse_blocks() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (uint32_t)(sms > 0 ? sms : 1) * 8u;
}

cudaError_t launch_reuse_match(dev::TreeHeader* hdr, const dev::TreeHeader* prev, uint32_t* src, uint32_t* list,
                               uint32_t level, cudaStream_t stream) {
    dev::reuse_match_kernel<<<reuse_blocks(), 128, 0, stream>>>(hdr, prev, src, list, level);
    return cudaGetLastError();
}

cudaError_t launch_reuse_copy(dev::TreeHeader* hdr, const dev::TreeHeader* prev, uint32_t* src, uint32_t level,
                              cudaStream_t stream) {
    dev::reuse_copy_kernel<<<reuse_blocks(), 128, 0, stream>>>(hdr, prev, src, level);
    return cudaGetLastError();
}

}  // namespace frep
