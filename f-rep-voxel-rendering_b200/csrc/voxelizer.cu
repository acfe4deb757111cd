// Level passes of the sparse-tree voxelizer (sm_100a).
//
// Replaces vulkan/shaders/voxelizer/main.comp + tape/interval.comp +
// tape/shorten.comp + tape/point.comp and the host level loop of
// vulkan/src/engine/voxelizer.cpp:295-329, :429-440.
//
// Work decomposition: one WARP owns one work item = (node, 32 cells that form
// one word of the node's masks, in bit-index order z + dim*y + dim^2*x). All
// 32 lanes follow the same tape, so the opcode stream is warp-uniform:
//   * the tape is staged through shared memory 32 instructions at a time
//     (one coalesced 256-byte load per chunk, then broadcast reads);
//   * the slot file lives in shared memory as [slot][lane] float2 (interval) or
//     float (point) — conflict-free 8/4-byte accesses;
//   * MIN/MAX choices are kept as two 32-bit ballots per MIN/MAX instruction;
//   * leaf / interior mask words are written whole from ballots (no atomics);
//   * children are claimed with one warp-aggregated atomic per item, tapes with
//     one more; shortened tapes are written cooperatively by the warp, one
//     coalesced 256-byte store per 32 input instructions.
// Items are fetched in chunks from a device counter, so a level pass needs no
// host round trip: the node count of level l is read on the device.
#include "device_common.cuh"
#include "kernels.h"

namespace frep {
namespace dev {

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

__device__ __forceinline__ uint32_t level_count(const TreeHeader* H, uint32_t level,
                                                unsigned long long node_cap, uint32_t node_size) {
    // A pool overflow in the previous level may have counted children that
    // were never written; only the ones that fit exist.
    const unsigned long long ofs = H->node_ofs[level];
    const unsigned long long cap = node_cap > ofs ? (node_cap - ofs) / node_size : 0;
    return (uint32_t)min((unsigned long long)H->node_count[level], cap);
}

template <int ROUND, int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
interval_level_kernel(LevelArgs p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* wbase = smem + (size_t)warp * p.smem_per_warp;
    float2* slots = reinterpret_cast<float2*>(wbase);
    uint64_t* stage = reinterpret_cast<uint64_t*>(wbase + (size_t)p.n_slots * 256);
    uint2* mmb = reinterpret_cast<uint2*>(wbase + (size_t)p.n_slots * 256 + 256);
    uint32_t* live = reinterpret_cast<uint32_t*>(wbase + (size_t)p.n_slots * 256 + 256 + (size_t)p.mm_cap * 8);
    const uint32_t live_words = (p.n_slots + 31) / 32;

    TreeHeader* H = p.hdr;
    const uint32_t L = p.level;
    const uint32_t dim = p.dim;
    const uint32_t groups = dim * dim * dim / 32;
    const uint32_t count = level_count(H, L, p.node_cap, p.node_size);
    const unsigned long long ofs_l = H->node_ofs[L];
    const unsigned long long ofs_next = ofs_l + (unsigned long long)count * p.node_size;
    if (blockIdx.x == 0 && threadIdx.x == 0) H->node_ofs[L + 1] = ofs_next;
    const unsigned long long child_cap =
        p.node_cap > ofs_next ? (p.node_cap - ofs_next) / p.node_size_next : 0ull;
    const unsigned long long total = (unsigned long long)count * groups;
    const uint32_t grid_warps = gridDim.x * WARPS;
    const uint32_t chunk = chunk_for(total, grid_warps);
    uint32_t* keep = p.keep_scratch + (size_t)(blockIdx.x * WARPS + warp) * p.keep_stride;
    const float cs = p.cell_size;

    unsigned long long stat_sum = 0, stat_work = 0;
    uint32_t stat_max = 0;

    unsigned long long first;
    uint32_t got;
    while ((got = fetch_items(&H->work_cursor[L], total, chunk, &first)) != 0) {
        for (uint32_t it = 0; it < got; it++) {
            const unsigned long long item = first + it;
            const uint32_t node = (uint32_t)(item / groups), grp = (uint32_t)(item % groups);
            uint32_t* rec = p.nodes + ofs_l + (size_t)node * p.node_size;
            const uint32_t tape_idx = rec[0];
            const uint32_t ncx = rec[1], ncy = rec[2], ncz = rec[3];
            const uint64_t* tape = p.tapes + tape_idx + 1;
            const uint32_t n = (uint32_t)p.tapes[tape_idx];

            const uint32_t cell = grp * 32 + lane;
            const uint32_t cz = cell % dim, cy = (cell / dim) % dim, cx = cell / (dim * dim);
            const uint32_t gx = ncx * dim + cx, gy = ncy * dim + cy, gz = ncz * dim + cz;
            // voxelizer/main.comp:113-116, :124-126
            const float lox = __fadd_rn(p.low[0], __fmul_rn((float)gx, cs));
            const float loy = __fadd_rn(p.low[1], __fmul_rn((float)gy, cs));
            const float loz = __fadd_rn(p.low[2], __fmul_rn((float)gz, cs));
            slots[0 * 32 + lane] = make_float2(lox, __fadd_rn(lox, cs));
            slots[1 * 32 + lane] = make_float2(loy, __fadd_rn(loy, cs));
            slots[2 * 32 + lane] = make_float2(loz, __fadd_rn(loz, cs));
            slots[3 * 32 + lane] = make_float2(p.tape_time, p.tape_time);

            // ---- forward interval pass (interval.comp:121-160) ----
            uint32_t mm = 0;
            for (uint32_t base = 0; base < n; base += 32) {
                const uint32_t m = min(32u, n - base);
                __syncwarp();
                if (lane < m) stage[lane] = tape[base + lane];
                __syncwarp();
                for (uint32_t j = 0; j < m; j++) {
                    const uint64_t w = stage[j];
                    const uint32_t op = w_op(w);
                    float2 a = make_float2(0.0f, 0.0f), b = a;
                    if (op != OP_CONST) {
                        a = slots[w_a(w) * 32 + lane];
                        b = slots[w_b(w) * 32 + lane];
                    }
                    slots[w_out(w) * 32 + lane] = iv_apply<ROUND>(op, w, a, b);
                    if (is_mm(op)) {
                        uint32_t c;
                        if (op == OP_MIN) c = a.y < b.x ? MM_FIRST : (b.y < a.x ? MM_SECOND : MM_BOTH);
                        else c = a.y < b.x ? MM_SECOND : (b.y < a.x ? MM_FIRST : MM_BOTH);
                        const uint32_t b0 = __ballot_sync(0xFFFFFFFFu, c & 1u);
                        const uint32_t b1 = __ballot_sync(0xFFFFFFFFu, c & 2u);
                        if (lane == 0 && mm < p.mm_cap) mmb[mm] = make_uint2(b0, b1);
                        mm++;
                    }
                }
            }
            __syncwarp();
            stat_work += 32ull * n;

            // ---- classification (voxelizer/main.comp:88-108) ----
            const float2 d = slots[lane];
            const bool empty = d.x > 0.0f;
            const bool leaf = !empty && d.y < 0.0f;
            const bool amb = !empty && !leaf;
            const uint32_t leaf_w = __ballot_sync(0xFFFFFFFFu, leaf);
            const uint32_t amb_w = __ballot_sync(0xFFFFFFFFu, amb);

            // ---- child allocation (main.comp:138-148), warp-aggregated ----
            const uint32_t n_amb = __popc(amb_w);
            unsigned long long child_base = 0;
            if (n_amb) {
                if (lane == 0) child_base = atomicAdd(&H->node_count[L + 1], n_amb);
                child_base = __shfl_sync(0xFFFFFFFFu, child_base, 0);
            }
            const unsigned long long my_child = child_base + __popc(amb_w & lanemask_lt());
            const bool ok = amb && my_child < child_cap;
            const uint32_t ok_w = __ballot_sync(0xFFFFFFFFu, ok);
            if (ok_w != amb_w && lane == 0) atomicOr(&H->overflow, 1u);

            uint32_t child_tape = tape_idx;
            uint32_t child_len = n;
            if (ok_w && p.shorten) {
                // ---- backward liveness (shorten.comp:148-186) ----
                for (uint32_t wd = 0; wd < live_words; wd++) live[wd * 32 + lane] = 0u;
                if (ok) live[lane] = 1u;  // slot 0 is the output
                uint32_t kept = 0;
                int mmi = (int)mm - 1;
                for (int hi = (int)n; hi > 0; hi -= 32) {
                    const int lo = max(0, hi - 32);
                    const int m = hi - lo;
                    __syncwarp();
                    if ((int)lane < m) stage[lane] = tape[lo + lane];
                    __syncwarp();
                    for (int j = m - 1; j >= 0; j--) {
                        const uint64_t w = stage[j];
                        const uint32_t op = w_op(w), o = w_out(w);
                        uint32_t* lw = &live[(o >> 5) * 32 + lane];
                        const uint32_t lv = *lw;
                        const bool k = (lv >> (o & 31)) & 1u;
                        if (k) {
                            *lw = lv & ~(1u << (o & 31));
                            uint32_t c;
                            if (op == OP_CONST) c = 0;
                            else if (op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_DIV) c = MM_BOTH;
                            else if (is_mm(op)) {
                                const uint2 cb = mmb[mmi];
                                c = ((cb.x >> lane) & 1u) | (((cb.y >> lane) & 1u) << 1);
                            } else c = MM_FIRST;
                            if (c & MM_FIRST) {
                                const uint32_t s = w_a(w);
                                live[(s >> 5) * 32 + lane] |= 1u << (s & 31);
                            }
                            if (c & MM_SECOND) {
                                const uint32_t s = w_b(w);
                                live[(s >> 5) * 32 + lane] |= 1u << (s & 31);
                            }
                            kept++;
                        }
                        const uint32_t kb = __ballot_sync(0xFFFFFFFFu, k);
                        if (lane == 0) keep[lo + j] = kb;
                        if (is_mm(op)) mmi--;
                    }
                }
                __syncwarp();

                // ---- claim output tapes (shorten.comp:136-142), one atomic per warp ----
                const bool do_short = ok && kept < n;  // "not shorter -> reuse" (:188-191)
                const uint32_t words = do_short ? (1 + kept + TAPE_ALIGN_WORDS - 1) / TAPE_ALIGN_WORDS * TAPE_ALIGN_WORDS : 0;
                uint32_t incl = words;
                for (int off = 1; off < 32; off <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xFFFFFFFFu, incl, off);
                    if ((int)lane >= off) incl += v;
                }
                const uint32_t total_words = __shfl_sync(0xFFFFFFFFu, incl, 31);
                unsigned long long tbase = 0;
                if (total_words) {
                    if (lane == 0) tbase = atomicAdd(&H->tape_top, (unsigned long long)total_words);
                    tbase = __shfl_sync(0xFFFFFFFFu, tbase, 0);
                }
                const unsigned long long my_tape = tbase + (incl - words);
                const bool tape_ok = do_short && my_tape + words <= p.tape_cap;
                if (do_short && !tape_ok) atomicOr(&H->overflow, 2u);
                const uint32_t short_w = __ballot_sync(0xFFFFFFFFu, tape_ok);

                // ---- cooperative copy of each shortened tape (shorten.comp:193-221) ----
                uint32_t pending = short_w;
                while (pending) {
                    const int sel = __ffs(pending) - 1;
                    pending &= pending - 1;
                    const unsigned long long dst = __shfl_sync(0xFFFFFFFFu, my_tape, sel);
                    const uint32_t ksz = __shfl_sync(0xFFFFFFFFu, kept, sel);
                    if (lane == 0) p.tapes[dst] = (uint64_t)ksz;
                    uint32_t run = 0, mm_run = 0;
                    for (uint32_t b = 0; b < n; b += 32) {
                        const uint32_t idx = b + lane;
                        const bool valid = idx < n;
                        uint64_t w = valid ? tape[idx] : 0ull;
                        const bool kb = valid && ((keep[idx] >> sel) & 1u);
                        const bool ism = valid && is_mm(w_op(w));
                        const uint32_t mball = __ballot_sync(0xFFFFFFFFu, ism);
                        if (kb && ism) {
                            const uint2 cb = mmb[mm_run + __popc(mball & lanemask_lt())];
                            const uint32_t c = ((cb.x >> sel) & 1u) | (((cb.y >> sel) & 1u) << 1);
                            if (c == MM_FIRST) {
                                w = (w & ~0xFFull) | OP_COPY;
                            } else if (c == MM_SECOND) {  // COPY of B; the B field is kept
                                w = (w & ~0xFFull & ~(0xFFFFull << 32)) | OP_COPY | ((uint64_t)w_b(w) << 32);
                            }
                        }
                        const uint32_t kball = __ballot_sync(0xFFFFFFFFu, kb);
                        if (kb) p.tapes[dst + 1 + run + __popc(kball & lanemask_lt())] = w;
                        run += __popc(kball);
                        mm_run += __popc(mball);
                    }
                }
                if (tape_ok) {
                    child_tape = (uint32_t)my_tape;
                    child_len = kept;
                }
            }

            // ---- node records: masks, child list, children ----
            if (ok) {
                uint32_t* crec = p.nodes + ofs_next + (size_t)my_child * p.node_size_next;
                crec[0] = child_tape;
                crec[1] = gx;
                crec[2] = gy;
                crec[3] = gz;
            }
            rec[4 + 2 * groups + cell] = ok ? (uint32_t)my_child : 0xFFFFFFFFu;
            if (lane == 0) {
                rec[4 + grp] = leaf_w;
                rec[4 + groups + grp] = ok_w;
            }
            if (ok) {
                stat_sum += child_len;
                stat_max = max(stat_max, child_len);
            }
        }
    }

    // Per-warp statistics, flushed once (stats_buf of main.comp:146-147).
    for (int off = 16; off > 0; off >>= 1) {
        stat_sum += __shfl_down_sync(0xFFFFFFFFu, stat_sum, off);
        stat_max = max(stat_max, __shfl_down_sync(0xFFFFFFFFu, stat_max, off));
    }
    if (lane == 0) {
        if (stat_sum) atomicAdd(&H->tape_size_sum[L + 1], stat_sum);
        if (stat_max) atomicMax(&H->tape_size_max[L + 1], stat_max);
        if (stat_work) atomicAdd(&H->cell_instr[L], stat_work);
    }
}

// Last level: the leaf bit is the sign of the point value at the cell's low
// corner (voxelize_point, main.comp:74-83; tape_eval_point, point.comp:2-63).
template <int WARPS>
__global__ void __launch_bounds__(WARPS * 32)
point_level_kernel(LevelArgs p) {
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned char* wbase = smem + (size_t)warp * p.smem_per_warp;
    float* slots = reinterpret_cast<float*>(wbase);
    uint64_t* stage = reinterpret_cast<uint64_t*>(wbase + (size_t)p.n_slots * 128);

    TreeHeader* H = p.hdr;
    const uint32_t L = p.level;
    const uint32_t dim = p.dim;
    const uint32_t groups = dim * dim * dim / 32;
    const uint32_t count = level_count(H, L, p.node_cap, p.node_size);
    const unsigned long long ofs_l = H->node_ofs[L];
    const unsigned long long total = (unsigned long long)count * groups;
    const uint32_t chunk = chunk_for(total, gridDim.x * WARPS);
    const float cs = p.cell_size;
    unsigned long long stat_work = 0;

    unsigned long long first;
    uint32_t got;
    while ((got = fetch_items(&H->work_cursor[L], total, chunk, &first)) != 0) {
        for (uint32_t it = 0; it < got; it++) {
            const unsigned long long item = first + it;
            const uint32_t node = (uint32_t)(item / groups), grp = (uint32_t)(item % groups);
            uint32_t* rec = p.nodes + ofs_l + (size_t)node * p.node_size;
            const uint32_t tape_idx = rec[0];
            const uint64_t* tape = p.tapes + tape_idx + 1;
            const uint32_t n = (uint32_t)p.tapes[tape_idx];
            const uint32_t cell = grp * 32 + lane;
            const uint32_t cz = cell % dim, cy = (cell / dim) % dim, cx = cell / (dim * dim);
            const uint32_t gx = rec[1] * dim + cx, gy = rec[2] * dim + cy, gz = rec[3] * dim + cz;
            slots[0 * 32 + lane] = __fadd_rn(p.low[0], __fmul_rn((float)gx, cs));
            slots[1 * 32 + lane] = __fadd_rn(p.low[1], __fmul_rn((float)gy, cs));
            slots[2 * 32 + lane] = __fadd_rn(p.low[2], __fmul_rn((float)gz, cs));
            slots[3 * 32 + lane] = p.tape_time;
            for (uint32_t base = 0; base < n; base += 32) {
                const uint32_t m = min(32u, n - base);
                __syncwarp();
                if (lane < m) stage[lane] = tape[base + lane];
                __syncwarp();
                for (uint32_t j = 0; j < m; j++) {
                    const uint64_t w = stage[j];
                    const uint32_t op = w_op(w);
                    float a = 0.0f, b = 0.0f;
                    if (op != OP_CONST) {
                        a = slots[w_a(w) * 32 + lane];
                        b = slots[w_b(w) * 32 + lane];
                    }
                    slots[w_out(w) * 32 + lane] = pt_apply(op, w, a, b);
                }
            }
            __syncwarp();
            stat_work += 32ull * n;
            const uint32_t leaf_w = __ballot_sync(0xFFFFFFFFu, slots[lane] < 0.0f);
            if (lane == 0) {
                rec[4 + grp] = leaf_w;
                rec[4 + groups + grp] = 0u;  // the unused second mask word range
            }
        }
    }
    // stat_work is warp-uniform: lane 0 reports it.
    if (lane == 0 && stat_work) atomicAdd(&H->cell_instr[L], stat_work);
}

// Resets the header and writes the root node (Voxelizer::Voxelize sets
// interiorNodeCount[0] = 1 and relies on a zeroed root, voxelizer.cpp:432-435).
__global__ void tree_init_kernel(TreeHeader* H, uint32_t* nodes, uint32_t root_n, uint32_t root_words) {
    const uint32_t t = threadIdx.x;
    for (uint32_t l = t; l < MAX_LEVELS; l += blockDim.x) {
        H->node_count[l] = l == 0 ? 1u : 0u;
        H->work_cursor[l] = 0;
        H->node_ofs[l] = 0;
        H->tape_size_sum[l] = l == 0 ? root_n : 0;
        H->tape_size_max[l] = l == 0 ? root_n : 0;
        H->cell_instr[l] = 0;
    }
    if (t == 0) {
        H->tape_top = root_words;
        H->overflow = 0;
        H->status = 0;
        nodes[0] = 0;  // root tape at word 0 of the tape pool
        nodes[1] = 0;
        nodes[2] = 0;
        nodes[3] = 0;
    }
}

}  // namespace dev

namespace {

template <typename K>
cudaError_t occupancy(K kernel, int threads, size_t smem, int* blocks) {
    cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    *blocks = per_sm * sms;
    return cudaSuccess;
}

}  // namespace

cudaError_t plan_levels(uint32_t n_slots, uint32_t mm_cap, int rounding, LevelPlan* plan) {
    const uint32_t live_words = (n_slots + 31) / 32;
    const uint32_t iv = (n_slots * 256 + 256 + mm_cap * 8 + live_words * 128 + 15) / 16 * 16;
    const uint32_t pt = (n_slots * 128 + 256 + 15) / 16 * 16;
    plan->smem_per_warp = iv;
    plan->point_smem_per_warp = pt;
    // Four warps per block when they fit in shared memory, else one.
    const bool four = 4ull * iv <= 200 * 1024;
    plan->warps_per_block = four ? 4 : 1;
    if (!four && iv > 227 * 1024) return cudaErrorInvalidValue;
    cudaError_t e;
    if (four) {
        e = rounding ? occupancy(dev::interval_level_kernel<1, 4>, 128, 4 * iv, &plan->blocks)
                     : occupancy(dev::interval_level_kernel<0, 4>, 128, 4 * iv, &plan->blocks);
    } else {
        e = rounding ? occupancy(dev::interval_level_kernel<1, 1>, 32, iv, &plan->blocks)
                     : occupancy(dev::interval_level_kernel<0, 1>, 32, iv, &plan->blocks);
    }
    if (e != cudaSuccess) return e;
    plan->point_warps_per_block = 4ull * pt <= 200 * 1024 ? 4 : 1;
    if (pt > 227 * 1024) return cudaErrorInvalidValue;
    if (plan->point_warps_per_block == 4)
        return occupancy(dev::point_level_kernel<4>, 128, 4 * pt, &plan->point_blocks);
    return occupancy(dev::point_level_kernel<1>, 32, pt, &plan->point_blocks);
}

cudaError_t launch_tree_init(dev::TreeHeader* hdr, uint32_t* nodes, uint32_t root_n_instr,
                             uint32_t root_words, cudaStream_t stream) {
    dev::tree_init_kernel<<<1, 32, 0, stream>>>(hdr, nodes, root_n_instr, root_words);
    return cudaGetLastError();
}

cudaError_t launch_level(const LevelArgs& a, const LevelPlan& plan, int rounding, bool last,
                         cudaStream_t stream) {
    if (last) {
        LevelArgs b = a;
        b.smem_per_warp = plan.point_smem_per_warp;
        if (plan.point_warps_per_block == 4)
            dev::point_level_kernel<4><<<plan.point_blocks, 128, 4 * plan.point_smem_per_warp, stream>>>(b);
        else
            dev::point_level_kernel<1><<<plan.point_blocks, 32, plan.point_smem_per_warp, stream>>>(b);
        return cudaGetLastError();
    }
    LevelArgs b = a;
    b.smem_per_warp = plan.smem_per_warp;
    const int w = plan.warps_per_block;
    const size_t smem = (size_t)w * plan.smem_per_warp;
    if (w == 4) {
        if (rounding) dev::interval_level_kernel<1, 4><<<plan.blocks, 128, smem, stream>>>(b);
        else dev::interval_level_kernel<0, 4><<<plan.blocks, 128, smem, stream>>>(b);
    } else {
        if (rounding) dev::interval_level_kernel<1, 1><<<plan.blocks, 32, smem, stream>>>(b);
        else dev::interval_level_kernel<0, 1><<<plan.blocks, 32, smem, stream>>>(b);
    }
    return cudaGetLastError();
}

}  // namespace frep
