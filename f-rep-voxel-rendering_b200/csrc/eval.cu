// Tape evaluation on the device over caller-given points and boxes.
//
// frep_tape_eval_device replaces csg::Tape::Eval (vulkan/src/csg/tape.cpp:
// 274-302) for many points at once; frep_tape_eval_intervals exposes the
// interval extension the level passes compute (tape_eval_interval,
// vulkan/shaders/tape/interval.comp:8-160) for arbitrary boxes. Both run the
// same per-instruction device functions as the voxelizer (pt_apply, iv_apply
// in device_common.cuh), so a value or interval returned here is the one a
// level pass computes for the same tape and box. They are what the soundness
// checks of the outward mode measure: every interval must contain the tape's
// value at any point of its box.
//
// One thread per point or box; the slot file lives in global memory as rows
// [slot][item] (coalesced), allocated per call.
#include "capi_internal.h"

namespace frep {
namespace dev {

__global__ void eval_points_kernel(const uint64_t* __restrict__ tape, uint32_t n_instr, uint32_t n_slots,
                                   const float4* __restrict__ xyzt, uint32_t n, float* __restrict__ slots,
                                   float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = xyzt[i];
    // point.comp:4-7: slots 0..3 = x, y, z, t
    slots[0 * (size_t)n + i] = p.x;
    slots[1 * (size_t)n + i] = p.y;
    slots[2 * (size_t)n + i] = p.z;
    slots[3 * (size_t)n + i] = p.w;
    for (uint32_t j = 0; j < n_instr; j++) {
        const uint64_t w = __ldg(&tape[j]);
        const uint32_t op = w_op(w);
        const float a = op == OP_CONST ? 0.0f : slots[(size_t)w_a(w) * n + i];
        const float b = is_binary(op) ? slots[(size_t)w_b(w) * n + i] : 0.0f;
        slots[(size_t)w_out(w) * n + i] = pt_apply(op, w, a, b);
    }
    out[i] = slots[i];
    (void)n_slots;
}

template <int ROUND>
__global__ void eval_intervals_kernel(const uint64_t* __restrict__ tape, uint32_t n_instr,
                                      const float* __restrict__ boxes, uint32_t n, float tape_time,
                                      float2* __restrict__ slots, float2* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* b6 = boxes + 6 * (size_t)i;
    // interval.comp:121-128: slots 0..3 = X, Y, Z over the box, T = [t, t]
    slots[0 * (size_t)n + i] = make_float2(b6[0], b6[3]);
    slots[1 * (size_t)n + i] = make_float2(b6[1], b6[4]);
    slots[2 * (size_t)n + i] = make_float2(b6[2], b6[5]);
    slots[3 * (size_t)n + i] = make_float2(tape_time, tape_time);
    for (uint32_t j = 0; j < n_instr; j++) {
        const uint64_t w = __ldg(&tape[j]);
        const uint32_t op = w_op(w);
        const float2 a = op == OP_CONST ? make_float2(0.0f, 0.0f) : slots[(size_t)w_a(w) * n + i];
        const float2 b = is_binary(op) ? slots[(size_t)w_b(w) * n + i] : make_float2(0.0f, 0.0f);
        slots[(size_t)w_out(w) * n + i] = iv_apply<ROUND>(op, w, a, b);
    }
    out[i] = slots[i];
}

// The hybrid affine mode (FREP_ROUND_HYBRID): each slot row holds the
// interval and the affine form, 8 floats (lo, hi, c, x | y, z, e, 0).
__global__ void eval_hybrid_kernel(const uint64_t* __restrict__ tape, uint32_t n_instr,
                                   const float* __restrict__ boxes, uint32_t n, float tape_time,
                                   float4* __restrict__ slots, float2* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* b6 = boxes + 6 * (size_t)i;
    auto row = [&](uint32_t s) { return slots + 2 * ((size_t)s * n + i); };
    for (int k = 0; k < 3; k++) {
        const Af f = af_axis(b6[k], b6[3 + k], k);
        row(k)[0] = make_float4(b6[k], b6[3 + k], f.c, f.x);
        row(k)[1] = make_float4(f.y, f.z, f.e, 0.0f);
    }
    row(3)[0] = make_float4(tape_time, tape_time, tape_time, 0.0f);
    row(3)[1] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (uint32_t j = 0; j < n_instr; j++) {
        const uint64_t w = __ldg(&tape[j]);
        const uint32_t op = w_op(w);
        float2 v;
        Af f;
        if (op == OP_CONST) {
            v = make_float2(w_const(w), w_const(w));
            f = Af{v.x, 0.0f, 0.0f, 0.0f, 0.0f};
        } else {
            const uint32_t sb = is_binary(op) ? w_b(w) : 0u;
            const float4 a0 = row(w_a(w))[0], a1 = row(w_a(w))[1];
            const float4 b0 = row(sb)[0], b1 = row(sb)[1];
            const float2 a = make_float2(a0.x, a0.y), b = make_float2(b0.x, b0.y);
            const Af fa{a0.z, a0.w, a1.x, a1.y, a1.z}, fb{b0.z, b0.w, b1.x, b1.y, b1.z};
            const uint32_t c = is_mm(op) ? mm_choice(op, a, b) : 0u;
            v = hy_apply(op, w, a, b, fa, fb, op == OP_MUL && w_a(w) == w_b(w), c, &f);
        }
        row(w_out(w))[0] = make_float4(v.x, v.y, f.c, f.x);
        row(w_out(w))[1] = make_float4(f.y, f.z, f.e, 0.0f);
    }
    out[i] = make_float2(row(0)[0].x, row(0)[0].y);
}

}  // namespace dev
}  // namespace frep

using frep::detail::align_up;
using frep::detail::cuda_fail;
using frep::detail::fail;

namespace {

// Device buffers of one evaluation call, released on every path.
struct EvalBuffers {
    void* p = nullptr;
    ~EvalBuffers() {
        if (p) cudaFree(p);
    }
};

frep_status eval_common(frep_ctx* ctx, const frep_tape* tape, uint32_t n, uint64_t in_bytes, uint64_t slot_bytes,
                        uint64_t out_bytes, EvalBuffers* buf, uint8_t** in, uint8_t** slots, uint8_t** out,
                        const char* who) {
    // Every slot an instruction names must be a row of the slot file the
    // kernels index with it.
    const uint32_t n_slots = std::max<uint32_t>(tape->ct.n_slots, 4);
    for (const uint64_t w : tape->ct.instrs) {
        const uint32_t op = (uint32_t)w & 0xFFu, o = ((uint32_t)w >> 16) & 0xFFFFu;
        const uint32_t a = (uint32_t)(w >> 32) & 0xFFFFu, b = (uint32_t)(w >> 48);
        if (op > FREP_TAPE_COPY || o >= n_slots || (op != FREP_TAPE_CONST && a >= n_slots) ||
            (frep::dev::is_binary(op) && b >= n_slots))
            return fail(FREP_ERR_INVALID_ARG, "%s: instruction names a slot outside the tape's %u slots", who, n_slots);
    }
    const uint64_t tape_bytes = align_up(tape->ct.instrs.size() * 8 + 8, 256);
    const uint64_t total = tape_bytes + align_up(in_bytes, 256) + align_up(slot_bytes, 256) + align_up(out_bytes, 256);
    if (ctx->used + total > ctx->budget)
        return fail(FREP_ERR_OOM, "%s: %llu bytes of working memory exceed the context's budget", who,
                    (unsigned long long)total);
    FREP_CUDA(cudaSetDevice(ctx->device));
    cudaError_t e = cudaMalloc(&buf->p, total);
    if (e != cudaSuccess) {
        buf->p = nullptr;
        return fail(FREP_ERR_OOM, "%s: cudaMalloc of %llu bytes failed (%s)", who, (unsigned long long)total,
                    cudaGetErrorString(e));
    }
    uint8_t* base = static_cast<uint8_t*>(buf->p);
    FREP_CUDA(cudaMemcpy(base, tape->ct.instrs.data(), tape->ct.instrs.size() * 8, cudaMemcpyHostToDevice));
    *in = base + tape_bytes;
    *slots = *in + align_up(in_bytes, 256);
    *out = *slots + align_up(slot_bytes, 256);
    (void)n;
    return FREP_OK;
}

}  // namespace

extern "C" frep_status frep_tape_eval_device(frep_ctx* ctx, const frep_tape* tape, const float* xyzt, uint32_t n,
                                             float* out) {
    if (!ctx || !tape || (n && (!xyzt || !out))) return fail(FREP_ERR_INVALID_ARG, "frep_tape_eval_device: null argument");
    if (n == 0) return FREP_OK;
    if (tape->ct.instrs.empty()) return fail(FREP_ERR_INVALID_ARG, "frep_tape_eval_device: empty tape");
    const uint32_t n_slots = std::max<uint32_t>(tape->ct.n_slots, 4);
    EvalBuffers buf;
    uint8_t *d_in, *d_slots, *d_out;
    frep_status st = eval_common(ctx, tape, n, (uint64_t)n * 16, (uint64_t)n * n_slots * 4, (uint64_t)n * 4, &buf,
                                 &d_in, &d_slots, &d_out, "frep_tape_eval_device");
    if (st != FREP_OK) return st;
    FREP_CUDA(cudaMemcpy(d_in, xyzt, (size_t)n * 16, cudaMemcpyHostToDevice));
    const uint32_t threads = 128, blocks = (n + threads - 1) / threads;
    frep::dev::eval_points_kernel<<<blocks, threads>>>(static_cast<const uint64_t*>(buf.p),
                                                        (uint32_t)tape->ct.instrs.size(), n_slots,
                                                        reinterpret_cast<const float4*>(d_in), n,
                                                        reinterpret_cast<float*>(d_slots),
                                                        reinterpret_cast<float*>(d_out));
    FREP_CUDA(cudaGetLastError());
    FREP_CUDA(cudaMemcpy(out, d_out, (size_t)n * 4, cudaMemcpyDeviceToHost));
    return FREP_OK;
}

extern "C" frep_status frep_tape_eval_intervals(frep_ctx* ctx, const frep_tape* tape, const float* boxes, uint32_t n,
                                                float tape_time, uint32_t rounding, float* out) {
    if (!ctx || !tape || (n && (!boxes || !out)))
        return fail(FREP_ERR_INVALID_ARG, "frep_tape_eval_intervals: null argument");
    if (rounding > FREP_ROUND_HYBRID) return fail(FREP_ERR_INVALID_ARG, "frep_tape_eval_intervals: rounding %u", rounding);
    if (n == 0) return FREP_OK;
    if (tape->ct.instrs.empty()) return fail(FREP_ERR_INVALID_ARG, "frep_tape_eval_intervals: empty tape");
    const uint32_t n_slots = std::max<uint32_t>(tape->ct.n_slots, 4);
    EvalBuffers buf;
    uint8_t *d_in, *d_slots, *d_out;
    const uint64_t row_bytes = rounding == FREP_ROUND_HYBRID ? 32 : 8;
    frep_status st = eval_common(ctx, tape, n, (uint64_t)n * 24, (uint64_t)n * n_slots * row_bytes, (uint64_t)n * 8,
                                 &buf, &d_in, &d_slots, &d_out, "frep_tape_eval_intervals");
    if (st != FREP_OK) return st;
    FREP_CUDA(cudaMemcpy(d_in, boxes, (size_t)n * 24, cudaMemcpyHostToDevice));
    const uint32_t threads = 128, blocks = (n + threads - 1) / threads;
    const auto* t = static_cast<const uint64_t*>(buf.p);
    const uint32_t ni = (uint32_t)tape->ct.instrs.size();
    if (rounding == FREP_ROUND_HYBRID)
        frep::dev::eval_hybrid_kernel<<<blocks, threads>>>(t, ni, reinterpret_cast<const float*>(d_in), n, tape_time,
                                                           reinterpret_cast<float4*>(d_slots),
                                                           reinterpret_cast<float2*>(d_out));
    else if (rounding == FREP_ROUND_OUTWARD)
        frep::dev::eval_intervals_kernel<1><<<blocks, threads>>>(t, ni, reinterpret_cast<const float*>(d_in), n,
                                                                  tape_time, reinterpret_cast<float2*>(d_slots),
                                                                  reinterpret_cast<float2*>(d_out));
    else
        frep::dev::eval_intervals_kernel<0><<<blocks, threads>>>(t, ni, reinterpret_cast<const float*>(d_in), n,
                                                                  tape_time, reinterpret_cast<float2*>(d_slots),
                                                                  reinterpret_cast<float2*>(d_out));
    FREP_CUDA(cudaGetLastError());
    FREP_CUDA(cudaMemcpy(out, d_out, (size_t)n * 8, cudaMemcpyDeviceToHost));
    return FREP_OK;
}
