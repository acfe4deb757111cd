// Device-side definitions shared by the voxelizer and raytracer kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "frep/frep_math.h"

namespace frep {
namespace dev {

constexpr uint32_t OP_CONST = 0, OP_SIN = 1, OP_COS = 2, OP_ADD = 3, OP_SUB = 4, OP_MUL = 5,
                   OP_DIV = 6, OP_MIN = 7, OP_MAX = 8, OP_EXP = 9, OP_NEG = 10, OP_SQRT = 11,
                   OP_COPY = 12;
constexpr uint32_t MM_FIRST = 1, MM_SECOND = 2, MM_BOTH = 3;
constexpr float EPS = 0.0001f;                    // utils.comp:19
constexpr float PI_F = 3.141592653589793238f;     // utils.comp:2
constexpr uint32_t MAX_LEVELS = 8;
constexpr uint32_t MAX_DDA_STEPS = 1u << 16;      // bound on every DDA loop
constexpr uint32_t TAPE_ALIGN_WORDS = 16;         // tape records start on 128-byte lines

// Device-resident state of one tree (one per frep_tree). The first block is
// written once when the tree is created; the rest is reset by the init kernel
// at the start of every voxelization. Level passes read a tree entirely from
// here, so one launch can serve many trees.
struct TreeHeader {
    // ---- static: set at creation ----
    uint32_t* nodes;                           // node pool
    uint64_t* tapes;                           // tape pool
    unsigned long long node_cap;               // u32 words
    unsigned long long tape_cap;               // u64 words
    uint32_t levels;
    uint32_t shorten;
    uint32_t share_tapes;                      // identical child tapes of a group stored once
    uint32_t dims[MAX_LEVELS];
    uint32_t node_size[MAX_LEVELS];            // u32 words
    float cell_size[MAX_LEVELS];
    float low[3];
    uint32_t point_k;                          // last-level pass: cells per lane (2 or 4)
    // ---- per voxelization ----
    float tape_time;
    uint32_t node_count[MAX_LEVELS];           // interiorNodeCount
    unsigned long long node_ofs[MAX_LEVELS];   // u32 words
    unsigned long long tape_top;               // u64 words
    unsigned long long tape_size_sum[MAX_LEVELS];
    uint32_t tape_size_max[MAX_LEVELS];
    unsigned long long cell_instr[MAX_LEVELS]; // cell-instructions evaluated per level
    unsigned long long fp32_ops[MAX_LEVELS];   // op-weighted FP32 work per level (count_ops_kernel)
    uint32_t overflow;                         // bit 0 node pool, bit 1 tape pool
    uint32_t status;                           // reserved for bounded-wait failures
    uint32_t reuse_eval[MAX_LEVELS];           // reuse: nodes of each level listed for
                                               //   evaluation (the others are copies)
};

__device__ __forceinline__ uint32_t level_count(const TreeHeader* H, uint32_t level,
                                                unsigned long long node_cap, uint32_t node_size) {
    // A pool overflow in the previous level may have counted children that
    // were never written; only the ones that fit exist.
    const unsigned long long ofs = H->node_ofs[level];
    const unsigned long long cap = node_cap > ofs ? (node_cap - ofs) / node_size : 0;
    return (uint32_t)min((unsigned long long)H->node_count[level], cap);
}

// Entry of a node in a tree's reuse side array (one u32 per node: the
// previous tree's node it is copied from, or ~0). Nodes are at least 8 words
// (dims are multiples of 4), so word offset / 8 is unique per node.
__host__ __device__ inline unsigned long long reuse_slot(unsigned long long level_ofs, uint32_t node,
                                                         uint32_t node_size) {
    return (level_ofs + (unsigned long long)node * node_size) >> 3;
}

__host__ __device__ inline uint32_t node_words(uint32_t dim, bool last) {
    const uint32_t c3 = dim * dim * dim;       // node.comp:4-15
    return last ? 4 + (c3 >> 4) : 4 + 17 * (c3 >> 4);
}

// Algorithmic FP32 operations per cell for one tape instruction: the weights
// of the reference's interval formulas (interval.comp:36-111) and of the point
// interpreter (point.comp:41-81). Used only for work accounting.
//                                  CONST SIN COS ADD SUB MUL DIV MIN MAX EXP NEG SQRT COPY
__device__ __constant__ const uint8_t kIntervalOps[16] = {0, 18, 18, 2, 2, 10, 16, 4, 4, 2, 0, 4, 0, 0, 0, 0};
__device__ __constant__ const uint8_t kPointOps[16]    = {0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0};

__device__ __forceinline__ uint32_t w_op(uint64_t w) { return (uint32_t)w & 0xFFu; }
__device__ __forceinline__ uint32_t w_out(uint64_t w) { return ((uint32_t)w >> 16) & 0xFFFFu; }
__device__ __forceinline__ uint32_t w_a(uint64_t w) { return (uint32_t)(w >> 32) & 0xFFFFu; }
__device__ __forceinline__ uint32_t w_b(uint64_t w) { return (uint32_t)(w >> 48); }
__device__ __forceinline__ float w_const(uint64_t w) { return __uint_as_float((uint32_t)(w >> 32)); }
__device__ __forceinline__ bool is_mm(uint32_t op) { return op == OP_MIN || op == OP_MAX; }
__host__ __device__ constexpr bool is_binary(uint32_t op) {
    return op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_DIV || op == OP_MIN || op == OP_MAX;
}

// glm's min/max selection rules (the oracle uses the same selects).
__device__ __forceinline__ float min_sel(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float max_sel(float a, float b) { return (a < b) ? b : a; }

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// ---- interval arithmetic (interval.comp:8-111) --------------------------------
// ROUND = 0: the reference's round-to-nearest; ROUND = 1: outward (directed
// rounding intrinsics), conservative.
template <int ROUND>
__device__ __forceinline__ float2 iv_mul(float2 a, float2 b) {
    if (ROUND) {
        const float l0 = __fmul_rd(a.x, b.x), l1 = __fmul_rd(a.x, b.y), l2 = __fmul_rd(a.y, b.x),
                    l3 = __fmul_rd(a.y, b.y);
        const float h0 = __fmul_ru(a.x, b.x), h1 = __fmul_ru(a.x, b.y), h2 = __fmul_ru(a.y, b.x),
                    h3 = __fmul_ru(a.y, b.y);
        return make_float2(min_sel(min_sel(l0, l1), min_sel(l2, l3)),
                           max_sel(max_sel(h0, h1), max_sel(h2, h3)));
    } else {
        const float p0 = __fmul_rn(a.x, b.x), p1 = __fmul_rn(a.x, b.y), p2 = __fmul_rn(a.y, b.x),
                    p3 = __fmul_rn(a.y, b.y);
        return make_float2(min_sel(min_sel(p0, p1), min_sel(p2, p3)),
                           max_sel(max_sel(p0, p1), max_sel(p2, p3)));
    }
}

__device__ __forceinline__ bool contains_multiple(float lo, float hi, float x) {
    const float ql = __fdiv_rn(lo, x), qh = __fdiv_rn(hi, x);
    const float fl = floorf(ql), fh = floorf(qh);
    return fl < fh || fl == ql || fh == qh;
}

static __device__ __noinline__ float2 iv_sincos_rn(float2 a, bool is_cos) {
    const float two_pi = 2.0f * PI_F, half_pi = PI_F / 2.0f;
    if (!is_cos) {
        const float s_lo = frep_sinf(a.x), s_hi = frep_sinf(a.y);
        const float lo = contains_multiple(__fadd_rn(a.x, half_pi), __fadd_rn(a.y, half_pi), two_pi)
                             ? -1.0f : min_sel(s_lo, s_hi);
        const float hi = contains_multiple(__fsub_rn(a.x, half_pi), __fsub_rn(a.y, half_pi), two_pi)
                             ? 1.0f : max_sel(s_lo, s_hi);
        return make_float2(lo, hi);
    }
    const float c_lo = frep_cosf(a.x), c_hi = frep_cosf(a.y);
    const float lo = contains_multiple(__fsub_rn(a.x, PI_F), __fsub_rn(a.y, PI_F), two_pi)
                         ? -1.0f : min_sel(c_lo, c_hi);
    const float hi = contains_multiple(a.x, a.y, two_pi) ? 1.0f : max_sel(c_lo, c_hi);
    return make_float2(lo, hi);
}

__device__ __forceinline__ bool critical_in(double lo, double hi, double phase) {
    const double two_pi = 6.283185307179586;
    const double kl = ceil(__dsub_rn(__ddiv_rn(__dsub_rn(lo, phase), two_pi), 1e-9));
    const double kh = floor(__dadd_rn(__ddiv_rn(__dsub_rn(hi, phase), two_pi), 1e-9));
    return kl <= kh;
}

static __device__ __noinline__ float2 iv_sincos_out(float2 a, bool is_cos) {
    const double lo = a.x, hi = a.y;
    if (!(__dsub_rn(hi, lo) < 6.0) || !(fabs(lo) < 1048576.0) || !(fabs(hi) < 1048576.0))
        return make_float2(-1.0f, 1.0f);
    const double ph_max = is_cos ? 0.0 : 1.5707963267948966;
    const double ph_min = is_cos ? 3.141592653589793 : -1.5707963267948966;
    const float f_lo = is_cos ? frep_cosf(a.x) : frep_sinf(a.x);
    const float f_hi = is_cos ? frep_cosf(a.y) : frep_sinf(a.y);
    const float l = critical_in(lo, hi, ph_min) ? -1.0f : max_sel(-1.0f, frep_next_down(min_sel(f_lo, f_hi)));
    const float h = critical_in(lo, hi, ph_max) ? 1.0f : min_sel(1.0f, frep_next_up(max_sel(f_lo, f_hi)));
    return make_float2(l, h);
}

template <int ROUND>
__device__ __noinline__ float2 iv_div(float2 a, float2 b) {
    const float inf = __int_as_float(0x7f800000);
    if ((b.x == 0.0f && b.y == 0.0f) || (b.x < 0.0f && b.y > 0.0f)) return make_float2(-inf, inf);
    float2 r;
    if (b.x == 0.0f) r = make_float2(ROUND ? __fdiv_rd(1.0f, b.y) : __fdiv_rn(1.0f, b.y), inf);
    else if (b.y == 0.0f) r = make_float2(-inf, ROUND ? __fdiv_ru(1.0f, b.x) : __fdiv_rn(1.0f, b.x));
    else r = make_float2(ROUND ? __fdiv_rd(1.0f, b.y) : __fdiv_rn(1.0f, b.y),
                         ROUND ? __fdiv_ru(1.0f, b.x) : __fdiv_rn(1.0f, b.x));
    return iv_mul<ROUND>(a, r);
}

template <int ROUND>
__device__ __noinline__ float2 iv_exp(float2 a) {
    const float el = frep_expf(a.x), eh = frep_expf(a.y);
    if (ROUND) return make_float2(max_sel(0.0f, frep_next_down(el)), frep_next_up(eh));
    return make_float2(el, eh);
}

// One interval instruction (INTERVAL_UPDATE_SLOTS, interval.comp:36-111).
template <int ROUND>
__device__ __forceinline__ float2 iv_apply(uint32_t op, uint64_t w, float2 a, float2 b) {
    switch (op) {
        case OP_CONST: { const float c = w_const(w); return make_float2(c, c); }
        case OP_ADD:
            return ROUND ? make_float2(__fadd_rd(a.x, b.x), __fadd_ru(a.y, b.y))
                         : make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
        case OP_SUB:
            return ROUND ? make_float2(__fsub_rd(a.x, b.y), __fsub_ru(a.y, b.x))
                         : make_float2(__fsub_rn(a.x, b.y), __fsub_rn(a.y, b.x));
        case OP_MUL: return iv_mul<ROUND>(a, b);
        case OP_MIN: return make_float2(min_sel(a.x, b.x), min_sel(a.y, b.y));
        case OP_MAX: return make_float2(max_sel(a.x, b.x), max_sel(a.y, b.y));
        case OP_NEG: return make_float2(-a.y, -a.x);
        case OP_SQRT: {
            const float l = max_sel(0.0f, a.x), h = max_sel(0.0f, a.y);
            return ROUND ? make_float2(__fsqrt_rd(l), __fsqrt_ru(h))
                         : make_float2(__fsqrt_rn(l), __fsqrt_rn(h));
        }
        case OP_DIV: return iv_div<ROUND>(a, b);
        case OP_EXP: return iv_exp<ROUND>(a);
        case OP_SIN: return ROUND ? iv_sincos_out(a, false) : iv_sincos_rn(a, false);
        case OP_COS: return ROUND ? iv_sincos_out(a, true) : iv_sincos_rn(a, true);
        default: return a;  // COPY
    }
}

// ---- hybrid affine mode (FREP_ROUND_HYBRID) ----------------------------------
// A slot carries its outward interval and an affine form over the cell's axes,
// A = c + x ex + y ey + z ez + [-e, e] (ex, ey, ez in [-1, 1]). Each
// instruction computes the outward interval of its operands' intervals (the
// formulas above) and the affine form; the slot keeps the interval intersected
// with the form's range. Centres and coefficients are rounded to nearest and
// every rounding error is added to e, rounded up (af_err bounds the error of
// a nearest-rounded result r by |r| 2^-23 + 2^-149). Sums of error terms run
// left to right, so the oracle (oracle/frep_oracle.cpp) computes the same bits.
struct Af {
    float c, x, y, z, e;
};
__device__ __forceinline__ float af_err(float r) { return __fadd_ru(__fmul_ru(fabsf(r), 0x1p-23f), 0x1p-149f); }
__device__ __forceinline__ float af_rad(const Af& a) {
    return __fadd_ru(__fadd_ru(__fadd_ru(fabsf(a.x), fabsf(a.y)), fabsf(a.z)), a.e);
}
__device__ __forceinline__ Af af_hull(float2 v) {
    const float c = __fmul_rn(__fadd_rn(v.x, v.y), 0.5f);
    return Af{c, 0.0f, 0.0f, 0.0f, max_sel(__fsub_ru(v.y, c), __fsub_ru(c, v.x))};
}
// The interval intersected with the form's range (a NaN form leaves it as is).
__device__ __forceinline__ float2 af_tighten(float2 v, const Af& a) {
    const float r = af_rad(a);
    return make_float2(max_sel(v.x, __fsub_rd(a.c, r)), min_sel(v.y, __fadd_ru(a.c, r)));
}
__device__ __forceinline__ Af af_addsub(const Af& a, const Af& b, bool sub) {
    Af r;
    r.c = sub ? __fsub_rn(a.c, b.c) : __fadd_rn(a.c, b.c);
    r.x = sub ? __fsub_rn(a.x, b.x) : __fadd_rn(a.x, b.x);
    r.y = sub ? __fsub_rn(a.y, b.y) : __fadd_rn(a.y, b.y);
    r.z = sub ? __fsub_rn(a.z, b.z) : __fadd_rn(a.z, b.z);
    r.e = __fadd_ru(__fadd_ru(a.e, b.e),
                    __fadd_ru(__fadd_ru(af_err(r.c), af_err(r.x)), __fadd_ru(af_err(r.y), af_err(r.z))));
    return r;
}
__device__ __forceinline__ Af af_mul(const Af& a, const Af& b, bool square) {
    Af r;
    const float ra = af_rad(a);
    if (square) {  // (c + s)^2 = c^2 + 2 c s + s^2 with s^2 in [0, ra^2] = h +- h
        const float h = __fmul_ru(__fmul_ru(ra, ra), 0.5f);
        const float cc = __fmul_rn(a.c, a.c);
        r.c = __fadd_rn(cc, h);
        r.x = __fmul_rn(__fmul_rn(a.c, a.x), 2.0f);
        r.y = __fmul_rn(__fmul_rn(a.c, a.y), 2.0f);
        r.z = __fmul_rn(__fmul_rn(a.c, a.z), 2.0f);
        const float lin = __fmul_ru(__fmul_ru(fabsf(a.c), 2.0f), a.e);
        r.e = __fadd_ru(__fadd_ru(__fadd_ru(lin, h), __fadd_ru(af_err(cc), af_err(r.c))),
                        __fadd_ru(__fadd_ru(af_err(r.x), af_err(r.y)), af_err(r.z)));
        return r;
    }
    const float rb = af_rad(b);
    r.c = __fmul_rn(a.c, b.c);
    const float x1 = __fmul_rn(a.c, b.x), x2 = __fmul_rn(b.c, a.x);
    const float y1 = __fmul_rn(a.c, b.y), y2 = __fmul_rn(b.c, a.y);
    const float z1 = __fmul_rn(a.c, b.z), z2 = __fmul_rn(b.c, a.z);
    r.x = __fadd_rn(x1, x2);
    r.y = __fadd_rn(y1, y2);
    r.z = __fadd_rn(z1, z2);
    const float lin = __fadd_ru(__fmul_ru(fabsf(a.c), b.e), __fmul_ru(fabsf(b.c), a.e));
    const float rnd = __fadd_ru(__fadd_ru(__fadd_ru(af_err(x1), af_err(x2)), __fadd_ru(af_err(y1), af_err(y2))),
                                __fadd_ru(__fadd_ru(af_err(z1), af_err(z2)),
                                          __fadd_ru(__fadd_ru(af_err(r.x), af_err(r.y)), af_err(r.z))));
    r.e = __fadd_ru(__fadd_ru(lin, __fmul_ru(ra, rb)), __fadd_ru(af_err(r.c), rnd));
    return r;
}
// The form of an input axis k (0, 1, 2) over [lo, hi].
__device__ __forceinline__ Af af_axis(float lo, float hi, int k) {
    const float c = __fmul_rn(__fadd_rn(lo, hi), 0.5f);
    const float r = max_sel(__fsub_ru(hi, c), __fsub_ru(c, lo));
    return Af{c, k == 0 ? r : 0.0f, k == 1 ? r : 0.0f, k == 2 ? r : 0.0f, 0.0f};
}
// One hybrid instruction: the outward interval of the operands' intervals and
// the form (MIN/MAX: the chosen operand's form when the choice is decided).
// Returns the tightened interval; *f receives the form.
__device__ __forceinline__ float2 hy_apply(uint32_t op, uint64_t w, float2 a, float2 b, const Af& fa, const Af& fb,
                                           bool square, uint32_t choice, Af* f) {
    const float2 v = op == OP_CONST ? make_float2(w_const(w), w_const(w)) : iv_apply<1>(op, w, a, b);
    switch (op) {
        case OP_CONST: *f = Af{v.x, 0.0f, 0.0f, 0.0f, 0.0f}; break;
        case OP_ADD: *f = af_addsub(fa, fb, false); break;
        case OP_SUB: *f = af_addsub(fa, fb, true); break;
        case OP_NEG: *f = Af{-fa.c, -fa.x, -fa.y, -fa.z, fa.e}; break;
        case OP_MUL: *f = af_mul(fa, fb, square); break;
        case OP_COPY: *f = fa; break;
        case OP_MIN:
        case OP_MAX: *f = choice == MM_FIRST ? fa : (choice == MM_SECOND ? fb : af_hull(v)); break;
        default: *f = af_hull(v); break;  // DIV SQRT EXP SIN COS: the interval's hull
    }
    return af_tighten(v, *f);
}
// MIN/MAX choice from two intervals (interval.comp:140-155).
__device__ __forceinline__ uint32_t mm_choice(uint32_t op, float2 a, float2 b) {
    const bool first_low = a.y < b.x, second_low = b.y < a.x;
    return op == OP_MIN ? (first_low ? MM_FIRST : (second_low ? MM_SECOND : MM_BOTH))
                        : (first_low ? MM_SECOND : (second_low ? MM_FIRST : MM_BOTH));
}

// Point evaluation of one instruction (point.comp:41-81).
__device__ __forceinline__ float pt_apply(uint32_t op, uint64_t w, float a, float b) {
    switch (op) {
        case OP_CONST: return w_const(w);
        case OP_ADD: return __fadd_rn(a, b);
        case OP_SUB: return __fsub_rn(a, b);
        case OP_MUL: return __fmul_rn(a, b);
        case OP_MIN: return min_sel(a, b);
        case OP_MAX: return max_sel(a, b);
        case OP_NEG: return -a;
        case OP_SQRT: return __fsqrt_rn(a);
        case OP_DIV: return __fdiv_rn(a, b);
        case OP_EXP: return frep_expf(a);
        case OP_SIN: return frep_sinf(a);
        case OP_COS: return frep_cosf(a);
        default: return a;  // COPY
    }
}

}  // namespace dev
}  // namespace frep
