// CPU oracle — TEST INFRASTRUCTURE (see frep_oracle.h for scope and pins).
//
// A plain, single-cell-at-a-time restatement of the reference's shaders. It is
// deliberately simple: one std::vector of slots per evaluation, straight
// switch dispatch, node-parallel threads with a serial merge in node order.
#include "frep_oracle.h"

#include <algorithm>
#include <cfenv>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "frep/frep_math.h"

namespace {

enum : uint32_t {
    OP_CONST = 0, OP_SIN, OP_COS, OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_MIN, OP_MAX,
    OP_EXP, OP_NEG, OP_SQRT, OP_COPY
};
constexpr uint8_t MM_FIRST = 1, MM_SECOND = 2, MM_BOTH = 3;
constexpr float EPS = 0.0001f;                          // utils.comp:19
constexpr float PI_F = 3.141592653589793238f;           // utils.comp:2 (float)
constexpr uint32_t MAX_DDA_STEPS = 1u << 16;            // bound on every DDA loop

inline uint32_t i_op(uint64_t w) { return (uint32_t)(w & 0xFF); }
inline uint32_t i_out(uint64_t w) { return (uint32_t)((w >> 16) & 0xFFFF); }
inline uint32_t i_a(uint64_t w) { return (uint32_t)((w >> 32) & 0xFFFF); }
inline uint32_t i_b(uint64_t w) { return (uint32_t)((w >> 48) & 0xFFFF); }
inline float i_const(uint64_t w) {
    uint32_t u = (uint32_t)(w >> 32);
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline bool is_mm(uint32_t op) { return op == OP_MIN || op == OP_MAX; }

// glm's min/max selection rules; the GPU code uses the same selects.
inline float min_sel(float a, float b) { return (b < a) ? b : a; }
inline float max_sel(float a, float b) { return (a < b) ? b : a; }

struct Iv {
    float lo, hi;
};

// ---- directed rounding -----------------------------------------------------
// The outward evaluator runs with the SSE rounding mode set to FE_DOWNWARD;
// upward results use RU(x) = -RD(-x). sqrt (not odd) switches to FE_UPWARD.
struct RoundMode {
    int saved;
    explicit RoundMode(int mode) : saved(std::fegetround()) { std::fesetround(mode); }
    ~RoundMode() { std::fesetround(saved); }
};
inline float add_dn(float a, float b) { return a + b; }
inline float add_up(float a, float b) { return -((-a) - b); }
inline float sub_dn(float a, float b) { return a - b; }
inline float sub_up(float a, float b) { return -(b - a); }
inline float mul_dn(float a, float b) { return a * b; }
inline float mul_up(float a, float b) { return -((-a) * b); }
inline float div_dn(float a, float b) { return a / b; }
inline float div_up(float a, float b) { return -((-a) / b); }
inline float sqrt_dn(float a) { return std::sqrt(a); }
inline float sqrt_up(float a) {
    std::fesetround(FE_UPWARD);
    float r = std::sqrt(a);
    std::fesetround(FE_DOWNWARD);
    return r;
}

// ---- interval operators (interval.comp:8-111) --------------------------------
inline Iv mul_rn(Iv a, Iv b) {
    const float p0 = a.lo * b.lo, p1 = a.lo * b.hi, p2 = a.hi * b.lo, p3 = a.hi * b.hi;
    return {min_sel(min_sel(p0, p1), min_sel(p2, p3)), max_sel(max_sel(p0, p1), max_sel(p2, p3))};
}
inline Iv mul_out(Iv a, Iv b) {
    const float l0 = mul_dn(a.lo, b.lo), l1 = mul_dn(a.lo, b.hi), l2 = mul_dn(a.hi, b.lo),
                l3 = mul_dn(a.hi, b.hi);
    const float h0 = mul_up(a.lo, b.lo), h1 = mul_up(a.lo, b.hi), h2 = mul_up(a.hi, b.lo),
                h3 = mul_up(a.hi, b.hi);
    return {min_sel(min_sel(l0, l1), min_sel(l2, l3)), max_sel(max_sel(h0, h1), max_sel(h2, h3))};
}

// contains_multiple (interval.comp:20-25), float round-to-nearest.
inline bool contains_multiple(float lo, float hi, float x) {
    const float ql = lo / x, qh = hi / x;
    const float fl = std::floor(ql), fh = std::floor(qh);
    return fl < fh || fl == ql || fh == qh;
}

Iv sin_rn(Iv a) {
    const float half_pi = PI_F / 2, two_pi = 2 * PI_F;
    const float s_lo = frep_sinf(a.lo), s_hi = frep_sinf(a.hi);
    Iv r;
    r.lo = contains_multiple(a.lo + half_pi, a.hi + half_pi, two_pi) ? -1.0f : min_sel(s_lo, s_hi);
    r.hi = contains_multiple(a.lo - half_pi, a.hi - half_pi, two_pi) ? 1.0f : max_sel(s_lo, s_hi);
    return r;
}
Iv cos_rn(Iv a) {
    const float two_pi = 2 * PI_F;
    const float c_lo = frep_cosf(a.lo), c_hi = frep_cosf(a.hi);
    Iv r;
    r.lo = contains_multiple(a.lo - PI_F, a.hi - PI_F, two_pi) ? -1.0f : min_sel(c_lo, c_hi);
    r.hi = contains_multiple(a.lo, a.hi, two_pi) ? 1.0f : max_sel(c_lo, c_hi);
    return r;
}

// Outward sin/cos: the extreme is +-1 if a critical point may lie in [lo, hi]
// (tested in double with a 1e-9 margin in units of periods), else the
// endpoint values widened by one ulp (frep_sinf/frep_cosf are within 1 ulp).
// Evaluated in round-to-nearest.
bool critical_in(double lo, double hi, double phase) {
    const double two_pi = 6.283185307179586;
    const double kl = std::ceil((lo - phase) / two_pi - 1e-9);
    const double kh = std::floor((hi - phase) / two_pi + 1e-9);
    return kl <= kh;
}
Iv sincos_out(Iv a, bool is_cos) {
    const double lo = a.lo, hi = a.hi;
    if (!(hi - lo < 6.0) || !(std::fabs(lo) < 1048576.0) || !(std::fabs(hi) < 1048576.0))
        return {-1.0f, 1.0f};
    const double ph_max = is_cos ? 0.0 : 1.5707963267948966;
    const double ph_min = is_cos ? 3.141592653589793 : -1.5707963267948966;
    const float f_lo = is_cos ? frep_cosf(a.lo) : frep_sinf(a.lo);
    const float f_hi = is_cos ? frep_cosf(a.hi) : frep_sinf(a.hi);
    Iv r;
    r.lo = critical_in(lo, hi, ph_min) ? -1.0f : max_sel(-1.0f, frep_next_down(min_sel(f_lo, f_hi)));
    r.hi = critical_in(lo, hi, ph_max) ? 1.0f : min_sel(1.0f, frep_next_up(max_sel(f_lo, f_hi)));
    return r;
}

// One interval instruction. rounding: 0 nearest, 1 outward (FE_DOWNWARD active).
inline Iv interval_op(uint32_t op, uint64_t w, Iv a, Iv b, int rounding) {
    const float inf = INFINITY;
    switch (op) {
        case OP_CONST: { const float c = i_const(w); return {c, c}; }
        case OP_ADD:
            return rounding ? Iv{add_dn(a.lo, b.lo), add_up(a.hi, b.hi)} : Iv{a.lo + b.lo, a.hi + b.hi};
        case OP_SUB:
            return rounding ? Iv{sub_dn(a.lo, b.hi), sub_up(a.hi, b.lo)} : Iv{a.lo - b.hi, a.hi - b.lo};
        case OP_MUL: return rounding ? mul_out(a, b) : mul_rn(a, b);
        case OP_DIV: {
            if ((b.lo == 0 && b.hi == 0) || (b.lo < 0 && b.hi > 0)) return {-inf, inf};
            Iv rcp;
            if (b.lo == 0) rcp = {rounding ? div_dn(1.0f, b.hi) : 1.0f / b.hi, inf};
            else if (b.hi == 0) rcp = {-inf, rounding ? div_up(1.0f, b.lo) : 1.0f / b.lo};
            else rcp = {rounding ? div_dn(1.0f, b.hi) : 1.0f / b.hi, rounding ? div_up(1.0f, b.lo) : 1.0f / b.lo};
            return rounding ? mul_out(a, rcp) : mul_rn(a, rcp);
        }
        case OP_MIN: return {min_sel(a.lo, b.lo), min_sel(a.hi, b.hi)};
        case OP_MAX: return {max_sel(a.lo, b.lo), max_sel(a.hi, b.hi)};
        case OP_NEG: return {-a.hi, -a.lo};
        case OP_SQRT: {
            const float l = max_sel(0.0f, a.lo), h = max_sel(0.0f, a.hi);
            return rounding ? Iv{sqrt_dn(l), sqrt_up(h)} : Iv{std::sqrt(l), std::sqrt(h)};
        }
        case OP_COPY: return a;
        case OP_EXP: {
            if (!rounding) return {frep_expf(a.lo), frep_expf(a.hi)};
            std::fesetround(FE_TONEAREST);
            const float el = frep_expf(a.lo), eh = frep_expf(a.hi);
            std::fesetround(FE_DOWNWARD);
            return {max_sel(0.0f, frep_next_down(el)), frep_next_up(eh)};
        }
        case OP_SIN:
        case OP_COS: {
            if (!rounding) return op == OP_SIN ? sin_rn(a) : cos_rn(a);
            std::fesetround(FE_TONEAREST);
            Iv r = sincos_out(a, op == OP_COS);
            std::fesetround(FE_DOWNWARD);
            return r;
        }
    }
    return a;
}

// ---- hybrid affine mode (rounding 2; this library's own, see frep.h) --------
// Each slot carries its outward interval and an affine form over the cell's
// axes, A = c + x ex + y ey + z ez + [-e, e] (ex, ey, ez in [-1, 1]); every
// instruction computes the outward interval of its operands' intervals and the
// affine form, and the slot keeps the interval intersected with the form's
// range. Forms take their centre and coefficients rounded to nearest and add
// every rounding error to e, rounded up. Evaluated with FE_DOWNWARD active
// (as the outward intervals are); nearest operations switch the mode.
struct Af {
    float c, x, y, z, e;
};
inline float rn_add(float a, float b) { std::fesetround(FE_TONEAREST); const float r = a + b; std::fesetround(FE_DOWNWARD); return r; }
inline float rn_sub(float a, float b) { std::fesetround(FE_TONEAREST); const float r = a - b; std::fesetround(FE_DOWNWARD); return r; }
inline float rn_mul(float a, float b) { std::fesetround(FE_TONEAREST); const float r = a * b; std::fesetround(FE_DOWNWARD); return r; }
// bound on the error of a round-to-nearest result r: |r| 2^-23 + 2^-149, up
inline float af_err(float r) { return add_up(mul_up(std::fabs(r), 0x1p-23f), 0x1p-149f); }
// radius of the non-constant part, summed left to right, rounded up
inline float af_rad(const Af& a) {
    return add_up(add_up(add_up(std::fabs(a.x), std::fabs(a.y)), std::fabs(a.z)), a.e);
}
inline Af af_hull(Iv v) {
    const float c = rn_mul(rn_add(v.lo, v.hi), 0.5f);
    return {c, 0.0f, 0.0f, 0.0f, max_sel(sub_up(v.hi, c), sub_up(c, v.lo))};
}
// the interval intersected with the form's range (NaN forms leave it as is)
inline Iv af_tighten(Iv v, const Af& a) {
    const float r = af_rad(a);
    return {max_sel(v.lo, sub_dn(a.c, r)), min_sel(v.hi, add_up(a.c, r))};
}
inline Af af_addsub(const Af& a, const Af& b, bool sub) {
    Af r;
    r.c = sub ? rn_sub(a.c, b.c) : rn_add(a.c, b.c);
    r.x = sub ? rn_sub(a.x, b.x) : rn_add(a.x, b.x);
    r.y = sub ? rn_sub(a.y, b.y) : rn_add(a.y, b.y);
    r.z = sub ? rn_sub(a.z, b.z) : rn_add(a.z, b.z);
    r.e = add_up(add_up(a.e, b.e), add_up(add_up(af_err(r.c), af_err(r.x)), add_up(af_err(r.y), af_err(r.z))));
    return r;
}
inline Af af_mul(const Af& a, const Af& b, bool square) {
    Af r;
    const float ra = af_rad(a);
    if (square) {  // (c + s)^2 = c^2 + 2 c s + s^2, s^2 in [0, ra^2] = h +- h
        const float h = mul_up(mul_up(ra, ra), 0.5f);
        const float cc = rn_mul(a.c, a.c);
        r.c = rn_add(cc, h);
        r.x = rn_mul(rn_mul(a.c, a.x), 2.0f);
        r.y = rn_mul(rn_mul(a.c, a.y), 2.0f);
        r.z = rn_mul(rn_mul(a.c, a.z), 2.0f);
        const float lin = mul_up(mul_up(std::fabs(a.c), 2.0f), a.e);
        r.e = add_up(add_up(add_up(lin, h), add_up(af_err(cc), af_err(r.c))),
                     add_up(add_up(af_err(r.x), af_err(r.y)), af_err(r.z)));
        return r;
    }
    const float rb = af_rad(b);
    r.c = rn_mul(a.c, b.c);
    const float x1 = rn_mul(a.c, b.x), x2 = rn_mul(b.c, a.x);
    const float y1 = rn_mul(a.c, b.y), y2 = rn_mul(b.c, a.y);
    const float z1 = rn_mul(a.c, b.z), z2 = rn_mul(b.c, a.z);
    r.x = rn_add(x1, x2);
    r.y = rn_add(y1, y2);
    r.z = rn_add(z1, z2);
    const float lin = add_up(mul_up(std::fabs(a.c), b.e), mul_up(std::fabs(b.c), a.e));
    const float rnd = add_up(add_up(add_up(af_err(x1), af_err(x2)), add_up(af_err(y1), af_err(y2))),
                             add_up(add_up(af_err(z1), af_err(z2)),
                                    add_up(add_up(af_err(r.x), af_err(r.y)), af_err(r.z))));
    r.e = add_up(add_up(lin, mul_up(ra, rb)), add_up(af_err(r.c), rnd));
    return r;
}

Iv eval_hybrid(const uint64_t* tape, uint32_t n, std::vector<Iv>& slots, std::vector<Af>& forms,
               const float* lo3, const float* hi3, float t, uint8_t* choices) {
    RoundMode mode(FE_DOWNWARD);
    for (int k = 0; k < 3; k++) {
        slots[k] = {lo3[k], hi3[k]};
        const float c = rn_mul(rn_add(lo3[k], hi3[k]), 0.5f);
        const float r = max_sel(sub_up(hi3[k], c), sub_up(c, lo3[k]));
        forms[k] = {c, k == 0 ? r : 0.0f, k == 1 ? r : 0.0f, k == 2 ? r : 0.0f, 0.0f};
    }
    slots[3] = {t, t};
    forms[3] = {t, 0.0f, 0.0f, 0.0f, 0.0f};
    uint32_t mm = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint64_t w = tape[i];
        const uint32_t op = i_op(w);
        const Iv a = op == OP_CONST ? Iv{0, 0} : slots[i_a(w)];
        const Iv b = op == OP_CONST ? Iv{0, 0} : slots[i_b(w)];
        const Af fa = op == OP_CONST ? Af{} : forms[i_a(w)];
        const Af fb = op == OP_CONST ? Af{} : forms[i_b(w)];
        const Iv v = interval_op(op, w, a, b, 1);
        Af f;
        switch (op) {
            case OP_CONST: f = {v.lo, 0.0f, 0.0f, 0.0f, 0.0f}; break;
            case OP_ADD: f = af_addsub(fa, fb, false); break;
            case OP_SUB: f = af_addsub(fa, fb, true); break;
            case OP_NEG: f = {-fa.c, -fa.x, -fa.y, -fa.z, fa.e}; break;
            case OP_MUL: f = af_mul(fa, fb, i_a(w) == i_b(w)); break;
            case OP_COPY: f = fa; break;
            case OP_MIN:
            case OP_MAX: {
                const bool first_low = a.hi < b.lo, second_low = b.hi < a.lo;
                const uint8_t c = op == OP_MIN ? (first_low ? MM_FIRST : (second_low ? MM_SECOND : MM_BOTH))
                                               : (first_low ? MM_SECOND : (second_low ? MM_FIRST : MM_BOTH));
                if (choices) choices[mm] = c;
                mm++;
                f = c == MM_FIRST ? fa : (c == MM_SECOND ? fb : af_hull(v));
                break;
            }
            default: f = af_hull(v); break;  // DIV SQRT EXP SIN COS: the interval's hull
        }
        slots[i_out(w)] = af_tighten(v, f);
        forms[i_out(w)] = f;
    }
    return slots[0];
}

// tape_eval_interval (interval.comp:121-160): slots 0..3 = box x, y, z and
// [t, t]; MIN/MAX record FIRST/SECOND/BOTH with strict comparisons.
// rounding 2 = the hybrid affine mode (eval_hybrid).
Iv eval_interval(const uint64_t* tape, uint32_t n, std::vector<Iv>& slots, const float* lo3,
                 const float* hi3, float t, int rounding, uint8_t* choices, Iv* trace = nullptr) {
    if (rounding == 2) {
        std::vector<Af> forms(slots.size());
        return eval_hybrid(tape, n, slots, forms, lo3, hi3, t, choices);
    }
    slots[0] = {lo3[0], hi3[0]};
    slots[1] = {lo3[1], hi3[1]};
    slots[2] = {lo3[2], hi3[2]};
    slots[3] = {t, t};
    RoundMode mode(rounding ? FE_DOWNWARD : FE_TONEAREST);
    uint32_t mm = 0;
    for (uint32_t i = 0; i < n; i++) {
        const uint64_t w = tape[i];
        const uint32_t op = i_op(w);
        // CONST carries its value in the operand fields: read no slots for it.
        const Iv a = op == OP_CONST ? Iv{0, 0} : slots[i_a(w)];
        const Iv b = op == OP_CONST ? Iv{0, 0} : slots[i_b(w)];
        slots[i_out(w)] = interval_op(op, w, a, b, rounding);
        if (trace) trace[i] = slots[i_out(w)];
        if (op == OP_MIN) {
            const uint8_t c = a.hi < b.lo ? MM_FIRST : (b.hi < a.lo ? MM_SECOND : MM_BOTH);
            if (choices) choices[mm] = c;
            mm++;
        } else if (op == OP_MAX) {
            const uint8_t c = a.hi < b.lo ? MM_SECOND : (b.hi < a.lo ? MM_FIRST : MM_BOTH);
            if (choices) choices[mm] = c;
            mm++;
        }
    }
    return slots[0];
}

// tape_eval_point (point.comp:2-63).
float eval_point(const uint64_t* tape, uint32_t n, std::vector<float>& s, float x, float y,
                 float z, float t) {
    s[0] = x;
    s[1] = y;
    s[2] = z;
    s[3] = t;
    for (uint32_t i = 0; i < n; i++) {
        const uint64_t w = tape[i];
        const uint32_t op = i_op(w);
        const float a = op == OP_CONST ? 0.0f : s[i_a(w)];
        const float b = op == OP_CONST ? 0.0f : s[i_b(w)];
        float r;
        switch (op) {
            case OP_CONST: r = i_const(w); break;
            case OP_SIN: r = frep_sinf(a); break;
            case OP_COS: r = frep_cosf(a); break;
            case OP_ADD: r = a + b; break;
            case OP_SUB: r = a - b; break;
            case OP_MUL: r = a * b; break;
            case OP_DIV: r = a / b; break;
            case OP_MIN: r = min_sel(a, b); break;
            case OP_MAX: r = max_sel(a, b); break;
            case OP_EXP: r = frep_expf(a); break;
            case OP_NEG: r = -a; break;
            case OP_SQRT: r = std::sqrt(a); break;
            default: r = a; break;  // COPY
        }
        s[i_out(w)] = r;
    }
    return s[0];
}

struct V4 {
    float x, y, z, w;
};

// tape_eval_gradient (gradient.comp:4-88): forward mode, slot = (d/dx, d/dy, d/dz, value).
void eval_gradient(const uint64_t* tape, uint32_t n, std::vector<V4>& s, float x, float y,
                   float z, float t, float* g) {
    s[0] = {1, 0, 0, x};
    s[1] = {0, 1, 0, y};
    s[2] = {0, 0, 1, z};
    s[3] = {0, 0, 0, t};
    for (uint32_t i = 0; i < n; i++) {
        const uint64_t w = tape[i];
        const uint32_t op = i_op(w);
        const V4 a = op == OP_CONST ? V4{0, 0, 0, 0} : s[i_a(w)];
        const V4 b = op == OP_CONST ? V4{0, 0, 0, 0} : s[i_b(w)];
        V4 r;
        switch (op) {
            case OP_CONST: r = {0, 0, 0, i_const(w)}; break;
            case OP_SIN: {
                const float c = frep_cosf(a.w);
                r = {c * a.x, c * a.y, c * a.z, frep_sinf(a.w)};
                break;
            }
            case OP_COS: {
                const float ms = -frep_sinf(a.w);
                r = {ms * a.x, ms * a.y, ms * a.z, frep_cosf(a.w)};
                break;
            }
            case OP_ADD: r = {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; break;
            case OP_SUB: r = {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; break;
            case OP_MUL:
                r = {a.x * b.w + a.w * b.x, a.y * b.w + a.w * b.y, a.z * b.w + a.w * b.z, a.w * b.w};
                break;
            case OP_DIV: {
                const float d = b.w * b.w;
                r = {(a.x * b.w - a.w * b.x) / d, (a.y * b.w - a.w * b.y) / d,
                     (a.z * b.w - a.w * b.z) / d, a.w / b.w};
                break;
            }
            case OP_MIN: r = (a.w < b.w) ? a : b; break;
            case OP_MAX: r = (a.w > b.w) ? a : b; break;
            case OP_EXP: {
                const float e = frep_expf(a.w);
                r = {e * a.x, e * a.y, e * a.z, e};
                break;
            }
            case OP_NEG: r = {-a.x, -a.y, -a.z, -a.w}; break;
            case OP_SQRT: {
                const float sq = std::sqrt(a.w);
                const float d = 2.0f * sq;
                r = {a.x / d, a.y / d, a.z / d, sq};
                break;
            }
            default: r = a; break;  // COPY
        }
        s[i_out(w)] = r;
    }
    g[0] = s[0].x;
    g[1] = s[0].y;
    g[2] = s[0].z;
}

// tape_shorten (shorten.comp:148-191): backward liveness from slot 0 through
// the MIN/MAX choices; kept MIN/MAX with one live side become COPY of it
// (keeping the inB field as it was). Returns the kept count; fills out only
// when it is shorter than the input.
uint32_t shorten(const uint64_t* tape, uint32_t n, uint32_t n_slots, const uint8_t* choices,
                 uint32_t n_mm, std::vector<uint8_t>& live, std::vector<uint8_t>& keep,
                 uint64_t* out) {
    live.assign(std::max<uint32_t>(n_slots, 4), 0);
    keep.assign(n, 0);
    live[0] = 1;
    uint32_t kept = 0;
    int64_t mm = (int64_t)n_mm - 1;
    for (int64_t i = (int64_t)n - 1; i >= 0; i--) {
        const uint64_t w = tape[i];
        const uint32_t op = i_op(w);
        if (live[i_out(w)]) {
            keep[i] = 1;
            kept++;
            uint8_t c;
            switch (op) {
                case OP_CONST: c = 0; break;
                case OP_SIN: case OP_COS: case OP_EXP: case OP_NEG: case OP_SQRT: case OP_COPY:
                    c = MM_FIRST; break;
                case OP_MIN: case OP_MAX: c = choices[mm]; break;
                default: c = MM_BOTH; break;
            }
            live[i_out(w)] = 0;
            if (c & MM_FIRST) live[i_a(w)] = 1;
            if (c & MM_SECOND) live[i_b(w)] = 1;
        }
        if (is_mm(op)) mm--;
    }
    if (kept >= n) return n;
    uint32_t o = 0;
    mm = 0;
    for (uint32_t i = 0; i < n; i++) {
        uint64_t w = tape[i];
        const uint32_t op = i_op(w);
        if (keep[i]) {
            if (is_mm(op)) {
                const uint8_t c = choices[mm];
                if (c == MM_FIRST) {
                    w = (w & ~0xFFull) | OP_COPY;
                } else if (c == MM_SECOND) {
                    w = (w & ~0xFFull & ~(0xFFFFull << 32)) | OP_COPY | ((uint64_t)i_b(w) << 32);
                }
            }
            out[o++] = w;
        }
        if (is_mm(op)) mm++;
    }
    return kept;
}

// ---- tree --------------------------------------------------------------------
struct Tree {
    uint32_t levels = 0;
    uint32_t dims[8] = {};
    float low[3] = {};
    float world_size = 0;
    float cell_size[8] = {};
    uint32_t node_size[8] = {};
    uint32_t node_count[8] = {};
    uint64_t node_ofs[8] = {};
    uint32_t n_slots = 4;
    float tape_time = 0;
    std::vector<uint32_t> nodes;
    std::vector<uint64_t> tapes;
    uint64_t work[8] = {};
};

uint64_t tape_record_words(uint32_t n_instr) { return (1 + (uint64_t)n_instr + 15) / 16 * 16; }

uint64_t append_tape(std::vector<uint64_t>& pool, const uint64_t* instrs, uint32_t n) {
    const uint64_t at = pool.size();
    pool.resize(at + tape_record_words(n), 0);
    pool[at] = n;
    std::memcpy(&pool[at + 1], instrs, (size_t)n * 8);
    return at;
}

struct ChildRec {
    uint32_t cell;
    uint32_t coords[3];
    int64_t new_tape;  // index into NodeOut::tapes, or -1 = parent's tape
};

struct NodeOut {
    std::vector<uint32_t> leaf, interior;
    std::vector<ChildRec> children;
    std::vector<std::vector<uint64_t>> tapes;
    uint64_t work = 0;
};

template <typename F>
void parallel_for(uint32_t n, int threads, F f) {
    if (threads <= 1 || n < 2) {
        for (uint32_t i = 0; i < n; i++) f(i, 0);
        return;
    }
    const uint32_t nt = std::min<uint32_t>((uint32_t)threads, n);
    std::vector<std::thread> pool;
    for (uint32_t k = 0; k < nt; k++) {
        pool.emplace_back([&, k] {
            for (uint32_t i = k; i < n; i += nt) f(i, k);
        });
    }
    for (auto& th : pool) th.join();
}

void process_node(const Tree& T, uint32_t level, uint32_t node, int rounding, int do_shorten,
                  NodeOut& out) {
    const uint32_t dim = T.dims[level];
    const uint32_t cells = dim * dim * dim;
    const uint32_t* rec = &T.nodes[T.node_ofs[level] + (uint64_t)node * T.node_size[level]];
    const uint64_t tape_idx = rec[0];
    const uint32_t n = (uint32_t)T.tapes[tape_idx];
    const uint64_t* tape = &T.tapes[tape_idx + 1];
    const bool last = level == T.levels - 1;
    const float cs = T.cell_size[level];
    out.leaf.assign(cells / 32, 0);
    out.interior.assign(cells / 32, 0);
    out.work = (uint64_t)cells * n;
    uint32_t n_mm = 0;
    for (uint32_t i = 0; i < n; i++) n_mm += is_mm(i_op(tape[i]));
    std::vector<Iv> slots(std::max<uint32_t>(T.n_slots, 4));
    std::vector<float> pslots(std::max<uint32_t>(T.n_slots, 4));
    std::vector<uint8_t> choices(n_mm + 1), live, keep;
    std::vector<uint64_t> short_tape(n);
    for (uint32_t idx = 0; idx < cells; idx++) {
        // bit index z + dim*y + dim^2*x (utils.comp:6)
        const uint32_t cz = idx % dim, cy = (idx / dim) % dim, cx = idx / (dim * dim);
        const uint32_t cc[3] = {rec[1] * dim + cx, rec[2] * dim + cy, rec[3] * dim + cz};
        float lo[3], hi[3];
        for (int k = 0; k < 3; k++) {
            lo[k] = T.low[k] + (float)cc[k] * cs;   // voxelizer/main.comp:115-116
            hi[k] = lo[k] + cs;                      // :125
        }
        if (last) {  // voxelize_point (main.comp:74-83)
            const float d = eval_point(tape, n, pslots, lo[0], lo[1], lo[2], T.tape_time);
            if (d < 0.0f) out.leaf[idx >> 5] |= 1u << (idx & 31);
            continue;
        }
        const Iv d = eval_interval(tape, n, slots, lo, hi, T.tape_time, rounding, choices.data());
        if (d.lo > 0) continue;                                               // empty
        if (d.hi < 0) { out.leaf[idx >> 5] |= 1u << (idx & 31); continue; }   // leaf
        out.interior[idx >> 5] |= 1u << (idx & 31);                          // ambiguous
        ChildRec cr{idx, {cc[0], cc[1], cc[2]}, -1};
        if (do_shorten) {
            const uint32_t k = shorten(tape, n, T.n_slots, choices.data(), n_mm, live, keep, short_tape.data());
            if (k < n) {
                out.tapes.emplace_back(short_tape.begin(), short_tape.begin() + k);
                cr.new_tape = (int64_t)out.tapes.size() - 1;
            }
        }
        out.children.push_back(cr);
    }
}

}  // namespace

extern "C" {

void oracle_eval_interval(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots,
                          const float* lo3, const float* hi3, float t, int rounding,
                          float* out_lohi, uint8_t* choices) {
    std::vector<Iv> slots(std::max<uint32_t>(n_slots, 4));
    Iv r = eval_interval(tape, n_instr, slots, lo3, hi3, t, rounding, choices);
    out_lohi[0] = r.lo;
    out_lohi[1] = r.hi;
}

void oracle_eval_interval_trace(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots,
                                const float* lo3, const float* hi3, float t, int rounding,
                                float* trace) {
    std::vector<Iv> slots(std::max<uint32_t>(n_slots, 4));
    eval_interval(tape, n_instr, slots, lo3, hi3, t, rounding, nullptr, reinterpret_cast<Iv*>(trace));
}

float oracle_eval_point(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots, float x,
                        float y, float z, float t) {
    std::vector<float> s(std::max<uint32_t>(n_slots, 4));
    return eval_point(tape, n_instr, s, x, y, z, t);
}

void oracle_eval_gradient(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots, float x,
                          float y, float z, float t, float* out_grad3) {
    std::vector<V4> s(std::max<uint32_t>(n_slots, 4));
    eval_gradient(tape, n_instr, s, x, y, z, t, out_grad3);
}

uint32_t oracle_shorten(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots,
                        const uint8_t* choices, uint32_t n_minmax, uint64_t* out) {
    std::vector<uint8_t> live, keep;
    return shorten(tape, n_instr, n_slots, choices, n_minmax, live, keep, out);
}

float oracle_directed(int op, int dir, float a, float b) {
    RoundMode mode(FE_DOWNWARD);
    switch (op) {
        case 0: return dir < 0 ? add_dn(a, b) : add_up(a, b);
        case 1: return dir < 0 ? sub_dn(a, b) : sub_up(a, b);
        case 2: return dir < 0 ? mul_dn(a, b) : mul_up(a, b);
        case 3: return dir < 0 ? div_dn(a, b) : div_up(a, b);
        default: return dir < 0 ? sqrt_dn(a) : sqrt_up(a);
    }
}

void* oracle_voxelize(const uint64_t* tape, uint32_t n_instr, uint32_t n_slots,
                      const uint32_t* dims, uint32_t levels, const float* low_vertex,
                      float world_size, float tape_time, int rounding, int do_shorten,
                      int threads) {
    if (levels == 0 || levels > 8 || n_instr == 0) return nullptr;
    auto* T = new Tree();
    T->levels = levels;
    T->n_slots = n_slots;
    T->tape_time = tape_time;
    T->world_size = world_size;
    std::memcpy(T->low, low_vertex, sizeof(T->low));
    float cs = world_size;  // voxelizer.cpp:209-220: successive divisions
    for (uint32_t l = 0; l < levels; l++) {
        T->dims[l] = dims[l];
        cs /= (float)dims[l];
        T->cell_size[l] = cs;
        const uint32_t c3 = dims[l] * dims[l] * dims[l];
        T->node_size[l] = (l == levels - 1) ? 4 + (c3 >> 4) : 4 + 17 * (c3 >> 4);  // node.comp:4-15
    }
    append_tape(T->tapes, tape, n_instr);
    T->node_count[0] = 1;
    T->node_ofs[0] = 0;
    T->nodes.assign(T->node_size[0], 0);  // root: tape 0, coords 0
    for (uint32_t l = 0; l < levels; l++) {
        const uint32_t count = T->node_count[l];
        const uint32_t dim = T->dims[l];
        const uint32_t c3 = dim * dim * dim;
        std::vector<NodeOut> outs(count);
        parallel_for(count, threads, [&](uint32_t i, uint32_t) {
            process_node(*T, l, i, rounding, do_shorten, outs[i]);
        });
        const bool last = l == levels - 1;
        uint64_t next_ofs = T->node_ofs[l] + (uint64_t)count * T->node_size[l];
        uint32_t next_count = 0;
        for (uint32_t i = 0; i < count; i++) next_count += (uint32_t)outs[i].children.size();
        if (!last) {
            T->node_ofs[l + 1] = next_ofs;
            T->node_count[l + 1] = next_count;
            T->nodes.resize(next_ofs + (uint64_t)next_count * T->node_size[l + 1], 0);
        }
        uint32_t child = 0;
        for (uint32_t i = 0; i < count; i++) {
            NodeOut& o = outs[i];
            T->work[l] += o.work;
            uint32_t* rec = &T->nodes[T->node_ofs[l] + (uint64_t)i * T->node_size[l]];
            std::memcpy(rec + 4, o.leaf.data(), (c3 / 32) * 4);
            if (last) continue;
            std::memcpy(rec + 4 + c3 / 32, o.interior.data(), (c3 / 32) * 4);
            uint32_t* list = rec + 4 + c3 / 16;
            for (uint32_t c = 0; c < c3; c++) list[c] = 0xFFFFFFFFu;
            for (const ChildRec& cr : o.children) {
                uint64_t tidx = rec[0];
                if (cr.new_tape >= 0) {
                    const auto& tv = o.tapes[(size_t)cr.new_tape];
                    tidx = append_tape(T->tapes, tv.data(), (uint32_t)tv.size());
                }
                list[cr.cell] = child;
                uint32_t* crec = &T->nodes[T->node_ofs[l + 1] + (uint64_t)child * T->node_size[l + 1]];
                crec[0] = (uint32_t)tidx;
                crec[1] = cr.coords[0];
                crec[2] = cr.coords[1];
                crec[3] = cr.coords[2];
                child++;
            }
        }
    }
    return T;
}

void oracle_tree_free(void* tree) { delete (Tree*)tree; }

void oracle_tree_info(void* tree, uint64_t* info) {
    const Tree* T = (const Tree*)tree;
    info[0] = T->levels;
    for (int l = 0; l < 8; l++) {
        info[1 + l] = T->node_count[l];
        info[9 + l] = T->node_size[l];
        info[17 + l] = T->node_ofs[l];
    }
    info[25] = T->nodes.size();
    info[26] = T->tapes.size();
}

void oracle_tree_nodes(void* tree, uint32_t* dst) {
    const Tree* T = (const Tree*)tree;
    std::memcpy(dst, T->nodes.data(), T->nodes.size() * 4);
}

void oracle_tree_tapes(void* tree, uint64_t* dst) {
    const Tree* T = (const Tree*)tree;
    std::memcpy(dst, T->tapes.data(), T->tapes.size() * 8);
}

void oracle_tree_work(void* tree, uint64_t* cell_instr8) {
    const Tree* T = (const Tree*)tree;
    for (int l = 0; l < 8; l++) cell_instr8[l] = T->work[l];
}

}  // extern "C"

// ---- compaction (vulkan/src/engine/scene_builder.cpp) --------------------------
namespace {

enum : uint8_t { ST_EMPTY = 0, ST_KEPT = 1, ST_FULL = 2 };

struct Compactor {
    const Tree& S;
    int prune;
    std::vector<std::vector<uint8_t>> status;  // per level, per source node (prune only)
    Tree* D = nullptr;
    std::vector<uint32_t> next;                 // LayoutNode's nextNodeIdx

    const uint32_t* rec(uint32_t l, uint32_t node) const {
        return &S.nodes[S.node_ofs[l] + (uint64_t)node * S.node_size[l]];
    }

    // A node's masks after its children are compacted. BuildNode
    // (scene_builder.cpp:91-156): a child whose cells are all leaves becomes a
    // leaf bit (:132-137, HasAllLeafChildren :79-89), an empty child (nullptr,
    // :151-154) clears its bit, any other child stays an interior child.
    void masks(uint32_t l, uint32_t node, std::vector<uint32_t>& leaf, std::vector<uint32_t>& inter) const {
        const uint32_t dim = S.dims[l], c3 = dim * dim * dim, W = c3 / 32;
        const bool last = l == S.levels - 1;
        const uint32_t* r = rec(l, node);
        leaf.assign(r + 4, r + 4 + W);
        inter.assign(W, 0);
        if (last) return;
        for (uint32_t w = 0; w < W; w++) inter[w] = r[4 + W + w];
        if (!prune) return;
        const uint32_t* list = r + 4 + c3 / 16;
        for (uint32_t w = 0; w < W; w++) {
            for (uint32_t b = 0; b < 32; b++) {
                if (!((inter[w] >> b) & 1u)) continue;
                const uint8_t st = status[l + 1][list[w * 32 + b]];
                if (st == ST_FULL) {
                    leaf[w] |= 1u << b;
                    inter[w] &= ~(1u << b);
                } else if (st == ST_EMPTY) {
                    inter[w] &= ~(1u << b);
                }
            }
        }
    }

    void compute_status() {
        status.assign(S.levels, {});
        std::vector<uint32_t> leaf, inter;
        for (int l = (int)S.levels - 1; l >= 0; l--) {
            status[l].assign(S.node_count[l], ST_KEPT);
            for (uint32_t i = 0; i < S.node_count[l]; i++) {
                masks((uint32_t)l, i, leaf, inter);
                bool any = false, full = true;
                for (size_t w = 0; w < leaf.size(); w++) {
                    any = any || leaf[w] || inter[w];
                    full = full && leaf[w] == 0xFFFFFFFFu;
                }
                status[l][i] = !any ? ST_EMPTY : (full ? ST_FULL : ST_KEPT);
            }
        }
    }

    // CountInteriorNodes (scene_builder.cpp:158-168) over the compacted tree.
    void count(uint32_t l, uint32_t node, std::vector<uint32_t>& counts) const {
        counts[l]++;
        if (l == S.levels - 1) return;
        std::vector<uint32_t> leaf, inter;
        masks(l, node, leaf, inter);
        const uint32_t* list = rec(l, node) + 4 + S.dims[l] * S.dims[l] * S.dims[l] / 16;
        for (uint32_t w = 0; w < inter.size(); w++)
            for (uint32_t b = 0; b < 32; b++)
                if ((inter[w] >> b) & 1u) count(l + 1, list[w * 32 + b], counts);
    }

    // LayoutNode (scene_builder.cpp:199-238): the node's index at its level is
    // claimed before its children, which follow in cell order (x, y, z loops =
    // ascending bit index), so every level is numbered in depth-first preorder.
    uint32_t layout(uint32_t l, uint32_t node) {
        const uint32_t idx = next[l]++;
        const uint32_t dim = S.dims[l], c3 = dim * dim * dim, W = c3 / 32;
        std::vector<uint32_t> leaf, inter;
        masks(l, node, leaf, inter);
        const uint32_t* r = rec(l, node);
        uint32_t* d = &D->nodes[D->node_ofs[l] + (uint64_t)idx * D->node_size[l]];
        d[0] = r[0];
        d[1] = r[1];
        d[2] = r[2];
        d[3] = r[3];
        std::memcpy(d + 4, leaf.data(), W * 4);
        if (l == S.levels - 1) return idx;
        std::memcpy(d + 4 + W, inter.data(), W * 4);
        const uint32_t* list = r + 4 + c3 / 16;
        uint32_t* dlist = d + 4 + c3 / 16;
        for (uint32_t c = 0; c < c3; c++) dlist[c] = 0xFFFFFFFFu;
        for (uint32_t w = 0; w < W; w++)
            for (uint32_t b = 0; b < 32; b++)
                if ((inter[w] >> b) & 1u) dlist[w * 32 + b] = layout(l + 1, list[w * 32 + b]);
        return idx;
    }
};

}  // namespace

extern "C" void* oracle_compact(void* tree, int prune) {
    const Tree& S = *(const Tree*)tree;
    Compactor C{S, prune, {}, nullptr, {}};
    if (prune) C.compute_status();
    std::vector<uint32_t> counts(S.levels, 0);
    C.count(0, 0, counts);  // the root is always kept (BuildScene asserts it exists, :24-25)
    auto* D = new Tree();
    D->levels = S.levels;
    std::memcpy(D->dims, S.dims, sizeof(D->dims));
    std::memcpy(D->low, S.low, sizeof(D->low));
    D->world_size = S.world_size;
    std::memcpy(D->cell_size, S.cell_size, sizeof(D->cell_size));
    std::memcpy(D->node_size, S.node_size, sizeof(D->node_size));
    D->n_slots = S.n_slots;
    D->tape_time = S.tape_time;
    std::memcpy(D->work, S.work, sizeof(D->work));
    uint64_t ofs = 0;
    for (uint32_t l = 0; l < S.levels; l++) {
        D->node_count[l] = counts[l];
        D->node_ofs[l] = ofs;
        ofs += (uint64_t)counts[l] * S.node_size[l];
    }
    D->nodes.assign(ofs, 0);
    D->tapes = S.tapes;
    C.D = D;
    C.next.assign(S.levels, 0);
    C.layout(0, 0);
    return D;
}

// ---- raytracer (raytracer/main.comp) -----------------------------------------
namespace {

struct F3 {
    float x, y, z;
};
inline F3 cross3(F3 a, F3 b) {  // glm::cross component order
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 normalize3(F3 v) {
    const float inv = 1.0f / std::sqrt(dot3(v, v));
    return {v.x * inv, v.y * inv, v.z * inv};
}

struct Hit {
    float t;
    uint32_t node, level, cell, steps;
};

struct Tracer {
    const Tree& T;
    uint32_t leaf_bit(uint32_t node, uint32_t lvl, uint32_t idx) const {
        const uint32_t* rec = &T.nodes[T.node_ofs[lvl] + (uint64_t)node * T.node_size[lvl]];
        return (rec[4 + (idx >> 5)] >> (idx & 31)) & 1;
    }
    uint32_t interior_bit(uint32_t node, uint32_t lvl, uint32_t idx) const {
        if (lvl >= T.levels - 1) return 0;
        const uint32_t c3 = T.dims[lvl] * T.dims[lvl] * T.dims[lvl];
        const uint32_t* rec = &T.nodes[T.node_ofs[lvl] + (uint64_t)node * T.node_size[lvl]];
        return (rec[4 + c3 / 32 + (idx >> 5)] >> (idx & 31)) & 1;
    }
    uint32_t child(uint32_t node, uint32_t lvl, uint32_t idx) const {
        const uint32_t c3 = T.dims[lvl] * T.dims[lvl] * T.dims[lvl];
        const uint32_t* rec = &T.nodes[T.node_ofs[lvl] + (uint64_t)node * T.node_size[lvl]];
        return rec[4 + c3 / 16 + idx];
    }

    // raygrid_intersect (main.comp:24-43)
    bool grid_intersect(F3 o, F3 d, float& t_enter, float& t_leave) const {
        const F3 inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
        const float gs = T.world_size;
        float t0x = ((T.low[0] + EPS) - o.x) * inv.x, t0y = ((T.low[1] + EPS) - o.y) * inv.y,
              t0z = ((T.low[2] + EPS) - o.z) * inv.z;
        float t1x = (((T.low[0] + gs) - EPS) - o.x) * inv.x, t1y = (((T.low[1] + gs) - EPS) - o.y) * inv.y,
              t1z = (((T.low[2] + gs) - EPS) - o.z) * inv.z;
        if (inv.x < 0.0f) std::swap(t0x, t1x);
        if (inv.y < 0.0f) std::swap(t0y, t1y);
        if (inv.z < 0.0f) std::swap(t0z, t1z);
        t_enter = max_sel(t0x, max_sel(t0y, t0z));
        t_leave = min_sel(t1x, min_sel(t1y, t1z));
        return t_enter <= t_leave && t_leave >= 0.0f;
    }

    // dda (main.comp:46-111), kd-restart. Deviations, shared with the GPU code:
    // cell coordinates are clamped to [0, dim) so that a rounding slip cannot
    // index outside the node, and the total step count is bounded.
    bool dda(F3 o, F3 d, Hit& hit) const {
        hit.steps = 0;
        float g_enter, g_leave;
        if (!grid_intersect(o, d, g_enter, g_leave)) return false;
        const F3 inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
        const float sx = inv.x >= 0.0f ? 1.0f : 0.0f, sy = inv.y >= 0.0f ? 1.0f : 0.0f,
                    sz = inv.z >= 0.0f ? 1.0f : 0.0f;
        float t_curr = max_sel(g_enter, 0.0f) + EPS;
        float t_max = t_curr;
        uint32_t steps = 0;
        while (t_max < g_leave - EPS) {
            uint32_t lvl = 0, node = 0;
            F3 np = {T.low[0], T.low[1], T.low[2]};
            t_curr = t_max + EPS;
            t_max = g_leave;
            while (t_curr < t_max - EPS) {
                if (++steps > MAX_DDA_STEPS) { hit.steps = steps; return false; }
                const float cs = T.cell_size[lvl];
                const int dim = (int)T.dims[lvl];
                const float te = t_curr + EPS;
                const float nx = ((o.x + te * d.x) - np.x) / cs;
                const float ny = ((o.y + te * d.y) - np.y) / cs;
                const float nz = ((o.z + te * d.z) - np.z) / cs;
                int cx = (int)std::floor(nx), cy = (int)std::floor(ny), cz = (int)std::floor(nz);
                cx = std::min(std::max(cx, 0), dim - 1);
                cy = std::min(std::max(cy, 0), dim - 1);
                cz = std::min(std::max(cz, 0), dim - 1);
                const float tnx = te + ((((float)cx + sx) - nx) * cs) * inv.x;
                const float tny = te + ((((float)cy + sy) - ny) * cs) * inv.y;
                const float tnz = te + ((((float)cz + sz) - nz) * cs) * inv.z;
                const uint32_t idx = (uint32_t)(cz + dim * cy + dim * dim * cx);
                if (leaf_bit(node, lvl, idx)) {
                    hit.t = t_curr;
                    hit.node = node;
                    hit.level = lvl;
                    hit.cell = idx;
                    hit.steps = steps;
                    return true;
                } else if (interior_bit(node, lvl, idx)) {
                    node = child(node, lvl, idx);
                    np.x = np.x + (float)cx * cs;
                    np.y = np.y + (float)cy * cs;
                    np.z = np.z + (float)cz * cs;
                    t_max = min_sel(tnx, min_sel(tny, tnz));
                    lvl++;
                } else {
                    t_curr = min_sel(tnx, min_sel(tny, tnz));
                }
            }
        }
        hit.steps = steps;
        return false;
    }
};

// rand() of random.comp:10-15 with the library's sine.
inline float rand_step(float& seed, uint32_t gx, uint32_t gy) {
    const float dotv = (float)gx * 12.9898f + (float)gy * 78.233f;
    const float v = frep_sinf(seed / 100.0f * dotv) * 43758.5453f;
    seed += 1.0f;
    return v - std::floor(v);
}

inline uint8_t to_unorm8(float c) {
    if (!(c > 0.0f)) return 0;
    if (c >= 1.0f) return 255;
    return (uint8_t)(c * 255.0f + 0.5f);
}

}  // namespace

extern "C" void oracle_render(void* tree, const float* cam, uint32_t n_lights,
                              const float* light_dir, const float* light_color,
                              const float* ambient, const float* background, uint32_t shadow_mask,
                              float tape_time, uint8_t* rgba8, uint32_t* hits, int threads) {
    const Tree& T = *(const Tree*)tree;
    Tracer tr{T};
    const F3 pos = {cam[0], cam[1], cam[2]};
    // Camera::Init + Right() + Up() (camera.cpp:8-27)
    const F3 fwd = normalize3({cam[3], cam[4], cam[5]});
    const F3 up0 = normalize3({cam[6], cam[7], cam[8]});
    const F3 right = normalize3(cross3(fwd, up0));
    const F3 up = cross3(right, fwd);
    const float fov = cam[9], ortho_w = cam[10];
    const uint32_t proj = (uint32_t)cam[11], W = (uint32_t)cam[12], H = (uint32_t)cam[13];
    const uint32_t jitter = (uint32_t)cam[14];
    const float seed0 = cam[15];
    // raytracer.cpp:177-181 (glm::radians multiplies by pi/180 in float)
    const float sws_x = 2.0f * std::tan((fov * 0.01745329251994329577f) / 2.0f);
    const float aspect = (float)H / (float)W;
    const float sws_y = sws_x * aspect;
    const float half_w = ortho_w / 2.0f, half_h = (ortho_w * aspect) / 2.0f;
    std::vector<F3> L(n_lights);
    for (uint32_t i = 0; i < n_lights; i++)
        L[i] = normalize3({light_dir[3 * i], light_dir[3 * i + 1], light_dir[3 * i + 2]});

    parallel_for(H, threads, [&](uint32_t y, uint32_t) {
        std::vector<V4> gslots(std::max<uint32_t>(T.n_slots, 4));
        for (uint32_t x = 0; x < W; x++) {
            float ox = 0.0f, oy = 0.0f;
            if (jitter) {
                float seed = seed0;
                const float r0 = rand_step(seed, x, y);
                const float r1 = rand_step(seed, x, y);
                ox = 2.0f * (r0 - 0.5f);
                oy = 2.0f * (r1 - 0.5f);
            }
            const float dx = 2.0f * (((float)x + ox) / (float)W) - 1.0f;
            const float dy = 2.0f * (((float)y + oy) / (float)H) - 1.0f;
            F3 o, d;
            if (proj == 0) {  // main.comp:173-178
                o = pos;
                const float ax = dx * sws_x, ay = dy * sws_y;
                d = normalize3({(fwd.x + ax * right.x) + ay * up.x, (fwd.y + ax * right.y) + ay * up.y,
                                (fwd.z + ax * right.z) + ay * up.z});
            } else {  // orthographic: parallel rays through the pixel
                const float ax = dx * half_w, ay = dy * half_h;
                o = {(pos.x + ax * right.x) + ay * up.x, (pos.y + ax * right.y) + ay * up.y,
                     (pos.z + ax * right.z) + ay * up.z};
                d = fwd;
            }
            Hit h{};
            float col[4];
            float nrm[3] = {0, 0, 0};
            const bool did = tr.dda(o, d, h);
            if (!did) {
                for (int c = 0; c < 4; c++) col[c] = background[c];
            } else if (h.t < 0.0f) {  // main.comp:149-151
                for (int c = 0; c < 4; c++) col[c] = 1.0f;
            } else {  // shade (main.comp:115-139)
                const uint32_t* rec = &T.nodes[T.node_ofs[h.level] + (uint64_t)h.node * T.node_size[h.level]];
                const uint64_t tidx = rec[0];
                const F3 p = {o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z};
                float g[3];
                eval_gradient(&T.tapes[tidx + 1], (uint32_t)T.tapes[tidx], gslots, p.x, p.y, p.z,
                              tape_time, g);
                const F3 n = normalize3({g[0], g[1], g[2]});
                nrm[0] = n.x; nrm[1] = n.y; nrm[2] = n.z;
                float diff[4] = {0, 0, 0, 0};
                for (uint32_t i = 0; i < n_lights; i++) {
                    if (shadow_mask & (1u << i)) {
                        const float ts = h.t - EPS;
                        const F3 so = {o.x + ts * d.x, o.y + ts * d.y, o.z + ts * d.z};
                        Hit sh{};
                        if (tr.dda(so, {-L[i].x, -L[i].y, -L[i].z}, sh)) continue;
                    }
                    const float dd = (-L[i].x) * n.x + (-L[i].y) * n.y + (-L[i].z) * n.z;
                    const float inten = std::fmax(dd, 0.0f);
                    for (int c = 0; c < 4; c++) diff[c] = diff[c] + inten * light_color[4 * i + c];
                }
                for (int c = 0; c < 4; c++) col[c] = ambient[c] + diff[c];
            }
            const size_t pix = (size_t)y * W + x;
            if (rgba8)
                for (int c = 0; c < 4; c++) rgba8[4 * pix + c] = to_unorm8(col[c]);
            if (hits) {
                uint32_t* hr = &hits[8 * pix];
                float tt = did ? h.t : 0.0f;
                std::memcpy(&hr[0], &tt, 4);
                std::memcpy(&hr[1], nrm, 12);
                hr[4] = did ? h.level : 0xFFFFFFFFu;
                hr[5] = did ? h.node : 0xFFFFFFFFu;
                hr[6] = did ? h.cell : 0xFFFFFFFFu;
                hr[7] = h.steps;
            }
        }
    });
}
