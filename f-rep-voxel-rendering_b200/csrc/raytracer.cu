// Raytracer kernel (sm_100a): one thread per pixel.
//
// Replaces vulkan/shaders/raytracer/main.comp (+ tape/gradient.comp,
// random.comp) and Raytracer::Trace (vulkan/src/engine/raytracer.cpp:243-272):
// ray generation, kd-restart DDA through the multi-level tree, forward-mode
// gradient of the hit node's tape for the normal, diffuse + ambient shading,
// optional shadow rays, rgba8 (and hit records) into device buffers.
//
// Blocks are 8 x 8 pixel tiles, so that neighbouring rays (which walk the same
// nodes and usually share the hit node's tape) sit in the same warp.
#include <algorithm>
#include "device_common.cuh"
#include "kernels.h"

namespace frep {
namespace dev {

struct RHit {
    float t;
    uint32_t node, level, cell, steps;
};

struct Tree {
    const uint32_t* nodes;
    const RenderArgs* a;
    unsigned long long ofs[MAX_LEVELS];

    __device__ const uint32_t* rec(uint32_t lvl, uint32_t node) const {
        return nodes + ofs[lvl] + (size_t)node * a->node_size[lvl];
    }
};

// Where a node record keeps its masks and children. CMP = false: the
// reference's layout (node.comp:4-72), [tape, coords, leaf, interior,
// childList[dim^3]]; CMP = true: the compact layout, [tape, leaf[W],
// interior[W], prefix[W], base] (last level [tape, leaf[W]]), W = dim^3 / 32,
// whose interior children are numbered consecutively from `base` in cell
// order, prefix[w] = interior cells before word w.
template <bool CMP>
struct Layout;
template <>
struct Layout<false> {
    static __device__ __forceinline__ bool leaf(const uint32_t* r, uint32_t c3, uint32_t idx) {
        return (__ldg(&r[4 + (idx >> 5)]) >> (idx & 31)) & 1u;
    }
    // The child node of an interior cell, or ~0 when the cell is not interior.
    static __device__ __forceinline__ uint32_t child(const uint32_t* r, uint32_t c3, uint32_t idx) {
        if (!((__ldg(&r[4 + c3 / 32 + (idx >> 5)]) >> (idx & 31)) & 1u)) return ~0u;
        return __ldg(&r[4 + c3 / 16 + idx]);
    }
};
template <>
struct Layout<true> {
    static __device__ __forceinline__ bool leaf(const uint32_t* r, uint32_t c3, uint32_t idx) {
        return (__ldg(&r[1 + (idx >> 5)]) >> (idx & 31)) & 1u;
    }
    static __device__ __forceinline__ uint32_t child(const uint32_t* r, uint32_t c3, uint32_t idx) {
        const uint32_t W = c3 >> 5;
        const uint32_t iw = __ldg(&r[1 + W + (idx >> 5)]);
        if (!((iw >> (idx & 31)) & 1u)) return ~0u;
        return __ldg(&r[1 + 3 * W]) + __ldg(&r[1 + 2 * W + (idx >> 5)]) + __popc(iw & ((1u << (idx & 31)) - 1u));
    }
};

// raygrid_intersect (main.comp:24-43).
__device__ bool grid_intersect(const RenderArgs& A, float3 o, float3 inv, float& te, float& tl) {
    const float gs = A.world_size;
    float t0x = __fmul_rn(__fsub_rn(__fadd_rn(A.low[0], EPS), o.x), inv.x);
    float t0y = __fmul_rn(__fsub_rn(__fadd_rn(A.low[1], EPS), o.y), inv.y);
    float t0z = __fmul_rn(__fsub_rn(__fadd_rn(A.low[2], EPS), o.z), inv.z);
    float t1x = __fmul_rn(__fsub_rn(__fsub_rn(__fadd_rn(A.low[0], gs), EPS), o.x), inv.x);
    float t1y = __fmul_rn(__fsub_rn(__fsub_rn(__fadd_rn(A.low[1], gs), EPS), o.y), inv.y);
    float t1z = __fmul_rn(__fsub_rn(__fsub_rn(__fadd_rn(A.low[2], gs), EPS), o.z), inv.z);
    if (inv.x < 0.0f) { const float t = t0x; t0x = t1x; t1x = t; }
    if (inv.y < 0.0f) { const float t = t0y; t0y = t1y; t1y = t; }
    if (inv.z < 0.0f) { const float t = t0z; t0z = t1z; t1z = t; }
    te = max_sel(t0x, max_sel(t0y, t0z));
    tl = min_sel(t1x, min_sel(t1y, t1z));
    return te <= tl && tl >= 0.0f;
}

// dda (main.comp:46-111), kd-restart. Cell coordinates are clamped to
// [0, dim) and the step count is bounded (both also in the oracle).
template <bool CMP>
__device__ bool dda(const Tree& T, float3 o, float3 d, RHit& hit) {
    const RenderArgs& A = *T.a;
    hit.steps = 0;
    const float3 inv = make_float3(__fdiv_rn(1.0f, d.x), __fdiv_rn(1.0f, d.y), __fdiv_rn(1.0f, d.z));
    float g_enter, g_leave;
    if (!grid_intersect(A, o, inv, g_enter, g_leave)) return false;
    const float sx = inv.x >= 0.0f ? 1.0f : 0.0f, sy = inv.y >= 0.0f ? 1.0f : 0.0f,
                sz = inv.z >= 0.0f ? 1.0f : 0.0f;
    float t_curr = __fadd_rn(max_sel(g_enter, 0.0f), EPS);
    float t_max = t_curr;
    uint32_t steps = 0;
    const uint32_t last = A.levels - 1;
    while (t_max < __fsub_rn(g_leave, EPS)) {
        uint32_t lvl = 0, node = 0;
        float npx = A.low[0], npy = A.low[1], npz = A.low[2];
        t_curr = __fadd_rn(t_max, EPS);
        t_max = g_leave;
        while (t_curr < __fsub_rn(t_max, EPS)) {
            if (++steps > MAX_DDA_STEPS) { hit.steps = steps; return false; }
            const float cs = A.cell_size[lvl];
            const int dim = (int)A.dims[lvl];
            const float te = __fadd_rn(t_curr, EPS);
            const float nx = __fdiv_rn(__fsub_rn(__fadd_rn(o.x, __fmul_rn(te, d.x)), npx), cs);
            const float ny = __fdiv_rn(__fsub_rn(__fadd_rn(o.y, __fmul_rn(te, d.y)), npy), cs);
            const float nz = __fdiv_rn(__fsub_rn(__fadd_rn(o.z, __fmul_rn(te, d.z)), npz), cs);
            int cx = (int)floorf(nx), cy = (int)floorf(ny), cz = (int)floorf(nz);
            cx = min(max(cx, 0), dim - 1);
            cy = min(max(cy, 0), dim - 1);
            cz = min(max(cz, 0), dim - 1);
            const float tnx = __fadd_rn(te, __fmul_rn(__fmul_rn(__fsub_rn(__fadd_rn((float)cx, sx), nx), cs), inv.x));
            const float tny = __fadd_rn(te, __fmul_rn(__fmul_rn(__fsub_rn(__fadd_rn((float)cy, sy), ny), cs), inv.y));
            const float tnz = __fadd_rn(te, __fmul_rn(__fmul_rn(__fsub_rn(__fadd_rn((float)cz, sz), nz), cs), inv.z));
            const uint32_t idx = (uint32_t)(cz + dim * cy + dim * dim * cx);
            const uint32_t* r = T.rec(lvl, node);
            const uint32_t c3 = (uint32_t)(dim * dim * dim);
            if (Layout<CMP>::leaf(r, c3, idx)) {
                hit.t = t_curr;
                hit.node = node;
                hit.level = lvl;
                hit.cell = idx;
                hit.steps = steps;
                return true;
            }
            const uint32_t ch = lvl < last ? Layout<CMP>::child(r, c3, idx) : ~0u;
            if (ch != ~0u) {
                node = ch;
                npx = __fadd_rn(npx, __fmul_rn((float)cx, cs));
                npy = __fadd_rn(npy, __fmul_rn((float)cy, cs));
                npz = __fadd_rn(npz, __fmul_rn((float)cz, cs));
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

// tape_eval_gradient (gradient.comp:4-88) with a per-thread slot array of NS
// entries (local memory).
template <int NS>
__device__ float3 gradient(const uint64_t* tape, uint32_t n, float x, float y, float z, float t) {
    float4 s[NS];
    s[0] = make_float4(1, 0, 0, x);
    s[1] = make_float4(0, 1, 0, y);
    s[2] = make_float4(0, 0, 1, z);
    s[3] = make_float4(0, 0, 0, t);
    for (uint32_t i = 0; i < n; i++) {
        const uint64_t w = __ldg(&tape[i]);
        const uint32_t op = w_op(w);
        float4 r;
        if (op == OP_CONST) {
            r = make_float4(0, 0, 0, w_const(w));
        } else {
            const float4 a = s[w_a(w)], b = s[w_b(w)];
            switch (op) {
                case OP_SIN: {
                    const float c = frep_cosf(a.w);
                    r = make_float4(__fmul_rn(c, a.x), __fmul_rn(c, a.y), __fmul_rn(c, a.z), frep_sinf(a.w));
                    break;
                }
                case OP_COS: {
                    const float ms = -frep_sinf(a.w);
                    r = make_float4(__fmul_rn(ms, a.x), __fmul_rn(ms, a.y), __fmul_rn(ms, a.z), frep_cosf(a.w));
                    break;
                }
                case OP_ADD:
                    r = make_float4(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z), __fadd_rn(a.w, b.w));
                    break;
                case OP_SUB:
                    r = make_float4(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z), __fsub_rn(a.w, b.w));
                    break;
                case OP_MUL:
                    r = make_float4(__fadd_rn(__fmul_rn(a.x, b.w), __fmul_rn(a.w, b.x)),
                                    __fadd_rn(__fmul_rn(a.y, b.w), __fmul_rn(a.w, b.y)),
                                    __fadd_rn(__fmul_rn(a.z, b.w), __fmul_rn(a.w, b.z)), __fmul_rn(a.w, b.w));
                    break;
                case OP_DIV: {
                    const float dd = __fmul_rn(b.w, b.w);
                    r = make_float4(__fdiv_rn(__fsub_rn(__fmul_rn(a.x, b.w), __fmul_rn(a.w, b.x)), dd),
                                    __fdiv_rn(__fsub_rn(__fmul_rn(a.y, b.w), __fmul_rn(a.w, b.y)), dd),
                                    __fdiv_rn(__fsub_rn(__fmul_rn(a.z, b.w), __fmul_rn(a.w, b.z)), dd),
                                    __fdiv_rn(a.w, b.w));
                    break;
                }
                case OP_MIN: r = (a.w < b.w) ? a : b; break;
                case OP_MAX: r = (a.w > b.w) ? a : b; break;
                case OP_EXP: {
                    const float e = frep_expf(a.w);
                    r = make_float4(__fmul_rn(e, a.x), __fmul_rn(e, a.y), __fmul_rn(e, a.z), e);
                    break;
                }
                case OP_NEG: r = make_float4(-a.x, -a.y, -a.z, -a.w); break;
                case OP_SQRT: {
                    const float sq = __fsqrt_rn(a.w);
                    const float dd = __fmul_rn(2.0f, sq);
                    r = make_float4(__fdiv_rn(a.x, dd), __fdiv_rn(a.y, dd), __fdiv_rn(a.z, dd), sq);
                    break;
                }
                default: r = a; break;  // COPY
            }
        }
        s[w_out(w)] = r;
    }
    return make_float3(s[0].x, s[0].y, s[0].z);
}

__device__ __forceinline__ float dot3(float3 a, float3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ float3 normalize3(float3 v) {
    const float inv = __fdiv_rn(1.0f, __fsqrt_rn(dot3(v, v)));
    return make_float3(__fmul_rn(v.x, inv), __fmul_rn(v.y, inv), __fmul_rn(v.z, inv));
}

// rand() of random.comp:10-15, with the library's sine.
__device__ __forceinline__ float rand_step(float& seed, uint32_t gx, uint32_t gy) {
    const float dotv = __fadd_rn(__fmul_rn((float)gx, 12.9898f), __fmul_rn((float)gy, 78.233f));
    const float v = __fmul_rn(frep_sinf(__fmul_rn(__fdiv_rn(seed, 100.0f), dotv)), 43758.5453f);
    seed = __fadd_rn(seed, 1.0f);
    return __fsub_rn(v, floorf(v));
}

__device__ __forceinline__ uint8_t to_unorm8(float c) {
    if (!(c > 0.0f)) return 0;
    if (c >= 1.0f) return 255;
    return (uint8_t)__fadd_rn(__fmul_rn(c, 255.0f), 0.5f);
}

struct HitRecord {  // == frep_hit
    float t;
    float n[3];
    uint32_t level, node, cell, steps;
};

template <int NS, bool CMP>
__device__ __forceinline__ void render_pixel(const RenderArgs& A, uint32_t x, uint32_t y) {
    Tree T;
    T.nodes = A.nodes;
    T.a = &A;
    for (uint32_t l = 0; l < A.levels; l++) T.ofs[l] = CMP ? A.node_ofs[l] : A.hdr->node_ofs[l];

    // Ray generation (main.comp:168-178).
    float ox = 0.0f, oy = 0.0f;
    if (A.jitter) {
        float seed = A.jitter_seed;
        const float r0 = rand_step(seed, x, y);
        const float r1 = rand_step(seed, x, y);
        ox = __fmul_rn(2.0f, __fsub_rn(r0, 0.5f));
        oy = __fmul_rn(2.0f, __fsub_rn(r1, 0.5f));
    }
    const float dx = __fsub_rn(__fmul_rn(2.0f, __fdiv_rn(__fadd_rn((float)x, ox), (float)A.width)), 1.0f);
    const float dy = __fsub_rn(__fmul_rn(2.0f, __fdiv_rn(__fadd_rn((float)y, oy), (float)A.height)), 1.0f);
    float3 o, d;
    if (A.projection == 0) {
        o = make_float3(A.pos[0], A.pos[1], A.pos[2]);
        const float ax = __fmul_rn(dx, A.sws_x), ay = __fmul_rn(dy, A.sws_y);
        d = normalize3(make_float3(__fadd_rn(__fadd_rn(A.fwd[0], __fmul_rn(ax, A.right[0])), __fmul_rn(ay, A.up[0])),
                                   __fadd_rn(__fadd_rn(A.fwd[1], __fmul_rn(ax, A.right[1])), __fmul_rn(ay, A.up[1])),
                                   __fadd_rn(__fadd_rn(A.fwd[2], __fmul_rn(ax, A.right[2])), __fmul_rn(ay, A.up[2]))));
    } else {
        const float ax = __fmul_rn(dx, A.half_w), ay = __fmul_rn(dy, A.half_h);
        o = make_float3(__fadd_rn(__fadd_rn(A.pos[0], __fmul_rn(ax, A.right[0])), __fmul_rn(ay, A.up[0])),
                        __fadd_rn(__fadd_rn(A.pos[1], __fmul_rn(ax, A.right[1])), __fmul_rn(ay, A.up[1])),
                        __fadd_rn(__fadd_rn(A.pos[2], __fmul_rn(ax, A.right[2])), __fmul_rn(ay, A.up[2])));
        d = make_float3(A.fwd[0], A.fwd[1], A.fwd[2]);
    }

    RHit h;
    const bool did = dda<CMP>(T, o, d, h);
    float col[4];
    float3 n = make_float3(0.0f, 0.0f, 0.0f);
    if (!did) {
        for (int c = 0; c < 4; c++) col[c] = A.background[c];
    } else if (h.t < 0.0f) {  // main.comp:149-151
        for (int c = 0; c < 4; c++) col[c] = 1.0f;
    } else {  // shade (main.comp:115-139)
        const uint32_t tidx = __ldg(&T.rec(h.level, h.node)[0]);
        const uint32_t tn = (uint32_t)__ldg(&A.tapes[tidx]);
        const float px = __fadd_rn(o.x, __fmul_rn(h.t, d.x));
        const float py = __fadd_rn(o.y, __fmul_rn(h.t, d.y));
        const float pz = __fadd_rn(o.z, __fmul_rn(h.t, d.z));
        n = normalize3(gradient<NS>(A.tapes + tidx + 1, tn, px, py, pz, A.tape_time));
        float diff[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        for (uint32_t i = 0; i < A.n_lights; i++) {
            const float3 L = make_float3(A.light_dir[i][0], A.light_dir[i][1], A.light_dir[i][2]);
            if (A.shadow_mask & (1u << i)) {
                const float ts = __fsub_rn(h.t, EPS);
                const float3 so = make_float3(__fadd_rn(o.x, __fmul_rn(ts, d.x)), __fadd_rn(o.y, __fmul_rn(ts, d.y)),
                                              __fadd_rn(o.z, __fmul_rn(ts, d.z)));
                RHit sh;
                if (dda<CMP>(T, so, make_float3(-L.x, -L.y, -L.z), sh)) continue;
            }
            const float dd = dot3(make_float3(-L.x, -L.y, -L.z), n);
            const float inten = fmaxf(dd, 0.0f);
            for (int c = 0; c < 4; c++) diff[c] = __fadd_rn(diff[c], __fmul_rn(inten, A.light_color[i][c]));
        }
        for (int c = 0; c < 4; c++) col[c] = __fadd_rn(A.ambient[c], diff[c]);
    }
    const size_t pix = (size_t)y * A.width + x;
    if (A.rgba8) {
        uchar4 v = make_uchar4(to_unorm8(col[0]), to_unorm8(col[1]), to_unorm8(col[2]), to_unorm8(col[3]));
        reinterpret_cast<uchar4*>(A.rgba8)[pix] = v;
    }
    if (A.hits) {
        HitRecord r;
        r.t = did ? h.t : 0.0f;
        r.n[0] = n.x;
        r.n[1] = n.y;
        r.n[2] = n.z;
        r.level = did ? h.level : 0xFFFFFFFFu;
        r.node = did ? h.node : 0xFFFFFFFFu;
        r.cell = did ? h.cell : 0xFFFFFFFFu;
        r.steps = h.steps;
        reinterpret_cast<HitRecord*>(A.hits)[pix] = r;
    }
}

template <int NS, bool CMP = false>
__global__ void __launch_bounds__(64) render_kernel(const RenderArgs A) {
    const uint32_t x = blockIdx.x * 8 + (threadIdx.x & 7);
    const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 3);
    if (x >= A.width || y >= A.height) return;
    render_pixel<NS, CMP>(A, x, y);
}

// Many frames in one launch: blockIdx.z selects the frame.
template <int NS>
__global__ void __launch_bounds__(64) render_batch_kernel(const RenderArgs* args) {
    const RenderArgs& A = args[blockIdx.z];
    const uint32_t x = blockIdx.x * 8 + (threadIdx.x & 7);
    const uint32_t y = blockIdx.y * 8 + (threadIdx.x >> 3);
    if (x >= A.width || y >= A.height) return;
    render_pixel<NS, false>(A, x, y);
}

// Temporal resolve (renderer/triangle.frag:14-23): the pixel is the mean of
// the layers' rgb with alpha 1. The mean is exact (integer sum) and rounded
// to nearest, ties up: (2 sum + n) / 2n; the reference leaves the float ->
// unorm rounding to the driver. One thread per pixel, 4 bytes each.
__global__ void resolve_layers_kernel(const uchar4* __restrict__ layers, uint32_t n, uint32_t pixels,
                                      uchar4* __restrict__ out) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < pixels; p += gridDim.x * blockDim.x) {
        uint32_t r = 0, g = 0, b = 0;
        for (uint32_t i = 0; i < n; i++) {
            const uchar4 v = layers[(size_t)i * pixels + p];
            r += v.x;
            g += v.y;
            b += v.z;
        }
        const uint32_t den = 2 * n;
        out[p] = make_uchar4((uint8_t)((2 * r + n) / den), (uint8_t)((2 * g + n) / den), (uint8_t)((2 * b + n) / den),
                             255);
    }
}

}  // namespace dev

cudaError_t launch_resolve_layers(const uint8_t* layers, uint32_t n, uint32_t pixels, uint8_t* out,
                                  cudaStream_t stream) {
    if (n == 0 || pixels == 0) return cudaSuccess;
    const uint32_t blocks = (uint32_t)std::min<uint64_t>((pixels + 255) / 256, 148ull * 16);
    dev::resolve_layers_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<const uchar4*>(layers), n, pixels,
                                                            reinterpret_cast<uchar4*>(out));
    return cudaGetLastError();
}

cudaError_t launch_render(const RenderArgs& a, cudaStream_t stream) {
    const dim3 grid((a.width + 7) / 8, (a.height + 7) / 8);
    const uint32_t ns = a.n_slots;
    if (a.compact) {
        if (ns <= 32) dev::render_kernel<32, true><<<grid, 64, 0, stream>>>(a);
        else if (ns <= 64) dev::render_kernel<64, true><<<grid, 64, 0, stream>>>(a);
        else if (ns <= 128) dev::render_kernel<128, true><<<grid, 64, 0, stream>>>(a);
        else if (ns <= 256) dev::render_kernel<256, true><<<grid, 64, 0, stream>>>(a);
        else if (ns <= 512) dev::render_kernel<512, true><<<grid, 64, 0, stream>>>(a);
        else if (ns <= 1024) dev::render_kernel<1024, true><<<grid, 64, 0, stream>>>(a);
        else return cudaErrorInvalidValue;
        return cudaGetLastError();
    }
    if (ns <= 32) dev::render_kernel<32><<<grid, 64, 0, stream>>>(a);
    else if (ns <= 64) dev::render_kernel<64><<<grid, 64, 0, stream>>>(a);
    else if (ns <= 128) dev::render_kernel<128><<<grid, 64, 0, stream>>>(a);
    else if (ns <= 256) dev::render_kernel<256><<<grid, 64, 0, stream>>>(a);
    else if (ns <= 512) dev::render_kernel<512><<<grid, 64, 0, stream>>>(a);
    else if (ns <= 1024) dev::render_kernel<1024><<<grid, 64, 0, stream>>>(a);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

cudaError_t launch_render_batch(const RenderArgs* args, uint32_t n, uint32_t max_w, uint32_t max_h,
                                uint32_t max_slots, cudaStream_t stream) {
    if (n == 0) return cudaSuccess;
    if (n > 65535) return cudaErrorInvalidValue;
    const dim3 grid((max_w + 7) / 8, (max_h + 7) / 8, n);
    if (max_slots <= 32) dev::render_batch_kernel<32><<<grid, 64, 0, stream>>>(args);
    else if (max_slots <= 64) dev::render_batch_kernel<64><<<grid, 64, 0, stream>>>(args);
    else if (max_slots <= 128) dev::render_batch_kernel<128><<<grid, 64, 0, stream>>>(args);
    else if (max_slots <= 256) dev::render_batch_kernel<256><<<grid, 64, 0, stream>>>(args);
    else if (max_slots <= 512) dev::render_batch_kernel<512><<<grid, 64, 0, stream>>>(args);
    else if (max_slots <= 1024) dev::render_batch_kernel<1024><<<grid, 64, 0, stream>>>(args);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace frep
