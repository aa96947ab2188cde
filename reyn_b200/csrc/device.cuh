// Device-side building blocks of the reyn_b200 engine: smoothing kernels,
// the uniform-grid view and the fixed-radius neighbour traversal.
#pragma once

#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>

#include "reyn_b200.h"

namespace reyn {

// ---- smoothing kernels ----------------------------------------------------
// Kernel<D> (reference kernels.cuh:19-65) precomputes 1/h, alpha/h^3 and
// alpha/h^4; the four shape functions w(q), dw(q) follow kernels.cuh:78-165.

enum KernelKind : int { K_C2 = 0, K_B3 = 1, K_W6 = 2, K_COS = 3 };

struct KernelConst {
    float h_inv;    // 1 / h_bar
    float w_scale;  // alpha / h_bar^3
    float dw_scale; // alpha / h_bar^4
};

// normalisation alpha of each kernel, rounded to float exactly as the
// reference's constructors do (kernels.cuh:81, 104, 124, 151)
inline float kernel_alpha(int kind)
{
    switch (kind) {
    case K_C2: return (float)(21.f / 2.f * M_1_PI);
    case K_B3: return (float)(16.f * M_1_PI);
    case K_W6: return (float)(1365.f / 64.f * M_1_PI);
    case K_COS: return (float)(M_PI / (4.f * M_PI * M_PI - 30.f));
    default: return 0.f;
    }
}

inline KernelConst make_kernel(int kind, float h_bar)
{
    const float a = kernel_alpha(kind);
    return KernelConst { 1.0f / h_bar, a / (h_bar * h_bar * h_bar),
        a / (h_bar * h_bar * h_bar * h_bar) };
}

// clamp to [0, 1]: __saturatef on the device, fmin/fmax on the host (the
// same split as the reference's `sat`, vector.cuh:236-243)
__host__ __device__ __forceinline__ float sat01(float a)
{
#ifdef __CUDA_ARCH__
    return __saturatef(a);
#else
    return fminf(fmaxf(a, 0.f), 1.f);
#endif
}

template <int KIND> struct Shape;

template <> struct Shape<K_C2> { // w = (1-q)_+^4 (4q+1)
    __host__ __device__ static float w(float q)
    {
        const float t = fmaxf(0.f, 1.f - q);
        const float t2 = t * t;
        return t2 * t2 * (4.f * q + 1.f);
    }
    __host__ __device__ static float dw(float q)
    {
        const float t = fmaxf(0.f, 1.f - q);
        return t * t * t * (-20.f * q);
    }
    // dw(q) / q: the gradient's 1/|x| cancels against q = |x| / h_bar
    static constexpr bool kDwOverQ = true;
    __host__ __device__ static float dw_over_q(float q)
    {
        const float t = fmaxf(0.f, 1.f - q);
        return t * t * t * -20.f;
    }
};

template <> struct Shape<K_B3> { // w = (1-q)_+^3 - 4 (1/2-q)_+^3
    __host__ __device__ static float w(float q)
    {
        const float t = fmaxf(0.f, 1.f - q);
        const float u = sat01(0.5f - q);
        return t * t * t - 4.f * u * u * u;
    }
    __host__ __device__ static float dw(float q)
    {
        const float t = fmaxf(0.f, 1.f - q);
        const float u = sat01(0.5f - q);
        return -3.f * t * t + 12.f * u * u;
    }
};

template <> struct Shape<K_W6> { // w = (1-q)_+^8 (32q^3 + 25q^2 + 8q + 1)
    __host__ __device__ static float w(float q)
    {
        const float t = fmaxf(0.f, 1.f - q);
        const float t2 = t * t;
        const float t4 = t2 * t2;
        const float q2 = q * q;
        return (t4 * t4) * (32.f * q2 * q + 25.f * q2 + 8.f * q + 1.f);
    }
    __host__ __device__ static float dw(float q)
    {
        const float t = fmaxf(0.f, 1.f - q);
        const float t2 = t * t;
        const float t7 = t2 * t2 * t2 * t;
        return t7 * ((16.f * q * q + 7.f * q + 1.f) * (-22.f * q));
    }
    static constexpr bool kDwOverQ = true;
    __host__ __device__ static float dw_over_q(float q)
    {
        const float t = fmaxf(0.f, 1.f - q);
        const float t2 = t * t;
        const float t7 = t2 * t2 * t2 * t;
        return t7 * ((16.f * q * q + 7.f * q + 1.f) * -22.f);
    }
};

template <> struct Shape<K_COS> { // w = 4 cos(pi q) + cos(2 pi q) + 3
    __host__ __device__ static float w(float q)
    {
        const float s = (float)M_PI * fminf(1.f, q);
        return 4.f * cosf(s) + cosf(2.f * s) + 3.f;
    }
    __host__ __device__ static float dw(float q)
    {
        const float s = (float)M_PI * fminf(1.f, q);
        const float tp = (float)(2.0 * M_PI);
        return -2.f * tp * sinf(s) - sinf(2.f * s) * tp;
    }
};

// W and the gradient factor g (grad W = g * x_ij) for a neighbour pair with
// squared distance 0 <= l2 <= r^2 (the traversal guarantees the range).
// len = l2 * rsqrt(l2) replaces the reference's norm3df; the self pair
// (l2 = 0) has W = W(0) and a zero gradient, as kernels.cuh:60-63 defines.
template <int KIND>
__device__ __forceinline__ float pair_w(const KernelConst& k, float l2)
{
    const float len = l2 > 0.f ? l2 * rsqrtf(l2) : 0.f;
    return k.w_scale * Shape<KIND>::w(__saturatef(len * k.h_inv));
}

template <int KIND, class = void> struct HasDwOverQ {
    static constexpr bool value = false;
};
template <int KIND>
struct HasDwOverQ<KIND, decltype(void(Shape<KIND>::kDwOverQ))> {
    static constexpr bool value = Shape<KIND>::kDwOverQ;
};

// the gradient factor g with grad W(x) = g x. For the Wendland kernels dw(q)
// carries a factor q, so g = dw_scale / h_bar * dw(q) / q needs no division
// by |x|; at x = 0 it is finite and multiplies a zero vector. Otherwise the
// reference's form dw_scale * dw(q) / |x| with its non-finite guard
// (kernels.cuh:51-64).
template <int KIND>
__device__ __forceinline__ float pair_g(const KernelConst& k, float l2)
{
    const float inv = rsqrtf(l2);
    if constexpr (HasDwOverQ<KIND>::value) {
        // coincident points (l2 = 0) get the finite g at q = 0
        const float len = l2 > 0.f ? l2 * inv : 0.f;
        return (k.dw_scale * k.h_inv) * Shape<KIND>::dw_over_q(len * k.h_inv);
    } else {
        const float len = l2 * inv;
        const float g = k.dw_scale * Shape<KIND>::dw(len * k.h_inv) * inv;
        return (l2 > 0.f && isfinite(g)) ? g : 0.f;
    }
}

template <int KIND>
__device__ __forceinline__ void pair_wg(
    const KernelConst& k, float l2, float& w, float& g)
{
    const float inv = rsqrtf(l2);
    const float len = l2 > 0.f ? l2 * inv : 0.f;
    const float q = len * k.h_inv;
    w = k.w_scale * Shape<KIND>::w(__saturatef(q));
    const float gg = k.dw_scale * Shape<KIND>::dw(q) * inv;
    g = (l2 > 0.f && isfinite(gg)) ? gg : 0.f;
}

// ---- uniform grid view ----------------------------------------------------
// The device POD of a built grid, UniformGrid<Resort::yes>
// (uniformgrid.cuh:84-97): lower bound (with margin), cell size, r^2, cell
// counts and the prefix over all cell keys (keys + 1 entries).
struct GridView {
    float lox, loy, loz;
    float cell;
    float inv_cell; // 1 / cell, for the strip trimming only (never for keys)
    float r2;
    int nx, ny, nz, nxny;
    int order;      // REYN_ORDER_XYZ or REYN_ORDER_ZORDER
    int tx, txy;    // Z-order: 32-cell tiles along x, per xy layer
    const uint32_t* __restrict__ prefix;
    // batched scenes: scene of each point (null for one scene) and each
    // scene's own grid geometry, whose cell keys start at its key_base
    const uint16_t* __restrict__ sid;
    const struct SceneGeom* __restrict__ scenes;
    uint32_t key_base; // of the scene this view is narrowed to
};

// one scene of a batch: its grid's lower bound (with margin), cell counts
// and the first of its cell keys
struct SceneGeom {
    float lox, loy, loz;
    int nx, ny, nz, nxny, tx, txy;
    uint32_t key_base;
};

__device__ __forceinline__ uint32_t scene_of(const GridView& g, uint32_t i)
{
    return g.sid ? uint32_t(__ldg(g.sid + i)) : 0u;
}

// the view of scene s alone: its geometry, and its prefix slice
__device__ __forceinline__ GridView at_scene(GridView g, uint32_t s)
{
    if (g.scenes) {
        const SceneGeom q = g.scenes[s];
        g.lox = q.lox;
        g.loy = q.loy;
        g.loz = q.loz;
        g.nx = q.nx;
        g.ny = q.ny;
        g.nz = q.nz;
        g.nxny = q.nxny;
        g.tx = q.tx;
        g.txy = q.txy;
        g.key_base = q.key_base;
        g.prefix += q.key_base;
    }
    g.sid = nullptr;
    g.scenes = nullptr;
    return g;
}

// Z-order cell keys: cells are grouped into bricks of 4x4x4 (x fastest
// inside a brick, so x-runs of up to 4 cells stay contiguous), bricks follow
// the Morton curve inside tiles of 8x8x8 bricks (32^3 cells), and tiles are
// in XYZ order. Consecutive particles in this order fill compact 3-D blocks.
constexpr int ZTILE = 32;

__host__ __device__ __forceinline__ uint32_t spread3(uint32_t v) // 3 bits -> bits 0, 3, 6
{
    return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4);
}

__host__ __device__ __forceinline__ uint32_t zorder_key(int tx, int txy, int cx, int cy, int cz)
{
    const uint32_t tile = uint32_t(cz >> 5) * uint32_t(txy) + uint32_t(cy >> 5) * uint32_t(tx)
        + uint32_t(cx >> 5);
    const uint32_t brick = spread3(uint32_t(cx >> 2) & 7u) | (spread3(uint32_t(cy >> 2) & 7u) << 1)
        | (spread3(uint32_t(cz >> 2) & 7u) << 2);
    const uint32_t local = uint32_t(cx & 3) | (uint32_t(cy & 3) << 2) | (uint32_t(cz & 3) << 4);
    return (((tile << 9) | brick) << 6) | local;
}

// the key of cell (cx, cy, cz) in the grid's cell order (_linearize,
// uniformgrid.cuh:33-40, for XYZ)
__device__ __forceinline__ uint32_t cell_key(const GridView& g, int cx, int cy, int cz)
{
    if (g.order == REYN_ORDER_ZORDER)
        return zorder_key(g.tx, g.txy, cx, cy, cz);
    return (uint32_t)cz * (uint32_t)g.nxny + ((uint32_t)cy * (uint32_t)g.nx + (uint32_t)cx);
}

// _index3 (uniformgrid.cuh:17-22): floor((x - min) / cell), IEEE division so
// that keys agree with the reference bit for bit
__device__ __forceinline__ int3 cell_of(const GridView& g, float x, float y, float z)
{
    return make_int3((int)floorf((x - g.lox) / g.cell),
        (int)floorf((y - g.loy) / g.cell), (int)floorf((z - g.loz) / g.cell));
}

__device__ __forceinline__ bool cell_inside(const GridView& g, int3 c, int R)
{
    return c.x >= R && c.y >= R && c.z >= R && c.x < g.nx - R && c.y < g.ny - R
        && c.z < g.nz - R;
}

__device__ __forceinline__ int3 clamp_cell(const GridView& g, int3 c, int R)
{
    return make_int3(min(max(c.x, R), g.nx - 1 - R), min(max(c.y, R), g.ny - 1 - R),
        min(max(c.z, R), g.nz - 1 - R));
}

// The rows of the fixed-radius traversal (the role of UniformGrid::ff_nbrs,
// uniformgrid.cuh:113-178): (2R+1)^2 rows of cells, each a run of x-cells,
// visited in the reference's order (z, then y). run(k0, ncell) gets the key
// of a run's first cell and its length: the run's particles are the sorted
// range prefix[k0] .. prefix[k0 + ncell]. In XYZ order every row is one run;
// in Z-order a row that crosses a brick boundary is two.
//
// Each row is trimmed to the part the search sphere can reach: rows whose
// (y, z) distance from the point exceeds r are skipped, and the x-run is cut
// to the cells overlapping the sphere's chord at that distance. The trimming
// is conservative by a margin of 1e-3 cells (far above the rounding of the
// approximate square root used for the chord), so exactly the candidates
// within r are still visited, in the same order; only provably empty cells
// are skipped.

// the point in cell units relative to its own cell's lower corner, and the
// squared search radius in cells with the trimming margin
struct RowFrame {
    float fx, fy, fz, rr;
};

__device__ __forceinline__ RowFrame row_frame(const GridView& g, int3 c, float xi, float yi,
    float zi)
{
    constexpr float EPS = 1e-3f;
    RowFrame fr;
    fr.fx = (xi - g.lox) * g.inv_cell - (float)c.x;
    fr.fy = (yi - g.loy) * g.inv_cell - (float)c.y;
    fr.fz = (zi - g.loz) * g.inv_cell - (float)c.z;
    fr.rr = g.r2 * g.inv_cell * g.inv_cell * (1.f + EPS) + EPS;
    return fr;
}

// squared distance (cells) from the point to the slab of cells at c.z + dz
__device__ __forceinline__ float slab_gap2(const RowFrame& fr, int dz)
{
    const float gz = dz > 0 ? fmaxf((float)dz - fr.fz, 0.f)
                            : (dz < 0 ? fmaxf(fr.fz - (float)(dz + 1), 0.f) : 0.f);
    return gz * gz;
}

// the x-cells [x0, x1] (relative to c.x) of row dy in a slab at squared gap
// gz2 that the sphere can reach; false when the row is skipped
template <int R>
__device__ __forceinline__ bool row_span(const RowFrame& fr, float gz2, int dy, int& x0, int& x1)
{
    constexpr float EPS = 1e-3f;
    const float gy = dy > 0 ? fmaxf((float)dy - fr.fy, 0.f)
                            : (dy < 0 ? fmaxf(fr.fy - (float)(dy + 1), 0.f) : 0.f);
    const float d2 = fmaf(gy, gy, gz2);
    if (d2 > fr.rr)
        return false;
    const float t = fr.rr - d2;
    const float w = (t > 0.f ? t * rsqrtf(t) : 0.f) + EPS; // half chord, cells
    x0 = max(-R, (int)floorf(fr.fx - w));
    x1 = min(R, (int)floorf(fr.fx + w));
    return x0 <= x1; // empty only for points clamped into the grid from outside
}

template <int R, class Run>
__device__ __forceinline__ void for_each_row(const GridView& g, int3 c, float xi, float yi,
    float zi, Run&& run)
{
    const RowFrame fr = row_frame(g, c, xi, yi, zi);
#pragma unroll 1
    for (int dz = -R; dz <= R; ++dz) {
        const float gz2 = slab_gap2(fr, dz);
        if (gz2 > fr.rr)
            continue;
        const int plane = (c.z + dz) * g.nxny;
#pragma unroll 1
        for (int dy = -R; dy <= R; ++dy) {
            int x0, x1;
            if (!row_span<R>(fr, gz2, dy, x0, x1))
                continue;
            // one run per row, two where a Z-order row crosses a brick; one
            // call site, so the caller's candidate loop is inlined once
            uint32_t k0 = uint32_t(plane + (c.y + dy) * g.nx + c.x + x0);
            int n0 = x1 - x0 + 1;
            uint32_t k1 = 0;
            int n1 = 0;
            if (g.order == REYN_ORDER_ZORDER) {
                const int xa = c.x + x0, xb = c.x + x1, y = c.y + dy, z = c.z + dz;
                k0 = zorder_key(g.tx, g.txy, xa, y, z);
                if ((xa >> 2) != (xb >> 2)) {
                    n0 = 4 - (xa & 3);
                    k1 = zorder_key(g.tx, g.txy, xb & ~3, y, z);
                    n1 = (xb & 3) + 1;
                }
            }
#pragma unroll 1
            for (int q = 0; q < 2; ++q) {
                if (q == 1) {
                    if (!n1)
                        break;
                    k0 = k1;
                    n0 = n1;
                }
                run(k0, n0);
            }
        }
    }
}

// Fixed-radius neighbour traversal: f(j, pts[j], dx, dy, dz, l2) for every
// candidate with l2 <= r^2 (self included, as the reference's accumulation
// does), in the reference's row order. `pts` are packed (x, y, z, mass) in
// grid order.
template <int R, class F>
__device__ __forceinline__ void for_each_neighbour(const GridView& g, int3 c,
    float xi, float yi, float zi, const float4* __restrict__ pts, F&& f)
{
    for_each_row<R>(g, c, xi, yi, zi, [&](uint32_t k0, int ncell) {
        const uint32_t s = __ldg(g.prefix + k0);
        const uint32_t e = __ldg(g.prefix + k0 + ncell);
        for (uint32_t j = s; j < e; ++j) {
            const float4 q = __ldg(pts + j);
            const float dx = xi - q.x, dy_ = yi - q.y, dz_ = zi - q.z;
            const float l2 = fmaf(dx, dx, fmaf(dy_, dy_, dz_ * dz_));
            if (l2 <= g.r2)
                f(j, q, dx, dy_, dz_, l2);
        }
    });
}

// ---- counter-based random numbers ------------------------------------------
// Value k of stream t under seed s is SplitMix64 (Steele, Lea, Flood 2014) of
// s + 0x9E3779B97F4A7C15 (t 2^40 + k + 1): a pure function of (s, t, k), so
// results never depend on the launch and the host reproduces them exactly.

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t stream_bits(uint64_t seed, uint64_t t, uint64_t k)
{
    return splitmix64(seed + 0x9E3779B97F4A7C15ull * ((t << 40) + k + 1));
}

// uniform in [0, 1) from the top 24 bits (an exact float)
__device__ __forceinline__ float uniform01(uint64_t seed, uint64_t t, uint64_t k)
{
    return float(uint32_t(stream_bits(seed, t, k) >> 40)) * (1.f / 16777216.f);
}

// uniform in (0, 1] from the top 53 bits (an exact double)
__device__ __forceinline__ double uniform_open0(uint64_t seed, uint64_t t, uint64_t k)
{
    return double((stream_bits(seed, t, k) >> 11) + 1) * (1.0 / 9007199254740992.0);
}

// uniform in [-a, a]: (2u - 1) a, explicitly rounded
__device__ __forceinline__ float symmetric(float u, float a)
{
    return __fmul_rn(__fsub_rn(__fmul_rn(2.f, u), 1.f), a);
}

// ---- reductions -------------------------------------------------------------

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ unsigned warp_sum(unsigned v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
        v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// atomic max on non-negative floats through their ordered bit patterns
__device__ __forceinline__ void atomic_max_nonneg(float* addr, float v)
{
    if (v > 0.f)
        atomicMax(reinterpret_cast<unsigned*>(addr), __float_as_uint(v));
}

} // namespace reyn
