// The neighbour passes of the SESPH / PCISPH / IISPH steps and the step
// driver, templated on the largest block size the passes are compiled for
// (solver.cu instantiates 128 threads, solver_wide.cu 512). Each including
// file gets its own copies of the kernels (anonymous namespace).
// SESPH / PCISPH / IISPH steps on the B200. Each pass is one fixed-radius
// neighbour kernel over the packed (x, y, z, m) copy in grid order; work the
// reference spreads over separate kernels is fused where no neighbour reads
// the value being written:
//   * density also caches, per particle, the boundary sums rho_b = sum m_b W
//     and g_b = sum m_b grad W (positions are fixed within a step, so every
//     later boundary term of the step is a multiply by g_b);
//   * the non-pressure pass writes v* = v + dt a into a second velocity
//     buffer (integrate_a_v_only fused);
//   * PCISPH's pressure pass applies v += dt a in place (it reads no
//     neighbour velocity), so the next prediction and the final integrate
//     see the same velocities as the reference's separate kernels;
//   * IISPH's diagonal pass also applies the warm start; the final pressure
//     pass integrates (v, x) and writes the SoA state.
// Reference: solver.cuh:18-105, solver.cu, SESPH.cu:6-95, PCISPH.cuh:49-77,
// PCISPH.cu:15-111, IISPH.cu:11-262.
#pragma once
#include "engine.cuh"

#include <cuda_fp16.h>

#include <cmath>
#include <type_traits>
#include <vector>

namespace reyn {

namespace {

// Per-step neighbour list: the fluid neighbours (self excluded) of every
// particle, in traversal order, written by the density pass and read by every
// later pass of the step (positions are fixed until the final integration).
// Slot k of particle i lives at list_slot(i, k): blocks of 128 particles
// store their slot rows contiguously, so that a warp reads one 128-byte row
// per slot. A particle with more than KMAX neighbours keeps its count
// (> KMAX) and is served by the cell traversal instead. Each block of 128
// particles owns LROWS = KMAX + 4 rows, so that a loop may load the indices
// of the next four slots past a particle's last one without a bound check
// (the values are not used).
constexpr int KMAX = 64;
constexpr int LROWS = KMAX + 4;
// (the layout is independent of the block size of the passes)

__host__ __device__ __forceinline__ size_t list_slot(uint32_t i, uint32_t k)
{
    return size_t(i >> 7) * (LROWS * 128) + size_t(k) * 128 + (i & 127u);
}

inline size_t list_capacity(uint32_t n) { return size_t((n + 127) / 128) * LROWS * 128; }

struct Fluid {
    GridView g;
    KernelConst kc;
    const float4* __restrict__ pm; // (x, y, z, m), grid order
    uint32_t* status;
    uint32_t* __restrict__ nbr;    // neighbour list (list_slot layout)
    uint32_t* __restrict__ ncount; // neighbours per particle
    // MIXED: per particle its pressure acceleration as FP16 (scaled by
    // ACC_SCALE) for the Jacobi sweeps, and the FP32 accelerations for
    // particles off the list
    const uint2* __restrict__ acch;
    const float4* __restrict__ acc32;
    // batched scenes: per-scene flag, 0 once the scene's iteration has
    // converged (its particles then sit out the remaining sweeps)
    const uint8_t* __restrict__ active;
};

// ---- mixed precision ----------------------------------------------------------
// MIXED_POS16 records are 16 bytes: each position coordinate as a 16-bit
// wrapped fixed-point number, the position in cells modulo 4 at a resolution
// of 1/16384 cell, and 10 bytes of the quantity the reading pass needs.
// Neighbours lie within 2 cells (r), so the 16-bit difference u_i - u_j, read
// as a signed number, is the pair vector x_ij in units of 1/16384 cell
// exactly, with no cell index stored. (A coordinate difference of exactly 2
// cells reads as -2; such a pair lies on the support's edge, where the kernel
// and its gradient vanish.) Both ends use their quantised records, so
// x_ji = -x_ij holds exactly and pair forces stay antisymmetric. The
// quantisation error is at most 1/32768 cell per coordinate (FP16 offsets
// within a cell would round to 1/4096).
constexpr float FIXQ = 16384.f;

// storage modes of the neighbour loops (the template argument MIX):
// 0 FP32; MIX_F16 FP16 velocities, densities and pressure accelerations of
// neighbours; MIX_POS16 the 16-byte records (16-bit positions, FP16
// velocities and accelerations, FP32 pressures)
constexpr int MIX_F16 = 1;
constexpr int MIX_POS16 = 2;

__device__ __forceinline__ float4 half4_to_float4(uint2 u)
{
    __half2 a, b;
    memcpy(&a, &u.x, 4);
    memcpy(&b, &u.y, 4);
    const float2 fa = __half22float2(a), fb = __half22float2(b);
    return make_float4(fa.x, fa.y, fb.x, fb.y);
}

__device__ __forceinline__ uint2 float4_to_half4(float4 v)
{
    const __half2 a = __floats2half2_rn(v.x, v.y), b = __floats2half2_rn(v.z, v.w);
    uint2 u;
    memcpy(&u.x, &a, 4);
    memcpy(&u.y, &b, 4);
    return u;
}

__device__ __forceinline__ uint32_t half2_bits(float a, float b)
{
    const __half2 h = __floats2half2_rn(a, b);
    uint32_t u;
    memcpy(&u, &h, 4);
    return u;
}

__device__ __forceinline__ float2 bits_half2(uint32_t u)
{
    __half2 h;
    memcpy(&h, &u, 4);
    return __half22float2(h);
}

// the FP16 number in the upper half of u
__device__ __forceinline__ float upper_half(uint32_t u)
{
    return __half2float(__ushort_as_half((unsigned short)(u >> 16)));
}

// one coordinate: (cell index mod 4) * 16384 + the offset in the cell in
// units of 1/16384, modulo 2^16 (an offset that rounds up to 16384 carries
// into the cell index)
__device__ __forceinline__ uint32_t fix_coord(float p, float lo, float inv_cell, int c)
{
    const float o = __saturatef(__fsub_rn(__fmul_rn(__fsub_rn(p, lo), inv_cell), (float)c));
    return ((uint32_t(c) << 14) + __float2uint_rn(o * FIXQ)) & 0xffffu;
}

// words 0 and 1 of a record: x | y << 16 and z | a << 16 (a: 16 payload bits)
__device__ __forceinline__ uint2 record_position(const GridView& g, int3 c, float x, float y,
    float z, uint32_t a)
{
    const uint32_t ux = fix_coord(x, g.lox, g.inv_cell, c.x);
    const uint32_t uy = fix_coord(y, g.loy, g.inv_cell, c.y);
    const uint32_t uz = fix_coord(z, g.loz, g.inv_cell, c.z);
    return make_uint2(ux | (uy << 16), uz | (a << 16));
}

// Record layouts (word 0 = x | y << 16 and the low half of word 1 = z are the
// position in every layout):
//   NP (density -> non-pressure): w1 hi m/m_0 (FP16), w2 (vx, vy), w3 (vz, rho)
//   DG (non-pressure -> diagonal): w1 hi, w2 = m v* / m_0 (3 x FP16),
//      w3 = m p_old (FP32)
//   Y (pressure accelerations -> Jacobi): w1 hi m/m_0, w2, w3 lo =
//      m a ACC_SCALE / m_0 (3 x FP16)
//   X (Jacobi -> pressure accelerations): w1 hi m/m_0, w2 = p (FP32),
//      w3 = (m/m_0) p (FP32)
__device__ __forceinline__ uint32_t half_bits(float a)
{
    return __half_as_ushort(__float2half_rn(a));
}

// the FP16 number in the lower half of u
__device__ __forceinline__ float lower_half(uint32_t u)
{
    return __half2float(__ushort_as_half((unsigned short)(u & 0xffffu)));
}

__device__ __forceinline__ uint4 rec_np(const GridView& g, int3 c, const float4& me,
    uint32_t m16, float vx, float vy, float vz, float rho)
{
    const uint2 p = record_position(g, c, me.x, me.y, me.z, m16);
    return make_uint4(p.x, p.y, half2_bits(vx, vy), half2_bits(vz, rho));
}

// word 1 of a record with the mass ratio m16 in its upper half
__device__ __forceinline__ uint32_t rec_w1(const uint4& r, uint32_t m16)
{
    return (r.y & 0xffffu) | (m16 << 16);
}

__device__ __forceinline__ uint4 rec_dg(const uint4& prev, float vx, float vy, float vz, float mp)
{
    return make_uint4(prev.x, (prev.y & 0xffffu) | (half_bits(vx) << 16), half2_bits(vy, vz),
        __float_as_uint(mp));
}

__device__ __forceinline__ float3 rec_dg_vec(const uint4& r)
{
    const float2 yz = bits_half2(r.z);
    return make_float3(upper_half(r.y), yz.x, yz.y);
}

__device__ __forceinline__ float rec_dg_mp(const uint4& r) { return __uint_as_float(r.w); }

__device__ __forceinline__ uint4 rec_y(uint32_t w0, uint32_t w1, float ax, float ay, float az)
{
    return make_uint4(w0, w1, half2_bits(ax, ay), half_bits(az));
}

__device__ __forceinline__ float3 rec_y_vec(const uint4& r)
{
    const float2 xy = bits_half2(r.z);
    return make_float3(xy.x, xy.y, lower_half(r.w));
}

__device__ __forceinline__ uint4 rec_x(uint32_t w0, uint32_t w1, float p)
{
    return make_uint4(w0, w1, __float_as_uint(p), __float_as_uint(upper_half(w1) * p));
}

__device__ __forceinline__ float rec_x_p(const uint4& r) { return __uint_as_float(r.z); }

// (m/m_0) p of an X record: the product a neighbour's pressure enters the
// pressure accelerations with, rounded as the reader would round it
__device__ __forceinline__ float rec_x_mp(const uint4& r) { return __uint_as_float(r.w); }

// the mass ratio m/m_0 of a NP, Y or X record
__device__ __forceinline__ float rec_m16(const uint4& r) { return upper_half(r.y); }

// A particle's own coordinates, offset by half the 16-bit range, laid out so
// that one 32-bit subtraction per coordinate leaves (u_i - u_j + 2^15) mod
// 2^16 in one half of the result: x and z in the low half, y in the high half
// (its low half 0xffff, so that no borrow crosses into it).
struct Own16 {
    uint32_t bx, by, bz;
};

__device__ __forceinline__ Own16 own16(const uint4& r)
{
    return Own16 { (r.x + 0x8000u) & 0xffffu, ((r.x + 0x80000000u) & 0xffff0000u) | 0xffffu,
        (r.y + 0x8000u) & 0xffffu };
}

// x_i - x_j in units of 1/FIXQ cell, exactly: the 16-bit half t of each
// difference is placed under the exponent of 2^23 (a float 2^23 + t, built by
// one byte permutation), and 2^23 + 2^15 is subtracted. No integer-to-float
// conversion instruction is needed.
__device__ __forceinline__ float3 delta16(const Own16& o, const uint4& rj)
{
    constexpr float BIAS = 8421376.f; // 2^23 + 2^15
    const uint32_t tx = o.bx - rj.x, ty = o.by - rj.x, tz = o.bz - rj.y;
    return make_float3(__uint_as_float(__byte_perm(tx, 0x4B000000u, 0x7610)) - BIAS,
        __uint_as_float(__byte_perm(ty, 0x4B000000u, 0x7632)) - BIAS,
        __uint_as_float(__byte_perm(tz, 0x4B000000u, 0x7610)) - BIAS);
}

// the kernel constants for pair vectors in units of 1/FIXQ cell: with
// h_inv scaled by the unit, pair_w gives W and pair_g gives g' = g * unit,
// so that grad W = g' d for the pair vector d in those units
__host__ __device__ __forceinline__ KernelConst kernel_in_units(KernelConst k, float unit)
{
    k.h_inv *= unit;
    return k;
}

// accelerations are stored as FP16 of a * 2^-6: up to 4e6 m/s^2 before
// overflow, 11 significant bits
constexpr float ACC_SCALE = 0.015625f;

__device__ __forceinline__ uint2 pack_acc(float ax, float ay, float az)
{
    return float4_to_half4(make_float4(ax * ACC_SCALE, ay * ACC_SCALE, az * ACC_SCALE, 0.f));
}

// the stored (scaled) acceleration: a * ACC_SCALE
__device__ __forceinline__ float3 unpack_acc_scaled(uint2 u)
{
    const float4 a = half4_to_float4(u);
    return make_float3(a.x, a.y, a.z);
}

// compensated (Kahan) summation for the mixed modes' density and divergence
// sums: sum + comp carries the rounding the plain sum would drop
struct Kahan {
    float sum = 0.f, comp = 0.f;
    __device__ __forceinline__ void add(float v)
    {
        const float y = __fsub_rn(v, comp);
        const float t = __fadd_rn(sum, y);
        comp = __fsub_rn(__fsub_rn(t, sum), y);
        sum = t;
    }
};

// a neighbour's velocity/density record: FP32 or FP16 storage
template <int MIX>
__device__ __forceinline__ float4 nbr_vel(const float4* __restrict__ v32,
    const uint2* __restrict__ v16, uint32_t j)
{
    if constexpr (MIX)
        return half4_to_float4(__ldg(v16 + j));
    else
        return __ldg(v32 + j);
}

struct Bdy {
    GridView g;
    const float4* __restrict__ pm;
    const uint8_t* __restrict__ near; // cells with samples within reach
    uint32_t n;
};

// the cell of particle i in the fluid grid; positions outside it are
// clamped (results are then meaningless) and reported through `status`
template <int R>
__device__ __forceinline__ int3 fluid_cell(const Fluid& f, const float4& me)
{
    int3 c = cell_of(f.g, me.x, me.y, me.z);
    if (!cell_inside(f.g, c, R) || !(isfinite(me.x) && isfinite(me.y) && isfinite(me.z))) {
        atomicOr(f.status, STATUS_OUT_OF_GRID);
        c = clamp_cell(f.g, c, R);
    }
    return c;
}

// batched scenes: narrows the views to particle i's scene (its grid keys,
// its boundary grid and near-flags) and returns the scene; 0 for one scene
__device__ __forceinline__ uint32_t enter_scene(Fluid& f, uint32_t i)
{
    if (!f.g.sid)
        return 0;
    const uint32_t s = __ldg(f.g.sid + i);
    f.g = at_scene(f.g, s);
    return s;
}

__device__ __forceinline__ uint32_t enter_scene(Fluid& f, Bdy& b, uint32_t i)
{
    const uint32_t s = enter_scene(f, i);
    if (b.n && b.g.sid) {
        b.g = at_scene(b.g, s);
        b.near += b.g.key_base;
    }
    return s;
}

__device__ __forceinline__ bool scene_live(const Fluid& f, uint32_t s)
{
    return !f.active || __ldg(f.active + s);
}

// the fluid neighbours j != i of particle i from the step's list (or, for a
// particle whose list overflowed, from the cell traversal); fn(j, q, dx, dy,
// dz, l2) in the traversal order of the cells, q.w the neighbour's mass. q.xyz
// is the neighbour's position on the FP32 path; on the mixed path with ACC it
// is the neighbour's pressure acceleration times ACC_SCALE (from the FP16
// record, or FP32 for a particle off the list).
template <int R, int MIX = 0, bool ACC = false, bool BATCH = false, class F>
__device__ __forceinline__ void for_each_listed(const Fluid& f, uint32_t i, const float4& me,
    F&& fn)
{
    static_assert(MIX || !ACC, "accelerations travel with the mixed records only");
    static_assert(MIX != MIX_POS16, "the 16-byte records have their own loop (for_each_rec)");
    const uint32_t cnt = __ldg(f.ncount + i);
    if (cnt <= KMAX) {
        const uint32_t* __restrict__ row = f.nbr + list_slot(i, 0);
        // one neighbour: index, position data, the pair
        auto pair = [&](uint32_t j, float4& q, float& dx, float& dy, float& dz) {
            q = __ldg(f.pm + j);
            dx = me.x - q.x;
            dy = me.y - q.y;
            dz = me.z - q.z;
            if constexpr (ACC) {
                const float3 a = unpack_acc_scaled(__ldg(f.acch + j));
                q.x = a.x;
                q.y = a.y;
                q.z = a.z;
            }
        };
        uint32_t k = 0;
        // four neighbours per round: their index and position loads are
        // independent, which keeps more of the latency-bound loads in flight
        for (; k + 4 <= cnt; k += 4) {
            uint32_t j[4];
            float4 q[4];
            float dx[4], dy[4], dz[4];
#pragma unroll
            for (int u = 0; u < 4; ++u)
                j[u] = __ldg(row + size_t(k + u) * 128);
#pragma unroll
            for (int u = 0; u < 4; ++u)
                pair(j[u], q[u], dx[u], dy[u], dz[u]);
#pragma unroll
            for (int u = 0; u < 4; ++u)
                fn(j[u], q[u], dx[u], dy[u], dz[u],
                    fmaf(dx[u], dx[u], fmaf(dy[u], dy[u], dz[u] * dz[u])));
        }
        for (; k < cnt; ++k) {
            const uint32_t j = __ldg(row + size_t(k) * 128);
            float4 q;
            float dx, dy, dz;
            pair(j, q, dx, dy, dz);
            fn(j, q, dx, dy, dz, fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
        }
    } else {
        // the cell traversal: the particle's (scene's) grid and cell, found
        // only here, as the density pass already checked the positions
        GridView g = f.g;
        if constexpr (BATCH)
            g = at_scene(g, scene_of(g, i));
        int3 c = cell_of(g, me.x, me.y, me.z);
        if (!cell_inside(g, c, R)) // flagged by the density pass already
            c = clamp_cell(g, c, R);
        for_each_neighbour<R>(g, c, me.x, me.y, me.z, f.pm,
            [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
                if (j == i)
                    return;
                if constexpr (ACC) {
                    const float4 a = __ldg(f.acc32 + j);
                    fn(j, make_float4(a.x * ACC_SCALE, a.y * ACC_SCALE, a.z * ACC_SCALE, q.w),
                        dx, dy, dz, l2);
                } else {
                    fn(j, q, dx, dy, dz, l2);
                }
            });
    }
}

// The kernel-gradient factor of a record pair up to a factor that is the
// same for every pair of a pass: for Wendland C2 the cube of (1 - q), the
// constant dw(q)/q / (1 - q)^3 = -20 times dw_scale h_inv being applied once
// to each particle's sums (rec_gscale); for the other kernels pair_g itself.
// At l2 = 0 (a coincident pair, whose d is 0) the C2 factor is 0.
template <int KIND>
__device__ __forceinline__ float rec_g(const KernelConst& k, float l2)
{
    if constexpr (KIND == K_C2) {
        const float t = fmaxf(0.f, fmaf(-k.h_inv, l2 * rsqrtf(l2), 1.f));
        return t * t * t;
    } else {
        return pair_g<KIND>(k, l2);
    }
}

template <int KIND>
__device__ __forceinline__ float rec_gscale(const KernelConst& k)
{
    if constexpr (KIND == K_C2)
        return (k.dw_scale * k.h_inv) * Shape<KIND>::dw_over_q(0.f);
    else
        return 1.f;
}

// MIXED_POS16: the fluid neighbours j != i of particle i with their 16-byte
// records: fn(j, rec_j, d, g) with d = x_i - x_j in units of 1/FIXQ cell and
// g = rec_g, the kernel-gradient factor of the pair in those units up to the
// pass-wide rec_gscale (grad W_ij = rec_gscale g d; kc holds the kernel
// constants in record units), in the traversal order of
// the cells. ri is the particle's own record in `rec`. A particle whose list
// overflowed walks the cell traversal over the FP32 positions, its pair
// vectors converted to the record units.
template <int KIND, int R, bool BATCH = false, class F>
__device__ __forceinline__ void for_each_rec(const Fluid& f, const KernelConst& kc,
    const uint4* __restrict__ rec, uint32_t i, const uint4& ri, F&& fn)
{
    const uint32_t cnt = __ldg(f.ncount + i);
    {
        // ask the L2 for the warp's list rows up front (one 128-byte segment
        // per row and lane), so that the loop's index loads do not each wait
        // for DRAM
        const unsigned m = __activemask();
        const uint32_t mc = __reduce_max_sync(m, min(cnt, uint32_t(KMAX)));
        const uint32_t lane = threadIdx.x & 31u;
        const uint32_t* seg = f.nbr + list_slot(i & ~31u, 0);
        if (lane < mc)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(seg + size_t(lane) * 128));
        if (lane + 32u < mc)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(seg + size_t(lane + 32u) * 128));
    }
    if (cnt <= KMAX) {
        const Own16 o = own16(ri);
        const uint32_t* __restrict__ row = f.nbr + list_slot(i, 0);
        uint32_t k = 0;
        // four neighbours per round, the next round's indices loaded before
        // this round's records are used (the list streams from DRAM and each
        // record load depends on its index); the rows past a particle's last
        // slot are padding, read but not used
        uint32_t jn[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
            jn[u] = __ldg(row + size_t(u) * 128);
        for (; k + 4 <= cnt; k += 4) {
            uint32_t j[4];
            uint4 r[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                j[u] = jn[u];
                r[u] = __ldg(rec + j[u]);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
                jn[u] = __ldg(row + size_t(k + 4 + u) * 128);
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const float3 d = delta16(o, r[u]);
                fn(j[u], r[u], d, rec_g<KIND>(kc, fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z))));
            }
        }
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            if (k + u < cnt) {
                const uint4 r = __ldg(rec + jn[u]);
                const float3 d = delta16(o, r);
                fn(jn[u], r, d, rec_g<KIND>(kc, fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z))));
            }
        }
    } else {
        const float4 me = f.pm[i];
        GridView gv = f.g;
        if constexpr (BATCH)
            gv = at_scene(gv, scene_of(gv, i));
        int3 c = cell_of(gv, me.x, me.y, me.z);
        if (!cell_inside(gv, c, R)) // flagged by the density pass already
            c = clamp_cell(gv, c, R);
        const float to_units = FIXQ / gv.cell;
        for_each_neighbour<R>(gv, c, me.x, me.y, me.z, f.pm,
            [&](uint32_t j, const float4&, float dx, float dy, float dz, float) {
                if (j == i)
                    return;
                const float3 d = make_float3(dx * to_units, dy * to_units, dz * to_units);
                fn(j, __ldg(rec + j), d,
                    rec_g<KIND>(kc, fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z))));
            });
    }
}

// boundary neighbours of a point; a point whose cell is outside the
// boundary grid's searchable range is farther than r from every sample
template <class F>
__device__ __forceinline__ void for_each_boundary(const Bdy& b, float x, float y, float z, F&& f)
{
    if (b.n == 0)
        return;
    const int3 c = cell_of(b.g, x, y, z);
    if (!cell_inside(b.g, c, 2))
        return;
    if (!__ldg(b.near + (c.z * b.g.nxny + c.y * b.g.nx + c.x)))
        return;
    for_each_neighbour<2>(b.g, c, x, y, z, b.pm, f);
}

// The density pass's boundary sums (rb = sum_b m_b W_ib and
// g = sum_b m_b grad W_ib) for every lane of the warp whose cell has samples
// within reach, computed by the whole warp: for each such lane in turn, lanes
// 0-24 take one row each of that point's 5x5 rows of boundary cells (the
// rows and trim of for_each_boundary) and the warp adds the rows up. A lane
// walking its 25 rows alone holds its warp for all of them; in the batched
// workloads three warps in four hold a lane near a wall (scene boxes are a
// few dozen particles wide), so the batched density pass uses this; in one
// large scene few warps do, and the lanes walk alone there. Every lane of the
// warp must call this (no lane may have returned); `need_point` says whether
// the lane's own point is a fluid particle. The sums run over the samples
// for_each_boundary visits, added in another order. Batched scenes: each
// point uses its own scene's boundary grid.
template <int KIND, bool BATCH>
__device__ __forceinline__ float4 boundary_sums_warp(const Bdy& b0, const KernelConst& kc,
    bool need_point, uint32_t scene, float x, float y, float z)
{
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    bool need = false;
    if (need_point && b0.n) {
        Bdy b = b0;
        if constexpr (BATCH) {
            if (b.g.sid) {
                b.g = at_scene(b.g, scene);
                b.near += b.g.key_base;
            }
        }
        const int3 c = cell_of(b.g, x, y, z);
        need = cell_inside(b.g, c, 2)
            && __ldg(b.near + (c.z * b.g.nxny + c.y * b.g.nx + c.x)) != 0;
    }
    unsigned m = __ballot_sync(FULL, need);
    float4 mine = make_float4(0.f, 0.f, 0.f, 0.f);
    while (m) {
        const int src = __ffs(m) - 1;
        m &= m - 1;
        const float px = __shfl_sync(FULL, x, src), py = __shfl_sync(FULL, y, src),
                    pz = __shfl_sync(FULL, z, src);
        Bdy b = b0;
        if constexpr (BATCH) {
            const uint32_t s = __shfl_sync(FULL, scene, src);
            if (b.g.sid) {
                b.g = at_scene(b.g, s);
                b.near += b.g.key_base;
            }
        }
        float rb = 0.f, gx = 0.f, gy = 0.f, gz = 0.f;
        if (lane < 25) {
            const int3 c = cell_of(b.g, px, py, pz);
            const RowFrame fr = row_frame(b.g, c, px, py, pz);
            const int dz = lane / 5 - 2, dy = lane % 5 - 2;
            const float gz2 = slab_gap2(fr, dz);
            int x0, x1;
            if (gz2 <= fr.rr && row_span<2>(fr, gz2, dy, x0, x1)) {
                const uint32_t k0 =
                    uint32_t((c.z + dz) * b.g.nxny + (c.y + dy) * b.g.nx + c.x + x0);
                const uint32_t e = __ldg(b.g.prefix + k0 + uint32_t(x1 - x0 + 1));
                for (uint32_t j = __ldg(b.g.prefix + k0); j < e; ++j) {
                    const float4 q = __ldg(b.pm + j);
                    const float dx = px - q.x, dyy = py - q.y, dzz = pz - q.z;
                    const float l2 = fmaf(dx, dx, fmaf(dyy, dyy, dzz * dzz));
                    if (l2 <= b.g.r2) {
                        float w, g;
                        pair_wg<KIND>(kc, l2, w, g);
                        rb += q.w * w;
                        const float mg = q.w * g;
                        gx += mg * dx;
                        gy += mg * dyy;
                        gz += mg * dzz;
                    }
                }
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            rb += __shfl_xor_sync(FULL, rb, o);
            gx += __shfl_xor_sync(FULL, gx, o);
            gy += __shfl_xor_sync(FULL, gy, o);
            gz += __shfl_xor_sync(FULL, gz, o);
        }
        if (lane == src)
            mine = make_float4(gx, gy, gz, rb);
    }
    return mine;
}

// jacobi_update (IISPH.cu:108-117). The reference compares the float a_ii
// with the double 1e-6; `tiny` is the smallest float above 1e-6, for which
// a < tiny holds exactly when (double)a < 1e-6 does (tiny_threshold()).
__device__ __forceinline__ float jacobi_update(float omega, float a_ii, float Ap, float s,
    float tiny)
{
    return (a_ii < tiny && a_ii > -tiny) ? 0.f : fmaxf(0.f, omega * (s - Ap) / a_ii);
}

float tiny_threshold()
{
    float t = (float)1e-6;
    while ((double)t < 1e-6)
        t = std::nextafterf(t, INFINITY);
    return t;
}

// per-sweep reductions (one slot per sweep, zeroed before use)
struct SweepStats {
    unsigned long long over; // particles with predicted error above eta rho0
    double err_sum;          // sum of max(0, predicted error)
    double rho_sum;          // PCISPH: sum of predicted densities
    float err_max;
    float pad;
};

__device__ __forceinline__ void block_accumulate(SweepStats* st, unsigned over, double err,
    double rho, float emax)
{
    __shared__ unsigned s_over[NBR_MAX_THREADS / 32];
    __shared__ double s_err[NBR_MAX_THREADS / 32], s_rho[NBR_MAX_THREADS / 32];
    __shared__ float s_max[NBR_MAX_THREADS / 32];
    over = warp_sum(over);
    err = warp_sum(err);
    rho = warp_sum(rho);
    emax = warp_max(emax);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) {
        s_over[w] = over;
        s_err[w] = err;
        s_rho[w] = rho;
        s_max[w] = emax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (unsigned k = 1; k < blockDim.x / 32; ++k) {
            over += s_over[k];
            err += s_err[k];
            rho += s_rho[k];
            emax = fmaxf(emax, s_max[k]);
        }
        if (over)
            atomicAdd(&st->over, (unsigned long long)over);
        if (err != 0.0)
            atomicAdd(&st->err_sum, err);
        if (rho != 0.0)
            atomicAdd(&st->rho_sum, rho);
        atomic_max_nonneg(&st->err_max, emax);
    }
}

// the same sums per scene (batched scenes, one slot per scene): a warp
// inside one scene reduces first, a warp across a scene boundary adds per lane
__device__ __forceinline__ void scene_accumulate(SweepStats* st, uint32_t s, bool valid,
    unsigned over, double err, double rho, float emax)
{
    const uint32_t s0 = __shfl_sync(0xffffffffu, s, 0);
    if (__all_sync(0xffffffffu, valid && s == s0)) {
        over = warp_sum(over);
        err = warp_sum(err);
        rho = warp_sum(rho);
        emax = warp_max(emax);
        if ((threadIdx.x & 31) != 0)
            return;
    } else if (!valid) {
        return;
    }
    SweepStats* t = st + s;
    if (over)
        atomicAdd(&t->over, (unsigned long long)over);
    if (err != 0.0)
        atomicAdd(&t->err_sum, err);
    if (rho != 0.0)
        atomicAdd(&t->rho_sum, rho);
    atomic_max_nonneg(&t->err_max, emax);
}

// per-scene convergence after a sweep (batched scenes): a scene that meets
// its criterion stops iterating; n_active counts the scenes that go on.
// mode 0: PCISPH average density (PCISPH.cu:101); 1: IISPH average error;
// 2: IISPH any particle above eta rho0 (IISPH.cu:246)
// In a captured step the sweep count lives on the device (iter_dev: sweeps
// finished before this one) and the kernel does nothing before min_iter, as
// the host loop does not call it then.
__global__ void k_scene_converge(uint32_t ns, const SweepStats* __restrict__ st,
    const uint32_t* __restrict__ first, int mode, float eta, float rho0, uint32_t iter,
    uint8_t* __restrict__ active, uint32_t* __restrict__ iters_out,
    float* __restrict__ avg_err, float* __restrict__ max_err, uint32_t* __restrict__ n_active,
    const uint32_t* __restrict__ iter_dev, uint32_t min_iter, uint32_t max_iter)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (iter_dev) {
        iter = *iter_dev + 1;
        if (iter < min_iter && !(max_iter && iter >= max_iter))
            return;
    }
    if (s >= ns || !active[s])
        return;
    const uint32_t cnt = first[s + 1] - first[s];
    bool conv = true;
    if (cnt) {
        const SweepStats t = st[s];
        if (mode == 0) {
            const double a = t.rho_sum / cnt;
            conv = !((float)a > (eta + 1.f) * rho0);
            avg_err[s] = (float)fmax(0.0, a / rho0 - 1.0);
        } else {
            conv = mode == 1 ? !(t.err_sum / cnt > (double)eta * rho0) : t.over == 0;
            avg_err[s] = (float)(t.err_sum / cnt / rho0);
            max_err[s] = t.err_max / rho0;
        }
    }
    iters_out[s] = iter;
    if (conv)
        active[s] = 0;
    else
        atomicAdd(n_active, 1u);
}

// ---- captured steps: the iteration decision on the device ------------------
// After each sweep of a captured step: counts the sweep, applies the host
// loop's stopping rule (min_iter, max_iter, the scheme's criterion on this
// sweep's sums, or for a batch whether any scene goes on), records the step
// statistics and sets the while node's condition and the pressure-pass gate.
// scheme: REYN_PCISPH or REYN_IISPH; conv_any: IISPH's any-particle rule.
__global__ void k_graph_decide(int scheme, int conv_any, const SweepStats* __restrict__ slot,
    uint32_t n, float eta, float rho0, uint32_t min_iter, uint32_t max_iter,
    const uint32_t* __restrict__ n_active, GraphStats* gs, uint32_t* gate,
    cudaGraphConditionalHandle h)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
        return;
    const uint32_t it = gs->iters + 1;
    gs->iters = it;
    const bool last = max_iter && it >= max_iter;
    bool go;
    if (it < min_iter && !last) {
        go = true;
    } else if (n_active) { // a batch (IISPH.cu / PCISPH.cu loops per scene)
        const bool any = *n_active > 0;
        go = any && !last;
        if (any && last)
            gs->unconverged = 1;
    } else if (scheme == REYN_IISPH) {
        const SweepStats t = *slot;
        gs->avg_err = t.err_sum / n / rho0;
        gs->max_err = t.err_max / rho0;
        const bool more = conv_any ? t.over > 0 : t.err_sum / n > (double)eta * rho0;
        go = more && !last;
        if (more && last)
            gs->unconverged = 1;
    } else { // PCISPH (PCISPH.cu:95-102)
        const SweepStats t = *slot;
        const float avg = (float)(t.rho_sum / n);
        if (last) {
            if (it >= min_iter && !(avg <= (eta + 1.f) * rho0))
                gs->unconverged = 1;
            go = false;
        } else {
            gs->avg_err = fmax(0.0, t.rho_sum / n / rho0 - 1.0);
            go = avg > (eta + 1.f) * rho0;
        }
    }
    if (gate)
        *gate = go ? 1u : 0u;
    cudaGraphSetConditional(h, go ? 1u : 0u);
}

// a captured SESPH step: one pass, for the statistics and every scene
__global__ void k_graph_single_pass(GraphStats* gs, uint32_t* __restrict__ scene_iters,
    uint32_t ns)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s == 0)
        gs->iters = 1;
    if (s < ns)
        scene_iters[s] = 1;
}

// three SoA float arrays (an acceleration's components)
struct Soa3 {
    float* __restrict__ x;
    float* __restrict__ y;
    float* __restrict__ z;
};

// ---- step tail ---------------------------------------------------------------
// The reference's main loop follows every step with hard_enforce_bounds
// (scene.cu:466-483) and starts the next with simple_dt_controller, whose CFL
// part reduces max |v| over the state (cfl.cu:5-37). A bounded step does both
// in the kernel that writes the new state: the bounds are applied to each
// particle's new position and velocity before they are stored, and the
// norm of the stored velocity is max-reduced into `vmax`.
struct Tail {
    float3 lo, hi;
    float* vmax; // nullptr: no bounds, no reduction (the plain step)
    // batched scenes: each particle's scene and the scenes' boxes (3 floats
    // each), used instead of lo/hi
    const uint16_t* sid;
    const float* lo_s;
    const float* hi_s;
    // the next build of the step's grid, pre-keyed (keys != nullptr): each
    // stored position's cell key and the per-cell histogram, as that build's
    // k_keys_count would compute them (uniformgrid.cu:20-34), status bits to
    // kstatus
    GridView kg;
    uint32_t* keys;
    uint32_t* counts;
    uint32_t* kstatus;
};

// the cell key of a stored position and its histogram count (k_keys_count's
// arithmetic: IEEE division, clamping and status of points outside the grid)
__device__ __forceinline__ void prekey(const Tail& t, uint32_t i, float px, float py, float pz)
{
    int3 c = cell_of(t.kg, px, py, pz);
    const bool finite = isfinite(px) && isfinite(py) && isfinite(pz);
    const bool inside = finite && c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < t.kg.nx
        && c.y < t.kg.ny && c.z < t.kg.nz;
    if (!inside) {
        atomicOr(t.kstatus, finite ? STATUS_OUT_OF_GRID : STATUS_NONFINITE);
        c = finite ? make_int3(min(max(c.x, 0), t.kg.nx - 1), min(max(c.y, 0), t.kg.ny - 1),
                         min(max(c.z, 0), t.kg.nz - 1))
                   : make_int3(0, 0, 0);
    }
    const uint32_t key = cell_key(t.kg, c.x, c.y, c.z);
    t.keys[i] = key;
    atomicAdd(t.counts + key, 1u);
}

// stores the new state of particle i (bounds applied when tail.vmax is set)
// and returns |v| of what was stored
template <bool BATCH = false>
__device__ __forceinline__ float store_state(const Tail& t, uint32_t i, float px, float py,
    float pz, float nvx, float nvy, float nvz, float* __restrict__ x, float* __restrict__ y,
    float* __restrict__ z, float* __restrict__ vx, float* __restrict__ vy,
    float* __restrict__ vz)
{
    if (t.vmax) {
        float3 lo = t.lo, hi = t.hi;
        if (BATCH && t.sid) {
            const uint32_t sc = __ldg(t.sid + i);
            lo = make_float3(__ldg(t.lo_s + 3 * sc), __ldg(t.lo_s + 3 * sc + 1),
                __ldg(t.lo_s + 3 * sc + 2));
            hi = make_float3(__ldg(t.hi_s + 3 * sc), __ldg(t.hi_s + 3 * sc + 1),
                __ldg(t.hi_s + 3 * sc + 2));
        }
        // _hard_enforce_bounds, scene.cu:466-483
        if (px <= lo.x || py <= lo.y || pz <= lo.z || hi.x <= px || hi.y <= py || hi.z <= pz) {
            const float d = (float)-0.1;
            nvx = nvx * d;
            nvy = nvy * d;
            nvz = nvz * d;
        }
        px = fmaxf(fminf(px, hi.x), lo.x);
        py = fmaxf(fminf(py, hi.y), lo.y);
        pz = fmaxf(fminf(pz, hi.z), lo.z);
    }
    vx[i] = nvx;
    vy[i] = nvy;
    vz[i] = nvz;
    x[i] = px;
    y[i] = py;
    z[i] = pz;
    if (!BATCH && t.keys)
        prekey(t, i, px, py, pz);
    return t.vmax ? norm3df(nvx, nvy, nvz) : 0.f; // cfl.cu:13-18
}

// block maximum of v into *t.vmax (all threads of the block call this)
__device__ __forceinline__ void tail_reduce(const Tail& t, float v)
{
    if (!t.vmax)
        return;
    __shared__ float s_max[32];
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0)
        s_max[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (unsigned w = 1; w < (blockDim.x + 31) / 32; ++w)
            v = fmaxf(v, s_max[w]);
        // most blocks find a larger maximum already there: skip their atomic
        if (v > __ldcg(t.vmax))
            atomic_max_nonneg(t.vmax, v);
    }
}

// ---- batched scenes: persistent launches over the active tiles --------------
// The sweeps of a batch's pressure loop (PCISPH prediction and pressure,
// IISPH pressure accelerations and Jacobi) run as persistent launches: a
// fixed grid of blocks walks the tiles (blockDim.x consecutive particles) in
// order, block b taking tiles b, b + gridDim.x, ..., and skips a tile whose
// scenes have all converged, so converged scenes cost a few loads per tile
// and the equal-sized tiles spread the remaining work evenly over the SMs
// whatever the scenes' sizes. Tiles are walked in index order (neighbouring
// blocks work on neighbouring tiles, which share neighbour data in the L2).
struct Tiles {
    const uint16_t* sid;   // scene of each particle
    const uint8_t* active; // per scene: still iterating
    uint32_t n;            // particles
    uint32_t count;        // tiles: ceil(n / blockDim.x)
};

// whether tile t holds a particle of a scene still iterating (the same value
// in every thread of the block)
__device__ __forceinline__ bool tile_active(const Tiles& tl, uint32_t t)
{
    const uint32_t first = t * blockDim.x;
    const uint32_t last = min(first + blockDim.x, tl.n) - 1u;
    for (uint32_t s = __ldg(tl.sid + first), e = __ldg(tl.sid + last); s <= e; ++s)
        if (__ldg(tl.active + s))
            return true;
    return false;
}

// blocks of a persistent launch of `kern`: as many as the SMs hold at once
// (its occupancy at bs threads), at most one per tile
template <class Kern>
unsigned persistent_grid(Kern kern, unsigned bs, unsigned tiles)
{
    int dev = 0, sms = 0, per_sm = 0;
    REYN_CUDA(cudaGetDevice(&dev));
    REYN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    REYN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, int(bs), 0));
    return std::max(1u, std::min(tiles, unsigned(sms) * unsigned(std::max(per_sm, 1))));
}

// the persistent loop of a tile kernel: `body` runs for particle i of every
// active tile assigned to this block (all threads of a block take the same
// iterations, so bodies may synchronise the block)
#define REYN_TILE_LOOP(tl, body)                                                \
    for (uint32_t t_ = blockIdx.x; t_ < (tl).count; t_ += gridDim.x) {           \
        if (!tile_active(tl, t_))                                              \
            continue;                                                          \
        const uint32_t i = t_ * blockDim.x + threadIdx.x;                       \
        body;                                                                  \
    }

// ---- passes ----------------------------------------------------------------

// compute_densities (solver.cuh:18-38) + cached boundary sums + the step's
// neighbour list, written entry by entry (a block's rows form one 32 KB
// region, so the L2 merges the scattered 4-byte stores into full lines).
// MIXED: the particle's FP16 velocity/density record is written for later
// passes; MIXED_POS16: its 16-byte record for the non-pressure pass. The
// one-scene MIXED_POS16 form is held to 40 registers (12 blocks of 128 per
// SM, 16 bytes spilled) like the other modes' forms: on the 4M dam break
// 753 us per launch against 771 us at the compiler's 47 registers.
template <int KIND, int R, int MIX = 0, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB, ((MIX == MIX_POS16 && !BATCH) ? 65536 / 40 / MB : 0))
k_density(uint32_t n, Fluid f, Bdy b,
    float* __restrict__ rho, float4* __restrict__ vel, float4* __restrict__ bterm,
    uint4* __restrict__ rec_out, uint2* __restrict__ velh_out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    // batched scenes: every lane stays until the boundary sums, which its warp
    // forms together
    if constexpr (!BATCH) {
        if (i >= n)
            return;
    }
    const bool valid = i < n;
    uint32_t scene = 0;
    if constexpr (BATCH) {
        if (valid)
            scene = enter_scene(f, i);
    }
    const float4 me = valid ? f.pm[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    int3 c = make_int3(0, 0, 0);
    uint32_t cnt = 0;
    float rf = 0.f;
    if (valid) {
        c = fluid_cell<R>(f, me);
        uint32_t* __restrict__ row = f.nbr + list_slot(i, 0);
        [[maybe_unused]] Kahan rk; // mixed modes: compensated density sum
        for_each_neighbour<R>(f.g, c, me.x, me.y, me.z, f.pm,
            [&](uint32_t j, const float4& q, float, float, float, float l2) {
                if constexpr (MIX)
                    rk.add(q.w * pair_w<KIND>(f.kc, l2));
                else
                    rf += q.w * pair_w<KIND>(f.kc, l2);
                if (j != i) {
                    if (cnt < KMAX)
                        row[size_t(cnt) * 128] = j;
                    ++cnt;
                }
            });
        if constexpr (MIX)
            rf = rk.sum;
    }
    float4 bs = make_float4(0.f, 0.f, 0.f, 0.f);
    if constexpr (BATCH) {
        bs = boundary_sums_warp<KIND, BATCH>(b, f.kc, valid, scene, me.x, me.y, me.z);
        if (!valid)
            return;
    } else {
        for_each_boundary(b, me.x, me.y, me.z,
            [&](uint32_t, const float4& q, float dx, float dy, float dz, float l2) {
                float w, g;
                pair_wg<KIND>(f.kc, l2, w, g);
                bs.w += q.w * w;
                const float mg = q.w * g;
                bs.x += mg * dx;
                bs.y += mg * dy;
                bs.z += mg * dz;
            });
    }
    const float r = rf + bs.w;
    rho[i] = r;
    vel[i].w = r;
    bterm[i] = bs;
    f.ncount[i] = cnt;
    if constexpr (MIX == MIX_POS16) {
        const float4 v = vel[i];
        const float m0 = __ldg(&f.pm[0].w);
        rec_out[i] = rec_np(f.g, c, me, half_bits(me.w / (m0 != 0.f ? m0 : 1.f)), v.x, v.y, v.z,
            r);
    } else if constexpr (MIX) {
        const float4 v = vel[i];
        velh_out[i] = float4_to_half4(make_float4(v.x, v.y, v.z, r));
    }
}

// write_non_prs_acc_ff (solver.cuh:40-69): gravity + artificial viscosity;
// optionally fused with integrate_a_v_only (solver.cu:3-13) into vel_out
// (and its FP16 copy velh_out under mixed precision)
template <int KIND, int R, int MIX, bool BATCH>
__device__ __forceinline__ void nonpressure(uint32_t n, const Fluid& f,
    const float4* __restrict__ vel, const uint2* __restrict__ velh, float nu10, float eps,
    float3 grav, float dt, float4* __restrict__ acc, float4* __restrict__ vel_out,
    uint2* __restrict__ velh_out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float4 me = f.pm[i];
    const float4 vi = vel[i];
    float ax = grav.x, ay = grav.y, az = grav.z;
    for_each_listed<R, MIX, false, BATCH>(f, i, me,
        [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
            const float4 vj = nbr_vel<MIX>(vel, velh, j);
            const float vdx = fmaf(vi.x - vj.x, dx, fmaf(vi.y - vj.y, dy, (vi.z - vj.z) * dz));
            // one division per pair: (10 nu m_j v_ij.x_ij / rho_j) / (l2 + eps) g
            const float s = (nu10 * q.w * vdx * pair_g<KIND>(f.kc, l2)) / (vj.w * (l2 + eps));
            ax += s * dx;
            ay += s * dy;
            az += s * dz;
        });
    acc[i] = make_float4(ax, ay, az, 0.f);
    if (vel_out) {
        const float4 vs = make_float4(vi.x + dt * ax, vi.y + dt * ay, vi.z + dt * az, vi.w);
        vel_out[i] = vs;
        if constexpr (MIX)
            velh_out[i] = float4_to_half4(vs);
    }
}

__device__ __forceinline__ float eos_sesph(float rho, float k, float rho0)
{
    return fmaxf(0.f, k * (rho / rho0 - 1.f)); // SESPH.cu:6-12
}

// _compute_accelerations (SESPH.cu:15-65) fused with integrate (solver.cu:
// 15-32): writes the new SoA state
template <int KIND, int R, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB) k_sesph(uint32_t n, Fluid f,
    const float4* __restrict__ vel, const float4* __restrict__ bterm, float k, float rho0,
    float nu10, float eps, float3 grav, float dt, float4* __restrict__ acc,
    float* __restrict__ x, float* __restrict__ y, float* __restrict__ z,
    float* __restrict__ vx, float* __restrict__ vy, float* __restrict__ vz, Tail tail)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float vn = 0.f;
    if (i < n) {
    const float4 me = f.pm[i];
    const float4 vi = vel[i];
    const float pi = eos_sesph(vi.w, k, rho0);
    const float pri = pi / (vi.w * vi.w);
    float ax = grav.x, ay = grav.y, az = grav.z;
    for_each_listed<R, 0, false, BATCH>(f, i, me,
        [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
            const float4 vj = __ldg(vel + j);
            const float pj = eos_sesph(vj.w, k, rho0);
            const float vdx = fmaf(vi.x - vj.x, dx, fmaf(vi.y - vj.y, dy, (vi.z - vj.z) * dz));
            const float visc = (nu10 * q.w * vdx) / (vj.w * (l2 + eps));
            const float prs = q.w * (pri + pj / (vj.w * vj.w));
            const float s = (visc - prs) * pair_g<KIND>(f.kc, l2);
            ax += s * dx;
            ay += s * dy;
            az += s * dz;
        });
    const float4 bt = bterm[i];
    ax -= pri * bt.x;
    ay -= pri * bt.y;
    az -= pri * bt.z;
    acc[i] = make_float4(ax, ay, az, 0.f);
    const float nvx = vi.x + dt * ax, nvy = vi.y + dt * ay, nvz = vi.z + dt * az;
    vn = store_state<BATCH>(tail, i, me.x + dt * nvx, me.y + dt * nvy, me.z + dt * nvz, nvx, nvy, nvz,
        x, y, z, vx, vy, vz);
    }
    tail_reduce(tail, vn);
}

// predict_rho (solver.cuh:71-105); the boundary part uses the cached sums:
// sum_b m_b (W + dt grad W . v_i) = rho_b + dt g_b . v_i
#define REYN_PCISPH_PREDICT_ARGS uint32_t n, Fluid f, const float4* __restrict__ vel, \
    const float4* __restrict__ bterm, float dt, float* __restrict__ rho, float k, float rho0, \
    float* __restrict__ pr, SweepStats* stats
#define REYN_PCISPH_PREDICT_PASS n, f, vel, bterm, dt, rho, k, rho0, pr, stats

template <int KIND, int R, bool BATCH>
__device__ __forceinline__ void pcisph_predict(uint32_t i, REYN_PCISPH_PREDICT_ARGS)
{
    double contrib = 0.0;
    constexpr bool batched = BATCH;
    uint32_t sc = 0;
    bool live = i < n;
    if (live) {
        if constexpr (BATCH) {
            sc = scene_of(f.g, i);
            live = scene_live(f, sc);
        }
    }
    if (live) {
        const float4 me = f.pm[i];
        const float4 vi = vel[i];
        // the list excludes the particle itself: its term is m_i W(0)
        float r = me.w * pair_w<KIND>(f.kc, 0.f);
        for_each_listed<R, 0, false, BATCH>(f, i, me,
            [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
                const float4 vj = __ldg(vel + j);
                float w, g;
                pair_wg<KIND>(f.kc, l2, w, g);
                const float vdx = fmaf(vi.x - vj.x, dx, fmaf(vi.y - vj.y, dy, (vi.z - vj.z) * dz));
                r += q.w * (w + dt * (g * vdx));
            });
        const float4 bt = bterm[i];
        r += bt.w + dt * fmaf(bt.x, vi.x, fmaf(bt.y, vi.y, bt.z * vi.z));
        rho[i] = r;
        // the pressure term p / rho^2 of the next pass (_eos_pcisph,
        // PCISPH.cu:15-19), once per particle instead of once per pair
        pr[i] = fmaxf(0.f, k * (r - rho0)) / (r * r);
        contrib = r;
    }
    if constexpr (batched)
        scene_accumulate(stats, sc, live, 0u, 0.0, contrib, 0.f);
    else
        block_accumulate(stats, 0u, 0.0, contrib, 0.f);
}

template <int KIND, int R, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB) k_pcisph_predict(REYN_PCISPH_PREDICT_ARGS)
{
    pcisph_predict<KIND, R, BATCH>(blockIdx.x * blockDim.x + threadIdx.x,
        REYN_PCISPH_PREDICT_PASS);
}

template <int KIND, int R, int MB>
__global__ void __launch_bounds__(MB) k_pcisph_predict_tiles(REYN_PCISPH_PREDICT_ARGS, Tiles tl)
{
    REYN_TILE_LOOP(tl, (pcisph_predict<KIND, R, true>(i, REYN_PCISPH_PREDICT_PASS)));
}

// _write_pcisph_prs_acc (PCISPH.cu:21-56) + v += dt a in place
#define REYN_PCISPH_PRESSURE_ARGS uint32_t n, Fluid f, const float* __restrict__ rho, \
    const float* __restrict__ pr, const float4* __restrict__ bterm, float k, float rho0, \
    float r0i, float dt, float4* __restrict__ acc, float4* __restrict__ vel
#define REYN_PCISPH_PRESSURE_PASS n, f, rho, pr, bterm, k, rho0, r0i, dt, acc, vel

template <int KIND, int R, bool BATCH>
__device__ __forceinline__ void pcisph_pressure(uint32_t i, REYN_PCISPH_PRESSURE_ARGS)
{
    if (i >= n)
        return;
    if constexpr (BATCH) {
        if (!scene_live(f, scene_of(f.g, i)))
            return;
    }
    const float4 me = f.pm[i];
    const float ri = rho[i];
    const float pi = fmaxf(0.f, k * (ri - rho0));
    const float pri = pi / (ri * ri);
    float ax = 0.f, ay = 0.f, az = 0.f;
    for_each_listed<R, 0, false, BATCH>(f, i, me,
        [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
            const float s = q.w * (pri + __ldg(pr + j)) * pair_g<KIND>(f.kc, l2);
            ax += s * dx;
            ay += s * dy;
            az += s * dz;
        });
    const float4 bt = bterm[i];
    const float cb = 0.5f * (pri + pi * r0i);
    ax = -ax - cb * bt.x;
    ay = -ay - cb * bt.y;
    az = -az - cb * bt.z;
    acc[i] = make_float4(ax, ay, az, 0.f);
    float4 v = vel[i];
    v.x += dt * ax;
    v.y += dt * ay;
    v.z += dt * az;
    vel[i] = v;
}

template <int KIND, int R, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB) k_pcisph_pressure(REYN_PCISPH_PRESSURE_ARGS)
{
    pcisph_pressure<KIND, R, BATCH>(blockIdx.x * blockDim.x + threadIdx.x,
        REYN_PCISPH_PRESSURE_PASS);
}

template <int KIND, int R, int MB>
__global__ void __launch_bounds__(MB) k_pcisph_pressure_tiles(REYN_PCISPH_PRESSURE_ARGS, Tiles tl)
{
    REYN_TILE_LOOP(tl, (pcisph_pressure<KIND, R, true>(i, REYN_PCISPH_PRESSURE_PASS)));
}

// the final position update of integrate (solver.cu:15-32) when v already
// holds v + dt a
template <bool BATCH = false>
__global__ void k_advect(uint32_t n, const float4* __restrict__ pm,
    const float4* __restrict__ vel, float dt, float* __restrict__ x, float* __restrict__ y,
    float* __restrict__ z, float* __restrict__ vx, float* __restrict__ vy,
    float* __restrict__ vz, Tail tail)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float vn = 0.f;
    if (i < n) {
        const float4 p = pm[i];
        const float4 v = vel[i];
        vn = store_state<BATCH>(tail, i, p.x + dt * v.x, p.y + dt * v.y, p.z + dt * v.z, v.x, v.y, v.z,
            x, y, z, vx, vy, vz);
    }
    tail_reduce(tail, vn);
}

// _compute_diagonal_elem_and_source_term (IISPH.cu:11-66) + warm start
// (IISPH.cu:193-209)
template <int KIND, int R, int MIX = 0, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB) k_iisph_diag(uint32_t n, Fluid f,
    const float4* __restrict__ vel, const uint2* __restrict__ velh,
    const float4* __restrict__ bterm, float rho0, float dt,
    float omega, int warmstart, float tiny, float* __restrict__ aii, float* __restrict__ sii,
    float* __restrict__ p)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float4 me = f.pm[i];
    const float4 vi = vel[i];
    float gx = 0.f, gy = 0.f, gz = 0.f, vdiv = 0.f, gsq = 0.f;
    [[maybe_unused]] Kahan vk; // mixed modes: compensated divergence sum
    for_each_listed<R, MIX, false, BATCH>(f, i, me,
        [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
            const float4 vj = nbr_vel<MIX>(vel, velh, j);
            const float g = pair_g<KIND>(f.kc, l2);
            const float mg = q.w * g;
            gx += mg * dx;
            gy += mg * dy;
            gz += mg * dz;
            const float dv = mg * fmaf(dx, vi.x - vj.x, fmaf(dy, vi.y - vj.y, dz * (vi.z - vj.z)));
            if constexpr (MIX)
                vk.add(dv);
            else
                vdiv += dv;
            gsq += mg * g * l2;
        });
    if constexpr (MIX)
        vdiv = vk.sum;
    const float4 bt = bterm[i];
    gx += bt.x;
    gy += bt.y;
    gz += bt.z;
    const float gss = fmaf(gx, gx, fmaf(gy, gy, gz * gz));
    const float a = -dt * (gss + me.w * gsq) / (rho0 * rho0);
    const float s = (rho0 - vi.w) / dt - (vdiv + fmaf(vi.x, bt.x, fmaf(vi.y, bt.y, vi.z * bt.z)));
    aii[i] = a;
    sii[i] = s;
    p[i] = warmstart ? p[i] * 0.5f : jacobi_update(omega, a, 0.f, s, tiny);
}

// the diagonal pass fused with the first sweep's pressure accelerations
// under the warm start: every neighbour's warm-started pressure is half its
// carried pressure, so a_i = -(1/rho0^2)(sum m_j (p_i' + p_j') grad W_ij +
// p_i' g_b) with p' = 0.5 p can be summed in the same neighbour loop. p_old
// is read, p_new written (p_new = 0.5 p_old).
template <int KIND, int R, int MIX = 0, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB) k_iisph_diag_pacc(uint32_t n, Fluid f,
    const float4* __restrict__ vel, const uint2* __restrict__ velh,
    const float4* __restrict__ bterm, float rho0, float dt,
    float r0i, const float* __restrict__ p_old, float* __restrict__ aii,
    float* __restrict__ sii, float* __restrict__ p_new, float4* __restrict__ acc,
    uint2* __restrict__ acch_out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float4 me = f.pm[i];
    const float4 vi = vel[i];
    const float pi = p_old[i] * 0.5f;
    float gx = 0.f, gy = 0.f, gz = 0.f, vdiv = 0.f, gsq = 0.f;
    [[maybe_unused]] Kahan vk; // mixed modes: compensated divergence sum
    float ax = 0.f, ay = 0.f, az = 0.f;
    for_each_listed<R, MIX, false, BATCH>(f, i, me,
        [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
            const float4 vj = nbr_vel<MIX>(vel, velh, j);
            const float pj = __ldg(p_old + j) * 0.5f;
            const float g = pair_g<KIND>(f.kc, l2);
            const float mg = q.w * g;
            gx += mg * dx;
            gy += mg * dy;
            gz += mg * dz;
            const float dv = mg * fmaf(dx, vi.x - vj.x, fmaf(dy, vi.y - vj.y, dz * (vi.z - vj.z)));
            if constexpr (MIX)
                vk.add(dv);
            else
                vdiv += dv;
            gsq += mg * g * l2;
            const float sp = q.w * (pi + pj) * g;
            ax += sp * dx;
            ay += sp * dy;
            az += sp * dz;
        });
    if constexpr (MIX)
        vdiv = vk.sum;
    const float4 bt = bterm[i];
    const float4 ai = make_float4(-r0i * (ax + pi * bt.x), -r0i * (ay + pi * bt.y),
        -r0i * (az + pi * bt.z), 0.f);
    acc[i] = ai;
    if constexpr (MIX)
        acch_out[i] = pack_acc(ai.x, ai.y, ai.z);
    gx += bt.x;
    gy += bt.y;
    gz += bt.z;
    const float gss = fmaf(gx, gx, fmaf(gy, gy, gz * gz));
    aii[i] = -dt * (gss + me.w * gsq) / (rho0 * rho0);
    sii[i] = (rho0 - vi.w) / dt - (vdiv + fmaf(vi.x, bt.x, fmaf(vi.y, bt.y, vi.z * bt.z)));
    p_new[i] = pi;
}

// _set_pressure_accelerations (IISPH.cu:68-98)
template <int KIND, int R, int MIX, bool BATCH>
__device__ __forceinline__ void iisph_pacc(uint32_t i, uint32_t n, const Fluid& f,
    const float* __restrict__ p, const float4* __restrict__ bterm, float r0i,
    float4* __restrict__ acc, uint2* __restrict__ acch_out, const uint32_t* __restrict__ gate)
{
    // a captured step's loop body: the first sweep uses the accelerations of
    // the pass before the loop
    if (i >= n || (gate && !*gate))
        return;
    if constexpr (BATCH) {
        if (!scene_live(f, scene_of(f.g, i)))
            return;
    }
    const float4 me = f.pm[i];
    const float pi = p[i];
    float ax = 0.f, ay = 0.f, az = 0.f;
    for_each_listed<R, MIX, false, BATCH>(f, i, me,
        [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
            const float s = q.w * (pi + __ldg(p + j)) * pair_g<KIND>(f.kc, l2);
            ax += s * dx;
            ay += s * dy;
            az += s * dz;
        });
    const float4 bt = bterm[i];
    const float4 ai = make_float4(-r0i * (ax + pi * bt.x), -r0i * (ay + pi * bt.y),
        -r0i * (az + pi * bt.z), 0.f);
    acc[i] = ai;
    if constexpr (MIX)
        acch_out[i] = pack_acc(ai.x, ai.y, ai.z);
}

// _jacobi_update_pressures (IISPH.cu:119-162); the convergence bitmask of the
// reference becomes a count of particles above the threshold, reduced per
// block together with the FP64 sum of max(0, error)
template <int KIND, int R, int MIX, bool BATCH>
__device__ __forceinline__ void iisph_jacobi(uint32_t i, uint32_t n, const Fluid& f,
    const float4* __restrict__ acc, const float4* __restrict__ bterm,
    const float* __restrict__ aii, const float* __restrict__ sii, float* __restrict__ p,
    float dt, float omega, float tiny, float thr, SweepStats* stats)
{
    unsigned over = 0;
    double epos = 0.0;
    float emax = 0.f;
    constexpr bool batched = BATCH;
    uint32_t sc = 0;
    bool live = i < n;
    if (live) {
        if constexpr (BATCH) {
            sc = scene_of(f.g, i);
            live = scene_live(f, sc);
        }
    }
    if (live) {
        const float4 me = f.pm[i];
        const float4 ai = acc[i];
        // mixed: neighbour accelerations arrive scaled by ACC_SCALE; the own
        // one is scaled to match and the sum scaled back
        constexpr float AS = MIX ? ACC_SCALE : 1.f;
        const float3 as = make_float3(ai.x * AS, ai.y * AS, ai.z * AS);
        float sum = 0.f;
        for_each_listed<R, MIX, (MIX != 0), BATCH>(f, i, me,
            [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
                float3 aj;
                if constexpr (MIX) {
                    aj = make_float3(q.x, q.y, q.z);
                } else {
                    const float4 a = __ldg(acc + j);
                    aj = make_float3(a.x, a.y, a.z);
                }
                const float d = fmaf(as.x - aj.x, dx, fmaf(as.y - aj.y, dy, (as.z - aj.z) * dz));
                sum += q.w * (pair_g<KIND>(f.kc, l2) * d);
            });
        if constexpr (MIX)
            sum *= 1.f / ACC_SCALE;
        const float4 bt = bterm[i];
        const float Ap = dt * (sum + fmaf(ai.x, bt.x, fmaf(ai.y, bt.y, ai.z * bt.z)));
        const float s = sii[i];
        p[i] = p[i] + jacobi_update(omega, aii[i], Ap, s, tiny);
        const float err = (Ap - s) * dt;
        over = err > thr ? 1u : 0u;
        epos = err > 0.f ? (double)err : 0.0;
        emax = fmaxf(err, 0.f);
    }
    if constexpr (batched)
        scene_accumulate(stats, sc, live, over, epos, 0.0, emax);
    else
        block_accumulate(stats, over, epos, 0.0, emax);
}

template <int KIND, int R, int MIX = 0, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB) k_iisph_pacc(uint32_t n, Fluid f,
    const float* __restrict__ p, const float4* __restrict__ bterm, float r0i,
    float4* __restrict__ acc, uint2* __restrict__ acch_out, const uint32_t* __restrict__ gate)
{
    iisph_pacc<KIND, R, MIX, BATCH>(blockIdx.x * blockDim.x + threadIdx.x, n, f, p, bterm, r0i,
        acc, acch_out, gate);
}

template <int KIND, int R, int MIX = 0, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB) k_iisph_jacobi(uint32_t n, Fluid f,
    const float4* __restrict__ acc, const float4* __restrict__ bterm,
    const float* __restrict__ aii, const float* __restrict__ sii, float* __restrict__ p,
    float dt, float omega, float tiny, float thr, SweepStats* stats)
{
    iisph_jacobi<KIND, R, MIX, BATCH>(blockIdx.x * blockDim.x + threadIdx.x, n, f, acc, bterm,
        aii, sii, p, dt, omega, tiny, thr, stats);
}

template <int KIND, int R, int MIX, int MB>
__global__ void __launch_bounds__(MB) k_iisph_pacc_tiles(uint32_t n, Fluid f,
    const float* __restrict__ p, const float4* __restrict__ bterm, float r0i,
    float4* __restrict__ acc, uint2* __restrict__ acch_out, const uint32_t* __restrict__ gate,
    Tiles tl)
{
    REYN_TILE_LOOP(tl, (iisph_pacc<KIND, R, MIX, true>(i, n, f, p, bterm, r0i, acc, acch_out,
        gate)));
}

template <int KIND, int R, int MIX, int MB>
__global__ void __launch_bounds__(MB) k_iisph_jacobi_tiles(uint32_t n, Fluid f,
    const float4* __restrict__ acc, const float4* __restrict__ bterm,
    const float* __restrict__ aii, const float* __restrict__ sii, float* __restrict__ p,
    float dt, float omega, float tiny, float thr, SweepStats* stats, Tiles tl)
{
    REYN_TILE_LOOP(tl, (iisph_jacobi<KIND, R, MIX, true>(i, n, f, acc, bterm, aii, sii, p, dt,
        omega, tiny, thr, stats)));
}

// The mixed modes' sweep kernels for one scene and the polynomial kernels,
// compiled for 40 registers a thread (12 resident blocks of 128): the FP16
// neighbour records leave these passes waiting on load latency rather than
// on the L1 data pipe, and the extra resident warps cover it (Jacobi 0.315 ->
// 0.251 ms at 4M particles). The FP32 passes are L1-bound and keep the
// compiler's own register choice.
template <int KIND, int MIX>
constexpr bool occupancy_variant = MIX != 0 && KIND != K_COS;

template <int KIND, int R, int MIX, int MB>
__global__ void __launch_bounds__(MB, (65536 / 40) / MB) k_iisph_pacc_occ(uint32_t n, Fluid f,
    const float* __restrict__ p, const float4* __restrict__ bterm, float r0i,
    float4* __restrict__ acc, uint2* __restrict__ acch_out, const uint32_t* __restrict__ gate)
{
    iisph_pacc<KIND, R, MIX, false>(blockIdx.x * blockDim.x + threadIdx.x, n, f, p, bterm, r0i,
        acc, acch_out, gate);
}

template <int KIND, int R, int MIX, int MB>
__global__ void __launch_bounds__(MB, (65536 / 40) / MB) k_iisph_jacobi_occ(uint32_t n, Fluid f,
    const float4* __restrict__ acc, const float4* __restrict__ bterm,
    const float* __restrict__ aii, const float* __restrict__ sii, float* __restrict__ p,
    float dt, float omega, float tiny, float thr, SweepStats* stats)
{
    iisph_jacobi<KIND, R, MIX, false>(blockIdx.x * blockDim.x + threadIdx.x, n, f, acc, bterm,
        aii, sii, p, dt, omega, tiny, thr, stats);
}

// a batch's sweeps: persistent launches over the active tiles (tl)
template <int KIND, int R, int MIX, bool BATCH, int MB, class... A>
void launch_iisph_pacc(unsigned nb, unsigned bs, cudaStream_t q, Tiles tl, bool persist,
    A... a)
{
    if constexpr (BATCH) {
        if (persist)
            k_iisph_pacc_tiles<KIND, R, MIX, MB><<<persistent_grid(
                k_iisph_pacc_tiles<KIND, R, MIX, MB>, bs, nb), bs, 0, q>>>(a..., tl);
        else
            k_iisph_pacc<KIND, R, MIX, BATCH, MB><<<nb, bs, 0, q>>>(a...);
    } else if constexpr (occupancy_variant<KIND, MIX>) {
        k_iisph_pacc_occ<KIND, R, MIX, MB><<<nb, bs, 0, q>>>(a...);
    } else {
        k_iisph_pacc<KIND, R, MIX, BATCH, MB><<<nb, bs, 0, q>>>(a...);
    }
}

template <int KIND, int R, int MIX, bool BATCH, int MB, class... A>
void launch_iisph_jacobi(unsigned nb, unsigned bs, cudaStream_t q, Tiles tl, bool persist,
    A... a)
{
    if constexpr (BATCH) {
        if (persist)
            k_iisph_jacobi_tiles<KIND, R, MIX, MB><<<persistent_grid(
                k_iisph_jacobi_tiles<KIND, R, MIX, MB>, bs, nb), bs, 0, q>>>(a..., tl);
        else
            k_iisph_jacobi<KIND, R, MIX, BATCH, MB><<<nb, bs, 0, q>>>(a...);
    } else if constexpr (occupancy_variant<KIND, MIX>) {
        k_iisph_jacobi_occ<KIND, R, MIX, MB><<<nb, bs, 0, q>>>(a...);
    } else {
        k_iisph_jacobi<KIND, R, MIX, BATCH, MB><<<nb, bs, 0, q>>>(a...);
    }
}

#define REYN_NONPRESSURE_ARGS uint32_t n, Fluid f, const float4* __restrict__ vel, \
    const uint2* __restrict__ velh, float nu10, float eps, float3 grav, float dt, \
    float4* __restrict__ acc, float4* __restrict__ vel_out, uint2* __restrict__ velh_out

template <int KIND, int R, int MIX = 0, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB) k_nonpressure(REYN_NONPRESSURE_ARGS)
{
    nonpressure<KIND, R, MIX, BATCH>(n, f, vel, velh, nu10, eps, grav, dt, acc, vel_out,
        velh_out);
}

template <int KIND, int R, int MIX, int MB>
__global__ void __launch_bounds__(MB, (65536 / 48) / MB) k_nonpressure_occ(REYN_NONPRESSURE_ARGS)
{
    nonpressure<KIND, R, MIX, false>(n, f, vel, velh, nu10, eps, grav, dt, acc, vel_out,
        velh_out);
}

#undef REYN_NONPRESSURE_ARGS

// The non-pressure pass (viscosity) waits on gather latency at 9 resident
// blocks of 128 (54-56 registers); compiled for 48 registers (10 blocks) it
// runs 6-8 % faster in every precision mode without spilling.
template <int KIND>
constexpr bool occupancy_variant_np = KIND != K_COS;

template <int KIND, int R, int MIX, bool BATCH, int MB, class... A>
void launch_nonpressure(unsigned nb, unsigned bs, cudaStream_t q, A... a)
{
    if constexpr (!BATCH && occupancy_variant_np<KIND>)
        k_nonpressure_occ<KIND, R, MIX, MB><<<nb, bs, 0, q>>>(a...);
    else
        k_nonpressure<KIND, R, MIX, BATCH, MB><<<nb, bs, 0, q>>>(a...);
}

// final _set_pressure_accelerations + integrate (IISPH.cu:248-257); the
// accelerations go straight to the solver's SoA arrays
template <int KIND, int R, int MIX = 0, bool BATCH = false, int MB = NBR_THREADS>
__global__ void __launch_bounds__(MB) k_iisph_final(uint32_t n, Fluid f,
    const float* __restrict__ p, const float4* __restrict__ bterm, float r0i,
    const float4* __restrict__ vel, float dt, Soa3 acc,
    float* __restrict__ x, float* __restrict__ y, float* __restrict__ z,
    float* __restrict__ vx, float* __restrict__ vy, float* __restrict__ vz, Tail tail)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float vn = 0.f;
    if (i < n) {
    const float4 me = f.pm[i];
    const float pi = p[i];
    float ax = 0.f, ay = 0.f, az = 0.f;
    for_each_listed<R, MIX, false, BATCH>(f, i, me,
        [&](uint32_t j, const float4& q, float dx, float dy, float dz, float l2) {
            const float s = q.w * (pi + __ldg(p + j)) * pair_g<KIND>(f.kc, l2);
            ax += s * dx;
            ay += s * dy;
            az += s * dz;
        });
    const float4 bt = bterm[i];
    ax = -r0i * (ax + pi * bt.x);
    ay = -r0i * (ay + pi * bt.y);
    az = -r0i * (az + pi * bt.z);
    acc.x[i] = ax;
    acc.y[i] = ay;
    acc.z[i] = az;
    const float4 v = vel[i];
    const float nvx = v.x + dt * ax, nvy = v.y + dt * ay, nvz = v.z + dt * az;
    vn = store_state<BATCH>(tail, i, me.x + dt * nvx, me.y + dt * nvy, me.z + dt * nvz, nvx, nvy, nvz,
        x, y, z, vx, vy, vz);
    }
    tail_reduce(tail, vn);
}

// SESPH and PCISPH: the packed accelerations to the solver's SoA arrays
__global__ void k_unpack_acc(uint32_t n, const float4* __restrict__ acc, float* __restrict__ ax,
    float* __restrict__ ay, float* __restrict__ az)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float4 a = acc[i];
    ax[i] = a.x;
    ay[i] = a.y;
    az[i] = a.z;
}

__global__ void k_gather_p(uint32_t n, const uint32_t* __restrict__ perm,
    const float* __restrict__ src, float* __restrict__ dst)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[perm[i]];
}

#include "passes_rec.cuh"

template <class F> void dispatch(int kind, int range, F&& f)
{
    auto go = [&](auto K) {
        if (range == 2)
            f(K, std::integral_constant<int, 2> {});
        else
            f(K, std::integral_constant<int, 1> {});
    };
    switch (kind) {
    case K_C2: go(std::integral_constant<int, K_C2> {}); break;
    case K_B3: go(std::integral_constant<int, K_B3> {}); break;
    case K_W6: go(std::integral_constant<int, K_W6> {}); break;
    case K_COS: go(std::integral_constant<int, K_COS> {}); break;
    default: fail(REYN_ERR_INVALID, "unknown kernel");
    }
}

} // namespace

double pcisph_template_delta(int kind, float h);
template <int MB>
void solver_step_t(reyn_solver& sv, reyn_particles& st, const Grid& grid,
    const reyn_boundary* bdy, float dt, cudaStream_t s, const float* bmin, const float* bmax)
{
    const reyn_params& P = sv.prm;
    // max_iter 0 is unbounded as in the reference; a hard bound still ends a
    // loop that cannot converge (a non-finite state), far above any sweep
    // count a converging step needs
    constexpr uint32_t SWEEP_SAFETY_LIMIT = 100000;
    const uint32_t max_it = P.max_iter ? P.max_iter : SWEEP_SAFETY_LIMIT;
    const uint32_t n = st.n;
    sv.vmax_valid = false;
    require(n == sv.n, "particle count differs from the solver's");
    require(dt > 0.f && std::isfinite(dt), "dt must be positive and finite");
    // the solver's own copy in grid order (a step on a construct-built grid)
    const bool shadow = &st == sv.shadow.get() && grid.n == n;
    if (!shadow && !(grid.reordered && grid.reordered_state == &st && grid.reorder_epoch == st.epoch
            && grid.n == n))
        fail(REYN_ERR_NOT_READY,
            "the grid must come from construct_and_reorder or construct over this particle state");
    ensure_buffers(sv, n);
    if (!st.packed_valid)
        pack_state(st, s);
    // IISPH carries p across steps in particle order: follow the permutation
    if (sv.scheme == REYN_IISPH && n) {
        if (sv.p_state == &st && sv.p_epoch + 1 == st.epoch) {
            REYN_KERNEL("k_gather_p", s,
                k_gather_p<<<blocks_for(n, THREADS), THREADS, 0, s>>>(
                n, grid.sorted.get(), sv.p.get(), sv.p_tmp.get()));
            sv.p.swap(sv.p_tmp);
        } else if (!(sv.p_state == &st && sv.p_epoch == st.epoch)) {
            sv.p.zero(s); // no step on this ordering yet: cold start
        }
        sv.p_state = &st;
        sv.p_epoch = st.epoch;
    }
    sv.stats = reyn_step_stats {};
    GraphCtx* const gx = sv.graph; // non-null: this step is being captured
    const uint32_t ns = grid.n_scenes;
    require(!bdy || !bdy->nb || bdy->grid.n_scenes == ns,
        "batched grids need a boundary batched over the same scenes");
    sv.n_scenes = ns;
    if (ns) {
        sv.scene_stats.resize(size_t(ns) * sizeof(SweepStats));
        sv.scene_active.resize(ns);
        sv.scene_iters.resize(ns);
        sv.scene_avg.resize(ns);
        sv.scene_max.resize(ns);
        sv.scene_first.resize(ns + 1);
        sv.n_active.resize(1);
        if (!sv.n_active_host)
            sv.n_active_host = std::make_unique<PinnedArray<uint32_t>>(1);
        if (!gx) // a capture uploads the offsets before it starts
            REYN_CUDA(cudaMemcpyAsync(sv.scene_first.get(), grid.first.data(),
                (ns + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        REYN_CUDA(cudaMemsetAsync(sv.scene_active.get(), 1, ns, s));
        sv.scene_iters.zero(s);
        sv.scene_avg.zero(s);
        sv.scene_max.zero(s);
    }
    if (n == 0)
        return;

    Fluid f;
    f.g = grid.view(2.f * P.h);
    f.kc = make_kernel(P.kernel, 2.f * P.h);
    f.pm = st.pm.get();
    f.status = const_cast<uint32_t*>(grid.status.get());
    f.nbr = sv.nbr.get();
    f.ncount = sv.ncount.get();
    f.acch = nullptr;
    f.acc32 = sv.acc.get();
    f.active = ns ? sv.scene_active.get() : nullptr;
    Bdy b {};
    if (bdy && bdy->nb) {
        b.g = bdy->view();
        b.g.r2 = f.g.r2;
        b.pm = bdy->pm.get();
        b.near = bdy->near.get();
        b.n = bdy->nb;
    }
    Tail tail {};
    if (bmin && bmax) {
        if (sv.vmax.size() == 0) {
            sv.vmax.resize(1);
            sv.vmax_host = std::make_unique<PinnedArray<float>>(1);
            REYN_CUDA(cudaEventCreateWithFlags(&sv.vmax_ready, cudaEventDisableTiming));
        }
        REYN_CUDA(cudaMemsetAsync(sv.vmax.get(), 0, sizeof(float), s));
        tail.lo = make_float3(bmin[0], bmin[1], bmin[2]);
        tail.hi = make_float3(bmax[0], bmax[1], bmax[2]);
        tail.vmax = sv.vmax.get();
        if (ns) { // batched: every scene's own box
            tail.sid = grid.sid.get();
            tail.lo_s = grid.scene_lo.get();
            tail.hi_s = grid.scene_hi.get();
        }
    }
    // a bounded step on the grid's own reordered state (not captured, not a
    // batch) computes the keys and histogram of that grid's next build
    const bool prekeyed = tail.vmax && !gx && !ns && !shadow && grid.n == n
        && grid.reordered_state == &st && !grid.counts_dirty && !grid.prekey_pending
        && grid.counts.size() == size_t(grid.total_keys()) && grid.status.size() >= 3;
    if (prekeyed) {
        tail.kg = grid.view(grid.geom.r);
        tail.keys = grid.keys.get();
        tail.counts = grid.counts.get();
        tail.kstatus = grid.status.get() + 2;
    }
    const unsigned bs = P.block_size ? P.block_size : NBR_THREADS;
    const unsigned nb = blocks_for(n, bs);
    const float rho0 = P.rho0;
    const float r0i = 1.f / (rho0 * rho0);
    const float nu10 = 10.f * P.nu;
    const float eps = (float)(0.01 * (double)P.h * (double)P.h);
    const float3 grav = make_float3(P.g[0], P.g[1], P.g[2]);
    float* X = st.cur[FX].get();
    float* Y = st.cur[FY].get();
    float* Z = st.cur[FZ].get();
    float* VX = st.cur[FVX].get();
    float* VY = st.cur[FVY].get();
    float* VZ = st.cur[FVZ].get();
    SweepStats* slots = reinterpret_cast<SweepStats*>(sv.sweep_stats.get());
    SweepStats& host = *reinterpret_cast<SweepStats*>(sv.readback->get());
    auto readback = [&](SweepStats* slot) {
        REYN_CUDA(cudaMemcpyAsync(&host, slot, sizeof(SweepStats), cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaStreamSynchronize(s));
    };
    uint32_t iters = 0;
    bool converged = true;
    // batched scenes: per-scene sums of the current sweep, then the per-scene
    // convergence kernel; returns whether any scene iterates on
    SweepStats* scene_slot = reinterpret_cast<SweepStats*>(sv.scene_stats.get());
    // a batch whose scenes no longer all iterate runs its sweeps as
    // persistent launches over the active tiles (plain steps; a captured step
    // keeps the full launches, whose threads of converged scenes return at
    // once). While every scene iterates the full launches are faster.
    bool persist = false;
    auto scenes_go_on = [&](int mode) {
        REYN_CUDA(cudaMemsetAsync(sv.n_active.get(), 0, sizeof(uint32_t), s));
        REYN_KERNEL("k_scene_converge", s,
            k_scene_converge<<<blocks_for(ns, THREADS), THREADS, 0, s>>>(ns, scene_slot,
            sv.scene_first.get(), mode, P.eta, rho0, iters, sv.scene_active.get(),
            sv.scene_iters.get(), sv.scene_avg.get(), sv.scene_max.get(), sv.n_active.get(),
            nullptr, 0, 0));
        REYN_CUDA(cudaMemcpyAsync(sv.n_active_host->get(), sv.n_active.get(), sizeof(uint32_t),
            cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaStreamSynchronize(s));
        persist = *sv.n_active_host->get() < ns;
        return *sv.n_active_host->get() > 0;
    };
    // a captured step's sweep loop: a while node after the work captured so
    // far on s; `sweep(stream, handle)` enqueues one sweep and its decision
    // on the body stream
    auto graph_loop = [&](auto&& sweep) {
        cudaStreamCaptureStatus cs;
        cudaGraph_t cg = nullptr;
        const cudaGraphNode_t* deps = nullptr;
        size_t nd = 0;
        REYN_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &cg, &deps, &nd));
        require(cs == cudaStreamCaptureStatusActive, "no capture in progress");
        cudaGraphConditionalHandle h;
        REYN_CUDA(cudaGraphConditionalHandleCreate(&h, cg, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t node;
        REYN_CUDA(cudaGraphAddNode(&node, cg, deps, nd, &cp));
        REYN_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1,
            cudaStreamSetCaptureDependencies));
        const cudaStream_t bst = gx->body;
        REYN_CUDA(cudaStreamBeginCaptureToGraph(bst, cp.conditional.phGraph_out[0], nullptr,
            nullptr, 0, cudaStreamCaptureModeRelaxed));
        profile_record(&gx->body_names);
        sweep(bst, h);
        profile_record(&gx->top_names);
        cudaGraph_t body_out = nullptr;
        REYN_CUDA(cudaStreamEndCapture(bst, &body_out));
    };
    auto decide = [&](cudaStream_t q, cudaGraphConditionalHandle h, const SweepStats* slot) {
        REYN_KERNEL("k_graph_decide", q,
            k_graph_decide<<<1, 32, 0, q>>>(int(sv.scheme), P.convergence != REYN_CONV_AVERAGE,
            slot, n, P.eta, rho0, P.min_iter, max_it, ns ? sv.n_active.get() : nullptr,
            gx->stats, sv.scheme == REYN_IISPH ? gx->gate : nullptr, h));
    };
    auto scene_converge_dev = [&](cudaStream_t q, int mode) {
        REYN_CUDA(cudaMemsetAsync(sv.n_active.get(), 0, sizeof(uint32_t), q));
        REYN_KERNEL("k_scene_converge", q,
            k_scene_converge<<<blocks_for(ns, THREADS), THREADS, 0, q>>>(ns, scene_slot,
            sv.scene_first.get(), mode, P.eta, rho0, 0, sv.scene_active.get(),
            sv.scene_iters.get(), sv.scene_avg.get(), sv.scene_max.get(), sv.n_active.get(),
            &gx->stats->iters, P.min_iter, max_it));
    };

    // batched scenes: the pressure loop's sweeps run as persistent launches
    // over the tiles of the scenes still iterating
    Tiles tl {};
    if (ns)
        tl = Tiles { grid.sid.get(), sv.scene_active.get(), n, nb };
    const bool mixed = P.precision == REYN_PRECISION_MIXED;
    const bool rec16 = P.precision == REYN_PRECISION_MIXED_POS16;
    uint2* ACH = mixed ? sv.acch.get() : nullptr;
    uint2* VH = mixed ? sv.velh.get() : nullptr;
    uint2* VH2 = mixed ? sv.velh2.get() : nullptr;
    uint4* REC0 = rec16 ? sv.rec0.get() : nullptr;
    uint4* REC1 = rec16 ? sv.rec1.get() : nullptr;
    f.acch = ACH;
    auto body = [&](auto KC, auto RC, auto MC, auto BC) {
        constexpr int K = decltype(KC)::value;
        constexpr int R = decltype(RC)::value;
        constexpr int MIX = decltype(MC)::value;
        constexpr bool B = decltype(BC)::value;
        REYN_KERNEL("k_density", s,
            k_density<K, R, MIX, B, MB><<<nb, bs, 0, s>>>(n, f, b, sv.rho.get(), st.vel.get(),
            sv.bterm.get(), REC0, VH));
        if (sv.scheme == REYN_SESPH) {
            REYN_KERNEL("k_sesph", s,
                k_sesph<K, R, B, MB><<<nb, bs, 0, s>>>(n, f, st.vel.get(), sv.bterm.get(),
                P.k_sesph, rho0, nu10, eps, grav, dt, sv.acc.get(), X, Y, Z, VX, VY, VZ, tail));
            iters = 1;
            if (gx) {
                REYN_KERNEL("k_graph_single_pass", s,
                    k_graph_single_pass<<<blocks_for(std::max<uint32_t>(ns, 1), THREADS), THREADS,
                    0, s>>>(gx->stats, ns ? sv.scene_iters.get() : nullptr, ns));
            } else if (ns) { // one pass per scene
                const std::vector<uint32_t> ones(ns, 1u);
                REYN_CUDA(cudaMemcpyAsync(sv.scene_iters.get(), ones.data(), ns * sizeof(uint32_t),
                    cudaMemcpyHostToDevice, s));
                REYN_CUDA(cudaStreamSynchronize(s));
            }
        } else if (sv.scheme == REYN_PCISPH) {
            const float kp = (float)((sv.pcisph_delta / dt) / dt); // PCISPH.cu:65
            REYN_KERNEL("k_nonpressure", s,
                launch_nonpressure<K, R, 0, B, MB>(nb, bs, s, n, f, (const float4*)st.vel.get(),
                (const uint2*)nullptr, nu10, eps, grav, dt, sv.acc.get(), sv.vel2.get(),
                (uint2*)nullptr));
            float4* v = sv.vel2.get();
            // one PCISPH iteration: prediction and pressure (a batch: over
            // the tiles of the scenes still iterating)
            auto sweep = [&](cudaStream_t q, SweepStats* slot) {
                if (B && persist) {
                    REYN_KERNEL("k_pcisph_predict", q,
                        k_pcisph_predict_tiles<K, R, MB><<<persistent_grid(
                        k_pcisph_predict_tiles<K, R, MB>, bs, nb), bs, 0, q>>>(n, f, v,
                        sv.bterm.get(), dt, sv.rho.get(), kp, rho0, sv.p.get(), slot, tl));
                    REYN_KERNEL("k_pcisph_pressure", q,
                        k_pcisph_pressure_tiles<K, R, MB><<<persistent_grid(
                        k_pcisph_pressure_tiles<K, R, MB>, bs, nb), bs, 0, q>>>(n, f, sv.rho.get(),
                        sv.p.get(), sv.bterm.get(), kp, rho0, r0i, dt, sv.acc.get(), v, tl));
                } else {
                    REYN_KERNEL("k_pcisph_predict", q,
                        k_pcisph_predict<K, R, B, MB><<<nb, bs, 0, q>>>(n, f, v, sv.bterm.get(),
                        dt, sv.rho.get(), kp, rho0, sv.p.get(), slot));
                    REYN_KERNEL("k_pcisph_pressure", q,
                        k_pcisph_pressure<K, R, B, MB><<<nb, bs, 0, q>>>(n, f, sv.rho.get(),
                        sv.p.get(), sv.bterm.get(), kp, rho0, r0i, dt, sv.acc.get(), v));
                }
            };
            if (gx) {
                graph_loop([&](cudaStream_t q, cudaGraphConditionalHandle h) {
                    SweepStats* slot = ns ? scene_slot : slots;
                    REYN_CUDA(cudaMemsetAsync(slot, 0, sizeof(SweepStats) * (ns ? ns : 1), q));
                    sweep(q, slot);
                    if (ns)
                        scene_converge_dev(q, 0);
                    decide(q, h, slot);
                });
            }
            for (; !gx;) {
                SweepStats* slot = ns ? scene_slot : slots + (iters % 64);
                REYN_CUDA(cudaMemsetAsync(slot, 0, sizeof(SweepStats) * (ns ? ns : 1), s));
                sweep(s, slot);
                iters += 1;
                if (ns) {
                    const bool last = max_it && iters >= max_it;
                    if (iters < P.min_iter && !last)
                        continue;
                    if (!scenes_go_on(0))
                        break;
                    if (last) {
                        converged = false;
                        break;
                    }
                    continue;
                }
                if (max_it && iters >= max_it) {
                    if (iters >= P.min_iter) {
                        readback(slot);
                        converged = (float)(host.rho_sum / n) <= (P.eta + 1.f) * rho0;
                    }
                    break;
                }
                if (iters < P.min_iter)
                    continue;
                readback(slot);
                const float avg = (float)(host.rho_sum / n);
                sv.stats.avg_density_error = std::max(0.0, host.rho_sum / n / rho0 - 1.0);
                if (!(avg > (P.eta + 1.f) * rho0)) // PCISPH.cu:101
                    break;
            }
            REYN_KERNEL("k_advect", s,
                k_advect<B><<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, st.pm.get(), v, dt, X, Y, Z,
                VX, VY, VZ, tail));
        } else if constexpr (MIX == MIX_POS16) { // IISPH over 16-byte records
            RecConst rc;
            rc.unit = f.g.cell / FIXQ;
            rc.kc = kernel_in_units(f.kc, rc.unit);
            const float tiny = tiny_threshold();
            const float thr = P.eta * rho0;
            // the density pass wrote the non-pressure records into REC0
            REYN_KERNEL("k_np_rec", s,
                k_np_rec<K, R, B, MB><<<nb, bs, 0, s>>>(n, f, rc, st.vel.get(),
                (const float4*)sv.bterm.get(), sv.p.get(), nu10, eps, grav, dt, REC0, REC1,
                sv.vel2.get(), sv.gq.get()));
            // the sweeps alternate between RX (records with m p, read by the
            // pressure accelerations) and RY (records with m a, read by Jacobi)
            uint4* RX = REC1;
            uint4* RY = REC0;
            auto pacc = [&](cudaStream_t q, const uint32_t* gate) {
                if (B && persist)
                    REYN_KERNEL("k_pacc_rec", q,
                        k_pacc_rec_tiles<K, R, MB><<<persistent_grid(
                        k_pacc_rec_tiles<K, R, MB>, bs, nb), bs, 0, q>>>(n, f, rc,
                        (const float4*)sv.gq.get(), r0i, RX, RY, gate, tl));
                else
                    REYN_KERNEL("k_pacc_rec", q,
                        k_pacc_rec<K, R, B, MB><<<nb, bs, 0, q>>>(n, f, rc,
                        (const float4*)sv.gq.get(), r0i, RX, RY, gate));
            };
            auto jacobi = [&](cudaStream_t q, SweepStats* slot) {
                if (B && persist)
                    REYN_KERNEL("k_jacobi_rec", q,
                        k_jacobi_rec_tiles<K, R, MB><<<persistent_grid(
                        k_jacobi_rec_tiles<K, R, MB>, bs, nb), bs, 0, q>>>(n, f, rc,
                        (const float4*)sv.gq.get(), (const float*)sv.sii.get(), sv.p.get(), dt,
                        P.omega, tiny, thr, slot, RY, RX, tl));
                else
                    REYN_KERNEL("k_jacobi_rec", q,
                        k_jacobi_rec<K, R, B, MB><<<nb, bs, 0, q>>>(n, f, rc,
                        (const float4*)sv.gq.get(), (const float*)sv.sii.get(), sv.p.get(), dt,
                        P.omega, tiny, thr, slot, RY, RX));
            };
            if (P.warmstart) {
                REYN_KERNEL("k_diag_pacc_rec", s,
                    k_diag_pacc_rec<K, R, B, MB><<<nb, bs, 0, s>>>(n, f, rc, sv.vel2.get(),
                    sv.gq.get(), rho0, dt, r0i, sv.p.get(), sv.aii.get(), sv.sii.get(),
                    sv.p_tmp.get(), REC1, REC0));
                sv.p.swap(sv.p_tmp);
            } else {
                REYN_KERNEL("k_diag_rec", s,
                    k_diag_rec<K, R, B, MB><<<nb, bs, 0, s>>>(n, f, rc, sv.vel2.get(),
                    sv.gq.get(), rho0, dt, P.omega, tiny, sv.aii.get(), sv.sii.get(),
                    sv.p.get(), REC1, REC0));
                RX = REC0;
                RY = REC1;
                pacc(s, nullptr);
            }
            if (gx) {
                REYN_CUDA(cudaMemsetAsync(gx->gate, 0, sizeof(uint32_t), s));
                graph_loop([&](cudaStream_t q, cudaGraphConditionalHandle h) {
                    SweepStats* slot = ns ? scene_slot : slots;
                    pacc(q, gx->gate);
                    REYN_CUDA(cudaMemsetAsync(slot, 0, sizeof(SweepStats) * (ns ? ns : 1), q));
                    jacobi(q, slot);
                    if (ns)
                        scene_converge_dev(q, P.convergence == REYN_CONV_AVERAGE ? 1 : 2);
                    decide(q, h, slot);
                });
            }
            for (; !gx;) {
                SweepStats* slot = ns ? scene_slot : slots + (iters % 64);
                REYN_CUDA(cudaMemsetAsync(slot, 0, sizeof(SweepStats) * (ns ? ns : 1), s));
                jacobi(s, slot);
                iters += 1;
                const bool last = max_it && iters >= max_it;
                if (iters < P.min_iter && !last) {
                    pacc(s, nullptr);
                    continue;
                }
                if (ns) {
                    if (!scenes_go_on(P.convergence == REYN_CONV_AVERAGE ? 1 : 2))
                        break;
                    if (last) {
                        converged = false;
                        break;
                    }
                    pacc(s, nullptr);
                    continue;
                }
                readback(slot);
                sv.stats.avg_density_error = host.err_sum / n / rho0;
                sv.stats.max_density_error = host.err_max / rho0;
                const bool more = P.convergence == REYN_CONV_AVERAGE
                    ? host.err_sum / n > (double)P.eta * rho0
                    : host.over > 0; // IISPH.cu:246
                if (!more)
                    break;
                if (last) {
                    converged = false;
                    break;
                }
                pacc(s, nullptr);
            }
            REYN_KERNEL("k_final_rec", s,
                k_final_rec<K, R, B, MB><<<nb, bs, 0, s>>>(n, f, rc,
                (const float4*)sv.gq.get(), r0i, sv.vel2.get(), dt,
                Soa3 { sv.ax.get(), sv.ay.get(), sv.az.get() }, RX, X, Y, Z, VX, VY, VZ, tail));
        } else { // IISPH
            REYN_KERNEL("k_nonpressure", s,
                launch_nonpressure<K, R, MIX, B, MB>(nb, bs, s, n, f, (const float4*)st.vel.get(),
                (const uint2*)VH, nu10, eps, grav, dt, sv.acc.get(), sv.vel2.get(), VH2));
            const float tiny = tiny_threshold();
            auto pacc = [&] {
                REYN_KERNEL("k_iisph_pacc", s,
                    launch_iisph_pacc<K, R, MIX, B, MB>(nb, bs, s, tl, persist, n, f, sv.p.get(),
                    sv.bterm.get(), r0i, sv.acc.get(), ACH, (const uint32_t*)nullptr));
            };
            if (P.warmstart) {
                REYN_KERNEL("k_iisph_diag_pacc", s,
                    k_iisph_diag_pacc<K, R, MIX, B, MB><<<nb, bs, 0, s>>>(n, f, sv.vel2.get(),
                    VH2, sv.bterm.get(), rho0, dt, r0i, sv.p.get(), sv.aii.get(), sv.sii.get(),
                    sv.p_tmp.get(), sv.acc.get(), ACH));
                sv.p.swap(sv.p_tmp);
            } else {
                REYN_KERNEL("k_iisph_diag", s,
                    k_iisph_diag<K, R, MIX, B, MB><<<nb, bs, 0, s>>>(n, f, sv.vel2.get(),
                    VH2, sv.bterm.get(), rho0, dt, P.omega, P.warmstart, tiny, sv.aii.get(),
                    sv.sii.get(), sv.p.get()));
                pacc();
            }
            const float thr = P.eta * rho0;
            if (gx) {
                // the loop body: [gated pressure accelerations, Jacobi update,
                // decision]; the gate is closed for the first sweep
                REYN_CUDA(cudaMemsetAsync(gx->gate, 0, sizeof(uint32_t), s));
                graph_loop([&](cudaStream_t q, cudaGraphConditionalHandle h) {
                    SweepStats* slot = ns ? scene_slot : slots;
                    REYN_KERNEL("k_iisph_pacc", q,
                        launch_iisph_pacc<K, R, MIX, B, MB>(nb, bs, q, tl, persist, n, f, sv.p.get(),
                        sv.bterm.get(), r0i, sv.acc.get(), ACH, (const uint32_t*)gx->gate));
                    REYN_CUDA(cudaMemsetAsync(slot, 0, sizeof(SweepStats) * (ns ? ns : 1), q));
                    REYN_KERNEL("k_iisph_jacobi", q,
                        launch_iisph_jacobi<K, R, MIX, B, MB>(nb, bs, q, tl, persist, n, f,
                        (const float4*)sv.acc.get(), (const float4*)sv.bterm.get(),
                        (const float*)sv.aii.get(), (const float*)sv.sii.get(), sv.p.get(), dt,
                        P.omega, tiny, thr, slot));
                    if (ns)
                        scene_converge_dev(q, P.convergence == REYN_CONV_AVERAGE ? 1 : 2);
                    decide(q, h, slot);
                });
            }
            // IISPH.cu:219-250: [pressure accelerations, Jacobi update]* with
            // the first accelerations computed above
            for (; !gx;) {
                SweepStats* slot = ns ? scene_slot : slots + (iters % 64);
                REYN_CUDA(cudaMemsetAsync(slot, 0, sizeof(SweepStats) * (ns ? ns : 1), s));
                REYN_KERNEL("k_iisph_jacobi", s,
                    launch_iisph_jacobi<K, R, MIX, B, MB>(nb, bs, s, tl, persist, n, f,
                    (const float4*)sv.acc.get(), (const float4*)sv.bterm.get(),
                    (const float*)sv.aii.get(), (const float*)sv.sii.get(), sv.p.get(), dt,
                    P.omega, tiny, thr, slot));
                iters += 1;
                const bool last = max_it && iters >= max_it;
                if (iters < P.min_iter && !last) {
                    pacc();
                    continue;
                }
                if (ns) {
                    if (!scenes_go_on(P.convergence == REYN_CONV_AVERAGE ? 1 : 2))
                        break;
                    if (last) {
                        converged = false;
                        break;
                    }
                    pacc();
                    continue;
                }
                readback(slot);
                sv.stats.avg_density_error = host.err_sum / n / rho0;
                sv.stats.max_density_error = host.err_max / rho0;
                const bool more = P.convergence == REYN_CONV_AVERAGE
                    ? host.err_sum / n > (double)P.eta * rho0
                    : host.over > 0; // IISPH.cu:246
                if (!more)
                    break;
                if (last) {
                    converged = false;
                    break;
                }
                pacc();
            }
            REYN_KERNEL("k_iisph_final", s,
                k_iisph_final<K, R, MIX, B, MB><<<nb, bs, 0, s>>>(n, f, sv.p.get(), sv.bterm.get(),
                r0i, sv.vel2.get(), dt, Soa3 { sv.ax.get(), sv.ay.get(), sv.az.get() }, X, Y, Z,
                VX, VY, VZ, tail));
        }
    };
    dispatch(P.kernel, grid.geom.range, [&](auto KC, auto RC) {
        // batched scenes: the records of the mixed modes use each scene's own
        // grid origin (the cell size is shared), and neighbours never cross
        // scenes, so every mode runs batched
        if (ns && P.precision == REYN_PRECISION_MIXED_POS16)
            body(KC, RC, std::integral_constant<int, MIX_POS16> {}, std::true_type {});
        else if (ns && mixed)
            body(KC, RC, std::integral_constant<int, MIX_F16> {}, std::true_type {});
        else if (ns)
            body(KC, RC, std::integral_constant<int, 0> {}, std::true_type {});
        else if (P.precision == REYN_PRECISION_MIXED_POS16)
            body(KC, RC, std::integral_constant<int, MIX_POS16> {}, std::false_type {});
        else if (mixed)
            body(KC, RC, std::integral_constant<int, MIX_F16> {}, std::false_type {});
        else
            body(KC, RC, std::integral_constant<int, 0> {}, std::false_type {});
    });
    if (sv.scheme != REYN_IISPH) {
        REYN_KERNEL("k_unpack_acc", s,
            k_unpack_acc<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, sv.acc.get(), sv.ax.get(),
            sv.ay.get(), sv.az.get()));
    }
    st.packed_valid = false; // positions moved: the packed copy is stale
    st.version += 1;
    if (prekeyed) {
        Grid& gm = const_cast<Grid&>(grid);
        gm.prekey_pending = true;
        gm.prekey_state = &st;
        gm.prekey_version = st.version;
        gm.prekey_x = st.cur[FX].get();
        gm.prekey_n = n;
    }
    if (tail.vmax) {
        if (!gx) { // a captured step records these after each launch
            REYN_CUDA(cudaMemcpyAsync(sv.vmax_host->get(), tail.vmax, sizeof(float),
                cudaMemcpyDeviceToHost, s));
            REYN_CUDA(cudaEventRecord(sv.vmax_ready, s));
        }
        sv.vmax_state = &st;
        sv.vmax_version = st.version;
        sv.vmax_valid = true;
    }
    sv.stats.iters = iters;
    if (!converged)
        fail(REYN_ERR_ITER_LIMIT, "solver reached max_iter before converging (step completed)");
}


} // namespace reyn
