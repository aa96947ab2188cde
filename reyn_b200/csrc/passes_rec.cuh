// The IISPH passes of the MIXED_POS16 mode: every neighbour loop reads one
// 16-byte record per neighbour (16-bit positions plus the quantity the pass
// needs), so a pair costs one gather instead of two or three, and each pass
// reads little of the particle's own data. Included by passes.cuh inside its
// anonymous namespace.
//
// The pressure passes use the per-particle gradient moment
// G_i = sum_j m_j grad W_ij + g_b (fluid sum from the density pass plus the
// cached boundary sum), which lets the pair terms of the reference's
// equations be split into a per-particle part and a neighbour sum:
//   sum_j m_j (p_i + p_j) grad W_ij + p_i g_b = p_i G_i + sum_j (m_j p_j) grad W_ij
//   sum_j m_j (a_i - a_j).grad W_ij + a_i.g_b = a_i.G_i - sum_j (m_j a_j).grad W_ij
//   sum_j m_j (v_i - v_j).grad W_ij + v_i.g_b = v_i.G_i - sum_j (m_j v_j).grad W_ij
// (IISPH.cu:11-66, 68-98, 108-162). Masses travel as m / m_0 in FP16 (m_0
// the mass of particle 0; exactly 1 for equal masses), pressures in FP32,
// m v and m a in FP16.
//
// Record flow through one step (two buffers, every pass reads one and writes
// the other): density -> NP -> non-pressure -> DG -> diagonal + first
// pressure accelerations -> Y -> [Jacobi -> X -> pressure accelerations ->
// Y]* ... Jacobi -> X -> final pressure accelerations + integration.
// Per particle, the sweeps read gq = (G, a_ii) and the particle's own record
// besides the records of its neighbours: Jacobi takes its own m a from its Y
// record (rounded as its neighbours see it), the pressure pass its own p
// from its X record.
//
// Pair vectors are in units of 1/FIXQ cell, with the kernel constants scaled
// to match (kernel_in_units), so no pair is rescaled. G and gsq are summed by
// the non-pressure pass from the same record pair vectors that the pressure
// passes use, so the split forms above cancel exactly where the reference's
// differences vanish.

// resident blocks the one-scene record passes are compiled for: 56 registers
// a thread (9 blocks of 128 per SM). Measured on the 4M dam break against the
// compiler's own choice (71 registers, 237 us per Jacobi sweep) and caps of
// 48 (214 us) and 40 (217 us, with spills): 209 us.
template <int MB> constexpr int rec_min_blocks = 65536 / 56 / MB;
// the batched forms (scene lookups, per-scene sums) are held to 64 registers,
// 8 blocks of 128 per SM, against the 71 to 92 the compiler takes unbounded

// per-step constants of the record passes
struct RecConst {
    KernelConst kc; // kernel constants for pair vectors in record units
    float unit;     // the record unit (cell / FIXQ) in metres
};

__device__ __forceinline__ float rec_m0(const Fluid& f)
{
    const float m0 = __ldg(&f.pm[0].w);
    return m0 != 0.f ? m0 : 1.f;
}

// write_non_prs_acc_ff (solver.cuh:40-69) + integrate_a_v_only (solver.cu:
// 3-13) over NP records; writes v* (vel_out), gq = (G, gsq) with
// G = sum_j m_j grad W_ij + g_b and gsq = sum_j m_j |grad W_ij|^2, and the DG
// record with m v* and m p_old for the diagonal pass. In record units the
// viscosity term (10 nu m_j v_ij.x_ij g / (rho_j (|x_ij|^2 + eps))) x_ij
// becomes (10 nu m_j v_ij.d g' / (rho_j (unit |d|^2 + eps / unit))) d. The
// quotient is the fast division (2 ulp; its divisor stays far inside
// [2^-126, 2^126] here: rho_j times a distance term between eps / unit and
// 4 cells^2 / unit) where FP32 uses the IEEE one, since rho_j and v_j come
// from FP16 already.
template <int KIND, int R, bool BATCH, int MB>
__global__ void __launch_bounds__(MB, (BATCH ? 65536 / 64 / MB : rec_min_blocks<MB>))
k_np_rec(uint32_t n, Fluid f, RecConst rc,
    const float4* __restrict__ vel, const float4* __restrict__ bterm,
    const float* __restrict__ p_old, float nu10, float eps, float3 grav, float dt,
    const uint4* __restrict__ rec_in, uint4* __restrict__ rec_out,
    float4* __restrict__ vel_out, float4* __restrict__ gq)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float m0 = rec_m0(f);
    const float4 vi = vel[i];
    const uint4 ri = rec_in[i];
    const float eps_u = eps / rc.unit;
    // the pair sums carry m_j / m_0 and rec_g; m_0 and rec_gscale are
    // applied once per particle
    float ax = 0.f, ay = 0.f, az = 0.f, Gx = 0.f, Gy = 0.f, Gz = 0.f, gsq = 0.f;
    for_each_rec<KIND, R, BATCH>(f, rc.kc, rec_in, i, ri,
        [&](uint32_t, const uint4& rj, float3 d, float g) {
            const float l2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
            const float2 vxy = bits_half2(rj.z);
            const float2 vzr = bits_half2(rj.w);
            const float mg = rec_m16(rj) * g;
            const float vdx =
                fmaf(vi.x - vxy.x, d.x, fmaf(vi.y - vxy.y, d.y, (vi.z - vzr.x) * d.z));
            const float s = __fdividef(nu10 * mg * vdx, vzr.y * fmaf(rc.unit, l2, eps_u));
            ax += s * d.x;
            ay += s * d.y;
            az += s * d.z;
            Gx += mg * d.x;
            Gy += mg * d.y;
            Gz += mg * d.z;
            gsq += mg * g * l2;
        });
    const float gs = rec_gscale<KIND>(rc.kc), sm = gs * m0;
    ax = fmaf(ax, sm, grav.x);
    ay = fmaf(ay, sm, grav.y);
    az = fmaf(az, sm, grav.z);
    const float4 bt = bterm[i];
    gq[i] = make_float4(fmaf(Gx, sm, bt.x), fmaf(Gy, sm, bt.y), fmaf(Gz, sm, bt.z),
        gsq * (sm * gs));
    const float4 vs = make_float4(vi.x + dt * ax, vi.y + dt * ay, vi.z + dt * az, vi.w);
    vel_out[i] = vs;
    const float mr = rec_m16(ri);
    rec_out[i] = rec_dg(ri, mr * vs.x, mr * vs.y, mr * vs.z, m0 * mr * p_old[i]);
}

// _compute_diagonal_elem_and_source_term (IISPH.cu:11-66) fused with the
// warm start and the first sweep's pressure accelerations (IISPH.cu:68-98,
// 193-209) over DG records: a_ii needs no neighbour loop (G and gsq come
// from the non-pressure pass); the loop sums the divergence
// sum_j (m_j v*_j).grad W_ij (compensated) and sum_j (m_j p'_j) grad W_ij with
// the warm-started p' = p_old / 2. Writes a_ii (also into gq.w), s_i, p'
// (p_new) and the Y record.
template <int KIND, int R, bool BATCH, int MB>
__global__ void __launch_bounds__(MB, (BATCH ? 65536 / 64 / MB : rec_min_blocks<MB>))
k_diag_pacc_rec(uint32_t n, Fluid f, RecConst rc,
    const float4* __restrict__ vel, float4* __restrict__ gq, float rho0, float dt, float r0i,
    const float* __restrict__ p_old, float* __restrict__ aii, float* __restrict__ sii,
    float* __restrict__ p_new, const uint4* __restrict__ rec_in, uint4* __restrict__ rec_out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float m0 = rec_m0(f);
    const float mi = f.pm[i].w;
    const uint32_t m16 = half_bits(mi / m0);
    const float4 vi = vel[i];
    const float4 gt = gq[i];
    const uint4 ri = rec_in[i];
    const float pi = p_old[i] * 0.5f;
    Kahan vk;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for_each_rec<KIND, R, BATCH>(f, rc.kc, rec_in, i, ri,
        [&](uint32_t, const uint4& rj, float3 d, float g) {
        const float3 mv = rec_dg_vec(rj);
        vk.add(g * fmaf(mv.x, d.x, fmaf(mv.y, d.y, mv.z * d.z)));
        const float sp = g * rec_dg_mp(rj);
        sx += sp * d.x;
        sy += sp * d.y;
        sz += sp * d.z;
    });
    const float gs = rec_gscale<KIND>(rc.kc);
    sx *= gs;
    sy *= gs;
    sz *= gs;
    vk.sum *= gs;
    // the neighbours' pressures are half their carried ones
    const float ax = -r0i * fmaf(pi, gt.x, 0.5f * sx), ay = -r0i * fmaf(pi, gt.y, 0.5f * sy),
                az = -r0i * fmaf(pi, gt.z, 0.5f * sz);
    const float gss = fmaf(gt.x, gt.x, fmaf(gt.y, gt.y, gt.z * gt.z));
    const float a = -dt * (gss + mi * gt.w) / (rho0 * rho0);
    aii[i] = a;
    gq[i].w = a;
    const float vdiv = fmaf(vi.x, gt.x, fmaf(vi.y, gt.y, vi.z * gt.z)) - m0 * vk.sum;
    sii[i] = (rho0 - vi.w) / dt - vdiv;
    p_new[i] = pi;
    const float ma = __half2float(__ushort_as_half((unsigned short)m16)) * ACC_SCALE;
    rec_out[i] = rec_y(ri.x, rec_w1(ri, m16), ma * ax, ma * ay, ma * az);
}

// the diagonal pass without warm start (IISPH.cu:11-66, 193-209): p starts
// from the Jacobi update of zero; writes the X record for the pressure
// accelerations that follow
template <int KIND, int R, bool BATCH, int MB>
__global__ void __launch_bounds__(MB, (BATCH ? 65536 / 64 / MB : rec_min_blocks<MB>))
k_diag_rec(uint32_t n, Fluid f, RecConst rc,
    const float4* __restrict__ vel, float4* __restrict__ gq, float rho0, float dt,
    float omega, float tiny, float* __restrict__ aii, float* __restrict__ sii,
    float* __restrict__ p, const uint4* __restrict__ rec_in, uint4* __restrict__ rec_out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float m0 = rec_m0(f);
    const float mi = f.pm[i].w;
    const float4 vi = vel[i];
    const float4 gt = gq[i];
    const uint4 ri = rec_in[i];
    Kahan vk;
    for_each_rec<KIND, R, BATCH>(f, rc.kc, rec_in, i, ri,
        [&](uint32_t, const uint4& rj, float3 d, float g) {
        const float3 mv = rec_dg_vec(rj);
        vk.add(g * fmaf(mv.x, d.x, fmaf(mv.y, d.y, mv.z * d.z)));
    });
    vk.sum *= rec_gscale<KIND>(rc.kc);
    const float gss = fmaf(gt.x, gt.x, fmaf(gt.y, gt.y, gt.z * gt.z));
    const float a = -dt * (gss + mi * gt.w) / (rho0 * rho0);
    const float vdiv = fmaf(vi.x, gt.x, fmaf(vi.y, gt.y, vi.z * gt.z)) - m0 * vk.sum;
    const float s = (rho0 - vi.w) / dt - vdiv;
    aii[i] = a;
    gq[i].w = a;
    sii[i] = s;
    const float pn = jacobi_update(omega, a, 0.f, s, tiny);
    p[i] = pn;
    rec_out[i] = rec_x(ri.x, rec_w1(ri, half_bits(mi / m0)), pn);
}

// _set_pressure_accelerations (IISPH.cu:68-98) over X records:
// a_i = -(p_i G_i + sum_j (m_j p_j) grad W_ij) / rho0^2, with p_i from the
// particle's own X record; writes the Y record with m a. `gate`: a captured
// step's loop body skips the first sweep's pass.
#define REYN_PACC_REC_ARGS uint32_t n, Fluid f, RecConst rc, const float4* __restrict__ gq, \
    float r0i, const uint4* __restrict__ rec_in, uint4* __restrict__ rec_out, \
    const uint32_t* __restrict__ gate
#define REYN_PACC_REC_PASS n, f, rc, gq, r0i, rec_in, rec_out, gate

template <int KIND, int R, bool BATCH>
__device__ __forceinline__ void pacc_rec(uint32_t i, REYN_PACC_REC_ARGS)
{
    if (i >= n || (gate && !*gate))
        return;
    if constexpr (BATCH) {
        if (!scene_live(f, scene_of(f.g, i)))
            return;
    }
    const float m0 = rec_m0(f);
    const float4 gt = gq[i];
    const uint4 ri = rec_in[i];
    const float pi = rec_x_p(ri);
    float sx = 0.f, sy = 0.f, sz = 0.f;
    for_each_rec<KIND, R, BATCH>(f, rc.kc, rec_in, i, ri,
        [&](uint32_t, const uint4& rj, float3 d, float g) {
        const float sp = g * rec_x_mp(rj);
        sx += sp * d.x;
        sy += sp * d.y;
        sz += sp * d.z;
    });
    const float sm = m0 * rec_gscale<KIND>(rc.kc);
    const float ma = rec_m16(ri) * ACC_SCALE * -r0i;
    rec_out[i] = rec_y(ri.x, ri.y, ma * fmaf(pi, gt.x, sm * sx), ma * fmaf(pi, gt.y, sm * sy),
        ma * fmaf(pi, gt.z, sm * sz));
}

template <int KIND, int R, bool BATCH, int MB>
__global__ void __launch_bounds__(MB, (BATCH ? 65536 / 64 / MB : rec_min_blocks<MB>))
k_pacc_rec(REYN_PACC_REC_ARGS)
{
    pacc_rec<KIND, R, BATCH>(blockIdx.x * blockDim.x + threadIdx.x, REYN_PACC_REC_PASS);
}

template <int KIND, int R, int MB>
__global__ void __launch_bounds__(MB, 65536 / 64 / MB)
k_pacc_rec_tiles(REYN_PACC_REC_ARGS, Tiles tl)
{
    REYN_TILE_LOOP(tl, (pacc_rec<KIND, R, true>(i, REYN_PACC_REC_PASS)));
}

// _jacobi_update_pressures (IISPH.cu:108-162) over Y records:
// Ap = dt (a_i.G_i - sum_j (m_j a_j).grad W_ij) with a_i from the particle's
// own Y record; p += max(0, omega (s - Ap) / a_ii); writes p and the X record;
// the convergence sums as the FP32 sweep's.
#define REYN_JACOBI_REC_ARGS uint32_t n, Fluid f, RecConst rc, const float4* __restrict__ gq, \
    const float* __restrict__ sii, float* __restrict__ p, float dt, float omega, float tiny, \
    float thr, SweepStats* stats, const uint4* __restrict__ rec_in, uint4* __restrict__ rec_out
#define REYN_JACOBI_REC_PASS n, f, rc, gq, sii, p, dt, omega, tiny, thr, stats, rec_in, rec_out

template <int KIND, int R, bool BATCH>
__device__ __forceinline__ void jacobi_rec(uint32_t i, REYN_JACOBI_REC_ARGS)
{
    unsigned over = 0;
    double epos = 0.0;
    float emax = 0.f;
    uint32_t sc = 0;
    bool live = i < n;
    if (live) {
        if constexpr (BATCH) {
            sc = scene_of(f.g, i);
            live = scene_live(f, sc);
        }
    }
    if (live) {
        const float m0 = rec_m0(f);
        const float4 gt = gq[i];
        const uint4 ri = rec_in[i];
        float sum = 0.f;
        for_each_rec<KIND, R, BATCH>(f, rc.kc, rec_in, i, ri,
            [&](uint32_t, const uint4& rj, float3 d, float g) {
                const float3 ma = rec_y_vec(rj);
                sum += g * fmaf(ma.x, d.x, fmaf(ma.y, d.y, ma.z * d.z));
            });
        sum *= rec_gscale<KIND>(rc.kc);
        // m_i a_i ACC_SCALE / m_0 as stored: a_i.G_i = (that . G_i) / (m16_i ACC_SCALE)
        const float3 mai = rec_y_vec(ri);
        const float Ap = dt * (1.f / ACC_SCALE)
            * (fmaf(mai.x, gt.x, fmaf(mai.y, gt.y, mai.z * gt.z)) / rec_m16(ri)
                - m0 * sum);
        const float s = sii[i];
        const float pn = p[i] + jacobi_update(omega, gt.w, Ap, s, tiny);
        p[i] = pn;
        rec_out[i] = rec_x(ri.x, ri.y, pn);
        const float err = (Ap - s) * dt;
        over = err > thr ? 1u : 0u;
        epos = err > 0.f ? (double)err : 0.0;
        emax = fmaxf(err, 0.f);
    }
    if constexpr (BATCH)
        scene_accumulate(stats, sc, live, over, epos, 0.0, emax);
    else
        block_accumulate(stats, over, epos, 0.0, emax);
}

template <int KIND, int R, bool BATCH, int MB>
__global__ void __launch_bounds__(MB, (BATCH ? 65536 / 64 / MB : rec_min_blocks<MB>))
k_jacobi_rec(REYN_JACOBI_REC_ARGS)
{
    jacobi_rec<KIND, R, BATCH>(blockIdx.x * blockDim.x + threadIdx.x, REYN_JACOBI_REC_PASS);
}

template <int KIND, int R, int MB>
__global__ void __launch_bounds__(MB, 65536 / 64 / MB)
k_jacobi_rec_tiles(REYN_JACOBI_REC_ARGS, Tiles tl)
{
    REYN_TILE_LOOP(tl, (jacobi_rec<KIND, R, true>(i, REYN_JACOBI_REC_PASS)));
}

// the last _set_pressure_accelerations + integrate (IISPH.cu:248-257) over X
// records; writes a (SoA) and the SoA state (bounds and the max |v|
// reduction of a bounded step included)
template <int KIND, int R, bool BATCH, int MB>
__global__ void __launch_bounds__(MB, (BATCH ? 65536 / 64 / MB : rec_min_blocks<MB>))
k_final_rec(uint32_t n, Fluid f, RecConst rc,
    const float4* __restrict__ gq, float r0i, const float4* __restrict__ vel, float dt,
    Soa3 acc, const uint4* __restrict__ rec_in, float* __restrict__ x,
    float* __restrict__ y, float* __restrict__ z, float* __restrict__ vx,
    float* __restrict__ vy, float* __restrict__ vz, Tail tail)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    float vn = 0.f;
    if (i < n) {
        const float m0 = rec_m0(f);
        const float4 me = f.pm[i];
        const float4 gt = gq[i];
        const uint4 ri = rec_in[i];
        const float pi = rec_x_p(ri);
        float sx = 0.f, sy = 0.f, sz = 0.f;
        for_each_rec<KIND, R, BATCH>(f, rc.kc, rec_in, i, ri,
            [&](uint32_t, const uint4& rj, float3 d, float g) {
                const float sp = g * rec_x_mp(rj);
                sx += sp * d.x;
                sy += sp * d.y;
                sz += sp * d.z;
            });
        const float sm = m0 * rec_gscale<KIND>(rc.kc);
        const float ax = -r0i * fmaf(pi, gt.x, sm * sx), ay = -r0i * fmaf(pi, gt.y, sm * sy),
                    az = -r0i * fmaf(pi, gt.z, sm * sz);
        acc.x[i] = ax;
        acc.y[i] = ay;
        acc.z[i] = az;
        const float4 v = vel[i];
        const float nvx = v.x + dt * ax, nvy = v.y + dt * ay, nvz = v.z + dt * az;
        vn = store_state<BATCH>(tail, i, me.x + dt * nvx, me.y + dt * nvy, me.z + dt * nvz,
            nvx, nvy, nvz, x, y, z, vx, vy, vz);
    }
    tail_reduce(tail, vn);
}
