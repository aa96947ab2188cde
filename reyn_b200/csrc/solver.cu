// SESPH / PCISPH / IISPH steps on the B200: the 128-thread instantiation of
// the step and its non-template parts (the passes are in passes.cuh). Each
// pass is one fixed-radius neighbour kernel over the packed (x, y, z, m) copy
// in grid order; work the
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
#include "passes.cuh"

namespace reyn {

// k_c_pcisph (PCISPH.cuh:49-77): host evaluation of grad W on a 5^3 lattice
// template particle at spacing h, support 2h; returns delta*dt^2 (rounded to
// float, as the reference's return type does)
double pcisph_template_delta(int kind, float h)
{
    const KernelConst kc = make_kernel(kind, 2.f * h);
    auto dw = [&](float q) {
        switch (kind) {
        case K_C2: return Shape<K_C2>::dw(q);
        case K_B3: return Shape<K_B3>::dw(q);
        case K_W6: return Shape<K_W6>::dw(q);
        default: return Shape<K_COS>::dw(q);
        }
    };
    const double hd = h;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    double sum_of_sq = 0.0;
    for (int a = -2; a <= 2; ++a)
        for (int b = -2; b <= 2; ++b)
            for (int c = -2; c <= 2; ++c) {
                const float x = -((float)a * h), y = -((float)b * h), z = -((float)c * h);
                const float l2 = std::fmaf(x, x, std::fmaf(y, y, z * z));
                const float len = (float)std::sqrt((double)l2);
                const float sc = kc.dw_scale * dw(len * kc.h_inv) * (1.f / len);
                const float s = std::isfinite(sc) ? sc : 0.f;
                const float gx = x * s, gy = y * s, gz = z * s;
                sx += gx;
                sy += gy;
                sz += gz;
                sum_of_sq += (double)std::fmaf(gx, gx, std::fmaf(gy, gy, gz * gz));
            }
    const double sq_of_sum = (double)std::fmaf(sx, sx, std::fmaf(sy, sy, sz * sz));
    const double V0 = hd * hd * hd;
    const double beta = 2. * V0 * V0;
    return (double)(float)(1. / (beta * (sq_of_sum + sum_of_sq)));
}

void ensure_buffers(reyn_solver& sv, uint32_t n)
{
    sv.rho.resize(n);
    sv.aii.resize(n);
    sv.sii.resize(n);
    sv.ax.resize(n);
    sv.ay.resize(n);
    sv.az.resize(n);
    sv.acc.resize(n);
    sv.vel2.resize(n);
    sv.bterm.resize(n);
    sv.nbr.resize(list_capacity(n));
    sv.ncount.resize(n);
    if (sv.prm.precision == REYN_PRECISION_MIXED) {
        sv.acch.resize(n);
        sv.velh.resize(n);
        sv.velh2.resize(n);
    } else if (sv.prm.precision == REYN_PRECISION_MIXED_POS16) {
        sv.rec0.resize(n);
        sv.rec1.resize(n);
        sv.gq.resize(n);
    }
    if (sv.p.size() != n) {
        sv.p.resize(n);
        REYN_CUDA(cudaMemset(sv.p.get(), 0, size_t(n) * sizeof(float)));
    }
    sv.p_tmp.resize(n);
    constexpr size_t SLOTS = 64;
    if (sv.sweep_stats.size() == 0) {
        sv.sweep_stats.resize(SLOTS * sizeof(SweepStats));
        sv.readback = std::make_unique<PinnedArray<unsigned char>>(sizeof(SweepStats));
    }
}

// the step at the block size the parameters ask for: up to 128 threads here,
// larger blocks in solver_wide.cu
void solver_step_wide(reyn_solver& sv, reyn_particles& st, const Grid& grid,
    const reyn_boundary* bdy, float dt, cudaStream_t s, const float* bmin, const float* bmax);

void solver_step_sorted(reyn_solver& sv, reyn_particles& st, const Grid& grid,
    const reyn_boundary* bdy, float dt, cudaStream_t s, const float* bmin, const float* bmax)
{
    if (sv.prm.block_size > NBR_THREADS)
        solver_step_wide(sv, st, grid, bdy, dt, s, bmin, bmax);
    else
        solver_step_t<NBR_THREADS>(sv, st, grid, bdy, dt, s, bmin, bmax);
}

// dst[k][perm[s]] = src[k][s]: arrays in grid order back to the caller's order
__global__ void k_scatter_back(uint32_t n, const uint32_t* __restrict__ perm, GatherArgs a)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const uint32_t p = perm[s];
#pragma unroll
    for (int k = 0; k < MAX_GATHER; ++k)
        if (k < a.count)
            a.dst[k][p] = __ldg(a.src[k] + s);
}

// the grid's last build was construct over this state's current positions
// (the reference's UniformGrid<Resort::no>, uniformgrid.cuh:363-380)
bool built_unsorted(const Grid& g, const reyn_particles& st)
{
    return !g.reordered && g.n_scenes == 0 && g.n == st.n && g.built_pos[0] == st.cur[FX].get()
        && g.built_pos[1] == st.cur[FY].get() && g.built_pos[2] == st.cur[FZ].get();
}

// Solver::step with R = Resort::no (the solvers are instantiated for both,
// IISPH.cu:264-269): neighbours come through the grid's permutation while the
// particles keep the caller's order. The state is gathered into grid order in
// solver-owned arrays, stepped there by the passes of the sorted step, and
// positions, velocities and the solver's per-particle buffers are scattered
// back. Neighbour sums then run in the order the reference's Resort::no
// kernels visit them (cell by cell, each cell in the permutation's order).
// IISPH's carried pressure stays in the caller's order between steps.
void solver_step_unsorted(reyn_solver& sv, reyn_particles& st, const Grid& grid,
    const reyn_boundary* bdy, float dt, cudaStream_t s, const float* bmin, const float* bmax)
{
    const uint32_t n = st.n;
    require(n == sv.n, "particle count differs from the solver's");
    require(dt > 0.f && std::isfinite(dt), "dt must be positive and finite");
    require(!sv.graph, "a captured step reorders the state (construct_and_reorder)");
    ensure_buffers(sv, n);
    if (!sv.shadow)
        sv.shadow = std::make_unique<reyn_particles>();
    reyn_particles& sh = *sv.shadow;
    sh.n = n;
    sh.rho0 = st.rho0;
    for (auto& a : sh.cur)
        a.resize(n);
    sh.pm.resize(n);
    sh.vel.resize(n);
    const uint32_t* perm = grid.sorted.get();
    GatherArgs ga {};
    for (int k = 0; k < NFIELDS; ++k) {
        ga.src[k] = st.cur[k].get();
        ga.dst[k] = sh.cur[k].get();
    }
    ga.count = NFIELDS;
    ga.pm = sh.pm.get();
    ga.vel = sh.vel.get();
    launch_gather(n, perm, ga, s);
    sh.packed_valid = true;
    if (sv.scheme == REYN_IISPH) {
        if (sv.p_state == &st && sv.p_epoch == st.epoch) { // warm: p in the caller's order
            GatherArgs gp {};
            gp.src[0] = sv.p.get();
            gp.dst[0] = sv.p_tmp.get();
            gp.count = 1;
            launch_gather(n, perm, gp, s);
            sv.p.swap(sv.p_tmp);
        } else {
            sv.p.zero(s);
        }
        sv.p_state = &sh;
        sv.p_epoch = sh.epoch;
    }
    auto scatter = [&] {
        DevArray<float>* bufs[] = { &sv.rho, &sv.p, &sv.aii, &sv.sii, &sv.ax, &sv.ay, &sv.az };
        GatherArgs sa {};
        int k = 0;
        for (int f = FX; f <= FVZ; ++f, ++k) {
            sa.src[k] = sh.cur[f].get();
            sa.dst[k] = st.cur[f].get();
        }
        int nb = 0;
        for (DevArray<float>* b : bufs) {
            if (b->size() != n)
                continue;
            sv.shadow_out[nb].resize(n);
            sa.src[k] = b->get();
            sa.dst[k++] = sv.shadow_out[nb++].get();
        }
        sa.count = k;
        if (n)
            REYN_KERNEL("k_scatter_back", s,
                k_scatter_back<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, perm, sa));
        nb = 0;
        for (DevArray<float>* b : bufs)
            if (b->size() == n)
                b->swap(sv.shadow_out[nb++]);
        st.packed_valid = false;
        st.version += 1;
        if (sv.scheme == REYN_IISPH) {
            sv.p_state = &st;
            sv.p_epoch = st.epoch;
        }
        if (sv.vmax_state == &sh) {
            sv.vmax_state = &st;
            sv.vmax_version = st.version;
        }
    };
    try {
        solver_step_sorted(sv, sh, grid, bdy, dt, s, bmin, bmax);
    } catch (const Error& e) {
        if (e.code == REYN_ERR_ITER_LIMIT) // the step completed
            scatter();
        throw;
    }
    scatter();
}

void solver_step(reyn_solver& sv, reyn_particles& st, const Grid& grid,
    const reyn_boundary* bdy, float dt, cudaStream_t s, const float* bmin, const float* bmax)
{
    if (built_unsorted(grid, st) && &st != sv.shadow.get())
        solver_step_unsorted(sv, st, grid, bdy, dt, s, bmin, bmax);
    else
        solver_step_sorted(sv, st, grid, bdy, dt, s, bmin, bmax);
}

// ---- densities alone ------------------------------------------------------------

// compute_densities (solver.cuh:19-38): rho_i = sum_j m_j W_ij over the fluid
// neighbours within r (self included) + sum_b m_b W_ib over the boundary
// samples, per grid slot over packed points; `owner` maps a slot back to
// the caller's index on a grid built without reorder
template <int KIND, int R>
__global__ void __launch_bounds__(NBR_THREADS) k_compute_densities(uint32_t n, GridView g,
    KernelConst kc, const float4* __restrict__ pts, const uint32_t* __restrict__ owner, Bdy b,
    float* __restrict__ rho, uint32_t* __restrict__ status)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const float4 me = pts[s];
    int3 c = cell_of(g, me.x, me.y, me.z);
    if (!cell_inside(g, c, R) || !(isfinite(me.x) && isfinite(me.y) && isfinite(me.z))) {
        atomicOr(status, STATUS_OUT_OF_GRID);
        c = clamp_cell(g, c, R);
    }
    float rf = 0.f;
    for_each_neighbour<R>(g, c, me.x, me.y, me.z, pts,
        [&](uint32_t, const float4& q, float, float, float, float l2) {
            rf += q.w * pair_w<KIND>(kc, l2);
        });
    float rb = 0.f;
    for_each_boundary(b, me.x, me.y, me.z,
        [&](uint32_t, const float4& q, float, float, float, float l2) {
            rb += q.w * pair_w<KIND>(kc, l2);
        });
    rho[owner ? owner[s] : s] = rf + rb;
}

void compute_densities(const Grid& g, const float* x, const float* y, const float* z,
    const float* m, const reyn_boundary* bdy, int kind, float* rho, cudaStream_t s)
{
    require(g.n_scenes == 0, "batched grids: the batched solver step computes densities");
    const uint32_t n = g.n;
    Bdy b {};
    if (bdy && bdy->nb) {
        require(bdy->grid.n_scenes == 0, "batched boundaries need the batched solver step");
        require(bdy->grid.geom.r >= g.geom.r,
            "the boundary grid's radius is below the fluid grid's search radius");
        b.g = bdy->view();
        b.g.r2 = g.geom.r * g.geom.r;
        b.pm = bdy->pm.get();
        b.near = bdy->near.get();
        b.n = bdy->nb;
    }
    if (!n)
        return;
    DevArray<float4>& pts = g.pts_tmp;
    pts.resize(n);
    const uint32_t* order = g.reordered ? nullptr : g.sorted.get();
    pack_positions(n, order, x, y, z, m, pts.get(), s);
    const GridView v = g.view(g.geom.r);
    const KernelConst kc = make_kernel(kind, g.geom.r);
    const unsigned nb = blocks_for(n, NBR_THREADS);
    uint32_t* st = const_cast<uint32_t*>(g.status.get());
    auto go = [&](auto K) {
        constexpr int KIND = decltype(K)::value;
        if (g.geom.range == 2)
            k_compute_densities<KIND, 2><<<nb, NBR_THREADS, 0, s>>>(n, v, kc, pts.get(), order, b,
                rho, st);
        else
            k_compute_densities<KIND, 1><<<nb, NBR_THREADS, 0, s>>>(n, v, kc, pts.get(), order, b,
                rho, st);
    };
    ProfScope scope("k_compute_densities", s);
    switch (kind) {
    case K_C2: go(std::integral_constant<int, K_C2> {}); break;
    case K_B3: go(std::integral_constant<int, K_B3> {}); break;
    case K_W6: go(std::integral_constant<int, K_W6> {}); break;
    case K_COS: go(std::integral_constant<int, K_COS> {}); break;
    default: fail(REYN_ERR_INVALID, "unknown kernel");
    }
    REYN_LAUNCHED("k_compute_densities");
}

// ---- FP64 diagnostics ----------------------------------------------------------

// sum m, sum m v, sum m |v|^2 / 2 in FP64 (per-block FP64 partials, one
// atomic per block and quantity)
__global__ void k_diagnostics(uint32_t n, const float* __restrict__ vx,
    const float* __restrict__ vy, const float* __restrict__ vz, const float* __restrict__ m,
    double* __restrict__ out)
{
    double acc[5] = { 0.0, 0.0, 0.0, 0.0, 0.0 };
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += gridDim.x * blockDim.x) {
        const double mi = m[i], ux = vx[i], uy = vy[i], uz = vz[i];
        acc[0] += mi;
        acc[1] += mi * ux;
        acc[2] += mi * uy;
        acc[3] += mi * uz;
        acc[4] += 0.5 * mi * (ux * ux + uy * uy + uz * uz);
    }
    __shared__ double s_acc[5][THREADS / 32];
#pragma unroll
    for (int q = 0; q < 5; ++q) {
        const double v = warp_sum(acc[q]);
        if ((threadIdx.x & 31) == 0)
            s_acc[q][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 5) {
        double v = 0.0;
        for (int w = 0; w < THREADS / 32; ++w)
            v += s_acc[threadIdx.x][w];
        atomicAdd(out + threadIdx.x, v);
    }
}

void diagnostics(const reyn_particles& st, double out[5], cudaStream_t s)
{
    DevArray<double> d(5);
    REYN_CUDA(cudaMemsetAsync(d.get(), 0, 5 * sizeof(double), s));
    if (st.n) {
        REYN_KERNEL("k_diagnostics", s,
            k_diagnostics<<<std::min<unsigned>(blocks_for(st.n, THREADS), 148 * 8), THREADS, 0, s>>>(
            st.n, st.cur[FVX].get(), st.cur[FVY].get(), st.cur[FVZ].get(), st.cur[FM].get(),
            d.get()));
    }
    REYN_CUDA(cudaMemcpyAsync(out, d.get(), 5 * sizeof(double), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaStreamSynchronize(s));
}

// ---- time step and bounds ------------------------------------------------------

__global__ void k_vmax(uint32_t n, const float* __restrict__ vx, const float* __restrict__ vy,
    const float* __restrict__ vz, float* out)
{
    __shared__ float s_max[THREADS / 32];
    float v = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        v = fmaxf(v, norm3df(vx[i], vy[i], vz[i])); // cfl.cu:13-18
    v = warp_max(v);
    if ((threadIdx.x & 31) == 0)
        s_max[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < THREADS / 32; ++w)
            v = fmaxf(v, s_max[w]);
        atomic_max_nonneg(out, v);
    }
}

float state_vmax(reyn_solver* sv, reyn_particles& st, cudaStream_t s)
{
    if (sv && sv->vmax_valid && sv->vmax_state == &st && sv->vmax_version == st.version) {
        REYN_CUDA(cudaEventSynchronize(sv->vmax_ready));
        return *sv->vmax_host->get();
    }
    DevArray<float> d(1);
    d.zero(s);
    if (st.n) {
        REYN_KERNEL("k_vmax", s,
            k_vmax<<<std::min<unsigned>(blocks_for(st.n, THREADS), 148 * 8), THREADS, 0, s>>>(st.n, st.cur[FVX].get(),
            st.cur[FVY].get(), st.cur[FVZ].get(), d.get()));
    }
    float vmax = 0.f;
    REYN_CUDA(cudaMemcpyAsync(&vmax, d.get(), sizeof(float), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaStreamSynchronize(s));
    return vmax;
}

float cfl_time_step(reyn_particles& st, float lambda, float h, const float g[3], cudaStream_t s,
    reyn_solver* sv)
{
    const float vmax = state_vmax(sv, st, s);
    // cfl.cu:22-36
    const float dt_vel = lambda * h / vmax;
    const float gn = (float)std::sqrt((double)std::fmaf(g[0], g[0], std::fmaf(g[1], g[1], g[2] * g[2])));
    const float dt_g = std::sqrt((float)(2. * lambda * h / (double)gn));
    return std::fmin(dt_vel, dt_g);
}

// _hard_enforce_bounds (scene.cu:466-483)
__global__ void k_bounds_enforce(uint32_t n, float3 lo, float3 hi, float* __restrict__ x,
    float* __restrict__ y, float* __restrict__ z, float* __restrict__ vx,
    float* __restrict__ vy, float* __restrict__ vz)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float px = x[i], py = y[i], pz = z[i];
    if (px <= lo.x || py <= lo.y || pz <= lo.z || hi.x <= px || hi.y <= py || hi.z <= pz) {
        const float d = (float)-0.1;
        vx[i] = vx[i] * d;
        vy[i] = vy[i] * d;
        vz[i] = vz[i] * d;
    }
    x[i] = fmaxf(fminf(px, hi.x), lo.x);
    y[i] = fmaxf(fminf(py, hi.y), lo.y);
    z[i] = fmaxf(fminf(pz, hi.z), lo.z);
}

void enforce_bounds(reyn_particles& st, const float lo[3], const float hi[3], cudaStream_t s)
{
    if (!st.n)
        return;
    REYN_KERNEL("k_bounds_enforce", s,
        k_bounds_enforce<<<blocks_for(st.n, THREADS), THREADS, 0, s>>>(st.n,
        make_float3(lo[0], lo[1], lo[2]), make_float3(hi[0], hi[1], hi[2]), st.cur[FX].get(),
        st.cur[FY].get(), st.cur[FZ].get(), st.cur[FVX].get(), st.cur[FVY].get(),
        st.cur[FVZ].get()));
    st.packed_valid = false;
    st.version += 1;
}

} // namespace reyn
