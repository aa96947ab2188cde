// Test infrastructure only: a C-ABI driver around the reference's OWN CUDA
// code (reyn, src/), compiled unmodified for sm_100a by oracle/ref/Makefile.
// It exists to pin the CPU oracle and the engine against the reference's real
// outputs (golden fixtures under tests/golden/). Nothing in the product links
// it. All arrays crossing this ABI are HOST arrays; the driver copies them to
// the device, runs the reference's own builder/solver/kernels, copies back.
//
// The orchestration below mirrors the reference's main loop (main.cu:60-78):
//   dt -> Scene::get_grid (scene.cuh:149-156: construct_and_reorder at 2h)
//      -> Solver::step -> Scene::hard_enforce_bounds (scene.cu:485-491)
// Scene itself cannot be built without an OBJ file, so the two one-line
// Scene members are replayed here with the reference's own builder and its
// own `_hard_enforce_bounds` kernel.

#include "common.h"
#include "kernels.cuh"
#include "particles.cuh"
#include "buffer.cuh"
#include "datastructure/uniformgrid.cuh"
#include "scene/scene.cuh"
#include "scene/sample_boundary.cuh"
#include "solvers/SESPH.cuh"
#include "solvers/PCISPH.cuh"
#include "solvers/IISPH.cuh"
#include "timestep/cfl.cuh"
#include "scene/ply_io.cuh"
#include "datastructure/lbvh.cuh"

#include <thrust/copy.h>
#include <thrust/host_vector.h>
#include <cstring>
#include <string>
#include <vector>

// defined in the reference's scene.cu:466, not declared in any header
__global__ void _hard_enforce_bounds(const float3 bound_min,
    const float3 bound_max, uint N, float* __restrict__ xx,
    float* __restrict__ xy, float* __restrict__ xz, float* __restrict__ vx,
    float* __restrict__ vy, float* __restrict__ vz);

namespace {

std::string g_err;

void to_dev(DeviceBuffer<float>& d, const float* h, size_t n)
{
    d.resize(n);
    if (n)
        thrust::copy(h, h + n, d.get().begin());
}

void to_host(const DeviceBuffer<float>& d, float* h, size_t n)
{
    if (h && n)
        thrust::copy(d.get().begin(), d.get().begin() + n, h);
}

template <typename F> int guarded(F&& f)
{
    try {
        f();
        CUDA_CHECK(cudaDeviceSynchronize());
        return 0;
    } catch (std::exception const& e) {
        g_err = e.what();
        return -1;
    }
}

// neighbour counting exactly as the reference's own grid test kernel
// (uniformgrid.cu:185-207), through the reference's `ff_nbrs`
template <Resort R>
__global__ void _drv_count(const uint N, const float* __restrict__ xx,
    const float* __restrict__ xy, const float* __restrict__ xz,
    uint* __restrict__ count_out, float* __restrict__ len2_out,
    const UniformGrid<R> grid, const float r_c_2)
{
    auto i { blockIdx.x * blockDim.x + threadIdx.x };
    if (i >= N)
        return;
    const float3 x_i { v3(i, xx, xy, xz) };
    count_out[i] = grid.ff_nbrs(x_i, xx, xy, xz,
        [r_c_2, i] __device__(auto j, auto x_ij, auto x_ij_l2) {
            return (x_ij_l2 <= r_c_2) ? (i == j ? 0u : 1u) : 0u;
        });
    len2_out[i] = grid.ff_nbrs(x_i, xx, xy, xz,
        [r_c_2, i] __device__(auto j, auto x_ij, auto x_ij_l2) {
            return (x_ij_l2 <= r_c_2) ? dot(x_ij, x_ij) : 0.f;
        });
}

// fluid-fluid density exactly as compute_densities (solver.cuh:31-33)
template <IsKernel K, Resort R>
__global__ void _drv_density(const uint N, const float* __restrict__ xx,
    const float* __restrict__ xy, const float* __restrict__ xz,
    const float* __restrict__ m, float* __restrict__ rho, const K W,
    const UniformGrid<R> grid)
{
    auto i { blockIdx.x * blockDim.x + threadIdx.x };
    if (i >= N)
        return;
    const float3 x_i { v3(i, xx, xy, xz) };
    rho[i] = grid.ff_nbrs(x_i, xx, xy, xz,
        [=] __device__(auto j, auto x_ij, auto x_ij_l2) {
            return m[j] * W(x_ij);
        });
}

// the reference grid benchmark's query kernel (uniformgrid.cu:231-245)
template <IsKernel K, Resort R>
__global__ void _drv_query(const uint N, const float* __restrict__ xx,
    const float* __restrict__ xy, const float* __restrict__ xz,
    float* __restrict__ res_out, const UniformGrid<R> grid, const K W)
{
    auto i { blockIdx.x * blockDim.x + threadIdx.x };
    if (i >= N)
        return;
    const float3 x_i { v3(i, xx, xy, xz) };
    res_out[i] = grid.ff_nbrs(
        x_i, xx, xy, xz, [=] __device__(auto j, auto x_ij, auto x_ij_l2) {
            return xx[i] * xx[j] * W(x_ij);
        });
}

template <IsKernel K>
__global__ void _drv_kernel_eval(const uint N, const float* __restrict__ dx,
    const float* __restrict__ dy, const float* __restrict__ dz,
    float* __restrict__ w, float* __restrict__ gx, float* __restrict__ gy,
    float* __restrict__ gz, const K W)
{
    auto i { blockIdx.x * blockDim.x + threadIdx.x };
    if (i >= N)
        return;
    const float3 d { v3(dx[i], dy[i], dz[i]) };
    w[i] = W(d);
    const float3 g { W.nabla(d) };
    gx[i] = g.x;
    gy[i] = g.y;
    gz[i] = g.z;
}

template <typename F> void with_kernel(int kind, float h_bar, F&& f)
{
    switch (kind) {
    case 0:
        f(C2(h_bar));
        break;
    case 1:
        f(B3(h_bar));
        break;
    case 2:
        f(W6(h_bar));
        break;
    case 3:
        f(COS(h_bar));
        break;
    default:
        throw std::runtime_error("unknown kernel id");
    }
}

// Build the boundary exactly as sample_mesh does after sampling
// (sample_boundary.cu:413-436): bounds from the samples, a grid at 2h,
// construct_and_reorder of xs,ys,zs (+ masses when given), then optionally
// the reference's Akinci mass refinement.
BoundarySamples make_boundary(uint Nb, const float* bx, const float* by,
    const float* bz, const float* bm, float h, float rho0, uint mass_iters,
    DeviceBuffer<float>& tmp)
{
    DeviceBuffer<float> xs(1), ys(1), zs(1), m(1);
    to_dev(xs, bx, Nb);
    to_dev(ys, by, Nb);
    to_dev(zs, bz, Nb);
    DeviceBuffer<uint> prefix(1);
    const float3 bmin { v3(xs.min(), ys.min(), zs.min()) };
    const float3 bmax { v3(xs.max(), ys.max(), zs.max()) };
    UniformGridBuilder builder(bmin, bmax, 2.f * h);
    if (bm) {
        to_dev(m, bm, Nb);
        UniformGrid<Resort::yes> grid { builder.construct_and_reorder(
            2.f * h, tmp, prefix, xs, ys, zs, &m) };
        return BoundarySamples { std::move(xs), std::move(ys), std::move(zs),
            std::move(m), std::move(prefix), grid, bmin, bmax };
    }
    m.resize(Nb);
    UniformGrid<Resort::yes> grid { builder.construct_and_reorder(
        2.f * h, m, prefix, xs, ys, zs) };
    m.resize(Nb);
    BoundarySamples res { std::move(xs), std::move(ys), std::move(zs),
        std::move(m), std::move(prefix), grid, bmin, bmax };
    calculate_boundary_masses(res, h, h, rho0, mass_iters);
    return res;
}

} // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

/// Reference kernel function evaluated on the DEVICE (norm3df, __saturatef).
int ref_kernel_eval_device(int kind, float h_bar, uint n, const float* dx,
    const float* dy, const float* dz, float* w, float* gx, float* gy,
    float* gz)
{
    return guarded([&] {
        DeviceBuffer<float> ddx(1), ddy(1), ddz(1), dw(n), dgx(n), dgy(n),
            dgz(n);
        to_dev(ddx, dx, n);
        to_dev(ddy, dy, n);
        to_dev(ddz, dz, n);
        with_kernel(kind, h_bar, [&](auto W) {
            _drv_kernel_eval<<<BLOCKS(n), BLOCK_SIZE>>>(n, ddx.ptr(),
                ddy.ptr(), ddz.ptr(), dw.ptr(), dgx.ptr(), dgy.ptr(),
                dgz.ptr(), W);
            CUDA_CHECK(cudaGetLastError());
        });
        to_host(dw, w, n);
        to_host(dgx, gx, n);
        to_host(dgy, gy, n);
        to_host(dgz, gz, n);
    });
}

/// UniformGridBuilder(bmin,bmax,r).construct(r, x) (uniformgrid.cu:65-156)
/// followed by the grid test's neighbour count and Σ|x_ij|² (self excluded
/// from the count) and, when m != NULL, the fluid density Σ m_j W(x_ij) with
/// kernel `kind` at support r. `dims` receives nx, ny, nz; `prefix` must
/// hold nx*ny*nz entries (query dims first with prefix == NULL).
int ref_grid(uint N, const float* x, const float* y, const float* z,
    const float* bmin, const float* bmax, float r, int* dims, uint* prefix,
    uint* sorted, uint* count, float* len2, int kind, const float* m,
    float* rho)
{
    return guarded([&] {
        const float3 lo { v3(bmin[0], bmin[1], bmin[2]) };
        const float3 hi { v3(bmax[0], bmax[1], bmax[2]) };
        // geometry exactly as the builder's initializer list computes it
        const float cell { r / 2.f };
        const float3 lo_m { lo - v3(r * 2.) };
        const int3 n3 { ceil_div((hi + v3(r * 2.)) - lo_m, r / 2.f) };
        dims[0] = n3.x;
        dims[1] = n3.y;
        dims[2] = n3.z;
        (void)cell;
        if (!prefix)
            return;
        DeviceBuffer<float> xx(1), xy(1), xz(1), dm(1);
        to_dev(xx, x, N);
        to_dev(xy, y, N);
        to_dev(xz, z, N);
        UniformGridBuilder builder(lo, hi, r);
        const UniformGrid<Resort::no> grid { builder.construct(r, xx, xy, xz) };
        const size_t C { size_t(n3.x) * n3.y * n3.z };
        CUDA_CHECK(cudaMemcpy(prefix, grid.prefix, C * sizeof(uint),
            cudaMemcpyDeviceToHost));
        CUDA_CHECK(cudaMemcpy(sorted, grid.sorted, N * sizeof(uint),
            cudaMemcpyDeviceToHost));
        DeviceBuffer<uint> dcount(N, 0);
        DeviceBuffer<float> dlen2(N, 0.f);
        _drv_count<<<BLOCKS(N), BLOCK_SIZE>>>(N, xx.ptr(), xy.ptr(), xz.ptr(),
            dcount.ptr(), dlen2.ptr(), grid, r * r);
        CUDA_CHECK(cudaGetLastError());
        thrust::copy(dcount.get().begin(), dcount.get().end(), count);
        to_host(dlen2, len2, N);
        if (m && rho) {
            to_dev(dm, m, N);
            DeviceBuffer<float> drho(N, 0.f);
            with_kernel(kind, r, [&](auto W) {
                _drv_density<<<BLOCKS(N), BLOCK_SIZE>>>(N, xx.ptr(), xy.ptr(),
                    xz.ptr(), dm.ptr(), drho.ptr(), W, grid);
                CUDA_CHECK(cudaGetLastError());
            });
            to_host(drho, rho, N);
        }
    });
}

/// The reference boundary pipeline: grid at 2h over the samples, reorder,
/// Akinci masses by calculate_boundary_masses (sample_boundary.cu:267-297).
/// Outputs the reordered samples and their masses.
int ref_boundary_masses(uint Nb, const float* bx, const float* by,
    const float* bz, float h, float rho0, uint iters, float* ox, float* oy,
    float* oz, float* om)
{
    return guarded([&] {
        DeviceBuffer<float> tmp(1);
        BoundarySamples b { make_boundary(
            Nb, bx, by, bz, nullptr, h, rho0, iters, tmp) };
        to_host(b.xs, ox, Nb);
        to_host(b.ys, oy, Nb);
        to_host(b.zs, oz, Nb);
        to_host(b.m, om, Nb);
    });
}

/// cfl_time_step (cfl.cu:5-37) on the given velocities.
int ref_cfl(uint N, const float* vx, const float* vy, const float* vz,
    float lambda, float h, const float* g, float* dt_out)
{
    return guarded([&] {
        Particles state(N, 1.f);
        to_dev(state.vx, vx, N);
        to_dev(state.vy, vy, N);
        to_dev(state.vz, vz, N);
        *dt_out = cfl_time_step(lambda, h, state, v3(g[0], g[1], g[2]));
    });
}

/// save_to_ply (ply_io.cu:7-55) on the given positions.
int ref_save_ply(uint N, const float* x, const float* y, const float* z, const char* path)
{
    return guarded([&] {
        DeviceBuffer<float> xs(N), ys(N), zs(N);
        to_dev(xs, x, N);
        to_dev(ys, y, N);
        to_dev(zs, z, N);
        save_to_ply(path, xs, ys, zs);
    });
}

/// Runs `steps` iterations of the reference main loop with solver `scheme`
/// (0 SESPH, 1 PCISPH, 2 IISPH) and kernel `kind` at support 2h.
/// state: x,y,z,vx,vy,vz,m,id are N-arrays, updated in place (in the order
///   the reference leaves them; `id` is carried as an extra reorder buffer).
/// bdy: Nb samples with masses (used as given, reordered by the boundary grid).
/// scene_min/max: the Scene bounds used by hard_enforce_bounds and the fluid
///   grid builder. dt_fixed > 0 uses a fixed dt; otherwise the reference's
///   cfl_time_step(lambda=-dt_fixed...) is not used and dt must be > 0.
/// Per-particle solver buffers after the last step are written to rho, p,
/// aii, sii, ax, ay, az (any may be NULL); iters[k] = iterations of step k.
int ref_run(int scheme, int kind, uint N, float* x, float* y, float* z,
    float* vx, float* vy, float* vz, float* m, float* id, uint Nb,
    const float* bx, const float* by, const float* bz, const float* bm,
    const float* scene_min, const float* scene_max, float h, float rho0,
    float nu, float dt, uint steps, float* rho, float* p, float* aii,
    float* sii, float* ax, float* ay, float* az, uint* iters)
{
    return guarded([&] {
        DeviceBuffer<float> tmp(1);
        BoundarySamples bdy { make_boundary(
            Nb, bx, by, bz, bm, h, rho0, 1, tmp) };
        Particles state(N, rho0);
        to_dev(state.xx, x, N);
        to_dev(state.xy, y, N);
        to_dev(state.xz, z, N);
        to_dev(state.vx, vx, N);
        to_dev(state.vy, vy, N);
        to_dev(state.vz, vz, N);
        to_dev(state.m, m, N);
        DeviceBuffer<float> did(1), tmp1(1), b_rho(1), b_p(1), b_aii(1),
            b_sii(1), b_ax(1), b_ay(1), b_az(1);
        DeviceBuffer<uint32_t> b_bits(1);
        to_dev(did, id, N);
        const float3 smin { v3(scene_min[0], scene_min[1], scene_min[2]) };
        const float3 smax { v3(scene_max[0], scene_max[1], scene_max[2]) };
        UniformGridBuilder builder(smin, smax, 2.f * h);

        with_kernel(kind, 2.f * h, [&](auto W) {
            using K = decltype(W);
            auto bounds = [&] {
                _hard_enforce_bounds<<<BLOCKS(N), BLOCK_SIZE>>>(smin, smax, N,
                    state.xx.ptr(), state.xy.ptr(), state.xz.ptr(),
                    state.vx.ptr(), state.vy.ptr(), state.vz.ptr());
                CUDA_CHECK(cudaGetLastError());
            };
            if (scheme == 0) {
                SESPH<K, Resort::yes> solver(
                    W, N, nu, h, rho0, b_rho, b_ax, b_ay, b_az);
                for (uint s { 0 }; s < steps; ++s) {
                    const auto grid { builder.construct_and_reorder(
                        2.f * h, tmp1, state, &did) };
                    solver.step(state, grid, bdy, dt);
                    bounds();
                    iters[s] = 1;
                }
            } else if (scheme == 1) {
                PCISPH<K, Resort::yes> solver(
                    W, N, nu, h, rho0, b_rho, b_ax, b_ay, b_az);
                for (uint s { 0 }; s < steps; ++s) {
                    const auto grid { builder.construct_and_reorder(
                        2.f * h, tmp1, state, &did) };
                    iters[s] = solver.step(state, grid, bdy, dt);
                    bounds();
                }
            } else if (scheme == 2) {
                IISPH<K, Resort::yes> solver(W, N, nu, h, rho0, b_rho, b_aii,
                    b_sii, b_ax, b_ay, b_az, b_p, b_bits);
                for (uint s { 0 }; s < steps; ++s) {
                    const auto grid { builder.construct_and_reorder(
                        2.f * h, tmp1, state, &did, &b_p) };
                    iters[s] = solver.step(state, grid, bdy, dt);
                    bounds();
                }
            } else {
                throw std::runtime_error("unknown scheme id");
            }
        });
        CUDA_CHECK(cudaDeviceSynchronize());
        to_host(state.xx, x, N);
        to_host(state.xy, y, N);
        to_host(state.xz, z, N);
        to_host(state.vx, vx, N);
        to_host(state.vy, vy, N);
        to_host(state.vz, vz, N);
        to_host(state.m, m, N);
        to_host(did, id, N);
        if (b_rho.size() >= N)
            to_host(b_rho, rho, N);
        if (b_p.size() >= N)
            to_host(b_p, p, N);
        if (b_aii.size() >= N)
            to_host(b_aii, aii, N);
        if (b_sii.size() >= N)
            to_host(b_sii, sii, N);
        if (b_ax.size() >= N) {
            to_host(b_ax, ax, N);
            to_host(b_ay, ay, N);
            to_host(b_az, az, N);
        }
    });
}

/// Timing of the reference's own grid benchmark (uniformgrid.cu:385-423) on
/// the given points: `reps` x construct_and_reorder of x, y, z plus 4 extra
/// arrays, and `reps` x the query kernel Σ x_i x_j W_B3(x_ij) at support r.
/// Device time by CUDA events; ms_out[0] = construction, ms_out[1] = query
/// (averages per repetition).
int ref_grid_bench(uint N, const float* x, const float* y, const float* z,
    const float* bmin, const float* bmax, float r, uint reps, float* ms_out)
{
    return guarded([&] {
        DeviceBuffer<float> xx(1), xy(1), xz(1), tmp(1), e1(1), out(N, 0.f);
        to_dev(xx, x, N);
        to_dev(xy, y, N);
        to_dev(xz, z, N);
        e1.resize(N);
        tmp.resize(N);
        UniformGridBuilder builder(v3(bmin[0], bmin[1], bmin[2]), v3(bmax[0], bmax[1], bmax[2]), r);
        cudaEvent_t a, b;
        CUDA_CHECK(cudaEventCreate(&a));
        CUDA_CHECK(cudaEventCreate(&b));
        for (uint k = 0; k < 2; ++k) // warm-up
            builder.construct_and_reorder(r, tmp, xx, xy, xz, &e1, &e1, &e1, &e1);
        CUDA_CHECK(cudaEventRecord(a));
        for (uint k = 0; k < reps; ++k)
            builder.construct_and_reorder(r, tmp, xx, xy, xz, &e1, &e1, &e1, &e1);
        CUDA_CHECK(cudaEventRecord(b));
        CUDA_CHECK(cudaEventSynchronize(b));
        float t = 0.f;
        CUDA_CHECK(cudaEventElapsedTime(&t, a, b));
        ms_out[0] = t / reps;
        const UniformGrid<Resort::yes> grid { builder.construct_and_reorder(
            r, tmp, xx, xy, xz) };
        const B3 W(r);
        _drv_query<<<BLOCKS(N), BLOCK_SIZE>>>(N, xx.ptr(), xy.ptr(), xz.ptr(), out.ptr(), grid, W);
        CUDA_CHECK(cudaEventRecord(a));
        for (uint k = 0; k < reps; ++k)
            _drv_query<<<BLOCKS(N), BLOCK_SIZE>>>(N, xx.ptr(), xy.ptr(), xz.ptr(), out.ptr(),
                grid, W);
        CUDA_CHECK(cudaEventRecord(b));
        CUDA_CHECK(cudaEventSynchronize(b));
        CUDA_CHECK(cudaEventElapsedTime(&t, a, b));
        ms_out[1] = t / reps;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    });
}

/// ref_run with device timing of the step loop: ms_out = average device time
/// per main-loop step (grid build + reorder, solver step, bounds), CUDA events
/// around the loop (the reference's host syncs inside the solvers included).
int ref_run_timed(int scheme, int kind, uint N, float* x, float* y, float* z,
    float* vx, float* vy, float* vz, float* m, float* id, uint Nb,
    const float* bx, const float* by, const float* bz, const float* bm,
    const float* scene_min, const float* scene_max, float h, float rho0,
    float nu, float dt, uint steps, uint* iters, float* ms_out)
{
    return guarded([&] {
        DeviceBuffer<float> tmp(1);
        BoundarySamples bdy { make_boundary(
            Nb, bx, by, bz, bm, h, rho0, 1, tmp) };
        Particles state(N, rho0);
        to_dev(state.xx, x, N);
        to_dev(state.xy, y, N);
        to_dev(state.xz, z, N);
        to_dev(state.vx, vx, N);
        to_dev(state.vy, vy, N);
        to_dev(state.vz, vz, N);
        to_dev(state.m, m, N);
        DeviceBuffer<float> tmp1(1), b_rho(1), b_p(1), b_aii(1), b_sii(1), b_ax(1), b_ay(1),
            b_az(1);
        DeviceBuffer<uint32_t> b_bits(1);
        const float3 smin { v3(scene_min[0], scene_min[1], scene_min[2]) };
        const float3 smax { v3(scene_max[0], scene_max[1], scene_max[2]) };
        UniformGridBuilder builder(smin, smax, 2.f * h);
        cudaEvent_t a, b;
        CUDA_CHECK(cudaEventCreate(&a));
        CUDA_CHECK(cudaEventCreate(&b));
        with_kernel(kind, 2.f * h, [&](auto W) {
            using K = decltype(W);
            auto bounds = [&] {
                _hard_enforce_bounds<<<BLOCKS(N), BLOCK_SIZE>>>(smin, smax, N,
                    state.xx.ptr(), state.xy.ptr(), state.xz.ptr(),
                    state.vx.ptr(), state.vy.ptr(), state.vz.ptr());
                CUDA_CHECK(cudaGetLastError());
            };
            if (scheme != 2)
                throw std::runtime_error("ref_run_timed times IISPH only");
            IISPH<K, Resort::yes> solver(W, N, nu, h, rho0, b_rho, b_aii, b_sii, b_ax, b_ay,
                b_az, b_p, b_bits);
            CUDA_CHECK(cudaEventRecord(a));
            for (uint s { 0 }; s < steps; ++s) {
                const auto grid { builder.construct_and_reorder(2.f * h, tmp1, state, &b_p) };
                iters[s] = solver.step(state, grid, bdy, dt);
                bounds();
            }
            CUDA_CHECK(cudaEventRecord(b));
            CUDA_CHECK(cudaEventSynchronize(b));
            float t = 0.f;
            CUDA_CHECK(cudaEventElapsedTime(&t, a, b));
            *ms_out = t / (float)steps;
        });
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        to_host(state.xx, x, N);
        to_host(state.xy, y, N);
        to_host(state.xz, z, N);
        to_host(state.vx, vx, N);
        to_host(state.vy, vy, N);
        to_host(state.vz, vz, N);
    });
}

} // extern "C"

namespace {

Mesh host_mesh(uint nv, const double* vx, const double* vy, const double* vz, uint nf,
    const uint* faces)
{
    Mesh m;
    m.xs.assign(vx, vx + nv);
    m.ys.assign(vy, vy + nv);
    m.zs.assign(vz, vz + nv);
    m.faces.resize(nf);
    for (uint t = 0; t < nf; ++t)
        m.faces[t] = make_uint3(faces[3 * t], faces[3 * t + 1], faces[3 * t + 2]);
    return m;
}

void put_boxes(const thrust::host_vector<AABB>& b, float* out)
{
    for (size_t i = 0; out && i < b.size(); ++i) {
        const float v[6] = { b[i].mini.x, b[i].mini.y, b[i].mini.z, b[i].maxi.x, b[i].maxi.y,
            b[i].maxi.z };
        std::memcpy(out + 6 * i, v, sizeof(v));
    }
}

} // namespace

extern "C" {

/// DeviceMesh::get_volume (sample_boundary.cuh:40-60) and LBVH(&mesh)
/// (lbvh.cuh:646-723) over a host mesh: the faces as the constructor leaves
/// them (sorted by Morton code), the children in the ChildNode encoding, the
/// leaf and internal boxes (min xyz, max xyz) and the tree height; then
/// LBVH::project (lbvh.cuh:726-741) of n host points, in place.
int ref_lbvh(uint nv, const double* vx, const double* vy, const double* vz, uint nf,
    const uint* faces, uint* faces_sorted, uint* children_l, uint* children_r, float* leaf_box,
    float* node_box, uint* height, double* volume, uint n, float* x, float* y, float* z)
{
    return guarded([&] {
        DeviceMesh dm { DeviceMesh::from(host_mesh(nv, vx, vy, vz, nf, faces)) };
        if (volume)
            *volume = dm.get_volume();
        const LBVH lbvh(&dm);
        const thrust::host_vector<uint3> fs = dm.faces.get();
        for (uint t = 0; faces_sorted && t < nf; ++t) {
            faces_sorted[3 * t] = fs[t].x;
            faces_sorted[3 * t + 1] = fs[t].y;
            faces_sorted[3 * t + 2] = fs[t].z;
        }
        const thrust::host_vector<ChildNode> cl = lbvh.children_l.get();
        const thrust::host_vector<ChildNode> cr = lbvh.children_r.get();
        for (size_t i = 0; i < cl.size(); ++i) {
            if (children_l)
                children_l[i] = cl[i].__i;
            if (children_r)
                children_r[i] = cr[i].__i;
        }
        put_boxes(lbvh.aabbs_leaf.get(), leaf_box);
        put_boxes(lbvh.aabbs_internal.get(), node_box);
        if (height)
            *height = lbvh.get_pod().tree_height;
        if (n) {
            DeviceBuffer<float> xs(1), ys(1), zs(1);
            to_dev(xs, x, n);
            to_dev(ys, y, n);
            to_dev(zs, z, n);
            lbvh.project(xs, ys, zs);
            to_host(xs, x, n);
            to_host(ys, y, n);
            to_host(zs, z, n);
        }
    });
}

/// uniform_sample_mesh (sample_boundary.cu:299-389): *count samples (curand
/// Philox, the reference's seed), written when cap allows
int ref_mesh_sample(uint nv, const double* vx, const double* vy, const double* vz, uint nf,
    const uint* faces, float h, float oversampling, uint cap, float* x, float* y, float* z,
    uint* count)
{
    return guarded([&] {
        DeviceMesh dm { DeviceMesh::from(host_mesh(nv, vx, vy, vz, nf, faces)) };
        DeviceBuffer<float> xs(1), ys(1), zs(1);
        uniform_sample_mesh(xs, ys, zs, dm, h, oversampling);
        const uint n = static_cast<uint>(xs.size());
        *count = n;
        if (x && cap >= n) {
            to_host(xs, x, n);
            to_host(ys, y, n);
            to_host(zs, z, n);
        }
    });
}

} // extern "C"

extern "C" {

/// Timing of the reference's mesh path on the device (CUDA events): the
/// LBVH constructor (lbvh.cuh:646-723) once, then `reps` times a device copy
/// of the n pristine points followed by LBVH::project (lbvh.cuh:726-741);
/// and sample_mesh (sample_boundary.cu:391-439) at h, oversampling 2,
/// relax_iters sweeps, 5 mass refinements (best of two runs). ms[0] =
/// build, ms[1] = per copy + project, ms[2] = sample_mesh, ms[3] = upload
/// (DeviceMesh::from) + build, counts[0] = samples.
int ref_mesh_bench(uint nv, const double* vx, const double* vy, const double* vz, uint nf,
    const uint* faces, uint n, const float* x, const float* y, const float* z, uint reps,
    float h, int relax_iters, float* ms, uint* counts)
{
    return guarded([&] {
        cudaEvent_t e0, e1;
        CUDA_CHECK(cudaEventCreate(&e0));
        CUDA_CHECK(cudaEventCreate(&e1));
        const Mesh hm = host_mesh(nv, vx, vy, vz, nf, faces);
        {
            // untimed first construction: module loading, allocator warm-up
            DeviceMesh warm { DeviceMesh::from(hm) };
            const LBVH lw(&warm);
        }
        {
            CUDA_CHECK(cudaDeviceSynchronize());
            CUDA_CHECK(cudaEventRecord(e0));
            DeviceMesh up { DeviceMesh::from(hm) };
            const LBVH lu(&up);
            CUDA_CHECK(cudaEventRecord(e1));
            CUDA_CHECK(cudaEventSynchronize(e1));
            CUDA_CHECK(cudaEventElapsedTime(&ms[3], e0, e1));
        }
        DeviceMesh dm { DeviceMesh::from(hm) };
        CUDA_CHECK(cudaDeviceSynchronize());
        CUDA_CHECK(cudaEventRecord(e0));
        const LBVH lbvh(&dm);
        CUDA_CHECK(cudaEventRecord(e1));
        CUDA_CHECK(cudaEventSynchronize(e1));
        CUDA_CHECK(cudaEventElapsedTime(&ms[0], e0, e1));
        DeviceBuffer<float> px(1), py(1), pz(1), wx(n), wy(n), wz(n);
        to_dev(px, x, n);
        to_dev(py, y, n);
        to_dev(pz, z, n);
        auto once = [&] {
            thrust::copy(px.get().begin(), px.get().end(), wx.get().begin());
            thrust::copy(py.get().begin(), py.get().end(), wy.get().begin());
            thrust::copy(pz.get().begin(), pz.get().end(), wz.get().begin());
            lbvh.project(wx, wy, wz);
        };
        once(); // warm-up
        CUDA_CHECK(cudaDeviceSynchronize());
        CUDA_CHECK(cudaEventRecord(e0));
        for (uint r = 0; r < reps; ++r)
            once();
        CUDA_CHECK(cudaEventRecord(e1));
        CUDA_CHECK(cudaEventSynchronize(e1));
        CUDA_CHECK(cudaEventElapsedTime(&ms[1], e0, e1));
        ms[1] /= float(reps > 0 ? reps : 1);
        ms[2] = 1e30f;
        for (int run = 0; run < 2; ++run) {
            CUDA_CHECK(cudaDeviceSynchronize());
            CUDA_CHECK(cudaEventRecord(e0));
            BoundarySamples b { sample_mesh(hm, h, 1000.f, 2.f, nullptr, relax_iters, 1.f, 5) };
            CUDA_CHECK(cudaEventRecord(e1));
            CUDA_CHECK(cudaEventSynchronize(e1));
            float t = 0.f;
            CUDA_CHECK(cudaEventElapsedTime(&t, e0, e1));
            ms[2] = std::min(ms[2], t);
            counts[0] = static_cast<uint>(b.xs.size());
        }
        CUDA_CHECK(cudaEventDestroy(e0));
        CUDA_CHECK(cudaEventDestroy(e1));
    });
}

} // extern "C"
