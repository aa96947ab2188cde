// reyn_b200 C++ adapters: header-only wrappers over the C ABI (reyn_b200.h)
// that reproduce the reference's (reyn) C++ surface, so that a loop written
// against the reference —
//
//     Particles state(N, rho0);
//     UniformGridBuilder builder(bmin, bmax, 2.f * h);
//     IISPH<B3, Resort::yes> solver(W, N, nu, h, rho0);
//     dt = simple_dt_controller(iters, dt, 1.0, h, state, g, 10, 0.001f);
//     const auto grid { builder.construct_and_reorder(2.f * h, state) };
//     iters = solver.step(state, grid, bdy, dt);
//     hard_enforce_bounds(state, bmin, bmax);
//
// (main.cu:60-78) — compiles against this header with the reyn:: namespace.
// Differences from the reference, by design of the C ABI: the solvers own
// their per-particle buffers (the reference takes caller DeviceBuffers,
// SESPH.cuh:37-41 etc.), the IISPH pressure follows reorders automatically
// (main.cu:68 passes it as an extra buffer), errors are exceptions carrying
// the C status code instead of exit() (common.h:24-36), and every call takes
// an optional cudaStream_t.
#ifndef REYN_B200_HPP_
#define REYN_B200_HPP_

#include "reyn_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

namespace reyn {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg)
        : std::runtime_error("reyn_b200 error " + std::to_string(code) + ": " + msg)
        , code_(code)
    {
    }
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc)
{
    if (rc != REYN_OK)
        throw Error(rc, reyn_last_error());
}

// uniformgrid.cuh:70
enum class Resort : bool { no = false, yes = true };

// ---- smoothing kernels (kernels.cuh:78-165): tags carrying h_bar ----------
template <reyn_kernel KIND> struct KernelTag {
    static constexpr reyn_kernel kind = KIND;
    float h_bar;
    explicit KernelTag(float h) : h_bar(h) { }
};
using C2 = KernelTag<REYN_KERNEL_C2>;
using B3 = KernelTag<REYN_KERNEL_B3>;
using W6 = KernelTag<REYN_KERNEL_W6>;
using COS = KernelTag<REYN_KERNEL_COS>;

// ---- Particles (particles.cuh:25-75) ----------------------------------------
class Particles {
public:
    Particles(uint32_t n, float rho0) { check(reyn_particles_create(n, rho0, &h_)); }
    ~Particles() { reyn_particles_destroy(h_); }
    Particles(const Particles&) = delete;
    Particles& operator=(const Particles&) = delete;

    // SoA device pointers (DeviceBuffer::ptr()); they change after a reorder
    reyn_soa soa()
    {
        reyn_soa s {};
        check(reyn_particles_soa(h_, &s));
        return s;
    }
    uint32_t size() const { return n(); }
    void upload(const float* xx, const float* xy, const float* xz, const float* vx,
        const float* vy, const float* vz, const float* m, cudaStream_t s = nullptr)
    {
        check(reyn_particles_upload(h_, xx, xy, xz, vx, vy, vz, m, s));
        if (cudaStreamSynchronize(s) != cudaSuccess)
            throw Error(REYN_ERR_CUDA, "stream synchronisation after upload failed");
    }
    void download(float* xx, float* xy, float* xz, float* vx, float* vy, float* vz, float* m,
        cudaStream_t s = nullptr)
    {
        check(reyn_particles_download(h_, xx, xy, xz, vx, vy, vz, m, s));
    }
    // Particles::reorder (particles.cu:93-113): device permutation of n entries
    void reorder(const uint32_t* sorted, cudaStream_t s = nullptr)
    {
        check(reyn_particles_reorder(h_, sorted, s));
    }
    // resize_truncate / resize_uninit (particles.cu:35-91); new particles are zero
    void resize_truncate(uint32_t N, cudaStream_t s = nullptr)
    {
        check(reyn_particles_resize(h_, N, 1, s));
    }
    void resize_uninit(uint32_t N, cudaStream_t s = nullptr)
    {
        check(reyn_particles_resize(h_, N, 0, s));
    }
    reyn_particles* handle() { return h_; }

private:
    uint32_t n() const
    {
        uint32_t c = 0;
        reyn_particles_count(h_, &c);
        return c;
    }
    reyn_particles* h_ = nullptr;
};

// ---- UniformGrid<R> (uniformgrid.cuh:84-179) --------------------------------
// A POD passed by value to the caller's own kernels, as the reference's is:
// in nvcc-compiled code ff_nbrs maps over the neighbours of a point and
// reduces, like the reference's UniformGrid<R>::ff_nbrs.
template <Resort R> struct UniformGrid {
    reyn_grid_info info;
    const reyn_grid* grid;

#ifdef __CUDACC__
    // Resort::yes: the arrays are in grid order; Resort::no: the grid's
    // permutation maps a sorted slot to the caller's index
    __device__ uint32_t sorted_lookup(uint32_t index) const
    {
        if constexpr (R == Resort::yes)
            return index;
        else
            return info.sorted[index];
    }

    template <class MapOp>
    using AccType = std::invoke_result_t<MapOp, const uint32_t, const float3, const float>;

    // acc += map(j, x_i - x_j, |x_i - x_j|^2) for every j (self included)
    // with |x_i - x_j|^2 <= r^2, over the (2 range + 1)^2 rows of cells
    // around x_i in z, then y, then x order. xx, xy, xz are the arrays the
    // grid was built over. Unlike the reference (whose traversal has no
    // checks), a point outside the grid's searchable interior is mapped to
    // the nearest interior cell, so no access leaves the grid.
    template <class MapOp>
    __device__ AccType<MapOp> ff_nbrs(const float3 x_i, const float* __restrict__ xx,
        const float* __restrict__ xy, const float* __restrict__ xz, MapOp map,
        AccType<MapOp> initial_value = AccType<MapOp> {}) const
    {
        AccType<MapOp> acc { initial_value };
        const int rg = info.range;
        // _index3 (uniformgrid.cuh:17-22)
        int cx = (int)floorf((x_i.x - info.bound_min[0]) / info.cell_size);
        int cy = (int)floorf((x_i.y - info.bound_min[1]) / info.cell_size);
        int cz = (int)floorf((x_i.z - info.bound_min[2]) / info.cell_size);
        cx = min(max(cx, rg), info.nx - 1 - rg);
        cy = min(max(cy, rg), info.ny - 1 - rg);
        cz = min(max(cz, rg), info.nz - 1 - rg);
        const bool zorder = info.order == REYN_ORDER_ZORDER;
        const int tx = (info.nx + 31) / 32, txy = tx * ((info.ny + 31) / 32);
        for (int z = cz - rg; z <= cz + rg; ++z)
            for (int y = cy - rg; y <= cy + rg; ++y) {
                // one run of cells in XYZ order; in Z-order the cells of a
                // row are contiguous within each 4-cell brick
                for (int x = cx - rg; x <= cx + rg;) {
                    const int xe = zorder ? min(cx + rg, x | 3) : cx + rg;
                    const uint32_t k = zorder ? zorder_cell(tx, txy, x, y, z)
                                              : uint32_t(z) * uint32_t(info.nxny)
                            + uint32_t(y) * uint32_t(info.nx) + uint32_t(x);
                    const uint32_t end = info.prefix[k + uint32_t(xe - x + 1)];
                    for (uint32_t j = info.prefix[k]; j < end; ++j) {
                        const uint32_t s_j = sorted_lookup(j);
                        const float3 x_ij = make_float3(x_i.x - xx[s_j], x_i.y - xy[s_j],
                            x_i.z - xz[s_j]);
                        // the engine's |x_ij|^2, so that both prune alike
                        const float l2 = fmaf(x_ij.x, x_ij.x, fmaf(x_ij.y, x_ij.y,
                            x_ij.z * x_ij.z));
                        if (l2 <= info.r_c_2)
                            acc += map(s_j, x_ij, l2);
                    }
                    x = xe + 1;
                }
            }
        return acc;
    }

private:
    // the engine's Z-order cell key: 4x4x4 bricks (x fastest) on the Morton
    // curve inside 32^3-cell tiles, tiles in XYZ order
    __device__ static uint32_t spread3(uint32_t v)
    {
        return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4);
    }
    __device__ static uint32_t zorder_cell(int tx, int txy, int cx, int cy, int cz)
    {
        const uint32_t tile = uint32_t(cz >> 5) * uint32_t(txy) + uint32_t(cy >> 5) * uint32_t(tx)
            + uint32_t(cx >> 5);
        const uint32_t brick = spread3(uint32_t(cx >> 2) & 7u)
            | (spread3(uint32_t(cy >> 2) & 7u) << 1) | (spread3(uint32_t(cz >> 2) & 7u) << 2);
        const uint32_t local = uint32_t(cx & 3) | (uint32_t(cy & 3) << 2) | (uint32_t(cz & 3) << 4);
        return (((tile << 9) | brick) << 6) | local;
    }
#endif
};

// ---- UniformGridBuilder (uniformgrid.cuh:200-489) ---------------------------
class UniformGridBuilder {
public:
    UniformGridBuilder(float3 bound_min, float3 bound_max, float search_radius,
        float cell_ratio = 0.5f, reyn_cell_order order = REYN_ORDER_XYZ)
    {
        const float lo[3] = { bound_min.x, bound_min.y, bound_min.z };
        const float hi[3] = { bound_max.x, bound_max.y, bound_max.z };
        check(reyn_grid_create(lo, hi, search_radius, cell_ratio, order, &g_));
    }
    ~UniformGridBuilder() { reyn_grid_destroy(g_); }
    UniformGridBuilder(const UniformGridBuilder&) = delete;
    UniformGridBuilder& operator=(const UniformGridBuilder&) = delete;

    // construct (uniformgrid.cu:145-156): positions are not moved
    UniformGrid<Resort::no> construct(float search_radius, const float* xx, const float* xy,
        const float* xz, uint32_t n, cudaStream_t s = nullptr)
    {
        check(reyn_grid_construct(g_, search_radius, xx, xy, xz, n, s));
        return { info(), g_ };
    }

    // construct over a state's own positions: a solver step on the result
    // keeps the caller's particle order (the solvers' Resort::no form)
    UniformGrid<Resort::no> construct(float search_radius, Particles& state,
        cudaStream_t s = nullptr)
    {
        reyn_soa v {};
        check(reyn_particles_soa(state.handle(), &v));
        return construct(search_radius, v.xx, v.xy, v.xz, v.n, s);
    }

    // construct_and_reorder (uniformgrid.cuh:477-483): the state and any
    // extra device arrays of n floats are permuted into grid order
    template <class... Extra>
    UniformGrid<Resort::yes> construct_and_reorder(float search_radius, Particles& state,
        Extra*... extra)
    {
        float* ex[] = { static_cast<float*>(extra)..., nullptr };
        check(reyn_grid_construct_and_reorder(g_, search_radius, state.handle(), ex,
            (uint32_t)sizeof...(Extra), nullptr));
        return { info(), g_ };
    }
    UniformGrid<Resort::yes> construct_and_reorder_on(cudaStream_t s, float search_radius,
        Particles& state, std::vector<float*> extra = {})
    {
        check(reyn_grid_construct_and_reorder(g_, search_radius, state.handle(), extra.data(),
            (uint32_t)extra.size(), s));
        return { info(), g_ };
    }

    reyn_grid_info info() const
    {
        reyn_grid_info i {};
        check(reyn_grid_info_get(g_, &i));
        return i;
    }

    reyn_grid* handle() { return g_; }

private:
    reyn_grid* g_ = nullptr;
};

// ---- BoundarySamples (scene.cuh:29-46) ----------------------------------------
class BoundarySamples {
public:
    // device arrays of nb samples; masses computed (Akinci) when m == nullptr
    BoundarySamples(const float* xs, const float* ys, const float* zs, const float* m,
        uint32_t nb, float h, float rho0, uint32_t mass_iters = 5, cudaStream_t s = nullptr)
    {
        check(reyn_boundary_create(xs, ys, zs, m, nb, h, rho0, mass_iters, s, &b_));
    }
    ~BoundarySamples() { reyn_boundary_destroy(b_); }
    BoundarySamples(BoundarySamples&& o) noexcept : b_(std::exchange(o.b_, nullptr)) { }
    BoundarySamples(const BoundarySamples&) = delete;
    BoundarySamples& operator=(const BoundarySamples&) = delete;
    const reyn_boundary* handle() const { return b_; }
    // bound_min / bound_max (scene.cuh:35-36): the samples' bounds
    float3 bound_min() const { return bounds().first; }
    float3 bound_max() const { return bounds().second; }
    uint32_t size() const
    {
        const float *x, *y, *z, *m;
        uint32_t nb = 0;
        check(reyn_boundary_arrays(b_, &x, &y, &z, &m, &nb));
        return nb;
    }

private:
    std::pair<float3, float3> bounds() const
    {
        float lo[3], hi[3];
        check(reyn_boundary_bounds(b_, lo, hi));
        return { make_float3(lo[0], lo[1], lo[2]), make_float3(hi[0], hi[1], hi[2]) };
    }
    reyn_boundary* b_ = nullptr;
};

// ---- solvers -----------------------------------------------------------------
namespace detail {
    template <class K>
    reyn_params params(reyn_scheme scheme, const K& W, float nu, float h, float rho0)
    {
        if (W.h_bar != 2.f * h)
            throw Error(REYN_ERR_INVALID, "the engine's kernel support is 2h (main.cu:51)");
        reyn_params p {};
        check(reyn_params_reference(scheme, K::kind, h, rho0, nu, &p));
        return p;
    }

    class Solver {
    public:
        Solver(reyn_scheme scheme, const reyn_params& p, uint32_t n)
        {
            check(reyn_solver_create(scheme, &p, n, &s_));
        }
        ~Solver() { reyn_solver_destroy(s_); }
        Solver(const Solver&) = delete;
        Solver& operator=(const Solver&) = delete;
        uint32_t step(Particles& st, const reyn_grid* g, const BoundarySamples* bdy, float dt,
            cudaStream_t s)
        {
            uint32_t it = 0;
            check(reyn_solver_step(s_, st.handle(), g, bdy ? bdy->handle() : nullptr, dt, &it, s));
            return it;
        }
        // the step with hard_enforce_bounds and the next controller's
        // max-velocity reduction fused into its integrating kernel
        uint32_t step_bounded(Particles& st, const reyn_grid* g, const BoundarySamples* bdy,
            float dt, float3 bound_min, float3 bound_max, cudaStream_t s)
        {
            const float lo[3] = { bound_min.x, bound_min.y, bound_min.z };
            const float hi[3] = { bound_max.x, bound_max.y, bound_max.z };
            uint32_t it = 0;
            check(reyn_solver_step_bounded(s_, st.handle(), g, bdy ? bdy->handle() : nullptr, dt,
                lo, hi, &it, s));
            return it;
        }
        // simple_dt_controller (cfl.cu:39-52) from the last bounded step's max |v|
        float next_dt(Particles& st, uint32_t iter_last, float dt_last, float lambda, float h,
            float3 g, uint32_t iter_target = 5, float change_factor = 0.01f,
            cudaStream_t s = nullptr)
        {
            const float gg[3] = { g.x, g.y, g.z };
            float dt = 0.f;
            check(reyn_solver_next_dt(s_, st.handle(), iter_last, dt_last, lambda, h, gg,
                iter_target, change_factor, &dt, s));
            return dt;
        }
        reyn_solver_buffers buffers() const
        {
            reyn_solver_buffers b {};
            check(reyn_solver_buffers_get(s_, &b));
            return b;
        }
        reyn_step_stats stats() const
        {
            reyn_step_stats t {};
            check(reyn_solver_stats(s_, &t));
            return t;
        }
        reyn_solver* handle() { return s_; }

    private:
        reyn_solver* s_ = nullptr;
    };
} // namespace detail

// SESPH<K,R> (SESPH.cuh:11-68): step returns nothing, like the reference
template <class K, Resort R = Resort::yes> class SESPH : public detail::Solver {
public:
    SESPH(K W, uint32_t N, float nu, float h, float rho0,
        float3 g = make_float3(0.f, -9.81f, 0.f), float k = 500.f)
        : detail::Solver(REYN_SESPH, with(detail::params(REYN_SESPH, W, nu, h, rho0), g, k), N)
    {
    }
    void step(Particles& st, const UniformGrid<R>& grid, const BoundarySamples& bdy, float dt,
        cudaStream_t s = nullptr)
    {
        detail::Solver::step(st, grid.grid, &bdy, dt, s);
    }
    void step_bounded(Particles& st, const UniformGrid<R>& grid, const BoundarySamples& bdy,
        float dt, float3 bound_min, float3 bound_max, cudaStream_t s = nullptr)
    {
        detail::Solver::step_bounded(st, grid.grid, &bdy, dt, bound_min, bound_max, s);
    }

private:
    static reyn_params with(reyn_params p, float3 g, float k)
    {
        p.g[0] = g.x;
        p.g[1] = g.y;
        p.g[2] = g.z;
        p.k_sesph = k;
        return p;
    }
};

// PCISPH<K,R> (PCISPH.cuh:8-111): step returns the iteration count
template <class K, Resort R = Resort::yes> class PCISPH : public detail::Solver {
public:
    PCISPH(K W, uint32_t N, float nu, float h, float rho0)
        : detail::Solver(REYN_PCISPH, detail::params(REYN_PCISPH, W, nu, h, rho0), N)
    {
    }
    uint32_t step(Particles& st, const UniformGrid<R>& grid, const BoundarySamples& bdy,
        float dt, cudaStream_t s = nullptr)
    {
        return detail::Solver::step(st, grid.grid, &bdy, dt, s);
    }
    // step + hard_enforce_bounds in one pass; next_dt() then needs no pass
    uint32_t step_bounded(Particles& st, const UniformGrid<R>& grid,
        const BoundarySamples& bdy, float dt, float3 bound_min, float3 bound_max,
        cudaStream_t s = nullptr)
    {
        return detail::Solver::step_bounded(st, grid.grid, &bdy, dt, bound_min, bound_max, s);
    }
};

// IISPH<K,R> (IISPH.cuh:8-93): step returns the iteration count
template <class K, Resort R = Resort::yes> class IISPH : public detail::Solver {
public:
    IISPH(K W, uint32_t N, float nu, float h, float rho0)
        : detail::Solver(REYN_IISPH, detail::params(REYN_IISPH, W, nu, h, rho0), N)
    {
    }
    // the configurable form: any reyn_params (e.g. the average-error criterion)
    IISPH(const reyn_params& p, uint32_t N)
        : detail::Solver(REYN_IISPH, p, N)
    {
    }
    uint32_t step(Particles& st, const UniformGrid<R>& grid, const BoundarySamples& bdy,
        float dt, cudaStream_t s = nullptr)
    {
        return detail::Solver::step(st, grid.grid, &bdy, dt, s);
    }
    // step + hard_enforce_bounds in one pass; next_dt() then needs no pass
    uint32_t step_bounded(Particles& st, const UniformGrid<R>& grid,
        const BoundarySamples& bdy, float dt, float3 bound_min, float3 bound_max,
        cudaStream_t s = nullptr)
    {
        return detail::Solver::step_bounded(st, grid.grid, &bdy, dt, bound_min, bound_max, s);
    }
};

// ---- compute_densities<K, R> (solver.cuh:19-38) as a call ---------------------
// the densities of the N points the grid was built over (grid order after
// construct_and_reorder, the caller's order after construct); W's support
// is the grid's search radius
template <class K, Resort R>
void compute_densities(const float* xx, const float* xy, const float* xz, const float* m,
    float* rho, uint32_t N, const K&, const UniformGrid<R>& grid, const BoundarySamples& bdy,
    cudaStream_t s = nullptr)
{
    if (N != grid.info.n)
        throw Error(REYN_ERR_INVALID, "N differs from the grid's point count");
    check(reyn_compute_densities(grid.grid, xx, xy, xz, m, bdy.handle(), K::kind, rho, s));
}

// ---- time step and bounds (cfl.cuh:13-32, scene.cu:485-491) --------------------
inline float cfl_time_step(float lambda, float h, Particles& state, float3 g,
    cudaStream_t s = nullptr)
{
    const float gg[3] = { g.x, g.y, g.z };
    float dt = 0.f;
    check(reyn_cfl_time_step(state.handle(), lambda, h, gg, &dt, s));
    return dt;
}

inline float simple_dt_controller(uint32_t iter_last, float dt_last, float lambda, float h,
    Particles& state, float3 g, uint32_t iter_target = 5, float change_factor = 0.01f,
    cudaStream_t s = nullptr)
{
    const float gg[3] = { g.x, g.y, g.z };
    float dt = 0.f;
    check(reyn_dt_controller(state.handle(), iter_last, dt_last, lambda, h, gg, iter_target,
        change_factor, &dt, s));
    return dt;
}

inline void hard_enforce_bounds(Particles& state, float3 bound_min, float3 bound_max,
    cudaStream_t s = nullptr)
{
    const float lo[3] = { bound_min.x, bound_min.y, bound_min.z };
    const float hi[3] = { bound_max.x, bound_max.y, bound_max.z };
    check(reyn_enforce_bounds(state.handle(), lo, hi, s));
}

// ---- captured steps (no counterpart in the reference) --------------------------
// the loop body `construct_and_reorder(2h, state); step(...); hard bounds` at a
// fixed dt as CUDA graphs (reyn_step_graph_*): launch() replays one step
class StepGraph {
public:
    StepGraph(detail::Solver& solver, Particles& state, UniformGridBuilder& builder,
        const BoundarySamples* bdy, float dt, float3 bound_min, float3 bound_max)
    {
        const float lo[3] = { bound_min.x, bound_min.y, bound_min.z };
        const float hi[3] = { bound_max.x, bound_max.y, bound_max.z };
        check(reyn_step_graph_create(solver.handle(), state.handle(), builder.handle(),
            bdy ? bdy->handle() : nullptr, dt, lo, hi, &g_));
    }
    ~StepGraph() { reyn_step_graph_destroy(g_); }
    StepGraph(const StepGraph&) = delete;
    StepGraph& operator=(const StepGraph&) = delete;
    void launch(cudaStream_t s = nullptr) { check(reyn_step_graph_launch(g_, s)); }
    // sweeps of the last launched step, as IISPH::step / PCISPH::step return
    uint32_t iterations(cudaStream_t s = nullptr)
    {
        reyn_step_stats t {};
        check(reyn_step_graph_stats(g_, &t, s));
        return t.iters;
    }

private:
    reyn_step_graph* g_ = nullptr;
};

// ---- meshes (loader.h:11-20, sample_boundary.cuh:13-163, lbvh.cuh:614-760) --
// Mesh: the reference's host mesh, double vertex components and uint3 faces
struct Mesh {
    std::vector<double> xs, ys, zs;
    std::vector<uint3> faces;
    size_t vertex_count() const { return xs.size(); }
    size_t face_count() const { return faces.size(); }
};

// DeviceMesh together with its LBVH: reyn_mesh builds the tree at creation
class DeviceMesh {
public:
    static DeviceMesh from(const Mesh& m, cudaStream_t s = nullptr)
    {
        std::vector<uint32_t> f(3 * m.faces.size());
        for (size_t t = 0; t < m.faces.size(); ++t) {
            f[3 * t] = m.faces[t].x;
            f[3 * t + 1] = m.faces[t].y;
            f[3 * t + 2] = m.faces[t].z;
        }
        reyn_mesh* h = nullptr;
        check(reyn_mesh_create(m.xs.data(), m.ys.data(), m.zs.data(),
            static_cast<uint32_t>(m.xs.size()), f.data(), static_cast<uint32_t>(m.faces.size()),
            s, &h));
        return DeviceMesh(h);
    }
    // load_mesh_from_obj (loader.cpp) straight into a device mesh
    static DeviceMesh from_obj(const std::string& path, const std::vector<std::string>& ignore = {},
        const char* only_this_name = nullptr, cudaStream_t s = nullptr)
    {
        std::vector<const char*> ig;
        for (const auto& i : ignore)
            ig.push_back(i.c_str());
        reyn_mesh* h = nullptr;
        check(reyn_mesh_load_obj(path.c_str(), ig.data(), static_cast<uint32_t>(ig.size()),
            only_this_name, s, &h));
        return DeviceMesh(h);
    }
    DeviceMesh(DeviceMesh&& o) noexcept : m_(std::exchange(o.m_, nullptr)) { }
    DeviceMesh(const DeviceMesh&) = delete;
    DeviceMesh& operator=(const DeviceMesh&) = delete;
    ~DeviceMesh() { reyn_mesh_destroy(m_); }
    reyn_mesh_info info() const
    {
        reyn_mesh_info i {};
        check(reyn_mesh_info_get(m_, &i));
        return i;
    }
    double get_volume() const { return info().volume; } // sample_boundary.cuh:40-60
    const reyn_mesh* handle() const { return m_; }

private:
    explicit DeviceMesh(reyn_mesh* h) : m_(h) { }
    reyn_mesh* m_ = nullptr;
};

// LBVH (lbvh.cuh:614-760) over a DeviceMesh; the tree lives in the mesh
class LBVH {
public:
    explicit LBVH(const DeviceMesh* mesh) : mesh_(mesh) { }
    // LBVH::project (lbvh.cuh:726-741): n device points, in place
    void project(float* xs, float* ys, float* zs, uint32_t n, cudaStream_t s = nullptr) const
    {
        check(reyn_mesh_project(mesh_->handle(), xs, ys, zs, n, s));
    }
    uint32_t tree_height() const { return mesh_->info().tree_height; }

private:
    const DeviceMesh* mesh_;
};

// uniform_sample_mesh (sample_boundary.cu:299-389): the sample count for
// spacing h / oversampling_factor; writes the samples when xs != nullptr
inline uint32_t uniform_sample_mesh(float* xs, float* ys, float* zs, uint32_t capacity,
    const DeviceMesh& mesh, float h, float oversampling_factor, uint64_t seed = 1614201312,
    cudaStream_t s = nullptr)
{
    uint32_t n = 0;
    check(reyn_mesh_sample_uniform(mesh.handle(), h, oversampling_factor, seed, xs, ys, zs,
        capacity, &n, s));
    return n;
}

// relax_sampling (sample_boundary.cu:100-166); with a debug stream, one CSV
// line "sweep,max/min ratio,average" per sweep as the reference writes
template <class Stream>
void relax_sampling(float* xs, float* ys, float* zs, uint32_t n, const DeviceMesh& mesh,
    float h_bdy, Stream* debug_stream, float relaxation_factor, uint32_t relaxation_iters,
    cudaStream_t s = nullptr)
{
    std::vector<float> st(2 * static_cast<size_t>(relaxation_iters));
    check(reyn_mesh_relax(mesh.handle(), xs, ys, zs, n, h_bdy, relaxation_factor,
        relaxation_iters, st.data(), nullptr, s));
    if (debug_stream)
        for (uint32_t i = 0; i < relaxation_iters; ++i)
            (*debug_stream) << i + 1 << "," << st[2 * i] << "," << st[2 * i + 1] << "\n";
}

// sample_mesh (sample_boundary.cu:391-439; defaults of sample_boundary.cuh:
// 160-163): uniform samples at h / oversampling_factor, relaxed, then the
// boundary with its grid at support 2h and Akinci masses
inline BoundarySamples sample_mesh(const DeviceMesh& mesh, float h, float rho0,
    float oversampling_factor = 2.f, uint32_t relaxation_iters = 50,
    float relaxation_factor = 1.f, uint32_t mass_refinement_iterations = 5,
    uint64_t seed = 1614201312, cudaStream_t s = nullptr)
{
    const uint32_t n = uniform_sample_mesh(nullptr, nullptr, nullptr, 0, mesh, h,
        oversampling_factor, seed, s);
    float* d = nullptr;
    if (cudaMalloc(&d, 3 * sizeof(float) * std::max<size_t>(n, 1)) != cudaSuccess)
        throw Error(REYN_ERR_ALLOC, "sample_mesh: cudaMalloc");
    struct Free {
        float* p;
        ~Free() { cudaFree(p); }
    } guard { d };
    uniform_sample_mesh(d, d + n, d + 2 * size_t(n), n, mesh, h, oversampling_factor, seed, s);
    if (relaxation_iters > 0)
        check(reyn_mesh_relax(mesh.handle(), d, d + n, d + 2 * size_t(n), n,
            h / oversampling_factor, relaxation_factor, relaxation_iters, nullptr, nullptr, s));
    return BoundarySamples(d, d + n, d + 2 * size_t(n), nullptr, n, h, rho0,
        mass_refinement_iterations, s);
}

// ---- Scene (scene.cuh:48-157, scene.cu:255-464) ---------------------------------
// The reference's scene set-up on the engine's kernels. Differences: the
// temporary buffers of the reference's signatures are the engine's own; the
// fluid jitter is uniform with the reference's standard deviation
// (counter-based, seeded) where the reference draws normal jitter.
class Scene {
public:
    float rho0; // the reference's ρ₀
    const float h;
    uint32_t N;
    const BoundarySamples bdy;
    float3 bound_min;
    float3 bound_max;

    // a box [min, max) of fluid at close to N_desired particles inside the
    // boundary the OBJ file's shapes not named "fluid" describe (scene.cu:255-314)
    Scene(const std::string& path, uint32_t N_desired, float3 min, float3 max, float rho0_,
        Particles& state, float bdy_oversampling_factor = 2.f, float cull_bdy_radius = 1.f,
        float jitter_stddev = 0.01f, uint64_t seed = 1)
        : rho0(rho0_)
        , h(cbrtf((max.x - min.x) * (max.y - min.y) * (max.z - min.z) / float(N_desired)))
        , N(0)
        , bdy(sample_mesh(DeviceMesh::from_obj(path, { "fluid" }), h, rho0_,
              bdy_oversampling_factor))
        , bound_min(bdy.bound_min())
        , bound_max(bdy.bound_max())
        , grid_builder_(bound_min, bound_max, 2.f * h)
    {
        const int nx = (int)floorf((max.x - min.x) / h), ny = (int)floorf((max.y - min.y) / h),
                  nz = (int)floorf((max.z - min.z) / h);
        const uint64_t n = uint64_t(std::abs(nx)) * uint64_t(std::abs(ny)) * uint64_t(std::abs(nz));
        if (n == 0)
            throw std::domain_error("Initialization of box failed, zero particles placed");
        if (n > UINT32_MAX)
            throw Error(REYN_ERR_INVALID, "too many particles for one state");
        state.resize_uninit(uint32_t(n));
        const uint32_t counts[3] = { uint32_t(std::abs(nx)), uint32_t(std::abs(ny)),
            uint32_t(std::abs(nz)) };
        const float origin[3] = { min.x, min.y, min.z };
        check(reyn_scene_fluid_block(state.handle(), 0, counts, origin, h, rho0 * h * h * h, 0.f,
            0.f, seed, nullptr));
        N = cull_and_jitter(state, bdy, uint32_t(n), h, cull_bdy_radius, jitter_stddev, seed);
    }

    // Scene::from_obj (scene.cu:316-464): the watertight shape named "fluid"
    // filled at spacing h = cbrt(volume / N_desired), the other shapes sampled
    // as the boundary, the bounds grown to hold the fluid with h / 2 to spare
    static Scene from_obj(const std::string& path, uint32_t N_desired, float rho0,
        Particles& state, float bdy_oversampling_factor = 2.f, float cull_bdy_radius = 1.f,
        float jitter_stddev = 0.01f, uint64_t seed = 1)
    {
        const DeviceMesh fluid = DeviceMesh::from_obj(path, {}, "fluid");
        const reyn_mesh_info fi = fluid.info();
        const float h = static_cast<float>(std::cbrt(fi.volume / double(N_desired)));
        BoundarySamples bdy = sample_mesh(DeviceMesh::from_obj(path, { "fluid" }), h, rho0,
            bdy_oversampling_factor);
        const float e = 0.5f * h;
        const float3 blo = bdy.bound_min(), bhi = bdy.bound_max();
        const float3 lo = make_float3(std::min(blo.x, float(fi.bounds_min[0]) - e),
            std::min(blo.y, float(fi.bounds_min[1]) - e), std::min(blo.z, float(fi.bounds_min[2]) - e));
        const float3 hi = make_float3(std::max(bhi.x, float(fi.bounds_max[0]) + e),
            std::max(bhi.y, float(fi.bounds_max[1]) + e), std::max(bhi.z, float(fi.bounds_max[2]) + e));
        uint32_t n = 0;
        check(reyn_mesh_fill(fluid.handle(), h, 0.f, seed, nullptr, nullptr, nullptr, 0, &n,
            nullptr));
        if (n == 0)
            throw std::domain_error("Initialization of box failed, zero particles placed");
        state.resize_uninit(n);
        const reyn_soa v = state.soa();
        check(reyn_mesh_fill(fluid.handle(), h, 0.f, seed, v.xx, v.xy, v.xz, n, &n, nullptr));
        const std::vector<float> m(n, rho0 * h * h * h);
        state.upload(nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, m.data());
        n = cull_and_jitter(state, bdy, n, h, cull_bdy_radius, jitter_stddev, seed);
        return Scene(rho0, h, n, std::move(bdy), lo, hi);
    }

    // hard_enforce_bounds (scene.cu:485-491)
    void hard_enforce_bounds(Particles& state, cudaStream_t s = nullptr) const
    {
        const float lo[3] = { bound_min.x, bound_min.y, bound_min.z };
        const float hi[3] = { bound_max.x, bound_max.y, bound_max.z };
        check(reyn_enforce_bounds(state.handle(), lo, hi, s));
    }

    // get_grid (scene.cuh:150-157): construct_and_reorder at search_radius h
    template <class... Extra>
    UniformGrid<Resort::yes> get_grid(Particles& state, float search_radius = 2.f,
        Extra*... reorder)
    {
        return grid_builder_.construct_and_reorder(search_radius * h, state, reorder...);
    }

private:
    Scene(float rho0_, float h_, uint32_t n, BoundarySamples&& b, float3 lo, float3 hi)
        : rho0(rho0_)
        , h(h_)
        , N(n)
        , bdy(std::move(b))
        , bound_min(lo)
        , bound_max(hi)
        , grid_builder_(bound_min, bound_max, 2.f * h)
    {
    }
    // cull fluid within cull_bdy_radius h of the boundary (scene.cu:59-83,
    // 176-205), then jitter (scene.cu:232-253); returns the count left
    static uint32_t cull_and_jitter(Particles& state, const BoundarySamples& b, uint32_t n,
        float h, float cull_bdy_radius, float jitter_stddev, uint64_t seed)
    {
        if (cull_bdy_radius > 0.f)
            check(reyn_scene_cull(state.handle(), b.handle(), cull_bdy_radius * h, &n, nullptr));
        check(reyn_scene_jitter(state.handle(), 0, n, 1.7320508f * jitter_stddev * h, seed,
            nullptr));
        if (cudaDeviceSynchronize() != cudaSuccess)
            throw Error(REYN_ERR_CUDA, "scene set-up failed");
        return n;
    }
    UniformGridBuilder grid_builder_;
};

} // namespace reyn

#endif // REYN_B200_HPP_
