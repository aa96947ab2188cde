// The C ABI of reyn_b200 (include/reyn_b200.h): argument checks, handle
// management and error translation around the engine in grid.cu/solver.cu.
#include "engine.cuh"

#include <cmath>
#include <string>

namespace reyn {
namespace {
    thread_local std::string g_last_error;
}
void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }
} // namespace reyn

using namespace reyn;

namespace {

void check_kernel(int k) { require(k >= 0 && k <= 3, "unknown smoothing kernel"); }

void check_params(reyn_scheme scheme, const reyn_params* p)
{
    require(p != nullptr, "null params");
    require(scheme >= REYN_SESPH && scheme <= REYN_IISPH, "unknown solver scheme");
    check_kernel(p->kernel);
    require(p->h > 0.f && std::isfinite(p->h), "h must be positive and finite");
    require(p->rho0 > 0.f && std::isfinite(p->rho0), "rho0 must be positive and finite");
    require(std::isfinite(p->nu) && p->nu >= 0.f, "nu must be finite and non-negative");
    require(std::isfinite(p->g[0]) && std::isfinite(p->g[1]) && std::isfinite(p->g[2]),
        "gravity must be finite");
    require(std::isfinite(p->eta) && p->eta >= 0.f, "eta must be finite and non-negative");
    require(p->omega > 0.f && p->omega < 2.f, "omega must lie in (0, 2)");
    require(p->convergence == REYN_CONV_REFERENCE || p->convergence == REYN_CONV_AVERAGE,
        "unknown convergence criterion");
    require(p->precision == REYN_PRECISION_FP32 || p->precision == REYN_PRECISION_MIXED
            || p->precision == REYN_PRECISION_MIXED_POS16,
        "unknown precision");
    require(p->precision == REYN_PRECISION_FP32 || scheme == REYN_IISPH,
        "mixed precision is implemented for IISPH");
    require(p->block_size == 0 || p->block_size == 64 || p->block_size == 128
            || p->block_size == 256 || p->block_size == 512,
        "block_size must be 0, 64, 128, 256 or 512");
}

void check_vec3(const float* v, const char* what)
{
    require(v != nullptr, what);
    require(std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]), what);
}

} // namespace

extern "C" {

const char* reyn_last_error(void) { return reyn::last_error(); }

int reyn_abi_version(void) { return REYN_ABI_VERSION; }

int reyn_kernel_eval(reyn_kernel kernel, float h_bar, const float* dx, const float* dy,
    const float* dz, uint32_t n, float* w, float* gx, float* gy, float* gz, void* stream)
{
    return guard([&] {
        check_kernel(kernel);
        require(n == 0 || (dx && dy && dz && w && gx && gy && gz), "null array");
        kernel_eval(kernel, h_bar, dx, dy, dz, n, w, gx, gy, gz, as_stream(stream));
    });
}

// ---- particles ----------------------------------------------------------------

int reyn_particles_create(uint32_t n, float rho0, reyn_particles** out)
{
    return guard([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        require(rho0 > 0.f && std::isfinite(rho0), "rho0 must be positive and finite");
        auto p = std::make_unique<reyn_particles>();
        p->n = n;
        p->rho0 = rho0;
        for (auto& a : p->cur) {
            a.resize(n);
            if (n)
                REYN_CUDA(cudaMemset(a.get(), 0, size_t(n) * sizeof(float)));
        }
        *out = p.release();
    });
}

int reyn_particles_destroy(reyn_particles* p)
{
    return guard([&] { delete p; });
}

int reyn_particles_soa(reyn_particles* p, reyn_soa* out)
{
    return guard([&] {
        require(p && out, "null argument");
        out->xx = p->cur[FX].get();
        out->xy = p->cur[FY].get();
        out->xz = p->cur[FZ].get();
        out->vx = p->cur[FVX].get();
        out->vy = p->cur[FVY].get();
        out->vz = p->cur[FVZ].get();
        out->m = p->cur[FM].get();
        out->n = p->n;
        out->rho0 = p->rho0;
        // the caller may write through these pointers: what was derived from
        // the current state (the packed copy, the next build's keys and
        // histogram pre-computed by the last step, that step's max |v|) is
        // no longer trusted
        p->packed_valid = false;
        p->version += 1;
    });
}

int reyn_particles_count(const reyn_particles* p, uint32_t* n)
{
    return guard([&] {
        require(p && n, "null argument");
        *n = p->n;
    });
}

int reyn_particles_upload(reyn_particles* p, const float* xx, const float* xy, const float* xz,
    const float* vx, const float* vy, const float* vz, const float* m, void* stream)
{
    return guard([&] {
        require(p != nullptr, "null particles");
        const float* src[NFIELDS] = { xx, xy, xz, vx, vy, vz, m };
        const cudaStream_t s = as_stream(stream);
        for (int k = 0; k < NFIELDS; ++k)
            if (src[k] && p->n)
                REYN_CUDA(cudaMemcpyAsync(p->cur[k].get(), src[k], size_t(p->n) * sizeof(float),
                    cudaMemcpyHostToDevice, s));
        p->packed_valid = false;
        p->version += 1;
    });
}

int reyn_particles_reorder(reyn_particles* p, const uint32_t* sorted, void* stream)
{
    return guard([&] {
        require(p != nullptr, "null particles");
        reorder_by(*p, sorted, as_stream(stream));
    });
}

int reyn_particles_resize(reyn_particles* p, uint32_t n, int keep, void* stream)
{
    return guard([&] {
        require(p != nullptr, "null particles");
        resize_state(*p, n, keep != 0, as_stream(stream));
    });
}

static void download_fields(reyn_particles* p, float* const dst[NFIELDS], cudaStream_t s)
{
    for (int k = 0; k < NFIELDS; ++k)
        if (dst[k] && p->n)
            REYN_CUDA(cudaMemcpyAsync(dst[k], p->cur[k].get(), size_t(p->n) * sizeof(float),
                cudaMemcpyDeviceToHost, s));
}

int reyn_particles_download(reyn_particles* p, float* xx, float* xy, float* xz, float* vx,
    float* vy, float* vz, float* m, void* stream)
{
    return guard([&] {
        require(p != nullptr, "null particles");
        float* const dst[NFIELDS] = { xx, xy, xz, vx, vy, vz, m };
        const cudaStream_t s = as_stream(stream);
        download_fields(p, dst, s);
        REYN_CUDA(cudaStreamSynchronize(s));
    });
}

int reyn_particles_download_async(reyn_particles* p, float* xx, float* xy, float* xz,
    float* vx, float* vy, float* vz, float* m, void* stream)
{
    return guard([&] {
        require(p != nullptr, "null particles");
        float* const dst[NFIELDS] = { xx, xy, xz, vx, vy, vz, m };
        download_fields(p, dst, as_stream(stream));
    });
}

// ---- grid -----------------------------------------------------------------------

int reyn_grid_create(const float bound_min[3], const float bound_max[3], float search_radius,
    float cell_ratio, reyn_cell_order order, reyn_grid** out)
{
    return guard([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        check_vec3(bound_min, "bound_min must be 3 finite floats");
        check_vec3(bound_max, "bound_max must be 3 finite floats");
        require(order == REYN_ORDER_XYZ || order == REYN_ORDER_ZORDER, "unknown cell order");
        auto g = std::make_unique<reyn_grid>();
        g->geom = make_geom(bound_min, bound_max, search_radius, cell_ratio, order);
        g->ratio = cell_ratio;
        const size_t C = size_t(g->geom.keys());
        g->counts.resize(C);
        REYN_CUDA(cudaMemset(g->counts.get(), 0, C * sizeof(uint32_t)));
        g->prefix.resize(C + 1);
        g->status.resize(3);
        *out = g.release();
    });
}

int reyn_grid_create_batched(float search_radius, float cell_ratio, reyn_cell_order order,
    uint32_t n_scenes, const uint32_t* first, const float* scene_min, const float* scene_max,
    reyn_grid** out)
{
    return guard([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        require(first && scene_min && scene_max, "null scene arrays");
        require(n_scenes >= 1, "at least one scene");
        require(order == REYN_ORDER_XYZ || order == REYN_ORDER_ZORDER, "unknown cell order");
        for (uint32_t k = 0; k < 3 * n_scenes; ++k)
            require(std::isfinite(scene_min[k]) && std::isfinite(scene_max[k])
                    && scene_min[k] <= scene_max[k],
                "scene boxes must be finite and ordered");
        auto g = std::make_unique<reyn_grid>();
        std::vector<GridGeom> geoms(n_scenes);
        for (uint32_t k = 0; k < n_scenes; ++k) // each scene: the grid of its own box
            geoms[k] = make_geom(scene_min + 3 * k, scene_max + 3 * k, search_radius, cell_ratio,
                order);
        g->geom = geoms[0];
        g->ratio = cell_ratio;
        g->set_scenes(first, n_scenes, geoms.data(), nullptr);
        g->scene_lo.resize(3 * size_t(n_scenes));
        g->scene_hi.resize(3 * size_t(n_scenes));
        REYN_CUDA(cudaMemcpy(g->scene_lo.get(), scene_min, 3 * size_t(n_scenes) * sizeof(float),
            cudaMemcpyHostToDevice));
        REYN_CUDA(cudaMemcpy(g->scene_hi.get(), scene_max, 3 * size_t(n_scenes) * sizeof(float),
            cudaMemcpyHostToDevice));
        const size_t C = size_t(g->total_keys());
        g->counts.resize(C);
        REYN_CUDA(cudaMemset(g->counts.get(), 0, C * sizeof(uint32_t)));
        g->prefix.resize(C + 1);
        g->status.resize(3);
        *out = g.release();
    });
}

int reyn_grid_destroy(reyn_grid* g)
{
    return guard([&] { delete g; });
}

static void check_radius(const reyn_grid* g, float r)
{
    require(r > 0.f && std::isfinite(r), "search radius must be positive and finite");
    // the grid geometry (cell size, margin) was fixed for g->geom.r; a larger
    // radius would need more cells per strip than the traversal scans
    require(r <= g->geom.r, "search radius exceeds the radius the grid was created for");
}

int reyn_grid_construct(reyn_grid* g, float search_radius, const float* xx, const float* xy,
    const float* xz, uint32_t n, void* stream)
{
    return guard([&] {
        require(g != nullptr, "null grid");
        check_radius(g, search_radius);
        require(n == 0 || (xx && xy && xz), "null position array");
        const cudaStream_t s = as_stream(stream);
        g->build(xx, xy, xz, n, s);
        g->check_status(s, "construct");
    });
}

int reyn_grid_construct_and_reorder(reyn_grid* g, float search_radius, reyn_particles* state,
    float* const* extra, uint32_t n_extra, void* stream)
{
    return guard([&] {
        require(g && state, "null argument");
        check_radius(g, search_radius);
        require(n_extra == 0 || extra != nullptr, "null extra array list");
        const cudaStream_t s = as_stream(stream);
        g->build(state->cur[FX].get(), state->cur[FY].get(), state->cur[FZ].get(), state->n, s,
            state);
        reorder_state(*state, *g, extra, n_extra, s);
        g->check_status(s, "construct_and_reorder");
    });
}

int reyn_grid_reorder(reyn_grid* g, reyn_particles* state, float* const* extra,
    uint32_t n_extra, void* stream)
{
    return guard([&] {
        require(g && state, "null argument");
        require(n_extra == 0 || extra != nullptr, "null extra array list");
        if (!built_unsorted(*g, *state))
            fail(REYN_ERR_NOT_READY,
                "the grid's last build must be construct over this state's positions");
        const cudaStream_t s = as_stream(stream);
        reorder_state(*state, *g, extra, n_extra, s);
    });
}

int reyn_grid_info_get(const reyn_grid* g, reyn_grid_info* out)
{
    return guard([&] {
        require(g && out, "null argument");
        for (int a = 0; a < 3; ++a)
            out->bound_min[a] = g->geom.lo[a];
        out->cell_size = g->geom.cell;
        out->r_c_2 = g->geom.r * g->geom.r;
        out->nx = g->geom.n[0];
        out->ny = g->geom.n[1];
        out->nz = g->geom.n[2];
        out->nxny = g->geom.n[0] * g->geom.n[1];
        out->range = g->geom.range;
        out->n = g->n;
        out->prefix = g->prefix.get();
        out->sorted = g->reordered ? nullptr : g->sorted.get();
        out->order = g->geom.order;
        out->n_keys = uint32_t(g->total_keys());
    });
}

int reyn_grid_permutation(const reyn_grid* g, const uint32_t** perm)
{
    return guard([&] {
        require(g && perm, "null argument");
        *perm = g->sorted.get();
    });
}

int reyn_grid_neighbour_stats(const reyn_grid* g, const float* xx, const float* xy,
    const float* xz, const float* m, reyn_kernel kernel, uint32_t* count, float* len2,
    float* rho, void* stream)
{
    return guard([&] {
        require(g != nullptr, "null grid");
        require(g->n == 0 || (xx && xy && xz), "null position array");
        if (rho)
            check_kernel(kernel);
        const cudaStream_t s = as_stream(stream);
        neighbour_stats(*g, xx, xy, xz, m, kernel, count, len2, rho, s);
        const_cast<reyn_grid*>(g)->check_status(s, "neighbour_stats");
    });
}

int reyn_compute_densities(const reyn_grid* g, const float* xx, const float* xy,
    const float* xz, const float* m, const reyn_boundary* bdy, reyn_kernel kernel, float* rho,
    void* stream)
{
    return guard([&] {
        require(g != nullptr, "null grid");
        require(g->n == 0 || (xx && xy && xz && m && rho), "null array");
        check_kernel(kernel);
        const cudaStream_t s = as_stream(stream);
        compute_densities(*g, xx, xy, xz, m, bdy, kernel, rho, s);
        const_cast<reyn_grid*>(g)->check_status(s, "compute_densities");
    });
}

// ---- boundary -------------------------------------------------------------------

int reyn_boundary_create(const float* bx, const float* by, const float* bz, const float* bm,
    uint32_t nb, float h, float rho0, uint32_t mass_iters, void* stream, reyn_boundary** out)
{
    return guard([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        require(rho0 > 0.f && std::isfinite(rho0), "rho0 must be positive and finite");
        auto b = std::make_unique<reyn_boundary>();
        boundary_build(*b, bx, by, bz, bm, nb, h, rho0, mass_iters, as_stream(stream));
        *out = b.release();
    });
}

int reyn_boundary_create_batched(const float* bx, const float* by, const float* bz,
    const float* bm, uint32_t nb, uint32_t n_scenes, const uint32_t* first, float h, float rho0,
    uint32_t mass_iters, void* stream, reyn_boundary** out)
{
    return guard([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        require(rho0 > 0.f && std::isfinite(rho0), "rho0 must be positive and finite");
        require(first != nullptr && n_scenes >= 1, "scene offsets required");
        require(first[n_scenes] == nb, "scene offsets must end at the sample count");
        require(nb > 0, "a batched boundary needs samples");
        auto b = std::make_unique<reyn_boundary>();
        boundary_build(*b, bx, by, bz, bm, nb, h, rho0, mass_iters, as_stream(stream), first,
            n_scenes);
        *out = b.release();
    });
}

int reyn_boundary_destroy(reyn_boundary* b)
{
    return guard([&] { delete b; });
}

int reyn_boundary_bounds(const reyn_boundary* b, float bound_min[3], float bound_max[3])
{
    return guard([&] {
        require(b && bound_min && bound_max, "null argument");
        for (int a = 0; a < 3; ++a) {
            bound_min[a] = b->lo[a];
            bound_max[a] = b->hi[a];
        }
    });
}

int reyn_boundary_arrays(const reyn_boundary* b, const float** bx, const float** by,
    const float** bz, const float** bm, uint32_t* nb)
{
    return guard([&] {
        require(b != nullptr, "null boundary");
        if (bx)
            *bx = b->x.get();
        if (by)
            *by = b->y.get();
        if (bz)
            *bz = b->z.get();
        if (bm)
            *bm = b->m.get();
        if (nb)
            *nb = b->nb;
    });
}

// ---- solvers ----------------------------------------------------------------------

int reyn_params_reference(reyn_scheme scheme, reyn_kernel kernel, float h, float rho0,
    float nu, reyn_params* out)
{
    return guard([&] {
        require(out != nullptr, "null params");
        require(scheme >= REYN_SESPH && scheme <= REYN_IISPH, "unknown solver scheme");
        check_kernel(kernel);
        reyn_params p {};
        p.kernel = kernel;
        p.h = h;
        p.rho0 = rho0;
        p.nu = nu;
        p.g[0] = 0.f; // SESPH.cuh:41 (default), PCISPH.cuh:27, IISPH.cuh:37
        p.g[1] = -9.81f;
        p.g[2] = 0.f;
        p.k_sesph = 500.f; // SESPH.cuh:50
        p.eta = scheme == REYN_PCISPH ? 0.001f : 0.005f; // PCISPH.cuh:36, IISPH.cuh:41
        p.min_iter = 3; // PCISPH.cuh:38, IISPH.cuh:43
        p.max_iter = 0;
        p.omega = 0.5f; // IISPH.cuh:45
        p.warmstart = 1; // IISPH.cuh:48
        p.convergence = REYN_CONV_REFERENCE;
        p.precision = REYN_PRECISION_FP32;
        p.block_size = 0;
        *out = p;
    });
}

int reyn_solver_create(reyn_scheme scheme, const reyn_params* params, uint32_t n,
    reyn_solver** out)
{
    return guard([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        check_params(scheme, params);
        auto s = std::make_unique<reyn_solver>();
        s->scheme = scheme;
        s->prm = *params;
        s->n = n;
        if (scheme == REYN_PCISPH)
            s->pcisph_delta = pcisph_template_delta(params->kernel, params->h);
        *out = s.release();
    });
}

int reyn_solver_destroy(reyn_solver* s)
{
    return guard([&] { delete s; });
}

static int step_impl(reyn_solver* s, reyn_particles* state, const reyn_grid* grid,
    const reyn_boundary* bdy, float dt, const float* bmin, const float* bmax, uint32_t* iters,
    void* stream)
{
    return guard([&] {
        require(s && state && grid, "null argument");
        if (bmin || bmax) {
            check_vec3(bmin, "bound_min must be 3 finite floats");
            check_vec3(bmax, "bound_max must be 3 finite floats");
        }
        const cudaStream_t st = as_stream(stream);
        if (iters)
            *iters = 0;
        int code = REYN_OK;
        std::string msg;
        try {
            solver_step(*s, *state, *grid, bdy, dt, st, bmin, bmax);
        } catch (const Error& e) {
            if (e.code != REYN_ERR_ITER_LIMIT)
                throw;
            code = e.code;
            msg = e.msg;
        }
        if (iters)
            *iters = s->stats.iters;
        const_cast<reyn_grid*>(grid)->check_status(st, "solver step");
        if (code)
            fail(code, msg);
    });
}

int reyn_solver_step(reyn_solver* s, reyn_particles* state, const reyn_grid* grid,
    const reyn_boundary* bdy, float dt, uint32_t* iters, void* stream)
{
    return step_impl(s, state, grid, bdy, dt, nullptr, nullptr, iters, stream);
}

int reyn_solver_step_batched(reyn_solver* s, reyn_particles* state, const reyn_grid* grid,
    const reyn_boundary* bdy, float dt, int bounded, uint32_t* scene_iters, void* stream)
{
    if (!grid || grid->n_scenes == 0) {
        set_last_error("reyn_solver_step_batched needs a batched grid");
        return REYN_ERR_INVALID;
    }
    // the per-scene boxes replace the bounds; these only switch them on
    const float on[3] = { 0.f, 0.f, 0.f };
    const int rc = step_impl(s, state, grid, bdy, dt, bounded ? on : nullptr,
        bounded ? on : nullptr, nullptr, stream);
    if (scene_iters && (rc == REYN_OK || rc == REYN_ERR_ITER_LIMIT)) {
        const int rc2 = guard([&] {
            REYN_CUDA(cudaMemcpy(scene_iters, s->scene_iters.get(),
                grid->n_scenes * sizeof(uint32_t), cudaMemcpyDeviceToHost));
        });
        if (rc2)
            return rc2;
    }
    return rc;
}

int reyn_solver_scene_stats(const reyn_solver* s, uint32_t n_scenes, reyn_step_stats* out)
{
    return guard([&] {
        require(s && out, "null argument");
        require(n_scenes == s->n_scenes && n_scenes > 0,
            "scene count differs from the last batched step's");
        std::vector<uint32_t> it(n_scenes);
        std::vector<float> avg(n_scenes), mx(n_scenes);
        REYN_CUDA(cudaMemcpy(it.data(), s->scene_iters.get(), n_scenes * sizeof(uint32_t),
            cudaMemcpyDeviceToHost));
        REYN_CUDA(cudaMemcpy(avg.data(), s->scene_avg.get(), n_scenes * sizeof(float),
            cudaMemcpyDeviceToHost));
        REYN_CUDA(cudaMemcpy(mx.data(), s->scene_max.get(), n_scenes * sizeof(float),
            cudaMemcpyDeviceToHost));
        for (uint32_t k = 0; k < n_scenes; ++k)
            out[k] = reyn_step_stats { it[k], avg[k], mx[k] };
    });
}

int reyn_solver_step_bounded(reyn_solver* s, reyn_particles* state, const reyn_grid* grid,
    const reyn_boundary* bdy, float dt, const float bound_min[3], const float bound_max[3],
    uint32_t* iters, void* stream)
{
    if (!bound_min || !bound_max) {
        set_last_error("null bounds");
        return REYN_ERR_INVALID;
    }
    return step_impl(s, state, grid, bdy, dt, bound_min, bound_max, iters, stream);
}

int reyn_solver_buffers_get(const reyn_solver* s, reyn_solver_buffers* out)
{
    return guard([&] {
        require(s && out, "null argument");
        out->rho = s->rho.get();
        out->p = s->p.get();
        out->aii = s->aii.get();
        out->sii = s->sii.get();
        out->ax = s->ax.get();
        out->ay = s->ay.get();
        out->az = s->az.get();
        out->n = s->n;
    });
}

int reyn_solver_pressure_download(const reyn_solver* s, float* host_p, void* stream)
{
    return guard([&] {
        require(s && host_p, "null argument");
        const cudaStream_t st = as_stream(stream);
        if (s->n && s->p.size() == s->n)
            REYN_CUDA(cudaMemcpyAsync(host_p, s->p.get(), size_t(s->n) * sizeof(float),
                cudaMemcpyDeviceToHost, st));
        else
            std::memset(host_p, 0, size_t(s->n) * sizeof(float));
        REYN_CUDA(cudaStreamSynchronize(st));
    });
}

int reyn_solver_pressure_upload(reyn_solver* s, const reyn_particles* state,
    const float* host_p, void* stream)
{
    return guard([&] {
        require(s && state && host_p, "null argument");
        require(state->n == s->n, "particle count differs from the solver's");
        const cudaStream_t st = as_stream(stream);
        s->p.resize(s->n);
        if (s->n)
            REYN_CUDA(cudaMemcpyAsync(s->p.get(), host_p, size_t(s->n) * sizeof(float),
                cudaMemcpyHostToDevice, st));
        REYN_CUDA(cudaStreamSynchronize(st));
        s->p_state = state;
        s->p_epoch = state->epoch;
    });
}

int reyn_solver_stats(const reyn_solver* s, reyn_step_stats* out)
{
    return guard([&] {
        require(s && out, "null argument");
        *out = s->stats;
    });
}

// ---- time step and bounds ------------------------------------------------------------

int reyn_cfl_time_step(reyn_particles* state, float lambda, float h, const float g[3],
    float* dt_out, void* stream)
{
    return guard([&] {
        require(state && dt_out, "null argument");
        check_vec3(g, "gravity must be 3 finite floats");
        *dt_out = cfl_time_step(*state, lambda, h, g, as_stream(stream));
    });
}

// simple_dt_controller, cfl.cu:39-52
static float dt_controller(reyn_solver* sv, reyn_particles& st, uint32_t iter_last,
    float dt_last, float lambda, float h, const float g[3], uint32_t iter_target,
    float change_factor, cudaStream_t s)
{
    const float f = iter_last < iter_target ? 1.f + change_factor : 1.f - change_factor;
    const float suggested = dt_last * f;
    const float cfl = cfl_time_step(st, lambda, h, g, s, sv);
    return std::min(cfl, suggested);
}

int reyn_dt_controller(reyn_particles* state, uint32_t iter_last, float dt_last, float lambda,
    float h, const float g[3], uint32_t iter_target, float change_factor, float* dt_out,
    void* stream)
{
    return guard([&] {
        require(state && dt_out, "null argument");
        check_vec3(g, "gravity must be 3 finite floats");
        *dt_out = dt_controller(nullptr, *state, iter_last, dt_last, lambda, h, g, iter_target,
            change_factor, as_stream(stream));
    });
}

int reyn_solver_next_dt(reyn_solver* s, reyn_particles* state, uint32_t iter_last,
    float dt_last, float lambda, float h, const float g[3], uint32_t iter_target,
    float change_factor, float* dt_out, void* stream)
{
    return guard([&] {
        require(s && state && dt_out, "null argument");
        check_vec3(g, "gravity must be 3 finite floats");
        *dt_out = dt_controller(s, *state, iter_last, dt_last, lambda, h, g, iter_target,
            change_factor, as_stream(stream));
    });
}

int reyn_diagnostics(reyn_particles* state, reyn_diag* out, void* stream)
{
    return guard([&] {
        require(state && out, "null argument");
        double d[5];
        diagnostics(*state, d, as_stream(stream));
        *out = reyn_diag { d[0], { d[1], d[2], d[3] }, d[4] };
    });
}

int reyn_enforce_bounds(reyn_particles* state, const float bound_min[3],
    const float bound_max[3], void* stream)
{
    return guard([&] {
        require(state != nullptr, "null particles");
        check_vec3(bound_min, "bound_min must be 3 finite floats");
        check_vec3(bound_max, "bound_max must be 3 finite floats");
        enforce_bounds(*state, bound_min, bound_max, as_stream(stream));
    });
}

} // extern "C"
