// The autotuner (no counterpart in the reference): picks the block size of
// the neighbour passes and the cell size of the grid (cell = r/2 or r) for
// the caller's own workload by timing it. For every combination the state
// is restored to the snapshot taken on entry, a fresh grid and solver are
// built, one untimed step warms them up, and `steps` steps (grid build with
// reorder + solver step) are timed with CUDA events on the caller's stream.
// The state is left as it was found. A second entry times the reorder
// frequency: the state reordered every K steps, the steps between on grids
// built without reorder (the solvers' Resort::no form).
#include "engine.cuh"

#include <vector>

namespace reyn {

namespace {

    struct Snapshot {
        std::array<DevArray<float>, NFIELDS> a;
        void take(const reyn_particles& st, cudaStream_t s)
        {
            for (int k = 0; k < NFIELDS; ++k) {
                a[k].resize(st.n);
                if (st.n)
                    REYN_CUDA(cudaMemcpyAsync(a[k].get(), st.cur[k].get(), st.n * sizeof(float),
                        cudaMemcpyDeviceToDevice, s));
            }
        }
        void restore(reyn_particles& st, cudaStream_t s) const
        {
            for (int k = 0; k < NFIELDS; ++k)
                if (st.n)
                    REYN_CUDA(cudaMemcpyAsync(st.cur[k].get(), a[k].get(), st.n * sizeof(float),
                        cudaMemcpyDeviceToDevice, s));
            st.packed_valid = false;
            st.version += 1;
        }
    };

    struct Event {
        cudaEvent_t e = nullptr;
        Event() { REYN_CUDA(cudaEventCreate(&e)); }
        ~Event() { cudaEventDestroy(e); }
    };

} // namespace

} // namespace reyn

using namespace reyn;

extern "C" int reyn_autotune(reyn_scheme scheme, const reyn_params* params,
    reyn_particles* state, const reyn_boundary* bdy, const float bound_min[3],
    const float bound_max[3], uint32_t n_scenes, const uint32_t* first, const float* scene_min,
    const float* scene_max, float dt, uint32_t steps, reyn_tune_point* best,
    reyn_tune_point* points, void* stream)
{
    return guard([&] {
        require(params && state && best, "null argument");
        require(steps >= 1, "at least one timed step");
        require(dt > 0.f && std::isfinite(dt), "dt must be positive and finite");
        require(n_scenes ? (first && scene_min && scene_max) : (bound_min && bound_max),
            "bounds (one scene) or scene arrays (a batch) required");
        const cudaStream_t s = as_stream(stream);
        Snapshot snap;
        snap.take(*state, s);
        const uint32_t blocks[4] = { 64, 128, 256, 512 };
        const float ratios[2] = { 0.5f, 1.0f };
        reyn_tune_point all[8] {};
        int k = 0;
        Event e0, e1;
        for (float ratio : ratios) {
            reyn_grid grid;
            if (n_scenes) {
                std::vector<GridGeom> geoms(n_scenes);
                for (uint32_t q = 0; q < n_scenes; ++q)
                    geoms[q] = make_geom(scene_min + 3 * q, scene_max + 3 * q, 2.f * params->h,
                        ratio);
                grid.geom = geoms[0];
                grid.set_scenes(first, n_scenes, geoms.data(), s);
            } else {
                grid.geom = make_geom(bound_min, bound_max, 2.f * params->h, ratio);
            }
            grid.ratio = ratio;
            for (uint32_t b : blocks) {
                reyn_params P = *params;
                P.block_size = b;
                reyn_solver sv;
                sv.scheme = scheme;
                sv.prm = P;
                sv.n = state->n;
                if (scheme == REYN_PCISPH)
                    sv.pcisph_delta = pcisph_template_delta(P.kernel, P.h);
                snap.restore(*state, s);
                auto one = [&] {
                    grid.build(state->cur[FX].get(), state->cur[FY].get(), state->cur[FZ].get(),
                        state->n, s);
                    reorder_state(*state, grid, nullptr, 0, s);
                    try {
                        solver_step(sv, *state, grid, bdy, dt, s);
                    } catch (const Error& e) {
                        if (e.code != REYN_ERR_ITER_LIMIT)
                            throw;
                    }
                };
                one(); // warm-up: buffers, caches
                REYN_CUDA(cudaEventRecord(e0.e, s));
                for (uint32_t t = 0; t < steps; ++t)
                    one();
                REYN_CUDA(cudaEventRecord(e1.e, s));
                REYN_CUDA(cudaEventSynchronize(e1.e));
                float ms = 0.f;
                REYN_CUDA(cudaEventElapsedTime(&ms, e0.e, e1.e));
                all[k++] = reyn_tune_point { b, ratio, ms / float(steps) };
            }
        }
        snap.restore(*state, s);
        int bi = 0;
        for (int q = 1; q < 8; ++q)
            if (all[q].ms_per_step < all[bi].ms_per_step)
                bi = q;
        *best = all[bi];
        if (points)
            for (int q = 0; q < 8; ++q)
                points[q] = all[q];
        REYN_CUDA(cudaStreamSynchronize(s));
    });
}

extern "C" int reyn_autotune_reorder(reyn_scheme scheme, const reyn_params* params,
    reyn_particles* state, const reyn_boundary* bdy, const float bound_min[3],
    const float bound_max[3], float cell_ratio, float dt, uint32_t steps, const uint32_t* every,
    uint32_t n_every, uint32_t* best_every, float* ms_per_step, void* stream)
{
    return guard([&] {
        require(params && state && best_every && every && bound_min && bound_max,
            "null argument");
        require(n_every >= 1 && steps >= 1, "at least one candidate and one timed step");
        require(dt > 0.f && std::isfinite(dt), "dt must be positive and finite");
        require(cell_ratio == 0.5f || cell_ratio == 1.0f, "cell ratio must be 0.5 or 1.0");
        for (uint32_t q = 0; q < n_every; ++q)
            require(every[q] >= 1, "a reorder interval is at least one step");
        const cudaStream_t s = as_stream(stream);
        Snapshot snap;
        snap.take(*state, s);
        reyn_grid grid;
        grid.geom = make_geom(bound_min, bound_max, 2.f * params->h, cell_ratio);
        grid.ratio = cell_ratio;
        Event e0, e1;
        std::vector<float> ms(n_every);
        for (uint32_t q = 0; q < n_every; ++q) {
            reyn_solver sv;
            sv.scheme = scheme;
            sv.prm = *params;
            sv.n = state->n;
            if (scheme == REYN_PCISPH)
                sv.pcisph_delta = pcisph_template_delta(params->kernel, params->h);
            snap.restore(*state, s);
            auto one = [&](bool reorder) {
                grid.build(state->cur[FX].get(), state->cur[FY].get(), state->cur[FZ].get(),
                    state->n, s);
                if (reorder)
                    reorder_state(*state, grid, nullptr, 0, s);
                try {
                    solver_step(sv, *state, grid, bdy, dt, s);
                } catch (const Error& e) {
                    if (e.code != REYN_ERR_ITER_LIMIT)
                        throw;
                }
            };
            // warm-up, two steps for every candidate so that all are timed
            // from the same state: buffers, caches, the unsorted step's own
            one(true);
            one(every[q] == 1);
            REYN_CUDA(cudaEventRecord(e0.e, s));
            for (uint32_t t = 0; t < steps; ++t)
                one(t % every[q] == 0);
            REYN_CUDA(cudaEventRecord(e1.e, s));
            REYN_CUDA(cudaEventSynchronize(e1.e));
            REYN_CUDA(cudaEventElapsedTime(&ms[q], e0.e, e1.e));
            ms[q] /= float(steps);
        }
        snap.restore(*state, s);
        uint32_t bi = 0;
        for (uint32_t q = 1; q < n_every; ++q)
            if (ms[q] < ms[bi])
                bi = q;
        *best_every = every[bi];
        if (ms_per_step)
            for (uint32_t q = 0; q < n_every; ++q)
                ms_per_step[q] = ms[q];
        REYN_CUDA(cudaStreamSynchronize(s));
    });
}
