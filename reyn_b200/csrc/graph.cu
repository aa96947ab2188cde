// Captured time steps: one full step of the main loop (main.cu:64-75) — the
// grid's construct_and_reorder over the state, then the solver step with hard
// bounds — recorded once as a CUDA graph and replayed. The pressure loop,
// which the host drives with one readback per sweep in a plain step, becomes
// a conditional WHILE node: a one-thread kernel after each sweep applies the
// loop's stopping rule to the sweep's sums and sets the node's condition
// (k_graph_decide), so a replay runs the whole step without returning to the
// host. dt is part of the graph (the fixed-dt configurations).
//
// A reorder swaps the state's current and spare arrays on the host, so two
// graphs are captured, one per buffer parity, and a launch picks the one that
// matches the state's current arrays. Capturing runs the step's host code
// without executing its kernels; every host-side effect of that run (buffer
// swaps, epochs, flags) is undone afterwards and replayed by each launch.
#include "engine.cuh"

#include <cstring>

using namespace reyn;

struct reyn_step_graph {
    reyn_solver* sv = nullptr;
    reyn_particles* st = nullptr;
    reyn_grid* g = nullptr;
    const reyn_boundary* bdy = nullptr;
    float dt = 0.f;
    float lo[3] = { 0, 0, 0 }, hi[3] = { 0, 0, 0 };
    bool bounded = false;
    uint32_t n = 0;
    cudaStream_t cap = nullptr;
    DevArray<GraphStats> stats;
    DevArray<uint32_t> gate;
    GraphCtx ctx;
    cudaGraph_t graph[2] = { nullptr, nullptr };
    cudaGraphExec_t exec[2] = { nullptr, nullptr };
    const float* key[2] = { nullptr, nullptr }; // state's current x array per graph
    const float* pkey[2] = { nullptr, nullptr }; // solver's p array per graph
    bool p_swaps = false; // one step swaps the solver's p and p_tmp an odd number of times
    uint64_t pending_body = 0; // launches whose loop kernels are not yet counted

    ~reyn_step_graph()
    {
        for (int k = 0; k < 2; ++k) {
            if (exec[k])
                cudaGraphExecDestroy(exec[k]);
            if (graph[k])
                cudaGraphDestroy(graph[k]);
        }
        if (ctx.body)
            cudaStreamDestroy(ctx.body);
        if (cap)
            cudaStreamDestroy(cap);
    }
};

namespace {

void swap_state(reyn_particles& st)
{
    for (int k = 0; k < NFIELDS; ++k)
        st.cur[k].swap(st.alt[k]);
}

// host-side fields a step changes, for restoring after a capture
struct HostState {
    const float* cur_x;
    const float* p;
    bool packed_valid;
    uint64_t epoch, version;
    uint32_t grid_n;
    bool reordered, counts_dirty;
    const reyn_particles* reordered_state;
    uint64_t reorder_epoch;
    const reyn_particles* p_state;
    uint64_t p_epoch;
    reyn_step_stats stats;
    bool vmax_valid;
    const reyn_particles* vmax_state;
    uint64_t vmax_version;
    uint32_t n_scenes;

    HostState(const reyn_particles& st, const Grid& g, const reyn_solver& sv)
        : cur_x(st.cur[FX].get())
        , p(sv.p.get())
        , packed_valid(st.packed_valid)
        , epoch(st.epoch)
        , version(st.version)
        , grid_n(g.n)
        , reordered(g.reordered)
        , counts_dirty(g.counts_dirty)
        , reordered_state(g.reordered_state)
        , reorder_epoch(g.reorder_epoch)
        , p_state(sv.p_state)
        , p_epoch(sv.p_epoch)
        , stats(sv.stats)
        , vmax_valid(sv.vmax_valid)
        , vmax_state(sv.vmax_state)
        , vmax_version(sv.vmax_version)
        , n_scenes(sv.n_scenes)
    {
    }
    void restore(reyn_particles& st, Grid& g, reyn_solver& sv) const
    {
        if (st.cur[FX].get() != cur_x)
            swap_state(st);
        if (sv.p.get() != p)
            sv.p.swap(sv.p_tmp);
        st.packed_valid = packed_valid;
        st.epoch = epoch;
        st.version = version;
        g.n = grid_n;
        g.reordered = reordered;
        g.counts_dirty = counts_dirty;
        g.reordered_state = reordered_state;
        g.reorder_epoch = reorder_epoch;
        sv.p_state = p_state;
        sv.p_epoch = p_epoch;
        sv.stats = stats;
        sv.vmax_valid = vmax_valid;
        sv.vmax_state = vmax_state;
        sv.vmax_version = vmax_version;
        sv.n_scenes = n_scenes;
    }
};

// records one step into gr.graph[k] / gr.exec[k] from the current host state
void capture(reyn_step_graph& gr, int k)
{
    reyn_particles& st = *gr.st;
    Grid& g = *gr.g;
    reyn_solver& sv = *gr.sv;
    const HostState before(st, g, sv);
    gr.key[k] = st.cur[FX].get();
    gr.pkey[k] = sv.p.get();
    // the gather branch of the pressure carried across the reorder
    sv.p_state = &st;
    sv.p_epoch = st.epoch;
    gr.ctx.top_names.clear();
    gr.ctx.body_names.clear();
    const cudaStream_t s = gr.cap;
    // the captured build computes its own keys: a histogram pre-keyed by
    // the last plain step is cleared before the capture starts
    g.drop_prekey(s);
    REYN_CUDA(cudaStreamSynchronize(s));
    REYN_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
    sv.graph = &gr.ctx;
    profile_record(&gr.ctx.top_names);
    try {
        REYN_CUDA(cudaMemsetAsync(gr.stats.get(), 0, sizeof(GraphStats), s));
        g.build(st.cur[FX].get(), st.cur[FY].get(), st.cur[FZ].get(), st.n, s);
        reorder_state(st, g, nullptr, 0, s);
        solver_step(sv, st, g, gr.bdy, gr.dt, s, gr.bounded ? gr.lo : nullptr,
            gr.bounded ? gr.hi : nullptr);
    } catch (...) {
        profile_record(nullptr);
        sv.graph = nullptr;
        cudaGraph_t dead = nullptr;
        cudaStreamEndCapture(s, &dead);
        if (dead)
            cudaGraphDestroy(dead);
        before.restore(st, g, sv);
        throw;
    }
    profile_record(nullptr);
    sv.graph = nullptr;
    gr.p_swaps = sv.p.get() != before.p;
    REYN_CUDA(cudaStreamEndCapture(s, &gr.graph[k]));
    REYN_CUDA(cudaGraphInstantiate(&gr.exec[k], gr.graph[k], 0));
    before.restore(st, g, sv);
}

} // namespace

extern "C" int reyn_step_graph_create(reyn_solver* sv, reyn_particles* st, reyn_grid* g,
    const reyn_boundary* bdy, float dt, const float bound_min[3], const float bound_max[3],
    reyn_step_graph** out)
{
    return guard([&] {
        require(out != nullptr, "null output handle");
        *out = nullptr;
        require(sv && st && g, "null argument");
        require(dt > 0.f && std::isfinite(dt), "dt must be positive and finite");
        require(st->n == sv->n, "particle count differs from the solver's");
        require(st->n > 0, "an empty state has no step to capture");
        require(!g->n_scenes || g->first.back() == st->n,
            "particle count differs from the scenes' total");
        auto gr = std::make_unique<reyn_step_graph>();
        gr->sv = sv;
        gr->st = st;
        gr->g = g;
        gr->bdy = bdy;
        gr->dt = dt;
        gr->n = st->n;
        require(!bound_min == !bound_max, "give both bounds or neither");
        gr->bounded = bound_min != nullptr;
        if (g->n_scenes) { // the scenes' own boxes; the bounds only switch them on
            for (int a = 0; a < 3; ++a)
                gr->lo[a] = gr->hi[a] = 0.f;
        } else if (gr->bounded) {
            for (int a = 0; a < 3; ++a) {
                require(std::isfinite(bound_min[a]) && std::isfinite(bound_max[a]),
                    "bounds must be finite");
                gr->lo[a] = bound_min[a];
                gr->hi[a] = bound_max[a];
            }
        }
        REYN_CUDA(cudaStreamCreateWithFlags(&gr->cap, cudaStreamNonBlocking));
        REYN_CUDA(cudaStreamCreateWithFlags(&gr->ctx.body, cudaStreamNonBlocking));
        gr->stats.resize(1);
        gr->gate.resize(1);
        gr->ctx.stats = gr->stats.get();
        gr->ctx.gate = gr->gate.get();
        // every buffer the step touches, sized before the capture: a grid
        // build over the current positions (grid arrays only), the reorder's
        // spare arrays, the solver's buffers and the batched and tail arrays
        const cudaStream_t s = gr->cap;
        g->build(st->cur[FX].get(), st->cur[FY].get(), st->cur[FZ].get(), st->n, s);
        for (auto& a : st->alt)
            a.resize(st->n);
        st->pm.resize(st->n);
        st->vel.resize(st->n);
        g->extra_tmp.resize(st->n);
        ensure_buffers(*sv, st->n);
        const uint32_t ns = g->n_scenes;
        if (ns) {
            sv->scene_stats.resize(size_t(ns) * SWEEP_STATS_BYTES);
            sv->scene_active.resize(ns);
            sv->scene_iters.resize(ns);
            sv->scene_avg.resize(ns);
            sv->scene_max.resize(ns);
            sv->scene_first.resize(ns + 1);
            sv->n_active.resize(1);
            if (!sv->n_active_host)
                sv->n_active_host = std::make_unique<PinnedArray<uint32_t>>(1);
            REYN_CUDA(cudaMemcpyAsync(sv->scene_first.get(), g->first.data(),
                (ns + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
        }
        if (gr->bounded && sv->vmax.size() == 0) {
            sv->vmax.resize(1);
            sv->vmax_host = std::make_unique<PinnedArray<float>>(1);
            REYN_CUDA(cudaEventCreateWithFlags(&sv->vmax_ready, cudaEventDisableTiming));
        }
        // the pressure carried across steps: zero unless it follows this state
        if (sv->scheme == REYN_IISPH && !(sv->p_state == st && sv->p_epoch == st->epoch))
            sv->p.zero(s);
        REYN_CUDA(cudaStreamSynchronize(s));
        g->check_status(s, "reyn_step_graph_create");
        capture(*gr, 0);
        // the other buffer parity: the host state after one step
        swap_state(*st);
        if (gr->p_swaps)
            sv->p.swap(sv->p_tmp);
        try {
            capture(*gr, 1);
        } catch (...) {
            swap_state(*st);
            if (gr->p_swaps)
                sv->p.swap(sv->p_tmp);
            throw;
        }
        swap_state(*st);
        if (gr->p_swaps)
            sv->p.swap(sv->p_tmp);
        if (sv->scheme == REYN_IISPH) { // p now follows this state
            sv->p_state = st;
            sv->p_epoch = st->epoch;
        }
        *out = gr.release();
    });
}

extern "C" int reyn_step_graph_launch(reyn_step_graph* gr, void* stream)
{
    return guard([&] {
        require(gr != nullptr, "null graph");
        reyn_particles& st = *gr->st;
        Grid& g = *gr->g;
        reyn_solver& sv = *gr->sv;
        require(st.n == gr->n && sv.n == gr->n, "the state was resized since the capture");
        const float* x = st.cur[FX].get();
        const int k = x == gr->key[0] ? 0 : (x == gr->key[1] ? 1 : -1);
        require(k >= 0 && sv.p.get() == gr->pkey[k],
            "the state's or solver's buffers changed since the capture (create a new graph)");
        if (sv.scheme == REYN_IISPH)
            require(sv.p_state == &st && sv.p_epoch == st.epoch,
                "the solver's pressure does not follow this state (create a new graph)");
        const cudaStream_t s = as_stream(stream);
        g.drop_prekey(s); // the replayed build computes its own keys
        REYN_CUDA(cudaGraphLaunch(gr->exec[k], s));
        // the host side of the replayed step: the reorder's swap and epochs,
        // the grid's ordering, the solver's pressure and max |v|
        swap_state(st);
        st.epoch += 1;
        st.version += 2;
        st.packed_valid = false;
        g.n = st.n;
        g.reordered = true;
        g.reordered_state = &st;
        g.reorder_epoch = st.epoch;
        g.counts_dirty = false;
        if (gr->p_swaps)
            sv.p.swap(sv.p_tmp);
        sv.p_state = &st;
        sv.p_epoch = st.epoch;
        sv.n_scenes = g.n_scenes;
        sv.stats = reyn_step_stats {};
        if (gr->bounded) {
            REYN_CUDA(cudaMemcpyAsync(sv.vmax_host->get(), sv.vmax.get(), sizeof(float),
                cudaMemcpyDeviceToHost, s));
            REYN_CUDA(cudaEventRecord(sv.vmax_ready, s));
            sv.vmax_state = &st;
            sv.vmax_version = st.version;
            sv.vmax_valid = true;
        } else {
            sv.vmax_valid = false;
        }
        profile_count(gr->ctx.top_names, 1);
        gr->pending_body += 1;
    });
}

extern "C" int reyn_step_graph_stats(reyn_step_graph* gr, reyn_step_stats* out, void* stream)
{
    return guard([&] {
        require(gr && out, "null argument");
        const cudaStream_t s = as_stream(stream);
        GraphStats h {};
        uint32_t status = 0;
        REYN_CUDA(cudaMemcpyAsync(&h, gr->stats.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaMemcpyAsync(&status, gr->g->status.get(), sizeof(status),
            cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaStreamSynchronize(s));
        // the loop's kernels ran h.iters times in the last launch; earlier
        // unread launches are counted with the same number
        profile_count(gr->ctx.body_names, gr->pending_body * h.iters);
        gr->pending_body = 0;
        out->iters = h.iters;
        out->avg_density_error = h.avg_err;
        out->max_density_error = h.max_err;
        gr->sv->stats = *out;
        if (status & STATUS_NONFINITE)
            fail(REYN_ERR_NONFINITE, "a particle position was not finite (clamped)");
        if (status & STATUS_OUT_OF_GRID)
            fail(REYN_ERR_OUT_OF_BOUNDS, "a particle lay outside the grid (clamped)");
        if (h.unconverged)
            fail(REYN_ERR_ITER_LIMIT, "solver reached max_iter before converging (step completed)");
    });
}

extern "C" int reyn_step_graph_info(const reyn_step_graph* gr, uint32_t* step_kernels,
    uint32_t* sweep_kernels)
{
    return guard([&] {
        require(gr != nullptr, "null graph");
        if (step_kernels)
            *step_kernels = uint32_t(gr->ctx.top_names.size());
        if (sweep_kernels)
            *sweep_kernels = uint32_t(gr->ctx.body_names.size());
    });
}

extern "C" int reyn_step_graph_destroy(reyn_step_graph* gr)
{
    delete gr;
    return REYN_OK;
}
