// Host-side engine objects behind the C ABI handles: particle state, uniform
// grid, boundary and solver. Kernels live in grid.cu and solver.cu.
#pragma once

#include "common.cuh"
#include "device.cuh"

#include <array>
#include <memory>
#include <vector>

namespace reyn {

// statistics of a captured step, kept on the device
struct GraphStats {
    uint32_t iters;       // sweeps of the pressure loop
    uint32_t unconverged; // 1: stopped by max_iter before converging
    double avg_err;       // last average density error (relative)
    double max_err;       // last maximum density error (IISPH)
};

// the capture of one step (reyn_step_graph): the loop bodies are captured on
// `body`; kernel names go to top_names / body_names instead of the launch
// counters
struct GraphCtx {
    cudaStream_t body = nullptr;
    GraphStats* stats = nullptr; // device
    uint32_t* gate = nullptr;    // device: IISPH pressure-pass gate
    std::vector<const char*> top_names, body_names;
};

// while sink is non-null, REYN_KERNEL appends each launch's name to it
// instead of counting and timing it (this thread only)
void profile_record(std::vector<const char*>* sink);
// adds `times` launches of each named kernel to the launch counters
void profile_count(const std::vector<const char*>& names, uint64_t times);

} // namespace reyn

// C-ABI handle types are the engine classes themselves
struct reyn_particles;
struct reyn_grid;
struct reyn_boundary;
struct reyn_solver;

namespace reyn {

enum Field : int { FX = 0, FY, FZ, FVX, FVY, FVZ, FM, NFIELDS };

// Geometry of UniformGridBuilder (uniformgrid.cu:65-96): cell = r * ratio,
// lower bound with a 2r margin, cell counts by ceil. All float arithmetic
// mirrors the reference so that cell keys match bit for bit.
struct GridGeom {
    float lo[3];
    float cell;
    float r;
    int n[3];
    int range; // 2 at ratio 0.5, 1 at ratio 1.0
    int order = REYN_ORDER_XYZ;
    int t[3] = { 0, 0, 0 }; // Z-order: tiles of ZTILE cells per axis
    int64_t cells() const { return int64_t(n[0]) * n[1] * n[2]; }
    // the key space (the prefix covers keys() + 1 entries)
    int64_t keys() const
    {
        return order == REYN_ORDER_ZORDER ? int64_t(t[0]) * t[1] * t[2] * ZTILE * ZTILE * ZTILE
                                          : cells();
    }
};

GridGeom make_geom(const float bmin[3], const float bmax[3], float r, float ratio,
    int order = REYN_ORDER_XYZ);

// The uniform grid over one set of positions.
struct Grid {
    GridGeom geom;
    float ratio = 0.5f;
    DevArray<uint32_t> counts; // C, all zero between builds
    DevArray<uint32_t> prefix; // C + 1
    DevArray<uint32_t> keys;   // n
    DevArray<uint32_t> slots;  // n, unordered counting-sort output
    DevArray<uint32_t> sorted; // n, canonical order (the permutation)
    DevArray<uint32_t> split;  // n, particles of cells split across warps
    DevArray<uint32_t> scan_part;
    DevArray<uint32_t> status; // StatusBits, the split-cell particle count, pre-key StatusBits
    DevArray<float> extra_tmp; // reorder staging of caller arrays
    mutable DevArray<float4> pts_tmp; // packed positions for statistics
    uint32_t n = 0;
    // batched scenes (n_scenes > 0): scene s owns points [first[s],
    // first[s + 1]) in every order the grid produces (its keys are
    // s * geom.keys() + the scene's own key, so a reorder keeps scenes
    // contiguous); sid holds each point's scene
    uint32_t n_scenes = 0;
    std::vector<uint32_t> first;
    DevArray<uint16_t> sid;
    std::vector<GridGeom> scene_geom; // each scene's own grid
    std::vector<uint32_t> key_base;   // first key of each scene (n_scenes + 1)
    DevArray<SceneGeom> scene_tab;
    DevArray<float> scene_lo, scene_hi; // per-scene boxes (3 floats each), fluid grids
    int64_t total_keys() const { return n_scenes ? int64_t(key_base[n_scenes]) : geom.keys(); }
    // scenes with their own geometries (n_scenes entries)
    void set_scenes(const uint32_t* first, uint32_t n_scenes, const GridGeom* geoms,
        cudaStream_t s);
    bool counts_dirty = false; // a build stopped between histogram and scatter
    bool reordered = false;    // last build was construct_and_reorder
    const reyn_particles* reordered_state = nullptr;
    uint64_t reorder_epoch = 0; // state epoch produced by that reorder
    const float* built_pos[3] = { nullptr, nullptr, nullptr }; // positions of the last build
    // Keys and histogram of the next build, computed by the integrating
    // kernel of a solver step on this grid's reordered state (status word 2
    // holds that kernel's status bits): valid while the state is unchanged
    // since (same arrays and version).
    bool prekey_pending = false;
    const reyn_particles* prekey_state = nullptr;
    uint64_t prekey_version = 0;
    const float* prekey_x = nullptr;
    uint32_t prekey_n = 0;

    GridView view(float search_radius) const;
    // counting-sort build over positions: keys, counts, prefix, canonical
    // `sorted`; flags particles outside the grid in `status`. With `st` (the
    // state whose current positions x, y, z are) a pending pre-keyed
    // histogram of that state is used instead of computing the keys.
    void build(const float* x, const float* y, const float* z, uint32_t n,
        cudaStream_t s, const reyn_particles* st = nullptr);
    // drops a pending pre-keyed histogram (its counts are cleared)
    void drop_prekey(cudaStream_t s);
    // host check of the status word (synchronises)
    void check_status(cudaStream_t s, const char* what);
};

} // namespace reyn

// particle state: the reference's SoA arrays (current + spare for the
// reorder swap) and the packed copies the neighbour loops read
struct reyn_particles {
    uint32_t n = 0;
    float rho0 = 1.f;
    std::array<reyn::DevArray<float>, reyn::NFIELDS> cur, alt;
    reyn::DevArray<float4> pm;  // (x, y, z, m) in grid order
    reyn::DevArray<float4> vel; // (vx, vy, vz, rho)
    bool packed_valid = false;
    uint64_t epoch = 0;   // number of reorders applied
    uint64_t version = 0; // changes through this library (uploads, reorders, steps, bounds)
};

struct reyn_grid : reyn::Grid { };

struct reyn_boundary {
    uint32_t nb = 0;
    float h = 0.f;
    float lo[3] = { 0.f, 0.f, 0.f }, hi[3] = { 0.f, 0.f, 0.f }; // the samples' bounds
    reyn::Grid grid;
    reyn::DevArray<float> x, y, z, m;
    reyn::DevArray<float4> pm;
    // per boundary-grid cell: 1 if a sample lies within its (2R+1)^3 block
    // of cells, so that fluid particles elsewhere skip the boundary walk
    reyn::DevArray<uint8_t> near;
    reyn::GridView view() const;
};

struct reyn_solver {
    reyn_scheme scheme;
    reyn_params prm;
    uint32_t n = 0;
    reyn::DevArray<float> rho, p, aii, sii, ax, ay, az;
    reyn::DevArray<float4> acc, vel2, bterm;
    reyn::DevArray<float> p_tmp;
    reyn::DevArray<uint32_t> nbr, ncount; // per-step neighbour list
    reyn::DevArray<uint2> acch, velh, velh2; // MIXED: FP16 neighbour records
    reyn::DevArray<uint4> rec0, rec1;        // MIXED_POS16: 16-byte neighbour records
    reyn::DevArray<float4> gq;               // MIXED_POS16: (G, gsq), then (G, a_ii)
    reyn::DevArray<unsigned char> sweep_stats; // per-sweep reductions
    std::unique_ptr<reyn::PinnedArray<unsigned char>> readback;
    uint64_t p_epoch = 0;      // particle epoch p is ordered for
    const reyn_particles* p_state = nullptr;
    reyn_step_stats stats {};
    double pcisph_delta = 0.0; // k_c_pcisph template stiffness
    // batched scenes: per-scene sweep sums, activity, iterations and errors
    uint32_t n_scenes = 0;
    reyn::DevArray<unsigned char> scene_stats;
    reyn::DevArray<uint8_t> scene_active;
    reyn::DevArray<uint32_t> scene_iters, scene_first, n_active;
    reyn::DevArray<float> scene_avg, scene_max;
    std::unique_ptr<reyn::PinnedArray<uint32_t>> n_active_host;
    // max |v| after the last bounded step, for the next dt controller
    reyn::DevArray<float> vmax;
    std::unique_ptr<reyn::PinnedArray<float>> vmax_host;
    cudaEvent_t vmax_ready = nullptr;
    const reyn_particles* vmax_state = nullptr;
    uint64_t vmax_version = 0;
    bool vmax_valid = false;
    // non-null while a step of this solver is being captured into a graph
    reyn::GraphCtx* graph = nullptr;
    // a step on a grid built by construct (the reference's Resort::no): the
    // state gathered into grid order, stepped there and scattered back
    std::unique_ptr<reyn_particles> shadow;
    std::array<reyn::DevArray<float>, 7> shadow_out; // buffers scattered back
    ~reyn_solver()
    {
        if (vmax_ready)
            cudaEventDestroy(vmax_ready);
    }
};

namespace reyn {

// gather of up to MAX_GATHER arrays by a permutation, plus optional packing
constexpr int MAX_GATHER = 16;
struct GatherArgs {
    const float* src[MAX_GATHER];
    float* dst[MAX_GATHER];
    int count;
    float4* pm;  // (x, y, z, m) from dst[FX..FZ], dst[FM]; may be null
    float4* vel; // (vx, vy, vz, 0) from dst[FVX..FVZ]; may be null
};
void launch_gather(uint32_t n, const uint32_t* perm, const GatherArgs& a,
    cudaStream_t s);

// exclusive prefix sum of C counts into out[0..C] (out[C] = total); `part`
// holds the per-tile partials
void exclusive_scan(const uint32_t* in, int64_t C, DevArray<uint32_t>& part, uint32_t* out,
    cudaStream_t s, uint32_t* fold_status = nullptr);

// packs the particle arrays into pm/vel (after a direct SoA write)
void pack_state(reyn_particles& st, cudaStream_t s);

// the grid's last build was construct over this state's current positions
bool built_unsorted(const Grid& g, const reyn_particles& st);
void reorder_state(reyn_particles& st, Grid& g, float* const* extra,
    uint32_t n_extra, cudaStream_t s);

// the solver's per-particle buffers for n particles (allocated once)
void ensure_buffers(reyn_solver& sv, uint32_t n);

// bytes of one scene's (or one sweep's) convergence sums, an upper bound
constexpr size_t SWEEP_STATS_BYTES = 64;

void kernel_eval(int kind, float h_bar, const float* dx, const float* dy,
    const float* dz, uint32_t n, float* w, float* gx, float* gy, float* gz,
    cudaStream_t s);

// Particles::reorder (particles.cu:93-113) by a caller's permutation, which
// is checked first (synchronises); the state is unchanged when it fails
void reorder_by(reyn_particles& st, const uint32_t* sorted, cudaStream_t s);
// resize_truncate / resize_uninit (particles.cu:35-91): keep the first
// min(old, n) particles or none; the others are zero
void resize_state(reyn_particles& st, uint32_t n, bool keep, cudaStream_t s);
// (x, y, z, m) of point order[s] (s when order is null) into pts[s]
void pack_positions(uint32_t n, const uint32_t* order, const float* x, const float* y,
    const float* z, const float* m, float4* pts, cudaStream_t s);
// compute_densities (solver.cuh:19-38) into rho[n], the caller's order
void compute_densities(const Grid& g, const float* x, const float* y, const float* z,
    const float* m, const reyn_boundary* bdy, int kind, float* rho, cudaStream_t s);
void neighbour_stats(const Grid& g, const float* x, const float* y,
    const float* z, const float* m, int kind, uint32_t* count, float* len2,
    float* rho, cudaStream_t s);

// scene_first/n_scenes (optional): batched boundaries, scene s owning
// samples [scene_first[s], scene_first[s + 1])
void boundary_build(reyn_boundary& b, const float* bx, const float* by,
    const float* bz, const float* bm, uint32_t nb, float h, float rho0,
    uint32_t mass_iters, cudaStream_t s, const uint32_t* scene_first = nullptr,
    uint32_t n_scenes = 0);

// one step; with bounds (bmin and bmax not null) the step also applies
// hard_enforce_bounds and records max |v| in sv.vmax (step tail fusion)
void solver_step(reyn_solver& sv, reyn_particles& st, const Grid& g,
    const reyn_boundary* bdy, float dt, cudaStream_t s, const float* bmin = nullptr,
    const float* bmax = nullptr);

// max |v| over the state: the recorded value of the solver's last bounded
// step when the state has not changed since, else a reduction pass
float state_vmax(reyn_solver* sv, reyn_particles& st, cudaStream_t s);

// cfl_time_step (cfl.cu:5-37); max |v| from state_vmax(sv, st)
float cfl_time_step(reyn_particles& st, float lambda, float h,
    const float g[3], cudaStream_t s, reyn_solver* sv = nullptr);

// total mass, momentum (3) and kinetic energy of the state, FP64
void diagnostics(const reyn_particles& st, double out[5], cudaStream_t s);

void enforce_bounds(reyn_particles& st, const float lo[3], const float hi[3],
    cudaStream_t s);

// host evaluation of k_c_pcisph's template stiffness (PCISPH.cuh:49-77)
double pcisph_template_delta(int kind, float h);

} // namespace reyn
