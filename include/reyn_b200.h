/* reyn_b200 — a B200 (sm_100a) SPH step engine behind the reference's
 * (reyn) interfaces. This is the C ABI: plain pointers, sizes and POD
 * structs; every entry point returns an int status (REYN_OK = 0, negative on
 * error) and never throws; reyn_last_error() describes the last failure of
 * the calling thread. Device pointers are CUDA device pointers; `stream` is a
 * cudaStream_t (NULL = legacy default stream). All work is enqueued on
 * `stream`; functions that must return a host value (iteration counts, dt)
 * synchronise that stream.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   smoothing kernels   src/kernels.cuh:19-165 (Kernel<D>, C2, B3, W6, COS)
 *   particle state      src/particles.cuh:25-75 (Particles, SoA xx..m)
 *   uniform grid        src/datastructure/uniformgrid.cuh:200-489
 *                       (UniformGridBuilder, construct, construct_and_reorder)
 *   grid query POD      src/datastructure/uniformgrid.cuh:84-179 (UniformGrid)
 *   boundary            src/scene/scene.cuh:14-46 (Boundary, BoundarySamples),
 *                       src/scene/sample_boundary.cu:267-297 (masses)
 *   solvers             src/solvers/SESPH.cuh:37-53, PCISPH.cuh:80-103,
 *                       IISPH.cuh:51-85 (constructors and step)
 *   time step           src/timestep/cfl.cuh:13-32
 *   bounds              src/scene/scene.cu:485-491 (Scene::hard_enforce_bounds)
 *   meshes              src/datastructure/lbvh.cuh:614-760 (LBVH),
 *                       src/scene/sample_boundary.cu:100-439 (sampling)
 */
#ifndef REYN_B200_H_
#define REYN_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define REYN_ABI_VERSION 1

/* ---- status ------------------------------------------------------------ */
enum reyn_status {
    REYN_OK = 0,
    REYN_ERR_INVALID = -1,       /* bad argument (null, size, enum, ...) */
    REYN_ERR_OUT_OF_BOUNDS = -2, /* a particle lay outside its grid */
    REYN_ERR_NONFINITE = -3,     /* NaN/Inf input where finite is required */
    REYN_ERR_ITER_LIMIT = -4,    /* solver hit max_iter before converging */
    REYN_ERR_CUDA = -5,          /* CUDA runtime error */
    REYN_ERR_ALLOC = -6,         /* device allocation failed */
    REYN_ERR_NOT_READY = -7      /* state used out of order */
};

/* message for the last failing call on this thread ("" if none) */
const char* reyn_last_error(void);
int reyn_abi_version(void);

/* ---- smoothing kernels (src/kernels.cuh:19-174, FOREACH_KERNEL) ---------- */
typedef enum reyn_kernel {
    REYN_KERNEL_C2 = 0, /* Wendland C2, alpha = 21/(2 pi)       kernels.cuh:78 */
    REYN_KERNEL_B3 = 1, /* cubic B-spline, alpha = 16/pi         kernels.cuh:101 */
    REYN_KERNEL_W6 = 2, /* Wendland C6, alpha = 1365/(64 pi)     kernels.cuh:121 */
    REYN_KERNEL_COS = 3 /* double cosine, alpha = pi/(4pi^2-30)  kernels.cuh:148 */
} reyn_kernel;

/* W(dx) and grad W(dx) at support h_bar for n offsets (device SoA arrays),
 * Kernel::operator() and Kernel::nabla (kernels.cuh:40-64). */
int reyn_kernel_eval(reyn_kernel kernel, float h_bar, const float* dx,
    const float* dy, const float* dz, uint32_t n, float* w, float* gx,
    float* gy, float* gz, void* stream);

/* ---- particle state (src/particles.cuh:25-75) ---------------------------- */
typedef struct reyn_particles reyn_particles;

/* current device pointers of the SoA arrays; they CHANGE after a reorder,
 * exactly as Particles' DeviceBuffers swap with `tmp` (buffer.cuh:205-207) */
typedef struct reyn_soa {
    float *xx, *xy, *xz, *vx, *vy, *vz, *m;
    uint32_t n;
    float rho0;
} reyn_soa;

/* Particles(N, rho0) (particles.cu:22): allocates 7 zeroed device arrays */
int reyn_particles_create(uint32_t n, float rho0, reyn_particles** out);
int reyn_particles_destroy(reyn_particles* p);
/* pointers for direct device access. The call counts as a change of the
 * state: what the engine derived from it (its packed copy, the next grid
 * build's keys pre-computed by the last step, that step's max |v|) is
 * recomputed. Fetch the pointers again after every reorder and before
 * writing through them. */
int reyn_particles_soa(reyn_particles* p, reyn_soa* out);
/* the particle count (no change to the state) */
int reyn_particles_count(const reyn_particles* p, uint32_t* n);
/* host <-> device copies of the 7 arrays (any host pointer may be NULL) */
int reyn_particles_upload(reyn_particles* p, const float* xx, const float* xy,
    const float* xz, const float* vx, const float* vy, const float* vz,
    const float* m, void* stream);
int reyn_particles_download(reyn_particles* p, float* xx, float* xy,
    float* xz, float* vx, float* vy, float* vz, float* m, void* stream);
/* reyn_particles_download without the final synchronisation: the copies are
 * enqueued on `stream` (asynchronous for page-locked host memory); the host
 * arrays are valid once the stream has passed this point. Copies of single
 * fields (the others NULL) on their own streams let a caller overlap the
 * download of one field with the upload of another. */
int reyn_particles_download_async(reyn_particles* p, float* xx, float* xy,
    float* xz, float* vx, float* vy, float* vz, float* m, void* stream);
/* Particles::reorder(sorted, tmp) (particles.cu:93-113): every attribute
 * gathered by `sorted` (device, n entries: new[i] = old[sorted[i]]). The
 * array must be a permutation of [0, n): it is checked first (the call
 * synchronises) and REYN_ERR_INVALID leaves the state unchanged. Like the
 * reference, solver buffers are not permuted: IISPH's next step on this
 * state starts from zero pressure. */
int reyn_particles_reorder(reyn_particles* p, const uint32_t* sorted,
    void* stream);
/* Particles::resize_truncate (keep != 0: the first min(old, n) particles
 * are kept) and resize_uninit (keep == 0) (particles.cu:35-91); particles
 * not kept are zero. A solver created for the old count rejects the state;
 * the positions_only form of resize_uninit is not offered (it leaves the
 * arrays at different sizes). Synchronises the stream. */
int reyn_particles_resize(reyn_particles* p, uint32_t n, int keep,
    void* stream);
/* save_to_ply (ply_io.cu:7-55): the positions as a binary PLY point cloud
 * (header: format binary_<native>_endian 1.0, element vertex n, float32
 * properties x, y, z; payload x y z per particle). Synchronises the stream. */
int reyn_particles_save_ply(reyn_particles* p, const char* path, void* stream);
/* (no counterpart in the reference) the whole state as a raw dump for
 * checkpoints: 8-byte magic "REYNSOA1", uint32 n, float rho0, uint32 field
 * count (7), then xx, xy, xz, vx, vy, vz, m as n native-endian floats each.
 * load_raw requires a file with this state's particle count. Both
 * synchronise the stream. */
int reyn_particles_save_raw(reyn_particles* p, const char* path, void* stream);
int reyn_particles_load_raw(reyn_particles* p, const char* path, void* stream);

/* ---- uniform grid (src/datastructure/uniformgrid.cuh:200-489) ----------- */
typedef struct reyn_grid reyn_grid;

typedef enum reyn_cell_order {
    REYN_ORDER_XYZ = 0, /* z*nx*ny + y*nx + x, uniformgrid.cuh:33-40 */
    /* (no counterpart in the reference) Z-order: cells grouped into bricks
     * of 4x4x4 (x fastest inside a brick), bricks along the Morton curve
     * inside tiles of 32x32x32 cells, tiles in XYZ order. A reorder then
     * places particles that are close in space close in memory in all three
     * directions. Keys run over the tiles covering the grid, so prefix has
     * n_keys + 1 entries, n_keys >= nx*ny*nz. */
    REYN_ORDER_ZORDER = 1
} reyn_cell_order;

/* Device-usable description of a built grid: UniformGrid<R>
 * (uniformgrid.cuh:84-179). `sorted` is NULL after construct_and_reorder
 * (Resort::yes: particle arrays are in grid order). prefix has n_keys + 1
 * entries (the last equals n); n_keys = nx*ny*nz in XYZ order. */
typedef struct reyn_grid_info {
    float bound_min[3]; /* lower bound INCLUDING the 2r safety margin */
    float cell_size;
    float r_c_2;        /* squared search radius */
    int32_t nx, ny, nz, nxny;
    int32_t range;      /* cells searched per side: 2 at r/2, 1 at r */
    uint32_t n;         /* particles indexed by the last construct */
    const uint32_t* prefix;
    const uint32_t* sorted;
    int32_t order;      /* reyn_cell_order */
    uint32_t n_keys;    /* cell keys (prefix has n_keys + 1 entries) */
} reyn_grid_info;

/* UniformGridBuilder(bound_min, bound_max, search_radius) (uniformgrid.cu:
 * 65-96). cell_ratio = cell size / search radius: 0.5 is the reference
 * geometry (5x5 strips of 5 cells), 1.0 gives 3x3 strips of 3 cells. */
int reyn_grid_create(const float bound_min[3], const float bound_max[3],
    float search_radius, float cell_ratio, reyn_cell_order order,
    reyn_grid** out);
int reyn_grid_destroy(reyn_grid* g);
/* (no counterpart in the reference) a grid over a batch of independent
 * scenes that share the smoothing kernel, spacing and solver parameters.
 * Scene s owns the particles [first[s], first[s+1]) of one reyn_particles
 * (n_scenes + 1 host offsets) and lies in its own box scene_min/max[3s..3s+2]
 * (host arrays; the boxes may overlap in space: scenes never see each
 * other). Each scene gets the grid a reyn_grid_create over its own box
 * would get, with its own range of cell keys after the previous scene's, so
 * one launch per phase serves every scene and a reorder keeps each scene's
 * particles in its own index range. The grid info's prefix covers all
 * scenes' keys. At most 65535 scenes. */
int reyn_grid_create_batched(float search_radius, float cell_ratio,
    reyn_cell_order order, uint32_t n_scenes, const uint32_t* first,
    const float* scene_min, const float* scene_max, reyn_grid** out);
/* construct (uniformgrid.cu:145-156): builds prefix + sorted for n
 * positions (device arrays), particles are not moved. Within a cell the
 * indices are ascending (a stable counting sort), which is the canonical
 * form of the reference's order. */
int reyn_grid_construct(reyn_grid* g, float search_radius, const float* xx,
    const float* xy, const float* xz, uint32_t n, void* stream);
/* construct_and_reorder (uniformgrid.cuh:477-483): builds the grid over
 * the particle positions, then permutes the 7 state arrays and the n_extra
 * caller arrays (device, n floats each, permuted in place) into grid order. */
int reyn_grid_construct_and_reorder(reyn_grid* g, float search_radius,
    reyn_particles* state, float* const* extra, uint32_t n_extra,
    void* stream);
/* the second half of construct_and_reorder: after reyn_grid_construct over
 * `state`'s own position arrays (reyn_particles_soa), permute the state and
 * the extra arrays by that build's permutation (Particles::reorder,
 * particles.cu:93-113), which makes the grid a reordered one. Between the
 * two calls the positions must not change; the other arrays may still be
 * arriving (a caller can build the grid while velocities upload). */
int reyn_grid_reorder(reyn_grid* g, reyn_particles* state,
    float* const* extra, uint32_t n_extra, void* stream);
int reyn_grid_info_get(const reyn_grid* g, reyn_grid_info* out);
/* after a construct_and_reorder: the permutation applied (new[i] =
 * old[perm[i]]), device array of n entries */
int reyn_grid_permutation(const reyn_grid* g, const uint32_t** perm);

/* neighbour statistics over a built grid (the reference grid test's
 * quantities, uniformgrid.cu:185-207): count of neighbours within r (self
 * excluded), sum of |x_ij|^2, and, if m != NULL, density sum m_j W(x_ij)
 * with `kernel` at support r. Positions/masses are the arrays the grid was
 * built over (in grid order after a reorder). Any output may be NULL. */
int reyn_grid_neighbour_stats(const reyn_grid* g, const float* xx,
    const float* xy, const float* xz, const float* m, reyn_kernel kernel,
    uint32_t* count, float* len2, float* rho, void* stream);

/* ---- uniform grid without allocation --------------------------------------
 * No counterpart in the reference: an added entry point for callers that
 * cannot allocate device memory — real-time loops that must not wait on the
 * device allocator, and hosts whose device memory belongs to another
 * runtime's pool (a game engine, a framework allocator) that only hands out
 * the buffers it created. It builds the same grid as reyn_grid_create +
 * reyn_grid_construct (identical prefix and canonical sorted indices) into
 * the caller's buffers, with its scratch in one file-scope device array of
 * REYN_GRID_NOALLOC_SCRATCH_WORDS 32-bit words (32 MiB) that every GPU
 * loading the library holds until exit. It calls no allocating routine.
 *
 * Limit: nx*ny*nz + 2 n + ceil(nx*ny*nz / 4096) + 2 <= the scratch words
 * (e.g. 1M particles over 5M cells); larger sizes fail with REYN_ERR_INVALID.
 * dims (may be NULL) receives nx, ny, nz; prefix == NULL only reports dims.
 * prefix needs nx*ny*nz + 1 entries (prefix_capacity); xx, xy, xz and sorted
 * n entries each. The first call on each device looks up the scratch array's
 * device address (cudaGetSymbolAddress) and should come before any stream
 * capture. All calls share the array and it keeps the last call's contents
 * (each call clears the counters it needs): calls that overlap on the GPU
 * race; serialise them. It synchronises `stream` (to report particles
 * outside the grid: REYN_ERR_OUT_OF_BOUNDS, REYN_ERR_NONFINITE). */
#define REYN_GRID_NOALLOC_SCRATCH_WORDS (8u * 1024u * 1024u)
int reyn_grid_construct_noalloc(const float bound_min[3],
    const float bound_max[3], float search_radius, float cell_ratio,
    const float* xx, const float* xy, const float* xz, uint32_t n,
    uint32_t* prefix, uint64_t prefix_capacity, uint32_t* sorted,
    int32_t dims[3], void* stream);

/* ---- boundary (src/scene/scene.cuh:14-46) -------------------------------- */
typedef struct reyn_boundary reyn_boundary;

/* Boundary samples at positions bx,by,bz (DEVICE arrays, nb entries) with
 * masses bm (device) or, if bm == NULL, Akinci masses computed as
 * calculate_boundary_masses does (sample_boundary.cu:267-297: B3 at 2h,
 * m = 1 then `mass_iters` refinements; double-buffered here). The samples
 * are copied and reordered into their own grid at support 2h over their own
 * bounds (sample_boundary.cu:413-428). nb == 0 is an empty boundary. */
int reyn_boundary_create(const float* bx, const float* by, const float* bz,
    const float* bm, uint32_t nb, float h, float rho0, uint32_t mass_iters,
    void* stream, reyn_boundary** out);
int reyn_boundary_destroy(reyn_boundary* b);
/* (no counterpart) the boundary of a batch: scene s owns samples [first[s],
 * first[s+1]) (host offsets); Akinci masses and every boundary term use
 * only the samples of the particle's own scene. */
int reyn_boundary_create_batched(const float* bx, const float* by,
    const float* bz, const float* bm, uint32_t nb, uint32_t n_scenes,
    const uint32_t* first, float h, float rho0, uint32_t mass_iters,
    void* stream, reyn_boundary** out);
/* device pointers of the reordered samples and masses */
int reyn_boundary_arrays(const reyn_boundary* b, const float** bx,
    const float** by, const float** bz, const float** bm, uint32_t* nb);

/* BoundarySamples::bound_min / bound_max (scene.cuh:35-36): the smallest
 * box holding every sample (zeros without samples) */
int reyn_boundary_bounds(const reyn_boundary* b, float bound_min[3],
    float bound_max[3]);

/* compute_densities<K, R> (solver.cuh:19-38): rho_i = sum_j m_j W(x_ij) over
 * the fluid neighbours within the grid's radius r (self included) plus
 * sum_b m_b W(x_ib) over the boundary samples (bdy may be NULL), `kernel` at
 * support r. Positions and masses are the arrays the grid was built over:
 * in grid order after construct_and_reorder, the caller's order after
 * reyn_grid_construct (rho is then in the caller's order too). Not for
 * batched grids. */
int reyn_compute_densities(const reyn_grid* g, const float* xx,
    const float* xy, const float* xz, const float* m, const reyn_boundary* bdy,
    reyn_kernel kernel, float* rho, void* stream);

/* ---- solvers (src/solvers/SESPH, PCISPH, IISPH) ------------------------- */
typedef enum reyn_scheme {
    REYN_SESPH = 0, /* SESPH.cu:68-95   */
    REYN_PCISPH = 1, /* PCISPH.cu:59-111 */
    REYN_IISPH = 2 /* IISPH.cu:165-262 */
} reyn_scheme;

typedef enum reyn_convergence {
    /* the reference's own criteria: PCISPH avg(rho) <= (1+eta) rho0
     * (PCISPH.cu:101); IISPH "no particle's predicted error above eta rho0"
     * (IISPH.cu:246-250) */
    REYN_CONV_REFERENCE = 0,
    /* IISPH: average of max(0, predicted density error) <= eta rho0,
     * reduced in FP64 */
    REYN_CONV_AVERAGE = 1
} reyn_convergence;

typedef enum reyn_precision {
    /* FP32 storage and arithmetic, as the reference */
    REYN_PRECISION_FP32 = 0,
    /* IISPH only: the velocities, densities and pressure accelerations the
     * neighbour loops read of a particle's neighbours are stored as FP16;
     * positions, the particle's own data and all arithmetic stay FP32, the
     * convergence reduction FP64. */
    REYN_PRECISION_MIXED = 1,
    /* IISPH only: as REYN_PRECISION_MIXED, and neighbour positions stored as
     * 16-bit fixed point relative to the grid (1/16384 cell) with FP16
     * masses (relative to particle 0's) */
    REYN_PRECISION_MIXED_POS16 = 2
} reyn_precision;

typedef struct reyn_params {
    reyn_kernel kernel;     /* support radius = 2h (main.cu:51) */
    float h;                /* particle spacing */
    float rho0;             /* rest density */
    float nu;               /* viscosity */
    float g[3];             /* gravity */
    float k_sesph;          /* SESPH stiffness (SESPH.cuh:50: 500) */
    float eta;              /* tolerance (PCISPH 0.001, IISPH 0.005) */
    uint32_t min_iter;      /* 3 (PCISPH.cuh:38, IISPH.cuh:43) */
    uint32_t max_iter;      /* 0 = unbounded, as the reference (a safety bound of
                             * 100000 sweeps still ends a step that cannot
                             * converge, with REYN_ERR_ITER_LIMIT) */
    float omega;            /* IISPH Jacobi weight (0.5, IISPH.cuh:45) */
    int32_t warmstart;      /* IISPH p *= 0.5 (IISPH.cuh:48) */
    reyn_convergence convergence;
    reyn_precision precision; /* REYN_PRECISION_FP32 unless set */
    uint32_t block_size;    /* threads per block of the neighbour passes:
                               64, 128, 256 or 512; 0 = 128 */
} reyn_params;

/* the reference's constants for `scheme` (gravity (0,-9.81,0)) */
int reyn_params_reference(reyn_scheme scheme, reyn_kernel kernel, float h,
    float rho0, float nu, reyn_params* out);

typedef struct reyn_solver reyn_solver;

/* SESPH/PCISPH/IISPH(W, N, nu, h, rho0, buffers...): the solver owns its
 * per-particle buffers (rho, a, p, a_ii, s_i). */
int reyn_solver_create(reyn_scheme scheme, const reyn_params* params,
    uint32_t n, reyn_solver** out);
int reyn_solver_destroy(reyn_solver* s);

/* Solver::step(state, grid, bdy, dt) on a grid built by
 * construct_and_reorder over `state` (the solvers' Resort::yes form), or by
 * reyn_grid_construct over `state`'s own position arrays (reyn_particles_soa;
 * Resort::no, IISPH.cu:264-266): the particles then keep the caller's order,
 * the step runs on a copy gathered into grid order and positions,
 * velocities and the solver buffers are scattered back (not batched grids,
 * not inside a step graph). IISPH's pressure is carried across steps in the
 * state's order and re-permuted with the grid's permutation automatically
 * (the reference passes it as an extra reorder buffer, main.cu:68). iters
 * (may be NULL) receives the iteration count (1 for SESPH); it synchronises
 * the stream for PCISPH/IISPH. */
int reyn_solver_step(reyn_solver* s, reyn_particles* state,
    const reyn_grid* grid, const reyn_boundary* bdy, float dt,
    uint32_t* iters, void* stream);

/* (no counterpart: the reference's main loop, main.cu:64-75, runs the step,
 * hard_enforce_bounds and the next dt controller's max-velocity reduction
 * as separate passes) The step with its tail fused: the kernel that writes
 * the new positions and velocities applies hard_enforce_bounds
 * (scene.cu:466-491) to them and max-reduces |v| of what it stores. The
 * result equals reyn_solver_step followed by reyn_enforce_bounds; the
 * recorded max |v| serves reyn_solver_next_dt. */
int reyn_solver_step_bounded(reyn_solver* s, reyn_particles* state,
    const reyn_grid* grid, const reyn_boundary* bdy, float dt,
    const float bound_min[3], const float bound_max[3], uint32_t* iters,
    void* stream);

/* per-particle solver buffers (device, in the particle order of the last
 * step's state: grid order after construct_and_reorder): rho
 * the (predicted) densities, ax..az the last accelerations; p the IISPH
 * pressure, for PCISPH the pressure term p / rho^2 of the last iteration
 * (_eos_pcisph, PCISPH.cu:15-19); aii, sii the IISPH diagonal and source */
typedef struct reyn_solver_buffers {
    const float *rho, *p, *aii, *sii, *ax, *ay, *az;
    uint32_t n;
} reyn_solver_buffers;
int reyn_solver_buffers_get(const reyn_solver* s, reyn_solver_buffers* out);

/* the pressure IISPH carries across steps (its warm start, IISPH.cuh:48),
 * copied to / from host memory: n floats in the particle order of `state`
 * at the time of the call. With the particle arrays (download/upload) this
 * is a complete checkpoint of a simulation. Upload binds the pressure to
 * the current order of `state`. Both synchronise the stream. */
int reyn_solver_pressure_download(const reyn_solver* s, float* host_p,
    void* stream);
int reyn_solver_pressure_upload(reyn_solver* s, const reyn_particles* state,
    const float* host_p, void* stream);

/* statistics of the last step: iterations and the last sweep's average
 * (max(0, .)) and maximum predicted density error, in units of rho0 */
typedef struct reyn_step_stats {
    uint32_t iters;
    double avg_density_error;
    double max_density_error;
} reyn_step_stats;
int reyn_solver_stats(const reyn_solver* s, reyn_step_stats* out);

/* (no counterpart) one step of every scene of a batched grid (after
 * construct_and_reorder over the batch): each phase is one launch over all
 * scenes; PCISPH/IISPH iterate per scene, a scene leaving the iteration once
 * it meets the criterion while the others go on (its particles then sit out
 * the remaining sweeps). bounded != 0 applies hard_enforce_bounds with each
 * scene's own box in the integrating kernel. scene_iters (host, n_scenes
 * entries, may be NULL) receives each scene's iteration count. One dt for
 * all scenes. */
int reyn_solver_step_batched(reyn_solver* s, reyn_particles* state,
    const reyn_grid* grid, const reyn_boundary* bdy, float dt, int bounded,
    uint32_t* scene_iters, void* stream);
/* per-scene iterations and density errors of the last batched step */
int reyn_solver_scene_stats(const reyn_solver* s, uint32_t n_scenes,
    reyn_step_stats* out);

/* ---- time step (src/timestep/cfl.cu) -------------------------------------- */
/* cfl_time_step (cfl.cu:5-37); synchronises the stream */
int reyn_cfl_time_step(reyn_particles* state, float lambda, float h,
    const float g[3], float* dt_out, void* stream);
/* simple_dt_controller (cfl.cu:39-52); synchronises the stream */
int reyn_dt_controller(reyn_particles* state, uint32_t iter_last,
    float dt_last, float lambda, float h, const float g[3],
    uint32_t iter_target, float change_factor, float* dt_out, void* stream);
/* simple_dt_controller with the max |v| that the solver's last
 * reyn_solver_step_bounded reduced, when `state` has not changed through
 * this library since (otherwise a reduction pass, as reyn_dt_controller).
 * Fetching the state's pointers (reyn_particles_soa) counts as a change;
 * writes through pointers fetched before the step are not seen: after such
 * writes use reyn_dt_controller. Waits for that step's last kernel. */
int reyn_solver_next_dt(reyn_solver* s, reyn_particles* state,
    uint32_t iter_last, float dt_last, float lambda, float h, const float g[3],
    uint32_t iter_target, float change_factor, float* dt_out, void* stream);

/* ---- diagnostics (no counterpart in the reference) ------------------------ */
typedef struct reyn_diag {
    double mass;        /* sum m */
    double momentum[3]; /* sum m v */
    double kinetic;     /* sum m |v|^2 / 2 */
} reyn_diag;
/* global mass, momentum and kinetic energy of the state, reduced in FP64;
 * synchronises the stream */
int reyn_diagnostics(reyn_particles* state, reyn_diag* out, void* stream);

/* ---- bounds (src/scene/scene.cu:466-491) ---------------------------------- */
int reyn_enforce_bounds(reyn_particles* state, const float bound_min[3],
    const float bound_max[3], void* stream);

/* ---- autotuner (no counterpart in the reference) -------------------------- */
typedef struct reyn_tune_point {
    uint32_t block_size;  /* threads per block of the neighbour passes */
    float cell_ratio;     /* cell size / search radius */
    float ms_per_step;    /* grid build with reorder + solver step */
} reyn_tune_point;
/* Times the caller's workload for every block size in {64, 128, 256, 512}
 * and cell ratio in {0.5, 1.0}: each from the state as it is on entry,
 * with a fresh grid and solver, one untimed step, then `steps` timed steps.
 * One scene: bound_min/max are its grid bounds; a batch: n_scenes > 0 with
 * the scene arrays of reyn_grid_create_batched (bdy batched likewise). The
 * state is restored before returning. *best is the fastest combination;
 * points (may be NULL) receives all eight. Synchronises the stream. */
int reyn_autotune(reyn_scheme scheme, const reyn_params* params,
    reyn_particles* state, const reyn_boundary* bdy, const float bound_min[3],
    const float bound_max[3], uint32_t n_scenes, const uint32_t* first,
    const float* scene_min, const float* scene_max, float dt, uint32_t steps,
    reyn_tune_point* best, reyn_tune_point* points, void* stream);

/* The reorder frequency for one scene at a chosen block size
 * (params->block_size) and cell ratio: for every candidate interval K in
 * every[0 .. n_every-1], from the state as it is on entry, with a fresh
 * solver, `steps` timed steps that reorder the state (construct_and_reorder)
 * when the step index is a multiple of K and otherwise build the grid
 * without reorder (reyn_grid_construct over the state's arrays: the solvers'
 * Resort::no form). A multiple of every K for `steps` times whole cycles.
 * The state is restored before returning. *best_every is the fastest
 * interval; ms_per_step (may be NULL) receives n_every times. Synchronises
 * the stream. */
int reyn_autotune_reorder(reyn_scheme scheme, const reyn_params* params,
    reyn_particles* state, const reyn_boundary* bdy, const float bound_min[3],
    const float bound_max[3], float cell_ratio, float dt, uint32_t steps,
    const uint32_t* every, uint32_t n_every, uint32_t* best_every,
    float* ms_per_step, void* stream);

/* ---- captured steps (no counterpart in the reference) -------------------- */
typedef struct reyn_step_graph reyn_step_graph;
/* Records one full step of the main loop at a fixed dt — construct_and_reorder
 * of `grid` over `state`, then the solver's step, with hard bounds when
 * bound_min/bound_max are given (for a batched grid each scene's own box; the
 * values are then unused) — as CUDA graphs, one per buffer parity of the
 * state. The pressure loop of PCISPH and IISPH runs as a conditional while
 * node whose condition a kernel sets after each sweep with the plain step's
 * stopping rule, so a launch needs no host round trip; results equal the
 * plain calls'. The solver, state, grid and boundary must outlive the graph,
 * and the state keeps its particle count. Synchronises. */
int reyn_step_graph_create(reyn_solver* s, reyn_particles* state, reyn_grid* grid,
    const reyn_boundary* bdy, float dt, const float bound_min[3],
    const float bound_max[3], reyn_step_graph** out);
/* one step: the graph launch on `stream` plus the host bookkeeping of the plain
 * calls (no synchronisation); plain steps may be interleaved */
int reyn_step_graph_launch(reyn_step_graph* g, void* stream);
/* the last launched step's sweeps and density errors (synchronises the
 * stream); returns the status the plain calls would have returned for it
 * (REYN_ERR_ITER_LIMIT, REYN_ERR_OUT_OF_BOUNDS, REYN_ERR_NONFINITE) */
int reyn_step_graph_stats(reyn_step_graph* g, reyn_step_stats* out,
    void* stream);
/* kernels per step outside the pressure loop, and per sweep inside it */
int reyn_step_graph_info(const reyn_step_graph* g, uint32_t* step_kernels,
    uint32_t* sweep_kernels);
int reyn_step_graph_destroy(reyn_step_graph* g);

/* ---- scene generation (src/scene/scene.cu) ------------------------------- */
/* _init_box_kernel (scene.cu:14-37) with seeded jitter (scene.cu:232-253):
 * particles first .. first + nx*ny*nz - 1 of the state become a lattice of
 * spacing `spacing` from `origin`, x fastest, each coordinate moved by a
 * uniform jitter in [-jitter, jitter] * spacing and each velocity component
 * uniform in [-velocity_noise, velocity_noise]. The random numbers are
 * counter-based (SplitMix64 of seed and particle index), so the result does
 * not depend on the launch and is reproducible on the host. mass <= 0 gives
 * the reference's rest mass rho0 spacing^3. */
int reyn_scene_fluid_block(reyn_particles* p, uint32_t first,
    const uint32_t counts[3], const float origin[3], float spacing, float mass,
    float jitter, float velocity_noise, uint64_t seed, void* stream);
/* (no counterpart in the reference, which samples boundaries from meshes,
 * sample_boundary.cu:100-248) one layer of boundary samples on the six faces
 * of an axis-aligned box, n = rint(extent / spacing) intervals per axis, no
 * duplicates at edges and corners. *count receives the number of samples;
 * with x == NULL nothing is written (size query). x, y, z: device arrays. */
int reyn_scene_box_walls(const float bound_min[3], const float bound_max[3],
    float spacing, float* x, float* y, float* z, uint64_t capacity,
    uint64_t* count, void* stream);
/* (no counterpart in the reference) a sphere sampled by the golden-angle
 * (Fibonacci) spiral, max(1, rint(4 pi r^2 / spacing^2)) samples; size query
 * with x == NULL as above. */
int reyn_scene_sphere(const float center[3], float radius, float spacing,
    float* x, float* y, float* z, uint32_t capacity, uint32_t* count,
    void* stream);
/* jitter_positions (scene.cu:232-253): particles first .. first + count - 1
 * move by a uniform [-amplitude, amplitude] per axis from the counter-based
 * streams 0..2 keyed by the particle index (the fluid blocks' jitter). The
 * reference draws normal jitter of standard deviation sigma; amplitude
 * sqrt(3) sigma gives the same standard deviation. */
int reyn_scene_jitter(reyn_particles* p, uint32_t first, uint32_t count,
    float amplitude, uint64_t seed, void* stream);
/* the reference's cull of fluid particles too close to the boundary
 * (CullPredicate + remove_if, scene.cu:59-83, 176-205): removes, keeping the
 * order of the rest, every particle with a boundary sample within `radius`
 * (at most the boundary grid's search radius 2h); the state's particle count
 * shrinks to *n_out. Synchronises the stream. */
int reyn_scene_cull(reyn_particles* p, const reyn_boundary* bdy, float radius,
    uint32_t* n_out, void* stream);

/* ---- triangle meshes: LBVH queries, boundary sampling, fluid fill ---------
 * src/scene/loader.{h,cpp} (Mesh, load_mesh_from_obj), sample_boundary.cuh:
 * 13-60 (DeviceMesh, get_volume), src/datastructure/lbvh.cuh:614-760 (LBVH),
 * src/scene/sample_boundary.cu:100-248, 299-389 (relax_sampling,
 * uniform_sample_mesh), src/scene/scene.cu:84-139, 316-425 (InsidePredicate,
 * Scene::from_obj's fluid fill). A mesh owns its vertices (double, as the
 * reference stores them), its triangles and the LBVH over them. */
typedef struct reyn_mesh reyn_mesh;

typedef struct reyn_mesh_info {
    uint32_t n_vertices;
    uint32_t n_faces;
    uint32_t tree_height;  /* edges from the root to the deepest leaf */
    uint32_t reserved;
    double bounds_min[3];  /* extent of all vertices (LBVH bounds_min/max) */
    double bounds_max[3];
    double area;           /* total surface area */
    double volume;         /* |signed volume|: closed, consistently wound meshes */
} reyn_mesh_info;

/* DeviceMesh::from + LBVH(DeviceMesh*) (sample_boundary.cuh:22-30,
 * lbvh.cuh:646-723): host vertex coordinates and host triangles (3 vertex
 * indices each). Builds the LBVH over the faces sorted by the 30-bit Morton
 * code of their centroids (ties by face index). Synchronises the stream. */
int reyn_mesh_create(const double* vx, const double* vy, const double* vz,
    uint32_t n_vertices, const uint32_t* faces, uint32_t n_faces, void* stream,
    reyn_mesh** out);
/* load_mesh_from_obj (loader.cpp) + reyn_mesh_create: a Wavefront OBJ file of
 * triangles ("v" and "f" records; "o"/"g" name the shapes). Shapes whose
 * lower-case name contains any of the n_ignore strings are skipped; with
 * `only` != NULL only shapes whose name contains it are kept. Every vertex
 * of the file is kept, as the reference's loader does. */
int reyn_mesh_load_obj(const char* path, const char* const* ignore,
    uint32_t n_ignore, const char* only, void* stream, reyn_mesh** out);
int reyn_mesh_destroy(reyn_mesh* mesh);
int reyn_mesh_info_get(const reyn_mesh* mesh, reyn_mesh_info* out);
/* the LBVH in the reference's layout, device arrays (any may be NULL):
 * order[j] = original face of leaf j (n_faces); children_l/r (n_faces - 1) in
 * the ChildNode encoding index << 1 | (1 for an internal node) of
 * lbvh.cuh:162-193; leaf_box (6 n_faces) and node_box (6 (n_faces - 1))
 * floats: min xyz, max xyz. */
int reyn_mesh_tree(const reyn_mesh* mesh, uint32_t* order, uint32_t* children_l,
    uint32_t* children_r, float* leaf_box, float* node_box, void* stream);
/* LBVH::project (lbvh.cuh:521-561, 726-741): each of the n points (device
 * arrays) moves to the closest point of the mesh */
int reyn_mesh_project(const reyn_mesh* mesh, float* x, float* y, float* z,
    uint32_t n, void* stream);
/* InsidePredicate (scene.cu:84-139): inside[i] = 1 when the step from point
 * i to the closest point of the mesh runs along that face's normal
 * (dot >= 0), i.e. i lies inside an outward-wound closed mesh. The
 * reference's predicate returns the negation (the points its remove_if
 * drops). */
int reyn_mesh_inside(const reyn_mesh* mesh, const float* x, const float* y,
    const float* z, uint32_t n, uint8_t* inside, void* stream);
/* uniform_sample_mesh (sample_boundary.cu:299-389): ceil(area / (1.5 sqrt(3)
 * h_bdy^2)) samples, h_bdy = h / oversampling, stratified along the summed
 * face areas and uniform inside each triangle. The random numbers are
 * counter-based (SplitMix64 of the seed and the sample index) instead of the
 * reference's curand Philox. *count receives the sample count; x == NULL is
 * a size query. */
int reyn_mesh_sample_uniform(const reyn_mesh* mesh, float h, float oversampling,
    uint64_t seed, float* x, float* y, float* z, uint32_t capacity,
    uint32_t* count, void* stream);
/* relax_sampling (sample_boundary.cu:100-166): `iters` sweeps that move every
 * sample down the gradient of its number density (B3 at support 2 h_bdy,
 * against the rest density of a hexagonal plane sampling), scaled by
 * relaxation_factor h_bdy^2, then back onto the mesh. Each sweep reads the
 * previous positions of all samples. The samples keep their order. stats
 * (host, may be NULL) receives per sweep the max/min number-density ratio and
 * the average number density; num_den (device, may be NULL) the number
 * densities of the last sweep. The mesh keeps the relaxation's grid (cell
 * 2 h_bdy over its box) and scratch for the next call until it is
 * destroyed. Synchronises the stream. */
int reyn_mesh_relax(const reyn_mesh* mesh, float* x, float* y, float* z,
    uint32_t n, float h_bdy, float relaxation_factor, uint32_t iters,
    float* stats, float* num_den, void* stream);
/* Scene::from_obj's fluid volume (scene.cu:336-425): lattice points of
 * spacing h over the mesh's bounds (x fastest), kept when inside, in lattice
 * order, each coordinate then moved by a uniform [-jitter h, jitter h]
 * (counter-based streams keyed by the lattice index). *count receives the
 * number kept; x == NULL is a size query. Synchronises the stream. */
int reyn_mesh_fill(const reyn_mesh* mesh, float h, float jitter, uint64_t seed,
    float* x, float* y, float* z, uint32_t capacity, uint32_t* count,
    void* stream);

/* ---- launch accounting (no counterpart in the reference, which has no
 * tracing): per-kernel launch counts and CUDA-event device time ----------- */
typedef struct reyn_profile_entry {
    char name[48];     /* kernel name */
    uint64_t launches; /* launches since the last reset */
    double total_ms;   /* summed device time while timing was enabled */
} reyn_profile_entry;

/* on != 0: bracket every engine kernel launch with CUDA events on its
 * stream (launches are always counted) */
int reyn_profile_enable(int on);
int reyn_profile_reset(void);
/* per-kernel totals; synchronises on the recorded events. Writes at most
 * cap entries to out (may be NULL) and the number of kernels to *count. */
int reyn_profile_read(reyn_profile_entry* out, uint32_t cap, uint32_t* count);

#ifdef __cplusplus
}
#endif

#endif /* REYN_B200_H_ */
