/* CPU ORACLE — test infrastructure only.
 *
 * A host C++/OpenMP restatement of the reference's (reyn) SPH hot path, used
 * as the checker for the CUDA engine in tests/, by __graft_entry__.smoke() and
 * as bench.py's CPU baseline. It is never linked into, loaded by or called
 * from the product (reyn_b200/). Every function cites the reference file:line
 * it restates. Parity of this oracle is pinned against the reference itself:
 * kernel values against the reference's own kernel classes compiled for the
 * host (oracle/ref/ref_kernels_host.cpp), grid and solver outputs against the
 * reference's CUDA code run on a B200 (fixtures in tests/golden/).
 *
 * Conventions: all arrays are host SoA arrays; status 0 = ok, < 0 = error.
 * The sort inside each grid cell is STABLE (ascending particle index), i.e.
 * the canonical form of the reference's atomicSub order (uniformgrid.cu:59).
 */
#ifndef REYN_ORACLE_H_
#define REYN_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* grid geometry, restating UniformGridBuilder's initializer list
 * (uniformgrid.cu:65-96); cell_ratio 0.5 is the reference geometry. */
typedef struct orc_geom {
    float bmin[3]; /* lower bound minus the 2r safety margin */
    float cell;    /* cell size */
    float r2;      /* squared search radius */
    int32_t nx, ny, nz;
    int32_t range; /* cells searched on each side: 2 at cell r/2, 1 at r */
    int32_t order; /* 0: XYZ keys (the reference's); 1: the engine's Z-order */
} orc_geom;

int orc_geometry(const float bmin[3], const float bmax[3], float r,
    float cell_ratio, orc_geom* g);
/* the same geometry with cell order `order`; orc_keys() gives the size of
 * its key space (prefix arrays hold orc_keys + 1 entries) */
int orc_geometry_order(const float bmin[3], const float bmax[3], float r,
    float cell_ratio, int order, orc_geom* g);
int64_t orc_keys(const orc_geom* g);

/* W(dx) and ∇W(dx) of kernel `kind` (0 C2, 1 B3, 2 W6, 3 COS) with support
 * h_bar, kernels.cuh:19-165 (host flavour: norm = sqrt(dot)). */
int orc_kernel_eval(int kind, float h_bar, uint32_t n, const float* dx,
    const float* dy, const float* dz, float* w, float* gx, float* gy,
    float* gz);

/* counting-sort grid build (uniformgrid.cu:20-63, 98-143), stable within a
 * cell. prefix: orc_keys + 1 entries (exclusive scan, last = N);
 * sorted: N particle indices; keys (optional): N cell keys. */
int orc_grid_build(const orc_geom* g, uint32_t n, const float* x,
    const float* y, const float* z, uint32_t* prefix, uint32_t* sorted,
    uint32_t* keys);

/* the grid test's neighbour count (self excluded) and Σ|x_ij|² over the
 * `ff_nbrs` traversal (uniformgrid.cu:185-207, uniformgrid.cuh:113-178),
 * plus the fluid density Σ m_j W(x_ij) (solver.cuh:31-33) when m != NULL. */
int orc_neighbours(const orc_geom* g, uint32_t n, const float* x,
    const float* y, const float* z, const uint32_t* prefix,
    const uint32_t* sorted, uint32_t* count, float* len2, int kind,
    const float* m, float* rho);

/* brute-force O(N^2) neighbour count (uniformgrid.cu:209-229) */
int orc_brute_count(uint32_t n, const float* x, const float* y,
    const float* z, float r, uint32_t* count, float* len2);

/* Akinci boundary masses (sample_boundary.cu:250-297): B3 at support 2h,
 * m0 = 1, `iters` refinements m_i <- rho0 m_i / Σ_j m_j W_ij. The reference
 * updates m in place while neighbours read it (a data race); this oracle uses
 * a double-buffered (Jacobi) update. Positions are given in any order. */
int orc_boundary_masses(uint32_t nb, const float* bx, const float* by,
    const float* bz, float h, float rho0, uint32_t iters, float* m);

/* the same refinement with smoothing kernel `kind` instead of B3 */
int orc_boundary_masses_kernel(uint32_t nb, const float* bx, const float* by,
    const float* bz, float h, float rho0, uint32_t iters, int kind, float* m);

/* cfl_time_step (cfl.cu:5-37) */
float orc_cfl(uint32_t n, const float* vx, const float* vy, const float* vz,
    float lambda, float h, const float g[3]);

/* simple_dt_controller (cfl.cu:39-52) */
float orc_dt_controller(uint32_t iter_last, float dt_last, float lambda,
    float h, uint32_t n, const float* vx, const float* vy, const float* vz,
    const float g[3], uint32_t iter_target, float change_factor);

/* solver parameters; orc_params_reference() gives the reference's hard-coded
 * constants (SESPH.cuh:50, PCISPH.cuh:27-38, IISPH.cuh:37-48). */
typedef struct orc_params {
    int scheme;         /* 0 SESPH, 1 PCISPH, 2 IISPH */
    int kind;           /* smoothing kernel, support 2h */
    float h, rho0, nu;
    float g[3];
    float k_sesph;      /* SESPH stiffness */
    float eta;          /* PCISPH: avg rho tolerance; IISPH: per-particle */
    uint32_t min_iter;
    uint32_t max_iter;  /* 0 = unbounded (reference) */
    float omega;        /* IISPH Jacobi weight */
    int warmstart;      /* IISPH: p *= 0.5 at step start */
    int iisph_avg;      /* IISPH: stop on average error <= eta instead of
                           "no particle above eta" (reference) */
    float cell_ratio;   /* 0.5 = reference */
    int projected;      /* IISPH: p = max(0, p + delta) instead of the
                           reference's p += max(0, delta) */
} orc_params;

void orc_params_reference(int scheme, int kind, float h, float rho0,
    float nu, orc_params* p);

/* `steps` iterations of the reference main loop (main.cu:60-78): grid build
 * + reorder of the state, id and (IISPH) pressure at 2h (scene.cuh:149-156),
 * solver step, hard_enforce_bounds (scene.cu:466-491), with a fixed dt.
 * State arrays are updated in place and left in the last grid order; solver
 * buffers after the last step go to rho/p/aii/sii/ax/ay/az (may be NULL);
 * iters[k] receives the iteration count of step k; p must hold the pressure
 * to warm-start from (zeros on the first step, like the reference). */
int orc_run(const orc_params* prm, uint32_t n, float* x, float* y, float* z,
    float* vx, float* vy, float* vz, float* m, float* id, float* p,
    uint32_t nb, const float* bx, const float* by, const float* bz,
    const float* bm, const float scene_min[3], const float scene_max[3],
    float dt, uint32_t steps, float* rho, float* aii, float* sii, float* ax,
    float* ay, float* az, uint32_t* iters);

/* number of OpenMP threads the oracle uses */
int orc_threads(void);


/* ---- triangle meshes (scene/sample_boundary.cu, datastructure/lbvh.cuh) ----
 * A mesh is nv double vertices (vx, vy, vz) and nf triangles (faces: 3 vertex
 * indices each). Boxes are 6 floats (min xyz, max xyz). */

/* 30-bit Morton code of each face centroid in the vertex bounds
 * (lbvh.cuh:17-45, 204-225) */
int orc_mesh_morton(const double* vx, const double* vy, const double* vz,
    uint32_t nv, const uint32_t* faces, uint32_t nf, uint32_t* codes);

/* the LBVH (lbvh.cuh:646-723, lbvh.cu:34-170): order[j] = original face of
 * leaf j (faces stably sorted by code); children in the ChildNode encoding
 * (index << 1 | 1 for an internal node, lbvh.cuh:162-193), nf - 1 each; leaf
 * and internal boxes; height = edges from the root to the deepest leaf.
 * Any output may be NULL. */
int orc_lbvh_build(const double* vx, const double* vy, const double* vz,
    uint32_t nv, const uint32_t* faces, uint32_t nf, uint32_t* order,
    uint32_t* children_l, uint32_t* children_r, float* leaf_box,
    float* node_box, uint32_t* height);

/* LBVH queries over n points: inside == NULL projects them in place onto
 * the closest point of the mesh (LBVH::project, lbvh.cuh:415-561); else
 * inside[i] = 1 when the step from point i to its closest point runs along
 * that face's normal (the negation of InsidePredicate, scene.cu:84-139,
 * which marks the points to remove) and the points are unchanged. */
int orc_lbvh_query(const double* vx, const double* vy, const double* vz,
    uint32_t nv, const uint32_t* faces, uint32_t nf, uint32_t n, float* x,
    float* y, float* z, uint8_t* inside);

/* the brute-force projection of the reference's LBVH test (lbvh.cu:276-306) */
int orc_project_brute(const double* vx, const double* vy, const double* vz,
    uint32_t nv, const uint32_t* faces, uint32_t nf, uint32_t n, float* x,
    float* y, float* z);

/* total area, |signed volume| and (optional, nf entries) the inclusive sum of
 * face areas (sample_boundary.cu:311-330, sample_boundary.cuh:40-60) */
int orc_mesh_measure(const double* vx, const double* vy, const double* vz,
    uint32_t nv, const uint32_t* faces, uint32_t nf, double* area,
    double* volume, double* cdf);

/* number of boundary samples for spacing h / oversampling
 * (sample_boundary.cu:339-346) */
uint32_t orc_mesh_sample_count(double area, float h, float oversampling);

/* area-stratified uniform samples (sample_boundary.cu:168-248, 299-389) with
 * the engine's counter-based random streams (SplitMix64: stream 8 the offset
 * inside the stratum, streams 9 and 10 the barycentric pair, each in (0, 1]
 * with 53 bits). x == NULL: count only. */
int orc_mesh_sample(const double* vx, const double* vy, const double* vz,
    uint32_t nv, const uint32_t* faces, uint32_t nf, float h,
    float oversampling, uint64_t seed, uint32_t cap, float* x, float* y,
    float* z, uint32_t* count);

/* rest number density of a hexagonal plane sampling (sample_boundary.cu:78-98) */
float orc_hex_plane_density(float h_bdy);

/* one relaxation sweep (sample_boundary.cu:20-71, 134-147) over all sample
 * pairs: number densities (out: num_den), the shift down their gradient
 * from the old positions (the reference shifts in place while neighbours
 * read, a data race), then the projection back onto the mesh */
int orc_mesh_relax_sweep(const double* vx, const double* vy, const double* vz,
    uint32_t nv, const uint32_t* faces, uint32_t nf, uint32_t n, float* x,
    float* y, float* z, float h_bdy, float k, float* num_den);

/* the fluid fill of Scene::from_obj (scene.cu:336-425): lattice points of
 * spacing h over the mesh's float bounds (x fastest) kept when inside, in
 * lattice order, optionally jittered by a uniform [-jitter h, jitter h] per
 * axis (streams 0..2 keyed by the lattice index). x == NULL: count only. */
int orc_mesh_fill(const double* vx, const double* vy, const double* vz,
    uint32_t nv, const uint32_t* faces, uint32_t nf, float h, float jitter,
    uint64_t seed, uint32_t cap, float* x, float* y, float* z,
    uint32_t* count);

#ifdef __cplusplus
}
#endif

#endif
