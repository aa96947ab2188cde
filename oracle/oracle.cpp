// CPU ORACLE — test infrastructure only (see oracle.h). A host C++/OpenMP
// restatement of the reference's (reyn) SPH hot path. Each function names the
// reference file:line it follows. Arithmetic types follow the reference
// expression by expression (float, with the double sub-expressions where the
// reference writes double literals) so that per-pair values match the
// reference's host flavour bit for bit; build with -ffp-contract=off.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {

#include "oracle_kernels.hpp"

// ---- uniform grid, uniformgrid.cuh:17-64/84-178, uniformgrid.cu:20-143 ----

struct Grid {
    orc_geom g;
    std::vector<uint32_t> prefix; // C + 1
    std::vector<uint32_t> sorted; // N (identity after a reorder)
    bool identity = false;
};

inline int cell_coord(float p, float lo, float cell)
{
    return (int)std::floor((p - lo) / cell); // floor_div, vector.cuh:137-141
}

// The engine's Z-order (no counterpart in the reference): 4x4x4-cell
// bricks, x fastest inside a brick; bricks numbered along the Morton curve
// inside 32x32x32-cell tiles (bit k of the brick's x, y, z index goes to bit
// 3k, 3k+1, 3k+2); tiles in XYZ order. key = (tile * 512 + brick) * 64 + cell.
inline int ztiles(int n) { return (n + 31) / 32; }

inline int64_t zorder_key(const orc_geom& g, int cx, int cy, int cz)
{
    const int64_t tx = ztiles(g.nx), ty = ztiles(g.ny);
    const int64_t tile = ((int64_t)(cz / 32) * ty + cy / 32) * tx + cx / 32;
    int64_t brick = 0;
    const int b[3] = { (cx / 4) % 8, (cy / 4) % 8, (cz / 4) % 8 };
    for (int bit = 0; bit < 3; ++bit)
        for (int a = 0; a < 3; ++a)
            brick |= (int64_t)((b[a] >> bit) & 1) << (3 * bit + a);
    const int64_t cell = (cx % 4) + 4 * (cy % 4) + 16 * (cz % 4);
    return (tile * 512 + brick) * 64 + cell;
}

inline int64_t cell_key(const orc_geom& g, int cx, int cy, int cz)
{
    if (g.order == 1)
        return zorder_key(g, cx, cy, cz);
    // _linearize, uniformgrid.cuh:33-40
    return (int64_t)cz * ((int64_t)g.nx * g.ny) + ((int64_t)cy * g.nx + cx);
}

inline int64_t n_keys(const orc_geom& g)
{
    if (g.order == 1)
        return (int64_t)ztiles(g.nx) * ztiles(g.ny) * ztiles(g.nz) * 32768;
    return (int64_t)g.nx * g.ny * g.nz;
}

inline int64_t linear_key(const orc_geom& g, float x, float y, float z)
{
    const int cx = cell_coord(x, g.bmin[0], g.cell);
    const int cy = cell_coord(y, g.bmin[1], g.cell);
    const int cz = cell_coord(z, g.bmin[2], g.cell);
    if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nx || cy >= g.ny || cz >= g.nz)
        return -1;
    return cell_key(g, cx, cy, cz);
}

int build(const orc_geom& g, uint32_t n, const float* x, const float* y,
    const float* z, Grid& out, uint32_t* keys_out)
{
    out.g = g;
    const int64_t C = n_keys(g);
    std::vector<uint32_t> keys(n);
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(+ : bad)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const int64_t k = linear_key(g, x[i], y[i], z[i]);
        if (k < 0)
            bad += 1;
        keys[i] = (uint32_t)(k < 0 ? 0 : k);
    }
    if (bad)
        return -2;
    // _count_particles_per_cell + exclusive_scan (uniformgrid.cu:115-134)
    out.prefix.assign(C + 1, 0);
    for (uint32_t i = 0; i < n; ++i)
        out.prefix[keys[i] + 1] += 1;
    for (int64_t c = 0; c < C; ++c)
        out.prefix[c + 1] += out.prefix[c];
    // _counting_sort (uniformgrid.cu:40-63), stable: slots in index order
    std::vector<uint32_t> fill(out.prefix.begin(), out.prefix.end() - 1);
    out.sorted.assign(n, 0);
    for (uint32_t i = 0; i < n; ++i)
        out.sorted[fill[keys[i]]++] = i;
    out.identity = false;
    if (keys_out)
        std::memcpy(keys_out, keys.data(), sizeof(uint32_t) * n);
    return 0;
}

// UniformGrid::ff_nbrs, uniformgrid.cuh:113-178: for each of the
// (2 range + 1)^2 (y,z) rows, one contiguous run of 2 range + 1 x-cells.
template <class Acc, class Map>
inline Acc ff_nbrs(const Grid& G, f3 xi, const float* x, const float* y,
    const float* z, Map map, Acc acc)
{
    const orc_geom& g = G.g;
    const int cx = cell_coord(xi.x, g.bmin[0], g.cell);
    const int cy = cell_coord(xi.y, g.bmin[1], g.cell);
    const int cz = cell_coord(xi.z, g.bmin[2], g.cell);
    const int R = g.range;
    const int64_t nxny = (int64_t)g.nx * g.ny;
    auto visit = [&](int64_t k0, int64_t k1) {
        for (uint32_t j = G.prefix[k0]; j < G.prefix[k1]; ++j) {
            const uint32_t sj = G.identity ? j : G.sorted[j];
            const f3 xij = xi - load(sj, x, y, z);
            const float l2 = dot(xij, xij);
            if (l2 <= g.r2)
                acc += map(sj, xij, l2);
        }
    };
    for (int zz = cz - R; zz <= cz + R; ++zz)
        for (int yy = cy - R; yy <= cy + R; ++yy) {
            if (g.order == 1) { // Z-order: cell by cell
                for (int xx = cx - R; xx <= cx + R; ++xx) {
                    const int64_t k = zorder_key(g, xx, yy, zz);
                    visit(k, k + 1);
                }
            } else {
                const int64_t cid = (int64_t)zz * nxny + ((int64_t)yy * g.nx + (cx - R));
                visit(cid, cid + (2 * R + 1));
            }
        }
    return acc;
}

// gather of an array by `sorted` (buffer.cuh:184-209)
void gather(float* a, const std::vector<uint32_t>& sorted, std::vector<float>& tmp)
{
    const size_t n = sorted.size();
    tmp.resize(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i)
        tmp[i] = a[sorted[i]];
    std::memcpy(a, tmp.data(), n * sizeof(float));
}

struct Bdy {
    Grid grid;
    std::vector<float> x, y, z, m;
    bool empty = true;
};

// boundary grid over the samples' own bounds at 2h, reordered
// (sample_boundary.cu:413-428)
int make_bdy(uint32_t nb, const float* bx, const float* by, const float* bz,
    const float* bm, float h, float cell_ratio, Bdy& b)
{
    b.empty = (nb == 0);
    if (nb == 0)
        return 0;
    float lo[3] = { bx[0], by[0], bz[0] }, hi[3] = { bx[0], by[0], bz[0] };
    for (uint32_t i = 0; i < nb; ++i) {
        lo[0] = std::min(lo[0], bx[i]);
        lo[1] = std::min(lo[1], by[i]);
        lo[2] = std::min(lo[2], bz[i]);
        hi[0] = std::max(hi[0], bx[i]);
        hi[1] = std::max(hi[1], by[i]);
        hi[2] = std::max(hi[2], bz[i]);
    }
    orc_geom g;
    if (orc_geometry(lo, hi, 2.f * h, cell_ratio, &g))
        return -1;
    if (int e = build(g, nb, bx, by, bz, b.grid, nullptr))
        return e;
    b.x.resize(nb);
    b.y.resize(nb);
    b.z.resize(nb);
    b.m.resize(nb);
    for (uint32_t i = 0; i < nb; ++i) {
        const uint32_t s = b.grid.sorted[i];
        b.x[i] = bx[s];
        b.y[i] = by[s];
        b.z[i] = bz[s];
        b.m[i] = bm ? bm[s] : 1.f;
    }
    b.grid.identity = true;
    return 0;
}

// Σ_k m_k (map) over boundary neighbours; a zero accumulator when there is no
// boundary (the fluid grid still bounds the query)
template <class Acc, class Map>
inline Acc bdy_nbrs(const Bdy& b, f3 xi, Map map, Acc acc)
{
    if (b.empty)
        return acc;
    // the fluid may lie outside the boundary grid; such queries see nothing
    const orc_geom& g = b.grid.g;
    const int cx = cell_coord(xi.x, g.bmin[0], g.cell);
    const int cy = cell_coord(xi.y, g.bmin[1], g.cell);
    const int cz = cell_coord(xi.z, g.bmin[2], g.cell);
    if (cx - g.range < 0 || cy - g.range < 0 || cz - g.range < 0
        || cx + g.range + 1 >= g.nx || cy + g.range >= g.ny
        || cz + g.range >= g.nz)
        return acc;
    return ff_nbrs(b.grid, xi, b.x.data(), b.y.data(), b.z.data(), map, acc);
}

// ---- solvers -------------------------------------------------------------

struct State {
    uint32_t n;
    float *x, *y, *z, *vx, *vy, *vz, *m;
};

// compute_densities, solver.cuh:18-38
template <class K>
void densities(const K& Wk, const State& s, const Grid& G, const Bdy& b,
    float* rho)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 xi = load(i, s.x, s.y, s.z);
        rho[i] = ff_nbrs(G, xi, s.x, s.y, s.z,
                     [&](uint32_t j, f3 xij, float) { return s.m[j] * W(Wk, xij); },
                     0.f)
            + bdy_nbrs(b, xi,
                [&](uint32_t j, f3 xij, float) { return b.m[j] * W(Wk, xij); },
                0.f);
    }
}

// the artificial viscosity term of solver.cuh:62-63 / SESPH.cu:259-260:
// float prefix / (double denominator), narrowed to float, times ∇W
inline float visc_scale(float nu, float mj, float rhoj, f3 vij, f3 xij, float h)
{
    const float num = 10.f * nu * mj / rhoj * dot(vij, xij);
    return (float)((double)num / ((double)dot(xij, xij) + 0.01 * h * h));
}

// write_non_prs_acc_ff, solver.cuh:40-69
template <class K>
void non_pressure_acc(const K& Wk, const State& s, const Grid& G,
    const float* rho, float h, float nu, f3 g, float* ax, float* ay, float* az)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 xi = load(i, s.x, s.y, s.z);
        const f3 vi = load(i, s.vx, s.vy, s.vz);
        const f3 a = ff_nbrs(G, xi, s.x, s.y, s.z,
            [&](uint32_t j, f3 xij, float) {
                const f3 vij = vi - load(j, s.vx, s.vy, s.vz);
                return visc_scale(nu, s.m[j], rho[j], vij, xij, h) * dW(Wk, xij);
            },
            g);
        store(a, i, ax, ay, az);
    }
}

// integrate_a_v_only, solver.cu:3-13
void integrate_v(const State& s, const float* ax, const float* ay,
    const float* az, float dt)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 v = load(i, s.vx, s.vy, s.vz);
        store(v + dt * load(i, ax, ay, az), i, s.vx, s.vy, s.vz);
    }
}

// integrate, solver.cu:15-32
void integrate(const State& s, const float* ax, const float* ay,
    const float* az, float dt)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 a = load(i, ax, ay, az);
        const f3 v = load(i, s.vx, s.vy, s.vz);
        const f3 x = load(i, s.x, s.y, s.z);
        const f3 vn = v + dt * a;
        store(vn, i, s.vx, s.vy, s.vz);
        store(x + dt * vn, i, s.x, s.y, s.z);
    }
}

// eos, SESPH.cu:6-12
inline float eos_sesph(float rho, float k, float rho0)
{
    return std::fmax(0.f, k * (rho / rho0 - 1.f));
}

// _compute_accelerations, SESPH.cu:15-65
template <class K>
void sesph_acc(const K& Wk, const State& s, const Grid& G, const Bdy& b,
    const float* rho, float k, float rho0, float nu, float h, f3 g, float* ax,
    float* ay, float* az)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 xi = load(i, s.x, s.y, s.z);
        const f3 vi = load(i, s.vx, s.vy, s.vz);
        const float rhoi = rho[i];
        const float pi = eos_sesph(rhoi, k, rho0);
        const float pr = pi / (rhoi * rhoi);
        const f3 af = ff_nbrs(G, xi, s.x, s.y, s.z,
            [&](uint32_t j, f3 xij, float) {
                const float rhoj = rho[j];
                const float mj = s.m[j];
                const f3 vij = vi - load(j, s.vx, s.vy, s.vz);
                const f3 dw = dW(Wk, xij);
                const float pj = eos_sesph(rhoj, k, rho0);
                const f3 visc = visc_scale(nu, mj, rhoj, vij, xij, h) * dw;
                return visc - (mj * (pr + pj / (rhoj * rhoj))) * dw;
            },
            g);
        const f3 ab = bdy_nbrs(b, xi,
            [&](uint32_t j, f3 xij, float) { return b.m[j] * dW(Wk, xij); },
            mk(0, 0, 0));
        store(af - pr * ab, i, ax, ay, az);
    }
}

// k_c_pcisph, PCISPH.cuh:49-77 (host evaluation of ∇W on a 5^3 lattice)
template <class K> double pcisph_delta(const K& Wk, double h)
{
    const float hf = (float)h;
    f3 sum = mk(0, 0, 0);
    double sum_of_sq = 0.;
    for (int x = -2; x <= 2; ++x)
        for (int y = -2; y <= 2; ++y)
            for (int z = -2; z <= 2; ++z) {
                const f3 xj = mk((float)x * hf, (float)y * hf, (float)z * hf);
                const f3 d = dW(Wk, -xj);
                sum += d;
                sum_of_sq += (double)dot(d, d);
            }
    const double sq_of_sum = (double)dot(sum, sum);
    const double V0 = h * h * h;
    const double beta = 2. * V0 * V0;
    return (double)(float)(1. / (beta * (sq_of_sum + sum_of_sq)));
}

// predict_rho, solver.cuh:71-105
template <class K>
void predict_rho(const K& Wk, const State& s, const Grid& G, const Bdy& b,
    float dt, float* rho)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 xi = load(i, s.x, s.y, s.z);
        const f3 vi = load(i, s.vx, s.vy, s.vz);
        rho[i] = ff_nbrs(G, xi, s.x, s.y, s.z,
                     [&](uint32_t j, f3 xij, float) {
                         const f3 vij = vi - load(j, s.vx, s.vy, s.vz);
                         return s.m[j] * (W(Wk, xij) + dt * dot(dW(Wk, xij), vij));
                     },
                     0.f)
            + bdy_nbrs(b, xi,
                [&](uint32_t j, f3 xij, float) {
                    return b.m[j] * (W(Wk, xij) + dt * dot(dW(Wk, xij), vi));
                },
                0.f);
    }
}

// _write_pcisph_prs_acc, PCISPH.cu:21-56
template <class K>
void pcisph_acc(const K& Wk, const State& s, const Grid& G, const Bdy& b,
    const float* rho, float k, float rho0, float* ax, float* ay, float* az)
{
    const float r0i = 1.f / (rho0 * rho0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 xi = load(i, s.x, s.y, s.z);
        const float rhoi = rho[i];
        const float pi = std::fmax(0.f, k * (rhoi - rho0));
        const float pr = pi / (rhoi * rhoi);
        const float p0 = pi * r0i;
        const f3 af = ff_nbrs(G, xi, s.x, s.y, s.z,
            [&](uint32_t j, f3 xij, float) {
                const float rhoj = rho[j];
                const float pj = std::fmax(0.f, k * (rhoj - rho0));
                return (s.m[j] * (pr + pj / (rhoj * rhoj))) * dW(Wk, xij);
            },
            mk(0, 0, 0));
        const f3 ab = bdy_nbrs(b, xi,
            [&](uint32_t j, f3 xij, float) { return b.m[j] * dW(Wk, xij); },
            mk(0, 0, 0));
        const float c = (float)(0.5 * (double)(pr + p0));
        store(-af - c * ab, i, ax, ay, az);
    }
}

// _compute_diagonal_elem_and_source_term, IISPH.cu:11-66
template <class K>
void iisph_diag(const K& Wk, const State& s, const Grid& G, const Bdy& b,
    const float* rho, float rho0, float dt, float* aii, float* sii)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 xi = load(i, s.x, s.y, s.z);
        const f3 vi = load(i, s.vx, s.vy, s.vz);
        float vel_div = 0.f, gsq = 0.f;
        const f3 gff = ff_nbrs(G, xi, s.x, s.y, s.z,
            [&](uint32_t j, f3 xij, float) {
                const f3 d = dW(Wk, xij);
                const f3 md = s.m[j] * d;
                vel_div += dot(md, vi - load(j, s.vx, s.vy, s.vz));
                gsq += dot(md, d);
                return md;
            },
            mk(0, 0, 0));
        const f3 gb = bdy_nbrs(b, xi,
            [&](uint32_t j, f3 xij, float) { return b.m[j] * dW(Wk, xij); },
            mk(0, 0, 0));
        const f3 grad = gff + gb;
        const float gss = dot(grad, grad);
        const float sgs = s.m[i] * gsq;
        aii[i] = -dt * (gss + sgs) / (rho0 * rho0);
        const float div = vel_div + dot(vi, gb);
        sii[i] = (rho0 - rho[i]) / dt - div;
    }
}

// _set_pressure_accelerations, IISPH.cu:68-98
template <class K>
void iisph_pacc(const K& Wk, const State& s, const Grid& G, const Bdy& b,
    const float* p, float r0i, float* ax, float* ay, float* az)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 xi = load(i, s.x, s.y, s.z);
        const float pi = p[i];
        const f3 af = ff_nbrs(G, xi, s.x, s.y, s.z,
            [&](uint32_t j, f3 xij, float) {
                return (s.m[j] * (pi + p[j])) * dW(Wk, xij);
            },
            mk(0, 0, 0));
        const f3 ab = bdy_nbrs(b, xi,
            [&](uint32_t j, f3 xij, float) { return b.m[j] * dW(Wk, xij); },
            mk(0, 0, 0));
        store((-r0i) * (af + pi * ab), i, ax, ay, az);
    }
}

// jacobi_update, IISPH.cu:108-117
inline float jacobi(float omega, float a_ii, float Ap, float s)
{
    return ((double)a_ii < 1e-6 && (double)a_ii > -1e-6)
        ? 0.f
        : std::fmax(0.f, omega * (s - Ap) / a_ii);
}

// _jacobi_update_pressures, IISPH.cu:119-162; returns the number of
// particles whose predicted density error exceeds `thr` and accumulates
// Σ max(0, err) into *err_sum (for the average-error criterion)
template <class K>
uint64_t iisph_jacobi(const K& Wk, const State& s, const Grid& G,
    const Bdy& b, const float* ax, const float* ay, const float* az,
    float* p, const float* aii, const float* sii, float dt, float omega,
    float thr, double* err_sum, int projected)
{
    uint64_t over = 0;
    double es = 0.;
    // Jacobi: every Ap_i reads a (not p), so p can be updated in place
#pragma omp parallel for schedule(static) reduction(+ : over, es)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 xi = load(i, s.x, s.y, s.z);
        const f3 ai = load(i, ax, ay, az);
        const float ff = ff_nbrs(G, xi, s.x, s.y, s.z,
            [&](uint32_t j, f3 xij, float) {
                const f3 aij = ai - load(j, ax, ay, az);
                return s.m[j] * dot(aij, dW(Wk, xij));
            },
            0.f);
        const f3 gb = bdy_nbrs(b, xi,
            [&](uint32_t j, f3 xij, float) { return b.m[j] * dW(Wk, xij); },
            mk(0, 0, 0));
        const float Ap = dt * (ff + dot(ai, gb));
        const float si = sii[i];
        if (projected) {
            const float a = aii[i];
            p[i] = ((double)a < 1e-6 && (double)a > -1e-6)
                ? p[i]
                : std::fmax(0.f, p[i] + omega * (si - Ap) / a);
        } else {
            p[i] = p[i] + jacobi(omega, aii[i], Ap, si);
        }
        const float err = (Ap - si) * dt;
        over += (err > thr) ? 1 : 0;
        es += std::max(0.0, (double)err);
    }
    *err_sum = es;
    return over;
}

// hard_enforce_bounds, scene.cu:466-483
void enforce_bounds(const State& s, const float* lo, const float* hi)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)s.n; ++i) {
        const f3 x = load(i, s.x, s.y, s.z);
        const bool touch = (x.x <= lo[0]) || (x.y <= lo[1]) || (x.z <= lo[2])
            || (hi[0] <= x.x) || (hi[1] <= x.y) || (hi[2] <= x.z);
        if (touch) {
            const f3 v = load(i, s.vx, s.vy, s.vz);
            store((float)-0.1 * v, i, s.vx, s.vy, s.vz);
        }
        store(mk(std::fmax(std::fmin(x.x, hi[0]), lo[0]),
                  std::fmax(std::fmin(x.y, hi[1]), lo[1]),
                  std::fmax(std::fmin(x.z, hi[2]), lo[2])),
            i, s.x, s.y, s.z);
    }
}

} // namespace

extern "C" {

int orc_threads(void) { return omp_get_max_threads(); }

int orc_geometry(const float bmin[3], const float bmax[3], float r,
    float cell_ratio, orc_geom* g)
{
    if (!(r > 0.f) || !(cell_ratio == 0.5f || cell_ratio == 1.0f))
        return -1;
    // uniformgrid.cu:69-80: cell = r/2, min' = min - 2r,
    // n = ceil(((max + 2r) - min') / cell)
    const float cell = cell_ratio == 0.5f ? r / 2.f : r;
    const float margin = (float)(r * 2.);
    int n[3];
    for (int a = 0; a < 3; ++a) {
        g->bmin[a] = bmin[a] - margin;
        n[a] = (int)std::ceil(((bmax[a] + margin) - g->bmin[a]) / cell);
        if (n[a] <= 0)
            return -1;
    }
    g->cell = cell;
    g->r2 = r * r;
    g->nx = n[0];
    g->ny = n[1];
    g->nz = n[2];
    g->range = cell_ratio == 0.5f ? 2 : 1;
    g->order = 0;
    return 0;
}

int orc_geometry_order(const float bmin[3], const float bmax[3], float r,
    float cell_ratio, int order, orc_geom* g)
{
    if (order != 0 && order != 1)
        return -1;
    if (int e = orc_geometry(bmin, bmax, r, cell_ratio, g))
        return e;
    g->order = order;
    return 0;
}

int64_t orc_keys(const orc_geom* g) { return n_keys(*g); }

int orc_kernel_eval(int kind, float h_bar, uint32_t n, const float* dx,
    const float* dy, const float* dz, float* w, float* gx, float* gy,
    float* gz)
{
    return with_kernel(kind, h_bar, [&](auto Wk) {
        for (uint32_t i = 0; i < n; ++i) {
            const f3 d = mk(dx[i], dy[i], dz[i]);
            w[i] = W(Wk, d);
            const f3 g = dW(Wk, d);
            gx[i] = g.x;
            gy[i] = g.y;
            gz[i] = g.z;
        }
    });
}

int orc_grid_build(const orc_geom* g, uint32_t n, const float* x,
    const float* y, const float* z, uint32_t* prefix, uint32_t* sorted,
    uint32_t* keys)
{
    Grid G;
    if (int e = build(*g, n, x, y, z, G, keys))
        return e;
    std::memcpy(prefix, G.prefix.data(), G.prefix.size() * sizeof(uint32_t));
    std::memcpy(sorted, G.sorted.data(), n * sizeof(uint32_t));
    return 0;
}

int orc_neighbours(const orc_geom* g, uint32_t n, const float* x,
    const float* y, const float* z, const uint32_t* prefix,
    const uint32_t* sorted, uint32_t* count, float* len2, int kind,
    const float* m, float* rho)
{
    Grid G;
    G.g = *g;
    const int64_t C = n_keys(*g);
    G.prefix.assign(prefix, prefix + C + 1);
    G.sorted.assign(sorted, sorted + n);
    const float r2 = g->r2;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const f3 xi = load(i, x, y, z);
        if (count)
            count[i] = ff_nbrs(G, xi, x, y, z,
                [&](uint32_t j, f3, float l2) {
                    return (l2 <= r2) ? (j == (uint32_t)i ? 0u : 1u) : 0u;
                },
                0u);
        if (len2)
            len2[i] = ff_nbrs(G, xi, x, y, z,
                [&](uint32_t, f3 xij, float l2) {
                    return (l2 <= r2) ? dot(xij, xij) : 0.f;
                },
                0.f);
    }
    if (m && rho) {
        const float r = std::sqrt(r2);
        return with_kernel(kind, r, [&](auto Wk) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < (int64_t)n; ++i) {
                const f3 xi = load(i, x, y, z);
                rho[i] = ff_nbrs(G, xi, x, y, z,
                    [&](uint32_t j, f3 xij, float) { return m[j] * W(Wk, xij); },
                    0.f);
            }
        });
    }
    return 0;
}

int orc_brute_count(uint32_t n, const float* x, const float* y,
    const float* z, float r, uint32_t* count, float* len2)
{
    const float r2 = r * r;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const f3 xi = load(i, x, y, z);
        uint32_t c = 0;
        float l = 0.f;
        for (uint32_t j = 0; j < n; ++j) {
            const f3 xij = xi - load(j, x, y, z);
            const float l2 = dot(xij, xij);
            if (l2 <= r2) {
                c += (j == (uint32_t)i) ? 0u : 1u;
                l += l2;
            }
        }
        count[i] = c;
        if (len2)
            len2[i] = l;
    }
    return 0;
}

int orc_boundary_masses_kernel(uint32_t nb, const float* bx, const float* by,
    const float* bz, float h, float rho0, uint32_t iters, int kind, float* m)
{
    if (iters == 0) // sample_boundary.cu:283-287
        return -1;
    Bdy b;
    if (int e = make_bdy(nb, bx, by, bz, nullptr, h, 0.5f, b))
        return e;
    std::vector<float> next(nb);
    const int st = with_kernel(kind, 2.f * h, [&](auto Wk) {
        for (uint32_t it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < (int64_t)nb; ++i) {
                const f3 xi = mk(b.x[i], b.y[i], b.z[i]);
                const float sum = ff_nbrs(b.grid, xi, b.x.data(), b.y.data(),
                    b.z.data(),
                    [&](uint32_t j, f3 xij, float) { return b.m[j] * W(Wk, xij); },
                    0.f);
                next[i] = rho0 * b.m[i] / sum;
            }
            b.m.swap(next);
        }
    });
    if (st)
        return st;
    // scatter back to the caller's order
    for (uint32_t i = 0; i < nb; ++i)
        m[b.grid.sorted[i]] = b.m[i];
    return 0;
}

int orc_boundary_masses(uint32_t nb, const float* bx, const float* by,
    const float* bz, float h, float rho0, uint32_t iters, float* m)
{
    // calculate_boundary_masses always refines with B3 (sample_boundary.cu:269)
    return orc_boundary_masses_kernel(nb, bx, by, bz, h, rho0, iters, 1, m);
}

float orc_cfl(uint32_t n, const float* vx, const float* vy, const float* vz,
    float lambda, float h, const float g[3])
{
    float vmax = 0.f;
#pragma omp parallel for schedule(static) reduction(max : vmax)
    for (int64_t i = 0; i < (int64_t)n; ++i)
        vmax = std::max(vmax, norm(load(i, vx, vy, vz)));
    const float dt_vel = lambda * h / vmax;
    const float dt_g
        = std::sqrt((float)(2. * lambda * h / (double)norm(mk(g[0], g[1], g[2]))));
    return std::fmin(dt_vel, dt_g);
}

float orc_dt_controller(uint32_t iter_last, float dt_last, float lambda,
    float h, uint32_t n, const float* vx, const float* vy, const float* vz,
    const float g[3], uint32_t iter_target, float change_factor)
{
    const float f = iter_last < iter_target ? 1.f + change_factor
                                            : 1.f - change_factor;
    const float suggested = dt_last * f;
    const float cfl = orc_cfl(n, vx, vy, vz, lambda, h, g);
    return std::min(cfl, suggested);
}

void orc_params_reference(int scheme, int kind, float h, float rho0,
    float nu, orc_params* p)
{
    std::memset(p, 0, sizeof(*p));
    p->scheme = scheme;
    p->kind = kind;
    p->h = h;
    p->rho0 = rho0;
    p->nu = nu;
    p->g[0] = 0.f; // gravity along -y: SESPH.cuh:41 default, PCISPH.cuh:27,
    p->g[1] = -9.81f; // IISPH.cuh:37
    p->g[2] = 0.f;
    p->k_sesph = 500.f; // SESPH.cuh:50
    p->eta = scheme == 1 ? 0.001f : 0.005f; // PCISPH.cuh:36, IISPH.cuh:41
    p->min_iter = 3; // PCISPH.cuh:38, IISPH.cuh:43
    p->max_iter = 0;
    p->omega = 0.5f; // IISPH.cuh:45
    p->warmstart = 1; // IISPH.cuh:48
    p->iisph_avg = 0;
    p->cell_ratio = 0.5f;
    p->projected = 0;
}

int orc_run(const orc_params* prm, uint32_t n, float* x, float* y, float* z,
    float* vx, float* vy, float* vz, float* m, float* id, float* p,
    uint32_t nb, const float* bx, const float* by, const float* bz,
    const float* bm, const float scene_min[3], const float scene_max[3],
    float dt, uint32_t steps, float* rho_out, float* aii_out, float* sii_out,
    float* ax_out, float* ay_out, float* az_out, uint32_t* iters)
{
    const float h = prm->h, rho0 = prm->rho0;
    Bdy b;
    if (int e = make_bdy(nb, bx, by, bz, bm, h, prm->cell_ratio, b))
        return e;
    orc_geom g;
    if (orc_geometry(scene_min, scene_max, 2.f * h, prm->cell_ratio, &g))
        return -1;
    std::vector<float> rho(n), aii(n), sii(n), ax(n), ay(n), az(n), tmp;
    std::vector<float> pbuf(n, 0.f);
    if (p)
        std::memcpy(pbuf.data(), p, n * sizeof(float));
    State s { n, x, y, z, vx, vy, vz, m };
    const f3 grav = mk(prm->g[0], prm->g[1], prm->g[2]);
    int status = 0;
    for (uint32_t step = 0; step < steps && status == 0; ++step) {
        // Scene::get_grid -> construct_and_reorder (uniformgrid.cuh:295-339):
        // extra buffers, then the state (particles.cu:93-113)
        Grid G;
        if (int e = build(g, n, x, y, z, G, nullptr))
            return e;
        if (id)
            gather(id, G.sorted, tmp);
        if (prm->scheme == 2)
            gather(pbuf.data(), G.sorted, tmp);
        for (float* a : { vx, vy, vz, m, x, y, z })
            gather(a, G.sorted, tmp);
        G.identity = true;
        uint32_t l = 0;
        status = with_kernel(prm->kind, 2.f * h, [&](auto Wk) {
            if (prm->scheme == 0) { // SESPH::step, SESPH.cu:68-95
                densities(Wk, s, G, b, rho.data());
                sesph_acc(Wk, s, G, b, rho.data(), prm->k_sesph, rho0, prm->nu,
                    h, grav, ax.data(), ay.data(), az.data());
                integrate(s, ax.data(), ay.data(), az.data(), dt);
                l = 1;
            } else if (prm->scheme == 1) { // PCISPH::step, PCISPH.cu:59-111
                const double dd = pcisph_delta(Wk, (double)h);
                const float k = (float)((dd / dt) / dt);
                densities(Wk, s, G, b, rho.data());
                non_pressure_acc(Wk, s, G, rho.data(), h, prm->nu, grav,
                    ax.data(), ay.data(), az.data());
                double avg = 0.;
                do {
                    integrate_v(s, ax.data(), ay.data(), az.data(), dt);
                    predict_rho(Wk, s, G, b, dt, rho.data());
                    pcisph_acc(Wk, s, G, b, rho.data(), k, rho0, ax.data(),
                        ay.data(), az.data());
                    l += 1;
                    double sum = 0.;
#pragma omp parallel for schedule(static) reduction(+ : sum)
                    for (int64_t i = 0; i < (int64_t)n; ++i)
                        sum += rho[i];
                    avg = sum / (double)n;
                } while ((l < prm->min_iter
                             || (float)avg > (prm->eta + 1.f) * rho0)
                    && (prm->max_iter == 0 || l < prm->max_iter));
                integrate(s, ax.data(), ay.data(), az.data(), dt);
            } else { // IISPH::step, IISPH.cu:165-262
                densities(Wk, s, G, b, rho.data());
                non_pressure_acc(Wk, s, G, rho.data(), h, prm->nu, grav,
                    ax.data(), ay.data(), az.data());
                integrate_v(s, ax.data(), ay.data(), az.data(), dt);
                iisph_diag(Wk, s, G, b, rho.data(), rho0, dt, aii.data(),
                    sii.data());
                if (prm->warmstart) {
                    for (uint32_t i = 0; i < n; ++i)
                        pbuf[i] = pbuf[i] * 0.5f;
                } else {
                    for (uint32_t i = 0; i < n; ++i)
                        pbuf[i] = jacobi(prm->omega, aii[i], 0.f, sii[i]);
                }
                const float r0i = 1.f / (rho0 * rho0);
                bool more = true;
                do {
                    iisph_pacc(Wk, s, G, b, pbuf.data(), r0i, ax.data(),
                        ay.data(), az.data());
                    double es = 0.;
                    const uint64_t over = iisph_jacobi(Wk, s, G, b, ax.data(),
                        ay.data(), az.data(), pbuf.data(), aii.data(),
                        sii.data(), dt, prm->omega, prm->eta * rho0, &es, prm->projected);
                    l += 1;
                    more = prm->iisph_avg
                        ? (es / (double)n > (double)prm->eta * rho0)
                        : (over > 0);
                } while ((l < prm->min_iter || more)
                    && (prm->max_iter == 0 || l < prm->max_iter));
                iisph_pacc(Wk, s, G, b, pbuf.data(), r0i, ax.data(), ay.data(),
                    az.data());
                integrate(s, ax.data(), ay.data(), az.data(), dt);
            }
        });
        enforce_bounds(s, scene_min, scene_max);
        if (iters)
            iters[step] = l;
    }
    if (status)
        return status;
    auto put = [n](float* dst, const std::vector<float>& src) {
        if (dst)
            std::memcpy(dst, src.data(), n * sizeof(float));
    };
    if (p)
        std::memcpy(p, pbuf.data(), n * sizeof(float));
    put(rho_out, rho);
    put(aii_out, aii);
    put(sii_out, sii);
    put(ax_out, ax);
    put(ay_out, ay);
    put(az_out, az);
    return 0;
}

} // extern "C"
