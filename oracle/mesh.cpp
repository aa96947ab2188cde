// CPU ORACLE — test infrastructure only (see oracle.h). Host restatement of
// the reference's triangle-mesh path: Morton codes and the LBVH
// (datastructure/lbvh.cuh:17-45, 204-350, 415-518; lbvh.cu:9-170), the
// brute-force closest-point query of its test (lbvh.cu:276-306), the inside
// predicate (scene/scene.cu:84-139), area-stratified surface sampling
// (scene/sample_boundary.cu:168-248, 299-389), one sweep of the sampling
// relaxation (sample_boundary.cu:20-166) and the fluid fill of a closed mesh
// (scene.cu:316-425).
//
// Float arithmetic is written operation by operation and built with
// -ffp-contract=off; the CUDA engine rounds every operation of these paths
// explicitly, so the two agree bit for bit. Dot products are the reference's
// nested fmaf (vector.cuh:152-160).
#include "oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include <omp.h>

namespace {

#include "oracle_kernels.hpp"

struct d3 {
    double x, y, z;
};
inline d3 dmk(double x, double y, double z) { return d3 { x, y, z }; }
inline d3 operator-(d3 a, d3 b) { return dmk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline d3 operator+(d3 a, d3 b) { return dmk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline d3 operator*(double s, d3 b) { return dmk(b.x * s, b.y * s, b.z * s); }
inline double ddot(d3 a, d3 b) { return std::fma(a.x, b.x, std::fma(a.y, b.y, a.z * b.z)); }
inline d3 dcross(d3 a, d3 b)
{
    return dmk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline f3 fcross(f3 a, f3 b)
{
    return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

struct Mesh {
    const double *vx, *vy, *vz;
    uint32_t nv;
    const uint32_t* f; // 3 per face, original order
    uint32_t nf;
    d3 vd(uint32_t v) const { return dmk(vx[v], vy[v], vz[v]); }
    f3 vf(uint32_t v) const { return mk((float)vx[v], (float)vy[v], (float)vz[v]); }
};

bool valid(const Mesh& m)
{
    if (!m.vx || !m.vy || !m.vz || !m.f || m.nf == 0)
        return false;
    for (uint64_t k = 0; k < 3ull * m.nf; ++k)
        if (m.f[k] >= m.nv)
            return false;
    return true;
}

// ---- Morton codes (lbvh.cuh:17-45, 204-225) ----------------------------------
// 10 bits of v spread to every third bit (bit i -> bit 3i)
uint32_t spread10(uint32_t v)
{
    uint32_t r = 0;
    for (int b = 0; b < 10; ++b)
        r |= ((v >> b) & 1u) << (3 * b);
    return r;
}

void bounds(const Mesh& m, d3& lo, d3& hi)
{
    lo = dmk(INFINITY, INFINITY, INFINITY);
    hi = dmk(-INFINITY, -INFINITY, -INFINITY);
    for (uint32_t v = 0; v < m.nv; ++v) {
        lo = dmk(std::fmin(lo.x, m.vx[v]), std::fmin(lo.y, m.vy[v]), std::fmin(lo.z, m.vz[v]));
        hi = dmk(std::fmax(hi.x, m.vx[v]), std::fmax(hi.y, m.vy[v]), std::fmax(hi.z, m.vz[v]));
    }
}

uint32_t quantise(double n)
{
    // static_cast<float>(min(max(n * 1024, 0), 1023)), then to an integer
    return (uint32_t)(float)std::fmin(std::fmax(n * 1024., 0.), 1023.);
}

std::vector<uint32_t> morton(const Mesh& m)
{
    d3 lo, hi;
    bounds(m, lo, hi);
    const d3 ext = hi - lo;
    const d3 inv = dmk(1. / ext.x, 1. / ext.y, 1. / ext.z);
    const double third = 1. / 3.;
    std::vector<uint32_t> codes(m.nf);
    for (uint32_t t = 0; t < m.nf; ++t) {
        const d3 a = m.vd(m.f[3 * t]), b = m.vd(m.f[3 * t + 1]), c = m.vd(m.f[3 * t + 2]);
        const d3 cen = third * (a + b + c) - lo;
        const uint32_t qx = quantise(cen.x * inv.x), qy = quantise(cen.y * inv.y),
                       qz = quantise(cen.z * inv.z);
        codes[t] = (spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz);
    }
    return codes;
}

// ---- the tree (lbvh.cuh:256-350, lbvh.cu:34-170) -----------------------------
struct Box {
    f3 lo, hi;
};

// the padded box of a flat extent (lbvh.cu:20-29). The reference's union
// operator (lbvh.cuh:58-68) pads the LEFT operand instead of the union when the
// union is flat; this restatement pads the union, as the engine does.
Box pad_if_flat(Box b)
{
    const f3 e = b.hi - b.lo;
    if (std::fmin(e.x, std::fmin(e.y, e.z)) == 0.f) {
        const f3 eps = mk(FLT_EPSILON, FLT_EPSILON, FLT_EPSILON);
        return Box { b.lo - eps, b.hi + eps };
    }
    return b;
}

Box unite(Box a, Box b)
{
    return pad_if_flat(Box { mk(std::fmin(a.lo.x, b.lo.x), std::fmin(a.lo.y, b.lo.y),
                                 std::fmin(a.lo.z, b.lo.z)),
        mk(std::fmax(a.hi.x, b.hi.x), std::fmax(a.hi.y, b.hi.y), std::fmax(a.hi.z, b.hi.z)) });
}

struct Tree {
    std::vector<uint32_t> order;  // leaf j holds original face order[j]
    std::vector<uint32_t> cl, cr; // ChildNode encoding: index << 1 | (internal ? 1 : 0)
    std::vector<Box> leaf, node;
    uint32_t height = 0;
};

inline int delta(const std::vector<uint64_t>& k, int i, int j)
{
    if (j < 0 || j >= (int)k.size())
        return -1;
    return __builtin_clzll(k[i] ^ k[j]);
}

Tree build_tree(const Mesh& m)
{
    Tree T;
    const uint32_t n = m.nf;
    const std::vector<uint32_t> codes = morton(m);
    T.order.resize(n);
    std::iota(T.order.begin(), T.order.end(), 0u);
    std::stable_sort(T.order.begin(), T.order.end(),
        [&](uint32_t a, uint32_t b) { return codes[a] < codes[b]; });
    std::vector<uint64_t> key(n);
    for (uint32_t j = 0; j < n; ++j)
        key[j] = ((uint64_t)codes[T.order[j]] << 32) | j;

    T.leaf.resize(n);
    for (uint32_t j = 0; j < n; ++j) {
        const uint32_t* f = m.f + 3 * T.order[j];
        const d3 a = m.vd(f[0]), b = m.vd(f[1]), c = m.vd(f[2]);
        Box bx { mk((float)std::fmin(std::fmin(a.x, b.x), c.x),
                     (float)std::fmin(std::fmin(a.y, b.y), c.y),
                     (float)std::fmin(std::fmin(a.z, b.z), c.z)),
            mk((float)std::fmax(std::fmax(a.x, b.x), c.x), (float)std::fmax(std::fmax(a.y, b.y), c.y),
                (float)std::fmax(std::fmax(a.z, b.z), c.z)) };
        T.leaf[j] = pad_if_flat(bx);
    }
    if (n < 2)
        return T;

    // Karras 2012, section 4: node i covers a key range with i at one end
    const int ni = (int)n - 1;
    T.cl.assign(ni, 0);
    T.cr.assign(ni, 0);
    std::vector<int> parent_node(ni, -1), parent_leaf(n, -1);
    for (int i = 0; i < ni; ++i) {
        int first, last;
        if (i == 0) {
            first = 0;
            last = (int)n - 1;
        } else {
            const int d = delta(key, i, i + 1) > delta(key, i, i - 1) ? 1 : -1;
            const int dmin = delta(key, i, i - d);
            int lmax = 2;
            while (delta(key, i, i + lmax * d) > dmin)
                lmax *= 2;
            int l = 0;
            for (int t = lmax / 2; t >= 1; t /= 2)
                if (delta(key, i, i + (l + t) * d) > dmin)
                    l += t;
            const int j = i + l * d;
            first = std::min(i, j);
            last = std::max(i, j);
        }
        // split: the last index of [first, last) sharing more than the
        // range's common prefix with key[first]
        const int common = delta(key, first, last);
        int split = first;
        int step = last - first;
        do {
            step = (step + 1) / 2;
            const int s = split + step;
            if (s < last && delta(key, first, s) > common)
                split = s;
        } while (step > 1);
        const bool l_leaf = split == first, r_leaf = split + 1 == last;
        T.cl[i] = ((uint32_t)split << 1) | (l_leaf ? 0u : 1u);
        T.cr[i] = ((uint32_t)(split + 1) << 1) | (r_leaf ? 0u : 1u);
        (l_leaf ? parent_leaf[split] : parent_node[split]) = i;
        (r_leaf ? parent_leaf[split + 1] : parent_node[split + 1]) = i;
    }
    // boxes bottom-up (recursion from the root)
    T.node.resize(ni);
    std::vector<int> stack { 0 };
    std::vector<char> done(ni, 0);
    while (!stack.empty()) {
        const int i = stack.back();
        const uint32_t l = T.cl[i], r = T.cr[i];
        bool ready = true;
        for (uint32_t c : { l, r })
            if ((c & 1u) && !done[c >> 1]) {
                stack.push_back((int)(c >> 1));
                ready = false;
            }
        if (!ready)
            continue;
        stack.pop_back();
        const Box bl = (l & 1u) ? T.node[l >> 1] : T.leaf[l >> 1];
        const Box br = (r & 1u) ? T.node[r >> 1] : T.leaf[r >> 1];
        T.node[i] = unite(bl, br);
        done[i] = 1;
    }
    // height: edges from the root to the deepest leaf (lbvh.cu:152-170)
    for (uint32_t j = 0; j < n; ++j) {
        uint32_t depth = 1;
        for (int p = parent_leaf[j]; p != 0; p = parent_node[p])
            ++depth;
        T.height = std::max(T.height, depth);
    }
    return T;
}

// ---- queries (lbvh.cuh:96-107, 415-518; geometry.cuh) -------------------------
float min_dist(const Box& b, f3 p)
{
    const f3 r = mk(std::fmin(std::fmax(p.x, b.lo.x), b.hi.x),
        std::fmin(std::fmax(p.y, b.lo.y), b.hi.y), std::fmin(std::fmax(p.z, b.lo.z), b.hi.z));
    const f3 d = r - p;
    return dot(d, d);
}

// closest point on triangle abc to p: the Voronoi-region walk of Ericson,
// Real-Time Collision Detection (2005), section 5.1.5
f3 closest_on_triangle(f3 p, f3 a, f3 b, f3 c)
{
    const f3 ab = b - a, ac = c - a, ap = p - a;
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f)
        return a;
    const f3 bp = p - b;
    const float d3_ = dot(ab, bp), d4 = dot(ac, bp);
    if (d3_ >= 0.f && d4 <= d3_)
        return b;
    const float vc = d1 * d4 - d3_ * d2;
    if (vc <= 0.f && d1 >= 0.f && d3_ <= 0.f)
        return a + (d1 / (d1 - d3_)) * ab;
    const f3 cp = p - c;
    const float d5 = dot(ab, cp), d6 = dot(ac, cp);
    if (d6 >= 0.f && d5 <= d6)
        return c;
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f)
        return a + (d2 / (d2 - d6)) * ac;
    const float va = d3_ * d6 - d5 * d4;
    if (va <= 0.f && (d4 - d3_) >= 0.f && (d5 - d6) >= 0.f)
        return b + ((d4 - d3_) / ((d4 - d3_) + (d5 - d6))) * (c - b);
    const float den = 1.f / (va + vb + vc);
    const float v = vb * den, w = vc * den;
    return (a + v * ab) + w * ac;
}

struct Hit {
    float d2;
    f3 q;       // closest point
    bool inside; // the step to the closest point runs along its face's normal
};

Hit leaf_hit(const Mesh& m, const Tree& T, uint32_t j, f3 p)
{
    const uint32_t* f = m.f + 3 * T.order[j];
    const f3 a = m.vf(f[0]), b = m.vf(f[1]), c = m.vf(f[2]);
    const f3 q = closest_on_triangle(p, a, b, c);
    const f3 d = q - p;
    const f3 nrm = fcross(b - a, c - a);
    // inside when the step to the surface runs along the outward normal; the
    // reference's predicate returns the negation, the points to remove
    // (scene.cu:120-133 with remove_if)
    return Hit { dot(d, d), q, dot(nrm, d) >= 0.f };
}

// stack traversal, nearer child first, pruning by the best squared distance
Hit traverse(const Mesh& m, const Tree& T, f3 p)
{
    Hit best { FLT_MAX, mk(0.f, 0.f, 0.f), false };
    if (m.nf == 1)
        return leaf_hit(m, T, 0, p);
    std::vector<uint32_t> idx { 0 };
    std::vector<float> md { min_dist(T.node[0], p) };
    auto visit = [&](float d, uint32_t c) {
        if (!(d <= best.d2))
            return;
        if (!(c & 1u)) {
            const Hit h = leaf_hit(m, T, c >> 1, p);
            if (h.d2 <= best.d2)
                best = h;
        } else {
            idx.push_back(c >> 1);
            md.push_back(d);
        }
    };
    while (!idx.empty()) {
        const uint32_t i = idx.back();
        const float d = md.back();
        idx.pop_back();
        md.pop_back();
        if (d > best.d2)
            continue;
        const uint32_t l = T.cl[i], r = T.cr[i];
        const float dl = min_dist((l & 1u) ? T.node[l >> 1] : T.leaf[l >> 1], p);
        const float dr = min_dist((r & 1u) ? T.node[r >> 1] : T.leaf[r >> 1], p);
        if (dl < dr) {
            visit(dr, r);
            visit(dl, l);
        } else {
            visit(dl, l);
            visit(dr, r);
        }
    }
    return best;
}

// ---- counter-based random numbers (the engine's SplitMix64 streams) ----------
uint64_t splitmix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
uint64_t stream_bits(uint64_t seed, uint64_t t, uint64_t k)
{
    return splitmix64(seed + 0x9E3779B97F4A7C15ull * ((t << 40) + k + 1));
}
// uniform in (0, 1] with 53 bits
double uniform_d(uint64_t seed, uint64_t t, uint64_t k)
{
    return (double)((stream_bits(seed, t, k) >> 11) + 1) * (1.0 / 9007199254740992.0);
}
// uniform in [0, 1) with 24 bits
float uniform_f(uint64_t seed, uint64_t t, uint64_t k)
{
    return (float)(uint32_t)(stream_bits(seed, t, k) >> 40) * (1.f / 16777216.f);
}

} // namespace

extern "C" {

int orc_mesh_morton(const double* vx, const double* vy, const double* vz, uint32_t nv,
    const uint32_t* faces, uint32_t nf, uint32_t* codes)
{
    const Mesh m { vx, vy, vz, nv, faces, nf };
    if (!valid(m) || !codes)
        return -1;
    const std::vector<uint32_t> c = morton(m);
    std::copy(c.begin(), c.end(), codes);
    return 0;
}

int orc_lbvh_build(const double* vx, const double* vy, const double* vz, uint32_t nv,
    const uint32_t* faces, uint32_t nf, uint32_t* order, uint32_t* children_l,
    uint32_t* children_r, float* leaf_box, float* node_box, uint32_t* height)
{
    const Mesh m { vx, vy, vz, nv, faces, nf };
    if (!valid(m))
        return -1;
    const Tree T = build_tree(m);
    auto put = [](const Box& b, float* o) {
        o[0] = b.lo.x;
        o[1] = b.lo.y;
        o[2] = b.lo.z;
        o[3] = b.hi.x;
        o[4] = b.hi.y;
        o[5] = b.hi.z;
    };
    if (order)
        std::copy(T.order.begin(), T.order.end(), order);
    if (children_l)
        std::copy(T.cl.begin(), T.cl.end(), children_l);
    if (children_r)
        std::copy(T.cr.begin(), T.cr.end(), children_r);
    for (uint32_t j = 0; leaf_box && j < nf; ++j)
        put(T.leaf[j], leaf_box + 6 * j);
    for (uint32_t i = 0; node_box && i + 1 < nf; ++i)
        put(T.node[i], node_box + 6 * i);
    if (height)
        *height = T.height;
    return 0;
}

int orc_lbvh_query(const double* vx, const double* vy, const double* vz, uint32_t nv,
    const uint32_t* faces, uint32_t nf, uint32_t n, float* x, float* y, float* z,
    uint8_t* inside)
{
    const Mesh m { vx, vy, vz, nv, faces, nf };
    if (!valid(m))
        return -1;
    const Tree T = build_tree(m);
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const Hit h = traverse(m, T, mk(x[i], y[i], z[i]));
        if (inside)
            inside[i] = h.inside ? 1 : 0;
        else
            store(h.q, (uint32_t)i, x, y, z);
    }
    return 0;
}

int orc_project_brute(const double* vx, const double* vy, const double* vz, uint32_t nv,
    const uint32_t* faces, uint32_t nf, uint32_t n, float* x, float* y, float* z)
{
    const Mesh m { vx, vy, vz, nv, faces, nf };
    if (!valid(m))
        return -1;
    const Tree T = build_tree(m); // the brute force scans faces in leaf order
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const f3 p = mk(x[i], y[i], z[i]);
        Hit best { FLT_MAX, mk(0.f, 0.f, 0.f), false };
        for (uint32_t j = 0; j < nf; ++j) {
            const Hit h = leaf_hit(m, T, j, p);
            if (h.d2 <= best.d2)
                best = h;
        }
        store(best.q, (uint32_t)i, x, y, z);
    }
    return 0;
}

int orc_mesh_measure(const double* vx, const double* vy, const double* vz, uint32_t nv,
    const uint32_t* faces, uint32_t nf, double* area, double* volume, double* cdf)
{
    const Mesh m { vx, vy, vz, nv, faces, nf };
    if (!valid(m))
        return -1;
    double acc = 0., vol = 0.;
    for (uint32_t t = 0; t < nf; ++t) {
        const d3 a = m.vd(faces[3 * t]), b = m.vd(faces[3 * t + 1]), c = m.vd(faces[3 * t + 2]);
        const d3 cr = dcross(b - a, c - a);
        acc += 0.5 * std::sqrt(ddot(cr, cr)); // sample_boundary.cu:317-330
        if (cdf)
            cdf[t] = acc;
        vol += ddot(a, dcross(b, c)); // sample_boundary.cuh:40-60
    }
    if (area)
        *area = acc;
    if (volume)
        *volume = std::fabs(vol) / 6.;
    return 0;
}

uint32_t orc_mesh_sample_count(double area, float h, float oversampling)
{
    // sample_boundary.cu:339-346
    const double h_bdy = (double)h / (double)oversampling;
    const float per = 1.5f * std::sqrt(3.f) * (float)h_bdy * (float)h_bdy;
    return (uint32_t)std::ceil(area / (double)per);
}

int orc_mesh_sample(const double* vx, const double* vy, const double* vz, uint32_t nv,
    const uint32_t* faces, uint32_t nf, float h, float oversampling, uint64_t seed,
    uint32_t cap, float* x, float* y, float* z, uint32_t* count)
{
    const Mesh m { vx, vy, vz, nv, faces, nf };
    if (!valid(m) || !count)
        return -1;
    std::vector<double> cdf(nf);
    double area = 0.;
    orc_mesh_measure(vx, vy, vz, nv, faces, nf, &area, nullptr, cdf.data());
    const uint32_t n = orc_mesh_sample_count(area, h, oversampling);
    *count = n;
    if (!x)
        return 0;
    if (cap < n)
        return -2;
    const double bin = area / (double)n;
    for (uint32_t i = 0; i < n; ++i) {
        // stratified position along the summed area (sample_boundary.cu:186-190)
        const double s_area = ((double)i / (double)n) * area + bin * uniform_d(seed, 8, i);
        // first face whose inclusive sum reaches it; the last face past the end
        const uint32_t t = (uint32_t)std::min<size_t>(
            std::lower_bound(cdf.begin(), cdf.end(), s_area) - cdf.begin(), nf - 1);
        const d3 a = m.vd(faces[3 * t]), b = m.vd(faces[3 * t + 1]), c = m.vd(faces[3 * t + 2]);
        double u = uniform_d(seed, 9, i), v = uniform_d(seed, 10, i);
        if (!(u + v <= 1.)) { // fold the parallelogram (sample_boundary.cu:226-235)
            u = 1. - u;
            v = 1. - v;
        }
        const d3 p = (a + u * (b - a)) + v * (c - a);
        x[i] = (float)p.x;
        y[i] = (float)p.y;
        z[i] = (float)p.z;
    }
    return 0;
}

float orc_hex_plane_density(float h_bdy)
{
    // _hex_plane_rest_density (sample_boundary.cu:78-98), B3 at support 2 h_bdy
    const B3 Wk(2.f * h_bdy);
    const f3 qa = h_bdy * mk(1.f, 0.f, 0.f);
    const f3 ra = h_bdy * mk(.5f, (float)(std::sqrt(3.) * .5), 0.f);
    float rho = 0.f;
    for (int q = -2; q <= 2; ++q)
        for (int r = -2; r <= 2; ++r)
            rho += W(Wk, (float)q * qa + (float)r * ra);
    return rho;
}

int orc_mesh_relax_sweep(const double* vx, const double* vy, const double* vz, uint32_t nv,
    const uint32_t* faces, uint32_t nf, uint32_t n, float* x, float* y, float* z, float h_bdy,
    float k, float* num_den)
{
    const Mesh m { vx, vy, vz, nv, faces, nf };
    if (!valid(m) || !num_den)
        return -1;
    const B3 Wk(2.f * h_bdy);
    const float r2 = (2.f * h_bdy) * (2.f * h_bdy);
    const float rho0 = orc_hex_plane_density(h_bdy);
    const float inv2 = 1.f / (rho0 * rho0);
    // number densities (sample_boundary.cu:30-44), all samples within 2 h_bdy
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const f3 p = load((uint32_t)i, x, y, z);
        float s = 0.f;
        for (uint32_t j = 0; j < n; ++j) {
            const f3 d = p - load(j, x, y, z);
            if (dot(d, d) <= r2)
                s += W(Wk, d);
        }
        num_den[i] = s;
    }
    // shift down the number-density gradient (sample_boundary.cu:46-71),
    // reading the old positions of every neighbour
    std::vector<float> nx(n), ny(n), nz(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const f3 p = load((uint32_t)i, x, y, z);
        const float ti = inv2 * num_den[i];
        f3 acc = mk(0.f, 0.f, 0.f);
        for (uint32_t j = 0; j < n; ++j) {
            const f3 d = p - load(j, x, y, z);
            if (dot(d, d) <= r2)
                acc += (ti + inv2 * num_den[j]) * dW(Wk, d);
        }
        const f3 q = p + ((-k * h_bdy) * h_bdy) * acc;
        nx[i] = q.x;
        ny[i] = q.y;
        nz[i] = q.z;
    }
    std::copy(nx.begin(), nx.end(), x);
    std::copy(ny.begin(), ny.end(), y);
    std::copy(nz.begin(), nz.end(), z);
    // back onto the surface (sample_boundary.cu:145-146)
    return orc_lbvh_query(vx, vy, vz, nv, faces, nf, n, x, y, z, nullptr);
}

int orc_mesh_fill(const double* vx, const double* vy, const double* vz, uint32_t nv,
    const uint32_t* faces, uint32_t nf, float h, float jitter, uint64_t seed, uint32_t cap,
    float* x, float* y, float* z, uint32_t* count)
{
    const Mesh m { vx, vy, vz, nv, faces, nf };
    if (!valid(m) || !count || !(h > 0.f))
        return -1;
    d3 lo, hi;
    bounds(m, lo, hi);
    // scene.cu:336-351: the lattice over the mesh's float bounds
    const f3 flo = mk((float)lo.x, (float)lo.y, (float)lo.z);
    const f3 fhi = mk((float)hi.x, (float)hi.y, (float)hi.z);
    const f3 ext = fhi - flo;
    const int64_t cx = (int64_t)std::floor(ext.x / h), cy = (int64_t)std::floor(ext.y / h),
                  cz = (int64_t)std::floor(ext.z / h);
    const int64_t total = std::max<int64_t>(cx, 0) * std::max<int64_t>(cy, 0) * std::max<int64_t>(cz, 0);
    std::vector<float> px(total), py(total), pz(total);
    for (int64_t g = 0; g < total; ++g) {
        const int64_t i = g % cx, j = (g / cx) % cy, kk = g / (cx * cy);
        px[g] = flo.x + (float)i * h;
        py[g] = flo.y + (float)j * h;
        pz[g] = flo.z + (float)kk * h;
    }
    std::vector<uint8_t> in(total);
    orc_lbvh_query(vx, vy, vz, nv, faces, nf, (uint32_t)total, px.data(), py.data(), pz.data(),
        in.data());
    uint32_t kept = 0;
    const float a = jitter * h;
    for (int64_t g = 0; g < total; ++g) {
        if (!in[g])
            continue;
        if (x && kept < cap) {
            float p[3] = { px[g], py[g], pz[g] };
            if (jitter > 0.f)
                for (int ax = 0; ax < 3; ++ax)
                    p[ax] = p[ax] + (2.f * uniform_f(seed, ax, (uint64_t)g) - 1.f) * a;
            x[kept] = p[0];
            y[kept] = p[1];
            z[kept] = p[2];
        }
        ++kept;
    }
    *count = kept;
    return (x && kept > cap) ? -2 : 0;
}

} // extern "C"
