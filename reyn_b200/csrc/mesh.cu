// Triangle meshes on the device: the LBVH over a mesh's faces and its
// closest-point queries, area-stratified surface sampling, the relaxation of
// a sampling, and the fluid fill of a closed mesh. The reference
// (datastructure/lbvh.cuh, lbvh.cu, scene/sample_boundary.cu, scene/scene.cu)
// builds its LBVH with thrust (transform, sort_by_key) and traverses separate
// arrays of child links and boxes. Here:
//  * the 30-bit Morton codes are sorted by an LSD radix sort of this file:
//    four stable 8-bit passes, digit ranks inside a tile from warp match
//    masks, tile offsets from the engine's exclusive scan;
//  * the tree is Karras' (2012) binary radix tree, one thread per internal
//    node, with the reference's node numbering; boxes are built bottom-up
//    with one arrival counter per node;
//  * a traversal reads one 64-byte record per internal node that holds both
//    children's boxes and links, and one 48-byte record per leaf holding the
//    triangle's float vertices, so a visited node is one cache line instead of
//    four scattered loads;
//  * every float operation of the queries and every double operation of the
//    Morton codes and the sampling is explicitly rounded, so the host oracle
//    reproduces the results bit for bit.
#include "engine.cuh"

#include <cctype>
#include <cfloat>
#include <cmath>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

namespace reyn {
namespace {

    constexpr int MESH_THREADS = 128;
    constexpr int RADIX_THREADS = 256; // one thread per 8-bit digit
    constexpr int RADIX_ITEMS = 8;
    constexpr int RADIX_TILE = RADIX_THREADS * RADIX_ITEMS;
    constexpr int DSCAN_THREADS = 256;
    constexpr int DSCAN_ITEMS = 8;
    constexpr int DSCAN_TILE = DSCAN_THREADS * DSCAN_ITEMS;
    constexpr uint32_t MAX_FACES = 1u << 30;

    struct Box {
        float lo[3], hi[3];
    };

    // one internal node: both children's boxes and links (ChildNode encoding:
    // index << 1 | 1 for an internal child, lbvh.cuh:162-193)
    struct __align__(16) Node {
        float4 a; // left lo.x lo.y lo.z hi.x
        float4 b; // left hi.y hi.z, right lo.x lo.y
        float4 c; // right lo.z hi.x hi.y hi.z
        uint4 d;  // left link, right link, -, -
    };
    static_assert(sizeof(Node) == 64, "a node record is one 64-byte line");

    struct MeshView {
        const Node* __restrict__ nodes;
        const float4* __restrict__ tri; // 3 records per leaf
        uint32_t n_internal;
        Box root;
        uint32_t* status; // MESH_STACK_FULL | MESH_BAD_TREE
    };

    // traversal and build faults (never expected; each stops the offending
    // thread instead of reading out of bounds or looping)
    constexpr uint32_t MESH_STACK_FULL = 1u;
    constexpr uint32_t MESH_BAD_TREE = 2u;

    // ---- explicitly rounded float vectors ------------------------------------
    struct V3 {
        float x, y, z;
    };
    __device__ __forceinline__ V3 mk3(float x, float y, float z) { return V3 { x, y, z }; }
    __device__ __forceinline__ V3 operator-(V3 a, V3 b)
    {
        return mk3(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z));
    }
    __device__ __forceinline__ V3 operator+(V3 a, V3 b)
    {
        return mk3(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z));
    }
    __device__ __forceinline__ V3 operator*(float s, V3 b)
    {
        return mk3(__fmul_rn(b.x, s), __fmul_rn(b.y, s), __fmul_rn(b.z, s));
    }
    // the reference's dot product: nested fmaf (vector.cuh:152-155)
    __device__ __forceinline__ float dot3(V3 a, V3 b)
    {
        return __fmaf_rn(a.x, b.x, __fmaf_rn(a.y, b.y, __fmul_rn(a.z, b.z)));
    }
    __device__ __forceinline__ V3 cross3(V3 a, V3 b)
    {
        return mk3(__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
            __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x)));
    }

    // closest point on triangle abc to p: the Voronoi-region walk of Ericson,
    // Real-Time Collision Detection (2005), section 5.1.5 (the method of
    // geometry.cuh:14-61)
    __device__ __forceinline__ V3 closest_on_triangle(V3 p, V3 a, V3 b, V3 c)
    {
        const V3 ab = b - a, ac = c - a, ap = p - a;
        const float d1 = dot3(ab, ap), d2 = dot3(ac, ap);
        if (d1 <= 0.f && d2 <= 0.f)
            return a;
        const V3 bp = p - b;
        const float d3 = dot3(ab, bp), d4 = dot3(ac, bp);
        if (d3 >= 0.f && d4 <= d3)
            return b;
        const float vc = __fsub_rn(__fmul_rn(d1, d4), __fmul_rn(d3, d2));
        if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f)
            return a + __fdiv_rn(d1, __fsub_rn(d1, d3)) * ab;
        const V3 cp = p - c;
        const float d5 = dot3(ab, cp), d6 = dot3(ac, cp);
        if (d6 >= 0.f && d5 <= d6)
            return c;
        const float vb = __fsub_rn(__fmul_rn(d5, d2), __fmul_rn(d1, d6));
        if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f)
            return a + __fdiv_rn(d2, __fsub_rn(d2, d6)) * ac;
        const float va = __fsub_rn(__fmul_rn(d3, d6), __fmul_rn(d5, d4));
        const float e43 = __fsub_rn(d4, d3), e56 = __fsub_rn(d5, d6);
        if (va <= 0.f && e43 >= 0.f && e56 >= 0.f)
            return b + __fdiv_rn(e43, __fadd_rn(e43, e56)) * (c - b);
        const float den = __fdiv_rn(1.f, __fadd_rn(__fadd_rn(va, vb), vc));
        return (a + __fmul_rn(vb, den) * ab) + __fmul_rn(vc, den) * ac;
    }

    // squared distance from p to a box (lbvh.cuh:96-107)
    __device__ __forceinline__ float box_dist(
        float lx, float ly, float lz, float hx, float hy, float hz, V3 p)
    {
        const V3 r = mk3(fminf(fmaxf(p.x, lx), hx), fminf(fmaxf(p.y, ly), hy),
            fminf(fmaxf(p.z, lz), hz));
        const V3 d = r - p;
        return dot3(d, d);
    }

    struct Hit {
        float d2;
        V3 q;
        bool inside;
    };

    template <bool INSIDE>
    __device__ __forceinline__ void leaf_test(const MeshView& m, uint32_t j, V3 p, Hit& best)
    {
        const float4 t0 = __ldg(m.tri + 3 * size_t(j));
        const float4 t1 = __ldg(m.tri + 3 * size_t(j) + 1);
        const float4 t2 = __ldg(m.tri + 3 * size_t(j) + 2);
        const V3 a = mk3(t0.x, t0.y, t0.z), b = mk3(t0.w, t1.x, t1.y), c = mk3(t1.z, t1.w, t2.x);
        const V3 q = closest_on_triangle(p, a, b, c);
        const V3 d = q - p;
        const float d2 = dot3(d, d);
        if (d2 <= best.d2) {
            best.d2 = d2;
            best.q = q;
            // inside when the step to the surface runs along the face's
            // (outward) normal; the reference's predicate returns the
            // negation, the points remove_if drops (scene.cu:120-133, 417-419)
            if constexpr (INSIDE)
                best.inside = dot3(cross3(b - a, c - a), d) >= 0.f;
        }
    }

    // bvh_find_closest (lbvh.cuh:415-518): a stack traversal that visits the
    // nearer child first and prunes by the best squared distance so far
    template <int STACK, bool INSIDE>
    __device__ __forceinline__ Hit closest(const MeshView& m, V3 p)
    {
        Hit best { FLT_MAX, mk3(0.f, 0.f, 0.f), false };
        if (m.n_internal == 0) {
            leaf_test<INSIDE>(m, 0, p, best);
            return best;
        }
        uint32_t st_node[STACK];
        float st_dist[STACK];
        st_node[0] = 0;
        st_dist[0] = box_dist(m.root.lo[0], m.root.lo[1], m.root.lo[2], m.root.hi[0],
            m.root.hi[1], m.root.hi[2], p);
        int sp = 1;
        auto visit = [&](uint32_t link, float dist) {
            if (!(dist <= best.d2))
                return;
            const uint32_t k = link >> 1;
            if (!(link & 1u)) {
                if (k <= m.n_internal) // leaves 0 .. n_internal
                    leaf_test<INSIDE>(m, k, p, best);
                else
                    atomicOr(m.status, MESH_BAD_TREE);
            } else if (k >= m.n_internal) {
                atomicOr(m.status, MESH_BAD_TREE);
            } else if (sp < STACK) {
                st_node[sp] = k;
                st_dist[sp] = dist;
                ++sp;
            } else {
                atomicOr(m.status, MESH_STACK_FULL); // not for STACK >= height + 2
            }
        };
        // a tree expands each internal node at most once
        uint32_t pops = 0;
        do {
            if (++pops > m.n_internal) {
                atomicOr(m.status, MESH_BAD_TREE);
                break;
            }
            --sp;
            if (st_dist[sp] > best.d2)
                continue;
            const Node* nd = m.nodes + st_node[sp];
            const float4 a = __ldg(&nd->a), b = __ldg(&nd->b), c = __ldg(&nd->c);
            const uint4 d = __ldg(&nd->d);
            const float dl = box_dist(a.x, a.y, a.z, a.w, b.x, b.y, p);
            const float dr = box_dist(b.z, b.w, c.x, c.y, c.z, c.w, p);
            // the farther child first, so that the nearer one is popped next
            if (dl < dr) {
                visit(d.y, dr);
                visit(d.x, dl);
            } else {
                visit(d.x, dl);
                visit(d.y, dr);
            }
        } while (sp > 0);
        return best;
    }

    // points from (x, y, z) or, with src, from packed float4 records; results
    // to index perm[i] (or i) of the output arrays
    template <int STACK, bool INSIDE>
    __global__ void __launch_bounds__(MESH_THREADS) k_mesh_query(uint32_t n, MeshView m,
        const float4* __restrict__ src, const uint32_t* __restrict__ perm, const float* xin,
        const float* yin, const float* zin, float* x, float* y, float* z,
        uint8_t* __restrict__ inside)
    {
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n)
            return;
        V3 p;
        if (src) {
            const float4 s = src[i];
            p = mk3(s.x, s.y, s.z);
        } else {
            p = mk3(xin[i], yin[i], zin[i]);
        }
        const Hit h = closest<STACK, INSIDE>(m, p);
        const uint32_t o = perm ? perm[i] : i;
        if constexpr (INSIDE) {
            inside[o] = h.inside ? 1 : 0;
        } else {
            x[o] = h.q.x;
            y[o] = h.q.y;
            z[o] = h.q.z;
        }
    }

    // 10 bits of v spread to every third bit (bit i -> bit 3i)
    __device__ __forceinline__ uint32_t spread10(uint32_t v)
    {
        v &= 0x3ffu;
        v = (v | (v << 16)) & 0x030000FFu;
        v = (v | (v << 8)) & 0x0300F00Fu;
        v = (v | (v << 4)) & 0x030C30C3u;
        v = (v | (v << 2)) & 0x09249249u;
        return v;
    }

    // Morton code of each query point in the mesh's box (clamped), for
    // ordering only: queries sorted by it traverse similar paths in a warp
    __global__ void k_query_keys(uint32_t n, const float* __restrict__ x,
        const float* __restrict__ y, const float* __restrict__ z, float3 lo, float3 scale,
        uint32_t* __restrict__ codes, uint32_t* __restrict__ ids)
    {
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n)
            return;
        auto q = [](float v, float l, float sc) {
            const float t = (v - l) * sc;
            return uint32_t(fminf(fmaxf(t, 0.f), 1023.f)); // NaN -> 0
        };
        codes[i] = (spread10(q(x[i], lo.x, scale.x)) << 2) | (spread10(q(y[i], lo.y, scale.y)) << 1)
            | spread10(q(z[i], lo.z, scale.z));
        ids[i] = i;
    }

    __global__ void k_query_gather(uint32_t n, const uint32_t* __restrict__ perm,
        const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
        float4* __restrict__ pts)
    {
        const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
        if (s >= n)
            return;
        const uint32_t p = perm[s];
        pts[s] = make_float4(x[p], y[p], z[p], 0.f);
    }

    // ---- face areas, volume and the sampling CDF -----------------------------
    struct D3 {
        double x, y, z;
    };
    __device__ __forceinline__ D3 dload(
        uint32_t v, const double* vx, const double* vy, const double* vz)
    {
        return D3 { vx[v], vy[v], vz[v] };
    }
    __device__ __forceinline__ D3 dsub(D3 a, D3 b)
    {
        return D3 { __dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y), __dsub_rn(a.z, b.z) };
    }
    __device__ __forceinline__ double ddot(D3 a, D3 b)
    {
        return __fma_rn(a.x, b.x, __fma_rn(a.y, b.y, __dmul_rn(a.z, b.z)));
    }
    __device__ __forceinline__ D3 dcross(D3 a, D3 b)
    {
        return D3 { __dsub_rn(__dmul_rn(a.y, b.z), __dmul_rn(a.z, b.y)),
            __dsub_rn(__dmul_rn(a.z, b.x), __dmul_rn(a.x, b.z)),
            __dsub_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)) };
    }

    // area of each face (sample_boundary.cu:317-330) and the signed volume of
    // its tetrahedron with the origin, times 6 (sample_boundary.cuh:40-60)
    __global__ void k_face_measure(uint32_t nf, const double* __restrict__ vx,
        const double* __restrict__ vy, const double* __restrict__ vz,
        const uint32_t* __restrict__ faces, double* __restrict__ area, double* __restrict__ vol)
    {
        const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= nf)
            return;
        const D3 a = dload(faces[3 * size_t(t)], vx, vy, vz);
        const D3 b = dload(faces[3 * size_t(t) + 1], vx, vy, vz);
        const D3 c = dload(faces[3 * size_t(t) + 2], vx, vy, vz);
        const D3 cr = dcross(dsub(b, a), dsub(c, a));
        area[t] = __dmul_rn(0.5, __dsqrt_rn(ddot(cr, cr)));
        vol[t] = ddot(a, dcross(b, c));
    }

    __device__ __forceinline__ double block_exclusive_scan_d(double v, double* total)
    {
        constexpr int NW = DSCAN_THREADS / 32;
        __shared__ double wsum[NW];
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        double inc = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double t = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o)
                inc = t + inc;
        }
        double exc = __shfl_up_sync(0xffffffffu, inc, 1);
        if (lane == 0)
            exc = 0.0;
        if (lane == 31)
            wsum[w] = inc;
        __syncthreads();
        if (w == 0) {
            double s = lane < NW ? wsum[lane] : 0.0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const double t = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o)
                    s = t + s;
            }
            double e = __shfl_up_sync(0xffffffffu, s, 1);
            if (lane == 0)
                e = 0.0;
            if (lane < NW)
                wsum[lane] = e;
            if (lane == NW - 1)
                *total = s;
        }
        __syncthreads();
        return wsum[w] + exc;
    }

    __global__ void __launch_bounds__(DSCAN_THREADS) k_dscan_tiles(
        const double* __restrict__ in, uint32_t n, double* __restrict__ part)
    {
        const size_t base = size_t(blockIdx.x) * DSCAN_TILE + size_t(threadIdx.x) * DSCAN_ITEMS;
        double s = 0.0;
        for (int k = 0; k < DSCAN_ITEMS; ++k)
            if (base + k < n)
                s += in[base + k];
        __shared__ double total;
        block_exclusive_scan_d(s, &total);
        if (threadIdx.x == 0)
            part[blockIdx.x] = total;
    }

    // exclusive scan of the tile sums in place (one block)
    __global__ void __launch_bounds__(DSCAN_THREADS) k_dscan_parts(double* part, uint32_t nparts)
    {
        const uint32_t per = (nparts + DSCAN_THREADS - 1) / DSCAN_THREADS;
        const uint32_t b = threadIdx.x * per;
        double s = 0.0;
        for (uint32_t k = 0; k < per && b + k < nparts; ++k)
            s += part[b + k];
        __shared__ double total;
        double run = block_exclusive_scan_d(s, &total);
        for (uint32_t k = 0; k < per && b + k < nparts; ++k) {
            const double t = part[b + k];
            part[b + k] = run;
            run += t;
        }
    }

    // inclusive output: the tile's offset, plus the thread's exclusive prefix,
    // plus its own running sum
    __global__ void __launch_bounds__(DSCAN_THREADS) k_dscan_apply(const double* __restrict__ in,
        uint32_t n, const double* __restrict__ part, double* __restrict__ out)
    {
        const size_t base = size_t(blockIdx.x) * DSCAN_TILE + size_t(threadIdx.x) * DSCAN_ITEMS;
        double s = 0.0;
        for (int k = 0; k < DSCAN_ITEMS; ++k)
            if (base + k < n)
                s += in[base + k];
        __shared__ double total;
        double run = part[blockIdx.x] + block_exclusive_scan_d(s, &total);
        for (int k = 0; k < DSCAN_ITEMS; ++k)
            if (base + k < n) {
                run += in[base + k];
                out[base + k] = run;
            }
    }

    inline uint32_t dscan_parts(uint32_t n) { return (n + DSCAN_TILE - 1) / DSCAN_TILE; }

    // inclusive scan of n doubles; `part` (dscan_parts(n) entries) holds the
    // tile sums and must outlive the enqueued kernels
    void inclusive_scan_d(const double* in, uint32_t n, double* part, double* out, cudaStream_t s)
    {
        const uint32_t nparts = dscan_parts(n);
        REYN_KERNEL("k_dscan_tiles", s,
            k_dscan_tiles<<<nparts, DSCAN_THREADS, 0, s>>>(in, n, part));
        REYN_KERNEL("k_dscan_parts", s, k_dscan_parts<<<1, DSCAN_THREADS, 0, s>>>(part, nparts));
        REYN_KERNEL("k_dscan_apply", s,
            k_dscan_apply<<<nparts, DSCAN_THREADS, 0, s>>>(in, n, part, out));
    }

    // ---- Morton codes and the radix sort ----------------------------------------
    __device__ __forceinline__ uint32_t quantise(double n)
    {
        return uint32_t(__double2float_rn(fmin(fmax(__dmul_rn(n, 1024.0), 0.0), 1023.0)));
    }

    // centroid Morton code of each face in the vertex bounds (lbvh.cuh:33-45,
    // 204-225): x, y, z bits interleaved with x highest
    __global__ void k_morton(uint32_t nf, const double* __restrict__ vx,
        const double* __restrict__ vy, const double* __restrict__ vz,
        const uint32_t* __restrict__ faces, double3 lo, double3 inv, uint32_t* __restrict__ codes,
        uint32_t* __restrict__ ids)
    {
        const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= nf)
            return;
        const D3 a = dload(faces[3 * size_t(t)], vx, vy, vz);
        const D3 b = dload(faces[3 * size_t(t) + 1], vx, vy, vz);
        const D3 c = dload(faces[3 * size_t(t) + 2], vx, vy, vz);
        const double third = 1.0 / 3.0;
        const double cx = __dsub_rn(__dmul_rn(__dadd_rn(__dadd_rn(a.x, b.x), c.x), third), lo.x);
        const double cy = __dsub_rn(__dmul_rn(__dadd_rn(__dadd_rn(a.y, b.y), c.y), third), lo.y);
        const double cz = __dsub_rn(__dmul_rn(__dadd_rn(__dadd_rn(a.z, b.z), c.z), third), lo.z);
        const uint32_t qx = quantise(__dmul_rn(cx, inv.x));
        const uint32_t qy = quantise(__dmul_rn(cy, inv.y));
        const uint32_t qz = quantise(__dmul_rn(cz, inv.z));
        codes[t] = (spread10(qx) << 2) | (spread10(qy) << 1) | spread10(qz);
        ids[t] = t;
    }

    // digit histogram of each tile, digit-major: hist[d * n_tiles + tile]
    __global__ void __launch_bounds__(RADIX_THREADS) k_radix_hist(uint32_t n,
        const uint32_t* __restrict__ keys, int shift, uint32_t n_tiles, uint32_t* __restrict__ hist)
    {
        __shared__ uint32_t h[RADIX_THREADS];
        h[threadIdx.x] = 0;
        __syncthreads();
        const size_t base = size_t(blockIdx.x) * RADIX_TILE;
        for (int it = 0; it < RADIX_ITEMS; ++it) {
            const size_t i = base + size_t(it) * RADIX_THREADS + threadIdx.x;
            if (i < n)
                atomicAdd(&h[(keys[i] >> shift) & 255u], 1u);
        }
        __syncthreads();
        hist[size_t(threadIdx.x) * n_tiles + blockIdx.x] = h[threadIdx.x];
    }

    // stable scatter of one tile: rounds of 256 keys in index order; inside a
    // round a key's rank is the number of earlier keys with its digit, from
    // its warp's match mask and the counts of the warps before it
    __global__ void __launch_bounds__(RADIX_THREADS) k_radix_scatter(uint32_t n,
        const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, int shift,
        uint32_t n_tiles, const uint32_t* __restrict__ offs, uint32_t* __restrict__ keys_out,
        uint32_t* __restrict__ vals_out)
    {
        constexpr int NW = RADIX_THREADS / 32;
        __shared__ uint32_t base[RADIX_THREADS];
        __shared__ uint32_t wcount[NW][RADIX_THREADS];
        const int t = threadIdx.x, lane = t & 31, w = t >> 5;
        base[t] = offs[size_t(t) * n_tiles + blockIdx.x];
        for (int k = 0; k < NW; ++k)
            wcount[k][t] = 0;
        __syncthreads();
        const size_t tile = size_t(blockIdx.x) * RADIX_TILE;
        for (int it = 0; it < RADIX_ITEMS; ++it) {
            const size_t i = tile + size_t(it) * RADIX_THREADS + t;
            const bool ok = i < n;
            const uint32_t key = ok ? keys_in[i] : 0u;
            // lanes past the end get distinct out-of-range digits
            const uint32_t dg = ok ? (key >> shift) & 255u : 256u + uint32_t(lane);
            const uint32_t peers = __match_any_sync(0xffffffffu, dg);
            const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
            if (ok && rank == 0)
                wcount[w][dg] = __popc(peers);
            __syncthreads();
            if (ok) {
                uint32_t pos = base[dg] + rank;
                for (int k = 0; k < w; ++k)
                    pos += wcount[k][dg];
                keys_out[pos] = key;
                vals_out[pos] = vals_in[i];
            }
            __syncthreads();
            uint32_t add = 0;
            for (int k = 0; k < NW; ++k) {
                add += wcount[k][t];
                wcount[k][t] = 0;
            }
            base[t] += add;
            __syncthreads();
        }
    }

    // 256-byte aligned sub-arrays of one device allocation: add() the sizes,
    // allocate bytes, then take the pointers at the returned offsets
    struct Carve {
        size_t bytes = 0;
        template <class T> size_t add(size_t n)
        {
            const size_t o = (bytes + 255) & ~size_t(255);
            bytes = o + std::max<size_t>(n, 1) * sizeof(T);
            return o;
        }
    };
    template <class T> T* at(const DevArray<unsigned char>& a, size_t off)
    {
        return reinterpret_cast<T*>(a.get() + off);
    }

    inline uint32_t radix_tiles(uint32_t n) { return (n + RADIX_TILE - 1) / RADIX_TILE; }

    // scratch of the radix sort of n pairs (all must outlive the kernels):
    // k2, v2: n each; hist: 256 radix_tiles(n); offs: that + 1
    struct SortBufs {
        uint32_t *k2, *v2, *hist, *offs;
    };
    struct SortLayout {
        size_t k2, v2, hist, offs;
        SortLayout(Carve& c, uint32_t n)
            : k2(c.add<uint32_t>(n))
            , v2(c.add<uint32_t>(n))
            , hist(c.add<uint32_t>(size_t(radix_tiles(n)) * 256))
            , offs(c.add<uint32_t>(size_t(radix_tiles(n)) * 256 + 1))
        {
        }
        SortBufs at(const DevArray<unsigned char>& a) const
        {
            return SortBufs { reyn::at<uint32_t>(a, k2), reyn::at<uint32_t>(a, v2),
                reyn::at<uint32_t>(a, hist), reyn::at<uint32_t>(a, offs) };
        }
    };

    // sorts (keys, vals) by the 32 key bits, stably; results in place
    void radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t n, const SortBufs& w,
        DevArray<uint32_t>& part, cudaStream_t s)
    {
        const uint32_t n_tiles = radix_tiles(n);
        uint32_t *ka = keys, *va = vals, *kb = w.k2, *vb = w.v2;
        for (int shift = 0; shift < 32; shift += 8) {
            REYN_KERNEL("k_radix_hist", s,
                k_radix_hist<<<n_tiles, RADIX_THREADS, 0, s>>>(n, ka, shift, n_tiles, w.hist));
            exclusive_scan(w.hist, int64_t(n_tiles) * 256, part, w.offs, s);
            REYN_KERNEL("k_radix_scatter", s,
                k_radix_scatter<<<n_tiles, RADIX_THREADS, 0, s>>>(n, ka, va, shift, n_tiles, w.offs,
                kb, vb));
            std::swap(ka, kb);
            std::swap(va, vb);
        }
        // four passes: the result is back in the caller's arrays
    }

    // ---- the tree (Karras 2012) ---------------------------------------------------
    // length of the common prefix of the unique keys (code << 32 | index) of
    // leaves i and j; -1 outside [0, n)
    __device__ __forceinline__ int prefix_len(const uint32_t* __restrict__ codes, int n, int i, int j)
    {
        if (j < 0 || j >= n)
            return -1;
        const uint64_t ki = (uint64_t(codes[i]) << 32) | uint32_t(i);
        const uint64_t kj = (uint64_t(codes[j]) << 32) | uint32_t(j);
        return __clzll(ki ^ kj);
    }

    // internal node i (lbvh.cu:34-75): its key range has i at one end; the
    // split is the last leaf of the range sharing more than the range's common
    // prefix with its first leaf
    __global__ void k_karras(uint32_t nf, const uint32_t* __restrict__ codes,
        uint32_t* __restrict__ cl, uint32_t* __restrict__ cr, uint32_t* __restrict__ parent_node,
        uint32_t* __restrict__ parent_leaf)
    {
        const int n = int(nf);
        const int i = int(blockIdx.x * blockDim.x + threadIdx.x);
        if (i >= n - 1)
            return;
        int first = 0, last = n - 1;
        if (i > 0) {
            const int d = prefix_len(codes, n, i, i + 1) > prefix_len(codes, n, i, i - 1) ? 1 : -1;
            const int dmin = prefix_len(codes, n, i, i - d);
            int lmax = 2;
            while (prefix_len(codes, n, i, i + lmax * d) > dmin)
                lmax <<= 1;
            int l = 0;
            for (int t = lmax >> 1; t >= 1; t >>= 1)
                if (prefix_len(codes, n, i, i + (l + t) * d) > dmin)
                    l += t;
            const int j = i + l * d;
            first = min(i, j);
            last = max(i, j);
        }
        const int common = prefix_len(codes, n, first, last);
        int split = first, step = last - first;
        do {
            step = (step + 1) >> 1;
            const int s = split + step;
            if (s < last && prefix_len(codes, n, first, s) > common)
                split = s;
        } while (step > 1);
        const bool l_leaf = split == first, r_leaf = split + 1 == last;
        cl[i] = (uint32_t(split) << 1) | (l_leaf ? 0u : 1u);
        cr[i] = (uint32_t(split + 1) << 1) | (r_leaf ? 0u : 1u);
        (l_leaf ? parent_leaf : parent_node)[split] = uint32_t(i);
        (r_leaf ? parent_leaf : parent_node)[split + 1] = uint32_t(i);
    }

    __device__ __forceinline__ Box pad_if_flat(Box b)
    {
        // zero extent along an axis: pad by FLT_EPSILON (lbvh.cu:20-31)
        const float ex = __fsub_rn(b.hi[0], b.lo[0]), ey = __fsub_rn(b.hi[1], b.lo[1]),
                    ez = __fsub_rn(b.hi[2], b.lo[2]);
        if (fminf(ex, fminf(ey, ez)) == 0.f) {
            for (int k = 0; k < 3; ++k) {
                b.lo[k] = __fsub_rn(b.lo[k], FLT_EPSILON);
                b.hi[k] = __fadd_rn(b.hi[k], FLT_EPSILON);
            }
        }
        return b;
    }

    // the union, padded when flat (the reference's union pads its left operand
    // instead, lbvh.cuh:58-68, which drops the right one)
    __device__ __forceinline__ Box unite(const Box& a, const Box& b)
    {
        Box u;
        for (int k = 0; k < 3; ++k) {
            u.lo[k] = fminf(a.lo[k], b.lo[k]);
            u.hi[k] = fmaxf(a.hi[k], b.hi[k]);
        }
        return pad_if_flat(u);
    }

    __device__ __forceinline__ Box load_box_cg(const Box* p)
    {
        const float* f = reinterpret_cast<const float*>(p);
        Box b;
        for (int k = 0; k < 3; ++k) {
            b.lo[k] = __ldcg(f + k);
            b.hi[k] = __ldcg(f + 3 + k);
        }
        return b;
    }

    // leaf boxes, then internal boxes bottom-up: the second child to arrive at
    // a node unites both boxes and climbs on (lbvh.cu:77-150)
    __global__ void k_lbvh_boxes(uint32_t nf, const uint32_t* __restrict__ order,
        const double* __restrict__ vx, const double* __restrict__ vy,
        const double* __restrict__ vz, const uint32_t* __restrict__ faces,
        const uint32_t* __restrict__ parent_node, const uint32_t* __restrict__ parent_leaf,
        const uint32_t* __restrict__ cl, const uint32_t* __restrict__ cr, uint32_t* visit,
        Box* leaf_box, Box* node_box, uint32_t* status)
    {
        const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
        if (j >= nf)
            return;
        const uint32_t f = order[j];
        const D3 a = dload(faces[3 * size_t(f)], vx, vy, vz);
        const D3 b = dload(faces[3 * size_t(f) + 1], vx, vy, vz);
        const D3 c = dload(faces[3 * size_t(f) + 2], vx, vy, vz);
        Box bx;
        bx.lo[0] = __double2float_rn(fmin(fmin(a.x, b.x), c.x));
        bx.lo[1] = __double2float_rn(fmin(fmin(a.y, b.y), c.y));
        bx.lo[2] = __double2float_rn(fmin(fmin(a.z, b.z), c.z));
        bx.hi[0] = __double2float_rn(fmax(fmax(a.x, b.x), c.x));
        bx.hi[1] = __double2float_rn(fmax(fmax(a.y, b.y), c.y));
        bx.hi[2] = __double2float_rn(fmax(fmax(a.z, b.z), c.z));
        bx = pad_if_flat(bx);
        leaf_box[j] = bx;
        if (nf < 2)
            return;
        uint32_t node = parent_leaf[j];
        uint32_t me = j << 1; // this subtree as a child link
        for (uint32_t guard = 0; guard < nf; ++guard) {
            if (node >= nf - 1) {
                atomicOr(status, MESH_BAD_TREE);
                return;
            }
            __threadfence();
            if (atomicAdd(visit + node, 1u) == 0)
                return; // the sibling finishes this node
            __threadfence();
            const uint32_t l = cl[node], r = cr[node];
            const uint32_t other = (l == me) ? r : l;
            if ((other >> 1) >= ((other & 1u) ? nf - 1 : nf)) {
                atomicOr(status, MESH_BAD_TREE);
                return;
            }
            const Box ob = load_box_cg(((other & 1u) ? node_box : leaf_box) + (other >> 1));
            bx = unite(bx, ob);
            node_box[node] = bx;
            if (node == 0)
                return;
            me = (node << 1) | 1u;
            node = parent_node[node];
        }
    }

    // traversal records: internal nodes with their children's boxes, leaves
    // with their triangle's float vertices
    __global__ void k_lbvh_pack(uint32_t nf, const uint32_t* __restrict__ order,
        const double* __restrict__ vx, const double* __restrict__ vy,
        const double* __restrict__ vz, const uint32_t* __restrict__ faces,
        const uint32_t* __restrict__ cl, const uint32_t* __restrict__ cr,
        const Box* __restrict__ leaf_box, const Box* __restrict__ node_box, Node* __restrict__ nodes,
        float4* __restrict__ tri, uint32_t* status)
    {
        const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
        if (j >= nf)
            return;
        const uint32_t f = order[j];
        float v[9];
        for (int k = 0; k < 3; ++k) {
            const uint32_t q = faces[3 * size_t(f) + k];
            v[3 * k] = __double2float_rn(vx[q]);
            v[3 * k + 1] = __double2float_rn(vy[q]);
            v[3 * k + 2] = __double2float_rn(vz[q]);
        }
        tri[3 * size_t(j)] = make_float4(v[0], v[1], v[2], v[3]);
        tri[3 * size_t(j) + 1] = make_float4(v[4], v[5], v[6], v[7]);
        tri[3 * size_t(j) + 2] = make_float4(v[8], 0.f, 0.f, 0.f);
        if (j + 1 >= nf)
            return;
        const uint32_t l = cl[j], r = cr[j];
        if ((l >> 1) >= ((l & 1u) ? nf - 1 : nf) || (r >> 1) >= ((r & 1u) ? nf - 1 : nf)) {
            atomicOr(status, MESH_BAD_TREE);
            return;
        }
        const Box L = ((l & 1u) ? node_box : leaf_box)[l >> 1];
        const Box R = ((r & 1u) ? node_box : leaf_box)[r >> 1];
        Node nd;
        nd.a = make_float4(L.lo[0], L.lo[1], L.lo[2], L.hi[0]);
        nd.b = make_float4(L.hi[1], L.hi[2], R.lo[0], R.lo[1]);
        nd.c = make_float4(R.lo[2], R.hi[0], R.hi[1], R.hi[2]);
        nd.d = make_uint4(l, r, 0u, 0u);
        nodes[j] = nd;
    }

    // edges from the root to each leaf (lbvh.cu:152-170), maximum
    __global__ void k_lbvh_height(uint32_t nf, const uint32_t* __restrict__ parent_node,
        const uint32_t* __restrict__ parent_leaf, uint32_t* height)
    {
        const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
        if (j >= nf || nf < 2)
            return;
        uint32_t p = parent_leaf[j], depth = 1;
        for (uint32_t k = 0; p != 0 && k < nf; ++k) {
            if (p >= nf - 1)
                break; // a malformed tree; the boxes pass has flagged it
            p = parent_node[p];
            ++depth;
        }
        atomicMax(height, depth);
    }

    // ---- sampling (sample_boundary.cu:168-248) ------------------------------------
    __global__ void k_mesh_sample(uint32_t n, uint32_t nf, const double* __restrict__ cdf,
        double area, double bin, uint64_t seed, const double* __restrict__ vx,
        const double* __restrict__ vy, const double* __restrict__ vz,
        const uint32_t* __restrict__ faces, float* __restrict__ x, float* __restrict__ y,
        float* __restrict__ z)
    {
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i >= n)
            return;
        // stratified position along the summed area: stratum i of n, uniform
        // inside it (stream 8)
        const double at = __dadd_rn(__dmul_rn(__ddiv_rn(double(i), double(n)), area),
            __dmul_rn(bin, uniform_open0(seed, 8, i)));
        // the first face whose inclusive area sum reaches it
        uint32_t lo = 0, hi = nf;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (cdf[mid] < at)
                lo = mid + 1;
            else
                hi = mid;
        }
        const uint32_t t = min(lo, nf - 1);
        const D3 a = dload(faces[3 * size_t(t)], vx, vy, vz);
        const D3 b = dload(faces[3 * size_t(t) + 1], vx, vy, vz);
        const D3 c = dload(faces[3 * size_t(t) + 2], vx, vy, vz);
        // a uniform point of the parallelogram, folded into the triangle
        // (streams 9, 10)
        double u = uniform_open0(seed, 9, i), v = uniform_open0(seed, 10, i);
        if (!(__dadd_rn(u, v) <= 1.0)) {
            u = __dsub_rn(1.0, u);
            v = __dsub_rn(1.0, v);
        }
        const D3 ab = dsub(b, a), ac = dsub(c, a);
        x[i] = __double2float_rn(__dadd_rn(__dadd_rn(a.x, __dmul_rn(ab.x, u)), __dmul_rn(ac.x, v)));
        y[i] = __double2float_rn(__dadd_rn(__dadd_rn(a.y, __dmul_rn(ab.y, u)), __dmul_rn(ac.y, v)));
        z[i] = __double2float_rn(__dadd_rn(__dadd_rn(a.z, __dmul_rn(ab.z, u)), __dmul_rn(ac.z, v)));
    }

    // ---- relaxation (sample_boundary.cu:20-71, 100-166) ----------------------------
    __global__ void k_relax_gather(uint32_t n, const uint32_t* __restrict__ perm,
        const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
        float4* __restrict__ pts)
    {
        const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
        if (s >= n)
            return;
        const uint32_t p = perm[s];
        pts[s] = make_float4(x[p], y[p], z[p], 0.f);
    }

    // number density: sum of W over all samples within 2 h_bdy, self included
    template <int R>
    __global__ void __launch_bounds__(MESH_THREADS) k_relax_density(uint32_t n, GridView g,
        KernelConst kc, const float4* __restrict__ pts, float* __restrict__ nd,
        uint32_t* __restrict__ status)
    {
        const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
        if (s >= n)
            return;
        const float4 me = pts[s];
        int3 c = cell_of(g, me.x, me.y, me.z);
        if (!cell_inside(g, c, R)) {
            atomicOr(status, STATUS_OUT_OF_GRID);
            c = clamp_cell(g, c, R);
        }
        float sum = 0.f;
        for_each_neighbour<R>(g, c, me.x, me.y, me.z, pts,
            [&](uint32_t, const float4&, float, float, float, float l2) {
                sum += pair_w<K_B3>(kc, l2);
            });
        nd[s] = sum;
    }

    // x_i - k h^2 sum_j (n_i + n_j) / rho0^2 grad W_ij, from the old positions
    template <int R>
    __global__ void __launch_bounds__(MESH_THREADS) k_relax_shift(uint32_t n, GridView g,
        KernelConst kc, const float4* __restrict__ pts, const float* __restrict__ nd,
        float inv_rho0_sq, float coef, const uint32_t* __restrict__ perm, float4* __restrict__ moved,
        float* __restrict__ nd_out)
    {
        const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
        if (s >= n)
            return;
        const float4 me = pts[s];
        const int3 c = clamp_cell(g, cell_of(g, me.x, me.y, me.z), R);
        const float ti = inv_rho0_sq * nd[s];
        float ax = 0.f, ay = 0.f, az = 0.f;
        for_each_neighbour<R>(g, c, me.x, me.y, me.z, pts,
            [&](uint32_t j, const float4&, float dx, float dy, float dz, float l2) {
                const float w = (ti + inv_rho0_sq * __ldg(nd + j)) * pair_g<K_B3>(kc, l2);
                ax = fmaf(w, dx, ax);
                ay = fmaf(w, dy, ay);
                az = fmaf(w, dz, az);
            });
        moved[s] = make_float4(fmaf(coef, ax, me.x), fmaf(coef, ay, me.y), fmaf(coef, az, me.z), 0.f);
        if (nd_out)
            nd_out[perm[s]] = nd[s];
    }

    __device__ __forceinline__ unsigned fbits(float f) { return __float_as_uint(f); }

    // min, max (as ordered bits of positive floats) and sum of number densities
    __global__ void k_relax_stats(uint32_t n, const float* __restrict__ nd, unsigned* __restrict__ mn,
        unsigned* __restrict__ mx, double* __restrict__ sum)
    {
        const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
        float v = s < n ? nd[s] : 0.f;
        float lo = s < n ? v : FLT_MAX, hi = v;
        double acc = v;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
            hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
            acc += __shfl_xor_sync(0xffffffffu, acc, o);
        }
        if ((threadIdx.x & 31) == 0 && s - (threadIdx.x & 31) < n) {
            atomicMin(mn, fbits(fmaxf(lo, 0.f)));
            atomicMax(mx, fbits(fmaxf(hi, 0.f)));
            atomicAdd(sum, acc);
        }
    }

    // ---- fluid fill (scene.cu:336-425) ------------------------------------------------
    struct Lattice {
        float3 lo;
        float h;
        uint32_t nx, ny;
    };
    __device__ __forceinline__ V3 lattice_point(const Lattice& L, uint32_t g)
    {
        const uint32_t i = g % L.nx, j = (g / L.nx) % L.ny, k = g / (L.nx * L.ny);
        return mk3(__fadd_rn(L.lo.x, __fmul_rn(float(i), L.h)),
            __fadd_rn(L.lo.y, __fmul_rn(float(j), L.h)), __fadd_rn(L.lo.z, __fmul_rn(float(k), L.h)));
    }

    template <int STACK>
    __global__ void __launch_bounds__(MESH_THREADS) k_fill_flag(
        uint32_t total, Lattice L, MeshView m, uint32_t* __restrict__ keep)
    {
        const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
        if (g >= total)
            return;
        keep[g] = closest<STACK, true>(m, lattice_point(L, g)).inside ? 1u : 0u;
    }

    __global__ void k_fill_write(uint32_t total, Lattice L, const uint32_t* __restrict__ keep,
        const uint32_t* __restrict__ pos, uint32_t cap, float a, uint64_t seed,
        float* __restrict__ x, float* __restrict__ y, float* __restrict__ z)
    {
        const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
        if (g >= total || !keep[g] || pos[g] >= cap)
            return;
        V3 p = lattice_point(L, g);
        if (a > 0.f) {
            p.x = __fadd_rn(p.x, symmetric(uniform01(seed, 0, g), a));
            p.y = __fadd_rn(p.y, symmetric(uniform01(seed, 1, g), a));
            p.z = __fadd_rn(p.z, symmetric(uniform01(seed, 2, g), a));
        }
        const uint32_t o = pos[g];
        x[o] = p.x;
        y[o] = p.y;
        z[o] = p.z;
    }

    // scratch of a query batch in Morton order (kept by the mesh, so that
    // the asynchronous queries never outlive it)
    struct QueryScratch {
        DevArray<unsigned char> buf; // codes, ids, pts, sort buffers
        DevArray<uint32_t> part;
        uint32_t cap = 0;
        uint32_t *codes = nullptr, *ids = nullptr;
        float4* pts = nullptr;
        SortBufs sort {};
        void reserve(uint32_t n)
        {
            if (n <= cap)
                return;
            Carve c;
            const size_t oc = c.add<uint32_t>(n), oi = c.add<uint32_t>(n), op = c.add<float4>(n);
            const SortLayout sl(c, n);
            buf.resize(c.bytes);
            codes = at<uint32_t>(buf, oc);
            ids = at<uint32_t>(buf, oi);
            pts = at<float4>(buf, op);
            sort = sl.at(buf);
            cap = n;
        }
    };

    // below this many points a query batch runs in the caller's order
    constexpr uint32_t QUERY_SORT_MIN = 1u << 15;

} // namespace
} // namespace reyn

using namespace reyn;

struct reyn_mesh {
    uint32_t nv = 0, nf = 0;
    DevArray<unsigned char> store; // one allocation holding every array below
    double *vx = nullptr, *vy = nullptr, *vz = nullptr;
    uint32_t* faces = nullptr;     // 3 per face, original order
    double* cdf = nullptr;         // inclusive area sums, original face order
    double area = 0.0, volume = 0.0;
    double lo[3] = { 0, 0, 0 }, hi[3] = { 0, 0, 0 };
    // the LBVH
    uint32_t* order = nullptr;     // original face of each leaf
    uint32_t *cl = nullptr, *cr = nullptr; // children of each internal node
    Box *leaf_box = nullptr, *node_box = nullptr;
    Node* nodes = nullptr;
    float4* tri = nullptr;
    uint32_t* status = nullptr;
    Box root {};
    uint32_t height = 0;
    mutable QueryScratch query;
    // the relaxation's uniform grid (rebuilt for another spacing) and its
    // scratch, kept for the next call: a surface's grid spans the mesh's box
    // at cell 2 h_bdy and can take a gigabyte, whose allocation would
    // otherwise dominate a call
    mutable std::unique_ptr<Grid> relax_grid;
    mutable float relax_r = 0.f;
    mutable DevArray<unsigned char> relax_tmp;

    void allocate()
    {
        const size_t ni = std::max<uint32_t>(nf - 1, 1);
        Carve c;
        const size_t o_vx = c.add<double>(nv), o_vy = c.add<double>(nv), o_vz = c.add<double>(nv);
        const size_t o_f = c.add<uint32_t>(3 * size_t(nf)), o_cdf = c.add<double>(nf);
        const size_t o_ord = c.add<uint32_t>(nf), o_cl = c.add<uint32_t>(ni),
                     o_cr = c.add<uint32_t>(ni);
        const size_t o_lb = c.add<Box>(nf), o_nb = c.add<Box>(ni), o_n = c.add<Node>(ni),
                     o_t = c.add<float4>(3 * size_t(nf)), o_s = c.add<uint32_t>(1);
        store.resize(c.bytes);
        vx = at<double>(store, o_vx);
        vy = at<double>(store, o_vy);
        vz = at<double>(store, o_vz);
        faces = at<uint32_t>(store, o_f);
        cdf = at<double>(store, o_cdf);
        order = at<uint32_t>(store, o_ord);
        cl = at<uint32_t>(store, o_cl);
        cr = at<uint32_t>(store, o_cr);
        leaf_box = at<Box>(store, o_lb);
        node_box = at<Box>(store, o_nb);
        nodes = at<Node>(store, o_n);
        tri = at<float4>(store, o_t);
        status = at<uint32_t>(store, o_s);
    }

    MeshView view() const { return MeshView { nodes, tri, nf - 1, root, status }; }
    int stack() const { return height + 2 <= 32 ? 32 : 64; }
};

namespace {

template <bool INSIDE>
void launch_query(const reyn_mesh& m, uint32_t n, const float4* src, const uint32_t* perm,
    const float* xin, const float* yin, const float* zin, float* x, float* y, float* z,
    uint8_t* inside, cudaStream_t s)
{
    if (!n)
        return;
    if (!src && n >= QUERY_SORT_MIN) {
        // queries in Morton order: the lanes of a warp then walk nearly the
        // same nodes, where random order makes each warp wait for its
        // costliest lane; results go back to the callers' slots
        QueryScratch& q = m.query;
        q.reserve(n);
        float lo[3], sc[3];
        for (int k = 0; k < 3; ++k) {
            lo[k] = float(m.lo[k]);
            const double ext = m.hi[k] - m.lo[k];
            sc[k] = ext > 0.0 ? float(1024.0 / ext) : 0.f;
        }
        REYN_KERNEL("k_query_keys", s,
            k_query_keys<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, xin, yin, zin,
            make_float3(lo[0], lo[1], lo[2]), make_float3(sc[0], sc[1], sc[2]), q.codes,
            q.ids));
        radix_sort_pairs(q.codes, q.ids, n, q.sort, q.part, s);
        REYN_KERNEL("k_query_gather", s,
            k_query_gather<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, q.ids, xin, yin, zin,
            q.pts));
        src = q.pts;
        perm = q.ids;
    }
    const unsigned b = blocks_for(n, MESH_THREADS);
    if (m.stack() == 32)
        REYN_KERNEL(INSIDE ? "k_mesh_inside" : "k_mesh_project", s,
            k_mesh_query<32, INSIDE><<<b, MESH_THREADS, 0, s>>>(n, m.view(), src, perm, xin, yin,
            zin, x, y, z, inside));
    else
        REYN_KERNEL(INSIDE ? "k_mesh_inside" : "k_mesh_project", s,
            k_mesh_query<64, INSIDE><<<b, MESH_THREADS, 0, s>>>(n, m.view(), src, perm, xin, yin,
            zin, x, y, z, inside));
}

void check_traversal(const reyn_mesh& m, cudaStream_t s)
{
    uint32_t st = 0;
    REYN_CUDA(cudaMemcpyAsync(&st, m.status, sizeof(st), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaStreamSynchronize(s));
    if (st)
        fail(REYN_ERR_CUDA, (st & MESH_BAD_TREE) ? "LBVH traversal met a malformed tree"
                                                 : "LBVH traversal stack exhausted");
}

void build_mesh(reyn_mesh& m, cudaStream_t s)
{
    const uint32_t nf = m.nf;
    const uint32_t ni = nf > 1 ? nf - 1 : 0;
    // the build's temporaries, one allocation
    Carve c;
    const size_t o_area = c.add<double>(nf), o_vol = c.add<double>(nf), o_vsum = c.add<double>(nf);
    const size_t o_pa = c.add<double>(dscan_parts(nf)), o_pv = c.add<double>(dscan_parts(nf));
    const size_t o_codes = c.add<uint32_t>(nf);
    const SortLayout sl(c, nf);
    const size_t o_pn = c.add<uint32_t>(std::max<uint32_t>(ni, 1)), o_pl = c.add<uint32_t>(nf);
    const size_t o_visit = c.add<uint32_t>(std::max<uint32_t>(ni, 1)), o_h = c.add<uint32_t>(1);
    DevArray<unsigned char> tmp(c.bytes);
    DevArray<uint32_t> part;
    double* area = at<double>(tmp, o_area);
    double* vol = at<double>(tmp, o_vol);
    double* vsum = at<double>(tmp, o_vsum);
    uint32_t* codes = at<uint32_t>(tmp, o_codes);
    uint32_t* parent_node = at<uint32_t>(tmp, o_pn);
    uint32_t* parent_leaf = at<uint32_t>(tmp, o_pl);
    uint32_t* visit = at<uint32_t>(tmp, o_visit);
    uint32_t* height = at<uint32_t>(tmp, o_h);
    REYN_CUDA(cudaMemsetAsync(visit, 0, std::max<uint32_t>(ni, 1) * sizeof(uint32_t), s));
    REYN_CUDA(cudaMemsetAsync(height, 0, sizeof(uint32_t), s));
    REYN_CUDA(cudaMemsetAsync(m.status, 0, sizeof(uint32_t), s));
    // areas, volume, sampling CDF
    REYN_KERNEL("k_face_measure", s,
        k_face_measure<<<blocks_for(nf, THREADS), THREADS, 0, s>>>(nf, m.vx, m.vy, m.vz, m.faces,
        area, vol));
    inclusive_scan_d(area, nf, at<double>(tmp, o_pa), m.cdf, s);
    inclusive_scan_d(vol, nf, at<double>(tmp, o_pv), vsum, s);
    // Morton codes, sorted with the face ids
    const double3 lo = make_double3(m.lo[0], m.lo[1], m.lo[2]);
    const double3 inv = make_double3(1.0 / (m.hi[0] - m.lo[0]), 1.0 / (m.hi[1] - m.lo[1]),
        1.0 / (m.hi[2] - m.lo[2]));
    REYN_KERNEL("k_morton", s,
        k_morton<<<blocks_for(nf, THREADS), THREADS, 0, s>>>(nf, m.vx, m.vy, m.vz, m.faces, lo, inv,
        codes, m.order));
    radix_sort_pairs(codes, m.order, nf, sl.at(tmp), part, s);
    // tree, boxes, traversal records, height
    if (ni)
        REYN_KERNEL("k_karras", s,
            k_karras<<<blocks_for(ni, THREADS), THREADS, 0, s>>>(nf, codes, m.cl, m.cr, parent_node,
            parent_leaf));
    REYN_KERNEL("k_lbvh_boxes", s,
        k_lbvh_boxes<<<blocks_for(nf, THREADS), THREADS, 0, s>>>(nf, m.order, m.vx, m.vy, m.vz,
        m.faces, parent_node, parent_leaf, m.cl, m.cr, visit, m.leaf_box, m.node_box, m.status));
    REYN_KERNEL("k_lbvh_pack", s,
        k_lbvh_pack<<<blocks_for(nf, THREADS), THREADS, 0, s>>>(nf, m.order, m.vx, m.vy, m.vz,
        m.faces, m.cl, m.cr, m.leaf_box, m.node_box, m.nodes, m.tri, m.status));
    REYN_KERNEL("k_lbvh_height", s,
        k_lbvh_height<<<blocks_for(nf, THREADS), THREADS, 0, s>>>(nf, parent_node, parent_leaf,
        height));
    // one readback: totals, height, root box, status
    double tot[2];
    uint32_t st = 0;
    REYN_CUDA(cudaMemcpyAsync(&tot[0], m.cdf + nf - 1, sizeof(double), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaMemcpyAsync(&tot[1], vsum + nf - 1, sizeof(double), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaMemcpyAsync(&m.height, height, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaMemcpyAsync(&m.root, ni ? m.node_box : m.leaf_box, sizeof(Box),
        cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaMemcpyAsync(&st, m.status, sizeof(st), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaStreamSynchronize(s));
    m.area = tot[0];
    m.volume = std::fabs(tot[1]) / 6.0;
    if (st)
        fail(REYN_ERR_CUDA, "LBVH construction produced a malformed tree");
    if (m.height + 2 > 64)
        fail(REYN_ERR_INVALID, "LBVH deeper than 62 levels");
}

std::string lower(std::string v)
{
    for (char& c : v)
        c = char(std::tolower(static_cast<unsigned char>(c)));
    return v;
}

// a Wavefront OBJ reader for triangle meshes (the subset load_mesh_from_obj
// uses, loader.cpp): vertices, triangles, shape names from "o" and "g"
void read_obj(const char* path, const std::vector<std::string>& ignore, const char* only,
    std::vector<double>& vx, std::vector<double>& vy, std::vector<double>& vz,
    std::vector<uint32_t>& faces)
{
    std::ifstream in(path);
    if (!in)
        fail(REYN_ERR_INVALID, std::string("cannot open mesh file ") + path);
    const std::string only_l = only ? lower(only) : std::string();
    std::string line, shape;
    bool keep = !only;
    auto decide = [&] {
        const std::string name = lower(shape);
        keep = !only || name.find(only_l) != std::string::npos;
        for (const std::string& ig : ignore)
            if (name.find(lower(ig)) != std::string::npos)
                keep = false;
    };
    decide();
    uint64_t lineno = 0;
    while (std::getline(in, line)) {
        ++lineno;
        const size_t hash = line.find('#');
        if (hash != std::string::npos)
            line.resize(hash);
        std::istringstream ls(line);
        std::string tag;
        if (!(ls >> tag))
            continue;
        if (tag == "v") {
            double c[3];
            if (!(ls >> c[0] >> c[1] >> c[2]))
                fail(REYN_ERR_INVALID, "malformed vertex in " + std::string(path) + " line "
                    + std::to_string(lineno));
            vx.push_back(c[0]);
            vy.push_back(c[1]);
            vz.push_back(c[2]);
        } else if (tag == "o" || tag == "g") {
            std::getline(ls >> std::ws, shape);
            while (!shape.empty() && std::isspace(static_cast<unsigned char>(shape.back())))
                shape.pop_back();
            decide();
        } else if (tag == "f") {
            std::string tok;
            uint32_t idx[3];
            int k = 0;
            while (ls >> tok) {
                if (k == 3)
                    fail(REYN_ERR_INVALID, "non-triangulated face in " + std::string(path) + " line "
                        + std::to_string(lineno));
                const long v = std::stol(tok.substr(0, tok.find('/')));
                const long nvert = long(vx.size());
                const long r = v > 0 ? v - 1 : nvert + v; // negative: relative to the end
                if (v == 0 || r < 0 || r >= nvert)
                    fail(REYN_ERR_INVALID, "face index out of range in " + std::string(path)
                        + " line " + std::to_string(lineno));
                idx[k++] = uint32_t(r);
            }
            if (k != 3)
                fail(REYN_ERR_INVALID, "face with fewer than 3 vertices in " + std::string(path));
            if (keep)
                faces.insert(faces.end(), idx, idx + 3);
        }
    }
}

void create_mesh(const double* vx, const double* vy, const double* vz, uint32_t nv,
    const uint32_t* faces, uint32_t nf, cudaStream_t s, reyn_mesh** out)
{
    require(out != nullptr, "null output handle");
    *out = nullptr;
    require(vx && vy && vz && faces, "null mesh array");
    require(nv > 0 && nf > 0, "a mesh needs vertices and faces");
    require(nf < MAX_FACES, "at most 2^30 faces");
    auto m = std::make_unique<reyn_mesh>();
    m->nv = nv;
    m->nf = nf;
    for (int k = 0; k < 3; ++k) {
        m->lo[k] = INFINITY;
        m->hi[k] = -INFINITY;
    }
    const double* v[3] = { vx, vy, vz };
    for (uint32_t i = 0; i < nv; ++i)
        for (int k = 0; k < 3; ++k) {
            require(std::isfinite(v[k][i]), "vertex coordinates must be finite");
            m->lo[k] = std::fmin(m->lo[k], v[k][i]);
            m->hi[k] = std::fmax(m->hi[k], v[k][i]);
        }
    for (uint64_t i = 0; i < 3ull * nf; ++i)
        require(faces[i] < nv, "face vertex index out of range");
    m->allocate();
    REYN_CUDA(cudaMemcpyAsync(m->vx, vx, nv * sizeof(double), cudaMemcpyHostToDevice, s));
    REYN_CUDA(cudaMemcpyAsync(m->vy, vy, nv * sizeof(double), cudaMemcpyHostToDevice, s));
    REYN_CUDA(cudaMemcpyAsync(m->vz, vz, nv * sizeof(double), cudaMemcpyHostToDevice, s));
    REYN_CUDA(cudaMemcpyAsync(m->faces, faces, 3 * size_t(nf) * sizeof(uint32_t),
        cudaMemcpyHostToDevice, s));
    build_mesh(*m, s);
    *out = m.release();
}

// the relaxation's rest density: B3 at support 2 h_bdy summed over a 5x5
// patch of the hexagonal lattice of spacing h_bdy (sample_boundary.cu:78-98)
float hex_plane_density(float h_bdy)
{
    const KernelConst kc = make_kernel(K_B3, 2.f * h_bdy);
    const float qa[3] = { h_bdy, 0.f, 0.f };
    const float ra[3] = { h_bdy * 0.5f, h_bdy * float(std::sqrt(3.0) * 0.5), 0.f };
    float rho = 0.f;
    for (int q = -2; q <= 2; ++q)
        for (int r = -2; r <= 2; ++r) {
            float d[3];
            for (int k = 0; k < 3; ++k)
                d[k] = float(q) * qa[k] + float(r) * ra[k];
            const float len = std::sqrt(std::fmaf(d[0], d[0], std::fmaf(d[1], d[1], d[2] * d[2])));
            rho += kc.w_scale * Shape<K_B3>::w(sat01(len * kc.h_inv));
        }
    return rho;
}

} // namespace

extern "C" int reyn_mesh_create(const double* vx, const double* vy, const double* vz,
    uint32_t n_vertices, const uint32_t* faces, uint32_t n_faces, void* stream, reyn_mesh** out)
{
    return guard([&] { create_mesh(vx, vy, vz, n_vertices, faces, n_faces, as_stream(stream), out); });
}

extern "C" int reyn_mesh_load_obj(const char* path, const char* const* ignore, uint32_t n_ignore,
    const char* only, void* stream, reyn_mesh** out)
{
    return guard([&] {
        require(path && out, "null argument");
        require(n_ignore == 0 || ignore, "null ignore list");
        std::vector<std::string> ig;
        for (uint32_t k = 0; k < n_ignore; ++k) {
            require(ignore[k] != nullptr, "null ignore entry");
            ig.emplace_back(ignore[k]);
        }
        std::vector<double> vx, vy, vz;
        std::vector<uint32_t> f;
        read_obj(path, ig, only, vx, vy, vz, f);
        require(!f.empty(), "the mesh file holds no (kept) faces");
        require(vx.size() < (size_t(1) << 32), "too many vertices");
        create_mesh(vx.data(), vy.data(), vz.data(), uint32_t(vx.size()), f.data(),
            uint32_t(f.size() / 3), as_stream(stream), out);
    });
}

extern "C" int reyn_mesh_destroy(reyn_mesh* mesh)
{
    delete mesh;
    return REYN_OK;
}

extern "C" int reyn_mesh_info_get(const reyn_mesh* mesh, reyn_mesh_info* out)
{
    return guard([&] {
        require(mesh && out, "null argument");
        reyn_mesh_info r {};
        r.n_vertices = mesh->nv;
        r.n_faces = mesh->nf;
        r.tree_height = mesh->height;
        for (int k = 0; k < 3; ++k) {
            r.bounds_min[k] = mesh->lo[k];
            r.bounds_max[k] = mesh->hi[k];
        }
        r.area = mesh->area;
        r.volume = mesh->volume;
        *out = r;
    });
}

extern "C" int reyn_mesh_tree(const reyn_mesh* mesh, uint32_t* order, uint32_t* children_l,
    uint32_t* children_r, float* leaf_box, float* node_box, void* stream)
{
    return guard([&] {
        require(mesh != nullptr, "null mesh");
        const cudaStream_t s = as_stream(stream);
        const size_t nf = mesh->nf, ni = nf - 1;
        auto copy = [&](void* dst, const void* src, size_t bytes) {
            if (dst && bytes)
                REYN_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
        };
        copy(order, mesh->order, nf * sizeof(uint32_t));
        copy(children_l, mesh->cl, ni * sizeof(uint32_t));
        copy(children_r, mesh->cr, ni * sizeof(uint32_t));
        copy(leaf_box, mesh->leaf_box, nf * sizeof(Box));
        copy(node_box, mesh->node_box, ni * sizeof(Box));
    });
}

extern "C" int reyn_mesh_project(const reyn_mesh* mesh, float* x, float* y, float* z, uint32_t n,
    void* stream)
{
    return guard([&] {
        require(mesh != nullptr, "null mesh");
        require(n == 0 || (x && y && z), "null point array");
        launch_query<false>(*mesh, n, nullptr, nullptr, x, y, z, x, y, z, nullptr,
            as_stream(stream));
    });
}

extern "C" int reyn_mesh_inside(const reyn_mesh* mesh, const float* x, const float* y,
    const float* z, uint32_t n, uint8_t* inside, void* stream)
{
    return guard([&] {
        require(mesh != nullptr, "null mesh");
        require(n == 0 || (x && y && z && inside), "null array");
        launch_query<true>(*mesh, n, nullptr, nullptr, x, y, z, nullptr, nullptr, nullptr, inside,
            as_stream(stream));
    });
}

extern "C" int reyn_mesh_sample_uniform(const reyn_mesh* mesh, float h, float oversampling,
    uint64_t seed, float* x, float* y, float* z, uint32_t capacity, uint32_t* count, void* stream)
{
    return guard([&] {
        require(mesh && count, "null argument");
        require(h > 0.f && oversampling > 0.f && std::isfinite(h) && std::isfinite(oversampling),
            "h and oversampling must be positive");
        require(mesh->area > 0.0, "the mesh has no area");
        // sample_boundary.cu:339-346: hexagonal packing of the surface
        const double h_bdy = double(h) / double(oversampling);
        const float per = 1.5f * std::sqrt(3.f) * float(h_bdy) * float(h_bdy);
        const double nd = std::ceil(mesh->area / double(per));
        require(nd < 4.0e9, "too many samples");
        const uint32_t n = uint32_t(nd);
        *count = n;
        if (!x)
            return; // size query
        require(y && z, "null output array");
        require(capacity >= n, "output arrays hold fewer samples than the mesh needs");
        const cudaStream_t s = as_stream(stream);
        REYN_KERNEL("k_mesh_sample", s,
            k_mesh_sample<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, mesh->nf, mesh->cdf,
            mesh->area, mesh->area / double(n), seed, mesh->vx, mesh->vy,
            mesh->vz, mesh->faces, x, y, z));
    });
}

extern "C" int reyn_mesh_relax(const reyn_mesh* mesh, float* x, float* y, float* z, uint32_t n,
    float h_bdy, float relaxation_factor, uint32_t iters, float* stats, float* num_den,
    void* stream)
{
    return guard([&] {
        require(mesh != nullptr, "null mesh");
        require(n == 0 || (x && y && z), "null point array");
        require(h_bdy > 0.f && std::isfinite(h_bdy), "h_bdy must be positive");
        require(std::isfinite(relaxation_factor), "relaxation factor must be finite");
        if (!iters || !n)
            return; // sample_boundary.cu:106-107
        const cudaStream_t s = as_stream(stream);
        // a grid of cell 2 h_bdy over the mesh bounds: projected samples lie
        // inside them, and the grid adds its own 2r margin
        if (!mesh->relax_grid || mesh->relax_r != 2.f * h_bdy) {
            auto ng = std::make_unique<Grid>();
            float bmin[3], bmax[3];
            for (int k = 0; k < 3; ++k) {
                bmin[k] = float(mesh->lo[k]);
                bmax[k] = float(mesh->hi[k]);
            }
            ng->geom = make_geom(bmin, bmax, 2.f * h_bdy, 1.0f);
            ng->ratio = 1.0f;
            require(ng->geom.range == 1, "unexpected relaxation grid range");
            mesh->relax_grid.reset(); // the old grid's memory first
            mesh->relax_grid = std::move(ng);
            mesh->relax_r = 2.f * h_bdy;
        }
        Grid& g = *mesh->relax_grid;
        const KernelConst kc = make_kernel(K_B3, 2.f * h_bdy);
        const float rho0 = hex_plane_density(h_bdy);
        const float inv2 = 1.f / (rho0 * rho0);
        const float coef = (-relaxation_factor * h_bdy) * h_bdy;
        Carve c;
        const size_t o_pts = c.add<float4>(n), o_mv = c.add<float4>(n), o_nd = c.add<float>(n);
        const size_t o_mm = c.add<unsigned>(2 * size_t(iters)), o_sum = c.add<double>(iters);
        const size_t o_st = c.add<uint32_t>(1);
        DevArray<unsigned char>& tmp = mesh->relax_tmp;
        tmp.resize(c.bytes);
        float4* pts = at<float4>(tmp, o_pts);
        float4* moved = at<float4>(tmp, o_mv);
        float* nd = at<float>(tmp, o_nd);
        unsigned* mnmx = at<unsigned>(tmp, o_mm);
        double* sums = at<double>(tmp, o_sum);
        uint32_t* status = at<uint32_t>(tmp, o_st);
        REYN_CUDA(cudaMemsetAsync(status, 0, sizeof(uint32_t), s));
        REYN_CUDA(cudaMemsetAsync(sums, 0, iters * sizeof(double), s));
        {
            std::vector<unsigned> init(2 * size_t(iters));
            const float big = FLT_MAX;
            for (uint32_t it = 0; it < iters; ++it) {
                std::memcpy(&init[2 * it], &big, sizeof(float));
                init[2 * it + 1] = 0u;
            }
            REYN_CUDA(cudaMemcpyAsync(mnmx, init.data(), init.size() * sizeof(unsigned),
                cudaMemcpyHostToDevice, s));
            REYN_CUDA(cudaStreamSynchronize(s)); // `init` leaves scope
        }
        const unsigned b = blocks_for(n, MESH_THREADS);
        for (uint32_t it = 0; it < iters; ++it) {
            g.build(x, y, z, n, s);
            const GridView v = g.view(g.geom.r);
            REYN_KERNEL("k_relax_gather", s,
                k_relax_gather<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, g.sorted.get(), x, y, z,
                pts));
            REYN_KERNEL("k_relax_density", s,
                k_relax_density<1><<<b, MESH_THREADS, 0, s>>>(n, v, kc, pts, nd,
                status));
            REYN_KERNEL("k_relax_stats", s,
                k_relax_stats<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, nd,
                mnmx + 2 * it, mnmx + 2 * it + 1, sums + it));
            REYN_KERNEL("k_relax_shift", s,
                k_relax_shift<1><<<b, MESH_THREADS, 0, s>>>(n, v, kc, pts, nd, inv2, coef,
                g.sorted.get(), moved, it + 1 == iters ? num_den : nullptr));
            // back onto the mesh, in grid order, results to the samples' slots
            launch_query<false>(*mesh, n, moved, g.sorted.get(), nullptr, nullptr, nullptr, x, y,
                z, nullptr, s);
        }
        std::vector<unsigned> mm(2 * size_t(iters));
        std::vector<double> sm(iters);
        uint32_t st = 0;
        REYN_CUDA(cudaMemcpyAsync(mm.data(), mnmx, mm.size() * sizeof(unsigned),
            cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaMemcpyAsync(sm.data(), sums, sm.size() * sizeof(double),
            cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaMemcpyAsync(&st, status, sizeof(st), cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaStreamSynchronize(s));
        check_traversal(*mesh, s);
        if (st)
            fail(REYN_ERR_OUT_OF_BOUNDS, "a sample left the relaxation grid");
        if (stats)
            for (uint32_t it = 0; it < iters; ++it) {
                float lo, hi;
                std::memcpy(&lo, &mm[2 * it], sizeof(float));
                std::memcpy(&hi, &mm[2 * it + 1], sizeof(float));
                stats[2 * it] = hi / lo;
                stats[2 * it + 1] = float(sm[it] / double(n));
            }
    });
}

extern "C" int reyn_mesh_fill(const reyn_mesh* mesh, float h, float jitter, uint64_t seed, float* x,
    float* y, float* z, uint32_t capacity, uint32_t* count, void* stream)
{
    return guard([&] {
        require(mesh && count, "null argument");
        require(h > 0.f && std::isfinite(h), "h must be positive");
        require(jitter >= 0.f && std::isfinite(jitter), "jitter must be >= 0");
        require(!x || (y && z), "null output array");
        const cudaStream_t s = as_stream(stream);
        // scene.cu:336-351: the lattice spans the mesh's float bounds
        Lattice L;
        L.lo = make_float3(float(mesh->lo[0]), float(mesh->lo[1]), float(mesh->lo[2]));
        L.h = h;
        const float hi[3] = { float(mesh->hi[0]), float(mesh->hi[1]), float(mesh->hi[2]) };
        const float lo[3] = { L.lo.x, L.lo.y, L.lo.z };
        int64_t cnt[3];
        for (int k = 0; k < 3; ++k)
            cnt[k] = std::max<int64_t>(0, int64_t(std::floor((hi[k] - lo[k]) / h)));
        const int64_t total = cnt[0] * cnt[1] * cnt[2];
        require(total < int64_t(UINT32_MAX), "more than 2^32 - 1 lattice candidates");
        L.nx = uint32_t(cnt[0]);
        L.ny = uint32_t(cnt[1]);
        *count = 0;
        if (!total)
            return;
        const uint32_t T = uint32_t(total);
        DevArray<uint32_t> keep(T), pos(size_t(T) + 1), part;
        const MeshView mv = mesh->view();
        const unsigned b = blocks_for(T, MESH_THREADS);
        if (mesh->stack() == 32)
            REYN_KERNEL("k_fill_flag", s,
                k_fill_flag<32><<<b, MESH_THREADS, 0, s>>>(T, L, mv, keep.get()));
        else
            REYN_KERNEL("k_fill_flag", s,
                k_fill_flag<64><<<b, MESH_THREADS, 0, s>>>(T, L, mv, keep.get()));
        exclusive_scan(keep.get(), T, part, pos.get(), s);
        uint32_t kept = 0;
        REYN_CUDA(cudaMemcpyAsync(&kept, pos.get() + T, sizeof(kept), cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaStreamSynchronize(s));
        check_traversal(*mesh, s);
        *count = kept;
        if (!x)
            return; // size query
        require(capacity >= kept, "output arrays hold fewer points than the fill keeps");
        REYN_KERNEL("k_fill_write", s,
            k_fill_write<<<blocks_for(T, THREADS), THREADS, 0, s>>>(T, L, keep.get(), pos.get(),
            capacity, jitter * h, seed, x, y, z));
        REYN_CUDA(cudaStreamSynchronize(s)); // keep/pos are freed on return
    });
}
