// On-device scene generation: fluid blocks on a jittered cubic lattice, box
// walls and Fibonacci spheres sampled with boundary particles, and the
// removal of fluid particles that lie too close to the boundary. The
// reference builds its scenes with _init_box_kernel (scene.cu:14-37), a
// thrust jitter pass (scene.cu:232-253) and a thrust remove_if against the
// boundary grid (scene.cu:59-83, 176-205); here each is one kernel writing
// straight into the caller's arrays.
//
// Random numbers are counter-based: value k of stream t under seed s is
// SplitMix64 (Steele, Lea, Flood 2014) applied to s + 0x9E3779B97F4A7C15 *
// (t * 2^40 + k + 1); its top 24 bits make an exact float in [0, 1). So a
// particle's jitter depends only on (seed, its index), never on launch
// shape, and a host restatement reproduces every value bit for bit. All
// position arithmetic is explicitly rounded for the same reason.
#include "engine.cuh"

#include <cmath>

namespace reyn {


// lattice + jitter (_init_box_kernel, scene.cu:14-37, x fastest): particle
// first + q of the block sits at origin + (i, j, k) h + jitter, jitter
// uniform in [-jitter h, jitter h] per axis (streams 0..2), velocity uniform
// in [-vnoise, vnoise] per axis (streams 3..5)
__global__ void k_fluid_block(uint32_t count, uint32_t first, uint3 n, float3 origin, float h,
    float mass, float jitter, float vnoise, uint64_t seed, float* __restrict__ x,
    float* __restrict__ y, float* __restrict__ z, float* __restrict__ vx,
    float* __restrict__ vy, float* __restrict__ vz, float* __restrict__ m)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count)
        return;
    const uint32_t i = q % n.x, j = (q / n.x) % n.y, k = q / (n.x * n.y);
    const uint64_t g = uint64_t(first) + q; // stream position: the particle index
    float px = __fadd_rn(origin.x, __fmul_rn(float(i), h));
    float py = __fadd_rn(origin.y, __fmul_rn(float(j), h));
    float pz = __fadd_rn(origin.z, __fmul_rn(float(k), h));
    if (jitter != 0.f) {
        const float a = __fmul_rn(jitter, h);
        px = __fadd_rn(px, symmetric(uniform01(seed, 0, g), a));
        py = __fadd_rn(py, symmetric(uniform01(seed, 1, g), a));
        pz = __fadd_rn(pz, symmetric(uniform01(seed, 2, g), a));
    }
    float ux = 0.f, uy = 0.f, uz = 0.f;
    if (vnoise != 0.f) {
        ux = symmetric(uniform01(seed, 3, g), vnoise);
        uy = symmetric(uniform01(seed, 4, g), vnoise);
        uz = symmetric(uniform01(seed, 5, g), vnoise);
    }
    const uint32_t o = first + q;
    x[o] = px;
    y[o] = py;
    z[o] = pz;
    vx[o] = ux;
    vy[o] = uy;
    vz[o] = uz;
    m[o] = mass;
}

// Box walls: one layer of samples on the six faces of [lo, hi] on a square
// lattice of n = rint((hi - lo) / spacing) intervals per axis, no duplicates
// at edges and corners. Sample order: the x faces (x = lo, then hi; all j,
// k), the y faces (interior i, all k), the z faces (interior i and j); inside
// a face the first index runs slowest. Sample (i, j, k) sits at lo + (i, j,
// k) * step, step = (hi - lo) / n per axis, in float arithmetic.
struct WallSpec {
    int3 n;
    float3 lo, step;
    uint64_t face_end[6]; // cumulative sample counts of the six faces
};

__host__ __device__ __forceinline__ uint64_t wall_face_size(const int3 n, int f)
{
    const int64_t nx = n.x + 1, ny = n.y + 1, nz = n.z + 1;
    if (f < 2)
        return uint64_t(ny * nz);
    if (f < 4)
        return uint64_t((nx - 2) * nz);
    return uint64_t((nx - 2) * (ny - 2));
}

__global__ void k_box_walls(uint64_t total, WallSpec w, float* __restrict__ x,
    float* __restrict__ y, float* __restrict__ z)
{
    const uint64_t q = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (q >= total)
        return;
    int f = 0;
    while (q >= w.face_end[f])
        ++f;
    const uint64_t r = q - (f ? w.face_end[f - 1] : 0);
    int i, j, k;
    if (f < 2) { // x faces: j slow, k fast
        i = f == 0 ? 0 : w.n.x;
        j = int(r / uint64_t(w.n.z + 1));
        k = int(r % uint64_t(w.n.z + 1));
    } else if (f < 4) { // y faces: interior i slow, k fast
        j = f == 2 ? 0 : w.n.y;
        i = 1 + int(r / uint64_t(w.n.z + 1));
        k = int(r % uint64_t(w.n.z + 1));
    } else { // z faces: interior i slow, interior j fast
        k = f == 4 ? 0 : w.n.z;
        i = 1 + int(r / uint64_t(w.n.y - 1));
        j = 1 + int(r % uint64_t(w.n.y - 1));
    }
    x[q] = __fadd_rn(w.lo.x, __fmul_rn(float(i), w.step.x));
    y[q] = __fadd_rn(w.lo.y, __fmul_rn(float(j), w.step.y));
    z[q] = __fadd_rn(w.lo.z, __fmul_rn(float(k), w.step.z));
}

// Fibonacci sphere: n points of the golden-angle spiral on a sphere of
// radius rad, n = max(1, rint(4 pi rad^2 / spacing^2)) (one sample per
// spacing^2 of area). Point k: height t_k = 1 - (2k + 1) / n along y, ring
// radius sqrt(1 - t_k^2), azimuth k * pi (3 - sqrt 5).
__global__ void k_sphere(uint32_t n, float3 c, float rad, float* __restrict__ x,
    float* __restrict__ y, float* __restrict__ z)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n)
        return;
    const double golden = 3.14159265358979323846 * (3.0 - 2.2360679774997896964);
    const double t = 1.0 - (2.0 * k + 1.0) / double(n);
    const double ring = sqrt(fmax(0.0, 1.0 - t * t));
    double sn, cs;
    sincos(golden * double(k), &sn, &cs);
    x[k] = float(double(c.x) + double(rad) * ring * cs);
    y[k] = float(double(c.y) + double(rad) * t);
    z[k] = float(double(c.z) + double(rad) * ring * sn);
}

// keep[i] = 1 unless a boundary sample lies within `radius` of particle i
// (CullPredicate, scene.cu:59-83)
__global__ void k_cull_mark(uint32_t n, const float* __restrict__ x, const float* __restrict__ y,
    const float* __restrict__ z, GridView bg, const float4* __restrict__ bpm,
    const uint8_t* __restrict__ near, float r2, uint32_t* __restrict__ keep)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float px = x[i], py = y[i], pz = z[i];
    uint32_t hit = 0;
    const int3 c = cell_of(bg, px, py, pz);
    if (cell_inside(bg, c, 2) && near[c.z * bg.nxny + c.y * bg.nx + c.x]) {
        for_each_neighbour<2>(bg, c, px, py, pz, bpm,
            [&](uint32_t, const float4&, float, float, float, float l2) {
                hit |= l2 <= r2 ? 1u : 0u;
            });
    }
    keep[i] = hit ? 0u : 1u;
}

// stable compaction of the seven state arrays by keep/prefix
__global__ void k_cull_scatter(uint32_t n, const uint32_t* __restrict__ keep,
    const uint32_t* __restrict__ pos, GatherArgs a)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !keep[i])
        return;
    const uint32_t o = pos[i];
#pragma unroll
    for (int k = 0; k < NFIELDS; ++k)
        a.dst[k][o] = a.src[k][i];
}

// jitter_positions (scene.cu:232-253) with the counter-based streams 0..2 of
// the fluid blocks: particle q of [first, first + count) moves by a uniform
// [-a, a] per axis, keyed by its index
__global__ void k_jitter(uint32_t count, uint32_t first, float a, uint64_t seed,
    float* __restrict__ x, float* __restrict__ y, float* __restrict__ z)
{
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count)
        return;
    const uint32_t o = first + q;
    x[o] = __fadd_rn(x[o], symmetric(uniform01(seed, 0, o), a));
    y[o] = __fadd_rn(y[o], symmetric(uniform01(seed, 1, o), a));
    z[o] = __fadd_rn(z[o], symmetric(uniform01(seed, 2, o), a));
}

} // namespace reyn

using namespace reyn;

extern "C" int reyn_scene_jitter(reyn_particles* p, uint32_t first, uint32_t count,
    float amplitude, uint64_t seed, void* stream)
{
    return guard([&] {
        require(p != nullptr, "null particles");
        require(amplitude >= 0.f && std::isfinite(amplitude), "amplitude must be >= 0");
        require(uint64_t(first) + count <= p->n, "range does not fit the particle state");
        if (!count || amplitude == 0.f)
            return;
        const cudaStream_t s = as_stream(stream);
        REYN_KERNEL("k_jitter", s,
            k_jitter<<<blocks_for(count, THREADS), THREADS, 0, s>>>(count, first, amplitude,
            seed, p->cur[FX].get(), p->cur[FY].get(), p->cur[FZ].get()));
        p->packed_valid = false;
        p->version += 1;
    });
}

extern "C" int reyn_scene_fluid_block(reyn_particles* p, uint32_t first, const uint32_t counts[3],
    const float origin[3], float spacing, float mass, float jitter, float velocity_noise,
    uint64_t seed, void* stream)
{
    return guard([&] {
        require(p && counts && origin, "null argument");
        require(spacing > 0.f && std::isfinite(spacing), "spacing must be positive");
        require(std::isfinite(origin[0]) && std::isfinite(origin[1]) && std::isfinite(origin[2]),
            "origin must be finite");
        require(jitter >= 0.f && velocity_noise >= 0.f, "jitter and noise must be >= 0");
        const uint64_t count = uint64_t(counts[0]) * counts[1] * counts[2];
        require(uint64_t(first) + count <= p->n, "block does not fit the particle state");
        if (!(mass > 0.f)) // the reference's rest mass rho0 h^3 (scene.cu:36)
            mass = p->rho0 * spacing * spacing * spacing;
        if (!count)
            return;
        const cudaStream_t s = as_stream(stream);
        REYN_KERNEL("k_fluid_block", s,
            k_fluid_block<<<blocks_for(uint32_t(count), THREADS), THREADS, 0, s>>>(
            uint32_t(count), first, make_uint3(counts[0], counts[1], counts[2]),
            make_float3(origin[0], origin[1], origin[2]), spacing, mass, jitter,
            velocity_noise, seed, p->cur[FX].get(), p->cur[FY].get(), p->cur[FZ].get(),
            p->cur[FVX].get(), p->cur[FVY].get(), p->cur[FVZ].get(), p->cur[FM].get()));
        p->packed_valid = false;
        p->version += 1;
    });
}

extern "C" int reyn_scene_box_walls(const float bound_min[3], const float bound_max[3],
    float spacing, float* x, float* y, float* z, uint64_t capacity, uint64_t* count,
    void* stream)
{
    return guard([&] {
        require(bound_min && bound_max && count, "null argument");
        require(spacing > 0.f && std::isfinite(spacing), "spacing must be positive");
        WallSpec w {};
        int n[3];
        for (int a = 0; a < 3; ++a) {
            const float ext = bound_max[a] - bound_min[a];
            require(std::isfinite(ext) && ext > 0.f, "box must have a positive extent");
            n[a] = int(std::nearbyint(double(ext) / double(spacing)));
            require(n[a] >= 2 && n[a] < (1 << 24), "box must span 2 .. 2^24 spacings");
        }
        w.n = make_int3(n[0], n[1], n[2]);
        w.lo = make_float3(bound_min[0], bound_min[1], bound_min[2]);
        w.step = make_float3((bound_max[0] - bound_min[0]) / float(n[0]),
            (bound_max[1] - bound_min[1]) / float(n[1]), (bound_max[2] - bound_min[2]) / float(n[2]));
        uint64_t total = 0;
        for (int f = 0; f < 6; ++f) {
            total += wall_face_size(w.n, f);
            w.face_end[f] = total;
        }
        *count = total;
        if (!x)
            return; // size query
        require(y && z, "null output array");
        require(capacity >= total, "output arrays hold fewer samples than the walls need");
        const cudaStream_t s = as_stream(stream);
        const unsigned blocks = unsigned((total + THREADS - 1) / THREADS);
        REYN_KERNEL("k_box_walls", s, k_box_walls<<<blocks, THREADS, 0, s>>>(total, w, x, y, z));
    });
}

extern "C" int reyn_scene_sphere(const float center[3], float radius, float spacing, float* x,
    float* y, float* z, uint32_t capacity, uint32_t* count, void* stream)
{
    return guard([&] {
        require(center && count, "null argument");
        require(radius > 0.f && spacing > 0.f && std::isfinite(radius) && std::isfinite(spacing),
            "radius and spacing must be positive");
        const double area = 4.0 * 3.14159265358979323846 * double(radius) * double(radius);
        const double nd = std::max(1.0, std::nearbyint(area / (double(spacing) * spacing)));
        require(nd < 4.0e9, "too many sphere samples");
        const uint32_t n = uint32_t(nd);
        *count = n;
        if (!x)
            return; // size query
        require(y && z, "null output array");
        require(capacity >= n, "output arrays hold fewer samples than the sphere needs");
        const cudaStream_t s = as_stream(stream);
        REYN_KERNEL("k_sphere", s,
            k_sphere<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n,
            make_float3(center[0], center[1], center[2]), radius, x, y, z));
    });
}

extern "C" int reyn_scene_cull(reyn_particles* p, const reyn_boundary* bdy, float radius,
    uint32_t* n_out, void* stream)
{
    return guard([&] {
        require(p && bdy, "null argument");
        require(radius >= 0.f && radius <= bdy->grid.geom.r,
            "cull radius must lie in [0, the boundary grid's search radius 2h]");
        const cudaStream_t s = as_stream(stream);
        const uint32_t n = p->n;
        if (n && bdy->nb) {
            DevArray<uint32_t> keep(n), pos(size_t(n) + 1), part;
            REYN_KERNEL("k_cull_mark", s,
                k_cull_mark<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, p->cur[FX].get(),
                p->cur[FY].get(), p->cur[FZ].get(), bdy->view(), bdy->pm.get(), bdy->near.get(),
                radius * radius, keep.get()));
            exclusive_scan(keep.get(), n, part, pos.get(), s);
            GatherArgs a {};
            for (int k = 0; k < NFIELDS; ++k) {
                p->alt[k].resize(n);
                a.src[k] = p->cur[k].get();
                a.dst[k] = p->alt[k].get();
            }
            a.count = NFIELDS;
            REYN_KERNEL("k_cull_scatter", s,
                k_cull_scatter<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, keep.get(),
                pos.get(), a));
            uint32_t kept = 0;
            REYN_CUDA(cudaMemcpyAsync(&kept, pos.get() + n, sizeof(kept), cudaMemcpyDeviceToHost, s));
            REYN_CUDA(cudaStreamSynchronize(s));
            for (int k = 0; k < NFIELDS; ++k)
                p->cur[k].swap(p->alt[k]);
            p->n = kept;
            p->packed_valid = false;
            p->version += 1;
        }
        if (n_out)
            *n_out = p->n;
    });
}
