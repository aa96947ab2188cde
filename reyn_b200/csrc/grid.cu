// Uniform-grid build on the B200: cell keys + warp-aggregated histogram,
// tiled prefix scan over all cells, counting-sort scatter, a canonicalising
// pass that makes the order inside each cell ascending (deterministic), and
// one fused gather that permutes every particle array and writes the packed
// (x, y, z, m) / (v, rho) copies the neighbour loops read.
//
// Reference: UniformGridBuilder (uniformgrid.cu:20-181, uniformgrid.cuh:
// 200-489). The reference's scatter slot comes from atomicSub and is
// nondeterministic inside a cell (uniformgrid.cu:59); here the final slot is
// the rank of the particle index inside its cell, i.e. the canonical form.
#include "engine.cuh"

#include <cmath>
#include <vector>

namespace reyn {

// ---- geometry -------------------------------------------------------------

GridGeom make_geom(const float bmin[3], const float bmax[3], float r, float ratio, int order)
{
    require(r > 0.f && std::isfinite(r), "search radius must be positive and finite");
    require(ratio == 0.5f || ratio == 1.0f, "cell_ratio must be 0.5 or 1.0");
    GridGeom g {};
    // uniformgrid.cu:69-80: cell = r/2, lower bound min - 2r,
    // n = ceil(((max + 2r) - lower) / cell), in float
    g.cell = ratio == 0.5f ? r / 2.f : r;
    g.r = r;
    g.range = ratio == 0.5f ? 2 : 1;
    const float margin = (float)(r * 2.);
    for (int a = 0; a < 3; ++a) {
        require(std::isfinite(bmin[a]) && std::isfinite(bmax[a]), "bounds must be finite");
        require(bmax[a] >= bmin[a], "bound_max must not be below bound_min");
        g.lo[a] = bmin[a] - margin;
        const float n = std::ceil(((bmax[a] + margin) - g.lo[a]) / g.cell);
        require(n > 0.f && n < 2.0e9f, "grid extent out of range");
        g.n[a] = (int)n;
    }
    require(order == REYN_ORDER_XYZ || order == REYN_ORDER_ZORDER, "unknown cell order");
    g.order = order;
    for (int a = 0; a < 3; ++a)
        g.t[a] = (g.n[a] + ZTILE - 1) / ZTILE;
    require(g.keys() < (int64_t(1) << 32) - 1, "grid has too many cells for 32-bit keys");
    return g;
}

GridView Grid::view(float search_radius) const
{
    GridView v;
    v.lox = geom.lo[0];
    v.loy = geom.lo[1];
    v.loz = geom.lo[2];
    v.cell = geom.cell;
    v.inv_cell = 1.f / geom.cell;
    v.r2 = search_radius * search_radius;
    v.nx = geom.n[0];
    v.ny = geom.n[1];
    v.nz = geom.n[2];
    v.nxny = geom.n[0] * geom.n[1];
    v.order = geom.order;
    v.tx = geom.t[0];
    v.txy = geom.t[0] * geom.t[1];
    v.prefix = prefix.get();
    v.sid = n_scenes ? sid.get() : nullptr;
    v.scenes = n_scenes ? scene_tab.get() : nullptr;
    v.key_base = 0;
    return v;
}

} // namespace reyn

reyn::GridView reyn_boundary::view() const { return grid.view(grid.geom.r); }

namespace reyn {

// ---- kernels --------------------------------------------------------------

// cell key of every particle + histogram (uniformgrid.cu:20-34). Lanes with
// equal keys are merged with match_any so that one atomic serves the group.
__global__ void k_keys_count(uint32_t n, const float* __restrict__ x,
    const float* __restrict__ y, const float* __restrict__ z, GridView g,
    uint32_t* __restrict__ keys, uint32_t* __restrict__ counts,
    uint32_t* __restrict__ status)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    uint32_t key = 0xffffffffu;
    if (valid) {
        const float px = x[i], py = y[i], pz = z[i];
        g = at_scene(g, scene_of(g, i)); // batched: the point's own scene grid
        int3 c = cell_of(g, px, py, pz);
        const bool finite = isfinite(px) && isfinite(py) && isfinite(pz);
        const bool inside = finite && c.x >= 0 && c.y >= 0 && c.z >= 0
            && c.x < g.nx && c.y < g.ny && c.z < g.nz;
        if (!inside) {
            atomicOr(status, finite ? STATUS_OUT_OF_GRID : STATUS_NONFINITE);
            c = finite ? make_int3(min(max(c.x, 0), g.nx - 1), min(max(c.y, 0), g.ny - 1),
                             min(max(c.z, 0), g.nz - 1))
                       : make_int3(0, 0, 0);
        }
        key = cell_key(g, c.x, c.y, c.z) + g.key_base;
        keys[i] = key;
    }
    const unsigned group = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    if (valid && lane == __ffs(group) - 1)
        atomicAdd(counts + key, (uint32_t)__popc(group));
}

// counting-sort scatter (uniformgrid.cu:40-63): slot = prefix[key] + a
// unique offset from atomicSub, which also returns `counts` to zero
__global__ void k_scatter(uint32_t n, const uint32_t* __restrict__ keys,
    const uint32_t* __restrict__ prefix, uint32_t* __restrict__ counts,
    uint32_t* __restrict__ slots)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const uint32_t key = valid ? keys[i] : 0xffffffffu;
    const unsigned group = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(group) - 1;
    uint32_t top = 0;
    if (valid && lane == leader)
        top = atomicSub(counts + key, (uint32_t)__popc(group));
    top = __shfl_sync(0xffffffffu, top, leader);
    if (valid) {
        const uint32_t rank = __popc(group & ((1u << lane) - 1u));
        slots[prefix[key] + top - __popc(group) + rank] = i;
    }
}

// canonical order inside each cell: the final slot of particle p is the
// start of its cell plus the number of smaller indices in the same cell
__global__ void k_canonical(uint32_t n, const uint32_t* __restrict__ slots,
    const uint32_t* __restrict__ keys, const uint32_t* __restrict__ prefix,
    uint32_t* __restrict__ sorted)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const uint32_t p = slots[s];
    const uint32_t key = keys[p];
    const uint32_t st = prefix[key], en = prefix[key + 1];
    if (en - st == 1) {
        sorted[st] = p;
        return;
    }
    uint32_t rank = 0;
    for (uint32_t t = st; t < en; ++t)
        rank += (slots[t] < p) ? 1u : 0u;
    sorted[st + rank] = p;
}

// counting-sort scatter straight into the canonical order (uniformgrid.cu:
// 40-63, with the order inside a cell made deterministic: ascending index).
// A warp's lanes hold consecutive indices, so a cell whose particles all lie
// in one warp (its count, prefix[key + 1] - prefix[key], equals the number of
// lanes holding its key) is placed by lane rank; the leader returns the
// cell's counter to zero. A cell split across warps takes counting-sort
// slots (atomicSub, which also returns its counter to zero) into `slots`,
// and its particles are listed in `split` (count in *nsplit) for
// k_rank_split. In a state reordered by the previous step's grid nearly
// every cell is whole. Blocks of THREADS threads.
__global__ void __launch_bounds__(THREADS) k_scatter_stable(uint32_t n,
    const uint32_t* __restrict__ keys,
    const uint32_t* __restrict__ prefix, uint32_t* __restrict__ counts,
    uint32_t* __restrict__ slots, uint32_t* __restrict__ sorted, uint32_t* __restrict__ split,
    uint32_t* __restrict__ nsplit)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < n;
    const uint32_t key = valid ? keys[i] : 0xffffffffu;
    const unsigned group = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(group) - 1;
    const uint32_t g = __popc(group);
    const uint32_t rank = __popc(group & ((1u << lane) - 1u));
    uint32_t st = 0, tot = 0;
    if (valid) {
        st = prefix[key];
        tot = prefix[key + 1] - st;
    }
    const bool whole = valid && g == tot;
    uint32_t top = 0;
    if (valid && lane == leader) {
        if (whole)
            counts[key] = 0u;
        else
            top = atomicSub(counts + key, g);
    }
    top = __shfl_sync(0xffffffffu, top, leader);
    if (valid) {
        if (whole)
            sorted[st + rank] = i;
        else
            slots[st + top - g + rank] = i;
    }
    // the split list: one atomic per block that has split cells (after a
    // developed flow's step a few percent of the particles land in cells
    // whose other particles sit in another warp; an atomic per warp then
    // serialises on the one counter)
    if (!__syncthreads_or(valid && !whole))
        return; // the block holds no particle of a split cell
    const unsigned sm = __ballot_sync(0xffffffffu, valid && !whole);
    __shared__ uint32_t warp_base[THREADS / 32];
    __shared__ uint32_t block_base;
    const int w = threadIdx.x >> 5;
    if (lane == 0)
        warp_base[w] = __popc(sm);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t tot = 0;
        for (int k = 0; k < int(blockDim.x >> 5); ++k) {
            const uint32_t c = warp_base[k];
            warp_base[k] = tot;
            tot += c;
        }
        block_base = atomicAdd(nsplit, tot);
    }
    __syncthreads();
    if (valid && !whole)
        split[block_base + warp_base[w] + __popc(sm & ((1u << lane) - 1u))] = i;
}

// the canonical place of each particle of a split cell: its cell's start plus
// the number of smaller indices among the cell's slots (grid-stride over the
// split list, whose length is known on the device only)
__global__ void k_rank_split(const uint32_t* __restrict__ nsplit,
    const uint32_t* __restrict__ split, const uint32_t* __restrict__ slots,
    const uint32_t* __restrict__ keys, const uint32_t* __restrict__ prefix,
    uint32_t* __restrict__ sorted)
{
    const uint32_t m = *nsplit;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        const uint32_t p = split[t];
        const uint32_t key = keys[p];
        const uint32_t st = prefix[key], en = prefix[key + 1];
        uint32_t rank = 0;
        for (uint32_t q = st; q < en; ++q)
            rank += (slots[q] < p) ? 1u : 0u;
        sorted[st + rank] = p;
    }
}

// ---- exclusive scan over all cells ----------------------------------------
// Two passes over tiles of SCAN_TILE counts: the tile sums, then the tile
// scans with their offsets. The last entry prefix[C] receives the total.
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_PER_THREAD = 16;
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_PER_THREAD;

__device__ __forceinline__ void load_tile_chunk(const uint32_t* __restrict__ in,
    int64_t C, int64_t base, uint32_t v[SCAN_PER_THREAD])
{
    if (base + SCAN_PER_THREAD <= C) {
        const uint4* q = reinterpret_cast<const uint4*>(in + base);
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD / 4; ++k) {
            const uint4 u = q[k];
            v[4 * k] = u.x;
            v[4 * k + 1] = u.y;
            v[4 * k + 2] = u.z;
            v[4 * k + 3] = u.w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; ++k)
            v[k] = (base + k < C) ? in[base + k] : 0u;
    }
}

// block-wide exclusive scan of one value per thread; returns the prefix and
// writes the block total to *total
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total)
{
    __shared__ uint32_t warp_tot[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o)
            inc += t;
    }
    if (lane == 31)
        warp_tot[w] = inc;
    __syncthreads();
    if (w == 0) {
        uint32_t t = lane < SCAN_THREADS / 32 ? warp_tot[lane] : 0u;
        uint32_t ti = t;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, ti, o);
            if (lane >= o)
                ti += u;
        }
        if (lane < SCAN_THREADS / 32)
            warp_tot[lane] = ti - t;
        if (lane == SCAN_THREADS / 32 - 1)
            *total = ti;
    }
    __syncthreads();
    return warp_tot[w] + inc - v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_tiles(
    const uint32_t* __restrict__ in, int64_t C, uint32_t* __restrict__ part,
    uint32_t* __restrict__ fold_status)
{
    // a pre-keyed build: the keys' status bits (word 2) become the build's
    if (fold_status && blockIdx.x == 0 && threadIdx.x == 0) {
        fold_status[0] = fold_status[2];
        fold_status[2] = 0u;
    }
    const int64_t base = int64_t(blockIdx.x) * SCAN_TILE + int64_t(threadIdx.x) * SCAN_PER_THREAD;
    uint32_t v[SCAN_PER_THREAD];
    load_tile_chunk(in, C, base, v);
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; ++k)
        s += v[k];
    __shared__ uint32_t total;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0)
        part[blockIdx.x] = total;
}

// the tiles' exclusive scans: each tile's offset is the sum of the tile sums
// before it, which the tile's block adds up itself (at most a few thousand
// values, from the L2); the last tile writes the total to out[C]
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_apply(
    const uint32_t* __restrict__ in, int64_t C, const uint32_t* __restrict__ part,
    uint32_t* __restrict__ out)
{
    uint32_t pre = 0;
    for (uint32_t t = threadIdx.x; t < blockIdx.x; t += SCAN_THREADS)
        pre += part[t];
    const int64_t base = int64_t(blockIdx.x) * SCAN_TILE + int64_t(threadIdx.x) * SCAN_PER_THREAD;
    uint32_t v[SCAN_PER_THREAD];
    load_tile_chunk(in, C, base, v);
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; ++k)
        s += v[k];
    __shared__ uint32_t offset, total;
    block_exclusive_scan(pre, &offset);
    uint32_t run = block_exclusive_scan(s, &total) + offset;
#pragma unroll
    for (int k = 0; k < SCAN_PER_THREAD; ++k) {
        const uint32_t t = v[k];
        v[k] = run;
        run += t;
    }
    if (base + SCAN_PER_THREAD <= C) {
        uint4* q = reinterpret_cast<uint4*>(out + base);
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD / 4; ++k)
            q[k] = make_uint4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_PER_THREAD; ++k)
            if (base + k < C)
                out[base + k] = v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
        out[C] = offset + total;
}

void exclusive_scan(const uint32_t* in, int64_t C, DevArray<uint32_t>& part,
    uint32_t* out, cudaStream_t s, uint32_t* fold_status)
{
    const uint32_t nparts = (uint32_t)((C + SCAN_TILE - 1) / SCAN_TILE);
    part.resize(size_t(nparts) + 1);
    REYN_KERNEL("k_scan_tiles", s,
        k_scan_tiles<<<nparts, SCAN_THREADS, 0, s>>>(in, C, part.get(), fold_status));
    REYN_KERNEL("k_scan_apply", s,
        k_scan_apply<<<nparts, SCAN_THREADS, 0, s>>>(in, C, part.get(), out));
}

void Grid::drop_prekey(cudaStream_t s)
{
    if (prekey_pending) {
        counts.zero(s);
        prekey_pending = false;
    }
}

void Grid::build(const float* x, const float* y, const float* z, uint32_t np,
    cudaStream_t s, const reyn_particles* st)
{
    const int64_t C = total_keys();
    require(!n_scenes || np == first[n_scenes], "particle count differs from the scenes' total");
    const bool prekeyed = prekey_pending && st && st == prekey_state
        && st->version == prekey_version && x == prekey_x && np == prekey_n
        && counts.size() == size_t(C) && !counts_dirty;
    if (!prekeyed)
        drop_prekey(s);
    prekey_pending = false;
    if (counts.size() != size_t(C) || counts_dirty) {
        // the scatter returns every count to zero; only a fresh array or an
        // interrupted build needs clearing
        counts.resize(size_t(C));
        counts.zero(s);
        prefix.resize(size_t(C) + 1);
        counts_dirty = false;
    }
    if (status.size() < 3)
        status.resize(3);
    // the status bits and the split-cell count (a pre-keyed build keeps word
    // 2, the keys' status, which the scan folds into word 0)
    REYN_CUDA(cudaMemsetAsync(status.get(), 0, (prekeyed ? 2 : 3) * sizeof(uint32_t), s));
    n = np;
    keys.resize(np);
    slots.resize(np);
    sorted.resize(np);
    split.resize(np);
    reordered = false;
    reordered_state = nullptr;
    built_pos[0] = x;
    built_pos[1] = y;
    built_pos[2] = z;
    const GridView g = view(geom.r);
    counts_dirty = true;
    if (np && !prekeyed) {
        REYN_KERNEL("k_keys_count", s,
            k_keys_count<<<blocks_for(np, THREADS), THREADS, 0, s>>>(
            np, x, y, z, g, keys.get(), counts.get(), status.get()));
    }
    exclusive_scan(counts.get(), C, scan_part, prefix.get(), s,
        prekeyed ? status.get() : nullptr);
    if (np) {
        REYN_KERNEL("k_scatter", s,
            k_scatter_stable<<<blocks_for(np, THREADS), THREADS, 0, s>>>(np, keys.get(),
            prefix.get(), counts.get(), slots.get(), sorted.get(), split.get(),
            status.get() + 1));
        // split cells are rare: a small fixed grid walks their list
        REYN_KERNEL("k_rank_split", s,
            k_rank_split<<<std::min<unsigned>(blocks_for(np, THREADS), 2 * 148), THREADS, 0,
            s>>>(status.get() + 1, split.get(), slots.get(), keys.get(), prefix.get(),
            sorted.get()));
    }
    counts_dirty = false;
}

// each point's scene from the scene offsets (binary search)
__global__ void k_fill_sid(uint32_t n, const uint32_t* __restrict__ first, uint32_t ns,
    uint16_t* __restrict__ sid)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    uint32_t lo = 0, hi = ns; // first[lo] <= i < first[hi]
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (first[mid] <= i)
            lo = mid;
        else
            hi = mid;
    }
    sid[i] = uint16_t(lo);
}

void Grid::set_scenes(const uint32_t* f, uint32_t ns, const GridGeom* geoms, cudaStream_t s)
{
    require(ns >= 1 && ns <= 65535, "1 .. 65535 scenes");
    require(f != nullptr && f[0] == 0, "scene offsets must start at 0");
    for (uint32_t k = 0; k < ns; ++k)
        require(f[k] <= f[k + 1], "scene offsets must not decrease");
    std::vector<SceneGeom> tab(ns);
    key_base.assign(ns + 1, 0);
    int64_t total = 0;
    for (uint32_t k = 0; k < ns; ++k) {
        const GridGeom& q = geoms[k];
        require(q.cell == geom.cell && q.range == geom.range && q.order == geom.order,
            "the scenes of a batch share the cell size and order");
        tab[k] = SceneGeom { q.lo[0], q.lo[1], q.lo[2], q.n[0], q.n[1], q.n[2], q.n[0] * q.n[1],
            q.t[0], q.t[0] * q.t[1], uint32_t(total) };
        key_base[k] = uint32_t(total);
        total += q.keys();
        require(total < (int64_t(1) << 32) - 1, "the scenes' cells exceed 32-bit keys");
    }
    key_base[ns] = uint32_t(total);
    scene_geom.assign(geoms, geoms + ns);
    scene_tab.resize(ns);
    REYN_CUDA(cudaMemcpy(scene_tab.get(), tab.data(), ns * sizeof(SceneGeom),
        cudaMemcpyHostToDevice));
    n_scenes = ns;
    first.assign(f, f + ns + 1);
    const uint32_t np_total = first[ns];
    sid.resize(np_total);
    if (np_total) {
        DevArray<uint32_t> fd(ns + 1);
        REYN_CUDA(cudaMemcpyAsync(fd.get(), first.data(), (ns + 1) * sizeof(uint32_t),
            cudaMemcpyHostToDevice, s));
        REYN_KERNEL("k_fill_sid", s,
            k_fill_sid<<<blocks_for(np_total, THREADS), THREADS, 0, s>>>(np_total, fd.get(), ns,
            sid.get()));
        REYN_CUDA(cudaStreamSynchronize(s));
    }
}

void Grid::check_status(cudaStream_t s, const char* what)
{
    uint32_t bits = 0;
    REYN_CUDA(cudaMemcpyAsync(&bits, status.get(), sizeof(bits), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaStreamSynchronize(s));
    if (bits & STATUS_NONFINITE)
        fail(REYN_ERR_NONFINITE, std::string(what) + ": non-finite particle position");
    if (bits & STATUS_OUT_OF_GRID)
        fail(REYN_ERR_OUT_OF_BOUNDS, std::string(what) + ": particle outside the grid bounds");
}

// ---- gather / pack ----------------------------------------------------------

__global__ void k_gather(uint32_t n, const uint32_t* __restrict__ perm, GatherArgs a)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const uint32_t p = perm[s];
    float v[MAX_GATHER];
#pragma unroll
    for (int k = 0; k < MAX_GATHER; ++k)
        if (k < a.count) {
            v[k] = __ldg(a.src[k] + p);
            a.dst[k][s] = v[k];
        }
    if (a.pm)
        a.pm[s] = make_float4(v[FX], v[FY], v[FZ], v[FM]);
    if (a.vel)
        a.vel[s] = make_float4(v[FVX], v[FVY], v[FVZ], 0.f);
}

void launch_gather(uint32_t n, const uint32_t* perm, const GatherArgs& a, cudaStream_t s)
{
    if (!n)
        return;
    REYN_KERNEL("k_gather", s,
        k_gather<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, perm, a));
}

__global__ void k_pack(uint32_t n, const float* __restrict__ x, const float* __restrict__ y,
    const float* __restrict__ z, const float* __restrict__ vx, const float* __restrict__ vy,
    const float* __restrict__ vz, const float* __restrict__ m, float4* __restrict__ pm,
    float4* __restrict__ vel)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    pm[i] = make_float4(x[i], y[i], z[i], m[i]);
    vel[i] = make_float4(vx[i], vy[i], vz[i], 0.f);
}

void pack_state(reyn_particles& st, cudaStream_t s)
{
    st.pm.resize(st.n);
    st.vel.resize(st.n);
    if (st.n) {
        REYN_KERNEL("k_pack", s,
            k_pack<<<blocks_for(st.n, THREADS), THREADS, 0, s>>>(st.n, st.cur[FX].get(),
            st.cur[FY].get(), st.cur[FZ].get(), st.cur[FVX].get(), st.cur[FVY].get(),
            st.cur[FVZ].get(), st.cur[FM].get(), st.pm.get(), st.vel.get()));
    }
    st.packed_valid = true;
}

void reorder_state(reyn_particles& st, Grid& g, float* const* extra, uint32_t n_extra,
    cudaStream_t s)
{
    require(n_extra + NFIELDS <= MAX_GATHER, "too many extra arrays to reorder (max 9)");
    const uint32_t n = st.n;
    for (auto& a : st.alt)
        a.resize(n);
    st.pm.resize(n);
    st.vel.resize(n);
    DevArray<float>& extra_tmp = g.extra_tmp;
    extra_tmp.resize(size_t(n) * std::max<uint32_t>(n_extra, 1));
    GatherArgs a {};
    a.count = NFIELDS + (int)n_extra;
    for (int k = 0; k < NFIELDS; ++k) {
        a.src[k] = st.cur[k].get();
        a.dst[k] = st.alt[k].get();
    }
    for (uint32_t k = 0; k < n_extra; ++k) {
        require(extra[k] != nullptr, "null extra array");
        a.src[NFIELDS + k] = extra[k];
        a.dst[NFIELDS + k] = extra_tmp.get() + size_t(k) * n;
    }
    a.pm = st.pm.get();
    a.vel = st.vel.get();
    launch_gather(n, g.sorted.get(), a, s);
    for (uint32_t k = 0; k < n_extra && n; ++k)
        REYN_CUDA(cudaMemcpyAsync(extra[k], extra_tmp.get() + size_t(k) * n,
            size_t(n) * sizeof(float), cudaMemcpyDeviceToDevice, s));
    for (int k = 0; k < NFIELDS; ++k)
        st.cur[k].swap(st.alt[k]);
    st.packed_valid = true;
    st.epoch += 1;
    st.version += 1;
    g.reordered = true;
    g.reordered_state = &st;
    g.reorder_epoch = st.epoch;
}

// a caller's permutation, checked before it is applied: bit 0 of `bad` for
// an index >= n, bit 1 for an index seen twice (`seen` holds n bits, zeroed)
__global__ void k_check_perm(uint32_t n, const uint32_t* __restrict__ perm,
    uint32_t* __restrict__ seen, uint32_t* __restrict__ bad)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const uint32_t p = perm[s];
    if (p >= n) {
        atomicOr(bad, 1u);
        return;
    }
    const uint32_t bit = 1u << (p & 31u);
    if (atomicOr(seen + (p >> 5), bit) & bit)
        atomicOr(bad, 2u);
}

void reorder_by(reyn_particles& st, const uint32_t* sorted, cudaStream_t s)
{
    const uint32_t n = st.n;
    if (!n)
        return;
    require(sorted != nullptr, "null permutation");
    {
        DevArray<uint32_t> seen((n + 31) / 32 + 1); // last word: the error bits
        seen.zero(s);
        uint32_t* bad = seen.get() + (n + 31) / 32;
        REYN_KERNEL("k_check_perm", s,
            k_check_perm<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, sorted, seen.get(), bad));
        uint32_t host = 0;
        REYN_CUDA(cudaMemcpyAsync(&host, bad, sizeof(host), cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaStreamSynchronize(s));
        if (host)
            fail(REYN_ERR_INVALID, (host & 1u) ? "permutation index out of range"
                                               : "permutation repeats an index");
    }
    for (auto& a : st.alt)
        a.resize(n);
    st.pm.resize(n);
    st.vel.resize(n);
    GatherArgs a {};
    a.count = NFIELDS;
    for (int k = 0; k < NFIELDS; ++k) {
        a.src[k] = st.cur[k].get();
        a.dst[k] = st.alt[k].get();
    }
    a.pm = st.pm.get();
    a.vel = st.vel.get();
    launch_gather(n, sorted, a, s);
    for (int k = 0; k < NFIELDS; ++k)
        st.cur[k].swap(st.alt[k]);
    st.packed_valid = true;
    st.epoch += 1;
    st.version += 1;
}

void resize_state(reyn_particles& st, uint32_t n, bool keep, cudaStream_t s)
{
    const uint32_t m = keep ? std::min(st.n, n) : 0u;
    // every new array first: a failed allocation leaves the state as it was
    std::array<DevArray<float>, NFIELDS> fresh;
    for (auto& a : fresh)
        a.resize(n);
    for (int k = 0; k < NFIELDS; ++k) {
        if (m)
            REYN_CUDA(cudaMemcpyAsync(fresh[k].get(), st.cur[k].get(), size_t(m) * sizeof(float),
                cudaMemcpyDeviceToDevice, s));
        if (n > m)
            REYN_CUDA(cudaMemsetAsync(fresh[k].get() + m, 0, size_t(n - m) * sizeof(float), s));
    }
    REYN_CUDA(cudaStreamSynchronize(s)); // the old arrays are freed below
    for (int k = 0; k < NFIELDS; ++k) {
        st.cur[k] = std::move(fresh[k]);
        st.alt[k] = DevArray<float>();
    }
    st.pm = DevArray<float4>();
    st.vel = DevArray<float4>();
    st.n = n;
    st.packed_valid = false;
    st.epoch += 1;
    st.version += 1;
}

// ---- kernel evaluation -------------------------------------------------------

// Kernel::operator() and Kernel::nabla (kernels.cuh:40-64) for arbitrary
// offsets: the norm is norm3df, as the reference computes it on the device
template <int KIND>
__global__ void k_kernel_eval(uint32_t n, KernelConst kc, const float* __restrict__ dx,
    const float* __restrict__ dy, const float* __restrict__ dz, float* __restrict__ w,
    float* __restrict__ gx, float* __restrict__ gy, float* __restrict__ gz)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float x = dx[i], y = dy[i], z = dz[i];
    const float len = norm3df(x, y, z);
    w[i] = kc.w_scale * Shape<KIND>::w(__saturatef(len * kc.h_inv));
    const float sc = kc.dw_scale * Shape<KIND>::dw(len * kc.h_inv) * (1.f / len);
    const float g = isfinite(sc) ? sc : 0.f;
    gx[i] = g * x;
    gy[i] = g * y;
    gz[i] = g * z;
}

void kernel_eval(int kind, float h_bar, const float* dx, const float* dy, const float* dz,
    uint32_t n, float* w, float* gx, float* gy, float* gz, cudaStream_t s)
{
    require(kind >= 0 && kind <= 3, "unknown kernel");
    require(h_bar > 0.f, "h_bar must be positive");
    if (!n)
        return;
    const KernelConst kc = make_kernel(kind, h_bar);
    const unsigned b = blocks_for(n, THREADS);
    ProfScope scope("k_kernel_eval", s);
    switch (kind) {
    case K_C2: k_kernel_eval<K_C2><<<b, THREADS, 0, s>>>(n, kc, dx, dy, dz, w, gx, gy, gz); break;
    case K_B3: k_kernel_eval<K_B3><<<b, THREADS, 0, s>>>(n, kc, dx, dy, dz, w, gx, gy, gz); break;
    case K_W6: k_kernel_eval<K_W6><<<b, THREADS, 0, s>>>(n, kc, dx, dy, dz, w, gx, gy, gz); break;
    default: k_kernel_eval<K_COS><<<b, THREADS, 0, s>>>(n, kc, dx, dy, dz, w, gx, gy, gz); break;
    }
    REYN_LAUNCHED("k_kernel_eval");
}

// ---- neighbour statistics ----------------------------------------------------

// the reference grid test's quantities (uniformgrid.cu:185-207) and the
// density sum (solver.cuh:31-33), evaluated per grid slot over packed points
template <int KIND, int R>
__global__ void __launch_bounds__(NBR_THREADS) k_neighbour_stats(uint32_t n, GridView g,
    KernelConst kc, const float4* __restrict__ pts, const uint32_t* __restrict__ owner,
    uint32_t* __restrict__ count, float* __restrict__ len2, float* __restrict__ rho,
    uint32_t* __restrict__ status)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const float4 me = pts[s];
    const uint32_t p = owner ? owner[s] : s;
    g = at_scene(g, scene_of(g, p)); // batched grids: the point's own scene
    int3 c = cell_of(g, me.x, me.y, me.z);
    if (!cell_inside(g, c, R) || !(isfinite(me.x) && isfinite(me.y) && isfinite(me.z))) {
        atomicOr(status, STATUS_OUT_OF_GRID);
        c = clamp_cell(g, c, R);
    }
    uint32_t cnt = 0;
    float l2sum = 0.f, dens = 0.f;
    for_each_neighbour<R>(g, c, me.x, me.y, me.z, pts,
        [&](uint32_t j, const float4& q, float, float, float, float l2) {
            cnt += (j == s) ? 0u : 1u;
            l2sum += l2;
            if (rho)
                dens += q.w * pair_w<KIND>(kc, l2);
        });
    if (count)
        count[p] = cnt;
    if (len2)
        len2[p] = l2sum;
    if (rho)
        rho[p] = dens;
}

__global__ void k_pack_positions(uint32_t n, const uint32_t* __restrict__ order,
    const float* __restrict__ x, const float* __restrict__ y, const float* __restrict__ z,
    const float* __restrict__ m, float4* __restrict__ pts)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n)
        return;
    const uint32_t p = order ? order[s] : s;
    pts[s] = make_float4(x[p], y[p], z[p], m ? m[p] : 0.f);
}

void pack_positions(uint32_t n, const uint32_t* order, const float* x, const float* y,
    const float* z, const float* m, float4* pts, cudaStream_t s)
{
    if (n)
        REYN_KERNEL("k_pack_positions", s,
            k_pack_positions<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, order, x, y, z, m, pts));
}

template <int KIND>
static void launch_stats(int range, unsigned b, cudaStream_t s, uint32_t n, GridView g,
    KernelConst kc, const float4* pts, const uint32_t* owner, uint32_t* count, float* len2,
    float* rho, uint32_t* status)
{
    if (range == 2)
        k_neighbour_stats<KIND, 2><<<b, NBR_THREADS, 0, s>>>(n, g, kc, pts, owner, count, len2, rho, status);
    else
        k_neighbour_stats<KIND, 1><<<b, NBR_THREADS, 0, s>>>(n, g, kc, pts, owner, count, len2, rho, status);
}

void neighbour_stats(const Grid& g, const float* x, const float* y, const float* z,
    const float* m, int kind, uint32_t* count, float* len2, float* rho, cudaStream_t s)
{
    const uint32_t n = g.n;
    if (!n)
        return;
    require(!(rho && !m), "density requires masses");
    require(!rho || (kind >= 0 && kind <= 3), "unknown kernel");
    DevArray<float4>& pts = g.pts_tmp;
    pts.resize(n);
    // the arrays are in grid order after a reorder, else gather them
    const uint32_t* order = g.reordered ? nullptr : g.sorted.get();
    REYN_KERNEL("k_pack_positions", s,
        k_pack_positions<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, order, x, y, z, m, pts.get()));
    const GridView v = g.view(g.geom.r);
    const KernelConst kc = make_kernel(rho ? kind : 0, g.geom.r);
    const unsigned b = blocks_for(n, NBR_THREADS);
    float* r = rho;
    uint32_t* st = const_cast<uint32_t*>(g.status.get());
    ProfScope scope("k_neighbour_stats", s);
    switch (rho ? kind : 0) {
    case K_C2: launch_stats<K_C2>(g.geom.range, b, s, n, v, kc, pts.get(), order, count, len2, r, st); break;
    case K_B3: launch_stats<K_B3>(g.geom.range, b, s, n, v, kc, pts.get(), order, count, len2, r, st); break;
    case K_W6: launch_stats<K_W6>(g.geom.range, b, s, n, v, kc, pts.get(), order, count, len2, r, st); break;
    default: launch_stats<K_COS>(g.geom.range, b, s, n, v, kc, pts.get(), order, count, len2, r, st); break;
    }
    REYN_LAUNCHED("k_neighbour_stats");
}

// ---- boundary ------------------------------------------------------------------

__device__ __forceinline__ unsigned ordered_bits(float f)
{
    const unsigned u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
inline float from_ordered_bits(unsigned u)
{
    const unsigned v = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
    float f;
    memcpy(&f, &v, sizeof(f));
    return f;
}

// bounding box of the samples (sample_boundary.cu:415-416: xs.min() ...)
__global__ void k_bounds(uint32_t n, const float* __restrict__ x, const float* __restrict__ y,
    const float* __restrict__ z, unsigned* __restrict__ box)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float v[3] = { x[i], y[i], z[i] };
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        atomicMin(box + a, ordered_bits(v[a]));
        atomicMax(box + 3 + a, ordered_bits(v[a]));
    }
}

// one Akinci mass refinement (sample_boundary.cu:250-265), double-buffered:
// m_i <- rho0 m_i / sum_j m_j W_B3(x_ij), support 2h
template <int R>
__global__ void __launch_bounds__(NBR_THREADS) k_boundary_mass(uint32_t n, GridView g,
    KernelConst kc, const float4* __restrict__ pts, float rho0, float4* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    g = at_scene(g, scene_of(g, i)); // batched boundaries: the sample's own scene
    const float4 me = pts[i];
    int3 c = clamp_cell(g, cell_of(g, me.x, me.y, me.z), R);
    float sum = 0.f;
    for_each_neighbour<R>(g, c, me.x, me.y, me.z, pts,
        [&](uint32_t, const float4& q, float, float, float, float l2) {
            sum += q.w * pair_w<K_B3>(kc, l2);
        });
    out[i] = make_float4(me.x, me.y, me.z, rho0 * me.w / sum);
}

// marks the (2R+1)^3 cells around every boundary sample
__global__ void k_mark_near(uint32_t n, GridView g, const float4* __restrict__ pts,
    uint8_t* __restrict__ near)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float4 me = pts[i];
    g = at_scene(g, scene_of(g, i)); // batched: the sample's own scene grid
    near += g.key_base;
    const int3 c = clamp_cell(g, cell_of(g, me.x, me.y, me.z), 2);
    for (int dz = -2; dz <= 2; ++dz)
        for (int dy = -2; dy <= 2; ++dy) {
            const int base = (c.z + dz) * g.nxny + (c.y + dy) * g.nx + c.x;
            for (int dx = -2; dx <= 2; ++dx)
                near[base + dx] = 1;
        }
}

__global__ void k_unpack_mass(uint32_t n, const float4* __restrict__ pts, float* __restrict__ m)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        m[i] = pts[i].w;
}

void boundary_build(reyn_boundary& b, const float* bx, const float* by, const float* bz,
    const float* bm, uint32_t nb, float h, float rho0, uint32_t mass_iters, cudaStream_t s,
    const uint32_t* scene_first, uint32_t n_scenes)
{
    require(h > 0.f && std::isfinite(h), "h must be positive");
    b.nb = nb;
    b.h = h;
    if (nb == 0)
        return;
    require(bx && by && bz, "null boundary positions");
    require(bm || mass_iters > 0, "at least one mass refinement iteration is required");
    DevArray<unsigned> box(6);
    const unsigned init[6] = { 0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u };
    REYN_CUDA(cudaMemcpyAsync(box.get(), init, sizeof(init), cudaMemcpyHostToDevice, s));
    REYN_KERNEL("k_bounds", s,
        k_bounds<<<blocks_for(nb, THREADS), THREADS, 0, s>>>(nb, bx, by, bz, box.get()));
    unsigned hb[6];
    REYN_CUDA(cudaMemcpyAsync(hb, box.get(), sizeof(hb), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaStreamSynchronize(s));
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        lo[a] = from_ordered_bits(hb[a]);
        hi[a] = from_ordered_bits(hb[3 + a]);
        b.lo[a] = lo[a];
        b.hi[a] = hi[a];
    }
    // the boundary grid: support 2h over the samples' own bounds, reference
    // geometry (sample_boundary.cu:420-428)
    b.grid.geom = make_geom(lo, hi, 2.f * h, 0.5f);
    if (n_scenes) {
        // batched: every scene's samples get the grid a boundary of their
        // own would get (over their own bounds), keyed scene after scene
        DevArray<unsigned> sbox(size_t(6) * n_scenes);
        std::vector<unsigned> sinit(size_t(6) * n_scenes);
        for (uint32_t k = 0; k < n_scenes; ++k)
            std::copy(init, init + 6, sinit.begin() + 6 * size_t(k));
        REYN_CUDA(cudaMemcpyAsync(sbox.get(), sinit.data(), sinit.size() * sizeof(unsigned),
            cudaMemcpyHostToDevice, s));
        for (uint32_t k = 0; k < n_scenes; ++k) {
            const uint32_t a = scene_first[k], cnt = scene_first[k + 1] - a;
            require(cnt > 0, "every scene of a batched boundary needs samples");
            REYN_KERNEL("k_bounds", s,
                k_bounds<<<blocks_for(cnt, THREADS), THREADS, 0, s>>>(cnt, bx + a, by + a, bz + a,
                sbox.get() + 6 * size_t(k)));
        }
        std::vector<unsigned> hsb(sinit.size());
        REYN_CUDA(cudaMemcpyAsync(hsb.data(), sbox.get(), hsb.size() * sizeof(unsigned),
            cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaStreamSynchronize(s));
        std::vector<GridGeom> geoms(n_scenes);
        for (uint32_t k = 0; k < n_scenes; ++k) {
            float slo[3], shi[3];
            for (int a = 0; a < 3; ++a) {
                slo[a] = from_ordered_bits(hsb[6 * k + a]);
                shi[a] = from_ordered_bits(hsb[6 * k + 3 + a]);
            }
            geoms[k] = make_geom(slo, shi, 2.f * h, 0.5f);
        }
        b.grid.set_scenes(scene_first, n_scenes, geoms.data(), s);
    }
    b.grid.build(bx, by, bz, nb, s);
    b.grid.check_status(s, "boundary grid");
    b.x.resize(nb);
    b.y.resize(nb);
    b.z.resize(nb);
    b.m.resize(nb);
    b.pm.resize(nb);
    DevArray<float> ones;
    if (!bm) {
        ones.resize(nb);
        std::vector<float> h1(nb, 1.f); // m_0 = 1 (sample_boundary.cu:277)
        REYN_CUDA(cudaMemcpyAsync(ones.get(), h1.data(), nb * sizeof(float),
            cudaMemcpyHostToDevice, s));
        REYN_CUDA(cudaStreamSynchronize(s));
    }
    GatherArgs a {};
    a.count = 4;
    a.src[0] = bx;
    a.src[1] = by;
    a.src[2] = bz;
    a.src[3] = bm ? bm : ones.get();
    a.dst[0] = b.x.get();
    a.dst[1] = b.y.get();
    a.dst[2] = b.z.get();
    a.dst[3] = b.m.get();
    launch_gather(nb, b.grid.sorted.get(), a, s);
    REYN_KERNEL("k_pack_positions", s,
        k_pack_positions<<<blocks_for(nb, THREADS), THREADS, 0, s>>>(
        nb, nullptr, b.x.get(), b.y.get(), b.z.get(), b.m.get(), b.pm.get()));
    b.grid.reordered = true;
    b.near.resize(size_t(b.grid.total_keys()));
    b.near.zero(s);
    REYN_KERNEL("k_mark_near", s,
        k_mark_near<<<blocks_for(nb, THREADS), THREADS, 0, s>>>(nb, b.view(), b.pm.get(),
            b.near.get()));
    if (!bm) {
        DevArray<float4> other(nb);
        const GridView v = b.view();
        const KernelConst kc = make_kernel(K_B3, 2.f * h);
        for (uint32_t it = 0; it < mass_iters; ++it) {
            REYN_KERNEL("k_boundary_mass", s,
                k_boundary_mass<2><<<blocks_for(nb, NBR_THREADS), NBR_THREADS, 0, s>>>(
                nb, v, kc, b.pm.get(), rho0, other.get()));
            b.pm.swap(other);
        }
        REYN_KERNEL("k_unpack_mass", s,
            k_unpack_mass<<<blocks_for(nb, THREADS), THREADS, 0, s>>>(nb, b.pm.get(), b.m.get()));
        REYN_CUDA(cudaStreamSynchronize(s));
    }
}

} // namespace reyn
