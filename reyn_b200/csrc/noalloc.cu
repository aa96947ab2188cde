// reyn_grid_construct_noalloc: the uniform-grid build for callers that must
// not allocate device memory.
//
// Some callers cannot call cudaMalloc: real-time loops that must not stall
// on the device allocator (cudaMalloc can synchronise the device and take
// milliseconds), and hosts whose device memory is owned by another runtime's
// pool (a game engine, a framework allocator) that only hand out the buffers
// they created and forbid allocations behind the pool's back.
// reyn_grid_construct keeps its scratch (per-cell counters, keys, unordered
// slots, scan partials) in device arrays the grid object allocates; this
// variant keeps it in one file-scope device array instead, so a call needs
// nothing but the caller's input and output buffers.
//
// The array is REYN_GRID_NOALLOC_SCRATCH_WORDS 32-bit words (32 MiB). It is
// part of this library's device image: every GPU that loads it holds the
// array until the process exits. Every call on a device shares the one array
// and leaves its contents behind; the counters and the status word are
// cleared at the start of each call. Calls that overlap on the GPU (two
// streams, two host threads) race on the array and corrupt each other's
// results: serialise them.
//
// Host code cannot use the array's name as a device address (on the host it
// names a host-side stand-in), so the device address is fetched with
// cudaGetSymbolAddress, once per device, on the first call made while that
// device is current. That first call therefore performs a CUDA runtime query
// and should come before any stream capture begins.
#include "engine.cuh"

#include <array>
#include <mutex>

namespace reyn {

// the grid-build kernels of grid.cu, launched here on the static scratch
__global__ void k_keys_count(uint32_t n, const float* __restrict__ x,
    const float* __restrict__ y, const float* __restrict__ z, GridView g,
    uint32_t* __restrict__ keys, uint32_t* __restrict__ counts,
    uint32_t* __restrict__ status);
__global__ void k_scatter(uint32_t n, const uint32_t* __restrict__ keys,
    const uint32_t* __restrict__ prefix, uint32_t* __restrict__ counts,
    uint32_t* __restrict__ slots);
__global__ void k_canonical(uint32_t n, const uint32_t* __restrict__ slots,
    const uint32_t* __restrict__ keys, const uint32_t* __restrict__ prefix,
    uint32_t* __restrict__ sorted);
__global__ void __launch_bounds__(256) k_scan_tiles(
    const uint32_t* __restrict__ in, int64_t C, uint32_t* __restrict__ part,
    uint32_t* __restrict__ fold_status);
__global__ void __launch_bounds__(256) k_scan_apply(const uint32_t* __restrict__ in, int64_t C,
    const uint32_t* __restrict__ part, uint32_t* __restrict__ out);

namespace {

    constexpr int64_t SCAN_TILE = 256 * 16; // k_scan_* tile: 256 threads x 16 counts

    static __device__ __align__(256) uint32_t g_grid_scratch[REYN_GRID_NOALLOC_SCRATCH_WORDS];

    std::mutex g_scratch_mu;
    std::array<uint32_t*, 256> g_scratch_addr {};

    // the device address of g_grid_scratch on the current device
    uint32_t* scratch_on_current_device()
    {
        int dev = 0;
        REYN_CUDA(cudaGetDevice(&dev));
        require(dev >= 0 && dev < (int)g_scratch_addr.size(), "device ordinal out of range");
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_grid_scratch);
            if (e != cudaSuccess || !p)
                fail(REYN_ERR_CUDA,
                    std::string("cudaGetSymbolAddress of the grid scratch failed: ")
                        + cudaGetErrorString(e));
            g_scratch_addr[dev] = static_cast<uint32_t*>(p);
        }
        return g_scratch_addr[dev];
    }

} // namespace
} // namespace reyn

using namespace reyn;

extern "C" int reyn_grid_construct_noalloc(const float bound_min[3], const float bound_max[3],
    float search_radius, float cell_ratio, const float* xx, const float* xy, const float* xz,
    uint32_t n, uint32_t* prefix, uint64_t prefix_capacity, uint32_t* sorted, int32_t dims[3],
    void* stream)
{
    return guard([&] {
        require(bound_min && bound_max, "null bounds");
        const GridGeom geom = make_geom(bound_min, bound_max, search_radius, cell_ratio);
        if (dims) {
            dims[0] = geom.n[0];
            dims[1] = geom.n[1];
            dims[2] = geom.n[2];
        }
        if (!prefix)
            return; // size query
        const int64_t C = geom.cells();
        require(prefix_capacity >= uint64_t(C) + 1, "prefix must hold nx*ny*nz + 1 entries");
        require(n == 0 || (xx && xy && xz && sorted), "null position or output array");
        const uint32_t nparts = uint32_t((C + SCAN_TILE - 1) / SCAN_TILE);
        // scratch layout: counts[C] | status[1] | parts[nparts + 1] | keys[n] | slots[n]
        const uint64_t need = uint64_t(C) + 1 + (uint64_t(nparts) + 1) + 2 * uint64_t(n);
        if (need > REYN_GRID_NOALLOC_SCRATCH_WORDS)
            fail(REYN_ERR_INVALID,
                "grid needs " + std::to_string(need) + " words of scratch (cells + 2 x particles "
                    + "+ scan partials); the no-alloc build holds at most "
                    + std::to_string(REYN_GRID_NOALLOC_SCRATCH_WORDS)
                    + ": use reyn_grid_construct");
        uint32_t* base = scratch_on_current_device();
        uint32_t* counts = base;
        uint32_t* status = counts + C;
        uint32_t* parts = status + 1;
        uint32_t* keys = parts + (nparts + 1);
        uint32_t* slots = keys + n;
        const cudaStream_t s = as_stream(stream);
        // the counters and the status word must start at zero; the rest is
        // fully overwritten before it is read
        REYN_CUDA(cudaMemsetAsync(counts, 0, size_t(C + 1) * sizeof(uint32_t), s));
        GridView v {};
        v.lox = geom.lo[0];
        v.loy = geom.lo[1];
        v.loz = geom.lo[2];
        v.cell = geom.cell;
        v.inv_cell = 1.f / geom.cell;
        v.r2 = geom.r * geom.r;
        v.nx = geom.n[0];
        v.ny = geom.n[1];
        v.nz = geom.n[2];
        v.nxny = geom.n[0] * geom.n[1];
        v.prefix = prefix;
        if (n) {
            REYN_KERNEL("k_keys_count", s,
                k_keys_count<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, xx, xy, xz, v, keys,
                counts, status));
        }
        REYN_KERNEL("k_scan_tiles", s,
            k_scan_tiles<<<nparts, 256, 0, s>>>(counts, C, parts, nullptr));
        REYN_KERNEL("k_scan_apply", s,
            k_scan_apply<<<nparts, 256, 0, s>>>(counts, C, parts, prefix));
        if (n) {
            REYN_KERNEL("k_scatter", s,
                k_scatter<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, keys, prefix, counts,
                slots));
            REYN_KERNEL("k_canonical", s,
                k_canonical<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, slots, keys, prefix,
                sorted));
        }
        uint32_t bits = 0;
        REYN_CUDA(cudaMemcpyAsync(&bits, status, sizeof(bits), cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaStreamSynchronize(s));
        if (bits & STATUS_NONFINITE)
            fail(REYN_ERR_NONFINITE, "construct_noalloc: non-finite particle position");
        if (bits & STATUS_OUT_OF_GRID)
            fail(REYN_ERR_OUT_OF_BOUNDS, "construct_noalloc: particle outside the grid bounds");
    });
}
