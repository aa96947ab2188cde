// UniformGrid<R>::ff_nbrs of the C++ adapters (include/reyn_b200.hpp) used
// from a user kernel, the way the reference's own kernels use theirs
// (solver.cuh:19-38): per point the neighbour count (self excluded) and the
// sum of |x_ij|^2, compared with the engine's reyn_grid_neighbour_stats on
// the same grid. Runs Resort::no (construct) and Resort::yes
// (construct_and_reorder) in the cell order given by argv[1] ("xyz" or
// "zorder") at the cell ratio argv[2]. Exit 0 when counts agree exactly and
// the sums within 1e-5 relative.
#include "reyn_b200.hpp"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace reyn;

struct CountL2 {
    unsigned count;
    float l2;
    __device__ CountL2& operator+=(const CountL2& o)
    {
        count += o.count;
        l2 += o.l2;
        return *this;
    }
};

template <Resort R>
__global__ void user_kernel(uint32_t n, UniformGrid<R> grid, const float* xx, const float* xy,
    const float* xz, unsigned* count, float* len2)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const float3 x_i = make_float3(xx[i], xy[i], xz[i]);
    const CountL2 r = grid.ff_nbrs(x_i, xx, xy, xz,
        [&](const uint32_t j, const float3, const float l2) {
            return CountL2 { j == i ? 0u : 1u, l2 };
        });
    count[i] = r.count;
    len2[i] = r.l2;
}

static bool compare(const char* what, uint32_t n, const unsigned* a, const float* al,
    const unsigned* b, const float* bl)
{
    std::vector<unsigned> ha(n), hb(n);
    std::vector<float> hal(n), hbl(n);
    cudaMemcpy(ha.data(), a, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hb.data(), b, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hal.data(), al, n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hbl.data(), bl, n * 4, cudaMemcpyDeviceToHost);
    size_t bad = 0;
    double mean = 0.0;
    for (uint32_t i = 0; i < n; ++i) {
        mean += ha[i];
        if (ha[i] != hb[i] || std::fabs(hal[i] - hbl[i]) > 1e-5f * std::fabs(hbl[i]) + 1e-12f)
            ++bad;
    }
    std::printf("%s: %zu/%u differ, mean count %.2f\n", what, bad, n, mean / n);
    return bad == 0 && mean / n > 20.0;
}

int main(int argc, char** argv)
{
    if (argc != 3)
        return 2;
    const reyn_cell_order order
        = std::strcmp(argv[1], "zorder") == 0 ? REYN_ORDER_ZORDER : REYN_ORDER_XYZ;
    const float ratio = std::stof(argv[2]);
    const uint32_t n = 200000;
    const float r = 0.0196f * 2.f; // about 33 neighbours at this density
    std::vector<float> h(3 * size_t(n));
    uint64_t z = 12345;
    for (auto& v : h) { // SplitMix64 uniforms in [0, 1)
        z += 0x9E3779B97F4A7C15ull;
        uint64_t t = z;
        t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
        t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
        t ^= t >> 31;
        v = float(uint32_t(t >> 40)) * (1.f / 16777216.f);
    }
    try {
        Particles state(n, 1000.f);
        state.upload(h.data(), h.data() + n, h.data() + 2 * size_t(n), nullptr, nullptr, nullptr,
            nullptr);
        UniformGridBuilder builder(make_float3(0, 0, 0), make_float3(1, 1, 1), r, ratio, order);
        unsigned *c0, *c1;
        float *l0, *l1;
        cudaMalloc(&c0, n * 4);
        cudaMalloc(&c1, n * 4);
        cudaMalloc(&l0, n * 4);
        cudaMalloc(&l1, n * 4);
        bool ok = true;
        {
            const UniformGrid<Resort::no> grid { builder.construct(r, state) };
            const reyn_soa v = state.soa();
            user_kernel<<<(n + 127) / 128, 128>>>(n, grid, v.xx, v.xy, v.xz, c0, l0);
            check(reyn_grid_neighbour_stats(grid.grid, v.xx, v.xy, v.xz, nullptr,
                REYN_KERNEL_C2, c1, l1, nullptr, nullptr));
            check(cudaDeviceSynchronize() == cudaSuccess ? REYN_OK : REYN_ERR_CUDA);
            ok = compare("Resort::no", n, c0, l0, c1, l1) && ok;
        }
        {
            const UniformGrid<Resort::yes> grid { builder.construct_and_reorder(r, state) };
            const reyn_soa v = state.soa();
            user_kernel<<<(n + 127) / 128, 128>>>(n, grid, v.xx, v.xy, v.xz, c0, l0);
            check(reyn_grid_neighbour_stats(grid.grid, v.xx, v.xy, v.xz, nullptr,
                REYN_KERNEL_C2, c1, l1, nullptr, nullptr));
            check(cudaDeviceSynchronize() == cudaSuccess ? REYN_OK : REYN_ERR_CUDA);
            ok = compare("Resort::yes", n, c0, l0, c1, l1) && ok;
        }
        cudaFree(c0);
        cudaFree(c1);
        cudaFree(l0);
        cudaFree(l1);
        return ok ? 0 : 1;
    } catch (const Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
}
