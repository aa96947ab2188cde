// The reference's main loop (main.cu:60-78) written against the reyn_b200
// C++ adapters (include/reyn_b200.hpp): dt controller, grid build with
// reorder (the particle ID carried as an extra array), IISPH step, hard
// bounds. Reads a scene from argv[1], writes the final state to argv[2].
// With a third argument "fused" the loop uses the fused tail (next_dt and
// step_bounded in place of simple_dt_controller, step and hard_enforce_bounds);
// "fixed" keeps dt fixed (no controller; the id array is not reordered) and
// "graph" runs that fixed-dt loop as replays of a StepGraph; "unsorted" is
// the default loop with IISPH<C2, Resort::no> on grids built by construct
// (the particles keep their order).
//
// input  (little-endian): u32 N, u32 Nb, u32 steps, f32 h, rho0, nu, dt0,
//        lambda, box_min[3], box_max[3], then N floats each of x y z vx vy vz
//        m id, then Nb floats each of bx by bz bm
// output: u32 steps, u32 iters[steps], f32 dt[steps], N floats each of
//        x y z vx vy vz id
#include "reyn_b200.hpp"

#include <cstdio>
#include <memory>
#include <string>
#include <vector>

using namespace reyn;

int main(int argc, char** argv)
{
    if (argc != 3 && argc != 4) {
        std::fprintf(stderr, "usage: main_loop in.bin out.bin [fused]\n");
        return 2;
    }
    const std::string mode = argc == 4 ? std::string(argv[3]) : std::string();
    const bool fused = mode == "fused";
    FILE* f = std::fopen(argv[1], "rb");
    if (!f)
        return 2;
    uint32_t hdr[3];
    float prm[11];
    if (std::fread(hdr, 4, 3, f) != 3 || std::fread(prm, 4, 11, f) != 11)
        return 2;
    const uint32_t N = hdr[0], Nb = hdr[1], steps = hdr[2];
    const float h = prm[0], rho0 = prm[1], nu = prm[2], lambda = prm[4];
    float dt = prm[3];
    const float3 bmin = make_float3(prm[5], prm[6], prm[7]);
    const float3 bmax = make_float3(prm[8], prm[9], prm[10]);
    std::vector<float> fl(size_t(N) * 8), bd(size_t(Nb) * 4);
    if (std::fread(fl.data(), 4, fl.size(), f) != fl.size()
        || std::fread(bd.data(), 4, bd.size(), f) != bd.size())
        return 2;
    std::fclose(f);
    auto col = [&](std::vector<float>& v, uint32_t n, int k) { return v.data() + size_t(k) * n; };

    try {
        Particles state(N, rho0);
        state.upload(col(fl, N, 0), col(fl, N, 1), col(fl, N, 2), col(fl, N, 3), col(fl, N, 4),
            col(fl, N, 5), col(fl, N, 6));
        float *d_id = nullptr, *d_b = nullptr;
        if (cudaMalloc(&d_id, N * sizeof(float)) != cudaSuccess
            || cudaMalloc(&d_b, size_t(Nb) * 4 * sizeof(float)) != cudaSuccess)
            throw Error(REYN_ERR_ALLOC, "cudaMalloc");
        cudaMemcpy(d_id, col(fl, N, 7), N * sizeof(float), cudaMemcpyHostToDevice);
        cudaMemcpy(d_b, bd.data(), bd.size() * sizeof(float), cudaMemcpyHostToDevice);
        BoundarySamples bdy(d_b, d_b + Nb, d_b + 2 * size_t(Nb), d_b + 3 * size_t(Nb), Nb, h, rho0);

        const C2 W(2.f * h);
        UniformGridBuilder builder(bmin, bmax, 2.f * h);
        IISPH<C2, Resort::yes> solver(W, N, nu, h, rho0);
        std::unique_ptr<IISPH<C2, Resort::no>> unsorted;
        if (mode == "unsorted")
            unsorted = std::make_unique<IISPH<C2, Resort::no>>(W, N, nu, h, rho0);
        const float3 g = make_float3(0.f, -9.81f, 0.f);
        std::vector<uint32_t> iters_log;
        std::vector<float> dt_log;
        uint32_t iters = 0;
        if (mode == "graph") {
            StepGraph graph(solver, state, builder, &bdy, dt, bmin, bmax);
            for (uint32_t s = 0; s < steps; ++s) {
                graph.launch();
                iters_log.push_back(graph.iterations());
                dt_log.push_back(dt);
            }
        }
        for (uint32_t s = 0; s < steps && mode != "graph"; ++s) {
            if (mode == "fixed") {
                const auto grid { builder.construct_and_reorder(2.f * h, state) };
                iters = solver.step_bounded(state, grid, bdy, dt, bmin, bmax);
            } else if (unsorted) {
                dt = simple_dt_controller(iters, dt, lambda, h, state, g, 10, 0.001f);
                const UniformGrid<Resort::no> grid { builder.construct(2.f * h, state) };
                iters = unsorted->step(state, grid, bdy, dt);
                hard_enforce_bounds(state, bmin, bmax);
            } else if (fused) {
                dt = solver.next_dt(state, iters, dt, lambda, h, g, 10, 0.001f);
                const auto grid { builder.construct_and_reorder(2.f * h, state, d_id) };
                iters = solver.step_bounded(state, grid, bdy, dt, bmin, bmax);
            } else {
                dt = simple_dt_controller(iters, dt, lambda, h, state, g, 10, 0.001f);
                const auto grid { builder.construct_and_reorder(2.f * h, state, d_id) };
                iters = solver.step(state, grid, bdy, dt);
                hard_enforce_bounds(state, bmin, bmax);
            }
            iters_log.push_back(iters);
            dt_log.push_back(dt);
        }
        std::vector<float> out(size_t(N) * 7);
        state.download(col(out, N, 0), col(out, N, 1), col(out, N, 2), col(out, N, 3),
            col(out, N, 4), col(out, N, 5), nullptr);
        cudaMemcpy(col(out, N, 6), d_id, N * sizeof(float), cudaMemcpyDeviceToHost);
        cudaFree(d_id);
        cudaFree(d_b);
        FILE* o = std::fopen(argv[2], "wb");
        if (!o)
            return 2;
        std::fwrite(&steps, 4, 1, o);
        std::fwrite(iters_log.data(), 4, steps, o);
        std::fwrite(dt_log.data(), 4, steps, o);
        std::fwrite(out.data(), 4, out.size(), o);
        std::fclose(o);
    } catch (const Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
