// The reference's main loop (main.cu:46-76) with its scene set-up, written
// against the C++ adapters (include/reyn_b200.hpp): Scene::from_obj (or the
// box constructor), IISPH<B3, Resort::yes> at support 2h, then steps of
// simple_dt_controller, scene.get_grid, solver.step and
// scene.hard_enforce_bounds.
//
// usage: scene_loop scene.obj out.bin obj|box N_desired steps
// output (little-endian): u32 N, u32 Nb, u32 steps, f32 h, f32 bound_min[3],
//        f32 bound_max[3], the set-up positions (N floats each of x y z),
//        the boundary samples (Nb floats each of x y z), u32 iters[steps],
//        the final positions (N floats each of x y z)
#include "reyn_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using namespace reyn;

static std::vector<float> to_host(const float* d, uint32_t n)
{
    std::vector<float> h(n);
    if (n)
        cudaMemcpy(h.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost);
    return h;
}

static void run(Scene& scene, Particles& state, const char* out, uint32_t steps)
{
    const uint32_t N = scene.N;
    reyn_soa v = state.soa();
    if (v.n != N)
        throw Error(REYN_ERR_INVALID, "state size differs from the scene's N");
    std::vector<float> x0 = to_host(v.xx, N), y0 = to_host(v.xy, N), z0 = to_host(v.xz, N);
    const float *bx, *by, *bz, *bm;
    uint32_t nb = 0;
    check(reyn_boundary_arrays(scene.bdy.handle(), &bx, &by, &bz, &bm, &nb));
    std::vector<float> hbx = to_host(bx, nb), hby = to_host(by, nb), hbz = to_host(bz, nb);

    const B3 W(2.f * scene.h);
    auto solver { IISPH<B3, Resort::yes>(W, scene.N, 0.001f, scene.h, scene.rho0) };
    std::vector<uint32_t> iters_log;
    uint32_t iters = 0;
    float dt = 0.0005f;
    for (uint32_t s = 0; s < steps; ++s) {
        dt = simple_dt_controller(iters, dt, 1.0f, scene.h, state, make_float3(0.f, -9.81f, 0.f),
            10, 0.001f);
        const auto grid { scene.get_grid(state, 2.f) };
        iters = solver.step(state, grid, scene.bdy, dt);
        scene.hard_enforce_bounds(state);
        iters_log.push_back(iters);
    }
    v = state.soa();
    std::vector<float> x1 = to_host(v.xx, N), y1 = to_host(v.xy, N), z1 = to_host(v.xz, N);
    FILE* o = std::fopen(out, "wb");
    if (!o)
        throw Error(REYN_ERR_INVALID, "cannot open the output file");
    const uint32_t hdr[3] = { N, nb, steps };
    const float geo[7] = { scene.h, scene.bound_min.x, scene.bound_min.y, scene.bound_min.z,
        scene.bound_max.x, scene.bound_max.y, scene.bound_max.z };
    std::fwrite(hdr, 4, 3, o);
    std::fwrite(geo, 4, 7, o);
    for (const auto* a : { &x0, &y0, &z0, &hbx, &hby, &hbz })
        std::fwrite(a->data(), 4, a->size(), o);
    std::fwrite(iters_log.data(), 4, iters_log.size(), o);
    for (const auto* a : { &x1, &y1, &z1 })
        std::fwrite(a->data(), 4, a->size(), o);
    std::fclose(o);
}

int main(int argc, char** argv)
{
    if (argc != 6)
        return 2;
    const std::string mode = argv[3];
    const uint32_t n_desired = uint32_t(std::atoi(argv[4]));
    const uint32_t steps = uint32_t(std::atoi(argv[5]));
    try {
        Particles state(1, 1000.f);
        if (mode == "box") {
            Scene scene(argv[1], n_desired, make_float3(0.05f, 0.05f, 0.05f),
                make_float3(0.45f, 0.4f, 0.4f), 1000.f, state, 3.f, 1.f);
            run(scene, state, argv[2], steps);
        } else {
            Scene scene { Scene::from_obj(argv[1], n_desired, 1000.f, state, 3.f, 1.f) };
            run(scene, state, argv[2], steps);
        }
    } catch (const std::exception& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
