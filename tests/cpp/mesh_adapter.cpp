// The mesh adapters of include/reyn_b200.hpp in the reference's own calling
// pattern (sample_mesh, sample_boundary.cu:391-439): a host Mesh (a unit
// octahedron scaled by argv[1]), DeviceMesh::from, uniform_sample_mesh,
// relax_sampling with a CSV debug stream, LBVH::project, BoundarySamples.
// Prints the sample count, the first and last relaxation lines and the
// largest distance of a projected sample from the surface |x|+|y|+|z| = r.
#include "reyn_b200.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <sstream>

using namespace reyn;

int main(int argc, char** argv)
{
    const double r = argc > 1 ? std::atof(argv[1]) : 1.0;
    Mesh m;
    const double v[6][3] = { { r, 0, 0 }, { -r, 0, 0 }, { 0, r, 0 }, { 0, -r, 0 }, { 0, 0, r },
        { 0, 0, -r } };
    for (auto& p : v) {
        m.xs.push_back(p[0]);
        m.ys.push_back(p[1]);
        m.zs.push_back(p[2]);
    }
    // outward winding: (x, y, z) octant faces
    const unsigned f[8][3] = { { 0, 2, 4 }, { 2, 1, 4 }, { 1, 3, 4 }, { 3, 0, 4 }, { 2, 0, 5 },
        { 1, 2, 5 }, { 3, 1, 5 }, { 0, 3, 5 } };
    for (auto& t : f)
        m.faces.push_back(make_uint3(t[0], t[1], t[2]));
    const DeviceMesh dm = DeviceMesh::from(m);
    const float h = 0.05f;
    const uint32_t n = uniform_sample_mesh(nullptr, nullptr, nullptr, 0, dm, h, 2.f);
    float *xs, *ys, *zs;
    cudaMalloc(&xs, n * sizeof(float));
    cudaMalloc(&ys, n * sizeof(float));
    cudaMalloc(&zs, n * sizeof(float));
    uniform_sample_mesh(xs, ys, zs, n, dm, h, 2.f);
    std::ostringstream csv;
    relax_sampling(xs, ys, zs, n, dm, h / 2.f, &csv, 1.f, 10);
    const LBVH lbvh(&dm);
    lbvh.project(xs, ys, zs, n);
    const BoundarySamples bdy(xs, ys, zs, nullptr, n, h, 1000.f);
    std::vector<float> hx(n), hy(n), hz(n);
    cudaMemcpy(hx.data(), xs, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(hy.data(), ys, n * sizeof(float), cudaMemcpyDeviceToHost);
    cudaMemcpy(hz.data(), zs, n * sizeof(float), cudaMemcpyDeviceToHost);
    double worst = 0.0;
    for (uint32_t i = 0; i < n; ++i)
        worst = std::fmax(worst, std::fabs(std::fabs(hx[i]) + std::fabs(hy[i]) + std::fabs(hz[i]) - r));
    const std::string lines = csv.str();
    const size_t first_end = lines.find('\n');
    const size_t last_start = lines.rfind('\n', lines.size() - 2) + 1;
    std::printf("%u\n%s\n%s%.3g\n%.17g\n", n, lines.substr(0, first_end).c_str(),
        lines.substr(last_start).c_str(), worst, dm.get_volume());
    cudaFree(xs);
    cudaFree(ys);
    cudaFree(zs);
    return 0;
}
