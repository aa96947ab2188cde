// Test infrastructure only: evaluates the reference's OWN smoothing-kernel
// classes (reyn src/kernels.cuh:19-165, compiled unmodified) on the HOST, so
// golden kernel vectors can be produced on a machine without a GPU. On the
// host the reference's `norm` is fsqrt(dot) and `sat` is fmin/fmax
// (src/utils/vector.cuh:236-268).
#include "kernels.cuh"

namespace {
template <typename K>
void eval(const K& W, unsigned n, const float* dx, const float* dy,
    const float* dz, float* w, float* gx, float* gy, float* gz)
{
    for (unsigned i = 0; i < n; ++i) {
        const float3 d = make_float3(dx[i], dy[i], dz[i]);
        w[i] = W(d);
        const float3 g = W.nabla(d);
        gx[i] = g.x;
        gy[i] = g.y;
        gz[i] = g.z;
    }
}
}

extern "C" int ref_kernel_eval_host(int kind, float h_bar, unsigned n,
    const float* dx, const float* dy, const float* dz, float* w, float* gx,
    float* gy, float* gz)
{
    switch (kind) {
    case 0: eval(C2(h_bar), n, dx, dy, dz, w, gx, gy, gz); return 0;
    case 1: eval(B3(h_bar), n, dx, dy, dz, w, gx, gy, gz); return 0;
    case 2: eval(W6(h_bar), n, dx, dy, dz, w, gx, gy, gz); return 0;
    case 3: eval(COS(h_bar), n, dx, dy, dz, w, gx, gy, gz); return 0;
    default: return -1;
    }
}
