// State export: particle positions as a binary PLY point cloud (the
// reference's save_to_ply, ply_io.cu:7-55) and the full SoA state as a raw
// dump for checkpoints (no counterpart in the reference).
//
// The PLY payload is the positions interleaved x0 y0 z0 x1 y1 z1 ... as
// native-endian float32. The interleave runs on the GPU (one kernel over the
// three SoA arrays into one staging array), so the host receives the payload
// in a single copy and writes it in one call instead of transposing element
// by element.
#include "engine.cuh"

#include <algorithm>
#include <cstdio>
#include <memory>
#include <vector>

namespace reyn {

__global__ void k_interleave_xyz(uint32_t n, const float* __restrict__ x,
    const float* __restrict__ y, const float* __restrict__ z, float* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    out[3 * size_t(i)] = x[i];
    out[3 * size_t(i) + 1] = y[i];
    out[3 * size_t(i) + 2] = z[i];
}

namespace {

    struct File {
        FILE* f = nullptr;
        explicit File(const char* path, const char* mode) : f(std::fopen(path, mode))
        {
            if (!f)
                fail(REYN_ERR_INVALID, std::string("cannot open ") + path);
        }
        ~File()
        {
            if (f)
                std::fclose(f);
        }
        void write(const void* p, size_t bytes)
        {
            if (bytes && std::fwrite(p, 1, bytes, f) != bytes)
                fail(REYN_ERR_INVALID, "short write");
        }
        void read(void* p, size_t bytes)
        {
            if (bytes && std::fread(p, 1, bytes, f) != bytes)
                fail(REYN_ERR_INVALID, "short read: not a complete raw state file");
        }
        void close()
        {
            if (f && std::fclose(f) != 0) {
                f = nullptr;
                fail(REYN_ERR_INVALID, "close failed");
            }
            f = nullptr;
        }
    };

    // raw state file: magic, particle count, rest density, field count, then
    // the fields in SoA order (xx, xy, xz, vx, vy, vz, m), native-endian
    constexpr char RAW_MAGIC[8] = { 'R', 'E', 'Y', 'N', 'S', 'O', 'A', '1' };

} // namespace

void save_ply(const reyn_particles& st, const char* path, cudaStream_t s)
{
    static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__
            || __BYTE_ORDER__ == __ORDER_BIG_ENDIAN__,
        "mixed-endian hosts are not supported");
    const uint32_t n = st.n;
    std::vector<float> host(size_t(n) * 3);
    if (n) {
        DevArray<float> staging(size_t(n) * 3);
        REYN_KERNEL("k_interleave_xyz", s,
            k_interleave_xyz<<<blocks_for(n, THREADS), THREADS, 0, s>>>(n, st.cur[FX].get(),
            st.cur[FY].get(), st.cur[FZ].get(), staging.get()));
        REYN_CUDA(cudaMemcpyAsync(host.data(), staging.get(), host.size() * sizeof(float),
            cudaMemcpyDeviceToHost, s));
        REYN_CUDA(cudaStreamSynchronize(s));
    }
    const char* endian = __BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__ ? "little" : "big";
    char header[512];
    const int len = std::snprintf(header, sizeof(header),
        "ply\nformat binary_%s_endian 1.0\n"
        "comment particle positions written by reyn_b200\n"
        "element vertex %u\nproperty float32 x\nproperty float32 y\nproperty float32 z\n"
        "end_header\n",
        endian, n);
    File f(path, "wb");
    f.write(header, size_t(len));
    f.write(host.data(), host.size() * sizeof(float));
    f.close();
}

void save_raw(const reyn_particles& st, const char* path, cudaStream_t s)
{
    const uint32_t n = st.n;
    std::vector<float> host(size_t(n) * NFIELDS);
    for (int k = 0; k < NFIELDS; ++k)
        if (n)
            REYN_CUDA(cudaMemcpyAsync(host.data() + size_t(k) * n, st.cur[k].get(),
                size_t(n) * sizeof(float), cudaMemcpyDeviceToHost, s));
    REYN_CUDA(cudaStreamSynchronize(s));
    File f(path, "wb");
    const uint32_t nf = NFIELDS;
    f.write(RAW_MAGIC, sizeof(RAW_MAGIC));
    f.write(&n, sizeof(n));
    f.write(&st.rho0, sizeof(st.rho0));
    f.write(&nf, sizeof(nf));
    f.write(host.data(), host.size() * sizeof(float));
    f.close();
}

void load_raw(reyn_particles& st, const char* path, cudaStream_t s)
{
    File f(path, "rb");
    char magic[8];
    uint32_t n = 0, nf = 0;
    float rho0 = 0.f;
    f.read(magic, sizeof(magic));
    require(std::equal(magic, magic + 8, RAW_MAGIC), "not a raw state file");
    f.read(&n, sizeof(n));
    f.read(&rho0, sizeof(rho0));
    f.read(&nf, sizeof(nf));
    require(nf == NFIELDS, "raw state file with an unexpected field count");
    require(n == st.n, "raw state file holds a different particle count");
    std::vector<float> host(size_t(n) * NFIELDS);
    f.read(host.data(), host.size() * sizeof(float));
    for (int k = 0; k < NFIELDS; ++k)
        if (n)
            REYN_CUDA(cudaMemcpyAsync(st.cur[k].get(), host.data() + size_t(k) * n,
                size_t(n) * sizeof(float), cudaMemcpyHostToDevice, s));
    // the host vector must outlive the copies
    REYN_CUDA(cudaStreamSynchronize(s));
    st.packed_valid = false;
    st.version += 1;
}

} // namespace reyn

using namespace reyn;

extern "C" int reyn_particles_save_ply(reyn_particles* p, const char* path, void* stream)
{
    return guard([&] {
        require(p && path, "null argument");
        save_ply(*p, path, as_stream(stream));
    });
}

extern "C" int reyn_particles_save_raw(reyn_particles* p, const char* path, void* stream)
{
    return guard([&] {
        require(p && path, "null argument");
        save_raw(*p, path, as_stream(stream));
    });
}

extern "C" int reyn_particles_load_raw(reyn_particles* p, const char* path, void* stream)
{
    return guard([&] {
        require(p && path, "null argument");
        load_raw(*p, path, as_stream(stream));
    });
}
