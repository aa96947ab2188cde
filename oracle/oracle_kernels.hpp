// CPU ORACLE — test infrastructure only (see oracle.h). Vector helpers and
// the four smoothing kernels (kernels.cuh:19-165, host flavour), shared by
// the oracle translation units. Included inside an anonymous namespace,
// after <cmath> and <cstdint>.
#pragma once

struct f3 {
    float x, y, z;
};
inline f3 mk(float x, float y, float z) { return f3 { x, y, z }; }
inline f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline f3& operator+=(f3& a, f3 b)
{
    a.x += b.x;
    a.y += b.y;
    a.z += b.z;
    return a;
}
inline f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }
// scalar * vector as in vector.cuh:184-191 (component * scalar)
inline f3 operator*(float s, f3 b) { return mk(b.x * s, b.y * s, b.z * s); }
// vector.cuh:152-155: nested fmaf
inline float dot(f3 a, f3 b)
{
    return std::fmaf(a.x, b.x, std::fmaf(a.y, b.y, a.z * b.z));
}
// host flavour of vector.cuh:261-268 (fsqrt of the float dot product)
inline float norm(f3 a) { return (float)std::sqrt((double)dot(a, a)); }
// host flavour of vector.cuh:236-243
inline float sat(float a) { return std::fmin(std::fmax(a, 0.f), 1.f); }
inline f3 load(uint32_t i, const float* x, const float* y, const float* z)
{
    return mk(x[i], y[i], z[i]);
}
inline void store(f3 v, uint32_t i, float* x, float* y, float* z)
{
    x[i] = v.x;
    y[i] = v.y;
    z[i] = v.z;
}

// ---- smoothing kernels, kernels.cuh:19-165 -------------------------------

struct KBase {
    float h_inv, w_scale, dw_scale;
    // kernels.cuh:32-37
    KBase(float h, float alpha)
        : h_inv(1.0f / h)
        , w_scale(alpha / (h * h * h))
        , dw_scale(alpha / (h * h * h * h))
    {
    }
};

struct C2 : KBase { // kernels.cuh:78-95
    explicit C2(float h) : KBase(h, (float)(21.f / 2.f * M_1_PI)) { }
    static float w(float q)
    {
        const float t1 = std::fmax(0.f, 1.f - q);
        const float t2 = 4.f * q + 1.f;
        const float t1_2 = t1 * t1;
        return t1_2 * t1_2 * t2;
    }
    static float dw(float q)
    {
        const float t1 = std::fmax(0.f, 1.f - q);
        const float t2 = -20.f * q;
        return t1 * t1 * t1 * t2;
    }
};
struct B3 : KBase { // kernels.cuh:101-118
    explicit B3(float h) : KBase(h, (float)(16.f * M_1_PI)) { }
    static float w(float q)
    {
        const float t1 = std::fmax(0.f, 1.f - q);
        const float t2 = sat(0.5f - q);
        return t1 * t1 * t1 - 4.f * t2 * t2 * t2;
    }
    static float dw(float q)
    {
        const float t1 = std::fmax(0.f, 1.f - q);
        const float t2 = sat(0.5f - q);
        return -3.f * t1 * t1 + 12.f * t2 * t2;
    }
};
struct W6 : KBase { // kernels.cuh:121-145
    explicit W6(float h) : KBase(h, (float)(1365.f / 64.f * M_1_PI)) { }
    static float w(float q)
    {
        const float t1 = std::fmax(0.f, 1.f - q);
        const float t1_2 = t1 * t1;
        const float t1_4 = t1_2 * t1_2;
        const float t1_8 = t1_4 * t1_4;
        const float q_2 = q * q;
        const float t2 = 32.f * q_2 * q + 25.f * q_2 + 8.f * q + 1.f;
        return t1_8 * t2;
    }
    static float dw(float q)
    {
        const float t1 = std::fmax(0.f, 1.f - q);
        const float t1_2 = t1 * t1;
        const float t1_4 = t1_2 * t1_2;
        const float t1_7 = t1_4 * t1_2 * t1;
        const float t2 = (16.f * q * q + 7.f * q + 1.f) * (-22.f * q);
        return t1_7 * t2;
    }
};
struct COS : KBase { // kernels.cuh:148-165
    explicit COS(float h)
        : KBase(h, (float)(M_PI / (4.f * M_PI * M_PI - 30.f)))
    {
    }
    static float w(float q)
    {
        const float PI = (float)M_PI;
        const float pi_s = PI * std::fmin(1.f, q);
        return 4.f * std::cos(pi_s) + std::cos(2.f * pi_s) + 3.f;
    }
    static float dw(float q)
    {
        const float PI = (float)M_PI;
        const float pi_s = PI * std::fmin(1.f, q);
        const float two_pi = (float)(2.f * M_PI);
        return -2.f * two_pi * std::sin(pi_s) - std::sin(2.f * pi_s) * two_pi;
    }
};

// kernels.cuh:40-49
template <class K> inline float W(const K& k, f3 dx)
{
    const float len = norm(dx);
    const float q = sat(len * k.h_inv);
    return k.w_scale * K::w(q);
}
// kernels.cuh:51-64
template <class K> inline f3 dW(const K& k, f3 dx)
{
    const float len = norm(dx);
    const float one_over_len = 1.f / len;
    const float q = len * k.h_inv;
    const float scale = k.dw_scale * K::dw(q) * one_over_len;
    const float safe = std::isfinite(scale) ? scale : 0.f;
    return safe * dx;
}

template <class F> int with_kernel(int kind, float h, F&& f)
{
    switch (kind) {
    case 0: f(C2(h)); return 0;
    case 1: f(B3(h)); return 0;
    case 2: f(W6(h)); return 0;
    case 3: f(COS(h)); return 0;
    default: return -1;
    }
}
