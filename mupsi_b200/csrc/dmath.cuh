// Device arithmetic shared by the kernels.
//
// The library is compiled with --fmad=false, so every float expression below
// rounds exactly as written (no silent a*b+c contraction); FMA is used only
// where a kernel asks for it explicitly with fmaf(). Vector reductions follow
// the reference's Eigen order for 3-vectors, v0 + (v1 + v2), so dot products,
// norms and normalisations reproduce the reference bit for bit.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define MD __device__ __forceinline__
#define MHD __host__ __device__ __forceinline__

struct v3 {
  float x, y, z;
};
MHD v3 mk3(float x, float y, float z) { return v3{x, y, z}; }
MHD v3 operator+(v3 a, v3 b) { return v3{a.x + b.x, a.y + b.y, a.z + b.z}; }
MHD v3 operator-(v3 a, v3 b) { return v3{a.x - b.x, a.y - b.y, a.z - b.z}; }
MHD v3 operator-(v3 a) { return v3{-a.x, -a.y, -a.z}; }
MHD v3 operator*(v3 a, float s) { return v3{a.x * s, a.y * s, a.z * s}; }
MHD v3 operator*(float s, v3 a) { return v3{s * a.x, s * a.y, s * a.z}; }
MHD v3 operator/(v3 a, float s) { return v3{a.x / s, a.y / s, a.z / s}; }
MHD v3 cmul(v3 a, v3 b) { return v3{a.x * b.x, a.y * b.y, a.z * b.z}; }
MHD float dot(v3 a, v3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
MHD float sqn(v3 a) { return dot(a, a); }
MHD float norm3(v3 a) { return sqrtf(sqn(a)); }
MHD v3 normalized(v3 a) {
  float z = sqn(a);
  return z > 0.0f ? a / sqrtf(z) : a;
}
MHD v3 cross(v3 a, v3 b) { return v3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
MHD float fmin_std(float a, float b) { return (b < a) ? b : a; }  // std::min
MHD float fmax_std(float a, float b) { return (a < b) ? b : a; }  // std::max
MHD float maxc(v3 a) { return fmax_std(a.x, fmax_std(a.y, a.z)); }
MHD float get(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
MHD v3 ld3(const float* p) { return v3{p[0], p[1], p[2]}; }
MHD void st3(float* p, v3 a) {
  p[0] = a.x;
  p[1] = a.y;
  p[2] = a.z;
}

// 4x4 column-major transform; products reduce over k as the reference's
// matrix-vector products do: rows of M*(p,w) as (m0 x + m1 y) + (m2 z + m3 w),
// 3x3 blocks as m0 x + (m1 y + m2 z).
struct m4 {
  float m[16];
};
MHD float M4(const m4& a, int i, int j) { return a.m[j * 4 + i]; }
MHD v3 apply4(const m4& a, v3 p) {
  return v3{(M4(a, 0, 0) * p.x + M4(a, 0, 1) * p.y) + (M4(a, 0, 2) * p.z + M4(a, 0, 3) * 1.0f),
            (M4(a, 1, 0) * p.x + M4(a, 1, 1) * p.y) + (M4(a, 1, 2) * p.z + M4(a, 1, 3) * 1.0f),
            (M4(a, 2, 0) * p.x + M4(a, 2, 1) * p.y) + (M4(a, 2, 2) * p.z + M4(a, 2, 3) * 1.0f)};
}
MHD v3 apply3(const m4& a, v3 v) {
  return v3{M4(a, 0, 0) * v.x + (M4(a, 0, 1) * v.y + M4(a, 0, 2) * v.z),
            M4(a, 1, 0) * v.x + (M4(a, 1, 1) * v.y + M4(a, 1, 2) * v.z),
            M4(a, 2, 0) * v.x + (M4(a, 2, 1) * v.y + M4(a, 2, 2) * v.z)};
}
// topLeftCorner<3,3>().transpose() * v
MHD v3 apply3t(const m4& a, v3 v) {
  return v3{M4(a, 0, 0) * v.x + (M4(a, 1, 0) * v.y + M4(a, 2, 0) * v.z),
            M4(a, 0, 1) * v.x + (M4(a, 1, 1) * v.y + M4(a, 2, 1) * v.z),
            M4(a, 0, 2) * v.x + (M4(a, 1, 2) * v.y + M4(a, 2, 2) * v.z)};
}

// ---- hashing and PCG32 (the reference's math/random.h) ----------------------
MHD void hash_combine(uint32_t& seed, uint32_t v) { seed ^= v + 0x9e3779b9u + (seed << 6) + (seed >> 2); }
MHD uint32_t make_seed4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  uint32_t h = 0;
  hash_combine(h, a);
  hash_combine(h, b);
  hash_combine(h, c);
  hash_combine(h, d);
  return h;
}
MHD uint32_t make_seed5(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t e) {
  uint32_t h = make_seed4(a, b, c, d);
  hash_combine(h, e);
  return h;
}

// XSH-RR output of the old state, LCG step with increment 1.
MHD uint32_t pcg_next(uint64_t& state) {
  uint64_t old = state;
  state = old * 6364136223846793005ULL + 1ULL;
  uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
  uint32_t rot = (uint32_t)(old >> 59u);
#ifdef __CUDA_ARCH__
  return __funnelshift_r(xs, xs, rot);
#else
  return (xs >> rot) | (xs << ((uint32_t)(-(int32_t)rot) & 31u));
#endif
}
// (i >> 9) | 0x3F800000 as a float, minus 1: uniform in [0, 1)
MHD float u01(uint32_t i) {
#ifdef __CUDA_ARCH__
  return __uint_as_float((i >> 9u) + 0x3F800000u) - 1.0f;
#else
  union {
    uint32_t u;
    float f;
  } c;
  c.u = (i >> 9u) | 0x3F800000u;
  return c.f - 1.0f;
#endif
}
MHD float pcg_next1d(uint64_t& state) { return u01(pcg_next(state)); }
// Random(seed): a zero seed becomes 1, then two warm-up draws.
MHD uint64_t pcg_seeded(uint64_t seed) {
  uint64_t s = seed == 0 ? 1 : seed;
  pcg_next(s);
  pcg_next(s);
  return s;
}
// ConstantSampler(seed).nextI(): the fifth output of Random(seed)'s stream
// (two warm-ups, x, y, then i).
MHD uint32_t constant_sampler_i(uint32_t seed) {
  uint64_t s = pcg_seeded(seed);
  pcg_next(s);
  pcg_next(s);
  return pcg_next(s);
}
