// Sparse-convolution GP noise psi / grad psi and the Renewal+ conditioning terms
// (the reference's gp/kernel.h:39-78, gp/gpnoise.cpp:51-87, gpnoise.h:31,44,
// medium/gpmedium.cpp:26-41).
//
// Bit-exact parts (shared with the reference): the grid cell of p
// (trunc(p/kr) with an IEEE division), the per-cell seed make_seed(cx,cy,cz,seed),
// the PCG stream started at cell_seed + 1 (32-bit wrap), the impulse positions
// s = cell*kr + U^3*kr and the +-1 weights, and the accumulation order
// (dx, dy, dz, i). The Gaussian h uses the SFU exp2 (ex2.approx) on the
// argument |p-s|^2 * (-log2(e)/L2); the reference calls glibc expf on
// -|p-s|^2 / L2. The resulting psi differs from the reference by ~1e-7 of the
// sum of |terms| (tested at 1e-5).
#pragma once
#include <climits>

#include "dmath.cuh"

struct KParams {
  float sigma;       // kernel sigma
  float kr;          // kernel radius = grid cell size
  float L2;          // |aniso|^2, computed as the reference does (a0^2 + (a1^2 + a2^2))
  float sqrt_var;    // sqrtf(float(ppc / kr^3 * pi^1.5)) (gpnoise.h:31,44)
  float k2;          // -log2(e) / L2: exp(-r2/L2) = exp2(r2 * k2)
  float c2;          // -2.0f / L2 (kernel.h:57)
  float c4;          // 4.0f / (L2 * L2) (kernel.h:64)
  float psi_bound;   // max over p of psi_bound_at(p) (<= sigma * 27 * ppc / sqrt_var)
  float gradh_max;   // max over r of |grad h| = sqrt(2/L2) * exp(-1/2)
  float psi_scale;   // sigma * ppc / sqrt_var
  int ppc;           // impulses per cell
};

MD float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Grid cell of p: (p / kr).cast<int>() (gpnoise.cpp:54), truncation toward zero.
MD void cell_of(const KParams& k, v3 p, int& cx, int& cy, int& cz) {
  cx = (int)(p.x / k.kr);
  cy = (int)(p.y / k.kr);
  cz = (int)(p.z / k.kr);
}

// Impulses of one cell, visited in the reference's order. F(s, w) is called per
// impulse with its position and sign (+1 / -1).
template <typename F>
MD void for_each_impulse(const KParams& k, int nx, int ny, int nz, uint32_t seed, F&& f) {
  uint32_t cs = make_seed4((uint32_t)nx, (uint32_t)ny, (uint32_t)nz, seed);
  uint64_t st = (uint64_t)(uint32_t)(cs + 1u);
  const float bx = (float)nx * k.kr, by = (float)ny * k.kr, bz = (float)nz * k.kr;
  for (int i = 0; i < k.ppc; ++i) {
    // Vector3f(next1D(), next1D(), next1D()) as the reference's build evaluates it:
    // constructor arguments right to left, so the first draw is z.
    float a = pcg_next1d(st);
    float b = pcg_next1d(st);
    float c = pcg_next1d(st);
    v3 s = v3{bx + c * k.kr, by + b * k.kr, bz + a * k.kr};
    float w = pcg_next1d(st) < 0.5f ? -1.0f : 1.0f;
    f(s, w);
  }
}

// Unnormalised InternalNoise sums over neighbour cells [c0, c1) of the 27, in
// the reference's (dx, dy, dz) order (cell c = 9(dx+1) + 3(dy+1) + (dz+1)).
// GRAD = false computes the value only.
template <bool GRAD>
MD void psi_sums_range(const KParams& k, v3 p, uint32_t seed, int c0, int c1, float& sv, float& sx, float& sy,
                       float& sz) {
  int cx, cy, cz;
  cell_of(k, p, cx, cy, cz);
  float v = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
#pragma unroll 1
  for (int c = c0; c < c1; ++c) {
    const int dx = c / 9 - 1, dy = (c / 3) % 3 - 1, dz = c % 3 - 1;
    for_each_impulse(k, cx + dx, cy + dy, cz + dz, seed, [&](v3 s, float w) {
      v3 d = p - s;
      float r2 = d.x * d.x + (d.y * d.y + d.z * d.z);
      float h = ex2_approx(r2 * k.k2);
      v = fmaf(w, h, v);  // w = +-1: w*h is exact, so this equals v + w*h
      if (GRAD) {
        float gs = h * k.c2;
        gx = fmaf(w, gs * d.x, gx);
        gy = fmaf(w, gs * d.y, gy);
        gz = fmaf(w, gs * d.z, gz);
      }
    });
  }
  sv = v;
  sx = gx;
  sy = gy;
  sz = gz;
}
template <bool GRAD>
MD void psi_sums(const KParams& k, v3 p, uint32_t seed, float& sv, float& sx, float& sy, float& sz) {
  psi_sums_range<GRAD>(k, p, seed, 0, 27, sv, sx, sy, sz);
}

// A group of G lanes (G a power of two, lanes gbase..gbase+G-1 of the warp)
// shares one evaluation: lane `sub` sums a contiguous block of the 27 cells and
// the block sums are added with a butterfly over the group, so every lane of the
// group ends with the same total. With G = 1 this is the sequential sum above.
struct Group {
  int G, sub;
  unsigned mask;
};
MD float group_sum(const Group& g, float v) {
  for (int off = 1; off < g.G; off <<= 1) v += __shfl_xor_sync(g.mask, v, off, g.G);
  return v;
}
MD void group_cells(const Group& g, int& c0, int& c1) {
  const int per = (27 + g.G - 1) / g.G;
  c0 = min(27, g.sub * per);
  c1 = min(27, c0 + per);
}
MD float raw_noise_value_group(const KParams& k, v3 p, uint32_t seed, const Group& g) {
  int c0, c1;
  group_cells(g, c0, c1);
  float v, x, y, z;
  psi_sums_range<false>(k, p, seed, c0, c1, v, x, y, z);
  v = group_sum(g, v);
  return (k.sigma * v) / k.sqrt_var;
}
MD float4 raw_noise_group(const KParams& k, v3 p, uint32_t seed, const Group& g) {
  int c0, c1;
  group_cells(g, c0, c1);
  float v, x, y, z;
  psi_sums_range<true>(k, p, seed, c0, c1, v, x, y, z);
  v = group_sum(g, v);
  x = group_sum(g, x);
  y = group_sum(g, y);
  z = group_sum(g, z);
  return make_float4((k.sigma * v) / k.sqrt_var, (k.sigma * x) / k.sqrt_var, (k.sigma * y) / k.sqrt_var,
                     (k.sigma * z) / k.sqrt_var);
}

// ---- impulse cache for marches --------------------------------------------
// Consecutive march steps of one ray share most of their 27 neighbour cells
// (dt = 0.5 against cells of size kr). A lane group keeps the impulses of the
// current 3x3x3 window in shared memory, one slot per cell of a mod-3 torus
// (slot = (cx mod 3, cy mod 3, cz mod 3)): moving the window by one cell
// replaces exactly the 9 slots of the layer it leaves. Lane `sub` owns the
// slots s with s % G == sub, so no slot is shared between lanes. A slot holds
// its cell's coordinates and ppc (s.x, s.y, s.z, w) records, computed exactly
// as for_each_impulse computes them.
#define CACHE_MAX_PPC 3
struct ImpCache {
  int* tag;      // [27 * 3]: cell coordinates held by each slot
  float4* imp;   // [27 * CACHE_MAX_PPC]
};
// per lane group: the float4 records first, then the tags; a multiple of 16 so
// every group's records start 16-byte aligned
constexpr int kCacheBytes = ((27 * CACHE_MAX_PPC * 16 + 27 * 3 * 4) + 15) / 16 * 16;
static_assert(kCacheBytes % 16 == 0, "lane-group cache stride must keep float4 alignment");

MD int mod3(int x) { return ((x % 3) + 3) % 3; }
MD void cache_clear(ImpCache c, const Group& g) {
  for (int s = g.sub; s < 27; s += g.G) c.tag[3 * s] = INT_MIN;
}
template <bool GRAD>
MD void psi_sums_cached(const KParams& k, v3 p, uint32_t seed, const Group& g, ImpCache c, float& sv, float& sx,
                        float& sy, float& sz) {
  int cx, cy, cz;
  cell_of(k, p, cx, cy, cz);
  float v = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
#pragma unroll 1
  for (int s = g.sub; s < 27; s += g.G) {
    // the cell of the window [c-1, c+1]^3 that maps to slot s
    const int ax = cx - 1 + mod3(s / 9 - (cx - 1));
    const int ay = cy - 1 + mod3((s / 3) % 3 - (cy - 1));
    const int az = cz - 1 + mod3(s % 3 - (cz - 1));
    int* t = c.tag + 3 * s;
    float4* I = c.imp + CACHE_MAX_PPC * s;
    if (t[0] != ax || t[1] != ay || t[2] != az) {
      int i = 0;
      for_each_impulse(k, ax, ay, az, seed, [&](v3 q, float w) { I[i++] = make_float4(q.x, q.y, q.z, w); });
      t[0] = ax;
      t[1] = ay;
      t[2] = az;
    }
    for (int i = 0; i < k.ppc; ++i) {
      const float4 q = I[i];
      v3 d = p - mk3(q.x, q.y, q.z);
      float r2 = d.x * d.x + (d.y * d.y + d.z * d.z);
      float h = ex2_approx(r2 * k.k2);
      v = fmaf(q.w, h, v);
      if (GRAD) {
        float gs = h * k.c2;
        gx = fmaf(q.w, gs * d.x, gx);
        gy = fmaf(q.w, gs * d.y, gy);
        gz = fmaf(q.w, gs * d.z, gz);
      }
    }
  }
  sv = v;
  sx = gx;
  sy = gy;
  sz = gz;
}
MD float raw_noise_value_cached(const KParams& k, v3 p, uint32_t seed, const Group& g, ImpCache c) {
  float v, x, y, z;
  psi_sums_cached<false>(k, p, seed, g, c, v, x, y, z);
  v = group_sum(g, v);
  return (k.sigma * v) / k.sqrt_var;
}
MD float4 raw_noise_cached(const KParams& k, v3 p, uint32_t seed, const Group& g, ImpCache c) {
  float v, x, y, z;
  psi_sums_cached<true>(k, p, seed, g, c, v, x, y, z);
  v = group_sum(g, v);
  x = group_sum(g, x);
  y = group_sum(g, y);
  z = group_sum(g, z);
  return make_float4((k.sigma * v) / k.sqrt_var, (k.sigma * x) / k.sqrt_var, (k.sigma * y) / k.sqrt_var,
                     (k.sigma * z) / k.sqrt_var);
}

// RawNoise(p, seed) = sigma * InternalNoise / sqrt(Var) (gpnoise.h:44)
MD float4 raw_noise(const KParams& k, v3 p, uint32_t seed) {
  float v, x, y, z;
  psi_sums<true>(k, p, seed, v, x, y, z);
  return make_float4((k.sigma * v) / k.sqrt_var, (k.sigma * x) / k.sqrt_var, (k.sigma * y) / k.sqrt_var,
                     (k.sigma * z) / k.sqrt_var);
}
MD float raw_noise_value(const KParams& k, v3 p, uint32_t seed) {
  float v, x, y, z;
  psi_sums<false>(k, p, seed, v, x, y, z);
  return (k.sigma * v) / k.sqrt_var;
}

struct Cond {
  v3 C;
  float u;
  v3 g;
  uint32_t active;
};

// h(C, p) with the accurate expf and the reference's division (kernel.h:52-54)
MD float h_exact(const KParams& k, v3 C, v3 p) { return expf(-sqn(p - C) / k.L2); }

// Value part of the conditioning: u*h(C,p) + g . grad h(C,p) (gpmedium.cpp:34-35)
MD float cond_value(const KParams& k, const Cond& c, v3 p) {
  float h = h_exact(k, c.C, p);
  v3 hg = (h * k.c2) * (p - c.C);
  return c.u * h + dot(c.g, hg);
}
// Conditioning terms added to (f, grad f) (gpmedium.cpp:32-39)
MD float4 add_cond(const KParams& k, const Cond& c, v3 p, float4 f) {
  if (!c.active) return f;
  float h = h_exact(k, c.C, p);
  v3 r = p - c.C;
  v3 hg = (h * k.c2) * r;
  f.x += c.u * h + dot(c.g, hg);
  // H_h g = h * ((-2/L2) g + (4/L2^2)(r.g) r)
  v3 a = k.c2 * c.g;
  v3 b = (k.c4 * dot(r, c.g)) * r;
  v3 Hg = h * (a + b);
  f.y += c.u * hg.x + Hg.x;
  f.z += c.u * hg.y + Hg.y;
  f.w += c.u * hg.z + Hg.z;
  return f;
}
// Bound on |u h + g . grad h| over all p (|h| <= 1, |grad h| <= gradh_max)
MD float cond_bound(const KParams& k, const Cond& c) {
  if (!c.active) return 0.0f;
  return fabsf(c.u) + norm3(c.g) * k.gradh_max;
}
// ... and at p: with r = |p - C|, h = exp(-r^2/L2) and |grad h| = h 2r/L2
MD float cond_bound_at(const KParams& k, const Cond& c, v3 p) {
  if (!c.active) return 0.0f;
  float r2 = sqn(p - c.C);
  float h = ex2_approx(r2 * k.k2);
  return (fabsf(c.u) + norm3(c.g) * (2.0f * sqrtf(r2) / k.L2)) * h;
}

// Bound on |psi(p)|. Every impulse of neighbour cell (cx+dx, cy+dy, cz+dz) lies
// in the box [cx+dx, cx+dx+1] x ... (times kr), and h factorises over the axes,
// so sum |w h| <= ppc * (sum_dx hx)(sum_dy hy)(sum_dz hz) with hx the largest
// exp(-(p.x - s.x)^2/L2) over the box's x range: 9 exponentials instead of the
// 27*ppc of psi itself.
MD float psi_bound_at(const KParams& k, v3 p) {
  int c[3];
  cell_of(k, p, c[0], c[1], c[2]);
  float prod = 1.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float pa = get(p, a);
    float sum = 0.0f;
#pragma unroll
    for (int d = -1; d <= 1; ++d) {
      const float lo = (float)(c[a] + d) * k.kr;
      const float hi = lo + k.kr;
      const float dist = fmaxf(0.0f, fmaxf(lo - pa, pa - hi));
      sum += ex2_approx(dist * dist * k.k2);
    }
    prod *= sum;
  }
  return k.psi_scale * prod;
}
