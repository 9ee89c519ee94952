// Sparse-convolution GP noise psi / grad psi and the Renewal+ conditioning terms
// (the reference's gp/kernel.h:39-78, gp/gpnoise.cpp:51-87, gpnoise.h:31,44,
// medium/gpmedium.cpp:26-41).
//
// Bit-exact parts (shared with the reference): the grid cell of p
// (trunc(p/kr) with an IEEE division), the per-cell seed make_seed(cx,cy,cz,seed),
// the PCG stream started at cell_seed + 1 (32-bit wrap), the impulse positions
// s = cell*kr + U^3*kr and the +-1 weights, and the accumulation order
// (dx, dy, dz, i). The Gaussian h uses the SFU exp2 (ex2.approx) on the
// argument |p-s|^2 * (-log2(e)/L2), |p-s|^2 formed with fused multiply-adds;
// the reference calls glibc expf on -|p-s|^2 / L2. The resulting psi differs from the reference by ~1e-7 of the
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
  int kr_pow2;       // kr is a power of two: p / kr == p * inv_kr, bit for bit
  float inv_kr;
};

MD float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// Grid cell of p: (p / kr).cast<int>() (gpnoise.cpp:54), truncation toward zero.
MD void cell_of(const KParams& k, v3 p, int& cx, int& cy, int& cz) {
  if (k.kr_pow2) {  // division by 2^e is the exact scaling by 2^-e, as the multiply is
    cx = (int)(p.x * k.inv_kr);
    cy = (int)(p.y * k.inv_kr);
    cz = (int)(p.z * k.inv_kr);
  } else {
    cx = (int)(p.x / k.kr);
    cy = (int)(p.y / k.kr);
    cz = (int)(p.z / k.kr);
  }
}

// Impulses of one cell, visited in the reference's order. F(s, wsign) is called
// per impulse with its position and the sign bit of its weight (0 for +1,
// 0x80000000 for -1).
template <typename F>
MD void cell_impulse(const KParams& k, uint64_t& st, float bx, float by, float bz, F&& f) {
  // Vector3f(next1D(), next1D(), next1D()) as the reference's build evaluates it:
  // constructor arguments right to left, so the first draw is z.
  float a = pcg_next1d(st);
  float b = pcg_next1d(st);
  float c = pcg_next1d(st);
  v3 s = v3{bx + c * k.kr, by + b * k.kr, bz + a * k.kr};
  // weight next1D() < 0.5 ? -1 : +1; next1D() = float((i >> 9) | 0x3F800000) - 1
  // is below 0.5 exactly when bit 31 of i is clear
  const uint32_t wsign = ~pcg_next(st) & 0x80000000u;
  f(s, wsign);
}
// The PCG32 state n steps after s0: s_n = A_n s0 + C_n (mod 2^64), A_n = M^n,
// C_n = M^(n-1) + ... + M + 1 for the LCG multiplier M and increment 1. Exact
// integer arithmetic: the same states as n sequential steps.
template <int N>
struct PcgAhead {
  static constexpr uint64_t A = PcgAhead<N - 1>::A * 6364136223846793005ULL;
  static constexpr uint64_t C = PcgAhead<N - 1>::C * 6364136223846793005ULL + 1ULL;
};
template <>
struct PcgAhead<0> {
  static constexpr uint64_t A = 1ULL, C = 0ULL;
};
// XSH-RR output of a state (the value pcg_next returns before stepping from it)
MD uint32_t pcg_output(uint64_t old) {
  const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
  const uint32_t rot = (uint32_t)(old >> 59u);
#ifdef __CUDA_ARCH__
  return __funnelshift_r(xs, xs, rot);
#else
  return (xs >> rot) | (xs << ((uint32_t)(-(int32_t)rot) & 31u));
#endif
}
// Impulse I of a cell whose stream starts at s0 (< 2^32: the cell seed + 1):
// draws 4I..4I+3, each from its own state computed from s0 (no chain of
// dependent LCG steps), the same values cell_impulse draws in sequence.
template <int I, typename F>
MD void cell_impulse_at(const KParams& k, uint64_t s0, float bx, float by, float bz, F&& f) {
  const float a = u01(pcg_output(PcgAhead<4 * I>::A * s0 + PcgAhead<4 * I>::C));
  const float b = u01(pcg_output(PcgAhead<4 * I + 1>::A * s0 + PcgAhead<4 * I + 1>::C));
  const float c = u01(pcg_output(PcgAhead<4 * I + 2>::A * s0 + PcgAhead<4 * I + 2>::C));
  const v3 s = v3{bx + c * k.kr, by + b * k.kr, bz + a * k.kr};
  const uint32_t wsign = ~pcg_output(PcgAhead<4 * I + 3>::A * s0 + PcgAhead<4 * I + 3>::C) & 0x80000000u;
  f(s, wsign);
}
template <int N, int I = 0, typename F>
MD void cell_impulses_ahead(const KParams& k, uint64_t s0, float bx, float by, float bz, F&& f) {
  if constexpr (I < N) {
    cell_impulse_at<I>(k, s0, bx, by, bz, f);
    cell_impulses_ahead<N, I + 1>(k, s0, bx, by, bz, f);
  }
}

// PPC > 0: k.ppc is known to be PPC at compile time (the batch entry's
// instantiations for the common counts); 0: a loop over k.ppc; -1: the same
// with the 3-impulse cell unrolled (the sphere-mean march kernels). Unrolled
// cells draw from jumped-ahead states (cell_impulse_at), the loop steps.
template <int PPC = 0, typename F>
MD void for_each_impulse(const KParams& k, int nx, int ny, int nz, uint32_t seed, F&& f) {
  uint32_t cs = make_seed4((uint32_t)nx, (uint32_t)ny, (uint32_t)nz, seed);
  uint64_t st = (uint64_t)(uint32_t)(cs + 1u);
  const float bx = (float)nx * k.kr, by = (float)ny * k.kr, bz = (float)nz * k.kr;
  if constexpr (PPC > 0) {
    cell_impulses_ahead<PPC>(k, st, bx, by, bz, f);
  } else {
    // the common count, unrolled: configuration-0 render 6.92 -> 6.71 ms.
    // Unrolling the 1- and 8-impulse cells as well made that render slower
    // (7.05 and 7.74 ms), unrolling the general loop by 2 or 4 gained nothing,
    // and in the mesh-mean march (32 registers) the unrolled cell cost 5%
    // (level-6 mesh render 704 -> 740 ms), so only PPC = -1 takes it.
    if constexpr (PPC < 0) {
      if (k.ppc == 3) {
        cell_impulses_ahead<3>(k, st, bx, by, bz, f);
        return;
      }
    }
    for (int i = 0; i < k.ppc; ++i) cell_impulse(k, st, bx, by, bz, f);
  }
}

#ifndef MUPSI_SLOT_PAIRS
#define MUPSI_SLOT_PAIRS 1  // value sums of a 3-impulse slot: both cells drawn at once
#endif
// One impulse's term w h (and w grad h when GRAD) added to the running sums.
template <bool GRAD>
struct PsiAcc {
  const KParams& k;
  v3 p;
  float v = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
  MD void operator()(v3 s, uint32_t wsign) {
    v3 d = p - s;
    // |p - s|^2 with two fused multiply-adds (psi carries the exp2
    // approximation's error already; the impulse positions stay exact)
    float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
    // w*h with w = +-1 and h >= 0: h with the weight's sign bit (exact)
    const float hs = __uint_as_float(__float_as_uint(ex2_approx(r2 * k.k2)) | wsign);
    v = v + hs;
    if (GRAD) {  // (w*h)*c2*d = w*((h*c2)*d) bit for bit: rounding is sign-symmetric
      float gs = hs * k.c2;
      gx = gx + gs * d.x;
      gy = gy + gs * d.y;
      gz = gz + gs * d.z;
    }
  }
};

// The signed terms w h of one cell's impulses in draw order, each formed as
// PsiAcc forms it (value only).
template <int N>
struct PsiTerms {
  const KParams& k;
  v3 p;
  float h[N];
  int n = 0;
  MD void operator()(v3 s, uint32_t wsign) {
    v3 d = p - s;
    float r2 = fmaf(d.x, d.x, fmaf(d.y, d.y, d.z * d.z));
    h[n++] = __uint_as_float(__float_as_uint(ex2_approx(r2 * k.k2)) | wsign);
  }
};
// The terms of cell c (0..27; 27 is outside the 27 neighbours and only ever
// drawn, never added) with 3 impulses per cell, from jumped-ahead states.
MD void cell_terms3(const KParams& k, int cx, int cy, int cz, uint32_t seed, int c, PsiTerms<3>& t) {
  const int nx = cx + c / 9 - 1, ny = cy + (c / 3) % 3 - 1, nz = cz + c % 3 - 1;
  const uint32_t cs = make_seed4((uint32_t)nx, (uint32_t)ny, (uint32_t)nz, seed);
  const uint64_t st = (uint64_t)(uint32_t)(cs + 1u);
  cell_impulses_ahead<3>(k, st, (float)nx * k.kr, (float)ny * k.kr, (float)nz * k.kr, t);
}
// Unnormalised InternalNoise sums over neighbour cells [c0, c1) of the 27, in
// the reference's (dx, dy, dz) order (cell c = 9(dx+1) + 3(dy+1) + (dz+1)).
// GRAD = false computes the value only.
template <bool GRAD, int PPC = 0>
MD void psi_sums_cells(const KParams& k, v3 p, int cx, int cy, int cz, uint32_t seed, int c0, int c1, float& sv,
                       float& sx, float& sy, float& sz) {
  if constexpr (!GRAD && PPC < 0 && MUPSI_SLOT_PAIRS) {
    if (k.ppc == 3 && c1 - c0 <= 2) {
      // a slot of one or two cells: both cells' impulses drawn at once (six
      // independent chains for the scheduler instead of two runs of three; a
      // one-cell slot's lanes wait for the two-cell ones anyway), then added
      // in the reference's order, so the same bits as the loop below
      PsiTerms<3> ta{k, p}, tb{k, p};
      cell_terms3(k, cx, cy, cz, seed, c0, ta);
      cell_terms3(k, cx, cy, cz, seed, c0 + 1, tb);
      float v = 0.0f;
      v = v + ta.h[0];
      v = v + ta.h[1];
      v = v + ta.h[2];
      if (c1 - c0 == 2) {
        v = v + tb.h[0];
        v = v + tb.h[1];
        v = v + tb.h[2];
      }
      sv = v;
      sx = sy = sz = 0.0f;
      return;
    }
  }
  PsiAcc<GRAD> acc{k, p};
#pragma unroll 1
  for (int c = c0; c < c1; ++c) {
    const int dx = c / 9 - 1, dy = (c / 3) % 3 - 1, dz = c % 3 - 1;
    for_each_impulse<PPC>(k, cx + dx, cy + dy, cz + dz, seed, acc);
  }
  sv = acc.v;
  sx = acc.gx;
  sy = acc.gy;
  sz = acc.gz;
}
template <bool GRAD, int PPC = 0>
MD void psi_sums_range(const KParams& k, v3 p, uint32_t seed, int c0, int c1, float& sv, float& sx, float& sy,
                       float& sz) {
  int cx, cy, cz;
  cell_of(k, p, cx, cy, cz);
  psi_sums_cells<GRAD, PPC>(k, p, cx, cy, cz, seed, c0, c1, sv, sx, sy, sz);
}
template <bool GRAD, int PPC = 0>
MD void psi_sums(const KParams& k, v3 p, uint32_t seed, float& sv, float& sx, float& sy, float& sz) {
  if constexpr (PPC > 0) {  // the same order with the dz cells unrolled (psi sweep 100 -> 81 ms)
    int cx, cy, cz;
    cell_of(k, p, cx, cy, cz);
    PsiAcc<GRAD> acc{k, p};
#pragma unroll 1
    for (int dx = -1; dx <= 1; ++dx) {
#pragma unroll 1
      for (int dy = -1; dy <= 1; ++dy) {
#pragma unroll
        for (int dz = -1; dz <= 1; ++dz) for_each_impulse<PPC>(k, cx + dx, cy + dy, cz + dz, seed, acc);
      }
    }
    sv = acc.v;
    sx = acc.gx;
    sy = acc.gy;
    sz = acc.gz;
  } else {
    psi_sums_range<GRAD, PPC>(k, p, seed, 0, 27, sv, sx, sy, sz);
  }
}

// A group of G lanes (G a power of two, lanes gbase..gbase+G-1 of the warp)
// shares one evaluation, and its sums are added in one fixed order whatever G
// is, so a ray's psi (and with it every march decision and hit normal) does not
// depend on the launch shape. The 27 cells are cut into 16 slots of one or two
// consecutive cells (sizes 2,2,2,1 | 2,2,2,1 | 2,2,2,1 | 2,2,1,1); a slot sums
// its cells' impulses from 0 in the reference's order, and the 16 slot sums are
// added by a perfect pairwise tree (slots 2i and 2i+1 first, then pairs of
// those, ...). Lane `sub` owns the V = max(1, 16/G) slots from sub V: it adds
// their subtree itself and the shuffles (offsets 1, 2, ..., up to 8) add the
// levels above; with G = 32, lanes 16-31 repeat lanes 0-15. Any 16/G
// consecutive slots hold at most ceil(27/G) cells for G = 4, 8, 16, so lanes
// are as evenly loaded as a plain split of the cells. Float addition commutes,
// so both lanes of a shuffle pair get the same bits.
struct Group {
  int G, sub;
  unsigned mask;
  // G = 1 only: a mesh mean's closest-point queries take the lane-group tie
  // rule (bvh_closest_lowtie), so a lane alone finds what a group of any size finds
  bool lowtie = false;
};
MD void slot_cells(int q, int& c0, int& c1) {
  const int r = q & 3;
  c0 = 7 * (q >> 2) + 2 * r - (q == 15 ? 1 : 0);
  c1 = c0 + ((r == 3 || q == 14) ? 1 : 2);
}
template <bool GRAD, int PPC = 0>
MD float4 slot_sums(const KParams& k, v3 p, int cx, int cy, int cz, uint32_t seed, int q) {
  int c0, c1;
  slot_cells(q, c0, c1);
  float4 x;
  psi_sums_cells<GRAD, PPC>(k, p, cx, cy, cz, seed, c0, c1, x.x, x.y, x.z, x.w);
  return x;
}
template <bool GRAD>
MD float4 add_s(float4 a, float4 b) {
  if (!GRAD) return make_float4(a.x + b.x, 0.0f, 0.0f, 0.0f);
  return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w);
}
// WIDE: the caller guarantees G >= 4 (V <= 4: the subtree is written out);
// otherwise a stack of partial sums walks the lane's V <= 16 slots.
template <bool GRAD, bool WIDE, int PPC = 0>
MD float4 psi_sums_group(const KParams& k, v3 p, uint32_t seed, const Group& g) {
  int cx, cy, cz;
  cell_of(k, p, cx, cy, cz);
  const int V = g.G >= 16 ? 1 : 16 / g.G;
  const int q0 = g.G >= 16 ? (g.sub & 15) : g.sub * V;
  float4 r;
  if (WIDE) {
    r = slot_sums<GRAD, PPC>(k, p, cx, cy, cz, seed, q0);
    if (V >= 2) r = add_s<GRAD>(r, slot_sums<GRAD, PPC>(k, p, cx, cy, cz, seed, q0 + 1));
    if (V >= 4) {
      const float4 a = slot_sums<GRAD, PPC>(k, p, cx, cy, cz, seed, q0 + 2);
      r = add_s<GRAD>(r, add_s<GRAD>(a, slot_sums<GRAD, PPC>(k, p, cx, cy, cz, seed, q0 + 3)));
    }
  } else {
    float4 st[5];
#pragma unroll 1
    for (int j = 0; j < V; ++j) {
      float4 x = slot_sums<GRAD, PPC>(k, p, cx, cy, cz, seed, q0 + j);
      bool carry = true;
#pragma unroll
      for (int l = 0; l < 5; ++l) {
        if (carry) {
          if (l < 4 && ((j >> l) & 1)) {
            x = add_s<GRAD>(st[l], x);
          } else {
            st[l] = x;
            carry = false;
          }
        }
      }
    }
    r = V == 1 ? st[0] : V == 2 ? st[1] : V == 4 ? st[2] : V == 8 ? st[3] : st[4];
  }
  const int top = min(g.G, 16);
  for (int off = 1; off < top; off <<= 1) {
    r.x += __shfl_xor_sync(g.mask, r.x, off, g.G);
    if (GRAD) {
      r.y += __shfl_xor_sync(g.mask, r.y, off, g.G);
      r.z += __shfl_xor_sync(g.mask, r.z, off, g.G);
      r.w += __shfl_xor_sync(g.mask, r.w, off, g.G);
    }
  }
  return r;
}
template <bool WIDE = false, int PPC = 0>
MD float raw_noise_value_group(const KParams& k, v3 p, uint32_t seed, const Group& g) {
  return (k.sigma * psi_sums_group<false, WIDE, PPC>(k, p, seed, g).x) / k.sqrt_var;
}
template <bool WIDE = false, int PPC = 0>
MD float4 raw_noise_group(const KParams& k, v3 p, uint32_t seed, const Group& g) {
  const float4 s = psi_sums_group<true, WIDE, PPC>(k, p, seed, g);
  return make_float4((k.sigma * s.x) / k.sqrt_var, (k.sigma * s.y) / k.sqrt_var, (k.sigma * s.z) / k.sqrt_var,
                     (k.sigma * s.w) / k.sqrt_var);
}

// RawNoise(p, seed) = sigma * InternalNoise / sqrt(Var) (gpnoise.h:44)
template <int PPC = 0>
MD float4 raw_noise(const KParams& k, v3 p, uint32_t seed) {
  float v, x, y, z;
  psi_sums<true, PPC>(k, p, seed, v, x, y, z);
  return make_float4((k.sigma * v) / k.sqrt_var, (k.sigma * x) / k.sqrt_var, (k.sigma * y) / k.sqrt_var,
                     (k.sigma * z) / k.sqrt_var);
}
template <int PPC = 0>
MD float raw_noise_value(const KParams& k, v3 p, uint32_t seed) {
  float v, x, y, z;
  psi_sums<false, PPC>(k, p, seed, v, x, y, z);
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
