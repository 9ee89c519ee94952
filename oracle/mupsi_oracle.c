/*
 * mupsi_oracle.c -- CPU restatement of the reference renderer's GPIS hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see mupsi_oracle.h). Compiled with
 * -ffp-contract=off so every float expression rounds exactly as written; the
 * expressions follow the reference's evaluation order (Eigen-style reductions
 * v0 + (v1 + v2), per-coefficient vector arithmetic, left-to-right scalar
 * products), which is what makes the integer outputs bit-exact and the float
 * outputs equal to the reference's parity build.
 */
#include "mupsi_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------ vectors -- */
typedef struct {
  float x, y, z;
} v3;
static inline v3 V3(float x, float y, float z) {
  v3 r = {x, y, z};
  return r;
}
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vneg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline v3 vmul(v3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
static inline v3 smul(float s, v3 a) { return V3(s * a.x, s * a.y, s * a.z); }
static inline v3 vdiv(v3 a, float s) { return V3(a.x / s, a.y / s, a.z / s); }
static inline v3 cmul(v3 a, v3 b) { return V3(a.x * b.x, a.y * b.y, a.z * b.z); }
/* Eigen reduction order for three coefficients: v0 + (v1 + v2) */
static inline float vdot(v3 a, v3 b) { return a.x * b.x + (a.y * b.y + a.z * b.z); }
static inline float vsqn(v3 a) { return vdot(a, a); }
static inline float vnorm(v3 a) { return sqrtf(vsqn(a)); }
static inline v3 vnormalized(v3 a) {
  float z = vsqn(a);
  return z > 0.0f ? vdiv(a, sqrtf(z)) : a;
}
static inline v3 vcross(v3 a, v3 b) {
  return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float fmin_std(float a, float b) { return (b < a) ? b : a; } /* std::min */
static inline float fmax_std(float a, float b) { return (a < b) ? b : a; } /* std::max */
static inline float vmaxc(v3 a) { return fmax_std(a.x, fmax_std(a.y, a.z)); }
static inline float vget(v3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
static inline v3 vload(const float* p) { return V3(p[0], p[1], p[2]); }
static inline void vstore(float* p, v3 a) {
  p[0] = a.x;
  p[1] = a.y;
  p[2] = a.z;
}

/* 4x4 matrices, column-major like Eigen; products reduce over k by halves. */
typedef struct {
  float m[16];
} m4;
static inline float M(const m4* a, int i, int j) { return a->m[j * 4 + i]; }
static m4 m4_identity(void) {
  m4 r;
  memset(&r, 0, sizeof r);
  for (int i = 0; i < 4; ++i) r.m[i * 4 + i] = 1.0f;
  return r;
}
/* Affine3f(Translation3f(t) * Scaling(s)).matrix() */
static m4 m4_translate_scale(v3 t, float s) {
  m4 r = m4_identity();
  r.m[0] = s;
  r.m[5] = s;
  r.m[10] = s;
  r.m[12] = t.x;
  r.m[13] = t.y;
  r.m[14] = t.z;
  return r;
}
static float det3f(const float a[9]) { /* row-major 3x3 */
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
}
/* cofactor inverse, same rounding sequence as the oracle's Eigen shim */
static m4 m4_inverse(const m4* a) {
  float cof[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      float sub[9];
      int ra = 0;
      for (int r = 0; r < 4; ++r) {
        if (r == i) continue;
        int cb = 0;
        for (int c = 0; c < 4; ++c) {
          if (c == j) continue;
          sub[ra * 3 + cb] = M(a, r, c);
          ++cb;
        }
        ++ra;
      }
      float minor = det3f(sub);
      cof[i][j] = ((i + j) % 2 == 0) ? minor : -minor;
    }
  float det = 0.0f;
  for (int j = 0; j < 4; ++j) det += M(a, 0, j) * cof[0][j];
  m4 r;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r.m[i * 4 + j] = cof[i][j] / det; /* r(j,i) */
  return r;
}
static int m4_is_identity(const m4* a) {
  for (int j = 0; j < 4; ++j)
    for (int i = 0; i < 4; ++i) {
      float v = M(a, i, j);
      if (i == j) {
        float lim = 1e-5f * fmin_std(fabsf(v), 1.0f);
        if (!(fabsf(v - 1.0f) <= lim)) return 0;
      } else if (!(fabsf(v) <= 1e-5f)) {
        return 0;
      }
    }
  return 1;
}
/* (M * (p, w)).head<3>(): each row reduced as (m0 x + m1 y) + (m2 z + m3 w) */
static v3 m4_apply(const m4* a, v3 p, float w) {
  float out[3];
  for (int i = 0; i < 3; ++i)
    out[i] = (M(a, i, 0) * p.x + M(a, i, 1) * p.y) + (M(a, i, 2) * p.z + M(a, i, 3) * w);
  return V3(out[0], out[1], out[2]);
}
/* topLeftCorner<3,3>() * v: m0 x + (m1 y + m2 z) */
static v3 m3_apply(const m4* a, v3 v) {
  float out[3];
  for (int i = 0; i < 3; ++i) out[i] = M(a, i, 0) * v.x + (M(a, i, 1) * v.y + M(a, i, 2) * v.z);
  return V3(out[0], out[1], out[2]);
}
/* topLeftCorner<3,3>().transpose() * v */
static v3 m3t_apply(const m4* a, v3 v) {
  float out[3];
  for (int i = 0; i < 3; ++i) out[i] = M(a, 0, i) * v.x + (M(a, 1, i) * v.y + M(a, 2, i) * v.z);
  return V3(out[0], out[1], out[2]);
}
static int m3_is_identity(const m4* a) {
  for (int j = 0; j < 3; ++j)
    for (int i = 0; i < 3; ++i) {
      float v = M(a, i, j);
      if (i == j) {
        float lim = 1e-5f * fmin_std(fabsf(v), 1.0f);
        if (!(fabsf(v - 1.0f) <= lim)) return 0;
      } else if (!(fabsf(v) <= 1e-5f)) {
        return 0;
      }
    }
  return 1;
}

/* ------------------------------------------------- math/random.h:13-119 -- */
static inline void hash_combine(uint32_t* seed, uint32_t v) { *seed ^= v + 0x9e3779b9u + (*seed << 6) + (*seed >> 2); }
uint32_t mo_make_seed4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  uint32_t h = 0;
  hash_combine(&h, a);
  hash_combine(&h, b);
  hash_combine(&h, c);
  hash_combine(&h, d);
  return h;
}
uint32_t mo_make_seed5(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t e) {
  uint32_t h = mo_make_seed4(a, b, c, d);
  hash_combine(&h, e);
  return h;
}

typedef struct {
  uint64_t state;
} pcg;
static inline uint32_t pcg_next(pcg* r) {
  uint64_t old = r->state;
  r->state = old * 6364136223846793005ULL + 1ULL;
  uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
  uint32_t rot = (uint32_t)(old >> 59u);
  return (xs >> rot) | (xs << ((uint32_t)(-(int32_t)rot) & 31u));
}
static inline float bits_to_float(uint32_t i) {
  float f;
  memcpy(&f, &i, 4);
  return f;
}
static inline float pcg_next1d(pcg* r) { return bits_to_float((pcg_next(r) >> 9u) | 0x3F800000u) - 1.0f; }
/* Random(seed): zero seed becomes 1, then two warm-up draws (random.h:77-80) */
static inline void pcg_init(pcg* r, uint64_t seed) {
  r->state = seed == 0 ? 1 : seed;
  pcg_next(r);
  pcg_next(r);
}

void mo_random_stream(uint64_t seed, int n, uint32_t* out_u32, float* out_f) {
  pcg a, b;
  pcg_init(&a, seed);
  pcg_init(&b, seed);
  for (int i = 0; i < n; ++i) {
    out_u32[i] = pcg_next(&a);
    out_f[i] = pcg_next1d(&b);
  }
}

typedef struct {
  float x, y;
  uint32_t i;
} csampler;
static csampler constant_sampler(uint32_t seed) { /* sampler.h:47-54 */
  pcg r;
  pcg_init(&r, seed);
  csampler c;
  c.x = pcg_next1d(&r);
  c.y = pcg_next1d(&r);
  c.i = pcg_next(&r);
  return c;
}
void mo_constant_sampler(uint32_t seed, float* x, float* y, uint32_t* i) {
  csampler c = constant_sampler(seed);
  *x = c.x;
  *y = c.y;
  *i = c.i;
}

/* --------------------------------------------------- gp/kernel.h, gpnoise -- */
typedef struct {
  float sigma, kr, L2, sqrt_var;
  int ppc;
} kparams;
static kparams kernel_params(const mupsi_kernel* k) {
  kparams p;
  p.sigma = k->sigma;
  p.kr = k->kernel_radius;
  p.L2 = vsqn(vload(k->aniso)); /* lengthScale_.squaredNorm() (kernel.h:53) */
  p.ppc = k->points_per_cell;
  /* Var() (gpnoise.h:31): int / pow(float,int) -> double, * pow(pi,1.5), returned as float */
  float var = (float)(((double)p.ppc / pow((double)p.kr, 3.0)) * pow(M_PI, 1.5));
  p.sqrt_var = sqrtf(var);
  return p;
}
/* h(s, p) = exp(-|p - s|^2 / L2) (kernel.h:52-54) */
static inline float kh(const kparams* k, v3 s, v3 p) { return expf(-vsqn(vsub(p, s)) / k->L2); }
/* h_grad(C, p) = h(C,p) * (-2/L2) * (p - C) (kernel.h:55-58) */
static inline v3 kh_grad(const kparams* k, v3 C, v3 p) { return smul(kh(k, C, p) * (-2.0f / k->L2), vsub(p, C)); }
/* H_h v = h * ((-2/L2) v + (4/L2^2)(r.v) r) (kernel.h:60-65) */
static inline v3 kh_hess_vec(const kparams* k, v3 C, v3 p, v3 v) {
  v3 r = vsub(p, C);
  float hv = kh(k, C, p);
  v3 a = smul(-2.0f / k->L2, v);
  v3 b = smul((4.0f / (k->L2 * k->L2)) * vdot(r, v), r);
  return smul(hv, vadd(a, b));
}

/* Impulses of one neighbour cell: the cell seed, the PCG stream started at
 * cell_seed + 1 (32-bit wrap, gpnoise.cpp:61-62), and per impulse three offset
 * draws and a sign draw (gpnoise.cpp:66-74). The offset is built as
 * Vector3f(next1D(), next1D(), next1D()); the reference's GCC build evaluates
 * those constructor arguments right to left, so the first draw is z. */
static inline v3 impulse_offset(pcg* r) {
  float a = pcg_next1d(r);
  float b = pcg_next1d(r);
  float c = pcg_next1d(r);
  return V3(c, b, a);
}

typedef struct {
  float v, gx, gy, gz;
} f4;

/* InternalNoise (gpnoise.cpp:51-87) */
static f4 internal_noise(const kparams* k, v3 p, uint32_t seed) {
  int cx = (int)(p.x / k->kr), cy = (int)(p.y / k->kr), cz = (int)(p.z / k->kr); /* cast<int>: truncation */
  f4 sum = {0, 0, 0, 0};
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz) {
        int nx = cx + dx, ny = cy + dy, nz = cz + dz;
        uint32_t cs = mo_make_seed4((uint32_t)nx, (uint32_t)ny, (uint32_t)nz, seed);
        pcg r;
        r.state = (uint64_t)(uint32_t)(cs + 1u);
        v3 ngbf = vmul(V3((float)nx, (float)ny, (float)nz), k->kr);
        for (int i = 0; i < k->ppc; ++i) {
          v3 off = impulse_offset(&r);
          v3 s = vadd(ngbf, vmul(off, k->kr));
          float w = pcg_next1d(&r) < 0.5f ? -1.0f : 1.0f;
          sum.v += w * kh(k, s, p);
          v3 g = kh_grad(k, s, p);
          sum.gx += w * g.x;
          sum.gy += w * g.y;
          sum.gz += w * g.z;
        }
      }
  return sum;
}
/* RawNoise = sigma * InternalNoise / sqrt(Var()) (gpnoise.h:44) */
static f4 raw_noise(const kparams* k, v3 p, uint32_t seed) {
  f4 s = internal_noise(k, p, seed);
  f4 r = {(k->sigma * s.v) / k->sqrt_var, (k->sigma * s.gx) / k->sqrt_var, (k->sigma * s.gy) / k->sqrt_var,
          (k->sigma * s.gz) / k->sqrt_var};
  return r;
}
/* The conditioning terms of evalWithGradient(p, seed, state) (gpmedium.cpp:32-39) */
static f4 add_cond(const kparams* k, f4 f, v3 p, const mupsi_cond* c) {
  if (!c || !c->active) return f;
  v3 C = vload(c->C), g = vload(c->g_tilde);
  v3 hg = kh_grad(k, C, p);
  f.v += c->u_tilde * kh(k, C, p) + vdot(g, hg);
  v3 Hg = kh_hess_vec(k, C, p, g);
  f.gx += c->u_tilde * hg.x + Hg.x;
  f.gy += c->u_tilde * hg.y + Hg.y;
  f.gz += c->u_tilde * hg.z + Hg.z;
  return f;
}

void mo_psi(const mupsi_kernel* kk, int64_t n, const float* p, const uint32_t* seed, const mupsi_cond* cond,
            float* out) {
  kparams k = kernel_params(kk);
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t i = 0; i < n; ++i) {
    v3 P = vload(p + 3 * i);
    f4 r = raw_noise(&k, P, seed[i]);
    r = add_cond(&k, r, P, cond ? cond + i : NULL);
    out[4 * i] = r.v;
    out[4 * i + 1] = r.gx;
    out[4 * i + 2] = r.gy;
    out[4 * i + 3] = r.gz;
  }
}

void mo_psi_f64(const mupsi_kernel* kk, int64_t n, const float* p, const uint32_t* seed, double* out,
                double* out_abs) {
  kparams k = kernel_params(kk);
  double L2 = (double)kk->aniso[0] * kk->aniso[0] + (double)kk->aniso[1] * kk->aniso[1] +
              (double)kk->aniso[2] * kk->aniso[2];
  double scale = (double)kk->sigma / sqrt(((double)k.ppc / pow((double)k.kr, 3.0)) * pow(M_PI, 1.5));
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t q = 0; q < n; ++q) {
    v3 P = vload(p + 3 * q);
    int cx = (int)(P.x / k.kr), cy = (int)(P.y / k.kr), cz = (int)(P.z / k.kr);
    double sv = 0, sg[3] = {0, 0, 0}, sa = 0, sga[3] = {0, 0, 0};
    for (int dx = -1; dx <= 1; ++dx)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dz = -1; dz <= 1; ++dz) {
          int nx = cx + dx, ny = cy + dy, nz = cz + dz;
          uint32_t cs = mo_make_seed4((uint32_t)nx, (uint32_t)ny, (uint32_t)nz, seed[q]);
          pcg r;
          r.state = (uint64_t)(uint32_t)(cs + 1u);
          v3 ngbf = vmul(V3((float)nx, (float)ny, (float)nz), k.kr);
          for (int i = 0; i < k.ppc; ++i) {
            v3 off = impulse_offset(&r);
            v3 s = vadd(ngbf, vmul(off, k.kr));
            double w = pcg_next1d(&r) < 0.5f ? -1.0 : 1.0;
            double d[3] = {(double)P.x - s.x, (double)P.y - s.y, (double)P.z - s.z};
            double h = exp(-(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) / L2);
            sv += w * h;
            sa += h;
            for (int c = 0; c < 3; ++c) {
              sg[c] += w * h * (-2.0 / L2) * d[c];
              sga[c] += fabs(h * (-2.0 / L2) * d[c]);
            }
          }
        }
    out[4 * q] = sv * scale;
    for (int c = 0; c < 3; ++c) out[4 * q + 1 + c] = sg[c] * scale;
    if (out_abs) {
      out_abs[4 * q] = sa * fabs(scale);
      for (int c = 0; c < 3; ++c) out_abs[4 * q + 1 + c] = sga[c] * fabs(scale);
    }
  }
}

void mo_psi_impulses(const mupsi_kernel* kk, const float* p, uint32_t seed, float* s_out, float* w_out,
                     int32_t* cells, uint32_t* cell_seed) {
  kparams k = kernel_params(kk);
  v3 P = vload(p);
  int cx = (int)(P.x / k.kr), cy = (int)(P.y / k.kr), cz = (int)(P.z / k.kr);
  int c = 0, m = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dz = -1; dz <= 1; ++dz, ++c) {
        int nx = cx + dx, ny = cy + dy, nz = cz + dz;
        uint32_t cs = mo_make_seed4((uint32_t)nx, (uint32_t)ny, (uint32_t)nz, seed);
        cells[3 * c] = nx;
        cells[3 * c + 1] = ny;
        cells[3 * c + 2] = nz;
        cell_seed[c] = cs;
        pcg r;
        r.state = (uint64_t)(uint32_t)(cs + 1u);
        v3 ngbf = vmul(V3((float)nx, (float)ny, (float)nz), k.kr);
        for (int i = 0; i < k.ppc; ++i, ++m) {
          v3 off = impulse_offset(&r);
          v3 s = vadd(ngbf, vmul(off, k.kr));
          s_out[3 * m] = s.x;
          s_out[3 * m + 1] = s.y;
          s_out[3 * m + 2] = s.z;
          w_out[m] = pcg_next1d(&r) < 0.5f ? -1.0f : 1.0f;
        }
      }
}

/* ----------------------------------------------------------- BVH build -- */
typedef struct {
  float mn[3], mx[3];
  uint32_t left, right;
} bnode;
#define LEAF_FLAG 0x80000000u

typedef struct {
  const v3* v;
  const int32_t* f;
  uint32_t* idx;
  bnode* nodes;
  int64_t count;
} bvh_builder;

static float tri_centroid(const bvh_builder* b, uint32_t ti, int axis) {
  const int32_t* f = b->f + 3 * ti;
  return (vget(b->v[f[0]], axis) + vget(b->v[f[1]], axis) + vget(b->v[f[2]], axis)) / 3.0f;
}
/* BVH::buildRecursive (bvh.cpp:132-193) */
static uint32_t build_rec(bvh_builder* b, uint32_t begin, uint32_t end) {
  uint32_t count = end - begin;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = begin; i < end; ++i) {
    const int32_t* f = b->f + 3 * b->idx[i];
    float tmn[3] = {INFINITY, INFINITY, INFINITY}, tmx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < 3; ++c) { /* AABB::extend per vertex (boudingbox.h:24-27) */
      v3 p = b->v[f[c]];
      for (int a = 0; a < 3; ++a) {
        tmn[a] = fmin_std(tmn[a], vget(p, a));
        tmx[a] = fmax_std(tmx[a], vget(p, a));
      }
    }
    for (int a = 0; a < 3; ++a) { /* box + triBounds: cwiseMin/Max (boudingbox.h:56-58) */
      mn[a] = fmin_std(mn[a], tmn[a]);
      mx[a] = fmax_std(mx[a], tmx[a]);
    }
  }
  if (count <= 4) {
    uint32_t id = (uint32_t)b->count++;
    bnode* nd = &b->nodes[id];
    memcpy(nd->mn, mn, sizeof mn);
    memcpy(nd->mx, mx, sizeof mx);
    nd->left = begin;
    nd->right = count | LEAF_FLAG;
    return id;
  }
  float d[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
  int axis = (d[0] > d[1] && d[0] > d[2]) ? 0 : (d[1] > d[2] ? 1 : 2); /* longestAxis (boudingbox.h:37-42) */
  float smin = INFINITY, smax = -INFINITY;
  for (uint32_t i = begin; i < end; ++i) {
    float c = tri_centroid(b, b->idx[i], axis);
    smin = fmin_std(smin, c);
    smax = fmax_std(smax, c);
  }
  float split = (smin + smax) * 0.5f;
  /* std::partition over a random-access range: the two-ended exchange scheme */
  uint32_t first = begin, last = end;
  for (;;) {
    for (;;) {
      if (first == last) goto partitioned;
      if (tri_centroid(b, b->idx[first], axis) < split)
        ++first;
      else
        break;
    }
    --last;
    for (;;) {
      if (first == last) goto partitioned;
      if (!(tri_centroid(b, b->idx[last], axis) < split))
        --last;
      else
        break;
    }
    uint32_t t = b->idx[first];
    b->idx[first] = b->idx[last];
    b->idx[last] = t;
    ++first;
  }
partitioned:;
  uint32_t mid = first;
  if (mid == begin || mid == end) mid = begin + count / 2;
  uint32_t l = build_rec(b, begin, mid);
  uint32_t r = build_rec(b, mid, end);
  uint32_t id = (uint32_t)b->count++;
  bnode* nd = &b->nodes[id];
  memcpy(nd->mn, mn, sizeof mn);
  memcpy(nd->mx, mx, sizeof mx);
  nd->left = l;
  nd->right = r;
  return id;
}

static int64_t bvh_build_into(int64_t nv, const v3* verts, int64_t nf, const int32_t* faces, bnode* nodes,
                              uint32_t* idx, uint32_t* root) {
  (void)nv;
  if (nf == 0) {
    *root = 0;
    return 0;
  }
  bvh_builder b = {verts, faces, idx, nodes, 0};
  for (int64_t i = 0; i < nf; ++i) idx[i] = (uint32_t)i;
  *root = build_rec(&b, 0, (uint32_t)nf);
  return b.count;
}

int64_t mo_bvh_build(int64_t nv, const float* verts, int64_t nf, const int32_t* faces, uint32_t* nodes_out,
                     uint32_t* tri_out, uint32_t* root) {
  return bvh_build_into(nv, (const v3*)verts, nf, faces, (bnode*)nodes_out, tri_out, root);
}

/* ------------------------------------------------------------- scenes -- */
typedef struct {
  int64_t nv, nf;
  v3* v;
  int32_t* f;
  v3* vn; /* nullable */
  v3* face_n;
  bnode* nodes;
  int64_t num_nodes;
  uint32_t* idx;
  uint32_t root;
  m4 T, Tinv;
  int identity;
  int normal_identity;
  float* cdf;
  float total_area;
} omesh;

typedef struct {
  mupsi_primitive_desc d;
  m4 T, Tinv;
  int identity;
  /* LambertianBsdf(BitmapTexture) albedo (bsdf.cpp:14-37, texture.cpp): RGB,
   * row 0 at the top; uvs [n*2] + face_uv [F*3] are the mesh's texcoords
   * (NULL: the hit's barycentrics are the uv, mesh.cpp:175-177) */
  float* tex;
  int tex_w, tex_h;
  float* uvs;
  int32_t* face_uv;
} oprim;

/* GridMeanFunction (meanfunction.h:45-55): res^3 samples, x-major */
typedef struct {
  float* data;
  int res;
  v3 bmin, inv;
} ogrid;

typedef struct {
  mupsi_medium_desc d;
  kparams k;
  int kind; /* mupsi_medium_kind */
  ogrid gmean, gvar; /* ExternalGPMedium grids (gvar.data NULL: no noise) */
  float noise_scale;
} omedium;

struct mo_scene {
  mupsi_scene_desc d;
  int nmesh, nprim, nmed;
  omesh* meshes;
  oprim* prims;
  omedium* media;
  int* lights;
  int nlights;
  /* camera (camera.h:13-19) */
  v3 cpos, cdir, cup, cright, ctrue_up;
  float fov, aspect;
  /* Skydrome(BitmapTexture) (skydrome.cpp, texture.cpp): RGB, row 0 at the top */
  float* sky_tex;
  int sky_w, sky_h;
  int skip_medium; /* PathTracerSettings::skip_medium (trace.h:22) */
};

/* Mesh::computeFaceNormals (mesh.cpp:140-154) */
static void mesh_face_normals(omesh* m) {
  for (int64_t i = 0; i < m->nf; ++i) {
    const int32_t* f = m->f + 3 * i;
    v3 e1 = vsub(m->v[f[1]], m->v[f[0]]);
    v3 e2 = vsub(m->v[f[2]], m->v[f[0]]);
    v3 n = vcross(e1, e2);
    float len = vnorm(n);
    m->face_n[i] = len > 1e-12f ? vdiv(n, len) : V3(0, 0, 0);
  }
}

mo_scene* mo_scene_create(const mupsi_scene_desc* d) {
  mo_scene* s = (mo_scene*)calloc(1, sizeof(mo_scene));
  s->d = *d;
  s->nmesh = d->num_meshes;
  s->nprim = d->num_primitives;
  s->nmed = d->num_media;
  s->meshes = (omesh*)calloc(s->nmesh > 0 ? s->nmesh : 1, sizeof(omesh));
  for (int i = 0; i < s->nmesh; ++i) {
    const mupsi_mesh_desc* md = &d->meshes[i];
    omesh* m = &s->meshes[i];
    m->nv = md->num_vertices;
    m->nf = md->num_faces;
    m->v = (v3*)malloc(sizeof(v3) * (m->nv ? m->nv : 1));
    memcpy(m->v, md->vertices, sizeof(v3) * m->nv);
    m->f = (int32_t*)malloc(sizeof(int32_t) * 3 * (m->nf ? m->nf : 1));
    memcpy(m->f, md->faces, sizeof(int32_t) * 3 * m->nf);
    if (md->vertex_normals) {
      m->vn = (v3*)malloc(sizeof(v3) * m->nv);
      memcpy(m->vn, md->vertex_normals, sizeof(v3) * m->nv);
    }
    m->face_n = (v3*)malloc(sizeof(v3) * (m->nf ? m->nf : 1));
    mesh_face_normals(m);
    m->nodes = (bnode*)malloc(sizeof(bnode) * (2 * m->nf + 1));
    m->idx = (uint32_t*)malloc(sizeof(uint32_t) * (m->nf ? m->nf : 1));
    m->num_nodes = bvh_build_into(m->nv, m->v, m->nf, m->f, m->nodes, m->idx, &m->root);
    m->T = m4_translate_scale(vload(md->position), md->scale);
    m->Tinv = m4_inverse(&m->T);
    m->identity = m4_is_identity(&m->Tinv);
    m->normal_identity = m3_is_identity(&m->Tinv); /* normalTransform_ = Tinv^T (mesh.h:27-30) */
    /* light-sampling CDF (mesh.cpp:308-318) */
    m->cdf = (float*)malloc(sizeof(float) * (m->nf ? m->nf : 1));
    float total = 0.0f;
    for (int64_t t = 0; t < m->nf; ++t) {
      const int32_t* f = m->f + 3 * t;
      v3 e1 = vsub(m->v[f[1]], m->v[f[0]]);
      v3 e2 = vsub(m->v[f[2]], m->v[f[0]]);
      total += 0.5f * vnorm(vcross(e1, e2));
      m->cdf[t] = total;
    }
    if (total > 0.0f)
      for (int64_t t = 0; t < m->nf; ++t) m->cdf[t] /= total;
    m->total_area = total;
  }
  s->prims = (oprim*)calloc(s->nprim > 0 ? s->nprim : 1, sizeof(oprim));
  s->lights = (int*)calloc(s->nprim > 0 ? s->nprim : 1, sizeof(int));
  for (int i = 0; i < s->nprim; ++i) {
    oprim* p = &s->prims[i];
    p->d = d->primitives[i];
    if (p->d.type == MUPSI_PRIM_SPHERE) {
      p->T = m4_translate_scale(vload(p->d.center), p->d.radius);
    } else {
      p->T = s->meshes[p->d.mesh].T;
    }
    p->Tinv = m4_inverse(&p->T);
    p->identity = m4_is_identity(&p->Tinv);
    if (p->d.has_emission) s->lights[s->nlights++] = i;
  }
  s->media = (omedium*)calloc(s->nmed > 0 ? s->nmed : 1, sizeof(omedium));
  for (int i = 0; i < s->nmed; ++i) {
    s->media[i].d = d->media[i];
    s->media[i].k = kernel_params(&d->media[i].kernel);
  }
  s->cpos = vload(d->cam_pos);
  s->cdir = vnormalized(vload(d->cam_dir));
  s->cup = vnormalized(vload(d->cam_up));
  s->fov = d->cam_fov;
  s->aspect = (float)d->width / (float)d->height;
  s->cright = vnormalized(vcross(s->cdir, s->cup));
  s->ctrue_up = vnormalized(vcross(s->cright, s->cdir));
  return s;
}

void mo_scene_free(mo_scene* s) {
  if (!s) return;
  for (int i = 0; i < s->nmesh; ++i) {
    omesh* m = &s->meshes[i];
    free(m->v);
    free(m->f);
    free(m->vn);
    free(m->face_n);
    free(m->nodes);
    free(m->idx);
    free(m->cdf);
  }
  free(s->meshes);
  for (int i = 0; i < s->nprim; ++i) {
    free(s->prims[i].tex);
    free(s->prims[i].uvs);
    free(s->prims[i].face_uv);
  }
  free(s->prims);
  free(s->lights);
  for (int i = 0; i < s->nmed; ++i) {
    free(s->media[i].gmean.data);
    free(s->media[i].gvar.data);
  }
  free(s->media);
  free(s->sky_tex);
  free(s);
}

void mo_scene_set_sky_texture(mo_scene* s, int w, int h, const float* rgb) {
  free(s->sky_tex);
  s->sky_tex = NULL;
  s->sky_w = s->sky_h = 0;
  if (w <= 0 || h <= 0 || !rgb) return;
  s->sky_tex = (float*)malloc(sizeof(float) * 3 * (size_t)w * h);
  memcpy(s->sky_tex, rgb, sizeof(float) * 3 * (size_t)w * h);
  s->sky_w = w;
  s->sky_h = h;
}

int mo_scene_set_albedo_texture(mo_scene* s, int prim, int64_t ntc, const float* tc, const int32_t* ftc, int w,
                                int h, const float* rgb) {
  if (prim < 0 || prim >= s->nprim) return -1;
  oprim* p = &s->prims[prim];
  if (p->d.type != MUPSI_PRIM_MESH || p->d.bsdf != MUPSI_BSDF_LAMBERTIAN) return -1;
  const int64_t nf = s->meshes[p->d.mesh].nf;
  if (w > 0 && ntc > 0)
    for (int64_t i = 0; i < 3 * nf; ++i)
      if (ftc[i] < 0 || ftc[i] >= ntc) return -1;
  free(p->tex);
  free(p->uvs);
  free(p->face_uv);
  p->tex = NULL;
  p->uvs = NULL;
  p->face_uv = NULL;
  p->tex_w = p->tex_h = 0;
  if (w <= 0 || h <= 0 || !rgb) return 0;
  p->tex = (float*)malloc(sizeof(float) * 3 * (size_t)w * h);
  memcpy(p->tex, rgb, sizeof(float) * 3 * (size_t)w * h);
  p->tex_w = w;
  p->tex_h = h;
  if (ntc > 0) {
    p->uvs = (float*)malloc(sizeof(float) * 2 * (size_t)ntc);
    memcpy(p->uvs, tc, sizeof(float) * 2 * (size_t)ntc);
    p->face_uv = (int32_t*)malloc(sizeof(int32_t) * 3 * (size_t)nf);
    memcpy(p->face_uv, ftc, sizeof(int32_t) * 3 * (size_t)nf);
  }
  return 0;
}

/* BitmapTexture::operator[] (texture.cpp:52-69): wrap to [0, 1), flip v (row
 * 0 is the top), nearest texel. */
static v3 tex_lookup(const float* tex, int w, int h, float u, float v) {
  u = u - floorf(u);
  v = v - floorf(v);
  v = 1.0f - v;
  int x = (int)(u * (float)w) % w;
  int y = (int)(v * (float)h) % h;
  if (x < 0) x += w;
  if (y < 0) y += h;
  const float* t = tex + 3 * ((size_t)y * w + x);
  return (v3){t[0], t[1], t[2]};
}

/* Skydrome::intersect (skydrome.cpp:8-17): equirectangular (u, v) of the
 * direction, then the texture lookup. */
static v3 sky_lookup(const mo_scene* s, v3 dir) {
  const double pi = 3.14159265358979323846;
  float u = (float)(((double)atan2f(dir.z, dir.x) + pi) / (2.0f * pi));
  float cy = -dir.y;
  cy = cy < -1.0f ? -1.0f : (cy > 1.0f ? 1.0f : cy);
  float v = (float)((double)acosf(cy) / pi);
  return tex_lookup(s->sky_tex, s->sky_w, s->sky_h, u, v);
}

/* --------------------------------------------------------- rays / BVH -- */
typedef struct {
  v3 o, d;
  float nt, ft;
} oray;
/* Ray(origin, direction): direction normalized (ray.h:12) */
static inline oray mkray(v3 o, v3 d) {
  oray r;
  r.o = o;
  r.d = vnormalized(d);
  r.nt = 0.0f;
  r.ft = FLT_MAX;
  return r;
}
static inline oray load_ray(const mupsi_ray* r) {
  oray q = mkray(vload(r->o), vload(r->d));
  q.nt = r->near_t;
  q.ft = r->far_t;
  return q;
}

/* AABB::intersect (boudingbox.cpp:6-38) */
static int aabb_hit(const bnode* b, const oray* r) {
  float tmin = -INFINITY, tmax = INFINITY;
  for (int a = 0; a < 3; ++a) {
    float d = vget(r->d, a), o = vget(r->o, a);
    if (fabsf(d) > 1e-8f) {
      float t1 = (b->mn[a] - o) / d;
      float t2 = (b->mx[a] - o) / d;
      tmin = fmax_std(tmin, fmin_std(t1, t2));
      tmax = fmin_std(tmax, fmax_std(t1, t2));
    } else if (o < b->mn[a] || o > b->mx[a]) {
      return 0;
    }
  }
  return tmax >= tmin && tmax >= r->nt && tmin <= r->ft;
}
/* BVH::rayTriIntersect, Moller-Trumbore (bvh.cpp:82-111) */
static int ray_tri(const oray* r, v3 v0, v3 v1, v3 v2, float* t, float* u, float* v) {
  v3 e1 = vsub(v1, v0), e2 = vsub(v2, v0);
  v3 h = vcross(r->d, e2);
  float a = vdot(e1, h);
  if (fabsf(a) < 1e-8f) return 0;
  float f = 1.0f / a;
  v3 s = vsub(r->o, v0);
  *u = f * vdot(s, h);
  if (*u < 0.0f || *u > 1.0f) return 0;
  v3 q = vcross(s, e1);
  *v = f * vdot(r->d, q);
  if (*v < 0.0f || *u + *v > 1.0f) return 0;
  *t = f * vdot(e2, q);
  return *t > r->nt && *t < r->ft;
}
static inline v3 node_centroid(const bnode* b) {
  return vmul(vadd(V3(b->mn[0], b->mn[1], b->mn[2]), V3(b->mx[0], b->mx[1], b->mx[2])), 0.5f);
}
static inline int node_axis(const bnode* b) {
  float d0 = b->mx[0] - b->mn[0], d1 = b->mx[1] - b->mn[1], d2 = b->mx[2] - b->mn[2];
  return (d0 > d1 && d0 > d2) ? 0 : (d1 > d2 ? 1 : 2);
}
#define OSTACK 256
/* BVH::intersect (bvh.cpp:197-250): narrows r->ft on hits */
static int bvh_intersect(const omesh* m, oray* r, uint32_t* tri, float* uu, float* vv, int64_t* visits) {
  if (m->num_nodes == 0) return 0;
  int hit = 0;
  uint32_t st[OSTACK];
  int sp = 0;
  st[sp++] = m->root;
  while (sp > 0) {
    const bnode* nd = &m->nodes[st[--sp]];
    if (visits) ++*visits;
    if (!aabb_hit(nd, r)) continue;
    if (nd->right & LEAF_FLAG) {
      uint32_t start = nd->left, cnt = nd->right & ~LEAF_FLAG;
      for (uint32_t i = start; i < start + cnt; ++i) {
        uint32_t ti = m->idx[i];
        const int32_t* f = m->f + 3 * ti;
        float t, u, v;
        if (ray_tri(r, m->v[f[0]], m->v[f[1]], m->v[f[2]], &t, &u, &v)) {
          r->ft = t;
          *tri = ti;
          *uu = u;
          *vv = v;
          hit = 1;
        }
      }
    } else {
      const bnode* ln = &m->nodes[nd->left];
      const bnode* rn = &m->nodes[nd->right];
      int axis = node_axis(nd);
      float lc = vget(node_centroid(ln), axis), rc = vget(node_centroid(rn), axis);
      int near_first = (vget(r->d, axis) > 0) ? (lc < rc) : (lc > rc);
      uint32_t first = near_first ? nd->left : nd->right;
      uint32_t second = near_first ? nd->right : nd->left;
      if (sp + 2 > OSTACK) return hit; /* the reference's fixed stack would overflow here */
      st[sp++] = second;
      st[sp++] = first;
    }
  }
  return hit;
}
/* BVH::occluded (bvh.cpp:254-300): the traversal starts at node 0 (bvh.cpp:259) */
static int bvh_occluded(const omesh* m, const oray* r) {
  if (m->num_nodes == 0) return 0;
  uint32_t st[OSTACK];
  int sp = 0;
  st[sp++] = 0;
  while (sp > 0) {
    const bnode* nd = &m->nodes[st[--sp]];
    if (!aabb_hit(nd, r)) continue;
    if (nd->right & LEAF_FLAG) {
      uint32_t start = nd->left, cnt = nd->right & ~LEAF_FLAG;
      for (uint32_t i = start; i < start + cnt; ++i) {
        const int32_t* f = m->f + 3 * m->idx[i];
        float t, u, v;
        if (ray_tri(r, m->v[f[0]], m->v[f[1]], m->v[f[2]], &t, &u, &v)) return 1;
      }
    } else {
      const bnode* ln = &m->nodes[nd->left];
      const bnode* rn = &m->nodes[nd->right];
      int axis = node_axis(nd);
      float lc = vget(node_centroid(ln), axis), rc = vget(node_centroid(rn), axis);
      int near_first = (vget(r->d, axis) > 0) ? (lc < rc) : (lc > rc);
      if (sp + 2 > OSTACK) return 0;
      st[sp++] = near_first ? nd->right : nd->left;
      st[sp++] = near_first ? nd->left : nd->right;
    }
  }
  return 0;
}
/* dist2ToAABB (bvh.cpp:20-25): std::max({a, 0, b}) */
static inline float max3_il(float a, float b, float c) {
  float m = a;
  if (m < b) m = b;
  if (m < c) m = c;
  return m;
}
static inline float dist2_aabb(v3 p, const bnode* b) {
  float dx = max3_il(b->mn[0] - p.x, 0.0f, p.x - b->mx[0]);
  float dy = max3_il(b->mn[1] - p.y, 0.0f, p.y - b->mx[1]);
  float dz = max3_il(b->mn[2] - p.z, 0.0f, p.z - b->mx[2]);
  return dx * dx + dy * dy + dz * dz;
}
/* dist2ToLine (bvh.cpp:27-40) */
static float dist2_line(v3 p, v3 a, v3 b, v3* out) {
  v3 ab = vsub(b, a), ap = vsub(p, a);
  if (vsqn(ab) < 1e-6f) {
    *out = a;
    return vsqn(ap);
  }
  float d = vdot(ap, ab);
  float t = d / vsqn(ab);
  t = t < 0.0f ? 0.0f : (1.0f < t ? 1.0f : t); /* std::clamp */
  v3 proj = vadd(a, smul(t, ab));
  *out = proj;
  return vsqn(vsub(p, proj));
}
/* dist2ToTriangle (bvh.cpp:42-80) */
static float dist2_tri(v3 p, const v3* v, const int32_t* f, v3* out) {
  v3 a = v[f[0]], b = v[f[1]], c = v[f[2]];
  v3 e1 = vsub(a, b), e2 = vsub(a, c);
  v3 n = vcross(e1, e2);
  if (vsqn(n) < 1e-6f) {
    *out = a;
    return vsqn(vsub(p, a));
  }
  n = vnormalized(n);
  float dp = vdot(vsub(p, a), n);
  v3 pj = vsub(p, smul(dp, n));
  v3 ab = vneg(e1), bc = vsub(c, b), ca = e2;
  v3 c1 = vcross(ab, vsub(pj, a));
  v3 c2 = vcross(bc, vsub(pj, b));
  v3 c3 = vcross(ca, vsub(pj, c));
  if (vdot(c1, n) >= 0 && vdot(c2, n) >= 0 && vdot(c3, n) >= 0) {
    *out = pj;
    return dp * dp;
  }
  float mn = INFINITY, d;
  v3 tmp;
  if ((d = dist2_line(p, a, b, &tmp)) < mn) {
    mn = d;
    *out = tmp;
  }
  if ((d = dist2_line(p, b, c, &tmp)) < mn) {
    mn = d;
    *out = tmp;
  }
  if ((d = dist2_line(p, c, a, &tmp)) < mn) {
    mn = d;
    *out = tmp;
  }
  return mn;
}
/* BVH::closest (bvh.cpp:302-353) */
static float bvh_closest(const omesh* m, v3 p, uint32_t* tri, v3* q) {
  if (m->num_nodes == 0) return 0.0f;
  uint32_t st[OSTACK];
  int sp = 0;
  st[sp++] = m->root;
  float best = FLT_MAX;
  while (sp > 0) {
    const bnode* nd = &m->nodes[st[--sp]];
    if (dist2_aabb(p, nd) >= best) continue;
    if (nd->right & LEAF_FLAG) {
      uint32_t start = nd->left, cnt = nd->right & ~LEAF_FLAG;
      for (uint32_t i = start; i < start + cnt; ++i) {
        uint32_t ti = m->idx[i];
        v3 tmp;
        float d = dist2_tri(p, m->v, m->f + 3 * ti, &tmp);
        if (d < best) {
          best = d;
          *tri = ti;
          *q = tmp;
        }
      }
    } else {
      float dl = dist2_aabb(p, &m->nodes[nd->left]);
      float dr = dist2_aabb(p, &m->nodes[nd->right]);
      if (sp + 2 > OSTACK) break;
      if (dl < dr) {
        if (dr < best) st[sp++] = nd->right;
        if (dl < best) st[sp++] = nd->left;
      } else {
        if (dl < best) st[sp++] = nd->left;
        if (dr < best) st[sp++] = nd->right;
      }
    }
  }
  return sqrtf(best);
}
/* Mesh::inside (mesh.cpp:341-362): parity of +x crossings */
static int mesh_inside(const omesh* m, v3 p) {
  v3 pl = m4_apply(&m->Tinv, p, 1.0f);
  oray r = mkray(pl, V3(1.0f, 0.0f, 0.0f));
  uint32_t tri;
  float u, v;
  int hits = 0;
  if (bvh_intersect(m, &r, &tri, &u, &v, NULL)) {
    ++hits;
    while (r.ft < INFINITY) {
      r.nt = r.ft + 1e-4f;
      r.ft = INFINITY;
      if (!bvh_intersect(m, &r, &tri, &u, &v, NULL)) break;
      ++hits;
    }
  }
  return (hits % 2) == 1;
}
/* Mesh::distToPoint (mesh.cpp:325-339) */
static float mesh_dist(const omesh* m, v3 p, uint32_t* tri, v3* q) {
  v3 pl = m4_apply(&m->Tinv, p, 1.0f);
  v3 ql = V3(0, 0, 0);
  bvh_closest(m, pl, tri, &ql);
  *q = m4_apply(&m->T, ql, 1.0f);
  return vnorm(vsub(*q, p));
}

void mo_bvh_intersect(const mo_scene* s, int mesh, int64_t n, const mupsi_ray* rays, uint32_t* out_tri,
                      float* out_tuv) {
  const omesh* m = &s->meshes[mesh];
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    oray r = load_ray(&rays[i]);
    uint32_t tri = 0;
    float u = 0, v = 0;
    int h = bvh_intersect(m, &r, &tri, &u, &v, NULL);
    out_tri[i] = h ? tri : 0xFFFFFFFFu;
    out_tuv[3 * i] = h ? r.ft : -1.0f;
    out_tuv[3 * i + 1] = h ? u : 0.0f;
    out_tuv[3 * i + 2] = h ? v : 0.0f;
  }
}
void mo_bvh_occluded(const mo_scene* s, int mesh, int64_t n, const mupsi_ray* rays, uint8_t* out) {
  const omesh* m = &s->meshes[mesh];
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    oray r = load_ray(&rays[i]);
    out[i] = (uint8_t)bvh_occluded(m, &r);
  }
}
void mo_bvh_closest(const mo_scene* s, int mesh, int64_t n, const float* p, uint32_t* out_tri, float* out_dq) {
  const omesh* m = &s->meshes[mesh];
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    uint32_t tri = 0xFFFFFFFFu;
    v3 q = V3(0, 0, 0);
    float d = bvh_closest(m, vload(p + 3 * i), &tri, &q);
    out_tri[i] = tri;
    out_dq[4 * i] = d;
    out_dq[4 * i + 1] = q.x;
    out_dq[4 * i + 2] = q.y;
    out_dq[4 * i + 3] = q.z;
  }
}
void mo_mesh_queries(const mo_scene* s, int mesh, int64_t n, const float* p, uint8_t* out_inside, uint32_t* out_tri,
                     float* out_dq) {
  const omesh* m = &s->meshes[mesh];
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    v3 P = vload(p + 3 * i);
    out_inside[i] = (uint8_t)mesh_inside(m, P);
    uint32_t tri = 0xFFFFFFFFu;
    v3 q = V3(0, 0, 0);
    out_dq[4 * i] = mesh_dist(m, P, &tri, &q);
    out_tri[i] = tri;
    out_dq[4 * i + 1] = q.x;
    out_dq[4 * i + 2] = q.y;
    out_dq[4 * i + 3] = q.z;
  }
}

/* ------------------------------------------------------ mean functions -- */
/* SphereMeanFunction / MeshMeanFunction (meanfunction.cpp:13-39) */
static float mean_eval(const mo_scene* s, const omedium* md, v3 p) {
  if (md->d.mean_type == MUPSI_MEAN_SPHERE) return vnorm(vsub(p, vload(md->d.mean_center))) - md->d.mean_radius;
  const omesh* m = &s->meshes[md->d.mean_mesh];
  float inside = mesh_inside(m, p) ? -1.0f : 1.0f;
  uint32_t tri;
  v3 q;
  return inside * mesh_dist(m, p, &tri, &q);
}
static v3 mean_grad(const mo_scene* s, const omedium* md, v3 p) {
  if (md->d.mean_type == MUPSI_MEAN_SPHERE) return vnormalized(vsub(p, vload(md->d.mean_center)));
  const omesh* m = &s->meshes[md->d.mean_mesh];
  float inside = mesh_inside(m, p) ? -1.0f : 1.0f;
  uint32_t tri = 0;
  v3 q;
  float d = mesh_dist(m, p, &tri, &q);
  if (d < 1e-6f) {
    v3 n = m->face_n[tri];
    if (!m->normal_identity) n = vnormalized(m3t_apply(&m->Tinv, n));
    return n;
  }
  return vnormalized(smul(inside, vsub(p, q)));
}

/* GPMedium::evalWithGradient (gpmedium.cpp:19-41) */
static f4 medium_eval(const mo_scene* s, const omedium* md, v3 p, uint32_t seed, const mupsi_cond* c) {
  float mean = mean_eval(s, md, p);
  v3 mg = mean_grad(s, md, p);
  f4 nz = raw_noise(&md->k, p, seed);
  f4 f = {mean + nz.v, mg.x + nz.gx, mg.y + nz.gy, mg.z + nz.gz};
  return add_cond(&md->k, f, p, c);
}

/* ------------------------------------------- field media evaluation -- */
static float clamp_std(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }
static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a < b ? b : a; }
/* (int)f as x86's cvttss2si: out of range / NaN -> INT_MIN (C leaves it undefined) */
static int f2i(float f) { return (f >= -2147483648.0f && f < 2147483648.0f) ? (int)f : INT32_MIN; }

/* GridMeanFunction::eval (meanfunction.cpp:58-78) */
static float grid_eval(const ogrid* g, v3 p) {
  float fx = (p.x - g->bmin.x) * g->inv.x - 0.5f;
  float fy = (p.y - g->bmin.y) * g->inv.y - 0.5f;
  float fz = (p.z - g->bmin.z) * g->inv.z - 0.5f;
  int i0 = imax(0, imin(g->res - 2, f2i(floorf(fx))));
  int j0 = imax(0, imin(g->res - 2, f2i(floorf(fy))));
  int k0 = imax(0, imin(g->res - 2, f2i(floorf(fz))));
  int i1 = i0 + 1, j1 = j0 + 1, k1 = k0 + 1;
  float wx = clamp_std(fx - (float)i0, 0.0f, 1.0f);
  float wy = clamp_std(fy - (float)j0, 0.0f, 1.0f);
  float wz = clamp_std(fz - (float)k0, 0.0f, 1.0f);
  size_t sy = (size_t)g->res, sx = (size_t)g->res * g->res;
#define AT(i, j, k) g->data[(size_t)(i) * sx + (size_t)(j) * sy + (size_t)(k)]
  float c00 = AT(i0, j0, k0) * (1 - wx) + AT(i1, j0, k0) * wx;
  float c01 = AT(i0, j0, k1) * (1 - wx) + AT(i1, j0, k1) * wx;
  float c10 = AT(i0, j1, k0) * (1 - wx) + AT(i1, j1, k0) * wx;
  float c11 = AT(i0, j1, k1) * (1 - wx) + AT(i1, j1, k1) * wx;
#undef AT
  float c0 = c00 * (1 - wy) + c10 * wy;
  float c1 = c01 * (1 - wy) + c11 * wy;
  return c0 * (1 - wz) + c1 * wz;
}
/* GridMeanFunction::gradient (meanfunction.cpp:80-86) */
static v3 grid_gradient(const ogrid* g, v3 p) {
  float eps = 1e-4f;
  float dx = grid_eval(g, V3(p.x + eps, p.y, p.z)) - grid_eval(g, V3(p.x - eps, p.y, p.z));
  float dy = grid_eval(g, V3(p.x, p.y + eps, p.z)) - grid_eval(g, V3(p.x, p.y - eps, p.z));
  float dz = grid_eval(g, V3(p.x, p.y, p.z + eps)) - grid_eval(g, V3(p.x, p.y, p.z - eps));
  return vdiv(V3(dx, dy, dz), 2.0f * eps);
}
/* hash11 (externalgpmedium.cpp:9-18) */
static float hash11(v3 p, uint32_t seed) {
  uint32_t h = seed, b;
  memcpy(&b, &p.x, 4);
  h = h * 0x9e3779b1u + b;
  memcpy(&b, &p.y, 4);
  h = h * 0x9e3779b1u + b;
  memcpy(&b, &p.z, 4);
  h = h * 0x9e3779b1u + b;
  h = (h ^ (h >> 16)) * 0x85ebca6bu;
  h = (h ^ (h >> 13)) * 0xc2b2ae35u;
  h = h ^ (h >> 16);
  return (float)(h & 0xFFFFFFu) / (float)0xFFFFFFu * 2.0f - 1.0f;
}
/* ExternalGPMedium::evalWithGradient(p, seed) (externalgpmedium.cpp:33-58) */
static f4 ext_eval(const omedium* md, v3 p, uint32_t seed) {
  float mu = grid_eval(&md->gmean, p);
  v3 mg = grid_gradient(&md->gmean, p);
  float noise = 0.0f;
  v3 ng = V3(0.0f, 0.0f, 0.0f);
  if (md->gvar.data && md->noise_scale > 0.0f) {
    float var = grid_eval(&md->gvar, p);
    if (var > 0.0f) {
      float amp = md->noise_scale * sqrtf(var);
      noise = amp * hash11(p, seed);
      float eps = 0.01f;
      ng.x = amp * (hash11(V3(p.x + eps, p.y, p.z), seed) - hash11(V3(p.x - eps, p.y, p.z), seed)) / (2.0f * eps);
      ng.y = amp * (hash11(V3(p.x, p.y + eps, p.z), seed) - hash11(V3(p.x, p.y - eps, p.z), seed)) / (2.0f * eps);
      ng.z = amp * (hash11(V3(p.x, p.y, p.z + eps), seed) - hash11(V3(p.x, p.y, p.z - eps), seed)) / (2.0f * eps);
    }
  }
  f4 f = {mu + noise, mg.x + ng.x, mg.y + ng.y, mg.z + ng.z};
  return f;
}
/* SDFMedium::evalWithGradient (sdfmedium.cpp:10-14) / ExternalGPMedium */
static f4 field_eval(const mo_scene* s, const omedium* md, v3 p, uint32_t seed) {
  if (md->kind == MUPSI_MEDIUM_SDF) {
    v3 g = mean_grad(s, md, p);
    f4 f = {mean_eval(s, md, p), g.x, g.y, g.z};
    return f;
  }
  return ext_eval(md, p, seed);
}
static float field_value(const mo_scene* s, const omedium* md, v3 p, uint32_t seed) {
  return md->kind == MUPSI_MEDIUM_SDF ? mean_eval(s, md, p) : ext_eval(md, p, seed).v;
}
void mo_mean(const mo_scene* s, int medium, int64_t n, const float* p, float* out) {
  const omedium* md = &s->media[medium];
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    v3 P = vload(p + 3 * i);
    int grid = md->kind == MUPSI_MEDIUM_EXTERNAL_GP;
    out[4 * i] = grid ? grid_eval(&md->gmean, P) : mean_eval(s, md, P);
    v3 g = grid ? grid_gradient(&md->gmean, P) : mean_grad(s, md, P);
    out[4 * i + 1] = g.x;
    out[4 * i + 2] = g.y;
    out[4 * i + 3] = g.z;
  }
}
void mo_medium_eval(const mo_scene* s, int medium, int64_t n, const float* p, const uint32_t* seed,
                    const mupsi_cond* cond, float* out) {
  const omedium* md = &s->media[medium];
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    f4 f = md->kind == MUPSI_MEDIUM_GP ? medium_eval(s, md, vload(p + 3 * i), seed[i], cond ? cond + i : NULL)
                                       : field_eval(s, md, vload(p + 3 * i), seed[i]);
    out[4 * i] = f.v;
    out[4 * i + 1] = f.gx;
    out[4 * i + 2] = f.gy;
    out[4 * i + 3] = f.gz;
  }
}

/* GPMedium::sampleDistance (gpmedium.cpp:46-103). The refinement loop at
 * gpmedium.cpp:67-73 computes a t_test that is never used; it is omitted. */
static void sample_distance(const mo_scene* s, const omedium* md, const oray* r, uint32_t seed, const mupsi_cond* c,
                            mupsi_medium_sample* out, int64_t* work) {
  float nt = r->nt, ft = r->ft;
  ft = fmin_std(ft, 2000.0f);
  float dt = fmin_std(0.5f, (ft - nt) / 100.0f);
  float t = nt;
  float f_prev = medium_eval(s, md, r->o, seed, c).v;
  if (work) work[1]++;
  while (t < ft) {
    v3 p = vadd(r->o, vmul(r->d, t));
    float fc = medium_eval(s, md, p, seed, c).v;
    if (work) {
      work[0]++;
      work[1]++;
    }
    if ((fc > 0.0f) != (f_prev > 0.0f) && (double)fabsf(f_prev - fc) > 1e-6) {
      out->exited = 0;
      out->t = t;
      v3 hp = vadd(r->o, vmul(r->d, t));
      f4 f = medium_eval(s, md, hp, seed, c);
      v3 nrm = vnormalized(V3(f.gx, f.gy, f.gz));
      out->p[0] = hp.x;
      out->p[1] = hp.y;
      out->p[2] = hp.z;
      out->normal[0] = nrm.x;
      out->normal[1] = nrm.y;
      out->normal[2] = nrm.z;
      return;
    }
    t += dt;
  }
  out->exited = 1;
}
/* GPMedium::transmittance (gpmedium.cpp:105-129) */
static float transmittance(const mo_scene* s, const omedium* md, const oray* r, uint32_t seed, const mupsi_cond* c) {
  float nt = r->nt, ft = r->ft;
  ft = fmin_std(ft, 2000.0f);
  float dt = fmin_std(0.5f, (ft - nt) / 100.0f);
  float t = nt;
  float f_prev = medium_eval(s, md, r->o, seed, c).v;
  while (t < ft) {
    v3 p = vadd(r->o, vmul(r->d, t));
    float fc = medium_eval(s, md, p, seed, c).v;
    if ((fc > 0.0f) != (f_prev > 0.0f) && (double)fabsf(f_prev - fc) > 1e-6) return 0.0f;
    t += dt;
  }
  return 1.0f;
}
/* GPMedium::sampleCondition (gpmedium.cpp:133-161) */
static void sample_condition(const mo_scene* s, const omedium* md, const mupsi_medium_sample* smp, uint32_t seed,
                             int renewal_plus, mupsi_cond* out) {
  out->active = 0;
  if (renewal_plus && !smp->exited) {
    v3 P = vload(smp->p);
    out->active = 1;
    out->C[0] = P.x;
    out->C[1] = P.y;
    out->C[2] = P.z;
    f4 psi = raw_noise(&md->k, P, seed);
    out->u_tilde = -mean_eval(s, md, P) / md->k.sigma - psi.v;
    float c2 = -md->k.L2 / 2.0f; /* oneOverSecondDerivative (kernel.h:66-68) */
    v3 g = smul(c2, vsub(vsub(vload(smp->normal), mean_grad(s, md, P)), V3(psi.gx, psi.gy, psi.gz)));
    out->g_tilde[0] = g.x;
    out->g_tilde[1] = g.y;
    out->g_tilde[2] = g.z;
  }
}

/* ------------------------------------------------------- field media -- */
void mo_scene_set_skip_medium(mo_scene* s, int skip) { s->skip_medium = skip != 0; }
int mo_scene_set_sdf_medium(mo_scene* s, int medium) {
  if (medium < 0 || medium >= s->nmed) return -1;
  s->media[medium].kind = MUPSI_MEDIUM_SDF;
  return 0;
}
int mo_scene_set_external_gp_medium(mo_scene* s, int medium, int res, const float* bmin, const float* bmax,
                                    const float* mean, const float* var, float noise_scale) {
  if (medium < 0 || medium >= s->nmed || res < 2 || !mean) return -1;
  omedium* md = &s->media[medium];
  size_t cells = (size_t)res * res * res;
  free(md->gmean.data);
  free(md->gvar.data);
  md->gmean.data = (float*)malloc(cells * sizeof(float));
  memcpy(md->gmean.data, mean, cells * sizeof(float));
  md->gvar.data = NULL;
  if (var) {
    md->gvar.data = (float*)malloc(cells * sizeof(float));
    memcpy(md->gvar.data, var, cells * sizeof(float));
  }
  /* inv_cell_size_ = Vector3f(res, res, res).cwiseQuotient(bmax - bmin) (meanfunction.cpp:44) */
  v3 lo = vload(bmin), hi = vload(bmax);
  v3 inv = V3((float)res / (hi.x - lo.x), (float)res / (hi.y - lo.y), (float)res / (hi.z - lo.z));
  md->gmean.res = md->gvar.res = res;
  md->gmean.bmin = md->gvar.bmin = lo;
  md->gmean.inv = md->gvar.inv = inv;
  md->noise_scale = noise_scale;
  md->kind = MUPSI_MEDIUM_EXTERNAL_GP;
  return 0;
}

static float max_std(float a, float b) { return (a < b) ? b : a; }

/* SDFMedium::sampleDistance (sdfmedium.cpp:16-63) */
static void sdf_sample_distance(const mo_scene* s, const omedium* md, const oray* r, mupsi_medium_sample* out) {
  float nt = r->nt, ft = fmin_std(r->ft, 2000.0f);
  const float minStep = 1e-3f;
  const int maxIter = 512;
  float t = nt;
  float f_c = field_value(s, md, r->o, 0);
  int iter = 0;
  while (t < ft && iter < maxIter) {
    v3 p = vadd(r->o, vmul(r->d, t));
    float f_prev = f_c, t_prev = t;
    f_c = field_value(s, md, p, 0);
    if (f_prev * f_c < 0.0f) {
      float lo = t_prev, hi = t, f_lo = f_prev;
      for (int b = 0; b < 16; b++) {
        float mid = (lo + hi) * 0.5f;
        float f_mid = field_value(s, md, vadd(r->o, vmul(r->d, mid)), 0);
        if (f_lo * f_mid <= 0.0f) {
          hi = mid;
        } else {
          lo = mid;
          f_lo = f_mid;
        }
      }
      v3 hp = vadd(r->o, vmul(r->d, hi));
      f4 f = field_eval(s, md, hp, 0);
      v3 n = vnormalized(V3(f.gx, f.gy, f.gz));
      out->exited = 0;
      out->t = hi;
      vstore(out->p, hp);
      vstore(out->normal, n);
      return;
    }
    float step = max_std(fabsf(f_c), minStep);
    t += step;
    iter++;
  }
  out->exited = 1;
}
/* ExternalGPMedium::sampleDistance (externalgpmedium.cpp:69-109) */
static void ext_sample_distance(const omedium* md, const oray* r, uint32_t seed, mupsi_medium_sample* out) {
  float nt = r->nt, ft = fmin_std(r->ft, 2000.0f);
  const float min_step = 0.005f;
  const int max_iter = 1024;
  float t = nt;
  float f_prev = ext_eval(md, r->o, seed).v;
  for (int iter = 0; iter < max_iter && t < ft; ++iter) {
    v3 p = vadd(r->o, vmul(r->d, t));
    float f_c = ext_eval(md, p, seed).v;
    if ((f_c > 0.0f) != (f_prev > 0.0f) && fabsf(f_prev - f_c) > 1e-6f) {
      float lo = t - max_std(fabsf(f_prev), min_step);
      float hi = t;
      for (int b = 0; b < 16; ++b) {
        float mid = (lo + hi) * 0.5f;
        float f_mid = ext_eval(md, vadd(r->o, vmul(r->d, mid)), seed).v;
        if ((f_mid > 0.0f) == (f_prev > 0.0f))
          lo = mid;
        else
          hi = mid;
      }
      v3 hp = vadd(r->o, vmul(r->d, hi));
      f4 f = ext_eval(md, hp, seed);
      v3 n = vnormalized(V3(f.gx, f.gy, f.gz));
      out->exited = 0;
      out->t = hi;
      vstore(out->p, hp);
      vstore(out->normal, n);
      return;
    }
    float step = max_std(fabsf(f_c), min_step);
    f_prev = f_c;
    t += step;
  }
  out->exited = 1;
}
/* SDFMedium::transmittance (sdfmedium.cpp:65-96) / ExternalGPMedium::transmittance
 * (externalgpmedium.cpp:111-130) */
static float field_transmittance(const mo_scene* s, const omedium* md, const oray* r, uint32_t seed) {
  float nt = r->nt, ft = fmin_std(r->ft, 2000.0f);
  float t = nt;
  if (md->kind == MUPSI_MEDIUM_SDF) {
    float f_c = field_value(s, md, r->o, 0);
    for (int iter = 0; t < ft && iter < 512; iter++) {
      v3 p = vadd(r->o, vmul(r->d, t));
      float f_prev = f_c;
      f_c = field_value(s, md, p, 0);
      if (f_prev * f_c < 0.0f) return 0.0f;
      t += max_std(fabsf(f_c), 1e-3f);
    }
    return 1.0f;
  }
  float f_prev = ext_eval(md, r->o, seed).v;
  for (int iter = 0; iter < 1024 && t < ft; ++iter) {
    v3 p = vadd(r->o, vmul(r->d, t));
    float f_c = ext_eval(md, p, seed).v;
    if ((f_c > 0.0f) != (f_prev > 0.0f) && fabsf(f_prev - f_c) > 1e-6f) return 0.0f;
    f_prev = f_c;
    t += max_std(fabsf(f_c), 0.005f);
  }
  return 1.0f;
}
/* Medium::sampleDistance / transmittance by medium kind */
static void any_sample_distance(const mo_scene* s, const omedium* md, const oray* r, uint32_t seed,
                                const mupsi_cond* c, mupsi_medium_sample* out, int64_t* work) {
  if (md->kind == MUPSI_MEDIUM_SDF)
    sdf_sample_distance(s, md, r, out);
  else if (md->kind == MUPSI_MEDIUM_EXTERNAL_GP)
    ext_sample_distance(md, r, seed, out);
  else
    sample_distance(s, md, r, seed, c, out, work);
}
static float any_transmittance(const mo_scene* s, const omedium* md, const oray* r, uint32_t seed,
                               const mupsi_cond* c) {
  return md->kind == MUPSI_MEDIUM_GP ? transmittance(s, md, r, seed, c) : field_transmittance(s, md, r, seed);
}

void mo_sample_distance(const mo_scene* s, int medium, int64_t n, const mupsi_ray* rays, const uint32_t* seed,
                        const mupsi_cond* cond, mupsi_medium_sample* out) {
  const omedium* md = &s->media[medium];
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < n; ++i) {
    oray r = load_ray(&rays[i]);
    memset(&out[i], 0, sizeof out[i]);
    any_sample_distance(s, md, &r, seed[i], cond ? cond + i : NULL, &out[i], NULL);
  }
}
void mo_transmittance(const mo_scene* s, int medium, int64_t n, const mupsi_ray* rays, const uint32_t* seed,
                      const mupsi_cond* cond, float* out) {
  const omedium* md = &s->media[medium];
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < n; ++i) {
    oray r = load_ray(&rays[i]);
    out[i] = any_transmittance(s, md, &r, seed[i], cond ? cond + i : NULL);
  }
}
void mo_sample_condition(const mo_scene* s, int medium, int64_t n, const mupsi_medium_sample* samples,
                         const uint32_t* seed, mupsi_cond* out) {
  const omedium* md = &s->media[medium];
  int rp = s->d.gp_mode == MUPSI_GP_RENEWAL_PLUS;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    memset(&out[i], 0, sizeof out[i]);
    sample_condition(s, md, &samples[i], seed[i], rp, &out[i]);
  }
}

/* ------------------------------------------------------- path tracing -- */
/* Camera::generateRay (camera.cpp:5-20) */
static oray camera_ray(const mo_scene* s, int x, int y) {
  float cx = ((float)x + 0.5f) / (float)s->d.width;
  float cy = ((float)y + 0.5f) / (float)s->d.height;
  float tf = tanf(s->fov / 2.0f);
  float nx = (2.0f * cx - 1.0f) * s->aspect * tf;
  float ny = (2.0f * cy - 1.0f) * tf;
  v3 dc = vnormalized(V3(nx, ny, 1.0f));
  v3 w = vnormalized(vadd(vadd(vmul(s->cright, dc.x), vmul(s->ctrue_up, dc.y)), vmul(s->cdir, dc.z)));
  return mkray(s->cpos, vnormalized(w));
}

/* TangentFrame(n) (sample.h:21-32) */
typedef struct {
  v3 n, t, b;
} frame;
static frame make_frame(v3 nn) {
  frame f;
  f.n = vnormalized(nn);
  float sign = copysignf(1.0f, f.n.z);
  float a = -1.0f / (sign + f.n.z);
  float b = f.n.x * f.n.y * a;
  f.t = vnormalized(V3(1.0f + sign * f.n.x * f.n.x * a, sign * b, -sign * f.n.x));
  f.b = vnormalized(V3(b, sign + f.n.y * f.n.y * a, -f.n.y));
  return f;
}
static v3 to_global(const frame* f, v3 p) { return vadd(vadd(vmul(f->t, p.x), vmul(f->b, p.y)), vmul(f->n, p.z)); }

typedef struct {
  int prim; /* -1 none */
  float t;
  v3 p, Ng;
  float tu, tv; /* texture coordinate (primitives with an albedo texture) */
} hitinfo;

/* intersectUnitSphere (sphere.cpp:11-30) */
static float unit_sphere(float nt, float ft, v3 O, v3 D) {
  float a = vsqn(D), b = vdot(O, D), c = vsqn(O) - 1.0f;
  float disc = b * b - a * c;
  if (disc < 0.0f) return -1.0f;
  float sq = sqrtf(disc);
  float t = (-b - sq) / a;
  if (t > nt && t < ft) return t;
  t = (-b + sq) / a;
  if (t > nt && t < ft) return t;
  return -1.0f;
}
/* mesh local-space ray (mesh.cpp:185-209) */
static int mesh_prim_intersect(const omesh* m, const oprim* p, oray* r, uint32_t* tri, float* u, float* v) {
  oray lr = *r;
  float tcorr = 1.0f;
  if (!p->identity) {
    v3 lo = m4_apply(&p->Tinv, r->o, 1.0f);
    v3 ld = m3_apply(&p->Tinv, r->d);
    float len = vnorm(ld);
    tcorr = vnorm(m3_apply(&p->T, vdiv(ld, len)));
    lr = mkray(lo, ld);
    lr.nt = r->nt * len;
    lr.ft = r->ft * len;
  }
  int h = bvh_intersect(m, &lr, tri, u, v, NULL);
  if (h) r->ft = lr.ft * tcorr;
  return h;
}
/* Scene::intersect (scene.cpp:25-39) with Sphere/Mesh intersect + intersectInfo */
static hitinfo scene_intersect(const mo_scene* s, oray* r) {
  hitinfo hi;
  hi.prim = -1;
  float mint = FLT_MAX;
  int have = 0;
  uint32_t tri = 0;
  float bu = 0, bv = 0;
  for (int i = 0; i < s->nprim; ++i) {
    const oprim* p = &s->prims[i];
    int h = 0;
    uint32_t ltri = 0;
    float lu = 0, lv = 0;
    if (p->d.type == MUPSI_PRIM_SPHERE) {
      v3 O = r->o, D = r->d;
      if (!p->identity) {
        O = m4_apply(&p->Tinv, O, 1.0f);
        D = m3_apply(&p->Tinv, D);
      }
      float t = unit_sphere(r->nt, r->ft, O, D);
      if (t >= 0.0f) {
        r->ft = t;
        h = 1;
      }
    } else {
      h = mesh_prim_intersect(&s->meshes[p->d.mesh], p, r, &ltri, &lu, &lv);
    }
    if (h) have = 1;
    /* data.primitive stays set once any primitive hit (scene.cpp:30) */
    if (have && h && r->ft < mint) {
      mint = r->ft;
      hi.prim = i;
      hi.t = r->ft;
      hi.p = vadd(r->o, vmul(r->d, r->ft));
      tri = ltri;
      bu = lu;
      bv = lv;
    }
  }
  if (hi.prim >= 0) {
    const oprim* p = &s->prims[hi.prim];
    if (p->d.type == MUPSI_PRIM_SPHERE) { /* Sphere::intersectInfo (sphere.cpp:56-76) */
      v3 pl = p->identity ? hi.p : m4_apply(&p->Tinv, hi.p, 1.0f);
      v3 ln = vnormalized(pl);
      hi.Ng = p->identity ? ln : vnormalized(m3t_apply(&p->Tinv, ln));
    } else { /* Mesh::intersectInfo (mesh.cpp:211-234) */
      const omesh* m = &s->meshes[p->d.mesh];
      v3 ln;
      if (!m->vn) {
        ln = m->face_n[tri];
      } else {
        const int32_t* f = m->f + 3 * tri;
        float w = 1.0f - bu - bv;
        v3 n = vadd(vadd(smul(w, m->vn[f[0]]), smul(bu, m->vn[f[1]])), smul(bv, m->vn[f[2]]));
        float len = vnorm(n);
        ln = len > 1e-12f ? vdiv(n, len) : m->face_n[tri];
      }
      hi.Ng = p->identity ? ln : vnormalized(m3t_apply(&p->Tinv, ln));
      if (p->tex) { /* Mesh::interpolateTexcoord (mesh.cpp:175-181) */
        if (!p->uvs) {
          hi.tu = bu;
          hi.tv = bv;
        } else {
          const int32_t* ft = p->face_uv + 3 * tri;
          const float *t0 = p->uvs + 2 * ft[0], *t1 = p->uvs + 2 * ft[1], *t2 = p->uvs + 2 * ft[2];
          float w = 1.0f - bu - bv;
          hi.tu = (w * t0[0] + bu * t1[0]) + bv * t2[0];
          hi.tv = (w * t0[1] + bu * t1[1]) + bv * t2[1];
        }
      }
    }
  }
  return hi;
}
/* Scene::occluded (scene.cpp:41-48) */
static int scene_occluded(const mo_scene* s, const oray* r) {
  for (int i = 0; i < s->nprim; ++i) {
    const oprim* p = &s->prims[i];
    if (p->d.type == MUPSI_PRIM_SPHERE) {
      v3 O = r->o, D = r->d;
      if (!p->identity) {
        O = m4_apply(&p->Tinv, O, 1.0f);
        D = m3_apply(&p->Tinv, D);
      }
      if (unit_sphere(r->nt, r->ft, O, D) >= 0.0f) return 1;
    } else {
      const omesh* m = &s->meshes[p->d.mesh];
      if (p->identity) {
        if (bvh_occluded(m, r)) return 1;
      } else {
        v3 lo = m4_apply(&p->Tinv, r->o, 1.0f);
        v3 ld = m3_apply(&p->Tinv, r->d);
        float len = vnorm(ld);
        oray lr = mkray(lo, ld);
        lr.nt = r->nt * len;
        lr.ft = r->ft * len;
        if (bvh_occluded(m, &lr)) return 1;
      }
    }
  }
  return 0;
}

typedef struct {
  v3 weight, d;
  float dist, pdf;
} lsample;

/* Scene::chooseLight (scene.cpp:50-61) + Sphere::sampleDirect (sphere.cpp:91-133) +
 * Mesh::sampleDirect (mesh.cpp:252-297) */
static int choose_light(const mo_scene* s, v3 p, pcg* smp, lsample* ls) {
  if (s->nprim == 0 || s->nlights == 0) return 0;
  uint32_t li = pcg_next(smp) % (uint32_t)s->nlights;
  const oprim* pr = &s->prims[s->lights[li]];
  v3 em = vload(pr->d.emission);
  if (pr->d.type == MUPSI_PRIM_SPHERE) {
    v3 pl = p;
    if (!pr->identity) pl = m4_apply(&pr->Tinv, p, 1.0f);
    v3 dir = vneg(pl);
    float dist2 = vsqn(dir);
    float d2 = dist2 - 1.0f;
    if (d2 < 1e-6f) return 0;
    float d = sqrtf(d2);
    float dist = sqrtf(dist2);
    dir = vdiv(dir, dist);
    float cos_t = d / dist;
    float x1 = pcg_next1d(smp), x2 = pcg_next1d(smp);
    /* uniformSphericalCap (sample.h:52-61) */
    float phi = (float)((double)(x1 * 2) * M_PI);
    float z = x2 * (1.0f - cos_t) + cos_t;
    float rr = sqrtf(fmax_std(1.0f - z * z, 0.0f));
    v3 sd = V3(cosf(phi) * rr, sinf(phi) * rr, z);
    float B = dist * sd.z;
    float det = sqrtf(fmax_std(B * B - d2, 0.0f));
    ls->dist = B - det;
    frame fr = make_frame(dir);
    ls->d = to_global(&fr, sd);
    if (!pr->identity) {
      v3 spl = vadd(pl, vmul(ls->d, ls->dist));
      v3 spw = m4_apply(&pr->T, spl, 1.0f);
      v3 wd = vsub(spw, p);
      ls->dist = vnorm(wd);
      ls->d = vdiv(wd, ls->dist);
    }
    ls->pdf = (float)(1.0f / (2.0f * M_PI * (1.0f - cos_t)));
    ls->weight = vdiv(em, fmax_std(ls->pdf, 1e-6f));
    return 1;
  } else {
    const omesh* m = &s->meshes[pr->d.mesh];
    if (m->nf == 0 || m->total_area <= 0.0f) return 0;
    float rnd = pcg_next1d(smp);
    int64_t lo = 0, hi = m->nf; /* std::lower_bound */
    while (lo < hi) {
      int64_t mid = lo + (hi - lo) / 2;
      if (m->cdf[mid] < rnd)
        lo = mid + 1;
      else
        hi = mid;
    }
    int64_t fi = lo >= m->nf ? m->nf - 1 : lo;
    float r1 = pcg_next1d(smp), r2 = pcg_next1d(smp);
    float sr1 = sqrtf(r1);
    float bu = 1.0f - sr1, bv = r2 * sr1;
    const int32_t* f = m->f + 3 * fi;
    v3 v0 = m->v[f[0]], e1 = vsub(m->v[f[1]], v0), e2 = vsub(m->v[f[2]], v0);
    v3 pt = vadd(vadd(v0, vmul(e1, bu)), vmul(e2, bv));
    if (!pr->identity) pt = m4_apply(&pr->T, pt, 1.0f);
    v3 dir = vsub(pt, p);
    float dist = sqrtf(vsqn(dir));
    ls->d = vdiv(dir, dist);
    ls->dist = dist;
    ls->pdf = 1.0f / m->total_area;
    ls->weight = vdiv(em, fmax_std(ls->pdf, 1e-6f));
    return 1;
  }
}

/* Bsdf::weight for the NEE direction (bsdf.cpp:14-77) */
static v3 bsdf_weight(int kind, v3 albedo, v3 wi, v3 wo, v3 n) {
  if (kind == MUPSI_BSDF_LAMBERTIAN) {
    float cd = vdot(wi, n);
    float pdf = (float)(fmax_std(cd, 0.0f) / M_PI);
    if (pdf == 0.0f) return V3(0, 0, 0);
    /* Vector3f / M_PI divides by the scalar converted to float */
    v3 ev = vdiv(vmul(albedo, cd), (float)M_PI);
    return vdiv(ev, pdf);
  }
  if (kind == MUPSI_BSDF_NULL) return vdot(wi, vneg(wo)) > 0.999f ? V3(1, 1, 1) : V3(0, 0, 0);
  v3 wr = vsub(smul(2.0f * vdot(wi, n), n), wi);
  return vdot(wr, wo) > 0.999f ? V3(1, 1, 1) : V3(0, 0, 0);
}
/* Bsdf::sample (bsdf.cpp:23-79): returns wi, sets weight */
static v3 bsdf_sample(int kind, v3 albedo, v3 wo, v3 n, pcg* smp, v3* weight) {
  if (kind == MUPSI_BSDF_LAMBERTIAN) {
    float r1 = pcg_next1d(smp), r2 = pcg_next1d(smp);
    float phi = (float)(2 * M_PI * r1);
    float ct = sqrtf(1 - r2);
    float st = sqrtf(r2);
    /* the reference's unqualified cos/sin take doubles here */
    v3 lw = V3((float)((double)st * cos((double)phi)), (float)((double)st * sin((double)phi)), ct);
    frame fr = make_frame(n);
    *weight = albedo;
    return to_global(&fr, lw);
  }
  *weight = V3(1, 1, 1);
  if (kind == MUPSI_BSDF_NULL) return vneg(wo);
  return vsub(smul(2.0f * vdot(wo, n), n), wo);
}

typedef struct {
  int64_t steps, evals;
} twork;

/* PathTracer::trace (trace.cpp:118-213) */
static v3 trace_sample(const mo_scene* s, int x, int y, int k, int64_t* work) {
  const uint32_t seed = 42;
  pcg ps;
  pcg_init(&ps, mo_make_seed4((uint32_t)x, (uint32_t)y, (uint32_t)k, seed));
  oray ray = camera_ray(s, x, y);
  v3 emission = V3(0, 0, 0), thr = V3(1, 1, 1);
  int has_hit, bounce = 0, medium = -1;
  mupsi_cond cond;
  memset(&cond, 0, sizeof cond);
  mupsi_medium_sample smp;
  memset(&smp, 0, sizeof smp);
  const float eps = s->d.eps, neart = s->d.nearteps;
  const int single = s->d.gp_mode == MUPSI_GP_SINGLE_REALIZATION;
  const v3 med_albedo = V3(0.8f, 0.8f, 0.8f); /* Medium::default_bsdf_ = Lambertian(0.8) */
  do {
    has_hit = 0;
    int exited = 1;
    if (medium >= 0 && !s->skip_medium) { /* trace.cpp:142 */
      const omedium* md = &s->media[medium];
      uint32_t ms = mo_make_seed5((uint32_t)x, (uint32_t)y, (uint32_t)k, seed, (uint32_t)bounce);
      csampler cs = constant_sampler(single ? seed : ms);
      any_sample_distance(s, md, &ray, cs.i, &cond, &smp, work);
      if (!smp.exited) {
        /* makeSurfaceEventFromMedium (medium.cpp:8-26) + handleVolume (trace.cpp:77-116) */
        v3 P = vload(smp.p), N = vload(smp.normal), wo = vneg(ray.d);
        lsample ls;
        if (choose_light(s, P, &ps, &ls)) {
          oray sr = mkray(vadd(P, vmul(N, eps)), ls.d);
          float bias = ls.dist - eps * fabsf(vdot(ls.d, N));
          sr.ft = bias * 0.99f;
          float tr = any_transmittance(s, md, &sr, cs.i, &cond);
          v3 f = bsdf_weight(MUPSI_BSDF_LAMBERTIAN, med_albedo, ls.d, wo, N);
          emission = vadd(emission, vmul(smul(tr, cmul(thr, cmul(f, ls.weight))), fabsf(vdot(ls.d, N))));
        }
        v3 w;
        v3 wi = bsdf_sample(MUPSI_BSDF_LAMBERTIAN, med_albedo, wo, N, &ps, &w);
        thr = cmul(thr, w);
        float surv = vmaxc(thr);
        if (pcg_next1d(&ps) > surv) break;
        thr = vdiv(thr, surv);
        uint32_t ns = mo_make_seed5((uint32_t)x, (uint32_t)y, (uint32_t)k, seed, (uint32_t)(bounce + 1));
        csampler ncs = constant_sampler(single ? seed : ns);
        if (md->kind == MUPSI_MEDIUM_GP) sample_condition(s, md, &smp, ncs.i, !single, &cond); /* trace.cpp:144-147 */
        ray = mkray(vadd(P, vmul(N, eps)), wi);
        ray.nt = neart;
        bounce++;
        exited = 0;
        has_hit = 1;
      }
    }
    if (exited) {
      hitinfo hi = scene_intersect(s, &ray);
      if (hi.prim >= 0) {
        const oprim* pr = &s->prims[hi.prim];
        v3 wo = vneg(ray.d), N = hi.Ng;
        v3 alb = pr->tex ? tex_lookup(pr->tex, pr->tex_w, pr->tex_h, hi.tu, hi.tv) : vload(pr->d.albedo);
        lsample ls;
        if (choose_light(s, hi.p, &ps, &ls)) { /* handleSurface NEE (trace.cpp:40-56) */
          oray sr = mkray(vadd(hi.p, vmul(N, eps)), ls.d);
          float bias = ls.dist - eps * fabsf(vdot(ls.d, N));
          sr.ft = bias * 0.99f;
          if (!scene_occluded(s, &sr)) {
            v3 a = bsdf_weight(pr->d.bsdf, alb, ls.d, wo, N);
            emission = vadd(emission, vmul(cmul(thr, cmul(a, ls.weight)), fabsf(vdot(ls.d, N))));
          }
        }
        v3 w;
        v3 wi = bsdf_sample(pr->d.bsdf, alb, wo, N, &ps, &w);
        if (pr->d.has_emission) {
          float c = fmax_std(0.0f, vdot(N, wi));
          emission = vadd(emission, cmul(thr, vmul(vload(pr->d.emission), c)));
        }
        thr = cmul(thr, w);
        float surv = vmaxc(thr);
        if (pcg_next1d(&ps) > surv) break;
        thr = vdiv(thr, surv);
        int back = vdot(wi, N) < 0;
        medium = back ? pr->d.int_medium : pr->d.ext_medium;
        float bs = back ? -1.0f : 1.0f;
        ray = mkray(vadd(hi.p, vmul(smul(bs, hi.Ng), eps)), wi);
        ray.nt = neart;
        bounce++;
        has_hit = 1;
      } else if (s->sky_tex) {
        emission = vadd(emission, cmul(thr, sky_lookup(s, ray.d)));
      } else if (s->d.has_sky) {
        emission = vadd(emission, cmul(thr, vload(s->d.sky)));
      }
    }
  } while (has_hit && bounce < s->d.max_bounce);
  return emission;
}

void mo_trace(const mo_scene* s, int64_t n, const int32_t* x, const int32_t* y, const int32_t* k, float* out_rgb) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < n; ++i) {
    v3 e = trace_sample(s, x[i], y[i], k[i], NULL);
    out_rgb[3 * i] = e.x;
    out_rgb[3 * i + 1] = e.y;
    out_rgb[3 * i + 2] = e.z;
  }
}

void mo_trace_work(const mo_scene* s, int64_t n, const int32_t* x, const int32_t* y, const int32_t* k,
                   int64_t* out) {
  int64_t steps = 0, evals = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : steps, evals)
  for (int64_t i = 0; i < n; ++i) {
    int64_t w[2] = {0, 0};
    trace_sample(s, x[i], y[i], k[i], w);
    steps += w[0];
    evals += w[1];
  }
  out[0] = steps;
  out[1] = evals;
}
