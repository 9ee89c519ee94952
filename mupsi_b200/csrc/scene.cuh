// Device scene and the per-ray routines of the GPIS trace loop: mean functions,
// the GP medium march (GPMedium::sampleDistance), Renewal+ conditioning,
// surface intersection, light sampling and BSDF sampling.
#pragma once
#include "dmath.cuh"
#include "geom.cuh"
#include "gp.cuh"

#define MAX_PRIMS 16
#define MAX_MEDIA 8
#define MAX_MESHES 16
#define TRACE_SEED 42u  // Renderer passes 42 as the hash seed (renderer.cpp:37)

struct DPrim {
  int type, mesh, bsdf, has_emission;
  v3 albedo, emission;
  int int_medium, ext_medium;
  int identity;
  m4 T, Tinv;
  // Lambertian BitmapTexture albedo of a mesh primitive (nullable; replaces
  // `albedo`): RGB texels, row 0 at the top, looked up at the hit's texture
  // coordinate: the mesh's texcoords `uvs` [n*2] interpolated over the face's
  // `face_uv` [F*3], or the hit's barycentrics when `uvs` is null
  const float* tex;
  const float* uvs;
  const int32_t* face_uv;
  int tex_w, tex_h;
};
// GridMeanFunction (gp/meanfunction.h:45-55): res^3 float samples, x-major,
// over [bmin, bmax]; inv = res / (bmax - bmin)
struct DGrid {
  const float* data;
  int res;
  v3 bmin, inv;
};
struct DMedium {
  int kind;  // mupsi_medium_kind
  int mean_type;
  int mesh;
  v3 center;
  float radius;
  v3 bs_c;     // mesh mean: bounding sphere of the world-space mesh (with slack)
  float bs_r;
  KParams k;
  // learned surrogate of a mesh mean (set by mupsi_gpu_scene_set_surrogate):
  // a prediction m with |m| > surr_band bounds the mean by
  // |m| / surr_scale - surr_add <= |mu| <= |m| * surr_scale + surr_add, same sign
  int surr;
  int surr_max;  // predictions per march
  int every_step;  // mesh mean queried exactly at every visited step (the plain form; no lazy mean)
  float surr_band, surr_scale, surr_add;
  // ExternalGPMedium: mean and variance grids (gvar.data null: deterministic)
  DGrid gmean, gvar;
  float noise_scale;
};

// error bits raised by device code
#define ERR_BVH_STACK 1
#define ERR_MARCH_GUARD 2

struct DScene {
  int width, height, max_bounce, gp_mode;
  v3 cpos, cdir, cright, cup;
  float tan_half, aspect;
  float eps, nearteps;
  int has_sky;
  v3 sky;
  // Skydrome with a BitmapTexture: RGB texels, row 0 at the top (nullable;
  // replaces the constant sky)
  const float* sky_tex;
  int sky_w, sky_h;
  int nprim, nmed, nmesh, nlights;
  int lights[MAX_PRIMS];
  DPrim prims[MAX_PRIMS];
  DMedium media[MAX_MEDIA];
  DMesh meshes[MAX_MESHES];
  // t_k of the march for rays with near_t == tab_nt and far_t clamped to tab_ft
  const float* tab;
  int tab_steps;  // K: tab[K] >= tab_ft, tab[k] < tab_ft for k < K
  float tab_nt, tab_ft, tab_dt;
  int* err;
  unsigned long long* counters;  // nullable: [0] march steps visited, [1] psi evaluations, [2] marches
  int min_group;                 // smallest lane group per march
  int sphere_only;               // every mean is a sphere: the march kernel without BVH code
  int field;                     // some medium is an SDF or external GP medium (k_march_field)
  int skip_medium;               // PathTracerSettings::skip_medium: media are passed through unmarched
};

// ------------------------------------------------------------ mean functions
// SphereMeanFunction / MeshMeanFunction::eval (meanfunction.cpp:13-26)
// MK: MEAN_ANY dispatches on the medium's mean type at run time; MEAN_SPHERE_ONLY
// compiles the sphere mean alone (a kernel for scenes without mesh means
// carries no BVH code and keeps its registers).
#define MEAN_ANY (-1)
#define MEAN_SPHERE_ONLY 0
// INL: the BVH traversals inline (the field march's sphere tracer)
template <int MK = MEAN_ANY, bool INL = false>
MD float mean_value(const DScene* S, const DMedium& md, v3 p, bool& ovf) {
  if constexpr (MK == MEAN_SPHERE_ONLY) return norm3(p - md.center) - md.radius;
  if (md.mean_type == MUPSI_MEAN_SPHERE) return norm3(p - md.center) - md.radius;
  const DMesh& m = S->meshes[md.mesh];
  float inside = mesh_inside<INL>(m, p, ovf) ? -1.0f : 1.0f;
  uint32_t tri;
  v3 q;
  return inside * mesh_dist<INL>(m, p, tri, q, ovf);
}
// eval + gradient (meanfunction.cpp:13-39); the mesh gradient reuses the single
// inside/closest query of the value (the reference repeats both queries).
template <int MK = MEAN_ANY, bool INL = false>
MD float4 mean_value_grad(const DScene* S, const DMedium& md, v3 p, bool& ovf) {
  if (MK == MEAN_SPHERE_ONLY || md.mean_type == MUPSI_MEAN_SPHERE) {
    v3 g = normalized(p - md.center);
    return make_float4(norm3(p - md.center) - md.radius, g.x, g.y, g.z);
  }
  if constexpr (MK == MEAN_SPHERE_ONLY) return make_float4(0, 0, 0, 0);
  const DMesh& m = S->meshes[md.mesh];
  float inside = mesh_inside<INL>(m, p, ovf) ? -1.0f : 1.0f;
  uint32_t tri = 0;
  v3 q;
  float d = mesh_dist<INL>(m, p, tri, q, ovf);
  v3 g;
  if (d < 1e-6f) {
    g = ld3(m.face_n + 3 * (int64_t)tri);
    if (!m.normal_identity) g = normalized(apply3t(m.Tinv, g));
  } else {
    g = normalized(inside * (p - q));
  }
  return make_float4(inside * d, g.x, g.y, g.z);
}

// GPMedium::evalWithGradient(p, seed, state) (gpmedium.cpp:19-41)
MD float4 medium_eval(const DScene* S, const DMedium& md, v3 p, uint32_t seed, const Cond& c, bool& ovf) {
  float4 mu = mean_value_grad(S, md, p, ovf);
  float4 nz = raw_noise(md.k, p, seed);
  float4 f = make_float4(mu.x + nz.x, mu.y + nz.y, mu.z + nz.z, mu.w + nz.w);
  return add_cond(md.k, c, p, f);
}

// ------------------------------------------------------------ field media
// SDFMedium (sdfmedium.cpp:16-98) and ExternalGPMedium (externalgpmedium.cpp:
// 9-130) march a scalar field by sphere tracing (step max(|f|, min_step)) and
// refine a sign change by 16 bisections. Both take the mean functions above or
// a GridMeanFunction; the conditioning state plays no part.

// float -> int as the reference's x86 build converts: out of range and NaN give
// INT_MIN (the GPU's own conversion saturates)
MD int f2i_x86(float f) { return (f >= -2147483648.0f && f < 2147483648.0f) ? (int)f : (int)0x80000000u; }
MD float clamp_std(float v, float lo, float hi) { return (v < lo) ? lo : ((hi < v) ? hi : v); }  // std::clamp

// GridMeanFunction::eval (meanfunction.cpp:58-78): trilinear, clamped to the grid
MD float grid_eval(const DGrid& g, v3 p) {
  const float fx = (p.x - g.bmin.x) * g.inv.x - 0.5f;
  const float fy = (p.y - g.bmin.y) * g.inv.y - 0.5f;
  const float fz = (p.z - g.bmin.z) * g.inv.z - 0.5f;
  const int i0 = max(0, min(g.res - 2, f2i_x86(floorf(fx))));
  const int j0 = max(0, min(g.res - 2, f2i_x86(floorf(fy))));
  const int k0 = max(0, min(g.res - 2, f2i_x86(floorf(fz))));
  const float wx = clamp_std(fx - (float)i0, 0.0f, 1.0f);
  const float wy = clamp_std(fy - (float)j0, 0.0f, 1.0f);
  const float wz = clamp_std(fz - (float)k0, 0.0f, 1.0f);
  const int64_t sy = g.res, sx = (int64_t)g.res * g.res;
  const float* a = g.data + i0 * sx + j0 * sy + k0;  // (i0, j0, k0); +sx: i1, +sy: j1, +1: k1
  const float c00 = __ldg(a) * (1.0f - wx) + __ldg(a + sx) * wx;
  const float c01 = __ldg(a + 1) * (1.0f - wx) + __ldg(a + sx + 1) * wx;
  const float c10 = __ldg(a + sy) * (1.0f - wx) + __ldg(a + sx + sy) * wx;
  const float c11 = __ldg(a + sy + 1) * (1.0f - wx) + __ldg(a + sx + sy + 1) * wx;
  const float c0 = c00 * (1.0f - wy) + c10 * wy;
  const float c1 = c01 * (1.0f - wy) + c11 * wy;
  return c0 * (1.0f - wz) + c1 * wz;
}
// GridMeanFunction::gradient (meanfunction.cpp:80-86): central differences, eps 1e-4
MD v3 grid_gradient(const DGrid& g, v3 p) {
  const float e = 1e-4f;
  const float dx = grid_eval(g, mk3(p.x + e, p.y, p.z)) - grid_eval(g, mk3(p.x - e, p.y, p.z));
  const float dy = grid_eval(g, mk3(p.x, p.y + e, p.z)) - grid_eval(g, mk3(p.x, p.y - e, p.z));
  const float dz = grid_eval(g, mk3(p.x, p.y, p.z + e)) - grid_eval(g, mk3(p.x, p.y, p.z - e));
  return mk3(dx, dy, dz) / (2.0f * e);
}
// hash11 (externalgpmedium.cpp:9-18): the coordinates' bit patterns folded
// into the seed, finalised, mapped to [-1, 1]
MD float hash11(v3 p, uint32_t seed) {
  uint32_t h = seed;
  h = h * 0x9e3779b1u + __float_as_uint(p.x);
  h = h * 0x9e3779b1u + __float_as_uint(p.y);
  h = h * 0x9e3779b1u + __float_as_uint(p.z);
  h = (h ^ (h >> 16)) * 0x85ebca6bu;
  h = (h ^ (h >> 13)) * 0xc2b2ae35u;
  h = h ^ (h >> 16);
  return (float)(h & 0xFFFFFFu) / 16777215.0f * 2.0f - 1.0f;
}
// ExternalGPMedium::evalWithGradient(p, seed).x (externalgpmedium.cpp:33-58)
MD float ext_value(const DMedium& md, v3 p, uint32_t seed) {
  const float mu = grid_eval(md.gmean, p);
  float noise = 0.0f;
  if (md.gvar.data && md.noise_scale > 0.0f) {
    const float var = grid_eval(md.gvar, p);
    if (var > 0.0f) noise = (md.noise_scale * sqrtf(var)) * hash11(p, seed);
  }
  return mu + noise;
}
// ExternalGPMedium::evalWithGradient(p, seed): value and gradient
MD float4 ext_value_grad(const DMedium& md, v3 p, uint32_t seed) {
  const float mu = grid_eval(md.gmean, p);
  const v3 mg = grid_gradient(md.gmean, p);
  float noise = 0.0f;
  v3 ng = mk3(0.0f, 0.0f, 0.0f);
  if (md.gvar.data && md.noise_scale > 0.0f) {
    const float var = grid_eval(md.gvar, p);
    if (var > 0.0f) {
      const float amp = md.noise_scale * sqrtf(var);
      noise = amp * hash11(p, seed);
      const float e = 0.01f;
      ng.x = amp * (hash11(mk3(p.x + e, p.y, p.z), seed) - hash11(mk3(p.x - e, p.y, p.z), seed)) / (2.0f * e);
      ng.y = amp * (hash11(mk3(p.x, p.y + e, p.z), seed) - hash11(mk3(p.x, p.y - e, p.z), seed)) / (2.0f * e);
      ng.z = amp * (hash11(mk3(p.x, p.y, p.z + e), seed) - hash11(mk3(p.x, p.y, p.z - e), seed)) / (2.0f * e);
    }
  }
  return make_float4(mu + noise, mg.x + ng.x, mg.y + ng.y, mg.z + ng.z);
}
// value of a field medium: SDFMedium::eval is the mean function itself
MD float field_value(const DScene* S, const DMedium& md, v3 p, uint32_t seed, bool& ovf) {
  return md.kind == MUPSI_MEDIUM_SDF ? mean_value<MEAN_ANY, true>(S, md, p, ovf) : ext_value(md, p, seed);
}
MD float4 field_value_grad(const DScene* S, const DMedium& md, v3 p, uint32_t seed, bool& ovf) {
  return md.kind == MUPSI_MEDIUM_SDF ? mean_value_grad<MEAN_ANY, true>(S, md, p, ovf) : ext_value_grad(md, p, seed);
}

// SDFMedium::sampleDistance (sdfmedium.cpp:16-63) / ExternalGPMedium::
// sampleDistance (externalgpmedium.cpp:69-109). A hit's normal is the
// normalised gradient there. Kept out of line: only field media reach it.
__device__ __noinline__ void field_sample_distance(const DScene* S, const DMedium& md, v3 o, v3 d, float nt, float ft,
                                                   uint32_t seed, mupsi_medium_sample& out, bool& ovf) {
  ft = fmin_std(ft, 2000.0f);
  out.exited = 1u;
  out.t = 0.0f;
  out.p[0] = out.p[1] = out.p[2] = 0.0f;
  out.normal[0] = out.normal[1] = out.normal[2] = 0.0f;
  float hit_t = 0.0f;
  bool hit = false;
  float t = nt;
  if (md.kind == MUPSI_MEDIUM_SDF) {
    float fc = field_value(S, md, o, seed, ovf);
    for (int iter = 0; t < ft && iter < 512; ++iter) {
      const float fp = fc, tp = t;
      fc = field_value(S, md, o + d * t, seed, ovf);
      if (fp * fc < 0.0f) {
        float lo = tp, hi = t, flo = fp;
        for (int b = 0; b < 16; ++b) {
          const float mid = (lo + hi) * 0.5f;
          const float fm = field_value(S, md, o + d * mid, seed, ovf);
          if (flo * fm <= 0.0f) {
            hi = mid;
          } else {
            lo = mid;
            flo = fm;
          }
        }
        hit_t = hi;
        hit = true;
        break;
      }
      t += fmax_std(fabsf(fc), 1e-3f);
    }
  } else {
    float fp = field_value(S, md, o, seed, ovf);
    for (int iter = 0; iter < 1024 && t < ft; ++iter) {
      const float fc = field_value(S, md, o + d * t, seed, ovf);
      if ((fc > 0.0f) != (fp > 0.0f) && fabsf(fp - fc) > 1e-6f) {
        float lo = t - fmax_std(fabsf(fp), 0.005f), hi = t;
        for (int b = 0; b < 16; ++b) {
          const float mid = (lo + hi) * 0.5f;
          const float fm = field_value(S, md, o + d * mid, seed, ovf);
          if ((fm > 0.0f) == (fp > 0.0f))
            lo = mid;
          else
            hi = mid;
        }
        hit_t = hi;
        hit = true;
        break;
      }
      const float step = fmax_std(fabsf(fc), 0.005f);
      fp = fc;
      t += step;
    }
  }
  if (hit) {
    const v3 p = o + d * hit_t;
    const float4 f = field_value_grad(S, md, p, seed, ovf);
    const v3 n = normalized(mk3(f.y, f.z, f.w));
    out.exited = 0u;
    out.t = hit_t;
    st3(out.p, p);
    st3(out.normal, n);
  }
}

// SDFMedium::transmittance (sdfmedium.cpp:65-96) / ExternalGPMedium::
// transmittance (externalgpmedium.cpp:111-130): 0 at the first sign change.
__device__ __noinline__ float field_transmittance(const DScene* S, const DMedium& md, v3 o, v3 d, float nt, float ft,
                                                  uint32_t seed, bool& ovf) {
  ft = fmin_std(ft, 2000.0f);
  float t = nt;
  if (md.kind == MUPSI_MEDIUM_SDF) {
    float fc = field_value(S, md, o, seed, ovf);
    for (int iter = 0; t < ft && iter < 512; ++iter) {
      const float fp = fc;
      fc = field_value(S, md, o + d * t, seed, ovf);
      if (fp * fc < 0.0f) return 0.0f;
      t += fmax_std(fabsf(fc), 1e-3f);
    }
  } else {
    float fp = field_value(S, md, o, seed, ovf);
    for (int iter = 0; iter < 1024 && t < ft; ++iter) {
      const float fc = field_value(S, md, o + d * t, seed, ovf);
      if ((fc > 0.0f) != (fp > 0.0f) && fabsf(fp - fc) > 1e-6f) return 0.0f;
      fp = fc;
      t += fmax_std(fabsf(fc), 0.005f);
    }
  }
  return 1.0f;
}

// ------------------------------------------------------------------ march
// GPMedium::sampleDistance (gpmedium.cpp:46-103). The reference steps t from
// nearT by dt (sequential float adds) while t < min(farT, 2000), evaluates
// f = mu + psi + conditioning at every step and stops at the first step whose
// sign(f > 0) differs from that of f at the ray origin with |f_origin - f| > 1e-6.
// Its refinement loop (gpmedium.cpp:67-73) computes an unused value and is not
// reproduced. Hit t is the step's t; the normal is normalize(grad f) there.
//
// Two exact work skips, both of which leave every output unchanged:
//  * |psi + conditioning| <= B for every p (|w h| <= 1 per impulse, |h| <= 1,
//    |grad h| <= gradh_max), so a step with |mu| > B has sign(f) = sign(mu)
//    and needs no psi evaluation;
//  * mu is a distance (1-Lipschitz along the unit ray), so after a step with
//    |mu| > B every later step within (|mu| - B) of it keeps that sign too and
//    is not evaluated at all. Step t values still come from the reference's
//    sequential additions (a precomputed table for the render's rays).
struct March {
  v3 o, d;
  float nt, ft, dt;
  uint32_t seed;
  Cond c;
  float B;        // bound on |psi + conditioning| at every p, with rounding slack
  float t;
  int k;
  bool use_tab;
  bool init;      // f at the origin not known yet
  bool fprev_pos;
  bool fprev_big; // |f_origin| > B: its value never decides the 1e-6 test
  float fprev;
  int status;     // 0 running, 1 hit, 2 exited, 3 suspended for a surrogate prediction at a
                  // step march_cheap reached, 4 ... in march_decide (psi of the step in spec_q),
                  // 5 waiting for the exact mean at a step march_cheap reached (defer_mu),
                  // 6 ... in march_decide (psi of the step in spec_q)
  int medium;
  uint32_t n_steps, n_psi;  // work counters: steps visited, psi evaluations
  uint32_t n_mu, n_par;     // mesh means: exact evaluations, parity casts among them
  // Lazy mean (meshes, where mu costs BVH traversals): the last exact mu and
  // its ray parameter bound |mu| at any later step; mu is only evaluated when
  // that bound cannot decide the sign of f.
  bool lazy;
  float mu_j, t_j;
  float mu_hi;      // upper bound on |mu| at t_j (|mu_j| when mu_j is exact)
  // surrogate predictions: allowed (this launch can suspend the march), made
  // so far, and the step at which the last one arrived (no second request there)
  bool may_request;
  int n_req;
  float t_resumed;
  // BVH queries of the lazy mean left to the caller (statuses 5 and 6), which
  // runs them for many marches at once (march_exact_step / march_exact_decide);
  // exact_here: mu_j is the exact mean at the current step
  bool defer_mu, exact_here;
  // pending step between the two phases
  bool pend_exact;  // pend_mu holds the exact mean at the pending point
  float pend_mu, pend_lb, pend_sgn;
  // psi of the next step, computed ahead by an otherwise idle half of a 32-lane
  // group (march_psi): valid for the step at spec_t
  bool spec_valid;
  float spec_t, spec_q;
};

// o, d: the Ray's origin and (already normalised) direction
MD void march_begin(const DScene* S, March& m, v3 o, v3 d, float near_t, float far_t, int medium, uint32_t seed,
                    const Cond& c) {
  m.o = o;
  m.d = d;
  m.nt = near_t;
  m.ft = fmin_std(far_t, 2000.0f);
  m.dt = fmin_std(0.5f, (m.ft - m.nt) / 100.0f);
  m.seed = seed;
  m.c = c;
  const KParams& k = S->media[medium].k;
  m.B = (k.psi_bound + cond_bound(k, c)) * 1.00001f + 1e-6f;
  m.t = m.nt;
  m.k = 0;
  m.use_tab = S->tab && m.nt == S->tab_nt && m.ft == S->tab_ft && m.dt == S->tab_dt;
  m.init = true;
  m.fprev_pos = false;
  m.fprev_big = false;
  m.fprev = 0.0f;
  m.status = 0;
  m.medium = medium;
  m.n_steps = 0;
  m.n_psi = 0;
  m.n_mu = 0;
  m.n_par = 0;
  m.lazy = S->media[medium].mean_type == MUPSI_MEAN_MESH && !S->media[medium].every_step;
  m.mu_j = 0.0f;
  m.t_j = 0.0f;
  m.mu_hi = 0.0f;
  m.may_request = false;
  m.defer_mu = false;
  m.exact_here = false;
  m.n_req = 0;
  m.t_resumed = -1.0f;
  m.pend_exact = false;
  m.spec_valid = false;
  m.spec_t = 0.0f;
  m.spec_q = 0.0f;
  m.pend_mu = 0.0f;
  m.pend_lb = 0.0f;
}

// Lower bound on |mu| at ray parameter t from the last exact value: mu is a
// distance along a unit-speed ray (1-Lipschitz); the slack covers the rounding
// of p = o + d t and of the distance computation.
MD float mu_lower(const March& m, float t) { return fabsf(m.mu_j) - fabsf(t - m.t_j) * 1.0001f - 1e-2f; }

// Exact mean at p = o + d t after an exact value mu_j at t_j on the same ray.
// For a mesh (MeshMeanFunction::eval = inside ? -dist : dist):
//  * dist: BVH::closest started from the bound (|mu_j| + |t - t_j|)^2 on the
//    squared distance instead of FLT_MAX (same minimum, fewer nodes);
//  * sign: when |t - t_j| < |mu_j| no surface lies between the two points and
//    the sign is mu_j's; otherwise the crossings of the march segment flip it
//    (for a closed mesh the parity test of Mesh::inside changes exactly there).
// mu_j == 0 (on the surface) or a transformed mesh use the full queries.
// BVH::closest spread over the G lanes of group g (every lane returns the same
// result): each lane keeps its own stack, a lane whose stack is empty takes the
// top entry of a lane holding two or more, and the best squared distance is
// shared after every node. Boxes are pruned only when strictly farther than the
// best, and among triangles at the best distance the lowest index wins, so the
// returned triangle and closest point do not depend on G or on which lane
// visited what. `found`: a triangle beat best_init.
// Out of line, as the single-lane traversals are (on its own this took a level-6
// mesh render at 512x512x4 from 358 to 263 ms).
template <bool CNT>
MD float bvh_closest_group_impl(const DMesh& m, v3 p, uint32_t& tri, v3& q, bool& overflow, float best_init,
                                bool& found, const Group& g) {
  BvhTally<CNT> tl;
  const int lane = (int)(threadIdx.x & 31);
  const unsigned gm = g.mask;
  uint32_t st[BVH_STACK];
  int sp = 0;
  if (g.sub == 0 && m.num_nodes > 0) st[sp++] = m.root;
  float bound = best_init;  // pruning bound shared by the group
  float lbest = best_init;  // this lane's best triangle: distance, index, point
  uint32_t btri = 0xffffffffu;
  v3 bq = mk3(0.0f, 0.0f, 0.0f);
  bool ovf = false;
  for (int guard = 0; guard < (1 << 22); ++guard) {
    const unsigned busy = __ballot_sync(gm, sp > 0) & gm;
    if (!busy || __any_sync(gm, ovf)) break;
    // idle lanes take the top entry of lanes holding two or more (the k-th
    // idle lane from the k-th donor)
    const unsigned idle = __ballot_sync(gm, sp == 0) & gm;
    const unsigned donors = __ballot_sync(gm, sp >= 2) & gm;
    const int k = min(__popc(idle), __popc(donors));
    const unsigned below = (1u << lane) - 1u;
    int src = lane;
    if (sp == 0) {
      const int r = __popc(idle & below);
      if (r < k) {
        unsigned d = donors;
        for (int i = 0; i < r; ++i) d &= d - 1u;
        src = __ffs(d) - 1;
      }
    }
    const bool give = sp >= 2 && __popc(donors & below) < k;
    const uint32_t got = __shfl_sync(gm, sp > 0 ? st[sp - 1] : 0u, src);
    if (give) --sp;
    if (sp == 0 && src != lane) st[sp++] = got;
    if (sp > 0) {
      const BNode nd = load_node(m.nodes, st[--sp]);
      tl.node();
      if (!(dist2_aabb(p, nd) > bound)) {
        if (nd.right & LEAF_FLAG) {
          const uint32_t start = nd.left, cnt = nd.right & ~LEAF_FLAG;
          for (uint32_t i = start; i < start + cnt; ++i) {
            tl.tri();
            v3 a, b, c, tmp;
            const uint32_t ti = leaf_tri(m, i, a, b, c);
            const float d = dist2_tri(p, a, b, c, tmp);
            if (d < best_init && (d < lbest || (d == lbest && ti < btri))) {
              lbest = d;
              btri = ti;
              bq = tmp;
            }
          }
          bound = fminf(bound, lbest);
        } else if (sp + 2 > BVH_STACK) {
          ovf = true;
        } else {
          BNode ln, rn;
          load_pair(m.nodes, nd.left, ln, rn);
          tl.node(2);
          const float dl = dist2_aabb(p, ln), dr = dist2_aabb(p, rn);
          if (dl < dr) {
            if (!(dr > bound)) st[sp++] = nd.right;
            if (!(dl > bound)) st[sp++] = nd.left;
          } else {
            if (!(dl > bound)) st[sp++] = nd.left;
            if (!(dr > bound)) st[sp++] = nd.right;
          }
        }
      }
    }
    for (int off = 1; off < g.G; off <<= 1) bound = fminf(bound, __shfl_xor_sync(gm, bound, off, g.G));
  }
  if (__any_sync(gm, ovf)) overflow = true;
  // the group's best distance, then the lowest triangle index at it
  float gbest = lbest;
  for (int off = 1; off < g.G; off <<= 1) gbest = fminf(gbest, __shfl_xor_sync(gm, gbest, off, g.G));
  uint32_t t = (btri != 0xffffffffu && lbest == gbest) ? btri : 0xffffffffu;
  for (int off = 1; off < g.G; off <<= 1) t = min(t, __shfl_xor_sync(gm, t, off, g.G));
  const unsigned win = __ballot_sync(gm, t != 0xffffffffu && btri == t && lbest == gbest) & gm;
  found = win != 0u;
  const int wl = found ? __ffs(win) - 1 : lane;
  const v3 wq = mk3(__shfl_sync(gm, bq.x, wl), __shfl_sync(gm, bq.y, wl), __shfl_sync(gm, bq.z, wl));
  if (found) {
    q = wq;
    tri = t;
  }
  if constexpr (CNT) {  // the group's tallies, added once by its first lane
    for (int off = 1; off < g.G; off <<= 1) {
      tl.n += __shfl_xor_sync(gm, tl.n, off, g.G);
      tl.t += __shfl_xor_sync(gm, tl.t, off, g.G);
    }
    if (g.sub == 0) tl.flush(m);
  }
  return gbest;
}
static __device__ __noinline__ float bvh_closest_group_counted(const DMesh& m, v3 p, uint32_t& tri, v3& q,
                                                                bool& overflow, float best_init, bool& found,
                                                                const Group& g) {
  return bvh_closest_group_impl<true>(m, p, tri, q, overflow, best_init, found, g);
}
static __device__ __noinline__ float bvh_closest_group(const DMesh& m, v3 p, uint32_t& tri, v3& q, bool& overflow,
                                                        float best_init, bool& found, const Group& g) {
  if (m.count) return bvh_closest_group_counted(m, p, tri, q, overflow, best_init, found, g);
  return bvh_closest_group_impl<false>(m, p, tri, q, overflow, best_init, found, g);
}

// g (nullable): the lane group marching this ray; with G > 1 the closest-point
// query is spread over its lanes (bvh_closest_group; measured in one run on the
// same GPU: -6% render time with 81,920 triangles, -34% with 1,310,720).
template <int MK = MEAN_ANY>
MD float mean_exact(const DScene* S, March& m, v3 p, float t, bool& ovf, const Group* g = nullptr) {
  const DMedium& md = S->media[m.medium];
  if constexpr (MK == MEAN_SPHERE_ONLY) return mean_value<MK>(S, md, p, ovf);
  if (!m.lazy) return mean_value(S, md, p, ovf);
  m.n_mu++;
  const DMesh& mesh = S->meshes[md.mesh];
  if (m.mu_j == 0.0f || !mesh.identity) {
    m.n_par++;
    return mean_value(S, md, p, ovf);
  }
  float sign = m.mu_j > 0.0f ? 1.0f : -1.0f;
  if (mu_lower(m, t) <= 0.0f && (segment_crossings(mesh, m.o, m.d, m.t_j, t, ovf) & 1)) sign = -sign;
  float ub = m.mu_hi + fabsf(t - m.t_j) * 1.0001f + 1e-2f;
  uint32_t tri;
  v3 q = mk3(0, 0, 0);
  bool found = false;
  if (g && g->G > 1) {
    bvh_closest_group(mesh, p, tri, q, ovf, ub * ub * 1.0001f + 1e-4f, found, *g);
    if (!found) bvh_closest_group(mesh, p, tri, q, ovf, 3.402823466e+38f, found, *g);  // bound too tight
  } else if (g && g->lowtie) {
    bvh_closest_lowtie(mesh, p, tri, q, ovf, ub * ub * 1.0001f + 1e-4f, &found);
    if (!found) bvh_closest_lowtie(mesh, p, tri, q, ovf, 3.402823466e+38f, &found);
  } else {
    bvh_closest(mesh, p, tri, q, ovf, ub * ub * 1.0001f + 1e-4f, &found);
    if (!found) bvh_closest(mesh, p, tri, q, ovf);  // the bound was too tight: full query
  }
  return sign * norm3(q - p);
}

// first step index after m.k whose t is >= target (at least m.k + 1)
MD void march_advance(const DScene* S, March& m, float target) {
  if (m.use_tab) {
    const int K = S->tab_steps;
    int kk = m.k + 1;
    if (target > m.t) {
      float est = ceilf((target - m.nt) / m.dt) - 1.0f;
      if (est > (float)kk) kk = est < (float)K ? (int)est : K;
    }
    if (kk > K) kk = K;
    while (kk > m.k + 1 && __ldg(S->tab + kk - 1) >= target) --kk;
    while (kk < K && __ldg(S->tab + kk) < target) ++kk;
    m.k = kk;
    m.t = __ldg(S->tab + kk);
  } else {
    // sequential t += dt, as the reference steps. If t + dt rounds back to t
    // the reference's loop never ends; here the march stops as exited and
    // raises ERR_MARCH_GUARD, and the add count is capped as well.
    const float t0 = m.t;
    int guard = 0;
    do {
      m.t += m.dt;
      m.k++;
    } while (m.t < target && m.t < m.ft && ++guard < (1 << 22));
    if (m.t == t0 || guard >= (1 << 22)) {
      atomicOr(S->err, ERR_MARCH_GUARD);
      m.status = 2;
    }
  }
}

// Bound on |psi + conditioning| at p (with rounding slack).
MD float noise_bound_at(const KParams& k, const Cond& c, v3 p) {
  return psi_bound_at(k, p) * 1.001f + cond_bound_at(k, c, p) * 1.001f + 2e-5f;
}

// Phase A: move through steps that need no psi evaluation. Returns true when
// the current point (origin if m.init, else step k) needs psi, with p set and
// the pending mean state (pend_*) filled.
//
// At a step with a lower bound lb on |mu|: lb > B (the bound over all p) lets the
// march jump to the first step that may have |mu| <= B; lb > noise_bound_at(p)
// settles this step's sign without psi. For a mesh mean lb comes from the last
// exact mu (Lipschitz) or the mesh's bounding sphere, and mu is re-evaluated
// (BVH) only when that is stale and cannot settle the step.
// budget: visited steps this call may settle; when it runs out the march is
// left running (status 0) at a step not yet visited, to continue in a later call.
template <int MK = MEAN_ANY>
MD bool march_cheap(const DScene* S, March& m, v3& p, bool& ovf, const Group* g = nullptr, int budget = 1 << 16) {
  const DMedium& md = S->media[m.medium];
  if (m.init) {
    p = m.o;
    if (MK != MEAN_SPHERE_ONLY && m.lazy) {
      // an origin outside the mesh's bounding sphere: mu > 0 (the parity test
      // reports outside) and |p - c| - r <= mu <= |p - c| + r; when that lower
      // bound exceeds the noise bound, sign(f) at the origin is settled
      // without a BVH query
      const float dc = norm3(p - md.bs_c);
      const float lbs = dc - md.bs_r;
      if (lbs * 0.999999f > noise_bound_at(md.k, m.c, p)) {
        m.mu_j = lbs;
        m.mu_hi = dc + md.bs_r;
        m.t_j = 0.0f;
        m.fprev_pos = true;
        m.fprev_big = true;
        m.init = false;
      }
    }
  }
  if (m.init) {
    float mu = mean_value<MK>(S, md, p, ovf);
    m.mu_j = mu;
    m.mu_hi = fabsf(mu);
    m.t_j = 0.0f;  // p(0) = o exactly
    if (fabsf(mu) * 0.999999f > noise_bound_at(md.k, m.c, p)) {
      m.fprev_pos = mu > 0.0f;
      m.fprev_big = true;
      m.init = false;
    } else {
      m.pend_exact = true;
      m.pend_mu = mu;
      m.pend_lb = fabsf(mu);
      m.pend_sgn = mu;
      return true;
    }
  }
  for (int guard = 0; guard < 1 << 16; ++guard) {
    if (guard >= budget) return false;  // continue later at this step
    if (!(m.t < m.ft)) {
      m.status = 2;
      return false;
    }
    p = m.o + m.d * m.t;
    m.n_steps++;
    float lb, sgn, mu = 0.0f;
    bool exact = MK == MEAN_SPHERE_ONLY || !m.lazy;
    if (exact) {
      mu = mean_value<MK>(S, md, p, ovf);
      m.mu_j = mu;
      m.mu_hi = fabsf(mu);
      m.t_j = m.t;
      lb = fabsf(mu);
      sgn = mu;
    } else if (m.exact_here) {  // resumed with the exact mean of this step (status 5)
      m.exact_here = false;
      mu = m.mu_j;
      lb = fabsf(mu);
      sgn = mu;
      exact = true;
    } else {
      lb = mu_lower(m, m.t);
      sgn = m.mu_j;
      // outside the mesh's bounding sphere every point of the mesh is farther
      // than |p - c| - r, and the parity test reports outside
      float lbs = norm3(p - md.bs_c) - md.bs_r;
      if (lbs > lb) {
        lb = lbs;
        sgn = 1.0f;
      }
      // a stale bound far from the last exact value: re-evaluate mu (BVH) so
      // a long jump can follow; near the surface the psi comparison decides
      if (lb * 0.999999f <= m.B && m.t - m.t_j >= fmaxf(16.0f, fabsf(m.mu_j))) {
        if (m.may_request && m.t != m.t_resumed && m.n_req < md.surr_max) {
          // ask the surrogate first: the march is suspended here and resumes
          // at this step with the prediction (march_apply_prediction)
          m.status = 3;
          return false;
        }
        if (m.defer_mu) {  // the caller queries the BVH (march_exact_step), then this step goes on
          m.n_steps--;
          m.status = 5;
          return false;
        }
        mu = mean_exact<MK>(S, m, p, m.t, ovf, g);
        m.mu_j = mu;
        m.mu_hi = fabsf(mu);
        m.t_j = m.t;
        lb = fabsf(mu);
        sgn = mu;
        exact = true;
      }
    }
    if (lb * 0.999999f > m.B) {
      if ((sgn > 0.0f) != m.fprev_pos) {  // sign(f) = sign(mu) differs: hit here
        m.status = 1;
        return false;
      }
      // mu is 1-Lipschitz: every step before `target` keeps |mu| > B
      march_advance(S, m, m.t + (lb - m.B) * 0.9999f - 2e-2f);
      if (m.status != 0) return false;
      continue;
    }
    if (lb * 0.999999f > noise_bound_at(md.k, m.c, p)) {  // this step's sign is sign(mu)
      if ((sgn > 0.0f) != m.fprev_pos) {
        m.status = 1;
        return false;
      }
      march_advance(S, m, -INFINITY);
      if (m.status != 0) return false;
      continue;
    }
    m.pend_exact = exact;
    m.pend_mu = mu;
    m.pend_lb = lb;
    m.pend_sgn = sgn;
    return true;
  }
  atomicOr(S->err, ERR_MARCH_GUARD);
  m.status = 2;
  return false;
}

// A surrogate prediction `pred` for the step where the march was suspended:
// outside the band it becomes the anchor of the lazy mean (a lower bound on
// |mu| with the prediction's sign, and an upper bound for the next exact
// query); inside the band, or too weak to bound anything, the march takes the
// exact mean at this step instead (t_resumed blocks a second request).
MD bool march_apply_prediction(const DMedium& md, March& m, float pred) {
  m.n_req++;
  m.t_resumed = m.t;
  const float a = fabsf(pred);
  const float lo = a / md.surr_scale - md.surr_add;
  if (a > md.surr_band && lo > 0.0f && isfinite(pred)) {
    m.mu_j = pred > 0.0f ? lo : -lo;
    m.mu_hi = a * md.surr_scale + md.surr_add;
    m.t_j = m.t;
    return true;
  }
  return false;
}

template <int MK>
MD void march_decide(const DScene* S, March& m, v3 p, float q, const Group* g, bool& ovf);

// f at the current step decided: the origin's value, a hit, or the next step.
MD void march_settle(const DScene* S, March& m, float f) {
  if (m.init) {
    m.fprev = f;
    m.fprev_pos = f > 0.0f;
    m.init = false;
    return;
  }
  if ((f > 0.0f) != m.fprev_pos && (m.fprev_big || (double)fabsf(m.fprev - f) > 1e-6)) {
    m.status = 1;
    return;
  }
  march_advance(S, m, -INFINITY);
}

// A march suspended in march_decide (status 4) resumes there: the step's psi q
// (saved with the march) and the prediction's anchor, or, without a usable
// prediction, the exact mean (t_resumed blocks a second request).
// Out of line: inlined into the refill path it doubled the mesh kernel's spills.
template <int MK>
static __device__ __noinline__ void march_resume_decide(const DScene* S, March& m, float q, const Group* g,
                                                        bool& ovf) {
  m.pend_exact = false;
  m.pend_lb = 0.0f;  // the |mu| bound of the step did not settle it before the suspension
  m.pend_sgn = 0.0f;
  march_decide<MK>(S, m, m.o + m.d * m.t, q, g, ovf);
}

// A march waiting for the exact mean at the step march_cheap reached (status
// 5): the BVH query, then the step goes on as march_cheap takes it with the
// exact value. Out of line, as march_resume_decide.
template <int MK>
static __device__ __noinline__ void march_exact_step(const DScene* S, March& m, const Group* g, bool& ovf) {
  const float mu = mean_exact<MK>(S, m, m.o + m.d * m.t, m.t, ovf, g);
  m.mu_j = mu;
  m.mu_hi = fabsf(mu);
  m.t_j = m.t;
  m.exact_here = true;
  m.status = 0;
}
// A march waiting for the exact mean in march_decide (status 6, the step's psi
// in spec_q): the BVH query and the rest of march_decide.
template <int MK>
static __device__ __noinline__ void march_exact_decide(const DScene* S, March& m, const Group* g, bool& ovf) {
  m.status = 0;
  const v3 p = m.o + m.d * m.t;
  const DMedium& md = S->media[m.medium];
  const float q = m.spec_q;
  float c = m.c.active ? cond_value(md.k, m.c, p) : 0.0f;
  float mu = mean_exact<MK>(S, m, p, m.t, ovf, g);
  m.mu_j = mu;
  m.mu_hi = fabsf(mu);
  m.t_j = m.t;
  float f = mu + q;
  if (m.c.active) f += c;
  march_settle(S, m, f);
}

// Phase B: f at the pending point (value only); decides hit or next step. The
// psi sum is shared by the lanes of group g (all of which hold the same march).
// WIDE: the group has G >= 4 lanes.
template <int MK = MEAN_ANY, bool WIDE = false>
MD void march_psi(const DScene* S, March& m, v3 p, const Group& g, bool& ovf) {
  const DMedium& md = S->media[m.medium];
  m.n_psi++;
  float q;
  if (m.spec_valid && m.spec_t == m.t) {
    q = m.spec_q;  // computed with the previous step (same point, same order)
    m.spec_valid = false;
  } else if (MK == MEAN_SPHERE_ONLY && WIDE && g.G == 32) {
    // The psi order keeps 16 lanes busy; the upper half evaluates the next step
    // (sphere-mean marches: in mesh marches the BVH queries set the pace)
    // (t as march_advance will produce it, the same point march_cheap will form)
    // for use if the march gets there next.
    float tn = m.t;
    bool ok;
    if (m.use_tab) {
      ok = m.k + 1 <= S->tab_steps;
      if (ok) tn = __ldg(S->tab + m.k + 1);
    } else {
      tn = m.t + m.dt;
      ok = tn < m.ft && tn != m.t;
    }
    const bool upper = g.sub >= 16;
    Group h;
    h.G = 16;
    h.sub = g.sub & 15;
    h.mask = upper ? 0xffff0000u : 0x0000ffffu;
    const v3 pe = upper && ok ? m.o + m.d * tn : p;
    const float v = (md.k.sigma * psi_sums_group<false, true, -1>(md.k, pe, m.seed, h).x) / md.k.sqrt_var;
    const float vo = __shfl_xor_sync(0xffffffffu, v, 16);
    q = upper ? vo : v;
    m.spec_q = upper ? v : vo;
    m.spec_t = tn;
    m.spec_valid = ok;
  } else {
    q = raw_noise_value_group<WIDE, MK == MEAN_SPHERE_ONLY ? -1 : 0>(md.k, p, m.seed, g);
  }
  march_decide<MK>(S, m, p, q, &g, ovf);
}

// Phase B after psi: q = RawNoise(p) at the pending point; f decides a hit or
// the next step.
template <int MK>
MD void march_decide(const DScene* S, March& m, v3 p, float q, const Group* g, bool& ovf) {
  const DMedium& md = S->media[m.medium];
  float c = m.c.active ? cond_value(md.k, m.c, p) : 0.0f;
  float f;
  if (m.pend_exact) {
    f = m.pend_mu + q;
    if (m.c.active) f += c;
  } else {
    // |mu| >= pend_lb > |psi + cond| (with rounding slack) gives sign(f) = sign(mu)
    // and |f| > 1e-6 without evaluating the mean
    float s = (fabsf(q) + fabsf(c)) * 1.00001f + 1e-5f;
    if (m.pend_lb * 0.999999f > s) {
      if ((m.pend_sgn > 0.0f) != m.fprev_pos) {
        m.status = 1;
        return;
      }
      march_advance(S, m, -INFINITY);
      return;
    }
    if (m.lazy) {
      // mu is a signed distance, 1-Lipschitz along the ray: from the anchor it
      // lies in [mu_lo, mu_hi] here. When that interval plus psi + cond keeps
      // the sign f had at the origin, this step is not a hit and needs no BVH
      // query (a sign change still takes the exact value below).
      const float d = fabsf(m.t - m.t_j) * 1.0001f + 1e-2f;
      const float lo = (m.mu_j > 0.0f ? m.mu_j : -m.mu_hi) - d;
      const float hi = (m.mu_j > 0.0f ? m.mu_hi : m.mu_j) + d;
      const float qc = q + c;
      const float slack = (fabsf(q) + fabsf(c) + fmaxf(fabsf(lo), fabsf(hi))) * 1e-5f + 1e-5f;
      if ((m.fprev_pos && lo + qc > slack) || (!m.fprev_pos && hi + qc < -slack)) {
        march_advance(S, m, -INFINITY);
        return;
      }
    }
    if (MK != MEAN_SPHERE_ONLY && m.may_request && m.t != m.t_resumed && m.n_req < md.surr_max) {
      // ask the surrogate before a BVH query here too: a prediction outside the
      // band bounds |mu| at this step, which may settle the sign with this psi
      // (march_resume_decide); the exact mean stays the fallback
      m.spec_q = q;
      m.status = 4;
      return;
    }
    if (m.defer_mu) {  // the caller queries the BVH (march_exact_decide)
      m.spec_q = q;
      m.status = 6;
      return;
    }
    float mu = mean_exact<MK>(S, m, p, m.t, ovf, g);
    m.mu_j = mu;
    m.mu_hi = fabsf(mu);
    m.t_j = m.t;
    f = mu + q;
    if (m.c.active) f += c;
  }
  march_settle(S, m, f);
}

// GPMedium::evalWithGradient with the psi sum shared by group g (WIDE: g.G >= 4)
template <int MK = MEAN_ANY, bool WIDE = false>
MD float4 medium_eval_group(const DScene* S, const DMedium& md, v3 p, uint32_t seed, const Cond& c, bool& ovf,
                            const Group& g) {
  float4 mu = mean_value_grad<MK>(S, md, p, ovf);
  float4 nz = raw_noise_group<WIDE, MK == MEAN_SPHERE_ONLY ? -1 : 0>(md.k, p, seed, g);
  float4 f = make_float4(mu.x + nz.x, mu.y + nz.y, mu.z + nz.z, mu.w + nz.w);
  return add_cond(md.k, c, p, f);
}

// hit point and normal of a finished march
// (an exited march leaves t, p and normal zero: sampleDistance does not write them)
template <int MK = MEAN_ANY, bool WIDE = false>
MD void march_result(const DScene* S, const March& m, mupsi_medium_sample& out, bool& ovf, const Group& g) {
  out.exited = m.status == 1 ? 0u : 1u;
  out.t = m.status == 1 ? m.t : 0.0f;
  if (m.status == 1) {
    v3 p = m.o + m.d * m.t;
    float4 f = medium_eval_group<MK, WIDE>(S, S->media[m.medium], p, m.seed, m.c, ovf, g);
    v3 n = normalized(mk3(f.y, f.z, f.w));
    st3(out.p, p);
    st3(out.normal, n);
  } else {
    st3(out.p, mk3(0, 0, 0));
    st3(out.normal, mk3(0, 0, 0));
  }
}

MD Group single_lane() {
  Group g;
  g.G = 1;
  g.sub = 0;
  g.mask = __activemask();
  return g;
}

// Whole march in one thread (batch entry, transmittance).
MD void march_full(const DScene* S, March& m, bool& ovf) {
  const Group g = single_lane();
  for (int guard = 0; m.status == 0 && guard < 1 << 16; ++guard) {
    v3 p;
    if (march_cheap(S, m, p, ovf)) march_psi(S, m, p, g, ovf);
  }
  if (m.status == 0) {
    atomicOr(S->err, ERR_MARCH_GUARD);
    m.status = 2;
  }
}

// GPMedium::sampleCondition (gpmedium.cpp:133-161)
MD Cond sample_condition(const DScene* S, const DMedium& md, v3 P, v3 N, bool exited, uint32_t seed, bool renewal,
                         bool& ovf) {
  Cond c;
  c.active = 0;
  c.C = mk3(0, 0, 0);
  c.u = 0.0f;
  c.g = mk3(0, 0, 0);
  if (renewal && !exited) {
    c.active = 1;
    c.C = P;
    float4 psi = raw_noise(md.k, P, seed);
    float4 mu = mean_value_grad(S, md, P, ovf);
    c.u = -mu.x / md.k.sigma - psi.x;
    float s = -md.k.L2 / 2.0f;  // oneOverSecondDerivative (kernel.h:66-68)
    c.g = s * ((N - mk3(mu.y, mu.z, mu.w)) - mk3(psi.y, psi.z, psi.w));
  }
  return c;
}

// --------------------------------------------------------------- surfaces
struct Hit {
  int prim;
  float t;
  v3 p, Ng;
  float tu, tv;  // texture coordinate (only for a primitive with an albedo texture)
};

// Scene::intersect (scene.cpp:25-39) with Sphere/Mesh intersect and intersectInfo
MD Hit scene_intersect(const DScene* S, Ray& r, bool& ovf) {
  Hit hi;
  hi.prim = -1;
  float mint = 3.402823466e+38f;
  uint32_t tri = 0;
  float bu = 0.0f, bv = 0.0f;
  for (int i = 0; i < S->nprim; ++i) {
    const DPrim& p = S->prims[i];
    bool h = false;
    uint32_t ltri = 0;
    float lu = 0.0f, lv = 0.0f;
    if (p.type == MUPSI_PRIM_SPHERE) {
      v3 O = r.o, D = r.d;
      if (!p.identity) {
        O = apply4(p.Tinv, O);
        D = apply3(p.Tinv, D);
      }
      float t = unit_sphere(r.nt, r.ft, O, D);
      if (t >= 0.0f) {
        r.ft = t;
        h = true;
      }
    } else {
      const DMesh& m = S->meshes[p.mesh];
      Ray lr = r;
      float tc = 1.0f;
      if (!p.identity) {  // mesh.cpp:185-209
        v3 lo = apply4(p.Tinv, r.o);
        v3 ld = apply3(p.Tinv, r.d);
        float len = norm3(ld);
        tc = norm3(apply3(p.T, ld / len));
        lr = make_ray(lo, ld);
        lr.nt = r.nt * len;
        lr.ft = r.ft * len;
      }
      if (bvh_intersect(m, lr, ltri, lu, lv, ovf)) {
        r.ft = lr.ft * tc;
        h = true;
      }
    }
    if (h && r.ft < mint) {
      mint = r.ft;
      hi.prim = i;
      hi.t = r.ft;
      hi.p = r.o + r.d * r.ft;
      tri = ltri;
      bu = lu;
      bv = lv;
    }
  }
  if (hi.prim >= 0) {
    const DPrim& p = S->prims[hi.prim];
    if (p.type == MUPSI_PRIM_SPHERE) {  // sphere.cpp:56-76
      v3 pl = p.identity ? hi.p : apply4(p.Tinv, hi.p);
      v3 ln = normalized(pl);
      hi.Ng = p.identity ? ln : normalized(apply3t(p.Tinv, ln));
    } else {  // mesh.cpp:211-234
      const DMesh& m = S->meshes[p.mesh];
      v3 ln;
      if (!m.vert_n) {
        ln = ld3(m.face_n + 3 * (int64_t)tri);
      } else {
        const int32_t* f = m.faces + 3 * (int64_t)tri;
        float w = 1.0f - bu - bv;
        v3 n = (w * ld3(m.vert_n + 3 * (int64_t)f[0]) + bu * ld3(m.vert_n + 3 * (int64_t)f[1])) +
               bv * ld3(m.vert_n + 3 * (int64_t)f[2]);
        float len = norm3(n);
        ln = len > 1e-12f ? n / len : ld3(m.face_n + 3 * (int64_t)tri);
      }
      hi.Ng = p.identity ? ln : normalized(apply3t(p.Tinv, ln));
      if (p.tex) {  // Mesh::interpolateTexcoord (mesh.cpp:175-181)
        if (!p.uvs) {
          hi.tu = bu;
          hi.tv = bv;
        } else {
          const int32_t* ft = p.face_uv + 3 * (int64_t)tri;
          const float* t0 = p.uvs + 2 * (int64_t)ft[0];
          const float* t1 = p.uvs + 2 * (int64_t)ft[1];
          const float* t2 = p.uvs + 2 * (int64_t)ft[2];
          float w = 1.0f - bu - bv;
          hi.tu = (w * t0[0] + bu * t1[0]) + bv * t2[0];
          hi.tv = (w * t0[1] + bu * t1[1]) + bv * t2[1];
        }
      }
    }
  }
  return hi;
}

// BitmapTexture::operator[] (texture.cpp:52-69): wrap (u, v) to [0, 1), flip v
// (row 0 is the top), nearest texel. Every int the casts produce lands inside
// the image after the modulo.
MD v3 tex_lookup(const float* tex, int w, int h, float u, float v) {
  u = u - floorf(u);
  v = v - floorf(v);
  v = 1.0f - v;
  int x = (int)(u * (float)w) % w;
  int y = (int)(v * (float)h) % h;
  if (x < 0) x += w;
  if (y < 0) y += h;
  const float* t = tex + 3 * ((int64_t)y * w + x);
  return mk3(__ldg(t), __ldg(t + 1), __ldg(t + 2));
}

// Skydrome::intersect (skydrome.cpp:8-17) + BitmapTexture::operator[]
// (texture.cpp:52-69): equirectangular (u, v) of the direction in the
// reference's float/double mix, nearest texel, v flipped (row 0 at the top).
MD v3 sky_lookup(const DScene* S, v3 dir) {
  const double pi = 3.14159265358979323846;
  float u = (float)(((double)atan2f(dir.z, dir.x) + pi) / (2.0f * pi));
  float cy = -dir.y;
  cy = cy < -1.0f ? -1.0f : (cy > 1.0f ? 1.0f : cy);
  float v = (float)((double)acosf(cy) / pi);
  return tex_lookup(S->sky_tex, S->sky_w, S->sky_h, u, v);
}

// Scene::occluded (scene.cpp:41-48)
MD bool scene_occluded(const DScene* S, const Ray& r, bool& ovf) {
  for (int i = 0; i < S->nprim; ++i) {
    const DPrim& p = S->prims[i];
    if (p.type == MUPSI_PRIM_SPHERE) {
      v3 O = r.o, D = r.d;
      if (!p.identity) {
        O = apply4(p.Tinv, O);
        D = apply3(p.Tinv, D);
      }
      if (unit_sphere(r.nt, r.ft, O, D) >= 0.0f) return true;
    } else {
      const DMesh& m = S->meshes[p.mesh];
      if (p.identity) {
        if (bvh_occluded(m, r, ovf)) return true;
      } else {
        v3 lo = apply4(p.Tinv, r.o);
        v3 ld = apply3(p.Tinv, r.d);
        float len = norm3(ld);
        Ray lr = make_ray(lo, ld);
        lr.nt = r.nt * len;
        lr.ft = r.ft * len;
        if (bvh_occluded(m, lr, ovf)) return true;
      }
    }
  }
  return false;
}

struct LSample {
  v3 weight, d;
  float dist, pdf;
};

// Scene::chooseLight (scene.cpp:50-61), Sphere::sampleDirect (sphere.cpp:91-133),
// Mesh::sampleDirect (mesh.cpp:252-297)
MD bool choose_light(const DScene* S, v3 p, uint64_t& rng, LSample& ls) {
  if (S->nprim == 0 || S->nlights == 0) return false;
  uint32_t li = pcg_next(rng) % (uint32_t)S->nlights;
  const DPrim& pr = S->prims[S->lights[li]];
  if (pr.type == MUPSI_PRIM_SPHERE) {
    v3 pl = pr.identity ? p : apply4(pr.Tinv, p);
    v3 dir = -pl;
    float dist2 = sqn(dir);
    float d2 = dist2 - 1.0f;
    if (d2 < 1e-6f) return false;
    float d = sqrtf(d2);
    float dist = sqrtf(dist2);
    dir = dir / dist;
    float ct = d / dist;
    float x1 = pcg_next1d(rng), x2 = pcg_next1d(rng);
    float phi = (float)((double)(x1 * 2.0f) * 3.14159265358979323846);
    float z = x2 * (1.0f - ct) + ct;
    float rr = sqrtf(fmax_std(1.0f - z * z, 0.0f));
    v3 sd = mk3(cosf(phi) * rr, sinf(phi) * rr, z);
    float Bq = dist * sd.z;
    float det = sqrtf(fmax_std(Bq * Bq - d2, 0.0f));
    ls.dist = Bq - det;
    Frame fr = make_frame(dir);
    ls.d = to_global(fr, sd);
    if (!pr.identity) {
      v3 spl = pl + ls.d * ls.dist;
      v3 wd = apply4(pr.T, spl) - p;
      ls.dist = norm3(wd);
      ls.d = wd / ls.dist;
    }
    ls.pdf = (float)(1.0 / (2.0 * 3.14159265358979323846 * (double)(1.0f - ct)));
    ls.weight = pr.emission / fmax_std(ls.pdf, 1e-6f);
    return true;
  }
  const DMesh& m = S->meshes[pr.mesh];
  if (m.num_faces == 0 || m.total_area <= 0.0f) return false;
  float rnd = pcg_next1d(rng);
  int64_t lo = 0, hi = m.num_faces;
  while (lo < hi) {
    int64_t mid = lo + (hi - lo) / 2;
    if (m.cdf[mid] < rnd)
      lo = mid + 1;
    else
      hi = mid;
  }
  int64_t fi = lo >= m.num_faces ? m.num_faces - 1 : lo;
  float r1 = pcg_next1d(rng), r2 = pcg_next1d(rng);
  float sr1 = sqrtf(r1);
  float bu = 1.0f - sr1, bv = r2 * sr1;
  const int32_t* f = m.faces + 3 * fi;
  v3 v0 = vert(m, f[0]);
  v3 pt = (v0 + (vert(m, f[1]) - v0) * bu) + (vert(m, f[2]) - v0) * bv;
  if (!pr.identity) pt = apply4(pr.T, pt);
  v3 dir = pt - p;
  float dist = sqrtf(sqn(dir));
  ls.d = dir / dist;
  ls.dist = dist;
  ls.pdf = 1.0f / m.total_area;
  ls.weight = pr.emission / fmax_std(ls.pdf, 1e-6f);
  return true;
}

// Bsdf::weight toward the light (bsdf.cpp:14-77)
MD v3 bsdf_weight(int kind, v3 albedo, v3 wi, v3 wo, v3 n) {
  if (kind == MUPSI_BSDF_LAMBERTIAN) {
    float cd = dot(wi, n);
    float pdf = (float)((double)fmax_std(cd, 0.0f) / 3.14159265358979323846);
    if (pdf == 0.0f) return mk3(0, 0, 0);
    v3 ev = (albedo * cd) / 3.14159265f;  // Vector3f / M_PI divides by (float)M_PI
    return ev / pdf;
  }
  if (kind == MUPSI_BSDF_NULL) return dot(wi, -wo) > 0.999f ? mk3(1, 1, 1) : mk3(0, 0, 0);
  v3 wr = (2.0f * dot(wi, n)) * n - wi;
  return dot(wr, wo) > 0.999f ? mk3(1, 1, 1) : mk3(0, 0, 0);
}

// Bsdf::sample (bsdf.cpp:23-79): returns wi, sets the weight
MD v3 bsdf_sample(int kind, v3 albedo, v3 wo, v3 n, uint64_t& rng, v3& weight) {
  if (kind == MUPSI_BSDF_LAMBERTIAN) {
    float r1 = pcg_next1d(rng), r2 = pcg_next1d(rng);
    float phi = (float)(2.0 * 3.14159265358979323846 * (double)r1);
    float ct = sqrtf(1.0f - r2);
    float st = sqrtf(r2);
    // the reference's build evaluates these cos/sin in double precision
    double sp, cp;
    sincos((double)phi, &sp, &cp);
    v3 lw = mk3((float)((double)st * cp), (float)((double)st * sp), ct);
    Frame fr = make_frame(n);
    weight = albedo;
    return to_global(fr, lw);
  }
  weight = mk3(1, 1, 1);
  if (kind == MUPSI_BSDF_NULL) return -wo;
  return (2.0f * dot(wo, n)) * n - wo;
}

// Camera::generateRay (camera.cpp:5-20)
MD Ray camera_ray(const DScene* S, int x, int y) {
  float cx = ((float)x + 0.5f) / (float)S->width;
  float cy = ((float)y + 0.5f) / (float)S->height;
  float nx = (2.0f * cx - 1.0f) * S->aspect * S->tan_half;
  float ny = (2.0f * cy - 1.0f) * S->tan_half;
  v3 dc = normalized(mk3(nx, ny, 1.0f));
  v3 w = normalized((S->cright * dc.x + S->cup * dc.y) + S->cdir * dc.z);
  return make_ray(S->cpos, normalized(w));
}
