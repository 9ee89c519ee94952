// Scenes, the GP-medium batch entry points and the wavefront path tracer
// (PathTracer::trace, rendering/trace.cpp:118-213, driven like
// Renderer::startRenderProgressive, rendering/renderer.cpp:22-49).
//
// Wavefront layout: a wave holds W*H*passes paths in structure-of-arrays state.
// Each bounce iteration runs two kernels:
//   k_march  - persistent warps march every path that is inside a GP medium;
//              idle lanes pull the next path from the medium queue, so long and
//              short marches never stall a warp;
//   k_shade  - every live path: medium event (NEE, Lambertian sample, Russian
//              roulette, Renewal+ conditioning) or surface event (scene
//              intersection, NEE, BSDF sample, RR, medium switch) or sky; the
//              survivors are appended to the next iteration's queues with
//              warp-aggregated atomics.
// Each path does exactly one bounce per iteration (or terminates), so a wave
// takes at most max_bounce iterations. Per-sample radiance is written to a
// buffer and summed per pixel in pass order (Framebuffer::accumulate order).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "core.cuh"
#include "scene.cuh"

namespace cg = cooperative_groups;

namespace mupsi {

// ------------------------------------------------------------ path state
struct Paths {
  float4* o;    // origin xyz, near_t
  float4* d;    // direction xyz, medium index (int bits; -1 none)
  float4* thr;  // throughput xyz
  float4* em;   // emission xyz
  uint2* rng;   // path sampler state (u64)
  float4* ca;   // conditioning C xyz, u
  float4* cb;   // conditioning g xyz, active
  int4* meta;   // x, y, k, bounce
  float4* ha;   // march: t, p xyz
  float4* hb;   // march: normal xyz, exited
  float* rad;   // final radiance [cap * 3]
  uint32_t* q[4];       // medium queue (2 buffers), live queue (2 buffers)
  uint32_t* counts;     // per iteration: [it*2+0] medium count, [it*2+1] live count
  uint32_t* cursors;    // per iteration: march work cursor
  int64_t cap;
};

MD uint64_t ld_rng(const uint2 v) { return ((uint64_t)v.y << 32) | v.x; }
MD uint2 st_rng(uint64_t s) { return make_uint2((uint32_t)s, (uint32_t)(s >> 32)); }

MD Cond load_cond(const Paths& P, uint32_t i) {
  float4 a = P.ca[i], b = P.cb[i];
  Cond c;
  c.C = mk3(a.x, a.y, a.z);
  c.u = a.w;
  c.g = mk3(b.x, b.y, b.z);
  c.active = __float_as_uint(b.w);
  return c;
}
MD void store_cond(const Paths& P, uint32_t i, const Cond& c) {
  P.ca[i] = make_float4(c.C.x, c.C.y, c.C.z, c.u);
  P.cb[i] = make_float4(c.g.x, c.g.y, c.g.z, __uint_as_float(c.active));
}

// ConstantSampler seed of bounce b's medium sampler (trace.cpp:146-147)
MD uint32_t medium_seed(const DScene* S, int x, int y, int k, int b) {
  uint32_t s = S->gp_mode == MUPSI_GP_SINGLE_REALIZATION
                   ? TRACE_SEED
                   : make_seed5((uint32_t)x, (uint32_t)y, (uint32_t)k, TRACE_SEED, (uint32_t)b);
  return constant_sampler_i(s);
}

// ------------------------------------------------------------ kernels
__global__ void k_raygen(const DScene* __restrict__ S, Paths P, int64_t n, int pass0, const int32_t* xs,
                         const int32_t* ys, const int32_t* ks) {
  const int64_t wh = (int64_t)S->width * S->height;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int x, y, k;
    if (xs) {
      x = xs[i];
      y = ys[i];
      k = ks[i];
    } else {
      int64_t pix = i % wh;
      k = pass0 + (int)(i / wh);
      x = (int)(pix % S->width);
      y = (int)(pix / S->width);
    }
    uint64_t rng = pcg_seeded(make_seed4((uint32_t)x, (uint32_t)y, (uint32_t)k, TRACE_SEED));
    Ray r = camera_ray(S, x, y);
    P.o[i] = make_float4(r.o.x, r.o.y, r.o.z, r.nt);
    P.d[i] = make_float4(r.d.x, r.d.y, r.d.z, __int_as_float(-1));
    P.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    P.em[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    P.rng[i] = st_rng(rng);
    P.ca[i] = make_float4(0, 0, 0, 0);
    P.cb[i] = make_float4(0, 0, 0, __uint_as_float(0u));
    P.meta[i] = make_int4(x, y, k, 0);
    P.q[2][i] = (uint32_t)i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.counts[0] = 0;
    P.counts[1] = (uint32_t)n;
  }
}

// Persistent march over the medium queue of iteration `it`. Each ray is
// marched by a group of G lanes that share its psi sums: G = 4 while the queue
// fills the resident threads, larger (up to 32) as the queue shrinks, so the
// late bounces' few long marches finish up to 8x sooner than on one lane.
template <bool CACHE, int MK>
__global__ void __launch_bounds__(128) k_march(const DScene* __restrict__ S, Paths P, int it) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t n = P.counts[2 * it];
  const uint32_t* q = P.q[it & 1];
  uint32_t* cursor = P.cursors + it;
  const unsigned lane = threadIdx.x & 31;
  const uint64_t resident = (uint64_t)gridDim.x * blockDim.x;
  Group grp;
  grp.G = S->min_group;
  while (grp.G < 32 && (uint64_t)n * (uint64_t)(2 * grp.G) <= resident) grp.G <<= 1;
  grp.sub = (int)(lane & (unsigned)(grp.G - 1));
  const unsigned gbase = lane & ~(unsigned)(grp.G - 1);
  grp.mask = grp.G == 32 ? 0xffffffffu : (((1u << grp.G) - 1u) << gbase);
  ImpCache cache;
  if (CACHE) {  // this group's slot table (G >= 4: at most 32 groups per block)
    unsigned char* base = smem + (size_t)(threadIdx.x / grp.G) * kCacheBytes;
    cache.tag = reinterpret_cast<int*>(base + 27 * CACHE_MAX_PPC * 16);
    cache.imp = reinterpret_cast<float4*>(base);
  }
  March m;
  uint32_t idx = 0;
  bool active = false;
  bool ovf = false;
  unsigned long long steps = 0, psis = 0, marches = 0, imps = 0, mus = 0, pars = 0;
  while (true) {
    // refill idle groups from the queue (warp-aggregated over group leaders)
    unsigned need = __ballot_sync(0xffffffffu, !active && grp.sub == 0);
    if (need) {
      uint32_t base = 0;
      int leader = __ffs(need) - 1;
      if ((int)lane == leader) base = atomicAdd(cursor, (uint32_t)__popc(need));
      base = __shfl_sync(0xffffffffu, base, leader);
      uint32_t j = base + __popc(need & ((1u << lane) - 1u));
      j = __shfl_sync(0xffffffffu, j, (int)gbase);
      if (!active) {
        if (j < n) {
          idx = q[j];
          float4 o = P.o[idx], d = P.d[idx];
          int4 meta = P.meta[idx];
          int med = __float_as_int(d.w);
          march_begin(S, m, mk3(o.x, o.y, o.z), mk3(d.x, d.y, d.z), o.w, 3.402823466e+38f, med,
                      medium_seed(S, meta.x, meta.y, meta.z, meta.w), load_cond(P, idx));
          if (CACHE) cache_clear(cache, grp);
          active = true;
          if (grp.sub == 0) marches++;
        }
      }
    }
    if (!__any_sync(0xffffffffu, active)) break;
    if (active) {
      v3 p;
      if (march_cheap<MK>(S, m, p, ovf)) march_psi<MK>(S, m, p, grp, ovf, CACHE ? &cache : nullptr);
      if (m.status != 0) {
        mupsi_medium_sample r;
        march_result<MK>(S, m, r, ovf, grp, CACHE ? &cache : nullptr);
        if (grp.sub == 0) {
          P.ha[idx] = make_float4(r.t, r.p[0], r.p[1], r.p[2]);
          P.hb[idx] = make_float4(r.normal[0], r.normal[1], r.normal[2], __uint_as_float(r.exited));
          steps += m.n_steps;
          psis += m.n_psi;
          imps += (unsigned long long)m.n_psi * 27ull * (unsigned long long)S->media[m.medium].k.ppc;
          mus += m.n_mu;
          pars += m.n_par;
        }
        active = false;
      }
    }
  }
  if (ovf) atomicOr(S->err, ERR_BVH_STACK);
  if (S->counters) {
    for (int o = 16; o > 0; o >>= 1) {
      steps += __shfl_down_sync(0xffffffffu, steps, o);
      psis += __shfl_down_sync(0xffffffffu, psis, o);
      marches += __shfl_down_sync(0xffffffffu, marches, o);
      imps += __shfl_down_sync(0xffffffffu, imps, o);
      mus += __shfl_down_sync(0xffffffffu, mus, o);
      pars += __shfl_down_sync(0xffffffffu, pars, o);
    }
    if (lane == 0) {
      atomicAdd(&S->counters[0], steps);
      atomicAdd(&S->counters[1], psis);
      atomicAdd(&S->counters[2], marches);
      atomicAdd(&S->counters[3], imps);
      atomicAdd(&S->counters[4], mus);
      atomicAdd(&S->counters[5], pars);
    }
  }
}

// GPMedium::transmittance (gpmedium.cpp:105-129): 0 at the first sign change.
MD float transmittance(const DScene* S, int medium, const Ray& r, uint32_t seed, const Cond& c, bool& ovf) {
  March m;
  march_begin(S, m, r.o, r.d, r.nt, r.ft, medium, seed, c);
  march_full(S, m, ovf);
  return m.status == 1 ? 0.0f : 1.0f;
}

MD void push(uint32_t* q, uint32_t* count, uint32_t v) {
  cg::coalesced_group g = cg::coalesced_threads();
  uint32_t base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(count, g.size());
  base = g.shfl(base, 0);
  q[base + g.thread_rank()] = v;
}

// One bounce of PathTracer::trace for every live path of iteration `it`.
__global__ void __launch_bounds__(128) k_shade(const DScene* __restrict__ S, Paths P, int it) {
  const uint32_t n = P.counts[2 * it + 1];
  const uint32_t* q = P.q[2 + (it & 1)];
  uint32_t* qm_next = P.q[(it + 1) & 1];
  uint32_t* qa_next = P.q[2 + ((it + 1) & 1)];
  uint32_t* cm_next = P.counts + 2 * (it + 1);
  uint32_t* ca_next = P.counts + 2 * (it + 1) + 1;
  const bool single = S->gp_mode == MUPSI_GP_SINGLE_REALIZATION;
  const v3 med_albedo = mk3(0.8f, 0.8f, 0.8f);  // Medium::default_bsdf_: Lambertian, albedo 0.8
  bool ovf = false;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t i = q[j];
    float4 o4 = P.o[i], d4 = P.d[i], t4 = P.thr[i], e4 = P.em[i];
    int4 meta = P.meta[i];
    int medium = __float_as_int(d4.w);
    uint64_t rng = ld_rng(P.rng[i]);
    v3 thr = mk3(t4.x, t4.y, t4.z), em = mk3(e4.x, e4.y, e4.z);
    Ray ray;
    ray.o = mk3(o4.x, o4.y, o4.z);
    ray.d = mk3(d4.x, d4.y, d4.z);
    ray.nt = o4.w;
    ray.ft = 3.402823466e+38f;
    int bounce = meta.w;
    bool has_hit = false, exited = true, dead = false;
    Cond cond = load_cond(P, i);
    if (medium >= 0) {
      float4 hb = P.hb[i];
      if (__float_as_uint(hb.w) == 0u) {
        // makeSurfaceEventFromMedium (medium.cpp:8-26) + handleVolume (trace.cpp:77-116)
        float4 ha = P.ha[i];
        v3 Pt = mk3(ha.y, ha.z, ha.w), N = mk3(hb.x, hb.y, hb.z), wo = -ray.d;
        LSample ls;
        if (choose_light(S, Pt, rng, ls)) {
          Ray sr = make_ray(Pt + N * S->eps, ls.d);
          float bias = ls.dist - S->eps * fabsf(dot(ls.d, N));
          sr.ft = bias * 0.99f;
          float tr = transmittance(S, medium, sr, medium_seed(S, meta.x, meta.y, meta.z, bounce), cond, ovf);
          v3 f = bsdf_weight(MUPSI_BSDF_LAMBERTIAN, med_albedo, ls.d, wo, N);
          em = em + (tr * cmul(thr, cmul(f, ls.weight))) * fabsf(dot(ls.d, N));
        }
        v3 w;
        v3 wi = bsdf_sample(MUPSI_BSDF_LAMBERTIAN, med_albedo, wo, N, rng, w);
        thr = cmul(thr, w);
        float surv = maxc(thr);
        if (pcg_next1d(rng) > surv) {
          dead = true;
        } else {
          thr = thr / surv;
          uint32_t ns = medium_seed(S, meta.x, meta.y, meta.z, bounce + 1);
          cond = sample_condition(S, S->media[medium], Pt, N, false, ns, !single, ovf);
          ray = make_ray(Pt + N * S->eps, wi);
          ray.nt = S->nearteps;
          bounce++;
          exited = false;
          has_hit = true;
        }
      }
    }
    if (!dead && exited) {
      Hit hi = scene_intersect(S, ray, ovf);
      if (hi.prim >= 0) {
        const DPrim& pr = S->prims[hi.prim];
        v3 wo = -ray.d, N = hi.Ng;
        LSample ls;
        if (choose_light(S, hi.p, rng, ls)) {  // handleSurface NEE (trace.cpp:40-56)
          Ray sr = make_ray(hi.p + N * S->eps, ls.d);
          float bias = ls.dist - S->eps * fabsf(dot(ls.d, N));
          sr.ft = bias * 0.99f;
          if (!scene_occluded(S, sr, ovf)) {
            v3 a = bsdf_weight(pr.bsdf, pr.albedo, ls.d, wo, N);
            em = em + cmul(thr, cmul(a, ls.weight)) * fabsf(dot(ls.d, N));
          }
        }
        v3 w;
        v3 wi = bsdf_sample(pr.bsdf, pr.albedo, wo, N, rng, w);
        if (pr.has_emission) em = em + cmul(thr, pr.emission * fmax_std(0.0f, dot(N, wi)));
        thr = cmul(thr, w);
        float surv = maxc(thr);
        if (pcg_next1d(rng) > surv) {
          dead = true;
        } else {
          thr = thr / surv;
          bool back = dot(wi, N) < 0.0f;
          medium = back ? pr.int_medium : pr.ext_medium;
          float bs = back ? -1.0f : 1.0f;
          ray = make_ray(hi.p + (bs * hi.Ng) * S->eps, wi);
          ray.nt = S->nearteps;
          bounce++;
          has_hit = true;
        }
      } else if (S->has_sky) {
        em = em + cmul(thr, S->sky);
      }
    }
    if (!dead && has_hit && bounce < S->max_bounce) {
      P.o[i] = make_float4(ray.o.x, ray.o.y, ray.o.z, ray.nt);
      P.d[i] = make_float4(ray.d.x, ray.d.y, ray.d.z, __int_as_float(medium));
      P.thr[i] = make_float4(thr.x, thr.y, thr.z, 0.0f);
      P.em[i] = make_float4(em.x, em.y, em.z, 0.0f);
      P.rng[i] = st_rng(rng);
      store_cond(P, i, cond);
      P.meta[i] = make_int4(meta.x, meta.y, meta.z, bounce);
      push(qa_next, ca_next, i);
      if (medium >= 0) push(qm_next, cm_next, i);
    } else {
      P.rad[3 * (int64_t)i] = em.x;
      P.rad[3 * (int64_t)i + 1] = em.y;
      P.rad[3 * (int64_t)i + 2] = em.z;
    }
  }
  if (ovf) atomicOr(S->err, ERR_BVH_STACK);
}

// Per-pixel running sum over the wave's passes in pass order (framebuffer.cpp:28-35),
// optional FP64 moments.
__global__ void k_accumulate(const float* __restrict__ rad, int passes, int64_t wh, float* __restrict__ sum,
                             double* __restrict__ moments) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < wh; p += (int64_t)gridDim.x * blockDim.x) {
    float s0 = sum[3 * p], s1 = sum[3 * p + 1], s2 = sum[3 * p + 2];
    double m[6] = {0, 0, 0, 0, 0, 0};
    for (int k = 0; k < passes; ++k) {
      const float* r = rad + 3 * ((int64_t)k * wh + p);
      float a = r[0], b = r[1], c = r[2];
      s0 += a;
      s1 += b;
      s2 += c;
      if (moments) {
        m[0] += a;
        m[1] += b;
        m[2] += c;
        m[3] += (double)a * a;
        m[4] += (double)b * b;
        m[5] += (double)c * c;
      }
    }
    sum[3 * p] = s0;
    sum[3 * p + 1] = s1;
    sum[3 * p + 2] = s2;
    if (moments)
      for (int c = 0; c < 6; ++c) moments[6 * p + c] += m[c];
  }
}

__global__ void k_average(const float* __restrict__ sum, int64_t n3, float inv, float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = sum[i] * inv;
}

// ---- batch kernels over a scene's medium ----
__global__ void k_mean(const DScene* S, int medium, int64_t n, const float* p, float* out) {
  bool ovf = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float4 r = mean_value_grad(S, S->media[medium], ld3(p + 3 * i), ovf);
    out[4 * i] = r.x;
    out[4 * i + 1] = r.y;
    out[4 * i + 2] = r.z;
    out[4 * i + 3] = r.w;
  }
  if (ovf) atomicOr(S->err, ERR_BVH_STACK);
}
__global__ void k_medium_eval(const DScene* S, int medium, int64_t n, const float* p, const uint32_t* seed,
                              const Cond* cond, float* out) {
  bool ovf = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Cond c;
    if (cond) {
      c = cond[i];
    } else {
      c.active = 0;
    }
    float4 r = medium_eval(S, S->media[medium], ld3(p + 3 * i), seed[i], c, ovf);
    out[4 * i] = r.x;
    out[4 * i + 1] = r.y;
    out[4 * i + 2] = r.z;
    out[4 * i + 3] = r.w;
  }
  if (ovf) atomicOr(S->err, ERR_BVH_STACK);
}
__global__ void k_sample_distance(const DScene* S, int medium, int64_t n, const mupsi_ray* rays, const uint32_t* seed,
                                  const Cond* cond, mupsi_medium_sample* out) {
  bool ovf = false;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Cond c;
    if (cond) {
      c = cond[i];
    } else {
      c.active = 0;
      c.C = mk3(0, 0, 0);
      c.u = 0;
      c.g = mk3(0, 0, 0);
    }
    const mupsi_ray& r = rays[i];
    March m;
    // Ray(origin, direction) normalises the direction (geometry/ray.h:12)
    march_begin(S, m, ld3(r.o), normalized(ld3(r.d)), r.near_t, r.far_t, medium, seed[i], c);
    march_full(S, m, ovf);
    mupsi_medium_sample res;
    march_result(S, m, res, ovf, single_lane());
    out[i] = res;
  }
  if (ovf) atomicOr(S->err, ERR_BVH_STACK);
}
__global__ void k_sample_condition(const DScene* S, int medium, int64_t n, const mupsi_medium_sample* smp,
                                   const uint32_t* seed, mupsi_cond* out) {
  bool ovf = false;
  const bool renewal = S->gp_mode == MUPSI_GP_RENEWAL_PLUS;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const mupsi_medium_sample& s = smp[i];
    Cond c = sample_condition(S, S->media[medium], ld3(s.p), ld3(s.normal), s.exited != 0, seed[i], renewal, ovf);
    mupsi_cond r;
    st3(r.C, c.C);
    r.u_tilde = c.u;
    st3(r.g_tilde, c.g);
    r.active = c.active;
    out[i] = r;
  }
  if (ovf) atomicOr(S->err, ERR_BVH_STACK);
}

}  // namespace mupsi

using namespace mupsi;

// ------------------------------------------------------------ scene handle
struct mupsi_scene {
  DScene h;                 // host copy (pointers are device pointers)
  DScene* d = nullptr;      // device copy
  std::vector<void*> allocs;
  int width = 0, height = 0, max_bounce = 0;
  // progressive framebuffer: running sum and passes so far
  float* sum = nullptr;
  int passes_done = 0;
  int next_pass = -1;  // pass after the last one accumulated
  // wave buffers (grow-only)
  Paths paths{};
  void* paths_mem = nullptr;
  size_t paths_bytes = 0;
  int64_t paths_cap = 0;
  int max_iters = 0;
  int* err = nullptr;
  unsigned long long* counters = nullptr;
  // profiling: per-launch event pairs, recorded while `profile` is set
  bool profile = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_march, ev_shade;
  size_t ev_used = 0;
  double march_ms = 0.0, shade_ms = 0.0;
  int64_t march_launches = 0, shade_launches = 0;
  // first profiled wave: queue sizes and march time per bounce iteration
  bool iter_pending = false, iter_done = false;
  std::vector<uint32_t> iter_counts;
  std::vector<float> iter_march_ms;
  cudaEvent_t next_event() {
    if (ev_used == ev_pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev_pool.push_back(e);
    }
    return ev_pool[ev_used++];
  }
  ~mupsi_scene();
};

namespace {

// Path-state buffers outlive their scenes in a small per-device pool, so a
// host that creates a scene per frame does not pay a cudaMalloc/cudaFree of a
// few hundred MB every time.
struct PoolEntry {
  int dev;
  void* ptr;
  size_t bytes;
};
std::mutex g_pool_mu;
std::vector<PoolEntry> g_pool;
constexpr size_t kPoolKeep = 4;

void* pool_take(size_t bytes, size_t* got) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_pool_mu);
  int best = -1;
  for (int i = 0; i < (int)g_pool.size(); ++i)
    if (g_pool[i].dev == dev && g_pool[i].bytes >= bytes && (best < 0 || g_pool[i].bytes < g_pool[best].bytes))
      best = i;
  if (best < 0) return nullptr;
  void* p = g_pool[best].ptr;
  *got = g_pool[best].bytes;
  g_pool.erase(g_pool.begin() + best);
  return p;
}
void pool_give(void* p, size_t bytes) {
  if (!p) return;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(g_pool_mu);
  g_pool.push_back({dev, p, bytes});
  while (g_pool.size() > kPoolKeep) {  // drop the smallest
    size_t k = 0;
    for (size_t i = 1; i < g_pool.size(); ++i)
      if (g_pool[i].bytes < g_pool[k].bytes) k = i;
    cudaFree(g_pool[k].ptr);
    g_pool.erase(g_pool.begin() + (long)k);
  }
}

}  // namespace

mupsi_scene::~mupsi_scene() {
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    for (void* p : allocs) cudaFree(p);
    if (d) cudaFree(d);
    if (sum) cudaFree(sum);
    if (paths_mem) pool_give(paths_mem, paths_bytes);
    if (err) cudaFree(err);
    if (counters) cudaFree(counters);
}

namespace {

bool desc_cacheable(const mupsi_scene_desc* desc) {
  for (int i = 0; i < desc->num_media; ++i)
    if (desc->media[i].kernel.points_per_cell > CACHE_MAX_PPC) return false;
  return true;
}

int build_scene(const mupsi_scene_desc* desc, mupsi_scene* s) {
  DScene& S = s->h;
  std::memset(&S, 0, sizeof S);
  if (desc->width <= 0 || desc->height <= 0) return fail(MUPSI_ERR_INVALID, "width/height must be positive");
  if ((int64_t)desc->width * desc->height > (1ll << 28)) return fail(MUPSI_ERR_INVALID, "image too large");
  if (desc->max_bounce < 0 || desc->max_bounce > 1024) return fail(MUPSI_ERR_INVALID, "max_bounce out of range");
  if (desc->num_primitives < 0 || desc->num_primitives > MAX_PRIMS)
    return fail(MUPSI_ERR_INVALID, "at most 16 primitives");
  if (desc->num_media < 0 || desc->num_media > MAX_MEDIA) return fail(MUPSI_ERR_INVALID, "at most 8 media");
  if (desc->num_meshes < 0 || desc->num_meshes > MAX_MESHES) return fail(MUPSI_ERR_INVALID, "at most 16 meshes");
  S.width = desc->width;
  S.height = desc->height;
  S.max_bounce = desc->max_bounce;
  S.gp_mode = desc->gp_mode;
  S.eps = desc->eps;
  S.nearteps = desc->nearteps;
  S.has_sky = desc->has_sky;
  S.sky = ld3(desc->sky);
  // Camera (camera.h:13-19)
  S.cpos = ld3(desc->cam_pos);
  S.cdir = normalized(ld3(desc->cam_dir));
  v3 up = normalized(ld3(desc->cam_up));
  S.cright = normalized(cross(S.cdir, up));
  S.cup = normalized(cross(S.cright, S.cdir));
  S.aspect = (float)desc->width / (float)desc->height;
  S.tan_half = std::tan(desc->cam_fov / 2.0f);  // fov taken as radians, as camera.cpp:10-11 does
  S.nmesh = desc->num_meshes;
  for (int i = 0; i < desc->num_meshes; ++i)
    if (int e = make_device_mesh(desc->meshes[i], S.meshes[i], s->allocs)) return e;
  S.nmed = desc->num_media;
  // lane groups share psi sums; a mesh mean's BVH queries would run on every
  // lane of a group, so scenes with mesh means start from single-lane marches
  // lane groups of >= 4 share psi sums and, when every medium has at most
  // CACHE_MAX_PPC impulses per cell, keep the impulse window in shared memory
  S.min_group = 4;
  S.sphere_only = 1;
  for (int i = 0; i < desc->num_media; ++i)
    if (desc->media[i].mean_type != MUPSI_MEAN_SPHERE) S.sphere_only = 0;
  // The shared-memory impulse cache measured slower than regenerating impulses
  // (the march is latency- rather than issue-bound); it stays selectable.
  S.cache = 0;
  if (const char* e = std::getenv("MUPSI_MARCH_CACHE")) S.cache = (std::atoi(e) != 0) && desc_cacheable(desc);
  for (int i = 0; i < desc->num_media; ++i) {
    const mupsi_medium_desc& m = desc->media[i];
    if (int e = check_kernel(&m.kernel)) return e;
    DMedium& dm = S.media[i];
    dm.mean_type = m.mean_type;
    dm.center = ld3(m.mean_center);
    dm.radius = m.mean_radius;
    dm.mesh = m.mean_mesh;
    dm.k = make_kparams(m.kernel);
    if (m.mean_type == MUPSI_MEAN_MESH && (m.mean_mesh < 0 || m.mean_mesh >= desc->num_meshes))
      return fail(MUPSI_ERR_INVALID, "medium mean_mesh out of range");
    dm.bs_c = mk3(0, 0, 0);
    dm.bs_r = INFINITY;
    if (m.mean_type == MUPSI_MEAN_MESH && desc->meshes[m.mean_mesh].num_vertices > 0) {
      // bounding sphere of the world-space vertices: centre of their box, radius
      // to the farthest vertex, in double with slack for the float comparisons
      const mupsi_mesh_desc& md = desc->meshes[m.mean_mesh];
      double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      auto world = [&](int64_t v, int a) { return (double)md.position[a] + (double)md.scale * md.vertices[3 * v + a]; };
      for (int64_t v = 0; v < md.num_vertices; ++v)
        for (int a = 0; a < 3; ++a) {
          lo[a] = std::min(lo[a], world(v, a));
          hi[a] = std::max(hi[a], world(v, a));
        }
      double c[3] = {(lo[0] + hi[0]) / 2, (lo[1] + hi[1]) / 2, (lo[2] + hi[2]) / 2}, r2 = 0.0;
      for (int64_t v = 0; v < md.num_vertices; ++v) {
        double d2 = 0.0;
        for (int a = 0; a < 3; ++a) d2 += (world(v, a) - c[a]) * (world(v, a) - c[a]);
        r2 = std::max(r2, d2);
      }
      dm.bs_c = mk3((float)c[0], (float)c[1], (float)c[2]);
      dm.bs_r = (float)(std::sqrt(r2) * (1.0 + 1e-5) + 1e-3 * (1.0 + std::fabs(c[0]) + std::fabs(c[1]) + std::fabs(c[2])));
    }
    if (m.mean_type != MUPSI_MEAN_MESH && m.mean_type != MUPSI_MEAN_SPHERE)
      return fail(MUPSI_ERR_INVALID, "unknown mean_type");
  }
  S.nprim = desc->num_primitives;
  for (int i = 0; i < desc->num_primitives; ++i) {
    const mupsi_primitive_desc& p = desc->primitives[i];
    DPrim& dp = S.prims[i];
    dp.type = p.type;
    dp.mesh = p.mesh;
    dp.bsdf = p.bsdf;
    dp.has_emission = p.has_emission;
    dp.albedo = ld3(p.albedo);
    dp.emission = ld3(p.emission);
    dp.int_medium = p.int_medium;
    dp.ext_medium = p.ext_medium;
    if (p.int_medium >= desc->num_media || p.ext_medium >= desc->num_media)
      return fail(MUPSI_ERR_INVALID, "primitive medium out of range");
    if (p.bsdf < 0 || p.bsdf > 2) return fail(MUPSI_ERR_INVALID, "unknown bsdf");
    HostM4 T;
    if (p.type == MUPSI_PRIM_SPHERE) {
      T = translate_scale(p.center, p.radius);
    } else if (p.type == MUPSI_PRIM_MESH) {
      if (p.mesh < 0 || p.mesh >= desc->num_meshes) return fail(MUPSI_ERR_INVALID, "primitive mesh out of range");
      T = translate_scale(desc->meshes[p.mesh].position, desc->meshes[p.mesh].scale);
    } else {
      return fail(MUPSI_ERR_INVALID, "unknown primitive type");
    }
    HostM4 Ti = inverse4(T);
    std::memcpy(dp.T.m, T.m, sizeof T.m);
    std::memcpy(dp.Tinv.m, Ti.m, sizeof Ti.m);
    dp.identity = is_identity4(Ti);
    if (p.has_emission) S.lights[S.nlights++] = i;
  }
  // march step table for the trace loop's medium rays: nearT = nearteps, farT = FLT_MAX
  {
    float nt = desc->nearteps, ft = 2000.0f;
    float dt = std::min(0.5f, (ft - nt) / 100.0f);
    std::vector<float> tab;
    float t = nt;
    while (t < ft && tab.size() < (1u << 20)) {
      tab.push_back(t);
      t += dt;
    }
    tab.push_back(t);
    const float* dtab = nullptr;
    void* p = nullptr;
    MUPSI_CUDA(cudaMalloc(&p, tab.size() * sizeof(float)));
    s->allocs.push_back(p);
    MUPSI_CUDA(cudaMemcpy(p, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice));
    dtab = (const float*)p;
    S.tab = dtab;
    S.tab_steps = (int)tab.size() - 1;
    S.tab_nt = nt;
    S.tab_ft = ft;
    S.tab_dt = dt;
  }
  MUPSI_CUDA(cudaMalloc(&s->err, sizeof(int)));
  MUPSI_CUDA(cudaMemset(s->err, 0, sizeof(int)));
  S.err = s->err;
  MUPSI_CUDA(cudaMalloc(&s->counters, 8 * sizeof(unsigned long long)));
  MUPSI_CUDA(cudaMemset(s->counters, 0, 8 * sizeof(unsigned long long)));
  S.counters = nullptr;
  MUPSI_CUDA(cudaMalloc(&s->d, sizeof(DScene)));
  MUPSI_CUDA(cudaMemcpy(s->d, &S, sizeof(DScene), cudaMemcpyHostToDevice));
  s->width = desc->width;
  s->height = desc->height;
  s->max_bounce = desc->max_bounce;
  MUPSI_CUDA(cudaMalloc(&s->sum, (size_t)3 * desc->width * desc->height * sizeof(float)));
  MUPSI_CUDA(cudaMemset(s->sum, 0, (size_t)3 * desc->width * desc->height * sizeof(float)));
  return MUPSI_OK;
}

// PathTracer::trace's do-while runs at least one bounce iteration
int wave_iters(const mupsi_scene* s) { return std::max(1, s->max_bounce); }

int ensure_paths(mupsi_scene* s, int64_t cap) {
  int iters = wave_iters(s) + 1;
  if (cap <= s->paths_cap && iters <= s->max_iters) return MUPSI_OK;
  if (s->paths_mem) {
    pool_give(s->paths_mem, s->paths_bytes);
    s->paths_mem = nullptr;
  }
  cap = std::max(cap, s->paths_cap);
  size_t bytes = 0;
  auto take = [&](size_t b) {
    size_t off = bytes;
    bytes += (b + 255) & ~(size_t)255;
    return off;
  };
  size_t o_o = take(cap * 16), o_d = take(cap * 16), o_t = take(cap * 16), o_e = take(cap * 16),
         o_r = take(cap * 8), o_ca = take(cap * 16), o_cb = take(cap * 16), o_m = take(cap * 16),
         o_ha = take(cap * 16), o_hb = take(cap * 16), o_rad = take(cap * 12), o_q0 = take(cap * 4),
         o_q1 = take(cap * 4), o_q2 = take(cap * 4), o_q3 = take(cap * 4), o_c = take((size_t)(iters + 1) * 8),
         o_cur = take((size_t)(iters + 1) * 4);
  size_t got = 0;
  char* base = static_cast<char*>(pool_take(bytes, &got));
  if (!base) {
    MUPSI_CUDA(cudaMalloc((void**)&base, bytes));
    got = bytes;
  }
  s->paths_mem = base;
  s->paths_bytes = got;
  Paths& P = s->paths;
  P.o = (float4*)(base + o_o);
  P.d = (float4*)(base + o_d);
  P.thr = (float4*)(base + o_t);
  P.em = (float4*)(base + o_e);
  P.rng = (uint2*)(base + o_r);
  P.ca = (float4*)(base + o_ca);
  P.cb = (float4*)(base + o_cb);
  P.meta = (int4*)(base + o_m);
  P.ha = (float4*)(base + o_ha);
  P.hb = (float4*)(base + o_hb);
  P.rad = (float*)(base + o_rad);
  P.q[0] = (uint32_t*)(base + o_q0);
  P.q[1] = (uint32_t*)(base + o_q1);
  P.q[2] = (uint32_t*)(base + o_q2);
  P.q[3] = (uint32_t*)(base + o_q3);
  P.counts = (uint32_t*)(base + o_c);
  P.cursors = (uint32_t*)(base + o_cur);
  P.cap = cap;
  s->paths_cap = cap;
  s->max_iters = iters;
  return MUPSI_OK;
}

// Persistent march grid: resident blocks per SM x SMs, for the cached (dynamic
// shared memory: one slot table per lane group of 4) or uncached kernel.
struct MarchLaunch {
  void (*fn)(const DScene*, Paths, int);
  int blocks;
  size_t smem;
};
// variant: bit 0 = impulse cache, bit 1 = sphere means only
MarchLaunch march_launch(bool cache, bool sphere_only) {
  static MarchLaunch ml[4] = {};
  const int v = (cache ? 1 : 0) | (sphere_only ? 2 : 0);
  MarchLaunch& m = ml[v];
  if (!m.blocks) {
    switch (v) {
      case 0: m.fn = k_march<false, MEAN_ANY>; break;
      case 1: m.fn = k_march<true, MEAN_ANY>; break;
      case 2: m.fn = k_march<false, MEAN_SPHERE_ONLY>; break;
      default: m.fn = k_march<true, MEAN_SPHERE_ONLY>; break;
    }
    m.smem = cache ? (size_t)(128 / 4) * kCacheBytes : 0;
    if (cache) cudaFuncSetAttribute(m.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m.smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, m.fn, 128, m.smem);
    m.blocks = std::max(1, per_sm) * num_sms();
  }
  return m;
}
void launch_march(const MarchLaunch& ml, const DScene* d, const Paths& P, int it, cudaStream_t st) {
  ml.fn<<<ml.blocks, 128, ml.smem, st>>>(d, P, it);
}

// One wave: n paths, from pass0 (or explicit x/y/k arrays). Leaves radiance in P.rad.
int run_wave(mupsi_scene* s, int64_t n, int pass0, const int32_t* xs, const int32_t* ys, const int32_t* ks,
             cudaStream_t st) {
  Paths& P = s->paths;
  const int iters = wave_iters(s);
  MUPSI_CUDA(cudaMemsetAsync(P.counts, 0, (size_t)(s->max_iters + 1) * 8, st));
  MUPSI_CUDA(cudaMemsetAsync(P.cursors, 0, (size_t)(s->max_iters + 1) * 4, st));
  count_launch(2);
  int gb = (int)std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 16);
  k_raygen<<<gb, 256, 0, st>>>(s->d, P, n, pass0, xs, ys, ks);
  count_launch();
  const MarchLaunch ml = march_launch(s->h.cache != 0, s->h.sphere_only != 0);
  int sb = (int)std::min<int64_t>((n + 127) / 128, (int64_t)num_sms() * 16);
  for (int it = 0; it < iters; ++it) {
    if (s->profile) {
      cudaEvent_t a = s->next_event(), b = s->next_event(), c = s->next_event();
      cudaEventRecord(a, st);
      launch_march(ml, s->d, P, it, st);
      cudaEventRecord(b, st);
      k_shade<<<sb, 128, 0, st>>>(s->d, P, it);
      cudaEventRecord(c, st);
      s->ev_march.push_back({a, b});
      s->ev_shade.push_back({b, c});
    } else {
      launch_march(ml, s->d, P, it, st);
      k_shade<<<sb, 128, 0, st>>>(s->d, P, it);
    }
    count_launch(2);
  }
  MUPSI_CUDA(cudaGetLastError());
  return MUPSI_OK;
}

void collect_events(mupsi_scene* s) {
  bool first = s->iter_pending && !s->iter_done;
  for (auto& pr : s->ev_march) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, pr.first, pr.second);
    s->march_ms += ms;
    s->march_launches++;
    if (first && (int)s->iter_march_ms.size() < s->max_iters) s->iter_march_ms.push_back(ms);
  }
  if (first && !s->ev_march.empty()) {
    s->iter_counts.resize(2 * (size_t)(s->max_iters + 1));
    cudaMemcpy(s->iter_counts.data(), s->paths.counts, s->iter_counts.size() * 4, cudaMemcpyDeviceToHost);
    s->iter_done = true;
  }
  for (auto& pr : s->ev_shade) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, pr.first, pr.second);
    s->shade_ms += ms;
    s->shade_launches++;
  }
  s->ev_march.clear();
  s->ev_shade.clear();
  s->ev_used = 0;
}

int check_err(mupsi_scene* s, cudaStream_t st) {
  int h = 0;
  MUPSI_CUDA(cudaMemcpyAsync(&h, s->err, sizeof(int), cudaMemcpyDeviceToHost, st));
  MUPSI_CUDA(cudaStreamSynchronize(st));
  collect_events(s);
  if (h) {
    cudaMemsetAsync(s->err, 0, sizeof(int), st);
    if (h & ERR_BVH_STACK) return fail(MUPSI_ERR_DEVICE_LIMIT, "BVH traversal exceeded the 64-entry stack");
    return fail(MUPSI_ERR_DEVICE_LIMIT, "march iteration cap reached");
  }
  return MUPSI_OK;
}

int grid_n(int64_t n) { return (int)std::min<int64_t>((n + 127) / 128, (int64_t)num_sms() * 32); }

const int64_t kDefaultWavePaths = 8ll << 20;

// ---------------------------------------------------------------------------
// Allocation-free trace (mupsi_gpu_trace_samples_noalloc). Some hosts cannot
// call cudaMalloc while they render: a render thread that must not block on
// the device-wide synchronisation cudaMalloc/cudaFree can imply, or a host that
// owns the GPU's memory budget through its own allocator. For them the wave's
// path state lives in one fixed device array, sized for kNoAllocMaxSamples
// samples per call and held by every GPU that loads this library until the
// process exits. Calls share the array: counters are cleared at the start of
// each call, and two calls that overlap on the GPU (different streams or host
// threads) race on it.
constexpr int64_t kNoAllocMaxSamples = 16384;
constexpr int kNoAllocMaxIters = 1025;  // max_bounce <= 1024, plus one
constexpr size_t na_align(size_t b) { return (b + 255) & ~(size_t)255; }
constexpr size_t kNoAllocBytes =
    10 * na_align(kNoAllocMaxSamples * 16) + na_align(kNoAllocMaxSamples * 8) + na_align(kNoAllocMaxSamples * 12) +
    4 * na_align(kNoAllocMaxSamples * 4) + na_align((size_t)(kNoAllocMaxIters + 1) * 8) +
    na_align((size_t)(kNoAllocMaxIters + 1) * 4);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[256] = {};

// Device address of the scratch array on the current device, looked up once per
// device (the first call on a device does this set-up).
int noalloc_scratch(void** out) {
  int dev = 0;
  MUPSI_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) return fail(MUPSI_ERR_UNSUPPORTED, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return fail(MUPSI_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return MUPSI_OK;
}

// Path-state view over the scratch array (same layout as ensure_paths).
Paths noalloc_paths(void* base_ptr) {
  char* base = static_cast<char*>(base_ptr);
  size_t off = 0;
  auto take = [&](size_t b) {
    char* p = base + off;
    off += na_align(b);
    return p;
  };
  const int64_t cap = kNoAllocMaxSamples;
  Paths P;
  P.o = (float4*)take(cap * 16);
  P.d = (float4*)take(cap * 16);
  P.thr = (float4*)take(cap * 16);
  P.em = (float4*)take(cap * 16);
  P.rng = (uint2*)take(cap * 8);
  P.ca = (float4*)take(cap * 16);
  P.cb = (float4*)take(cap * 16);
  P.meta = (int4*)take(cap * 16);
  P.ha = (float4*)take(cap * 16);
  P.hb = (float4*)take(cap * 16);
  P.rad = (float*)take(cap * 12);
  for (int i = 0; i < 4; ++i) P.q[i] = (uint32_t*)take(cap * 4);
  P.counts = (uint32_t*)take((size_t)(kNoAllocMaxIters + 1) * 8);
  P.cursors = (uint32_t*)take((size_t)(kNoAllocMaxIters + 1) * 4);
  P.cap = cap;
  return P;
}

}  // namespace

extern "C" {

int mupsi_gpu_scene_create(const mupsi_scene_desc* desc, mupsi_scene** out) {
  clear_error();
  if (!desc || !out) return fail(MUPSI_ERR_INVALID, "null argument");
  auto* s = new mupsi_scene();
  int e = build_scene(desc, s);
  if (e) {
    delete s;
    return e;
  }
  *out = s;
  return MUPSI_OK;
}

void mupsi_gpu_scene_destroy(mupsi_scene* scene) {
  if (scene) cudaDeviceSynchronize();
  delete scene;
}

int mupsi_gpu_mean(const mupsi_scene* scene, int32_t medium, int64_t n, const float* p, float* out, mupsi_mem mem,
                   void* stream) {
  clear_error();
  if (!scene || medium < 0 || medium >= scene->h.nmed || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!p || !out) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<float> dp(st), dout(st);
  MUPSI_CUDA(dp.in(p, 3 * n, mem));
  MUPSI_CUDA(dout.out(out, 4 * n, mem));
  k_mean<<<grid_n(n), 128, 0, st>>>(scene->d, medium, n, dp.ptr, dout.ptr);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dout.finish());
  return check_err(const_cast<mupsi_scene*>(scene), st);
}

int mupsi_gpu_medium_eval(const mupsi_scene* scene, int32_t medium, int64_t n, const float* p, const uint32_t* seed,
                          const mupsi_cond* cond, float* out, mupsi_mem mem, void* stream) {
  clear_error();
  if (!scene || medium < 0 || medium >= scene->h.nmed || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!p || !seed || !out) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<float> dp(st), dout(st);
  Staged<uint32_t> ds(st);
  Staged<mupsi_cond> dc(st);
  MUPSI_CUDA(dp.in(p, 3 * n, mem));
  MUPSI_CUDA(ds.in(seed, n, mem));
  if (cond) MUPSI_CUDA(dc.in(cond, n, mem));
  MUPSI_CUDA(dout.out(out, 4 * n, mem));
  k_medium_eval<<<grid_n(n), 128, 0, st>>>(scene->d, medium, n, dp.ptr, ds.ptr,
                                           cond ? reinterpret_cast<const Cond*>(dc.ptr) : nullptr, dout.ptr);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dout.finish());
  return check_err(const_cast<mupsi_scene*>(scene), st);
}

int mupsi_gpu_sample_distance(const mupsi_scene* scene, int32_t medium, int64_t n, const mupsi_ray* rays,
                              const uint32_t* seed, const mupsi_cond* cond, mupsi_medium_sample* out, mupsi_mem mem,
                              void* stream) {
  clear_error();
  if (!scene || medium < 0 || medium >= scene->h.nmed || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!rays || !seed || !out) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<mupsi_ray> dr(st);
  Staged<uint32_t> ds(st);
  Staged<mupsi_cond> dc(st);
  Staged<mupsi_medium_sample> dout(st);
  MUPSI_CUDA(dr.in(rays, n, mem));
  MUPSI_CUDA(ds.in(seed, n, mem));
  if (cond) MUPSI_CUDA(dc.in(cond, n, mem));
  MUPSI_CUDA(dout.out(out, n, mem));
  k_sample_distance<<<grid_n(n), 128, 0, st>>>(scene->d, medium, n, dr.ptr, ds.ptr,
                                               cond ? reinterpret_cast<const Cond*>(dc.ptr) : nullptr, dout.ptr);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dout.finish());
  return check_err(const_cast<mupsi_scene*>(scene), st);
}

int mupsi_gpu_sample_condition(const mupsi_scene* scene, int32_t medium, int64_t n, const mupsi_medium_sample* samples,
                               const uint32_t* seed, mupsi_cond* out, mupsi_mem mem, void* stream) {
  clear_error();
  if (!scene || medium < 0 || medium >= scene->h.nmed || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!samples || !seed || !out) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<mupsi_medium_sample> dsm(st);
  Staged<uint32_t> ds(st);
  Staged<mupsi_cond> dout(st);
  MUPSI_CUDA(dsm.in(samples, n, mem));
  MUPSI_CUDA(ds.in(seed, n, mem));
  MUPSI_CUDA(dout.out(out, n, mem));
  k_sample_condition<<<grid_n(n), 128, 0, st>>>(scene->d, medium, n, dsm.ptr, ds.ptr, dout.ptr);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dout.finish());
  return check_err(const_cast<mupsi_scene*>(scene), st);
}

int mupsi_gpu_trace_samples(mupsi_scene* scene, int64_t n, const int32_t* x, const int32_t* y, const int32_t* k,
                            float* out_rgb, mupsi_mem mem, void* stream) {
  clear_error();
  if (!scene || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!x || !y || !k || !out_rgb) return fail(MUPSI_ERR_INVALID, "null buffer");
  if (n > kDefaultWavePaths * 4) return fail(MUPSI_ERR_INVALID, "too many samples in one call");
  cudaStream_t st = resolve_stream(stream);
  if (int e = ensure_paths(scene, n)) return e;
  Staged<int32_t> dx(st), dy(st), dk(st);
  MUPSI_CUDA(dx.in(x, n, mem));
  MUPSI_CUDA(dy.in(y, n, mem));
  MUPSI_CUDA(dk.in(k, n, mem));
  if (int e = run_wave(scene, n, 0, dx.ptr, dy.ptr, dk.ptr, st)) return e;
  if (mem == MUPSI_MEM_DEVICE) {
    MUPSI_CUDA(cudaMemcpyAsync(out_rgb, scene->paths.rad, n * 12, cudaMemcpyDeviceToDevice, st));
  } else {
    MUPSI_CUDA(cudaMemcpyAsync(out_rgb, scene->paths.rad, n * 12, cudaMemcpyDeviceToHost, st));
  }
  return check_err(scene, st);
}

int mupsi_gpu_render(mupsi_scene* scene, const mupsi_render_args* a) {
  clear_error();
  if (!scene || !a) return fail(MUPSI_ERR_INVALID, "null argument");
  if (a->spp_begin < 0 || a->spp_end < a->spp_begin) return fail(MUPSI_ERR_INVALID, "bad pass range");
  cudaStream_t st = resolve_stream(a->stream);
  const int64_t wh = (int64_t)scene->width * scene->height;
  // a call that does not start where the previous one ended starts a new image
  if (a->spp_begin == 0 || a->spp_begin != scene->next_pass) {
    MUPSI_CUDA(cudaMemsetAsync(scene->sum, 0, wh * 12, st));
    scene->passes_done = 0;
  }
  double* dmom = nullptr;
  if (a->moments_out) {
    MUPSI_CUDA(cudaMallocAsync((void**)&dmom, wh * 6 * sizeof(double), st));
    MUPSI_CUDA(cudaMemsetAsync(dmom, 0, wh * 6 * sizeof(double), st));
  }
  int total = a->spp_end - a->spp_begin;
  int per_wave = (int)std::max<int64_t>(1, std::min<int64_t>(total, kDefaultWavePaths / wh));
  if (total > 0) {
    if (int e = ensure_paths(scene, (int64_t)per_wave * wh)) return e;
  }
  int rc = MUPSI_OK;
  for (int k0 = a->spp_begin; k0 < a->spp_end; k0 += per_wave) {
    if (a->cancel && *a->cancel) {
      rc = fail(MUPSI_ERR_CANCELLED, "render cancelled");
      break;
    }
    int passes = std::min(per_wave, a->spp_end - k0);
    if ((rc = run_wave(scene, (int64_t)passes * wh, k0, nullptr, nullptr, nullptr, st))) break;
    k_accumulate<<<grid_n(wh), 128, 0, st>>>(scene->paths.rad, passes, wh, scene->sum, dmom);
    count_launch();
    scene->passes_done += passes;
    scene->next_pass = k0 + passes;
    if (a->on_spp) {
      cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) {
        rc = fail(MUPSI_ERR_CUDA, cudaGetErrorString(e));
        break;
      }
      a->on_spp(k0 + passes, a->user);
    }
  }
  if (rc == MUPSI_OK && a->rgb_out && scene->passes_done > 0) {
    float inv = 1.0f / (float)scene->passes_done;
    if (a->out_mem == MUPSI_MEM_DEVICE) {
      k_average<<<grid_n(wh * 3), 128, 0, st>>>(scene->sum, wh * 3, inv, a->rgb_out);
      count_launch();
    } else {
      float* tmp = nullptr;
      MUPSI_CUDA(cudaMallocAsync((void**)&tmp, wh * 12, st));
      k_average<<<grid_n(wh * 3), 128, 0, st>>>(scene->sum, wh * 3, inv, tmp);
      count_launch();
      MUPSI_CUDA(cudaMemcpyAsync(a->rgb_out, tmp, wh * 12, cudaMemcpyDeviceToHost, st));
      MUPSI_CUDA(cudaFreeAsync(tmp, st));
    }
  }
  if (dmom) {
    if (rc == MUPSI_OK) MUPSI_CUDA(cudaMemcpyAsync(a->moments_out, dmom, wh * 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
    MUPSI_CUDA(cudaFreeAsync(dmom, st));
  }
  int e = check_err(scene, st);
  return rc ? rc : e;
}

// Allocation-free variant of mupsi_gpu_trace_samples (no counterpart in the
// reference): same kernels and results, path state in the library's static
// scratch array, device buffers only, at most kNoAllocMaxSamples samples.
int mupsi_gpu_trace_samples_noalloc(mupsi_scene* scene, int64_t n, const int32_t* x, const int32_t* y,
                                    const int32_t* k, float* out_rgb, void* stream) {
  clear_error();
  if (!scene || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n > kNoAllocMaxSamples)
    return fail(MUPSI_ERR_INVALID, "trace_samples_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                                       std::to_string(kNoAllocMaxSamples) + " samples per call");
  if (n == 0) return MUPSI_OK;
  if (!x || !y || !k || !out_rgb) return fail(MUPSI_ERR_INVALID, "null buffer");
  for (const void* ptr : {(const void*)x, (const void*)y, (const void*)k, (const void*)out_rgb}) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess || at.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      return fail(MUPSI_ERR_INVALID, "trace_samples_noalloc takes device buffers only");
    }
  }
  void* scratch = nullptr;
  if (int e = noalloc_scratch(&scratch)) return e;
  cudaStream_t st = (cudaStream_t)stream;  // NULL: the default stream (no stream is created here)
  Paths P = noalloc_paths(scratch);
  const int iters = std::max(1, scene->max_bounce);
  // the array keeps the previous call's contents: clear the queue counters and cursors
  MUPSI_CUDA(cudaMemsetAsync(P.counts, 0, (size_t)(iters + 1) * 8, st));
  MUPSI_CUDA(cudaMemsetAsync(P.cursors, 0, (size_t)(iters + 1) * 4, st));
  int gb = (int)std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 16);
  k_raygen<<<gb, 256, 0, st>>>(scene->d, P, n, 0, x, y, k);
  const MarchLaunch ml = march_launch(scene->h.cache != 0, scene->h.sphere_only != 0);
  int sb = (int)std::min<int64_t>((n + 127) / 128, (int64_t)num_sms() * 16);
  for (int it = 0; it < iters; ++it) {
    launch_march(ml, scene->d, P, it, st);
    k_shade<<<sb, 128, 0, st>>>(scene->d, P, it);
  }
  count_launch(1 + 2 * iters);
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(cudaMemcpyAsync(out_rgb, P.rad, n * 12, cudaMemcpyDeviceToDevice, st));
  return check_err(scene, st);
}

int mupsi_gpu_scene_profile(mupsi_scene* scene, int32_t enable) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  MUPSI_CUDA(cudaDeviceSynchronize());
  collect_events(scene);
  scene->profile = enable != 0;
  scene->iter_pending = enable != 0;
  scene->iter_done = false;
  scene->iter_counts.clear();
  scene->iter_march_ms.clear();
  scene->h.counters = enable ? scene->counters : nullptr;
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_scene_stats(mupsi_scene* scene, mupsi_render_stats* out, int32_t reset) {
  clear_error();
  if (!scene || !out) return fail(MUPSI_ERR_INVALID, "null argument");
  MUPSI_CUDA(cudaDeviceSynchronize());
  collect_events(scene);
  unsigned long long c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  MUPSI_CUDA(cudaMemcpy(c, scene->counters, sizeof c, cudaMemcpyDeviceToHost));
  out->march_steps = c[0];
  out->psi_evals = c[1];
  out->marches = c[2];
  out->impulse_evals = c[3];
  out->mean_evals = c[4];
  out->parity_casts = c[5];
  out->march_ms = scene->march_ms;
  out->shade_ms = scene->shade_ms;
  out->march_launches = scene->march_launches;
  out->shade_launches = scene->shade_launches;
  for (int i = 0; i < 16; ++i) {
    out->iter_medium[i] = 2 * i < (int)scene->iter_counts.size() ? scene->iter_counts[2 * i] : 0;
    out->iter_live[i] = 2 * i + 1 < (int)scene->iter_counts.size() ? scene->iter_counts[2 * i + 1] : 0;
    out->iter_march_ms[i] = i < (int)scene->iter_march_ms.size() ? scene->iter_march_ms[i] : 0.0f;
  }
  if (reset) {
    MUPSI_CUDA(cudaMemset(scene->counters, 0, sizeof c));
    scene->march_ms = scene->shade_ms = 0.0;
    scene->march_launches = scene->shade_launches = 0;
  }
  return MUPSI_OK;
}

}  // extern "C"
