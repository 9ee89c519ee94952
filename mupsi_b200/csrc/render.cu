// Scenes, the GP-medium batch entry points and the wavefront path tracer
// (PathTracer::trace, rendering/trace.cpp:118-213, driven like
// Renderer::startRenderProgressive, rendering/renderer.cpp:22-49).
//
// Wavefront layout: a wave holds W*H*passes paths in structure-of-arrays state.
// Each bounce iteration runs two kernels:
//   k_march  - persistent warps march every path that is inside a GP medium;
//              idle lanes pull the next path from the medium queue, so long and
//              short marches never stall a warp; (scenes with an SDF or
//              external GP medium add k_march_field, which sphere traces those
//              paths, one thread each)
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
  // surrogate rounds (rounds > 1): a march suspended for a prediction keeps its
  // state here, its request goes to req[round & 1] and the network's answer to
  // pred[round & 1]; the next round resumes it
  int rounds;
  float4* ms0;          // t, step index (int bits), f at the origin, flags | requests << 8
  float4* ms1;          // mu_j, mu_hi, t_j, -
  float4* req[2];       // point xyz, path index (uint bits)
  float* pred[2];
  uint32_t* rcounts;    // [it * rounds + r]: requests made in round r
  uint32_t* rcursors;   // [it * rounds + r]: work cursor of round r >= 1
  // deferred shadow rays (sh_a null: transmittance is marched inline in the
  // shading kernel): the NEE of a medium event at iteration it leaves a job at
  // its path's slot, queued in sq[(it + 1) & 1]; the march launch of iteration
  // it + 1 marches it and adds the term
  float4* sh_a;         // origin xyz, far_t
  float4* sh_b;         // direction xyz, medium (int bits)
  float4* sh_x;         // X = thr * f * light weight (xyz), c = |cos| (w): the term is (tr * X) * c
  float4* sh_ca;        // the conditioning at the event (C xyz, u)
  float4* sh_cb;        //   (g xyz, active)
  int4* sh_m;           // x: 1 = add to the final radiance (the path ended there), 0 = to its emission; y: seed
  uint32_t* sq[2];
  uint32_t* scounts;    // [it]: jobs for the march launch of iteration it
  uint32_t* scursors;
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

// The NEE term of shadow job `idx` with transmittance tr, added where the path
// stands: its final radiance if it ended at the event, else its emission.
MD void add_shadow_term(const Paths& P, uint32_t idx, float tr) {
  const float4 x = P.sh_x[idx];
  const float tx = (tr * x.x) * x.w, ty = (tr * x.y) * x.w, tz = (tr * x.z) * x.w;
  if (P.sh_m[idx].x) {
    float* r = P.rad + 3 * (int64_t)idx;
    r[0] = r[0] + tx;
    r[1] = r[1] + ty;
    r[2] = r[2] + tz;
  } else {
    const float4 e = P.em[idx];
    P.em[idx] = make_float4(e.x + tx, e.y + ty, e.z + tz, e.w);
  }
}


// ConstantSampler seed of bounce b's medium sampler (trace.cpp:146-147)
MD uint32_t medium_seed(const DScene* S, int x, int y, int k, int b) {
  uint32_t s = S->gp_mode == MUPSI_GP_SINGLE_REALIZATION
                   ? TRACE_SEED
                   : make_seed5((uint32_t)x, (uint32_t)y, (uint32_t)k, TRACE_SEED, (uint32_t)b);
  return constant_sampler_i(s);
}

// meta.w packs the bounce count (11 bits; max_bounce <= 1024) and the path's
// scene instance (a wave may hold paths of many scenes).
MD int meta_bounce(int w) { return w & 2047; }
MD int meta_inst(int w) { return w >> 11; }
MD int pack_meta(int bounce, int inst) { return bounce | (inst << 11); }

// A wave is a list of chunks: `passes` consecutive passes of one scene
// instance, stored at path indices [path0, path0 + passes * width * height);
// the chunk's pixels are [pix0, pix0 + wh) of the wave's accumulation range.
struct WaveChunk {
  int inst, pass0, passes, width;
  int64_t path0, wh, pix0;
};
// One wave of a device-resident wave plan: its paths, accumulated pixels and
// chunk range.
struct WaveDesc {
  int64_t n, npix;
  int chunk0, nchunks;
};
// Where a wave's paths come from: explicit (x, y, k) arrays, a chunk table, or
// (wave_idx != null) wave *wave_idx of a device wave plan, which lets one
// captured graph replay every wave of a plan.
struct WaveSrc {
  int64_t n = 0;
  const WaveChunk* chunks = nullptr;
  int nchunks = 0;
  const int32_t *xs = nullptr, *ys = nullptr, *ks = nullptr;
  const WaveDesc* waves = nullptr;
  const int* wave_idx = nullptr;
};
MD void resolve_wave(const WaveSrc& src, int64_t& n, int64_t& npix, const WaveChunk*& chunks, int& nchunks) {
  n = src.n;
  npix = 0;
  chunks = src.chunks;
  nchunks = src.nchunks;
  if (src.wave_idx) {
    const WaveDesc wd = src.waves[*src.wave_idx];
    n = wd.n;
    npix = wd.npix;
    chunks = src.chunks + wd.chunk0;
    nchunks = wd.nchunks;
  }
}
// last chunk whose start (member `start`) is <= i
template <typename F>
MD int find_chunk(const WaveChunk* chunks, int nchunks, int64_t i, F start) {
  int lo = 0, hi = nchunks - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (start(chunks[mid]) <= i)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------------ kernels
// Start of a wave: clear the queue counters and cursors of `iters` bounce
// iterations and step the plan's wave index.
__global__ void k_wave_begin(Paths P, int iters, int* wave_idx) {
  for (int i = threadIdx.x; i < 2 * (iters + 1); i += blockDim.x) P.counts[i] = 0;
  for (int i = threadIdx.x; i < iters + 1; i += blockDim.x) P.cursors[i] = 0;
  if (P.rounds > 1)
    for (int i = threadIdx.x; i < iters * P.rounds; i += blockDim.x) {
      P.rcounts[i] = 0;
      P.rcursors[i] = 0;
    }
  if (P.scounts)
    for (int i = threadIdx.x; i < iters + 1; i += blockDim.x) {
      P.scounts[i] = 0;
      P.scursors[i] = 0;
    }
  if (wave_idx && threadIdx.x == 0) *wave_idx += 1;
}

__global__ void k_raygen(const DScene* const* __restrict__ scenes, Paths P, WaveSrc src) {
  int64_t n, npix;
  const WaveChunk* chunks;
  int nchunks;
  resolve_wave(src, n, npix, chunks, nchunks);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int x, y, k, inst = 0;
    if (src.xs) {
      x = src.xs[i];
      y = src.ys[i];
      k = src.ks[i];
    } else {
      const WaveChunk& c = chunks[find_chunk(chunks, nchunks, i, [](const WaveChunk& w) { return w.path0; })];
      int64_t local = i - c.path0;
      int64_t pix = local % c.wh;
      inst = c.inst;
      k = c.pass0 + (int)(local / c.wh);
      x = (int)(pix % c.width);
      y = (int)(pix / c.width);
    }
    const DScene* S = scenes[inst];
    uint64_t rng = pcg_seeded(make_seed4((uint32_t)x, (uint32_t)y, (uint32_t)k, TRACE_SEED));
    Ray r = camera_ray(S, x, y);
    P.o[i] = make_float4(r.o.x, r.o.y, r.o.z, r.nt);
    P.d[i] = make_float4(r.d.x, r.d.y, r.d.z, __int_as_float(-1));
    P.thr[i] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    P.em[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    P.rng[i] = st_rng(rng);
    P.ca[i] = make_float4(0, 0, 0, 0);
    P.cb[i] = make_float4(0, 0, 0, __uint_as_float(0u));
    P.meta[i] = make_int4(x, y, k, pack_meta(0, inst));
    P.q[2][i] = (uint32_t)i;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.counts[0] = 0;
    P.counts[1] = (uint32_t)n;
  }
}

// Launch-wide settings of the march and shade kernels.
struct WaveCfg {
  int defer;                     // shading leaves GP-medium shadow rays as jobs for the next march launch
  int shadow_pass;               // this march launch marches the shadow jobs of iteration `it`
  int min_group;                 // smallest lane group per march
  int block_rays;                // block-per-ray marches while n <= block_rays * blocks (sphere means)
  int lane_rays;                 // > 0: one ray per lane for long sphere-mean queues (march_lanes), this
                                 // many visited steps per ray between the warp's psi rounds
  int mu_batch = 0;              // > 0: one-ray-per-lane mesh marches leave their BVH queries until this
                                 // many of a warp's marches wait for one (or all of them do)
  int* err;                      // device error word (ERR_* bits)
  unsigned long long* counters;  // nullable work counters
};

// Short queues of sphere-mean marches (the late bounces): one ray per block.
// Which steps of such a march need psi is settled without psi (the mean and
// the per-point bound decide every step, and a psi step without a hit moves
// the march on by exactly one step), so the block scans ahead for the next
// 2 x warps of them, each half-warp evaluates psi at one (the 16-slot sum
// order is the same for any group, so these are the values the one-group
// march computes), and the first sign change in step order is the hit. The
// origin, whose psi fixes the sign every step is compared with, goes first
// alone. Bounded by the march's own step and guard limits.
// Window positions below `stop` in warp w's lanes.
__device__ __forceinline__ unsigned below(int stop, int w) {
  const int b = stop - 32 * w;
  return b >= 32 ? 0xffffffffu : (b <= 0 ? 0u : ((1u << b) - 1u));
}
// Window position of the r-th (from 0) step needing psi below `stop`.
__device__ __forceinline__ int nth_need(const unsigned* need, int nw, int stop, int r) {
  for (int w = 0; w < nw; ++w) {
    unsigned msk = need[w] & below(stop, w);
    const int c = __popc(msk);
    if (r < c) {
      for (int i = 0; i < r; ++i) msk &= msk - 1u;
      return 32 * w + __ffs(msk) - 1;
    }
    r -= c;
  }
  return 0;  // not reached: r < the count of such steps
}

// SH: the rays are shadow jobs (GPMedium::transmittance: the result is the
// NEE term added where the path stands).
template <bool SH>
__device__ void march_block_rays(const DScene* const* __restrict__ scenes, Paths& P, uint32_t n,
                                 const uint32_t* __restrict__ q, uint32_t* cursor, const WaveCfg& cfg) {
  constexpr int kMaxWarps = 4, kWindow = 32 * kMaxWarps;
  __shared__ uint32_t s_j;
  __shared__ float s_tw[kWindow], s_mw[kWindow];
  __shared__ int s_cls[kWindow];
  __shared__ int s_hit[2 * kMaxWarps];
  __shared__ unsigned s_need[kMaxWarps], s_end[kMaxWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = min(kMaxWarps, (int)(blockDim.x >> 5));
  const int W = 32 * nw;  // window of steps classified per round
  const int ncand_max = 2 * nw;
  const int cand = 2 * warp + (lane >> 4);  // the candidate this half-warp evaluates
  Group half;
  half.G = 16;
  half.sub = lane & 15;
  half.mask = (lane >> 4) ? 0xffff0000u : 0x0000ffffu;
  Group full;
  full.G = 32;
  full.sub = lane;
  full.mask = 0xffffffffu;
  bool ovf = false;
  unsigned long long steps = 0, psis = 0, marches = 0, imps = 0;
  for (;;) {
    __syncthreads();  // every thread has read the previous s_j
    if (threadIdx.x == 0) s_j = atomicAdd(cursor, 1u);
    __syncthreads();
    const uint32_t j = s_j;
    if (j >= n) break;
    const uint32_t idx = q[j];
    const int4 meta = P.meta[idx];
    const DScene* S = scenes[meta_inst(meta.w)];
    March m;
    if constexpr (SH) {  // the job's shadow ray, medium, seed and conditioning
      const float4 a = P.sh_a[idx], b = P.sh_b[idx], ca = P.sh_ca[idx], cb = P.sh_cb[idx];
      const int med = __float_as_int(b.w);
      if (S->media[med].kind != MUPSI_MEDIUM_GP) continue;  // k_march_field's shadow pass
      Cond c;
      c.C = mk3(ca.x, ca.y, ca.z);
      c.u = ca.w;
      c.g = mk3(cb.x, cb.y, cb.z);
      c.active = __float_as_uint(cb.w);
      march_begin(S, m, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), 0.0f, a.w, med, (uint32_t)P.sh_m[idx].y, c);
    } else {
      const float4 o = P.o[idx], d = P.d[idx];
      const int med = __float_as_int(d.w);
      if (S->media[med].kind != MUPSI_MEDIUM_GP) continue;  // k_march_field marches it
      march_begin(S, m, mk3(o.x, o.y, o.z), mk3(d.x, d.y, d.z), o.w, 3.402823466e+38f, med,
                  medium_seed(S, meta.x, meta.y, meta.z, meta_bounce(meta.w)), load_cond(P, idx));
    }
    const DMedium& md = S->media[m.medium];
    m.may_request = false;
    marches++;
    {  // the origin (every warp alike)
      v3 p;
      if (m.init && march_cheap<MEAN_SPHERE_ONLY>(S, m, p, ovf, &full))
        march_psi<MEAN_SPHERE_ONLY, true>(S, m, p, full, ovf);
      m.spec_valid = false;
    }
    while (m.status == 0) {
      // candidate 0: the march's next psi step; jumps, certain hits and the
      // end are settled on the way exactly as the one-group march settles them
      v3 p0;
      if (!march_cheap<MEAN_SPHERE_ONLY>(S, m, p0, ovf, nullptr)) break;
      const int k0 = m.k;
      const float mu0 = m.pend_mu;
      // the next W steps (table marches), one per thread: 0 sign settled and
      // kept, 1 needs psi, 2 sign settled and changed (hit), 3 past the end
      int stop = W, total = 0, take = 0;
      {
        const int i = (int)threadIdx.x, kk = k0 + 1 + i;
        int cls = 3;
        // step k0 + 1 + i: from the table, or by the i + 1 sequential adds the
        // one-group march performs (a step that does not advance t ends the
        // march with ERR_MARCH_GUARD, as march_advance does)
        float tw = 0.0f;
        bool valid = false;
        if (m.use_tab) {
          valid = i < W && kk < S->tab_steps;
          if (valid) tw = __ldg(S->tab + kk);
        } else if (i < W) {
          tw = m.t;
          bool stuck = false;
          for (int s = 0; s <= i; ++s) {
            const float tn = tw + m.dt;
            stuck = stuck || tn == tw;
            tw = tn;
          }
          valid = !stuck && tw < m.ft;
          if (stuck) cls = 4;
        }
        if (valid) {
          const v3 pw = m.o + m.d * tw;
          const float mw = mean_value<MEAN_SPHERE_ONLY>(S, md, pw, ovf);
          const float lb = fabsf(mw);
          if (lb * 0.999999f > m.B || lb * 0.999999f > noise_bound_at(md.k, m.c, pw))
            cls = ((mw > 0.0f) != m.fprev_pos) ? 2 : 0;
          else
            cls = 1;
          s_mw[i] = mw;
        }
        if (i < W) s_tw[i] = tw;
        const unsigned need = __ballot_sync(0xffffffffu, cls == 1), end = __ballot_sync(0xffffffffu, cls >= 2);
        if (i < W && cls >= 2) s_cls[i] = cls;  // 2 hit, 3 past the end, 4 t stopped advancing
        if (lane == 0 && warp < kMaxWarps) {
          s_need[warp] = need;
          s_end[warp] = end;
        }
        __syncthreads();
        for (int w = 0; w < nw; ++w)
          if (s_end[w]) {
            stop = 32 * w + __ffs(s_end[w]) - 1;
            break;
          }
        for (int w = 0; w < nw; ++w) total += __popc(s_need[w] & below(stop, w));
        take = min(total, ncand_max - 1);
      }
      const int nc = 1 + take;
      if (cand < nc) {
        v3 myp = p0;
        float mymu = mu0;
        if (cand > 0) {
          const int pos = nth_need(s_need, nw, stop, cand - 1);
          myp = m.o + m.d * s_tw[pos];
          mymu = s_mw[pos];
        }
        const float qv = (md.k.sigma * psi_sums_group<false, true, -1>(md.k, myp, m.seed, half).x) / md.k.sqrt_var;
        float f = mymu + qv;
        if (m.c.active) f += cond_value(md.k, m.c, myp);
        const bool hit = (f > 0.0f) != m.fprev_pos && (m.fprev_big || (double)fabsf(m.fprev - f) > 1e-6);
        if (half.sub == 0) s_hit[cand] = hit ? 1 : 0;
      }
      __syncthreads();
      int first = -1;
      for (int c = 0; c < nc; ++c)
        if (s_hit[c]) {
          first = c;
          break;
        }
      if (first == 0) {  // at candidate 0's step, where march_cheap left the march
        m.status = 1;
      } else if (first > 0) {
        const int pos = nth_need(s_need, nw, stop, first - 1);
        m.k = k0 + 1 + pos;
        m.t = s_tw[pos];
        m.status = 1;
      } else if (take < total) {  // more psi steps in the window than candidates: resume after the last one
        const int pos = nth_need(s_need, nw, stop, take - 1) + 1;  // < stop <= W
        m.k = k0 + 1 + pos;
        m.t = m.use_tab ? __ldg(S->tab + m.k) : s_tw[pos];
      } else if (stop < W) {  // the window's first settled change of sign, or the end
        m.k = k0 + 1 + stop;
        if (s_cls[stop] == 2) {
          m.t = s_tw[stop];
          m.status = 1;
        } else {
          m.t = m.use_tab ? __ldg(S->tab + m.k) : s_tw[stop];
          if (s_cls[stop] == 4 && threadIdx.x == 0) atomicOr(S->err, ERR_MARCH_GUARD);
          m.status = 2;
        }
      } else {  // every window step keeps its sign: on after the window
        m.k = k0 + 1 + W;
        if (m.use_tab) {
          m.t = __ldg(S->tab + m.k);
        } else {
          const float tn = s_tw[W - 1] + m.dt;
          if (tn == s_tw[W - 1]) {
            if (threadIdx.x == 0) atomicOr(S->err, ERR_MARCH_GUARD);
            m.status = 2;
          }
          m.t = tn;
        }
      }
      m.n_steps += (uint32_t)min(stop, W);
      psis += (unsigned long long)nc;
      imps += (unsigned long long)nc * 27ull * (unsigned long long)md.k.ppc;
      __syncthreads();  // the shared candidate state is written again next round
    }
    if constexpr (SH) {
      if (threadIdx.x == 0) add_shadow_term(P, idx, m.status == 1 ? 0.0f : 1.0f);
    } else if (warp == 0) {
      mupsi_medium_sample r;
      march_result<MEAN_SPHERE_ONLY, true>(S, m, r, ovf, full);
      if (lane == 0) {
        P.ha[idx] = make_float4(r.t, r.p[0], r.p[1], r.p[2]);
        P.hb[idx] = make_float4(r.normal[0], r.normal[1], r.normal[2], __uint_as_float(r.exited));
      }
    }
    steps += m.n_steps;
  }
  if (ovf) atomicOr(cfg.err, ERR_BVH_STACK);
  if (cfg.counters && threadIdx.x == 0) {
    atomicAdd(&cfg.counters[0], steps);
    atomicAdd(&cfg.counters[1], psis);
    atomicAdd(&cfg.counters[2], marches);
    atomicAdd(&cfg.counters[3], imps);
  }
}

// Marches of a long queue: one ray per lane. Which steps need psi is settled
// per ray without psi (the mean, the global and per-point noise bounds, the
// Lipschitz jumps and, for mesh means, the lazy exact mean and its BVH
// queries: march_cheap), each lane on its own ray with no copy of that work on
// other lanes; the psi sums of every lane that reached a psi step are then
// evaluated by the whole warp, two points at a time, each by a half-warp in the
// 16-slot order (psi_sums_group with G = 16: the values the lane-group march
// computes for any group size, so the march outcome and the hit normal are the
// same bits). A hit's gradient sum goes the same way. A mesh mean's BVH queries
// run on the querying lane alone (their results do not depend on the group).
// `rays_per_warp` (a power of two <= 32) spreads a shorter queue over all warps:
// only every (32 / rays_per_warp)-th lane takes a ray. Each round a ray visits at
// most `budget` steps before the warp's psi round, so a ray far from the
// surface (Lipschitz jumps, settled steps) does not hold the others' psi.
// Round r >= 1 of a march with a surrogate resumes the marches suspended in
// round r - 1 with their predictions (req/pred lists); a march that asks for a
// prediction is saved and suspended as in the lane-group march.
#ifndef MUPSI_LANE_SPEC
#define MUPSI_LANE_SPEC 1  // sphere means: a round's idle half-warp computes psi at the next step ahead
#endif
template <int MK>
__device__ void march_lanes(const DScene* const* __restrict__ scenes, Paths& P, uint32_t n,
                            const uint32_t* __restrict__ q, uint32_t* cursor, const WaveCfg& cfg, int rays_per_warp,
                            int budget, int it, int round, bool resume, bool can_suspend) {
  const unsigned full = 0xffffffffu;
  const int lane = (int)(threadIdx.x & 31);
  const int stride = 32 / rays_per_warp;
  const bool owner = (lane & (stride - 1)) == 0;
  const int R = P.rounds;
  Group half;  // a half-warp evaluates one point's psi (16 slots, one per lane)
  half.G = 16;
  half.sub = lane & 15;
  half.mask = full;
  Group solo;  // this lane alone (mesh means: closest-point queries with the group tie rule)
  solo.G = 1;
  solo.sub = 0;
  solo.mask = 1u << lane;
  solo.lowtie = true;
  March m;
  const DScene* S = scenes[0];
  uint32_t idx = 0;
  bool active = false, ovf = false;
  // this lane's rays (32 bits suffice per lane)
  uint32_t steps = 0, psis = 0, marches = 0, imps = 0, mus = 0, pars = 0, reqs = 0, accs = 0;
  while (true) {
    // owners without a ray take the next ones from the queue (one atomic per warp)
    bool drew = false;
    const unsigned need = __ballot_sync(full, owner && !active);
    if (need) {
      uint32_t base = 0;
      const int leader = __ffs(need) - 1;
      if (lane == leader) base = atomicAdd(cursor, (uint32_t)__popc(need));
      base = __shfl_sync(full, base, leader);
      if (owner && !active) {
        const uint32_t j = base + __popc(need & ((1u << lane) - 1u));
        if (j < n) {
          drew = true;
          idx = resume ? __float_as_uint(P.req[(round - 1) & 1][j].w) : q[j];
          const float4 o = P.o[idx], d = P.d[idx];
          const int4 meta = P.meta[idx];
          const int med = __float_as_int(d.w);
          S = scenes[meta_inst(meta.w)];
          if (resume || S->media[med].kind == MUPSI_MEDIUM_GP) {  // else k_march_field marches it
            march_begin(S, m, mk3(o.x, o.y, o.z), mk3(d.x, d.y, d.z), o.w, 3.402823466e+38f, med,
                        medium_seed(S, meta.x, meta.y, meta.z, meta_bounce(meta.w)), load_cond(P, idx));
            m.may_request = MK != MEAN_SPHERE_ONLY && can_suspend && m.lazy && S->media[med].surr;
            m.defer_mu = MK != MEAN_SPHERE_ONLY && m.lazy && !m.may_request && cfg.mu_batch > 0;
            if (MK != MEAN_SPHERE_ONLY && resume) {
              const float4 a = P.ms0[idx], b = P.ms1[idx];
              const int fl = __float_as_int(a.w);
              m.t = a.x;
              m.k = __float_as_int(a.y);
              m.fprev = a.z;
              m.fprev_pos = (fl & 1) != 0;
              m.fprev_big = (fl & 2) != 0;
              m.n_req = fl >> 8;
              m.init = false;
              m.mu_j = b.x;
              m.mu_hi = b.y;
              m.t_j = b.z;
              if (march_apply_prediction(S->media[med], m, P.pred[(round - 1) & 1][j])) accs++;
              if (fl & 4) march_resume_decide<MK>(S, m, b.w, &solo, ovf);  // suspended in march_decide
            } else {
              marches++;
            }
            active = true;
          }
        }
      }
    }
    if (!__any_sync(full, active || drew)) break;
    // this lane's ray up to its next psi step (at most `budget` visited steps)
    v3 p = mk3(0.0f, 0.0f, 0.0f);
    // suspended (status 3 at a step march_cheap reached, 4 in march_decide with
    // the step's psi): save the march, request a prediction at p
    auto suspend = [&]() {
      const int fl = (m.fprev_pos ? 1 : 0) | (m.fprev_big ? 2 : 0) | (m.status == 4 ? 4 : 0) | (m.n_req << 8);
      P.ms0[idx] = make_float4(m.t, __int_as_float(m.k), m.fprev, __int_as_float(fl));
      P.ms1[idx] = make_float4(m.mu_j, m.mu_hi, m.t_j, m.status == 4 ? m.spec_q : 0.0f);
      const uint32_t slot = atomicAdd(&P.rcounts[it * R + round], 1u);
      P.req[round & 1][slot] = make_float4(p.x, p.y, p.z, __uint_as_float(idx));
      reqs++;
      steps += m.n_steps;
      psis += m.n_psi;
      imps += m.n_psi * 27u * (uint32_t)S->media[m.medium].k.ppc;
      mus += m.n_mu;
      pars += m.n_par;
      active = false;
    };
    // (a resumed march may have finished in march_resume_decide)
    const bool want = active && m.status == 0 && march_cheap<MK>(S, m, p, ovf, &solo, budget);
    if (MK != MEAN_SPHERE_ONLY && active && m.status == 3) suspend();
    // the warp's psi values, two points per round; the kernel parameters are
    // read once when every ray of the warp has the same scene and medium
    float qv = 0.0f;
    bool fresh = want;  // false: the step's psi was computed ahead (below)
    if constexpr (MUPSI_LANE_SPEC && MK == MEAN_SPHERE_ONLY) {
      if (want && m.spec_valid && m.spec_t == m.t) {
        qv = m.spec_q;  // the same point and order: the same bits
        fresh = false;
      }
      if (want) m.spec_valid = false;
    }
    const unsigned vmask = __ballot_sync(full, fresh);
    const int ref = vmask ? __ffs(vmask) - 1 : 0;
    const DScene* S0 = reinterpret_cast<const DScene*>(__shfl_sync(full, reinterpret_cast<unsigned long long>(S), ref));
    const int m0 = __shfl_sync(full, m.medium, ref);
    const bool uni = __all_sync(full, !fresh || (S == S0 && m.medium == m0));
    for (unsigned vm = vmask; vm;) {
      const int a = __ffs(vm) - 1;
      vm &= vm - 1u;
      int b = a;
      if (vm) {
        b = __ffs(vm) - 1;
        vm &= vm - 1u;
      }
      const int src = lane < 16 ? a : b;
      v3 ps = mk3(__shfl_sync(full, p.x, src), __shfl_sync(full, p.y, src), __shfl_sync(full, p.z, src));
      const uint32_t sd = __shfl_sync(full, m.seed, src);
      // one point left (a round with an idle half-warp; in the late part of a
      // launch most rounds): the upper half computes psi at the step after
      // a's, the step march_advance moves to when this one is no hit, so a
      // march that needs psi there too finds it ready (the 32-lane group's
      // speculation, march_psi)
      float tn = 0.0f;
      bool spec = false;
      if constexpr (MUPSI_LANE_SPEC && MK == MEAN_SPHERE_ONLY) {
        if (b == a) {
          bool ok;
          if (m.use_tab) {
            ok = active && m.k + 1 <= S->tab_steps;
            tn = ok ? __ldg(S->tab + m.k + 1) : m.t;
          } else {
            tn = m.t + m.dt;
            ok = active && tn < m.ft && tn != m.t;
          }
          const v3 pe = m.o + m.d * tn;
          spec = __shfl_sync(full, ok ? 1 : 0, a) != 0;
          const v3 pa = mk3(__shfl_sync(full, pe.x, a), __shfl_sync(full, pe.y, a), __shfl_sync(full, pe.z, a));
          if (spec && lane >= 16) ps = pa;
        }
      }
      const DScene* Ss = S0;
      int ms = m0;
      if (!uni) {
        Ss = reinterpret_cast<const DScene*>(__shfl_sync(full, reinterpret_cast<unsigned long long>(S), src));
        ms = __shfl_sync(full, m.medium, src);
      }
      const KParams& k = Ss->media[ms].k;
      const float v = raw_noise_value_group<true, MK == MEAN_SPHERE_ONLY ? -1 : 0>(k, ps, sd, half);
      const float va = __shfl_sync(full, v, 0), vb = __shfl_sync(full, v, 16);
      if (lane == a) qv = va;
      if (lane == b && b != a) qv = vb;
      if (MUPSI_LANE_SPEC && MK == MEAN_SPHERE_ONLY && spec && lane == a) {
        m.spec_q = vb;
        m.spec_t = tn;
        m.spec_valid = true;
      }
    }
    if (want) {
      m.n_psi++;
      march_decide<MK>(S, m, p, qv, &solo, ovf);
      if (MK != MEAN_SPHERE_ONLY && m.status == 4) suspend();
    }
    // hits: the gradient at the hit point (GPMedium::evalWithGradient), two per round
    const bool hit = active && m.status == 1;
    const v3 ph = hit ? m.o + m.d * m.t : mk3(0.0f, 0.0f, 0.0f);
    float4 nz = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    for (unsigned hm = __ballot_sync(full, hit); hm;) {
      const int a = __ffs(hm) - 1;
      hm &= hm - 1u;
      int b = a;
      if (hm) {
        b = __ffs(hm) - 1;
        hm &= hm - 1u;
      }
      const int src = lane < 16 ? a : b;
      const v3 ps = mk3(__shfl_sync(full, ph.x, src), __shfl_sync(full, ph.y, src), __shfl_sync(full, ph.z, src));
      const uint32_t sd = __shfl_sync(full, m.seed, src);
      const DScene* Ss = reinterpret_cast<const DScene*>(__shfl_sync(full, reinterpret_cast<unsigned long long>(S), src));
      const int ms = __shfl_sync(full, m.medium, src);
      const KParams& k = Ss->media[ms].k;
      const float4 g = raw_noise_group<true, MK == MEAN_SPHERE_ONLY ? -1 : 0>(k, ps, sd, half);
      const float4 ga = make_float4(__shfl_sync(full, g.x, 0), __shfl_sync(full, g.y, 0), __shfl_sync(full, g.z, 0),
                                    __shfl_sync(full, g.w, 0));
      const float4 gb = make_float4(__shfl_sync(full, g.x, 16), __shfl_sync(full, g.y, 16),
                                    __shfl_sync(full, g.z, 16), __shfl_sync(full, g.w, 16));
      if (lane == a) nz = ga;
      if (lane == b && b != a) nz = gb;
    }
    if (active && (m.status == 1 || m.status == 2)) {
      if (hit) {  // march_result: normalize(grad f) at the hit step
        const DMedium& md = S->media[m.medium];
        const float4 mu = mean_value_grad<MK>(S, md, ph, ovf);
        float4 f = make_float4(mu.x + nz.x, mu.y + nz.y, mu.z + nz.z, mu.w + nz.w);
        f = add_cond(md.k, m.c, ph, f);
        const v3 nn = normalized(mk3(f.y, f.z, f.w));
        P.ha[idx] = make_float4(m.t, ph.x, ph.y, ph.z);
        P.hb[idx] = make_float4(nn.x, nn.y, nn.z, __uint_as_float(0u));
      } else {  // exited: t, p and normal zero
        P.ha[idx] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        P.hb[idx] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(1u));
      }
      steps += m.n_steps;
      psis += m.n_psi;
      imps += m.n_psi * 27u * (uint32_t)S->media[m.medium].k.ppc;
      mus += m.n_mu;
      pars += m.n_par;
      active = false;
    }
    if constexpr (MK != MEAN_SPHERE_ONLY) {
      // marches waiting for an exact mean (statuses 5, 6) query the BVH together
      // once mu_batch of them wait, or every active one does: one lane's
      // traversal no longer holds the warp's other marches at each query
      // (deferring the origins' and the hits' queries the same way measured slower)
      const bool wait = active && (m.status == 5 || m.status == 6);
      const unsigned wm = __ballot_sync(full, wait);
      if (wm && (__popc(wm) >= cfg.mu_batch || wm == __ballot_sync(full, active))) {
        if (wait) {
          if (m.status == 5)
            march_exact_step<MK>(S, m, &solo, ovf);
          else
            march_exact_decide<MK>(S, m, &solo, ovf);
        }
      }
    }
  }
  if (ovf) atomicOr(cfg.err, ERR_BVH_STACK);
  if (cfg.counters) {
    unsigned long long c[8] = {steps, psis, marches, imps, mus, pars, reqs, accs};
    for (int i = 0; i < (MK == MEAN_SPHERE_ONLY ? 4 : 8); ++i) {
      for (int o = 16; o > 0; o >>= 1) c[i] += __shfl_down_sync(full, c[i], o);
      if (lane == 0) atomicAdd(&cfg.counters[i], c[i]);
    }
  }
}

// Persistent march over the medium queue of iteration `it`. Each ray is
// marched by a group of G lanes that share its psi sums: G = 4 while the queue
// fills the resident threads, larger (up to 32) as the queue shrinks, so the
// late bounces' few long marches finish up to 8x sooner than on one lane.
// SH: the shadow-pass instantiation (the medium march carries none of its code).
// The general (mesh-mean) march is bound by the latency of its BVH traversals
// and runs best with every thread resident (16 blocks per SM, 32 registers,
// the rest spilled to L1): 483 -> 331 ms for a level-6 mesh render at 512^2 x 4.
#ifndef MUPSI_SPHERE_MARCH_BLOCKS
#define MUPSI_SPHERE_MARCH_BLOCKS 4  // resident 128-thread blocks per SM of the sphere-mean march
#endif
#ifndef MUPSI_MESH_MARCH_BLOCKS
#define MUPSI_MESH_MARCH_BLOCKS 16  // ... of the general (mesh-mean) march with lane groups
#endif
#ifndef MUPSI_MESH_LANE_MARCH_BLOCKS
#define MUPSI_MESH_LANE_MARCH_BLOCKS 16  // ... and of the mesh-mean march with one ray per lane
#endif
// LANES: the instantiation carries march_lanes (one ray per lane); the mesh
// kernel without it keeps its registers for the lane-group march alone
template <int MK, bool SH, bool LANES = MK == MEAN_SPHERE_ONLY>
__global__ void __launch_bounds__(128, MK == MEAN_SPHERE_ONLY ? MUPSI_SPHERE_MARCH_BLOCKS
                                       : LANES               ? MUPSI_MESH_LANE_MARCH_BLOCKS
                                                             : MUPSI_MESH_MARCH_BLOCKS)
    k_march(const DScene* const* __restrict__ scenes, Paths P, int it, int round,
                                               WaveCfg cfg) {
  // round 0 marches the iteration's medium queue; round r >= 1 resumes the
  // marches suspended in round r - 1 with their surrogate predictions
  // (a scene with sphere means only has no surrogate: one round, no resumes)
  // a shadow pass marches the shadow jobs the shading of iteration it - 1 left
  // (GPMedium::transmittance, gpmedium.cpp:105-129) instead of the medium queue
  constexpr bool shadow = SH;
  const bool resume = MK != MEAN_SPHERE_ONLY && round > 0 && !shadow;
  const int R = P.rounds;
  const uint32_t n = shadow ? P.scounts[it] : resume ? P.rcounts[it * R + round - 1] : P.counts[2 * it];
  const uint32_t* q = shadow ? P.sq[it & 1] : P.q[it & 1];
  uint32_t* cursor = shadow ? P.scursors + it : resume ? P.rcursors + it * R + round : P.cursors + it;
  const bool can_suspend = round + 1 < R && !shadow;
  if constexpr (MK == MEAN_SPHERE_ONLY) {
    if ((uint64_t)n <= (uint64_t)gridDim.x * (uint64_t)cfg.block_rays) {
      march_block_rays<SH>(scenes, P, n, q, cursor, cfg);
      return;
    }
  }
  if (LANES && !SH && cfg.lane_rays) {
    // long queues: one ray per lane, at least 2 rays per warp on average (4, 8 or
    // 16 measured the same: the late bounces' time is their longest marches)
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    if ((uint64_t)n >= 2 * warps) {
      int r = 2;
      while (r < 32 && (uint64_t)n >= warps * (uint64_t)(2 * r)) r <<= 1;
      march_lanes<MK>(scenes, P, n, q, cursor, cfg, r, cfg.lane_rays, it, round, resume, can_suspend);
      return;
    }
  }
  const unsigned lane = threadIdx.x & 31;
  const uint64_t resident = (uint64_t)gridDim.x * blockDim.x;
  Group grp;
  grp.G = max(4, cfg.min_group);  // >= 4: march_result's WIDE gradient order
  while (grp.G < 32 && (uint64_t)n * (uint64_t)(2 * grp.G) <= resident) grp.G <<= 1;
  grp.sub = (int)(lane & (unsigned)(grp.G - 1));
  const unsigned gbase = lane & ~(unsigned)(grp.G - 1);
  grp.mask = grp.G == 32 ? 0xffffffffu : (((1u << grp.G) - 1u) << gbase);
  March m;
  const DScene* S = scenes[0];
  uint32_t idx = 0;
  bool active = false;
  bool ovf = false;
  unsigned long long steps = 0, psis = 0, marches = 0, imps = 0, mus = 0, pars = 0, reqs = 0, accs = 0;
  while (true) {
    bool skipped = false;  // this group drew a path of a field medium (k_march_field marches it)
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
          idx = resume ? __float_as_uint(P.req[(round - 1) & 1][j].w) : q[j];
          float4 o = P.o[idx], d = P.d[idx];
          int4 meta = P.meta[idx];
          int med = __float_as_int(d.w);
          S = scenes[meta_inst(meta.w)];
          if (shadow && S->media[__float_as_int(P.sh_b[idx].w)].kind != MUPSI_MEDIUM_GP) {
            skipped = true;  // a field medium's job: k_march_field's shadow pass
          } else if (shadow) {  // the shadow ray of the job (its own medium, seed and conditioning)
            const float4 a = P.sh_a[idx], b = P.sh_b[idx], ca = P.sh_ca[idx], cb = P.sh_cb[idx];
            med = __float_as_int(b.w);
            Cond c;
            c.C = mk3(ca.x, ca.y, ca.z);
            c.u = ca.w;
            c.g = mk3(cb.x, cb.y, cb.z);
            c.active = __float_as_uint(cb.w);
            march_begin(S, m, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), 0.0f, a.w, med, (uint32_t)P.sh_m[idx].y, c);
            m.may_request = false;
            if (grp.sub == 0) marches++;
            active = true;
          }
          if (!shadow) skipped = !resume && S->media[med].kind != MUPSI_MEDIUM_GP;  // k_march_field marches it
          if (!skipped && !shadow) {
            march_begin(S, m, mk3(o.x, o.y, o.z), mk3(d.x, d.y, d.z), o.w, 3.402823466e+38f, med,
                        medium_seed(S, meta.x, meta.y, meta.z, meta_bounce(meta.w)), load_cond(P, idx));
            m.may_request = MK != MEAN_SPHERE_ONLY && can_suspend && m.lazy && S->media[med].surr;
            if (MK != MEAN_SPHERE_ONLY && resume) {
              const float4 a = P.ms0[idx], b = P.ms1[idx];
              const int fl = __float_as_int(a.w);
              m.t = a.x;
              m.k = __float_as_int(a.y);
              m.fprev = a.z;
              m.fprev_pos = (fl & 1) != 0;
              m.fprev_big = (fl & 2) != 0;
              m.n_req = fl >> 8;
              m.init = false;
              m.mu_j = b.x;
              m.mu_hi = b.y;
              m.t_j = b.z;
              const bool used = march_apply_prediction(S->media[med], m, P.pred[(round - 1) & 1][j]);
              if (grp.sub == 0 && used) accs++;
              if (fl & 4) march_resume_decide<MK>(S, m, b.w, &grp, ovf);  // suspended in march_decide
            } else if (grp.sub == 0) {
              marches++;
            }
            active = true;
          }
        }
      }
    }
    if (!__any_sync(0xffffffffu, active || skipped)) break;
    if (active) {
      v3 p = mk3(0.0f, 0.0f, 0.0f);
      // (a resumed march may have finished in march_resume_decide)
      if (m.status == 0 && march_cheap<MK>(S, m, p, ovf, &grp)) march_psi<MK, true>(S, m, p, grp, ovf);
      if (MK != MEAN_SPHERE_ONLY && m.status >= 3) {
        // suspended (status 3 at a step march_cheap reached, 4 in march_decide
        // with the step's psi): save the march, request a prediction at p
        if (grp.sub == 0) {
          const int fl = (m.fprev_pos ? 1 : 0) | (m.fprev_big ? 2 : 0) | (m.status == 4 ? 4 : 0) | (m.n_req << 8);
          P.ms0[idx] = make_float4(m.t, __int_as_float(m.k), m.fprev, __int_as_float(fl));
          P.ms1[idx] = make_float4(m.mu_j, m.mu_hi, m.t_j, m.status == 4 ? m.spec_q : 0.0f);
          const uint32_t slot = atomicAdd(&P.rcounts[it * R + round], 1u);
          P.req[round & 1][slot] = make_float4(p.x, p.y, p.z, __uint_as_float(idx));
          reqs++;
          steps += m.n_steps;
          psis += m.n_psi;
          imps += (unsigned long long)m.n_psi * 27ull * (unsigned long long)S->media[m.medium].k.ppc;
          mus += m.n_mu;
          pars += m.n_par;
        }
        active = false;
      } else if (m.status != 0 && shadow) {
        if (grp.sub == 0) {  // transmittance 0 at a sign change: the NEE term (tr * X) * c
          add_shadow_term(P, idx, m.status == 1 ? 0.0f : 1.0f);
          steps += m.n_steps;
          psis += m.n_psi;
          imps += (unsigned long long)m.n_psi * 27ull * (unsigned long long)S->media[m.medium].k.ppc;
          mus += m.n_mu;
          pars += m.n_par;
        }
        active = false;
      } else if (m.status != 0) {
        mupsi_medium_sample r;
        march_result<MK, true>(S, m, r, ovf, grp);
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
  if (ovf) atomicOr(cfg.err, ERR_BVH_STACK);
  if (cfg.counters) {
    for (int o = 16; o > 0; o >>= 1) {
      steps += __shfl_down_sync(0xffffffffu, steps, o);
      psis += __shfl_down_sync(0xffffffffu, psis, o);
      marches += __shfl_down_sync(0xffffffffu, marches, o);
      imps += __shfl_down_sync(0xffffffffu, imps, o);
      mus += __shfl_down_sync(0xffffffffu, mus, o);
      pars += __shfl_down_sync(0xffffffffu, pars, o);
      reqs += __shfl_down_sync(0xffffffffu, reqs, o);
      accs += __shfl_down_sync(0xffffffffu, accs, o);
    }
    if (lane == 0) {
      atomicAdd(&cfg.counters[0], steps);
      atomicAdd(&cfg.counters[1], psis);
      atomicAdd(&cfg.counters[2], marches);
      atomicAdd(&cfg.counters[3], imps);
      atomicAdd(&cfg.counters[4], mus);
      atomicAdd(&cfg.counters[5], pars);
      atomicAdd(&cfg.counters[6], reqs);
      atomicAdd(&cfg.counters[7], accs);
    }
  }
}

// SDFMedium / ExternalGPMedium::sampleDistance for the paths of iteration `it`
// whose medium is a field medium (k_march leaves them): one thread per path,
// sphere tracing bounded by the reference's iteration limits (512 / 1024).
#ifndef MUPSI_FIELD_MARCH_BLOCKS
#define MUPSI_FIELD_MARCH_BLOCKS 6  // resident 128-thread blocks per SM the field march is compiled for
#endif
__global__ void __launch_bounds__(128, MUPSI_FIELD_MARCH_BLOCKS) k_march_field(const DScene* const* __restrict__ scenes, Paths P, int it,
                                                     WaveCfg cfg) {
  bool ovf = false;
  if (cfg.shadow_pass) {  // the shadow jobs of field media (SDFMedium / ExternalGPMedium::transmittance)
    const uint32_t n = P.scounts[it];
    const uint32_t* q = P.sq[it & 1];
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
      const uint32_t idx = q[j];
      const float4 a = P.sh_a[idx], b = P.sh_b[idx];
      const DScene* S = scenes[meta_inst(P.meta[idx].w)];
      const DMedium& md = S->media[__float_as_int(b.w)];
      if (md.kind == MUPSI_MEDIUM_GP) continue;  // the march kernel's shadow pass
      const float tr = field_transmittance(S, md, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), 0.0f, a.w,
                                           (uint32_t)P.sh_m[idx].y, ovf);
      add_shadow_term(P, idx, tr);
    }
    if (ovf) atomicOr(cfg.err, ERR_BVH_STACK);
    return;
  }
  const uint32_t n = P.counts[2 * it];
  const uint32_t* q = P.q[it & 1];
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t idx = q[j];
    const float4 d = P.d[idx];
    const int4 meta = P.meta[idx];
    const DScene* S = scenes[meta_inst(meta.w)];
    const DMedium& md = S->media[__float_as_int(d.w)];
    if (md.kind == MUPSI_MEDIUM_GP) continue;
    const float4 o = P.o[idx];
    mupsi_medium_sample r;
    field_sample_distance(S, md, mk3(o.x, o.y, o.z), mk3(d.x, d.y, d.z), o.w, 3.402823466e+38f,
                          medium_seed(S, meta.x, meta.y, meta.z, meta_bounce(meta.w)), r, ovf);
    P.ha[idx] = make_float4(r.t, r.p[0], r.p[1], r.p[2]);
    P.hb[idx] = make_float4(r.normal[0], r.normal[1], r.normal[2], __uint_as_float(r.exited));
  }
  if (ovf) atomicOr(cfg.err, ERR_BVH_STACK);
}

// Medium::transmittance: GPMedium (gpmedium.cpp:105-129) or a field medium;
// 0 at the first sign change.
MD float transmittance(const DScene* S, int medium, const Ray& r, uint32_t seed, const Cond& c, bool& ovf) {
  const DMedium& md = S->media[medium];
  if (md.kind != MUPSI_MEDIUM_GP) return field_transmittance(S, md, r.o, r.d, r.nt, r.ft, seed, ovf);
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
#ifndef MUPSI_SHADE_BLOCKS
#define MUPSI_SHADE_BLOCKS 4  // resident 128-thread blocks per SM the shading kernel is compiled for
#endif
__global__ void __launch_bounds__(128, MUPSI_SHADE_BLOCKS) k_shade(const DScene* const* __restrict__ scenes, Paths P, int it, WaveCfg cfg) {
  const uint32_t n = P.counts[2 * it + 1];
  const uint32_t* q = P.q[2 + (it & 1)];
  uint32_t* qm_next = P.q[(it + 1) & 1];
  uint32_t* qa_next = P.q[2 + ((it + 1) & 1)];
  uint32_t* cm_next = P.counts + 2 * (it + 1);
  uint32_t* ca_next = P.counts + 2 * (it + 1) + 1;
  const v3 med_albedo = mk3(0.8f, 0.8f, 0.8f);  // Medium::default_bsdf_: Lambertian, albedo 0.8
  bool ovf = false;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t i = q[j];
    bool job = false;  // this path's medium NEE left a shadow job
    uint32_t jseed = 0;
    float4 o4 = P.o[i], d4 = P.d[i], t4 = P.thr[i], e4 = P.em[i];
    int4 meta = P.meta[i];
    const int inst = meta_inst(meta.w);
    const DScene* S = scenes[inst];
    const bool single = S->gp_mode == MUPSI_GP_SINGLE_REALIZATION;
    int medium = __float_as_int(d4.w);
    uint64_t rng = ld_rng(P.rng[i]);
    v3 thr = mk3(t4.x, t4.y, t4.z), em = mk3(e4.x, e4.y, e4.z);
    Ray ray;
    ray.o = mk3(o4.x, o4.y, o4.z);
    ray.d = mk3(d4.x, d4.y, d4.z);
    ray.nt = o4.w;
    ray.ft = 3.402823466e+38f;
    int bounce = meta_bounce(meta.w);
    bool has_hit = false, exited = true, dead = false;
    Cond cond = load_cond(P, i);
    if (medium >= 0 && !S->skip_medium) {  // the medium branch (trace.cpp:142)
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
          const uint32_t sseed = medium_seed(S, meta.x, meta.y, meta.z, bounce);
          const v3 f = bsdf_weight(MUPSI_BSDF_LAMBERTIAN, med_albedo, ls.d, wo, N);
          const v3 X = cmul(thr, cmul(f, ls.weight));
          const float c = fabsf(dot(ls.d, N));
          if (cfg.defer) {
            // the next march launch marches the shadow ray (lane groups, the same
            // values) and adds (tr * X) * c before anything else reaches this path
            P.sh_a[i] = make_float4(sr.o.x, sr.o.y, sr.o.z, sr.ft);
            P.sh_b[i] = make_float4(sr.d.x, sr.d.y, sr.d.z, __int_as_float(medium));
            P.sh_x[i] = make_float4(X.x, X.y, X.z, c);
            P.sh_ca[i] = make_float4(cond.C.x, cond.C.y, cond.C.z, cond.u);
            P.sh_cb[i] = make_float4(cond.g.x, cond.g.y, cond.g.z, __uint_as_float(cond.active));
            job = true;
            jseed = sseed;
          } else {
            const float tr = transmittance(S, medium, sr, sseed, cond, ovf);
            em = em + (tr * X) * c;
          }
        }
        v3 w;
        v3 wi = bsdf_sample(MUPSI_BSDF_LAMBERTIAN, med_albedo, wo, N, rng, w);
        thr = cmul(thr, w);
        float surv = maxc(thr);
        if (pcg_next1d(rng) > surv) {
          dead = true;
        } else {
          thr = thr / surv;
          if (S->media[medium].kind == MUPSI_MEDIUM_GP) {  // only a GPMedium conditions (trace.cpp:144-147)
            uint32_t ns = medium_seed(S, meta.x, meta.y, meta.z, bounce + 1);
            cond = sample_condition(S, S->media[medium], Pt, N, false, ns, !single, ovf);
          }
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
        const v3 alb = pr.tex ? tex_lookup(pr.tex, pr.tex_w, pr.tex_h, hi.tu, hi.tv) : pr.albedo;
        LSample ls;
        if (choose_light(S, hi.p, rng, ls)) {  // handleSurface NEE (trace.cpp:40-56)
          Ray sr = make_ray(hi.p + N * S->eps, ls.d);
          float bias = ls.dist - S->eps * fabsf(dot(ls.d, N));
          sr.ft = bias * 0.99f;
          if (!scene_occluded(S, sr, ovf)) {
            v3 a = bsdf_weight(pr.bsdf, alb, ls.d, wo, N);
            em = em + cmul(thr, cmul(a, ls.weight)) * fabsf(dot(ls.d, N));
          }
        }
        v3 w;
        v3 wi = bsdf_sample(pr.bsdf, alb, wo, N, rng, w);
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
      } else if (S->sky_tex) {
        em = em + cmul(thr, sky_lookup(S, ray.d));
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
      P.meta[i] = make_int4(meta.x, meta.y, meta.z, pack_meta(bounce, inst));
      push(qa_next, ca_next, i);
      if (medium >= 0 && !S->skip_medium) push(qm_next, cm_next, i);
      if (job) P.sh_m[i] = make_int4(0, (int)jseed, 0, 0);
    } else {
      P.rad[3 * (int64_t)i] = em.x;
      P.rad[3 * (int64_t)i + 1] = em.y;
      P.rad[3 * (int64_t)i + 2] = em.z;
      if (job) P.sh_m[i] = make_int4(1, (int)jseed, 0, 0);
    }
    if (job) push(P.sq[(it + 1) & 1], P.scounts + it + 1, i);
  }
  if (ovf) atomicOr(cfg.err, ERR_BVH_STACK);
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

// k_accumulate over every chunk of a plan wave: chunk c adds its passes, in
// pass order, to the running sum of instance c.inst.
__global__ void k_accumulate_wave(const float* __restrict__ rad, WaveSrc src, float* const* __restrict__ sums) {
  int64_t n, npix;
  const WaveChunk* chunks;
  int nchunks;
  resolve_wave(src, n, npix, chunks, nchunks);
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < npix; q += (int64_t)gridDim.x * blockDim.x) {
    const WaveChunk& c = chunks[find_chunk(chunks, nchunks, q, [](const WaveChunk& w) { return w.pix0; })];
    const int64_t p = q - c.pix0;
    float* sum = sums[c.inst];
    float s0 = sum[3 * p], s1 = sum[3 * p + 1], s2 = sum[3 * p + 2];
    for (int k = 0; k < c.passes; ++k) {
      const float* r = rad + 3 * (c.path0 + (int64_t)k * c.wh + p);
      s0 += r[0];
      s1 += r[1];
      s2 += r[2];
    }
    sum[3 * p] = s0;
    sum[3 * p + 1] = s1;
    sum[3 * p + 2] = s2;
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
    const DMedium& md = S->media[medium];
    float4 r;
    if (md.kind == MUPSI_MEDIUM_EXTERNAL_GP) {  // its GridMeanFunction
      const v3 P3 = ld3(p + 3 * i);
      const v3 g = grid_gradient(md.gmean, P3);
      r = make_float4(grid_eval(md.gmean, P3), g.x, g.y, g.z);
    } else {
      r = mean_value_grad(S, md, ld3(p + 3 * i), ovf);
    }
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
    const DMedium& md = S->media[medium];
    float4 r = md.kind == MUPSI_MEDIUM_GP ? medium_eval(S, md, ld3(p + 3 * i), seed[i], c, ovf)
                                          : field_value_grad(S, md, ld3(p + 3 * i), seed[i], ovf);
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
    mupsi_medium_sample res;
    // Ray(origin, direction) normalises the direction (geometry/ray.h:12)
    if (S->media[medium].kind != MUPSI_MEDIUM_GP) {
      field_sample_distance(S, S->media[medium], ld3(r.o), normalized(ld3(r.d)), r.near_t, r.far_t, seed[i], res, ovf);
    } else {
      March m;
      march_begin(S, m, ld3(r.o), normalized(ld3(r.d)), r.near_t, r.far_t, medium, seed[i], c);
      march_full(S, m, ovf);
      march_result(S, m, res, ovf, single_lane());
    }
    out[i] = res;
  }
  if (ovf) atomicOr(S->err, ERR_BVH_STACK);
}
__global__ void k_transmittance(const DScene* S, int medium, int64_t n, const mupsi_ray* rays, const uint32_t* seed,
                                const Cond* cond, float* out) {
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
    Ray R = make_ray(ld3(r.o), ld3(r.d));
    R.nt = r.near_t;
    R.ft = r.far_t;
    out[i] = transmittance(S, medium, R, seed[i], c, ovf);
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
// Path state of one wave (SoA, grow-only) and the bounce iterations its queue
// counters were sized for.
struct PathBuf {
  Paths paths{};
  void* mem = nullptr;
  size_t bytes = 0;
  int64_t cap = 0;
  int iters = 0;
  int rounds = 1;  // surrogate rounds the round buffers were sized for
  bool shadow = false;  // shadow-job buffers present
};

struct mupsi_scene {
  DScene h;                 // host copy (pointers are device pointers)
  DScene* d = nullptr;      // device copy
  DScene** d_list = nullptr;  // device array {d}: the wave kernels' scene table
  WaveChunk* d_chunk = nullptr;  // device chunk table of one single-scene wave
  std::vector<void*> allocs;
  int width = 0, height = 0, max_bounce = 0;
  // progressive framebuffer: running sum and passes so far
  float* sum = nullptr;
  float* avg = nullptr;  // device staging of the averaged image for host output (kept: an
                         // allocation per render would be released and mapped again each time)
  int passes_done = 0;
  int next_pass = -1;  // pass after the last one accumulated
  PathBuf pb;  // wave buffers (grow-only)
  mupsi_mlp* surr_mlp = nullptr;  // surrogate of a mesh mean (not owned)
  void* sky_mem = nullptr;        // sky texture texels (owned)
  void* tex_mem[MAX_PRIMS] = {};  // albedo texture texels + texcoords per primitive (owned)
  void* grid_mem[MAX_MEDIA] = {};  // external GP mean + variance grids per medium (owned)
  int surr_rounds = 1;            // march rounds per bounce iteration with it: predictions + 1
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

void pool_release() {
  std::vector<PoolEntry> all;
  {
    std::lock_guard<std::mutex> lock(g_pool_mu);
    all.swap(g_pool);
  }
  int cur = 0;
  cudaGetDevice(&cur);
  for (const PoolEntry& e : all) {
    cudaSetDevice(e.dev);
    cudaFree(e.ptr);
  }
  cudaSetDevice(cur);
}

}  // namespace

mupsi_scene::~mupsi_scene() {
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    cudaDeviceSynchronize();  // nothing in flight reads the buffers handed back
    for (void* p : allocs) dev_give(p);
    dev_give(d);
    dev_give(d_list);
    dev_give(d_chunk);
    if (sky_mem) cudaFree(sky_mem);
    for (void* p : tex_mem)
      if (p) cudaFree(p);
    for (void* p : grid_mem)
      if (p) cudaFree(p);
    dev_give(sum);
    dev_give(avg);
    if (pb.mem) pool_give(pb.mem, pb.bytes);
    dev_give(err);
    dev_give(counters);
}

namespace {

// work counters of a scene: 8 march counters, then the BVH tallies
// (kBvhCountSlots pairs of nodes loaded, triangles tested)
constexpr int kSceneCounters = 8 + 2 * kBvhCountSlots;

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
  // lane groups of >= 4 share psi sums; scenes whose media all have sphere
  // means run the march specialised for them
  S.min_group = 4;
  S.sphere_only = 1;
  for (int i = 0; i < desc->num_media; ++i)
    if (desc->media[i].mean_type != MUPSI_MEAN_SPHERE) S.sphere_only = 0;
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
    MUPSI_CUDA(dev_take(&p, tab.size() * sizeof(float)));
    s->allocs.push_back(p);
    MUPSI_CUDA(cudaMemcpy(p, tab.data(), tab.size() * sizeof(float), cudaMemcpyHostToDevice));
    dtab = (const float*)p;
    S.tab = dtab;
    S.tab_steps = (int)tab.size() - 1;
    S.tab_nt = nt;
    S.tab_ft = ft;
    S.tab_dt = dt;
  }
  MUPSI_CUDA(dev_take((void**)&s->err, sizeof(int)));
  MUPSI_CUDA(cudaMemset(s->err, 0, sizeof(int)));
  S.err = s->err;
  MUPSI_CUDA(dev_take((void**)&s->counters, kSceneCounters * sizeof(unsigned long long)));
  MUPSI_CUDA(cudaMemset(s->counters, 0, kSceneCounters * sizeof(unsigned long long)));
  S.counters = nullptr;
  MUPSI_CUDA(dev_take((void**)&s->d, sizeof(DScene)));
  MUPSI_CUDA(cudaMemcpy(s->d, &S, sizeof(DScene), cudaMemcpyHostToDevice));
  MUPSI_CUDA(dev_take((void**)&s->d_list, sizeof(DScene*)));
  MUPSI_CUDA(cudaMemcpy(s->d_list, &s->d, sizeof(DScene*), cudaMemcpyHostToDevice));
  MUPSI_CUDA(dev_take((void**)&s->d_chunk, sizeof(WaveChunk)));
  s->width = desc->width;
  s->height = desc->height;
  s->max_bounce = desc->max_bounce;
  MUPSI_CUDA(dev_take((void**)&s->sum, (size_t)3 * desc->width * desc->height * sizeof(float)));
  MUPSI_CUDA(cudaMemset(s->sum, 0, (size_t)3 * desc->width * desc->height * sizeof(float)));
  return MUPSI_OK;
}

// PathTracer::trace's do-while runs at least one bounce iteration
int wave_iters(const mupsi_scene* s) { return std::max(1, s->max_bounce); }

int ensure_paths(PathBuf& b, int64_t cap, int iters, int rounds, bool shadow) {
  if (cap <= b.cap && iters <= b.iters && rounds <= b.rounds && (b.shadow || !shadow) && b.mem) return MUPSI_OK;
  if (b.mem) {
    pool_give(b.mem, b.bytes);
    b.mem = nullptr;
  }
  cap = std::max(cap, b.cap);
  iters = std::max(iters, b.iters);
  rounds = std::max(rounds, b.rounds);
  shadow = shadow || b.shadow;
  size_t bytes = 0;
  auto take = [&](size_t sz) {
    size_t off = bytes;
    bytes += (sz + 255) & ~(size_t)255;
    return off;
  };
  size_t o_o = take(cap * 16), o_d = take(cap * 16), o_t = take(cap * 16), o_e = take(cap * 16),
         o_r = take(cap * 8), o_ca = take(cap * 16), o_cb = take(cap * 16), o_m = take(cap * 16),
         o_ha = take(cap * 16), o_hb = take(cap * 16), o_rad = take(cap * 12), o_q0 = take(cap * 4),
         o_q1 = take(cap * 4), o_q2 = take(cap * 4), o_q3 = take(cap * 4), o_c = take((size_t)(iters + 1) * 8),
         o_cur = take((size_t)(iters + 1) * 4);
  const bool sr = rounds > 1;
  size_t o_s0 = sr ? take(cap * 16) : 0, o_s1 = sr ? take(cap * 16) : 0, o_rq0 = sr ? take(cap * 16) : 0,
         o_rq1 = sr ? take(cap * 16) : 0, o_pr0 = sr ? take(cap * 4) : 0, o_pr1 = sr ? take(cap * 4) : 0,
         o_rc = sr ? take((size_t)iters * rounds * 4) : 0, o_rr = sr ? take((size_t)iters * rounds * 4) : 0;
  size_t o_sa = shadow ? take(cap * 16) : 0, o_sb = shadow ? take(cap * 16) : 0, o_sx = shadow ? take(cap * 16) : 0,
         o_sca = shadow ? take(cap * 16) : 0, o_scb = shadow ? take(cap * 16) : 0, o_sm = shadow ? take(cap * 16) : 0,
         o_sq0 = shadow ? take(cap * 4) : 0, o_sq1 = shadow ? take(cap * 4) : 0,
         o_sc = shadow ? take((size_t)(iters + 1) * 4) : 0, o_scu = shadow ? take((size_t)(iters + 1) * 4) : 0;
  size_t got = 0;
  char* base = static_cast<char*>(pool_take(bytes, &got));
  if (!base) {
    MUPSI_CUDA(cudaMalloc((void**)&base, bytes));
    got = bytes;
  }
  b.mem = base;
  b.bytes = got;
  Paths& P = b.paths;
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
  P.rounds = 1;
  P.ms0 = sr ? (float4*)(base + o_s0) : nullptr;
  P.ms1 = sr ? (float4*)(base + o_s1) : nullptr;
  P.req[0] = sr ? (float4*)(base + o_rq0) : nullptr;
  P.req[1] = sr ? (float4*)(base + o_rq1) : nullptr;
  P.pred[0] = sr ? (float*)(base + o_pr0) : nullptr;
  P.pred[1] = sr ? (float*)(base + o_pr1) : nullptr;
  P.rcounts = sr ? (uint32_t*)(base + o_rc) : nullptr;
  P.rcursors = sr ? (uint32_t*)(base + o_rr) : nullptr;
  P.sh_a = shadow ? (float4*)(base + o_sa) : nullptr;
  P.sh_b = shadow ? (float4*)(base + o_sb) : nullptr;
  P.sh_x = shadow ? (float4*)(base + o_sx) : nullptr;
  P.sh_ca = shadow ? (float4*)(base + o_sca) : nullptr;
  P.sh_cb = shadow ? (float4*)(base + o_scb) : nullptr;
  P.sh_m = shadow ? (int4*)(base + o_sm) : nullptr;
  P.sq[0] = shadow ? (uint32_t*)(base + o_sq0) : nullptr;
  P.sq[1] = shadow ? (uint32_t*)(base + o_sq1) : nullptr;
  P.scounts = shadow ? (uint32_t*)(base + o_sc) : nullptr;
  P.scursors = shadow ? (uint32_t*)(base + o_scu) : nullptr;
  b.shadow = shadow;
  b.cap = cap;
  b.iters = iters;
  b.rounds = rounds;
  return MUPSI_OK;
}
bool needs_shadow_jobs(const DScene& h);
int ensure_paths(mupsi_scene* s, int64_t cap) {
  return ensure_paths(s->pb, cap, wave_iters(s) + 1, s->surr_mlp ? s->surr_rounds : 1, needs_shadow_jobs(s->h));
}

// Launch shapes of the wave kernels (mupsi_gpu_set_tuning; chosen by the
// project's autotuner, mupsi_b200/autotune.py).
mupsi_tuning g_tuning = {128, 4, 128, 0, 8, 1, 262144, 24};

// Persistent march grid: resident blocks per SM x SMs.
struct MarchLaunch {
  void (*fn)(const DScene* const*, Paths, int, int, WaveCfg);
  void (*fn_shadow)(const DScene* const*, Paths, int, int, WaveCfg);
  int blocks, block;
  int blocks_shadow;
};
// lanes: a mesh-mean wave marched one ray per lane (the sphere-mean kernel
// always carries that mode)
MarchLaunch march_launch(bool sphere_only, bool lanes = false) {
  static std::mutex mu;
  static std::vector<std::pair<int, MarchLaunch>> memo;  // key: variant | lanes << 1 | block << 2
  const int block = g_tuning.march_block;
  lanes = lanes && !sphere_only;
  const int key = (sphere_only ? 1 : 0) | (lanes ? 2 : 0) | (block << 2);
  std::lock_guard<std::mutex> lock(mu);
  for (auto& e : memo)
    if (e.first == key) return e.second;
  MarchLaunch m;
  m.fn = sphere_only ? k_march<MEAN_SPHERE_ONLY, false>
                     : (lanes ? k_march<MEAN_ANY, false, true> : k_march<MEAN_ANY, false, false>);
  m.fn_shadow = sphere_only ? k_march<MEAN_SPHERE_ONLY, true> : k_march<MEAN_ANY, true>;
  m.block = block;
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, m.fn, block, 0);
  m.blocks = std::max(1, per_sm) * num_sms();
  per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, m.fn_shadow, block, 0);
  m.blocks_shadow = std::max(1, per_sm) * num_sms();
  memo.push_back({key, m});
  return m;
}

// Everything one wave's kernels need besides where its paths come from.
struct WaveExec {
  const DScene* const* scenes;  // device scene table
  Paths P;
  int iters;                    // bounce iterations: max over the wave's scenes of max(1, max_bounce)
  bool sphere_only;
  bool field = false;           // some scene of the wave has a field medium: k_march_field runs too
  WaveCfg cfg;
  mupsi_mlp* mlp = nullptr;     // surrogate answering suspended marches (rounds > 1)
};

// The march of bounce iteration `it`: round 0, then, with a surrogate, the
// inference of the round's requests and the round that resumes them.
// The shadow jobs the shading of iteration it - 1 left (marched before the
// shading of iteration it reads the emission they add to).
void launch_shadow_pass(const WaveExec& w, const MarchLaunch& ml, int it, cudaStream_t st) {
  WaveCfg c = w.cfg;
  c.shadow_pass = 1;
  if (w.field) k_march_field<<<num_sms() * 16, 128, 0, st>>>(w.scenes, w.P, it, c);
  ml.fn_shadow<<<ml.blocks_shadow, ml.block, 0, st>>>(w.scenes, w.P, it, 0, c);
}

void launch_march_rounds(const WaveExec& w, const MarchLaunch& ml, int it, cudaStream_t st) {
  if (w.field) k_march_field<<<num_sms() * 16, 128, 0, st>>>(w.scenes, w.P, it, w.cfg);
  const int R = w.P.rounds;
  for (int r = 0; r < R; ++r) {
    ml.fn<<<ml.blocks, ml.block, 0, st>>>(w.scenes, w.P, it, r, w.cfg);
    if (r + 1 < R)
      mlp_infer_device(w.mlp, w.P.cap, reinterpret_cast<const float*>(w.P.req[r & 1]), 4, w.P.rcounts + it * R + r,
                       w.P.pred[r & 1], st);
  }
  if (w.cfg.defer && it > 0) launch_shadow_pass(w, ml, it, st);
}

// Launch one wave: clear the queue counters, generate the paths, then `iters`
// bounce iterations of march + shade. Grids do not depend on the wave's size
// (raygen and shade are grid-stride loops, the march is persistent), so the
// same launches serve every wave of a plan. `prof` (nullable) records CUDA
// events around each march and shade.
void launch_wave(const WaveExec& w, const WaveSrc& src, cudaStream_t st, mupsi_scene* prof) {
  k_wave_begin<<<1, 256, 0, st>>>(w.P, w.iters, const_cast<int*>(src.wave_idx));
  int64_t gb = (int64_t)num_sms() * 16;
  if (!src.wave_idx) gb = std::max<int64_t>(1, std::min<int64_t>(gb, (src.n + 255) / 256));
  k_raygen<<<(int)gb, 256, 0, st>>>(w.scenes, w.P, src);
  const MarchLaunch ml = march_launch(w.sphere_only, w.cfg.lane_rays != 0);
  const int sblock = g_tuning.shade_block;
  const int sb = num_sms() * (2048 / sblock);
  for (int it = 0; it < w.iters; ++it) {
    if (prof && prof->profile) {
      cudaEvent_t a = prof->next_event(), b = prof->next_event(), c = prof->next_event();
      cudaEventRecord(a, st);
      launch_march_rounds(w, ml, it, st);
      cudaEventRecord(b, st);
      k_shade<<<sb, sblock, 0, st>>>(w.scenes, w.P, it, w.cfg);
      cudaEventRecord(c, st);
      prof->ev_march.push_back({a, b});
      prof->ev_shade.push_back({b, c});
    } else {
      launch_march_rounds(w, ml, it, st);
      k_shade<<<sb, sblock, 0, st>>>(w.scenes, w.P, it, w.cfg);
    }
  }
  if (w.cfg.defer) {  // the last shading's shadow jobs
    if (prof && prof->profile) {
      cudaEvent_t a = prof->next_event(), b = prof->next_event();
      cudaEventRecord(a, st);
      launch_shadow_pass(w, ml, w.iters, st);
      cudaEventRecord(b, st);
      prof->ev_march.push_back({a, b});
    } else {
      launch_shadow_pass(w, ml, w.iters, st);
    }
  }
}
int wave_launches(int iters, int rounds = 1, bool field = false, bool defer = false) {
  return 2 + (2 * rounds + (field ? 1 : 0) + (defer ? (field ? 2 : 1) : 0)) * iters;
}

// Scenes whose medium events sample lights: their shadow rays are marched by
// the shadow passes (Paths::sh_*).
bool needs_shadow_jobs(const DScene& h) { return h.nlights > 0 && h.nmed > 0; }

// One ray per lane (lane_rays) unless a mesh mean of the scene is larger than
// lane_max_tris: a large mesh's closest-point queries are shared by lane groups.
int lane_rays_for(const DScene& S) {
  for (int i = 0; i < S.nmed; ++i)
    if (S.media[i].mean_type == MUPSI_MEAN_MESH && S.media[i].kind == MUPSI_MEDIUM_GP &&
        S.meshes[S.media[i].mesh].num_faces > g_tuning.lane_max_tris)
      return 0;
  return g_tuning.lane_rays;
}

WaveExec scene_exec(mupsi_scene* s) {
  WaveExec w;
  w.scenes = s->d_list;
  w.P = s->pb.paths;
  w.iters = wave_iters(s);
  w.sphere_only = s->h.sphere_only != 0;
  w.field = s->h.field != 0;
  w.cfg.defer = w.P.sh_a != nullptr && needs_shadow_jobs(s->h);
  w.cfg.shadow_pass = 0;
  w.cfg.min_group = g_tuning.min_group;
  w.cfg.block_rays = g_tuning.block_rays;
  w.cfg.lane_rays = lane_rays_for(s->h);
  w.cfg.mu_batch = g_tuning.mu_batch;
  w.cfg.err = s->err;
  w.cfg.counters = s->profile ? s->counters : nullptr;
  w.mlp = s->surr_mlp;
  w.P.rounds = s->surr_mlp ? s->surr_rounds : 1;  // ensure_paths sized the round buffers
  return w;
}

// One single-scene wave: n paths from pass0 (or explicit x/y/k arrays).
int run_wave(mupsi_scene* s, int64_t n, int pass0, const int32_t* xs, const int32_t* ys, const int32_t* ks,
             cudaStream_t st) {
  WaveExec w = scene_exec(s);
  WaveSrc src;
  src.n = n;
  if (xs) {
    src.xs = xs;
    src.ys = ys;
    src.ks = ks;
  } else {
    const int64_t wh = (int64_t)s->width * s->height;
    WaveChunk c{0, pass0, (int)(n / wh), s->width, 0, wh, 0};
    MUPSI_CUDA(cudaMemcpyAsync(s->d_chunk, &c, sizeof c, cudaMemcpyHostToDevice, st));
    src.chunks = s->d_chunk;
    src.nchunks = 1;
  }
  launch_wave(w, src, st, s);
  count_launch(wave_launches(w.iters, w.P.rounds, w.field, w.cfg.defer != 0));
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
    if (first && (int)s->iter_march_ms.size() < s->pb.iters) s->iter_march_ms.push_back(ms);
  }
  if (first && !s->ev_march.empty()) {
    s->iter_counts.resize(2 * (size_t)(s->pb.iters + 1));
    cudaMemcpy(s->iter_counts.data(), s->pb.paths.counts, s->iter_counts.size() * 4, cudaMemcpyDeviceToHost);
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
int64_t wave_paths() { return g_tuning.wave_paths > 0 ? g_tuning.wave_paths : kDefaultWavePaths; }

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
  P.rounds = 1;  // no surrogate rounds in the allocation-free path
  P.ms0 = P.ms1 = nullptr;
  P.req[0] = P.req[1] = nullptr;
  P.pred[0] = P.pred[1] = nullptr;
  P.rcounts = P.rcursors = nullptr;
  P.sh_a = P.sh_b = P.sh_x = P.sh_ca = P.sh_cb = nullptr;  // shadow rays marched inline
  P.sh_m = nullptr;
  P.sq[0] = P.sq[1] = nullptr;
  P.scounts = P.scursors = nullptr;
  return P;
}

}  // namespace

// ------------------------------------------------------------ batch
// Several scene instances rendered through one stream of waves. Each wave packs
// pass chunks of many instances into one path array with one shared queue per
// bounce iteration; every path carries its instance id (meta.w), so the
// persistent march balances rays of all instances over the whole GPU. The
// wave plan (chunks and per-wave ranges) is uploaded once per render and a
// device wave index steps through it, so one captured graph per bounce count
// replays every wave.
namespace {
struct BatchGraph {
  int iters;
  cudaGraphExec_t exec;
};
}  // namespace

struct mupsi_batch {
  std::vector<mupsi_scene*> inst;
  DScene** d_list = nullptr;
  float** d_sums = nullptr;
  int* d_wave_idx = nullptr;
  int* err = nullptr;
  WaveChunk* d_chunks = nullptr;
  size_t chunk_cap = 0;
  WaveDesc* d_waves = nullptr;
  size_t wave_cap = 0;
  PathBuf pb;
  bool sphere_only = true;     // k_march variant for every instance
  bool field = false;          // some instance has a field medium
  bool shadow = false;         // some instance leaves shadow jobs
  cudaStream_t bs = nullptr;  // graphs are captured and replayed on this stream
  std::vector<BatchGraph> graphs;
  mupsi_tuning graph_tuning{};  // launch shapes the graphs were captured with
  std::vector<cudaEvent_t> events;
  mupsi_batch_info info{};
  void drop_graphs() {
    for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
    graphs.clear();
  }
  ~mupsi_batch() {
    drop_graphs();
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    if (bs) cudaStreamDestroy(bs);
    if (d_list) cudaFree(d_list);
    if (d_sums) cudaFree(d_sums);
    if (d_wave_idx) cudaFree(d_wave_idx);
    if (err) cudaFree(err);
    if (d_chunks) cudaFree(d_chunks);
    if (d_waves) cudaFree(d_waves);
    if (pb.mem) pool_give(pb.mem, pb.bytes);
  }
};

namespace {

template <typename T>
int grow_device(T*& ptr, size_t& cap, size_t need, bool& moved) {
  if (need <= cap) return MUPSI_OK;
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = std::max(need, 2 * cap);
  MUPSI_CUDA(cudaMalloc((void**)&ptr, cap * sizeof(T)));
  moved = true;
  return MUPSI_OK;
}

int batch_lane_rays(const mupsi_batch* b) {
  int lr = g_tuning.lane_rays;
  for (const mupsi_scene* s : b->inst) lr = std::min(lr, lane_rays_for(s->h));
  return lr;
}

// One wave of the plan on stream bs: paths, bounces, accumulation.
void batch_wave_launches(mupsi_batch* b, int iters) {
  WaveExec w;
  w.scenes = b->d_list;
  w.P = b->pb.paths;
  w.iters = iters;
  w.sphere_only = b->sphere_only;
  w.field = b->field;
  w.cfg.defer = b->shadow && w.P.sh_a != nullptr;
  w.cfg.shadow_pass = 0;
  w.cfg.min_group = g_tuning.min_group;
  w.cfg.block_rays = g_tuning.block_rays;
  w.cfg.lane_rays = batch_lane_rays(b);
  w.cfg.mu_batch = g_tuning.mu_batch;
  w.cfg.err = b->err;
  w.cfg.counters = nullptr;
  WaveSrc src;
  src.chunks = b->d_chunks;
  src.waves = b->d_waves;
  src.wave_idx = b->d_wave_idx;
  launch_wave(w, src, b->bs, nullptr);
  k_accumulate_wave<<<num_sms() * 16, 128, 0, b->bs>>>(b->pb.paths.rad, src, b->d_sums);
}

bool same_tuning(const mupsi_tuning& a, const mupsi_tuning& c) {
  return a.march_block == c.march_block && a.min_group == c.min_group && a.shade_block == c.shade_block &&
         a.block_rays == c.block_rays && a.lane_rays == c.lane_rays && a.lane_max_tris == c.lane_max_tris &&
         a.mu_batch == c.mu_batch;
}

// The graph of a wave with `iters` bounce iterations, captured on first use.
// The instances' medium flags as they are now; graphs captured under others go.
void batch_flags(mupsi_batch* b) {
  bool so = true, fd = false, sh = false;
  for (mupsi_scene* s : b->inst) {
    so = so && s->h.sphere_only != 0;
    fd = fd || s->h.field != 0;
    sh = sh || needs_shadow_jobs(s->h);
  }
  if (so != b->sphere_only || fd != b->field || sh != b->shadow) b->drop_graphs();
  b->sphere_only = so;
  b->field = fd;
  b->shadow = sh;
}

int batch_graph(mupsi_batch* b, int iters, cudaGraphExec_t* out) {
  if (!same_tuning(b->graph_tuning, g_tuning)) {
    b->drop_graphs();
    b->graph_tuning = g_tuning;
  }
  for (auto& g : b->graphs)
    if (g.iters == iters) {
      *out = g.exec;
      return MUPSI_OK;
    }
  march_launch(b->sphere_only, batch_lane_rays(b) != 0);  // occupancy query outside the capture
  cudaGraph_t graph = nullptr;
  MUPSI_CUDA(cudaStreamBeginCapture(b->bs, cudaStreamCaptureModeThreadLocal));
  batch_wave_launches(b, iters);
  cudaError_t e = cudaStreamEndCapture(b->bs, &graph);
  if (e != cudaSuccess) return fail(MUPSI_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail(MUPSI_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  b->graphs.push_back({iters, exec});
  b->info.graphs_captured++;
  *out = exec;
  return MUPSI_OK;
}

int check_batch_err(mupsi_batch* b) {
  int h = 0;
  MUPSI_CUDA(cudaMemcpy(&h, b->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    cudaMemset(b->err, 0, sizeof(int));
    if (h & ERR_BVH_STACK) return fail(MUPSI_ERR_DEVICE_LIMIT, "BVH traversal exceeded the 64-entry stack");
    return fail(MUPSI_ERR_DEVICE_LIMIT, "march iteration cap reached");
  }
  for (mupsi_scene* s : b->inst)
    if (int e = check_err(s, b->bs)) return e;
  return MUPSI_OK;
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

int mupsi_gpu_transmittance(const mupsi_scene* scene, int32_t medium, int64_t n, const mupsi_ray* rays,
                            const uint32_t* seed, const mupsi_cond* cond, float* out, mupsi_mem mem, void* stream) {
  clear_error();
  if (!scene || medium < 0 || medium >= scene->h.nmed || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!rays || !seed || !out) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<mupsi_ray> dr(st);
  Staged<uint32_t> ds(st);
  Staged<mupsi_cond> dc(st);
  Staged<float> dout(st);
  MUPSI_CUDA(dr.in(rays, n, mem));
  MUPSI_CUDA(ds.in(seed, n, mem));
  if (cond) MUPSI_CUDA(dc.in(cond, n, mem));
  MUPSI_CUDA(dout.out(out, n, mem));
  k_transmittance<<<grid_n(n), 128, 0, st>>>(scene->d, medium, n, dr.ptr, ds.ptr,
                                             cond ? reinterpret_cast<const Cond*>(dc.ptr) : nullptr, dout.ptr);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dout.finish());
  return check_err(const_cast<mupsi_scene*>(scene), st);
}

int mupsi_gpu_sample_condition(const mupsi_scene* scene, int32_t medium, int64_t n, const mupsi_medium_sample* samples,
                               const uint32_t* seed, mupsi_cond* out, mupsi_mem mem, void* stream) {
  clear_error();
  if (scene && medium >= 0 && medium < scene->h.nmed && scene->h.media[medium].kind != MUPSI_MEDIUM_GP)
    return fail(MUPSI_ERR_INVALID, "only a GP medium conditions");
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
    MUPSI_CUDA(cudaMemcpyAsync(out_rgb, scene->pb.paths.rad, n * 12, cudaMemcpyDeviceToDevice, st));
  } else {
    MUPSI_CUDA(cudaMemcpyAsync(out_rgb, scene->pb.paths.rad, n * 12, cudaMemcpyDeviceToHost, st));
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
  int per_wave = (int)std::max<int64_t>(1, std::min<int64_t>(total, wave_paths() / wh));
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
    k_accumulate<<<grid_n(wh), 128, 0, st>>>(scene->pb.paths.rad, passes, wh, scene->sum, dmom);
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
      if (!scene->avg) MUPSI_CUDA(dev_take((void**)&scene->avg, wh * 12));
      k_average<<<grid_n(wh * 3), 128, 0, st>>>(scene->sum, wh * 3, inv, scene->avg);
      count_launch();
      MUPSI_CUDA(cudaMemcpyAsync(a->rgb_out, scene->avg, wh * 12, cudaMemcpyDeviceToHost, st));
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
// reference): same kernels, path state in the library's static scratch array,
// device buffers of the current device only, at most kNoAllocMaxSamples
// samples. Without surrogate rounds (P.rounds = 1) a scene's surrogate is not
// consulted, so results equal mupsi_gpu_trace_samples' for scenes without one.
int mupsi_gpu_trace_samples_noalloc(mupsi_scene* scene, int64_t n, const int32_t* x, const int32_t* y,
                                    const int32_t* k, float* out_rgb, void* stream) {
  clear_error();
  if (!scene || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n > kNoAllocMaxSamples)
    return fail(MUPSI_ERR_INVALID, "trace_samples_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                                       std::to_string(kNoAllocMaxSamples) + " samples per call");
  if (n == 0) return MUPSI_OK;
  if (!x || !y || !k || !out_rgb) return fail(MUPSI_ERR_INVALID, "null buffer");
  int cur_dev = 0;
  MUPSI_CUDA(cudaGetDevice(&cur_dev));
  for (const void* ptr : {(const void*)x, (const void*)y, (const void*)k, (const void*)out_rgb}) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess || at.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      return fail(MUPSI_ERR_INVALID, "trace_samples_noalloc takes device buffers only");
    }
    // the kernels run on the current device; another GPU's buffer would be
    // reached without peer access
    if (at.device != cur_dev)
      return fail(MUPSI_ERR_INVALID, "trace_samples_noalloc: buffer on device " + std::to_string(at.device) +
                                         ", current device " + std::to_string(cur_dev));
  }
  void* scratch = nullptr;
  if (int e = noalloc_scratch(&scratch)) return e;
  cudaStream_t st = (cudaStream_t)stream;  // NULL: the default stream (no stream is created here)
  WaveExec w = scene_exec(scene);
  w.P = noalloc_paths(scratch);  // launch_wave clears its queue counters and cursors
  w.cfg.defer = 0;               // no shadow-job buffers here: shadow rays are marched inline
  WaveSrc src;
  src.n = n;
  src.xs = x;
  src.ys = y;
  src.ks = k;
  launch_wave(w, src, st, nullptr);
  count_launch(wave_launches(w.iters, 1, w.field));
  MUPSI_CUDA(cudaGetLastError());
  const Paths& P = w.P;
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
  // enable == 2 also tallies BVH work (counted copies of the traversals)
  for (int i = 0; i < scene->h.nmesh; ++i) scene->h.meshes[i].count = enable == 2 ? scene->counters + 8 : nullptr;
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_scene_stats(mupsi_scene* scene, mupsi_render_stats* out, int32_t reset) {
  clear_error();
  if (!scene || !out) return fail(MUPSI_ERR_INVALID, "null argument");
  MUPSI_CUDA(cudaDeviceSynchronize());
  collect_events(scene);
  unsigned long long c[kSceneCounters] = {};
  MUPSI_CUDA(cudaMemcpy(c, scene->counters, sizeof c, cudaMemcpyDeviceToHost));
  out->bvh_nodes = out->bvh_tris = 0;
  for (int i = 0; i < kBvhCountSlots; ++i) {
    out->bvh_nodes += c[8 + 2 * i];
    out->bvh_tris += c[9 + 2 * i];
  }
  out->march_steps = c[0];
  out->psi_evals = c[1];
  out->marches = c[2];
  out->impulse_evals = c[3];
  out->mean_evals = c[4];
  out->parity_casts = c[5];
  out->surr_requests = c[6];
  out->surr_accepted = c[7];
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

int mupsi_gpu_set_tuning(const mupsi_tuning* t) {
  clear_error();
  if (!t) return fail(MUPSI_ERR_INVALID, "null tuning");
  if (t->march_block < 32 || t->march_block > 128 || t->march_block % 32)
    return fail(MUPSI_ERR_INVALID, "march_block must be 32, 64, 96 or 128");
  if (t->min_group < 4 || t->min_group > 32 || (t->min_group & (t->min_group - 1)))
    return fail(MUPSI_ERR_INVALID, "min_group must be 4, 8, 16 or 32");
  if (t->shade_block < 32 || t->shade_block > 128 || t->shade_block % 32)
    return fail(MUPSI_ERR_INVALID, "shade_block must be a multiple of 32 in [32, 128]");
  if (t->wave_paths < 0 || t->wave_paths > (1 << 28)) return fail(MUPSI_ERR_INVALID, "wave_paths out of range");
  if (t->block_rays < 0 || t->block_rays > 256) return fail(MUPSI_ERR_INVALID, "block_rays must be in [0, 256]");
  if (t->lane_rays < 0 || t->lane_rays > 64) return fail(MUPSI_ERR_INVALID, "lane_rays must be in [0, 64]");
  if (t->lane_max_tris < 0) return fail(MUPSI_ERR_INVALID, "lane_max_tris must be >= 0");
  if (t->mu_batch < 0 || t->mu_batch > 32) return fail(MUPSI_ERR_INVALID, "mu_batch must be in [0, 32]");
  g_tuning = *t;
  return MUPSI_OK;
}

int mupsi_gpu_get_tuning(mupsi_tuning* out) {
  clear_error();
  if (!out) return fail(MUPSI_ERR_INVALID, "null argument");
  *out = g_tuning;
  return MUPSI_OK;
}

int mupsi_gpu_batch_create(int32_t num_scenes, mupsi_scene* const* scenes, mupsi_batch** out) {
  clear_error();
  if (!out) return fail(MUPSI_ERR_INVALID, "null argument");
  *out = nullptr;
  if (num_scenes <= 0 || !scenes) return fail(MUPSI_ERR_INVALID, "a batch needs at least one scene");
  if (num_scenes > (1 << 20)) return fail(MUPSI_ERR_INVALID, "at most 2^20 scenes per batch");
  std::unique_ptr<mupsi_batch> b(new mupsi_batch);
  std::vector<DScene*> list;
  std::vector<float*> sums;
  for (int i = 0; i < num_scenes; ++i) {
    if (!scenes[i]) return fail(MUPSI_ERR_INVALID, "null scene in batch");
    b->inst.push_back(scenes[i]);
    list.push_back(scenes[i]->d);
    sums.push_back(scenes[i]->sum);
  }
  MUPSI_CUDA(cudaMalloc((void**)&b->d_list, list.size() * sizeof(DScene*)));
  MUPSI_CUDA(cudaMemcpy(b->d_list, list.data(), list.size() * sizeof(DScene*), cudaMemcpyHostToDevice));
  MUPSI_CUDA(cudaMalloc((void**)&b->d_sums, sums.size() * sizeof(float*)));
  MUPSI_CUDA(cudaMemcpy(b->d_sums, sums.data(), sums.size() * sizeof(float*), cudaMemcpyHostToDevice));
  MUPSI_CUDA(cudaMalloc((void**)&b->d_wave_idx, sizeof(int)));
  MUPSI_CUDA(cudaMalloc((void**)&b->err, sizeof(int)));
  MUPSI_CUDA(cudaMemset(b->err, 0, sizeof(int)));
  MUPSI_CUDA(cudaStreamCreateWithFlags(&b->bs, cudaStreamNonBlocking));
  *out = b.release();
  return MUPSI_OK;
}

int mupsi_gpu_batch_destroy(mupsi_batch* batch) {
  clear_error();
  if (!batch) return MUPSI_OK;
  cudaStreamSynchronize(batch->bs);
  delete batch;
  return MUPSI_OK;
}

int mupsi_gpu_batch_info(const mupsi_batch* batch, mupsi_batch_info* out) {
  clear_error();
  if (!batch || !out) return fail(MUPSI_ERR_INVALID, "null argument");
  *out = batch->info;
  return MUPSI_OK;
}

int mupsi_gpu_batch_render(mupsi_batch* b, const mupsi_batch_args* a) {
  clear_error();
  if (!b || !a || !a->spp) return fail(MUPSI_ERR_INVALID, "null argument");
  const int n = (int)b->inst.size();
  for (int i = 0; i < n; ++i)
    if (a->spp[i] < 0) return fail(MUPSI_ERR_INVALID, "negative spp");
  if (a->schedule != MUPSI_SCHEDULE_SHORTEST_FIRST && a->schedule != MUPSI_SCHEDULE_IN_ORDER &&
      a->schedule != MUPSI_SCHEDULE_INTERLEAVED)
    return fail(MUPSI_ERR_INVALID, "unknown schedule");
  b->info.waves = b->info.graph_launches = b->info.max_iters = 0;
  b->info.paths = 0;
  batch_flags(b);
  // ---- plan: instances in schedule order, their passes packed into waves of
  // at most wave_paths() paths (a pass is never split across waves)
  std::vector<int> order(n);
  for (int i = 0; i < n; ++i) order[i] = i;
  auto work = [&](int i) { return (int64_t)a->spp[i] * b->inst[i]->width * b->inst[i]->height; };
  if (a->schedule == MUPSI_SCHEDULE_SHORTEST_FIRST)
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return work(x) < work(y); });
  const int64_t W = wave_paths();
  // interleaved: every wave takes a share of every instance's passes, so all
  // instances progress together and complete in the last wave; K = total / W
  // waves, instance i contributing about spp_i / K passes to each (a wave can
  // exceed W by the passes rounding up; the path buffers are sized to the
  // largest wave)
  int K = 1;
  if (a->schedule == MUPSI_SCHEDULE_INTERLEAVED) {
    int64_t total = 0;
    for (int i = 0; i < n; ++i) total += work(i);
    K = (int)std::min<int64_t>(1 << 16, std::max<int64_t>(1, (total + W - 1) / W));
  }
  std::vector<WaveChunk> chunks;
  std::vector<WaveDesc> waves;
  std::vector<int> wave_iters_v, last_wave(n, -1);
  WaveDesc cur{0, 0, 0, 0};
  int cur_iters = 0;
  auto close_wave = [&]() {
    if (cur.nchunks == 0) return;
    waves.push_back(cur);
    wave_iters_v.push_back(cur_iters);
    cur = WaveDesc{0, 0, (int)chunks.size(), 0};
    cur_iters = 0;
  };
  if (a->schedule == MUPSI_SCHEDULE_INTERLEAVED) {
    for (int k = 0; k < K; ++k) {
      for (int i = 0; i < n; ++i) {
        mupsi_scene* s = b->inst[i];
        const int64_t wh = (int64_t)s->width * s->height;
        const int p0 = (int)((int64_t)a->spp[i] * k / K), p1 = (int)((int64_t)a->spp[i] * (k + 1) / K);
        if (p1 <= p0) continue;
        chunks.push_back(WaveChunk{i, p0, p1 - p0, s->width, cur.n, wh, cur.npix});
        cur.n += (int64_t)(p1 - p0) * wh;
        cur.npix += wh;
        cur.nchunks++;
        cur_iters = std::max(cur_iters, wave_iters(s));
        last_wave[i] = (int)waves.size();
      }
      close_wave();
    }
    order.clear();  // planned
  }
  for (int i : order) {
    mupsi_scene* s = b->inst[i];
    const int64_t wh = (int64_t)s->width * s->height;
    int pass = 0;
    while (pass < a->spp[i]) {
      int64_t fit = (W - cur.n) / wh;
      if (fit <= 0) {
        if (cur.n > 0) {
          close_wave();
          continue;
        }
        fit = 1;
      }
      const int take = (int)std::min<int64_t>(fit, a->spp[i] - pass);
      chunks.push_back(WaveChunk{i, pass, take, s->width, cur.n, wh, cur.npix});
      cur.n += (int64_t)take * wh;
      cur.npix += wh;
      cur.nchunks++;
      cur_iters = std::max(cur_iters, wave_iters(s));
      pass += take;
      last_wave[i] = (int)waves.size();
    }
  }
  close_wave();
  // ---- buffers
  int64_t max_n = 0;
  int max_it = 0;
  for (size_t w = 0; w < waves.size(); ++w) {
    max_n = std::max(max_n, waves[w].n);
    max_it = std::max(max_it, wave_iters_v[w]);
  }
  bool moved = false;
  if (!waves.empty()) {
    if (max_n > b->pb.cap || max_it + 1 > b->pb.iters) moved = true;
    if (int e = ensure_paths(b->pb, max_n, max_it + 1, 1, b->shadow)) return e;
    if (int e = grow_device(b->d_chunks, b->chunk_cap, chunks.size(), moved)) return e;
    if (int e = grow_device(b->d_waves, b->wave_cap, waves.size(), moved)) return e;
  }
  if (moved) b->drop_graphs();
  // events[0]: start of the first wave; events[1 + w]: end of wave w
  while (b->events.size() < waves.size() + 1) {
    cudaEvent_t e;
    MUPSI_CUDA(cudaEventCreate(&e));
    b->events.push_back(e);
  }
  cudaStream_t st = resolve_stream(a->stream);
  // the batch stream starts after the caller's stream's earlier work
  MUPSI_CUDA(cudaEventRecord(b->events[0], st));
  MUPSI_CUDA(cudaStreamWaitEvent(b->bs, b->events[0], 0));
  cudaStream_t bs = b->bs;
  if (!waves.empty()) {
    MUPSI_CUDA(cudaMemcpyAsync(b->d_chunks, chunks.data(), chunks.size() * sizeof(WaveChunk), cudaMemcpyHostToDevice, bs));
    MUPSI_CUDA(cudaMemcpyAsync(b->d_waves, waves.data(), waves.size() * sizeof(WaveDesc), cudaMemcpyHostToDevice, bs));
  }
  for (int i = 0; i < n; ++i) {
    mupsi_scene* s = b->inst[i];
    if (a->spp[i] > 0) MUPSI_CUDA(cudaMemsetAsync(s->sum, 0, (size_t)s->width * s->height * 12, bs));
    s->passes_done = a->spp[i];
    s->next_pass = a->spp[i];
  }
  MUPSI_CUDA(cudaMemsetAsync(b->d_wave_idx, 0xff, sizeof(int), bs));  // -1: k_wave_begin steps to 0
  MUPSI_CUDA(cudaEventRecord(b->events[0], bs));
  int rc = MUPSI_OK;
  for (size_t w = 0; w < waves.size(); ++w) {
    if (a->cancel && *a->cancel) {
      rc = fail(MUPSI_ERR_CANCELLED, "render cancelled");
      break;
    }
    const int iters = wave_iters_v[w];
    if (a->use_graphs) {
      cudaGraphExec_t exec = nullptr;
      if ((rc = batch_graph(b, iters, &exec))) break;
      cudaError_t e = cudaGraphLaunch(exec, bs);
      if (e != cudaSuccess) {
        rc = fail(MUPSI_ERR_CUDA, std::string("graph launch: ") + cudaGetErrorString(e));
        break;
      }
      b->info.graph_launches++;
    } else {
      batch_wave_launches(b, iters);
    }
    count_launch(wave_launches(iters, 1, b->field, b->shadow) + 1);
    b->info.waves++;
    b->info.max_iters = std::max(b->info.max_iters, iters);
    b->info.paths += waves[w].n;
    MUPSI_CUDA(cudaEventRecord(b->events[1 + w], bs));
  }
  if (rc == MUPSI_OK) {
    MUPSI_CUDA(cudaGetLastError());
    for (int i = 0; i < n; ++i) {
      mupsi_scene* s = b->inst[i];
      if (!a->rgb_out || !a->rgb_out[i] || a->spp[i] == 0) continue;
      const int64_t wh = (int64_t)s->width * s->height;
      const float inv = 1.0f / (float)a->spp[i];
      if (a->out_mem == MUPSI_MEM_DEVICE) {
        k_average<<<grid_n(wh * 3), 128, 0, bs>>>(s->sum, wh * 3, inv, a->rgb_out[i]);
        count_launch();
      } else {
        if (!s->avg) MUPSI_CUDA(dev_take((void**)&s->avg, wh * 12));
        k_average<<<grid_n(wh * 3), 128, 0, bs>>>(s->sum, wh * 3, inv, s->avg);
        count_launch();
        MUPSI_CUDA(cudaMemcpyAsync(a->rgb_out[i], s->avg, wh * 12, cudaMemcpyDeviceToHost, bs));
      }
    }
  }
  MUPSI_CUDA(cudaStreamSynchronize(bs));
  if (rc == MUPSI_OK && a->done_ms) {
    for (int i = 0; i < n; ++i) {
      float ms = 0.0f;
      if (last_wave[i] >= 0) MUPSI_CUDA(cudaEventElapsedTime(&ms, b->events[0], b->events[1 + last_wave[i]]));
      a->done_ms[i] = ms;
    }
  }
  int e = check_batch_err(b);
  return rc ? rc : e;
}

int mupsi_gpu_scene_set_surrogate(mupsi_scene* scene, int32_t medium, mupsi_mlp* mlp, float band, float scale,
                                  float margin, int32_t max_requests) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  if (medium < 0 || medium >= scene->h.nmed) return fail(MUPSI_ERR_INVALID, "medium out of range");
  DMedium& md = scene->h.media[medium];
  if (mlp) {
    if (md.mean_type != MUPSI_MEAN_MESH || md.kind != MUPSI_MEDIUM_GP)
      return fail(MUPSI_ERR_INVALID, "the surrogate stands in for a GP medium's mesh mean");
    if (!(band >= 0.0f) || !(scale >= 1.0f) || !(margin >= 0.0f) || !std::isfinite(band) || !std::isfinite(scale) ||
        !std::isfinite(margin))
      return fail(MUPSI_ERR_INVALID, "need band >= 0, scale >= 1, margin >= 0");
    if (max_requests < 1 || max_requests > 32) return fail(MUPSI_ERR_INVALID, "max_requests must be in [1, 32]");
    for (int i = 0; i < scene->h.nmed; ++i)
      if (i != medium) scene->h.media[i].surr = 0;  // one surrogate per scene
    md.surr = 1;
    md.surr_max = max_requests;
    md.surr_band = band;
    md.surr_scale = scale;
    md.surr_add = margin;
    scene->surr_mlp = mlp;
    scene->surr_rounds = max_requests + 1;
  } else {
    md.surr = 0;
    bool any = false;
    for (int i = 0; i < scene->h.nmed; ++i) any = any || scene->h.media[i].surr;
    if (!any) {
      scene->surr_mlp = nullptr;
      scene->surr_rounds = 1;
    }
  }
  MUPSI_CUDA(cudaDeviceSynchronize());
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_scene_set_mean_eval(mupsi_scene* scene, int32_t medium, int32_t mode) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  if (medium < 0 || medium >= scene->h.nmed) return fail(MUPSI_ERR_INVALID, "medium out of range");
  if (mode != MUPSI_MEAN_EVAL_LAZY && mode != MUPSI_MEAN_EVAL_EVERY_STEP)
    return fail(MUPSI_ERR_INVALID, "unknown mean evaluation mode");
  if (scene->h.media[medium].kind != MUPSI_MEDIUM_GP) return fail(MUPSI_ERR_INVALID, "not a GP medium");
  scene->h.media[medium].every_step = mode == MUPSI_MEAN_EVAL_EVERY_STEP;
  MUPSI_CUDA(cudaDeviceSynchronize());
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_scene_set_occlusion(mupsi_scene* scene, int32_t mode) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  if (mode != MUPSI_OCCLUSION_REFERENCE && mode != MUPSI_OCCLUSION_ROOT)
    return fail(MUPSI_ERR_INVALID, "unknown occlusion mode");
  for (int i = 0; i < scene->h.nmesh; ++i)
    scene->h.meshes[i].occl_start = mode == MUPSI_OCCLUSION_ROOT ? scene->h.meshes[i].root : scene->h.meshes[i].occl_ref;
  MUPSI_CUDA(cudaDeviceSynchronize());
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_scene_set_sky_texture(mupsi_scene* scene, int32_t width, int32_t height, const float* rgb) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  if (width < 0 || height < 0 || width > (1 << 15) || height > (1 << 15))
    return fail(MUPSI_ERR_INVALID, "sky texture size out of range");
  if ((width == 0) != (height == 0)) return fail(MUPSI_ERR_INVALID, "sky texture needs width and height");
  if (width > 0 && !rgb) return fail(MUPSI_ERR_INVALID, "null sky texels");
  MUPSI_CUDA(cudaDeviceSynchronize());
  if (scene->sky_mem) {
    cudaFree(scene->sky_mem);
    scene->sky_mem = nullptr;
  }
  scene->h.sky_tex = nullptr;
  scene->h.sky_w = scene->h.sky_h = 0;
  if (width > 0) {
    const size_t bytes = (size_t)width * height * 3 * sizeof(float);
    MUPSI_CUDA(cudaMalloc(&scene->sky_mem, bytes));
    MUPSI_CUDA(cudaMemcpy(scene->sky_mem, rgb, bytes, cudaMemcpyHostToDevice));
    scene->h.sky_tex = static_cast<const float*>(scene->sky_mem);
    scene->h.sky_w = width;
    scene->h.sky_h = height;
  }
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_release_pools(void) {
  clear_error();
  MUPSI_CUDA(cudaDeviceSynchronize());
  pool_release();
  dev_cache_release();
  return MUPSI_OK;
}

int mupsi_gpu_scene_get_size(const mupsi_scene* scene, int32_t* width, int32_t* height) {
  clear_error();
  if (!scene || !width || !height) return fail(MUPSI_ERR_INVALID, "null argument");
  *width = scene->width;
  *height = scene->height;
  return MUPSI_OK;
}

int mupsi_gpu_scene_set_gp_mode(mupsi_scene* scene, int32_t mode) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  if (mode != MUPSI_GP_SINGLE_REALIZATION && mode != MUPSI_GP_RENEWAL_PLUS) return fail(MUPSI_ERR_INVALID, "bad gp_mode");
  MUPSI_CUDA(cudaDeviceSynchronize());
  scene->h.gp_mode = mode;
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_scene_set_skip_medium(mupsi_scene* scene, int32_t skip) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  MUPSI_CUDA(cudaDeviceSynchronize());
  scene->h.skip_medium = skip ? 1 : 0;
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_scene_set_kernel(mupsi_scene* scene, int32_t medium, const mupsi_kernel* kernel) {
  clear_error();
  if (!scene || !kernel) return fail(MUPSI_ERR_INVALID, "null argument");
  if (medium < 0 || medium >= scene->h.nmed) return fail(MUPSI_ERR_INVALID, "medium out of range");
  if (int e = check_kernel(kernel)) return e;
  MUPSI_CUDA(cudaDeviceSynchronize());
  scene->h.media[medium].k = make_kparams(*kernel);
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

// The k_march variant: sphere means only among the GP media (field media are
// marched by k_march_field, which handles every mean).
static void update_medium_flags(DScene& S) {
  S.sphere_only = 1;
  S.field = 0;
  for (int i = 0; i < S.nmed; ++i) {
    if (S.media[i].kind != MUPSI_MEDIUM_GP)
      S.field = 1;
    else if (S.media[i].mean_type != MUPSI_MEAN_SPHERE)
      S.sphere_only = 0;
  }
}

int mupsi_gpu_scene_set_sdf_medium(mupsi_scene* scene, int32_t medium) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  if (medium < 0 || medium >= scene->h.nmed) return fail(MUPSI_ERR_INVALID, "medium out of range");
  if (scene->surr_mlp && scene->h.media[medium].surr) return fail(MUPSI_ERR_INVALID, "medium has a surrogate");
  MUPSI_CUDA(cudaDeviceSynchronize());
  DMedium& md = scene->h.media[medium];
  md.kind = MUPSI_MEDIUM_SDF;
  md.every_step = 0;
  update_medium_flags(scene->h);
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_scene_set_external_gp_medium(mupsi_scene* scene, int32_t medium, int32_t resolution,
                                           const float bounds_min[3], const float bounds_max[3],
                                           const float* mean_grid, const float* variance_grid, float noise_scale) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  if (medium < 0 || medium >= scene->h.nmed) return fail(MUPSI_ERR_INVALID, "medium out of range");
  if (scene->surr_mlp && scene->h.media[medium].surr) return fail(MUPSI_ERR_INVALID, "medium has a surrogate");
  if (resolution < 2 || resolution > 1024) return fail(MUPSI_ERR_INVALID, "resolution must be in [2, 1024]");
  if (!bounds_min || !bounds_max || !mean_grid) return fail(MUPSI_ERR_INVALID, "null argument");
  if (!std::isfinite(noise_scale)) return fail(MUPSI_ERR_INVALID, "bad noise scale");
  v3 bmin = ld3(bounds_min), bmax = ld3(bounds_max);
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(get(bmin, a)) || !std::isfinite(get(bmax, a)) || !(get(bmax, a) > get(bmin, a)))
      return fail(MUPSI_ERR_INVALID, "need finite bounds_min < bounds_max");
  MUPSI_CUDA(cudaDeviceSynchronize());
  if (scene->grid_mem[medium]) {
    cudaFree(scene->grid_mem[medium]);
    scene->grid_mem[medium] = nullptr;
  }
  const size_t cells = (size_t)resolution * resolution * resolution;
  float* mem = nullptr;
  MUPSI_CUDA(cudaMalloc(&mem, cells * sizeof(float) * (variance_grid ? 2 : 1)));
  scene->grid_mem[medium] = mem;
  MUPSI_CUDA(cudaMemcpy(mem, mean_grid, cells * sizeof(float), cudaMemcpyHostToDevice));
  if (variance_grid) MUPSI_CUDA(cudaMemcpy(mem + cells, variance_grid, cells * sizeof(float), cudaMemcpyHostToDevice));
  DMedium& md = scene->h.media[medium];
  md.kind = MUPSI_MEDIUM_EXTERNAL_GP;
  md.every_step = 0;
  // inv_cell_size_ = (res, res, res) / (bmax - bmin) (meanfunction.cpp:44)
  const float r = (float)resolution;
  const v3 inv = mk3(r / (bmax.x - bmin.x), r / (bmax.y - bmin.y), r / (bmax.z - bmin.z));
  md.gmean = DGrid{mem, resolution, bmin, inv};
  md.gvar = DGrid{variance_grid ? mem + cells : nullptr, resolution, bmin, inv};
  md.noise_scale = noise_scale;
  update_medium_flags(scene->h);
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

int mupsi_gpu_scene_set_albedo_texture(mupsi_scene* scene, int32_t primitive, int64_t num_texcoords,
                                       const float* texcoords, const int32_t* face_texcoords, int32_t width,
                                       int32_t height, const float* rgb) {
  clear_error();
  if (!scene) return fail(MUPSI_ERR_INVALID, "null scene");
  if (primitive < 0 || primitive >= scene->h.nprim) return fail(MUPSI_ERR_INVALID, "primitive out of range");
  DPrim& p = scene->h.prims[primitive];
  if (p.type != MUPSI_PRIM_MESH) return fail(MUPSI_ERR_INVALID, "albedo textures are on mesh primitives");
  if (p.bsdf != MUPSI_BSDF_LAMBERTIAN) return fail(MUPSI_ERR_INVALID, "albedo textures need a Lambertian BSDF");
  if (width < 0 || height < 0 || width > (1 << 15) || height > (1 << 15))
    return fail(MUPSI_ERR_INVALID, "albedo texture size out of range");
  if ((width == 0) != (height == 0)) return fail(MUPSI_ERR_INVALID, "albedo texture needs width and height");
  const int64_t nf = scene->h.meshes[p.mesh].num_faces;
  if (width > 0) {
    if (!rgb) return fail(MUPSI_ERR_INVALID, "null albedo texels");
    if (num_texcoords < 0 || num_texcoords > (int64_t(1) << 28)) return fail(MUPSI_ERR_INVALID, "bad texcoord count");
    if (num_texcoords > 0) {
      if (!texcoords || !face_texcoords) return fail(MUPSI_ERR_INVALID, "null texcoords");
      for (int64_t i = 0; i < 3 * nf; ++i)
        if (face_texcoords[i] < 0 || face_texcoords[i] >= num_texcoords)
          return fail(MUPSI_ERR_INVALID, "face texcoord index out of range");
    }
  }
  MUPSI_CUDA(cudaDeviceSynchronize());
  if (scene->tex_mem[primitive]) {
    cudaFree(scene->tex_mem[primitive]);
    scene->tex_mem[primitive] = nullptr;
  }
  p.tex = nullptr;
  p.uvs = nullptr;
  p.face_uv = nullptr;
  p.tex_w = p.tex_h = 0;
  if (width > 0) {
    auto up16 = [](size_t b) { return (b + 15) & ~size_t(15); };
    const size_t tb = up16((size_t)width * height * 3 * sizeof(float));
    const size_t ub = num_texcoords > 0 ? up16((size_t)num_texcoords * 2 * sizeof(float)) : 0;
    const size_t fb = num_texcoords > 0 ? (size_t)nf * 3 * sizeof(int32_t) : 0;
    char* mem = nullptr;
    MUPSI_CUDA(cudaMalloc(&mem, tb + ub + fb));
    scene->tex_mem[primitive] = mem;
    MUPSI_CUDA(cudaMemcpy(mem, rgb, (size_t)width * height * 3 * sizeof(float), cudaMemcpyHostToDevice));
    p.tex = reinterpret_cast<const float*>(mem);
    p.tex_w = width;
    p.tex_h = height;
    if (num_texcoords > 0) {
      MUPSI_CUDA(cudaMemcpy(mem + tb, texcoords, (size_t)num_texcoords * 2 * sizeof(float), cudaMemcpyHostToDevice));
      MUPSI_CUDA(cudaMemcpy(mem + tb + ub, face_texcoords, fb, cudaMemcpyHostToDevice));
      p.uvs = reinterpret_cast<const float*>(mem + tb);
      p.face_uv = reinterpret_cast<const int32_t*>(mem + tb + ub);
    }
  }
  MUPSI_CUDA(cudaMemcpy(scene->d, &scene->h, sizeof(DScene), cudaMemcpyHostToDevice));
  return MUPSI_OK;
}

}  // extern "C"
