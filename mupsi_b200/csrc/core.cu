// Library core: error state, launch accounting, transforms, the batched GP-noise
// entry points and the mesh/BVH entry points of include/mupsi_gpu.h.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "core.cuh"

namespace mupsi {

constexpr int kWideRowsHost = 8;  // float4 rows of a four-wide node (DMesh::wide)
static thread_local std::string g_last_error;
static std::atomic<int64_t> g_launches{0};

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
void clear_error() { g_last_error.clear(); }
void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

HostM4 translate_scale(const float t[3], float s) {
  HostM4 r;
  std::memset(r.m, 0, sizeof r.m);
  r.m[0] = s;
  r.m[5] = s;
  r.m[10] = s;
  r.m[15] = 1.0f;
  r.m[12] = t[0];
  r.m[13] = t[1];
  r.m[14] = t[2];
  return r;
}
static float det3(const float a[9]) {
  return a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) + a[2] * (a[3] * a[7] - a[4] * a[6]);
}
HostM4 inverse4(const HostM4& a) {
  auto at = [&](int i, int j) { return a.m[j * 4 + i]; };
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
          sub[ra * 3 + cb] = at(r, c);
          ++cb;
        }
        ++ra;
      }
      float minor = det3(sub);
      cof[i][j] = ((i + j) % 2 == 0) ? minor : -minor;
    }
  float det = 0.0f;
  for (int j = 0; j < 4; ++j) det += at(0, j) * cof[0][j];
  HostM4 r;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) r.m[i * 4 + j] = cof[i][j] / det;
  return r;
}
static bool ident(const HostM4& a, int n) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      float v = a.m[j * 4 + i];
      if (i == j) {
        float lim = 1e-5f * std::min(std::fabs(v), 1.0f);
        if (!(std::fabs(v - 1.0f) <= lim)) return false;
      } else if (!(std::fabs(v) <= 1e-5f)) {
        return false;
      }
    }
  return true;
}
bool is_identity4(const HostM4& a) { return ident(a, 4); }
bool is_identity3(const HostM4& a) { return ident(a, 3); }

KParams make_kparams(const mupsi_kernel& k) {
  KParams p;
  p.sigma = k.sigma;
  p.kr = k.kernel_radius;
  {
    int e = 0;
    const float m = std::frexp(p.kr, &e);  // kr = m * 2^e, m in [0.5, 1)
    p.kr_pow2 = (m == 0.5f && e > -125 && e < 126) ? 1 : 0;
    p.inv_kr = p.kr_pow2 ? std::ldexp(1.0f, 1 - e) : 0.0f;
  }
  p.L2 = k.aniso[0] * k.aniso[0] + (k.aniso[1] * k.aniso[1] + k.aniso[2] * k.aniso[2]);
  p.ppc = k.points_per_cell;
  // Var() (gpnoise.h:31): int / std::pow(float, int) -> double, * pow(pi, 1.5), returned as float
  float var = (float)(((double)p.ppc / std::pow((double)p.kr, 3.0)) * std::pow(M_PI, 1.5));
  p.sqrt_var = std::sqrt(var);
  p.k2 = (float)(-1.4426950408889634 / (double)p.L2);
  p.c2 = -2.0f / p.L2;
  p.c4 = 4.0f / (p.L2 * p.L2);
  p.psi_scale = (float)((double)p.sigma * p.ppc / (double)p.sqrt_var);
  // max over positions a in [0, kr] of 1 + exp(-a^2/L2) + exp(-(kr - a)^2/L2): the
  // largest per-axis factor of psi_bound_at (the cube is the largest bound)
  double smax = 0.0;
  for (int i = 0; i <= 4096; ++i) {
    double a = (double)p.kr * i / 4096.0;
    double s = 1.0 + std::exp(-a * a / p.L2) + std::exp(-((double)p.kr - a) * ((double)p.kr - a) / p.L2);
    smax = std::max(smax, s);
  }
  // the grid maximum can undershoot the true maximum by O(kr^2 / 4096^2 / L2)
  smax = std::min(3.0, smax * (1.0 + 1e-6));
  p.psi_bound = (float)((double)p.sigma * p.ppc / (double)p.sqrt_var * smax * smax * smax);
  p.gradh_max = (float)(std::sqrt(2.0 / (double)p.L2) * std::exp(-0.5));
  return p;
}

int check_kernel(const mupsi_kernel* k) {
  if (!k) return fail(MUPSI_ERR_INVALID, "kernel is null");
  if (!(k->kernel_radius > 0.0f) || !std::isfinite(k->kernel_radius))
    return fail(MUPSI_ERR_INVALID, "kernel_radius must be a positive finite number");
  if (k->points_per_cell < 0 || k->points_per_cell > 4096)
    return fail(MUPSI_ERR_INVALID, "points_per_cell must be in [0, 4096]");
  float L2 = k->aniso[0] * k->aniso[0] + (k->aniso[1] * k->aniso[1] + k->aniso[2] * k->aniso[2]);
  if (!(L2 > 0.0f) || !std::isfinite(L2)) return fail(MUPSI_ERR_INVALID, "aniso must have a positive norm");
  return MUPSI_OK;
}

cudaStream_t resolve_stream(void* s) {
  if (s) return (cudaStream_t)s;
  static cudaStream_t internal = nullptr;
  static std::once_flag once;
  std::call_once(once, [] { cudaStreamCreateWithFlags(&internal, cudaStreamNonBlocking); });
  return internal;
}

int num_sms() {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  return sms;
}

// ------------------------------------------------------------ GP noise batch
// PPC: the kernel's points per cell at compile time (0: read at run time)
template <bool GRAD, int PPC>
__global__ void __launch_bounds__(256) k_psi(KParams k, int64_t n, const float* __restrict__ p,
                                             const uint32_t* __restrict__ seed, const Cond* __restrict__ cond,
                                             float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    v3 P = v3{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    uint32_t s = seed[i];
    if (GRAD) {
      float4 f = raw_noise<PPC>(k, P, s);
      if (cond) f = add_cond(k, cond[i], P, f);
      out[4 * i] = f.x;
      out[4 * i + 1] = f.y;
      out[4 * i + 2] = f.z;
      out[4 * i + 3] = f.w;
    } else {
      float v = raw_noise_value<PPC>(k, P, s);
      if (cond && cond[i].active) v += cond_value(k, cond[i], P);
      out[i] = v;
    }
  }
}

static int psi_common(bool grad, const mupsi_kernel* kernel, int64_t n, const float* p, const uint32_t* seed,
                      const mupsi_cond* cond, float* out, mupsi_mem mem, void* stream) {
  clear_error();
  if (int e = check_kernel(kernel)) return e;
  if (n < 0) return fail(MUPSI_ERR_INVALID, "n must be >= 0");
  if (n == 0) return MUPSI_OK;
  if (!p || !seed || !out) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  KParams k = make_kparams(*kernel);
  const int ocomp = grad ? 4 : 1;
  Staged<float> dp(st), dout(st);
  Staged<uint32_t> ds(st);
  Staged<mupsi_cond> dc(st);
  MUPSI_CUDA(dp.in(p, 3 * n, mem));
  MUPSI_CUDA(ds.in(seed, n, mem));
  if (cond) MUPSI_CUDA(dc.in(cond, n, mem));
  MUPSI_CUDA(dout.out(out, ocomp * n, mem));
  int64_t blocks = std::min<int64_t>((n + 255) / 256, (int64_t)num_sms() * 64);
  const Cond* cptr = cond ? reinterpret_cast<const Cond*>(dc.ptr) : nullptr;
  auto fn = grad ? (k.ppc == 1 ? k_psi<true, 1> : k.ppc == 3 ? k_psi<true, 3> : k.ppc == 8 ? k_psi<true, 8> : k_psi<true, 0>)
                 : (k.ppc == 1 ? k_psi<false, 1> : k.ppc == 3 ? k_psi<false, 3> : k.ppc == 8 ? k_psi<false, 8>
                                                                                    : k_psi<false, 0>);
  fn<<<(unsigned)blocks, 256, 0, st>>>(k, n, dp.ptr, ds.ptr, cptr, dout.ptr);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dout.finish());
  MUPSI_CUDA(cudaStreamSynchronize(st));
  return MUPSI_OK;
}

// ----------------------------------------------- integer known-answer probes
// The hash, PCG32 and grid-cell routines the kernels use, exposed one query per
// thread so their outputs can be compared bit for bit with the reference
// (math/random.h:13-25,73-119, math/sampler.h:47-54, gp/gpnoise.cpp:54-62).
__global__ void k_probe_seed(int64_t n, int nargs, const uint32_t* __restrict__ a, uint32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t* v = a + i * nargs;
    out[i] = nargs == 4 ? make_seed4(v[0], v[1], v[2], v[3]) : make_seed5(v[0], v[1], v[2], v[3], v[4]);
  }
}
// Random(seed) then `draws` outputs: nextUInt as u32 and, from a second
// generator with the same seed, next1D as float; cs_i: ConstantSampler(seed).nextI()
__global__ void k_probe_random(int64_t n, const uint64_t* __restrict__ seeds, int draws, uint32_t* __restrict__ u,
                               float* __restrict__ f, uint32_t* __restrict__ cs_i) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t a = pcg_seeded(seeds[i]), b = a;
    for (int j = 0; j < draws; ++j) {
      u[i * draws + j] = pcg_next(a);
      f[i * draws + j] = pcg_next1d(b);
    }
    cs_i[i] = constant_sampler_i((uint32_t)seeds[i]);
  }
}
// Per point: the 27 neighbour cells (cell_of + (dx, dy, dz) in the psi order),
// their seeds, and every impulse's position and weight as the psi loop draws them.
template <int PPC>
__global__ void k_probe_impulses(KParams k, int64_t n, const float* __restrict__ p, const uint32_t* __restrict__ seed,
                                 int32_t* __restrict__ cells, uint32_t* __restrict__ cseed, float* __restrict__ s_out,
                                 float* __restrict__ w_out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const v3 P = v3{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    int cx, cy, cz;
    cell_of(k, P, cx, cy, cz);
    int64_t m = i * 27 * (int64_t)k.ppc;
    for (int c = 0; c < 27; ++c) {
      const int nx = cx + c / 9 - 1, ny = cy + (c / 3) % 3 - 1, nz = cz + c % 3 - 1;
      cells[(i * 27 + c) * 3] = nx;
      cells[(i * 27 + c) * 3 + 1] = ny;
      cells[(i * 27 + c) * 3 + 2] = nz;
      cseed[i * 27 + c] = make_seed4((uint32_t)nx, (uint32_t)ny, (uint32_t)nz, seed[i]);
      for_each_impulse<PPC>(k, nx, ny, nz, seed[i], [&](v3 s, uint32_t wsign) {
        s_out[3 * m] = s.x;
        s_out[3 * m + 1] = s.y;
        s_out[3 * m + 2] = s.z;
        w_out[m] = wsign ? -1.0f : 1.0f;
        ++m;
      });
    }
  }
}

// ------------------------------------------------------- buffer cache
namespace {
struct CachedBuf {
  int dev;
  size_t cls;
  void* p;
};
std::mutex g_buf_mu;
std::vector<CachedBuf> g_buf_free;
std::unordered_map<void*, CachedBuf> g_buf_live;
size_t g_buf_cached = 0;
constexpr size_t kBufMax = size_t(16) << 20, kBufCap = size_t(256) << 20;
}  // namespace

cudaError_t dev_take(void** out, size_t bytes) {
  if (bytes > kBufMax) return cudaMalloc(out, bytes);  // not cached: cudaFree'd by dev_give
  size_t cls = 256;
  while (cls < bytes) cls <<= 1;
  int dev = 0;
  cudaGetDevice(&dev);
  {
    std::lock_guard<std::mutex> lock(g_buf_mu);
    for (size_t i = 0; i < g_buf_free.size(); ++i)
      if (g_buf_free[i].dev == dev && g_buf_free[i].cls == cls) {
        const CachedBuf b = g_buf_free[i];
        g_buf_free[i] = g_buf_free.back();
        g_buf_free.pop_back();
        g_buf_cached -= cls;
        g_buf_live[b.p] = b;
        *out = b.p;
        return cudaSuccess;
      }
  }
  void* p = nullptr;
  const cudaError_t e = cudaMalloc(&p, cls);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(g_buf_mu);
  g_buf_live[p] = CachedBuf{dev, cls, p};
  *out = p;
  return cudaSuccess;
}

void dev_give(void* p) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lock(g_buf_mu);
    auto it = g_buf_live.find(p);
    if (it != g_buf_live.end()) {
      const CachedBuf b = it->second;
      g_buf_live.erase(it);
      if (g_buf_cached + b.cls <= kBufCap) {
        g_buf_free.push_back(b);
        g_buf_cached += b.cls;
        return;
      }
    }
  }
  cudaFree(p);
}

void dev_cache_release() {
  std::vector<CachedBuf> all;
  {
    std::lock_guard<std::mutex> lock(g_buf_mu);
    all.swap(g_buf_free);
    g_buf_cached = 0;
  }
  int cur = 0;
  cudaGetDevice(&cur);
  for (const CachedBuf& b : all) {
    cudaSetDevice(b.dev);
    cudaFree(b.p);
  }
  cudaSetDevice(cur);
}

// ------------------------------------------------------------ meshes / BVH
struct MeshStore {
  DMesh d;
  std::vector<void*> allocs;
  ~MeshStore() {
    cudaDeviceSynchronize();  // nothing in flight reads the buffers handed back
    for (void* p : allocs) dev_give(p);
  }
};

template <typename T>
static cudaError_t upload(std::vector<void*>& allocs, const T* src, size_t count, const T*& dst) {
  if (count == 0) {
    dst = nullptr;
    return cudaSuccess;
  }
  void* p = nullptr;
  cudaError_t e = dev_take(&p, count * sizeof(T));
  if (e != cudaSuccess) return e;
  allocs.push_back(p);
  e = cudaMemcpy(p, src, count * sizeof(T), cudaMemcpyHostToDevice);
  dst = static_cast<const T*>(p);
  return e;
}

// The binary tree four wide (DMesh::wide, WNode rows): each node takes the two
// children of a binary node and keeps replacing its inner child of largest box
// surface by that child's two children while it has fewer than four. Boxes and
// leaf ranges are the binary tree's own; node 0 is the root. Empty for a tree
// that is a single leaf or whose leaf slots exceed the child encoding.
static std::vector<float> build_wide(const std::vector<HostNode>& nodes, uint32_t root, int64_t num_faces) {
  std::vector<float> w;
  constexpr uint32_t kLeaf = 0x80000000u;
  if (nodes.empty() || (nodes[root].right & kLeaf) || num_faces >= (1ll << 28)) return w;
  auto area = [&](uint32_t i) {
    const HostNode& n = nodes[i];
    const float dx = n.mx[0] - n.mn[0], dy = n.mx[1] - n.mn[1], dz = n.mx[2] - n.mn[2];
    return dx * dy + dy * dz + dz * dx;
  };
  // nodes breadth first: (binary inner node, wide index)
  std::vector<std::pair<uint32_t, uint32_t>> order{{root, 0u}};
  w.assign(kWideRowsHost * 4, 0.0f);
  for (size_t h = 0; h < order.size(); ++h) {
    const uint32_t b = order[h].first, wi = order[h].second;
    uint32_t kids[4] = {nodes[b].left, nodes[b].right, 0, 0};
    int nk = 2;
    while (nk < 4) {
      int pick = -1;
      float pa = -1.0f;
      for (int i = 0; i < nk; ++i)
        if (!(nodes[kids[i]].right & kLeaf) && area(kids[i]) > pa) {
          pa = area(kids[i]);
          pick = i;
        }
      if (pick < 0) break;
      const uint32_t k = kids[pick];
      kids[pick] = nodes[k].left;
      kids[nk++] = nodes[k].right;
    }
    for (int i = 0; i < 4; ++i) {
      float* row = &w[(size_t)kWideRowsHost * 4 * wi];
      uint32_t ref = kLeaf;  // unused slot: count 0, empty box
      float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
      if (i < nk) {
        const HostNode& c = nodes[kids[i]];
        for (int a = 0; a < 3; ++a) {
          lo[a] = c.mn[a];
          hi[a] = c.mx[a];
        }
        if (c.right & kLeaf) {
          ref = kLeaf | ((c.right & ~kLeaf) << 28) | c.left;
        } else {
          ref = (uint32_t)(w.size() / (kWideRowsHost * 4));
          order.push_back({kids[i], ref});
          w.resize(w.size() + kWideRowsHost * 4, 0.0f);
          row = &w[(size_t)kWideRowsHost * 4 * wi];
        }
      }
      for (int a = 0; a < 3; ++a) {
        row[4 * a + i] = lo[a];
        row[4 * (3 + a) + i] = hi[a];
      }
      std::memcpy(&row[4 * 6 + i], &ref, 4);
    }
  }
  return w;
}

int make_device_mesh(const mupsi_mesh_desc& md, DMesh& d, std::vector<void*>& allocs) {
  if (md.num_vertices < 0 || md.num_faces < 0) return fail(MUPSI_ERR_INVALID, "negative mesh size");
  if ((md.num_vertices > 0 && !md.vertices) || (md.num_faces > 0 && !md.faces))
    return fail(MUPSI_ERR_INVALID, "mesh arrays are null");
  if (md.num_faces > 0x3FFFFFFF) return fail(MUPSI_ERR_INVALID, "too many faces");
  for (int64_t i = 0; i < 3 * md.num_faces; ++i)
    if (md.faces[i] < 0 || md.faces[i] >= md.num_vertices) return fail(MUPSI_ERR_INVALID, "face index out of range");
  d.count = nullptr;
  std::vector<HostNode> nodes;
  std::vector<uint32_t> idx;
  uint32_t root = build_bvh(md.vertices, md.faces, md.num_faces, nodes, idx);
  // face normals and the light-sampling CDF (mesh.cpp:140-154, :308-318)
  std::vector<float> fn(3 * md.num_faces), cdf(md.num_faces);
  float total = 0.0f;
  for (int64_t i = 0; i < md.num_faces; ++i) {
    const int32_t* f = md.faces + 3 * i;
    v3 a = ld3(md.vertices + 3 * (int64_t)f[0]), b = ld3(md.vertices + 3 * (int64_t)f[1]),
       c = ld3(md.vertices + 3 * (int64_t)f[2]);
    v3 n = cross(b - a, c - a);
    float len = norm3(n);
    v3 un = len > 1e-12f ? n / len : mk3(0, 0, 0);
    st3(&fn[3 * i], un);
    total += 0.5f * len;
    cdf[i] = total;
  }
  if (total > 0.0f)
    for (auto& c : cdf) c /= total;
  // device node order: breadth first from the root (node 0), a pad at 1, and
  // every inner node's children side by side at (left, left + 1), left even, so
  // a traversal reads both with one 64-byte load. Boxes, leaf ranges and the
  // tree are the reference's; only node positions change (traversal order
  // follows boxes and centroids, not positions).
  const std::vector<float> wide = build_wide(nodes, root, md.num_faces);
  std::vector<HostNode> dev_nodes;
  uint32_t occl_ref = 0;  // where the reference's node 0 (BVH::occluded's start) lands
  if (!nodes.empty()) {
    dev_nodes.reserve(nodes.size() + 1);
    dev_nodes.push_back(nodes[root]);
    dev_nodes.push_back(HostNode{});
    std::vector<std::pair<uint32_t, uint32_t>> order{{root, 0u}};  // (reference index, device index)
    for (size_t h = 0; h < order.size(); ++h) {
      const uint32_t o = order[h].first, di = order[h].second;
      if (o == 0) occl_ref = di;
      const HostNode n = nodes[o];
      if (n.right & 0x80000000u) continue;  // a leaf keeps (start, count | LEAF)
      const uint32_t l = (uint32_t)dev_nodes.size();
      dev_nodes.push_back(nodes[n.left]);
      dev_nodes.push_back(nodes[n.right]);
      dev_nodes[di].left = l;
      dev_nodes[di].right = l + 1;
      order.push_back({n.left, l});
      order.push_back({n.right, l + 1});
    }
    root = 0;
  }
  // the triangles in leaf order (DMesh::soup)
  std::vector<float> soup(12 * idx.size(), 0.0f);
  for (size_t i = 0; i < idx.size(); ++i) {
    const int32_t* f = md.faces + 3 * (int64_t)idx[i];
    float* q = &soup[12 * i];
    for (int k = 0; k < 3; ++k)
      for (int c = 0; c < 3; ++c) q[3 * k + c] = md.vertices[3 * (int64_t)f[k] + c];
    std::memcpy(&q[9], &idx[i], 4);
  }
  std::memset(&d, 0, sizeof d);
  const BNode* dn = nullptr;
  const float* dsoup = nullptr;
  cudaError_t e;
  if ((e = upload(allocs, reinterpret_cast<const BNode*>(dev_nodes.data()), dev_nodes.size(), dn)) != cudaSuccess ||
      (e = upload(allocs, soup.data(), soup.size(), dsoup)) != cudaSuccess ||
      (e = upload(allocs, idx.data(), idx.size(), d.tri_idx)) != cudaSuccess ||
      (e = upload(allocs, md.faces, 3 * md.num_faces, d.faces)) != cudaSuccess ||
      (e = upload(allocs, md.vertices, 3 * md.num_vertices, d.verts)) != cudaSuccess ||
      (e = upload(allocs, fn.data(), fn.size(), d.face_n)) != cudaSuccess ||
      (e = upload(allocs, cdf.data(), cdf.size(), d.cdf)) != cudaSuccess)
    return fail(e == cudaErrorMemoryAllocation ? MUPSI_ERR_OOM : MUPSI_ERR_CUDA,
                std::string("mesh upload: ") + cudaGetErrorString(e));
  if (md.vertex_normals) {
    if ((e = upload(allocs, md.vertex_normals, 3 * md.num_vertices, d.vert_n)) != cudaSuccess)
      return fail(MUPSI_ERR_CUDA, std::string("mesh upload: ") + cudaGetErrorString(e));
  }
  if (!wide.empty()) {
    const float* dw = nullptr;
    if ((e = upload(allocs, wide.data(), wide.size(), dw)) != cudaSuccess)
      return fail(e == cudaErrorMemoryAllocation ? MUPSI_ERR_OOM : MUPSI_ERR_CUDA,
                  std::string("mesh upload: ") + cudaGetErrorString(e));
    d.wide = reinterpret_cast<const float4*>(dw);
    d.wide_root = 0;
  }
  d.nodes = dn;
  d.soup = reinterpret_cast<const float4*>(dsoup);
  d.num_nodes = (int64_t)dev_nodes.size();
  d.num_faces = md.num_faces;
  d.root = root;
  d.occl_ref = occl_ref;
  d.occl_start = occl_ref;
  d.total_area = total;
  HostM4 T = translate_scale(md.position, md.scale), Ti = inverse4(T);
  std::memcpy(d.T.m, T.m, sizeof T.m);
  std::memcpy(d.Tinv.m, Ti.m, sizeof Ti.m);
  d.identity = is_identity4(Ti);
  d.normal_identity = is_identity3(Ti);
  return MUPSI_OK;
}

__global__ void k_bvh_intersect(DMesh m, int64_t n, const mupsi_ray* rays, uint32_t* out_tri, float* out_tuv,
                                int* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const mupsi_ray& q = rays[i];
    Ray r = make_ray(ld3(q.o), ld3(q.d));
    r.nt = q.near_t;
    r.ft = q.far_t;
    uint32_t tri = 0;
    float u = 0, v = 0;
    bool ovf = false;
    bool h = bvh_intersect(m, r, tri, u, v, ovf);
    if (ovf) atomicOr(err, 1);
    out_tri[i] = h ? tri : 0xFFFFFFFFu;
    out_tuv[3 * i] = h ? r.ft : -1.0f;
    out_tuv[3 * i + 1] = h ? u : 0.0f;
    out_tuv[3 * i + 2] = h ? v : 0.0f;
  }
}
__global__ void k_bvh_occluded(DMesh m, int64_t n, const mupsi_ray* rays, uint8_t* out, int* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const mupsi_ray& q = rays[i];
    Ray r = make_ray(ld3(q.o), ld3(q.d));
    r.nt = q.near_t;
    r.ft = q.far_t;
    bool ovf = false;
    out[i] = bvh_occluded(m, r, ovf) ? 1 : 0;
    if (ovf) atomicOr(err, 1);
  }
}
__global__ void k_bvh_closest(DMesh m, int64_t n, const float* p, uint32_t* out_tri, float* out_dq, int* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t tri = 0xFFFFFFFFu;
    v3 q = mk3(0, 0, 0);
    bool ovf = false;
    float d = bvh_closest(m, ld3(p + 3 * i), tri, q, ovf);
    if (ovf) atomicOr(err, 1);
    out_tri[i] = tri;
    out_dq[4 * i] = d;
    out_dq[4 * i + 1] = q.x;
    out_dq[4 * i + 2] = q.y;
    out_dq[4 * i + 3] = q.z;
  }
}
__global__ void k_mesh_queries(DMesh m, int64_t n, const float* p, uint8_t* out_inside, uint32_t* out_tri,
                               float* out_dq, int* err) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    v3 P = ld3(p + 3 * i);
    bool ovf = false;
    out_inside[i] = mesh_inside(m, P, ovf) ? 1 : 0;
    uint32_t tri = 0xFFFFFFFFu;
    v3 q = mk3(0, 0, 0);
    out_dq[4 * i] = mesh_dist(m, P, tri, q, ovf);
    out_tri[i] = tri;
    out_dq[4 * i + 1] = q.x;
    out_dq[4 * i + 2] = q.y;
    out_dq[4 * i + 3] = q.z;
    if (ovf) atomicOr(err, 1);
  }
}

}  // namespace mupsi

struct mupsi_mesh {
  mupsi::MeshStore store;
};

using namespace mupsi;

static int grid_for(int64_t n) { return (int)std::min<int64_t>((n + 127) / 128, (int64_t)num_sms() * 32); }

// Device error word for one batch call: allocated, cleared, read back.
struct ErrWord {
  int* d = nullptr;
  cudaStream_t s;
  explicit ErrWord(cudaStream_t st) : s(st) {}
  cudaError_t init() {
    cudaError_t e = cudaMallocAsync((void**)&d, sizeof(int), s);
    if (e != cudaSuccess) return e;
    return cudaMemsetAsync(d, 0, sizeof(int), s);
  }
  int read() {
    int h = 0;
    cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return h;
  }
  ~ErrWord() {
    if (d) cudaFreeAsync(d, s);
  }
};

extern "C" {

const char* mupsi_gpu_last_error(void) { return g_last_error.c_str(); }
int32_t mupsi_gpu_abi_version(void) { return MUPSI_GPU_ABI_VERSION; }
int64_t mupsi_gpu_launch_count(void) { return g_launches.load(); }

int mupsi_gpu_psi(const mupsi_kernel* kernel, int64_t n, const float* p, const uint32_t* seed, const mupsi_cond* cond,
                  float* out, mupsi_mem mem, void* stream) {
  return psi_common(true, kernel, n, p, seed, cond, out, mem, stream);
}
int mupsi_gpu_psi_value(const mupsi_kernel* kernel, int64_t n, const float* p, const uint32_t* seed,
                        const mupsi_cond* cond, float* out, mupsi_mem mem, void* stream) {
  return psi_common(false, kernel, n, p, seed, cond, out, mem, stream);
}

int mupsi_gpu_probe_make_seed(int64_t n, int32_t nargs, const uint32_t* args, uint32_t* out, mupsi_mem mem,
                              void* stream) {
  clear_error();
  if (n < 0 || (nargs != 4 && nargs != 5)) return fail(MUPSI_ERR_INVALID, "n >= 0 and nargs 4 or 5");
  if (n == 0) return MUPSI_OK;
  if (!args || !out) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<uint32_t> da(st), dout(st);
  MUPSI_CUDA(da.in(args, (size_t)n * nargs, mem));
  MUPSI_CUDA(dout.out(out, n, mem));
  k_probe_seed<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(n, nargs, da.ptr, dout.ptr);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dout.finish());
  MUPSI_CUDA(cudaStreamSynchronize(st));
  return MUPSI_OK;
}

int mupsi_gpu_probe_random(int64_t n, const uint64_t* seeds, int32_t draws, uint32_t* out_u32, float* out_f32,
                           uint32_t* out_cs_i, mupsi_mem mem, void* stream) {
  clear_error();
  if (n < 0 || draws < 0 || draws > 4096) return fail(MUPSI_ERR_INVALID, "n >= 0 and 0 <= draws <= 4096");
  if (n == 0) return MUPSI_OK;
  if (!seeds || !out_cs_i || (draws && (!out_u32 || !out_f32))) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<uint64_t> ds(st);
  Staged<uint32_t> du(st), dc(st);
  Staged<float> df(st);
  MUPSI_CUDA(ds.in(seeds, n, mem));
  MUPSI_CUDA(du.out(out_u32, (size_t)n * draws, mem));
  MUPSI_CUDA(df.out(out_f32, (size_t)n * draws, mem));
  MUPSI_CUDA(dc.out(out_cs_i, n, mem));
  k_probe_random<<<(unsigned)std::min<int64_t>((n + 255) / 256, 4096), 256, 0, st>>>(n, ds.ptr, draws, du.ptr,
                                                                                     df.ptr, dc.ptr);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(du.finish());
  MUPSI_CUDA(df.finish());
  MUPSI_CUDA(dc.finish());
  MUPSI_CUDA(cudaStreamSynchronize(st));
  return MUPSI_OK;
}

int mupsi_gpu_probe_impulses(const mupsi_kernel* kernel, int64_t n, const float* p, const uint32_t* seed,
                             int32_t* out_cells, uint32_t* out_cell_seeds, float* out_s, float* out_w, mupsi_mem mem,
                             void* stream) {
  clear_error();
  if (int e = check_kernel(kernel)) return e;
  if (n < 0) return fail(MUPSI_ERR_INVALID, "n must be >= 0");
  if (n == 0) return MUPSI_OK;
  if (!p || !seed || !out_cells || !out_cell_seeds || !out_s || !out_w) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  KParams k = make_kparams(*kernel);
  const size_t m = (size_t)n * 27 * k.ppc;
  Staged<float> dp(st), ds_(st), dw(st);
  Staged<uint32_t> dseed(st), dcs(st);
  Staged<int32_t> dcell(st);
  MUPSI_CUDA(dp.in(p, 3 * (size_t)n, mem));
  MUPSI_CUDA(dseed.in(seed, n, mem));
  MUPSI_CUDA(dcell.out(out_cells, (size_t)n * 81, mem));
  MUPSI_CUDA(dcs.out(out_cell_seeds, (size_t)n * 27, mem));
  MUPSI_CUDA(ds_.out(out_s, 3 * m, mem));
  MUPSI_CUDA(dw.out(out_w, m, mem));
  // the psi kernels' cell variants: unrolled for 1, 3 and 8 impulses (states
  // jumped ahead), a stepped loop for other counts
  auto fn = k.ppc == 1 ? k_probe_impulses<1> : k.ppc == 3 ? k_probe_impulses<3> : k.ppc == 8 ? k_probe_impulses<8>
                                                                                              : k_probe_impulses<0>;
  fn<<<(unsigned)std::min<int64_t>((n + 127) / 128, 4096), 128, 0, st>>>(k, n, dp.ptr, dseed.ptr, dcell.ptr, dcs.ptr,
                                                                          ds_.ptr, dw.ptr);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dcell.finish());
  MUPSI_CUDA(dcs.finish());
  MUPSI_CUDA(ds_.finish());
  MUPSI_CUDA(dw.finish());
  MUPSI_CUDA(cudaStreamSynchronize(st));
  return MUPSI_OK;
}

int mupsi_bvh_build_host(int64_t num_vertices, const float* vertices, int64_t num_faces, const int32_t* faces,
                         uint32_t* nodes_out, uint32_t* tri_indices_out, int64_t* num_nodes, uint32_t* root) {
  clear_error();
  if (num_faces < 0 || num_vertices < 0) return fail(MUPSI_ERR_INVALID, "negative size");
  if ((num_faces && (!faces || !vertices)) || !nodes_out || !tri_indices_out || !num_nodes || !root)
    return fail(MUPSI_ERR_INVALID, "null buffer");
  for (int64_t i = 0; i < 3 * num_faces; ++i)
    if (faces[i] < 0 || faces[i] >= num_vertices) return fail(MUPSI_ERR_INVALID, "face index out of range");
  std::vector<HostNode> nodes;
  std::vector<uint32_t> idx;
  *root = build_bvh(vertices, faces, num_faces, nodes, idx);
  *num_nodes = (int64_t)nodes.size();
  if (!nodes.empty()) std::memcpy(nodes_out, nodes.data(), nodes.size() * sizeof(HostNode));
  if (!idx.empty()) std::memcpy(tri_indices_out, idx.data(), idx.size() * sizeof(uint32_t));
  return MUPSI_OK;
}

int mupsi_gpu_mesh_create(const mupsi_mesh_desc* desc, mupsi_mesh** out) {
  clear_error();
  if (!desc || !out) return fail(MUPSI_ERR_INVALID, "null argument");
  auto* m = new mupsi_mesh();
  int e = make_device_mesh(*desc, m->store.d, m->store.allocs);
  if (e) {
    delete m;
    return e;
  }
  *out = m;
  return MUPSI_OK;
}
void mupsi_gpu_mesh_destroy(mupsi_mesh* mesh) { delete mesh; }

int mupsi_gpu_bvh_intersect(const mupsi_mesh* mesh, int64_t n, const mupsi_ray* rays, uint32_t* out_tri,
                            float* out_tuv, mupsi_mem mem, void* stream) {
  clear_error();
  if (!mesh || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!rays || !out_tri || !out_tuv) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<mupsi_ray> dr(st);
  Staged<uint32_t> dt(st);
  Staged<float> duv(st);
  ErrWord err(st);
  MUPSI_CUDA(err.init());
  MUPSI_CUDA(dr.in(rays, n, mem));
  MUPSI_CUDA(dt.out(out_tri, n, mem));
  MUPSI_CUDA(duv.out(out_tuv, 3 * n, mem));
  k_bvh_intersect<<<grid_for(n), 128, 0, st>>>(mesh->store.d, n, dr.ptr, dt.ptr, duv.ptr, err.d);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dt.finish());
  MUPSI_CUDA(duv.finish());
  if (err.read()) return fail(MUPSI_ERR_DEVICE_LIMIT, "BVH traversal exceeded the 64-entry stack");
  return MUPSI_OK;
}

int mupsi_gpu_mesh_set_occlusion(mupsi_mesh* mesh, int32_t mode) {
  clear_error();
  if (!mesh) return fail(MUPSI_ERR_INVALID, "null mesh");
  if (mode != MUPSI_OCCLUSION_REFERENCE && mode != MUPSI_OCCLUSION_ROOT)
    return fail(MUPSI_ERR_INVALID, "unknown occlusion mode");
  mesh->store.d.occl_start = mode == MUPSI_OCCLUSION_ROOT ? mesh->store.d.root : mesh->store.d.occl_ref;
  return MUPSI_OK;
}

int mupsi_gpu_bvh_occluded(const mupsi_mesh* mesh, int64_t n, const mupsi_ray* rays, uint8_t* out, mupsi_mem mem,
                           void* stream) {
  clear_error();
  if (!mesh || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!rays || !out) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<mupsi_ray> dr(st);
  Staged<uint8_t> dout(st);
  ErrWord err(st);
  MUPSI_CUDA(err.init());
  MUPSI_CUDA(dr.in(rays, n, mem));
  MUPSI_CUDA(dout.out(out, n, mem));
  k_bvh_occluded<<<grid_for(n), 128, 0, st>>>(mesh->store.d, n, dr.ptr, dout.ptr, err.d);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dout.finish());
  if (err.read()) return fail(MUPSI_ERR_DEVICE_LIMIT, "BVH traversal exceeded the 64-entry stack");
  return MUPSI_OK;
}

int mupsi_gpu_bvh_closest(const mupsi_mesh* mesh, int64_t n, const float* p, uint32_t* out_tri, float* out_dq,
                          mupsi_mem mem, void* stream) {
  clear_error();
  if (!mesh || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!p || !out_tri || !out_dq) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<float> dp(st), ddq(st);
  Staged<uint32_t> dt(st);
  ErrWord err(st);
  MUPSI_CUDA(err.init());
  MUPSI_CUDA(dp.in(p, 3 * n, mem));
  MUPSI_CUDA(dt.out(out_tri, n, mem));
  MUPSI_CUDA(ddq.out(out_dq, 4 * n, mem));
  k_bvh_closest<<<grid_for(n), 128, 0, st>>>(mesh->store.d, n, dp.ptr, dt.ptr, ddq.ptr, err.d);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(dt.finish());
  MUPSI_CUDA(ddq.finish());
  if (err.read()) return fail(MUPSI_ERR_DEVICE_LIMIT, "BVH traversal exceeded the 64-entry stack");
  return MUPSI_OK;
}

int mupsi_gpu_mesh_queries(const mupsi_mesh* mesh, int64_t n, const float* p, uint8_t* out_inside, uint32_t* out_tri,
                           float* out_dq, mupsi_mem mem, void* stream) {
  clear_error();
  if (!mesh || n < 0) return fail(MUPSI_ERR_INVALID, "bad argument");
  if (n == 0) return MUPSI_OK;
  if (!p || !out_inside || !out_tri || !out_dq) return fail(MUPSI_ERR_INVALID, "null buffer");
  cudaStream_t st = resolve_stream(stream);
  Staged<float> dp(st), ddq(st);
  Staged<uint32_t> dt(st);
  Staged<uint8_t> di(st);
  ErrWord err(st);
  MUPSI_CUDA(err.init());
  MUPSI_CUDA(dp.in(p, 3 * n, mem));
  MUPSI_CUDA(di.out(out_inside, n, mem));
  MUPSI_CUDA(dt.out(out_tri, n, mem));
  MUPSI_CUDA(ddq.out(out_dq, 4 * n, mem));
  k_mesh_queries<<<grid_for(n), 128, 0, st>>>(mesh->store.d, n, dp.ptr, di.ptr, dt.ptr, ddq.ptr, err.d);
  count_launch();
  MUPSI_CUDA(cudaGetLastError());
  MUPSI_CUDA(di.finish());
  MUPSI_CUDA(dt.finish());
  MUPSI_CUDA(ddq.finish());
  if (err.read()) return fail(MUPSI_ERR_DEVICE_LIMIT, "BVH traversal exceeded the 64-entry stack");
  return MUPSI_OK;
}

}  // extern "C"
