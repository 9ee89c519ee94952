// Declarations shared by core.cu and render.cu.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "dmath.cuh"
#include "geom.cuh"
#include "gp.cuh"
#include "host.h"

namespace mupsi {

KParams make_kparams(const mupsi_kernel& k);
int check_kernel(const mupsi_kernel* k);
cudaStream_t resolve_stream(void* s);
int num_sms();
int make_device_mesh(const mupsi_mesh_desc& md, DMesh& d, std::vector<void*>& allocs);

// Device buffers that live as long as a scene or mesh: released ones stay in a
// per-device cache (power-of-two size classes from 256 B, buffers up to 16 MB,
// 256 MB in all) and are handed out again, so a host that creates and
// releases a scene per frame pays no cudaMalloc / cudaFree (each may
// synchronise the device) after the first. dev_give's caller has
// synchronised: no work in flight uses the buffer.
cudaError_t dev_take(void** out, size_t bytes);
void dev_give(void* p);
void dev_cache_release();  // cudaFree every cached buffer

// A buffer of one batch call: aliases the caller's pointer for device memory,
// otherwise a stream-ordered device allocation with the copy in (in()) or the
// copy back (finish()); the caller synchronises the stream before returning.
template <typename T>
struct Staged {
  cudaStream_t s;
  T* ptr = nullptr;
  bool owned = false;
  T* host_dst = nullptr;
  size_t count = 0;
  explicit Staged(cudaStream_t st) : s(st) {}
  Staged(const Staged&) = delete;
  Staged& operator=(const Staged&) = delete;
  cudaError_t in(const T* src, size_t n, mupsi_mem mem) {
    if (mem == MUPSI_MEM_DEVICE) {
      ptr = const_cast<T*>(src);
      return cudaSuccess;
    }
    cudaError_t e = cudaMallocAsync((void**)&ptr, std::max<size_t>(n, 1) * sizeof(T), s);
    if (e != cudaSuccess) return e;
    owned = true;
    return cudaMemcpyAsync(ptr, src, n * sizeof(T), cudaMemcpyHostToDevice, s);
  }
  cudaError_t out(T* dst, size_t n, mupsi_mem mem) {
    if (mem == MUPSI_MEM_DEVICE) {
      ptr = dst;
      return cudaSuccess;
    }
    cudaError_t e = cudaMallocAsync((void**)&ptr, std::max<size_t>(n, 1) * sizeof(T), s);
    if (e != cudaSuccess) return e;
    owned = true;
    host_dst = dst;
    count = n;
    return cudaSuccess;
  }
  cudaError_t finish() {
    if (host_dst && owned) return cudaMemcpyAsync(host_dst, ptr, count * sizeof(T), cudaMemcpyDeviceToHost, s);
    return cudaSuccess;
  }
  ~Staged() {
    if (owned && ptr) cudaFreeAsync(ptr, s);
  }
};

// Surrogate inference (mlp.cu): mu_hat of the points P + i * pstride, i < n,
// or i < *n_dev when n_dev is set (a count written on the device, at most n).
int mlp_infer_device(mupsi_mlp* m, int64_t n, const float* p, int pstride, const uint32_t* n_dev, float* out,
                     cudaStream_t st);

}  // namespace mupsi
