// Headless progressive display: the render control of Controller
// (controller/controller.cpp:266-375) over the GPU path tracer. A host thread
// renders frames of passes through mupsi_gpu_render on its own stream; after
// each frame the averaged image goes device -> pinned back buffer and is
// swapped with the front buffer under a mutex (framebufferFront_ /
// framebufferBack_, displayMtx_), so a reader always copies a complete frame
// (copyDisplayRawTo, copyDisplayTo). sppPassDone_ / currentSpp_ report frames.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>

#include "host.h"

using namespace mupsi;

struct mupsi_display {
  mupsi_scene* scene = nullptr;
  int device = 0;
  int w = 0, h = 0;
  std::mutex mu;           // guards front (and has_frame)
  float* front = nullptr;  // pinned host w*h*3: the frame readers copy
  float* back = nullptr;   // pinned host w*h*3: the frame being filled
  float* dev = nullptr;    // device w*h*3: mupsi_gpu_render's averaged output
  cudaStream_t st = nullptr;
  std::thread th;
  volatile int32_t cancel = 0;  // polled by mupsi_gpu_render between waves
  std::atomic<int> spp_done{0};
  std::atomic<int> current{0};
  std::atomic<int> running{0};
  int status = MUPSI_OK;  // of the last render thread (read after join)
  std::string error;
};

namespace {

void set_cancel(mupsi_display* d, int v) { __atomic_store_n(&d->cancel, v, __ATOMIC_SEQ_CST); }

// Frames of `ppf` passes (the last one shorter) until `target` passes or a cancel.
void render_thread(mupsi_display* d, int target, int ppf) {
  cudaSetDevice(d->device);
  const size_t bytes = (size_t)d->w * d->h * 3 * sizeof(float);
  int rc = MUPSI_OK;
  for (int k = 0; k < target;) {
    if (__atomic_load_n(&d->cancel, __ATOMIC_SEQ_CST)) break;
    const int p = std::min(ppf, target - k);
    mupsi_render_args a;
    std::memset(&a, 0, sizeof a);
    a.spp_begin = k;
    a.spp_end = k + p;
    a.cancel = &d->cancel;
    a.rgb_out = d->dev;
    a.out_mem = MUPSI_MEM_DEVICE;
    a.stream = d->st;
    rc = mupsi_gpu_render(d->scene, &a);
    if (rc == MUPSI_ERR_CANCELLED) {  // the unfinished frame is dropped, as onSpp returns on cancel
      rc = MUPSI_OK;
      break;
    }
    if (rc != MUPSI_OK) {
      d->error = mupsi_gpu_last_error();
      break;
    }
    cudaError_t e = cudaMemcpyAsync(d->back, d->dev, bytes, cudaMemcpyDeviceToHost, d->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(d->st);
    if (e != cudaSuccess) {
      rc = MUPSI_ERR_CUDA;
      d->error = std::string("display copy: ") + cudaGetErrorString(e);
      break;
    }
    {
      std::lock_guard<std::mutex> lock(d->mu);
      std::swap(d->front, d->back);
    }
    k += p;
    d->current.store(k);
    d->spp_done.store(1);
  }
  d->status = rc;
  d->running.store(0);
}

int stop_thread(mupsi_display* d) {
  set_cancel(d, 1);
  if (d->th.joinable()) d->th.join();
  return d->status;
}

int copy_front(mupsi_display* d, float* dst, int32_t w, int32_t h, bool tonemap) {
  clear_error();
  if (!d || !dst) return fail(MUPSI_ERR_INVALID, "null argument");
  if (w != d->w || h != d->h) return fail(MUPSI_ERR_INVALID, "display size differs from the scene's");
  std::lock_guard<std::mutex> lock(d->mu);
  const size_t n = (size_t)w * h * 3;
  if (!tonemap) {
    std::memcpy(dst, d->front, n * sizeof(float));
  } else {  // Framebuffer::tonemapped (framebuffer.cpp:37-45): Reinhard v / (1 + v)
    for (size_t i = 0; i < n; ++i) dst[i] = d->front[i] / (1.0f + d->front[i]);
  }
  return MUPSI_OK;
}

}  // namespace

extern "C" {

int mupsi_gpu_display_create(mupsi_scene* scene, mupsi_display** out) {
  clear_error();
  if (!scene || !out) return fail(MUPSI_ERR_INVALID, "null argument");
  int32_t w = 0, h = 0;
  if (int e = mupsi_gpu_scene_get_size(scene, &w, &h)) return e;
  auto* d = new mupsi_display();
  d->scene = scene;
  d->w = w;
  d->h = h;
  cudaGetDevice(&d->device);
  const size_t bytes = (size_t)w * h * 3 * sizeof(float);
  cudaError_t e = cudaMallocHost((void**)&d->front, bytes);
  if (e == cudaSuccess) e = cudaMallocHost((void**)&d->back, bytes);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d->dev, bytes);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&d->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    mupsi_gpu_display_destroy(d);
    return fail(MUPSI_ERR_CUDA, std::string("display buffers: ") + cudaGetErrorString(e));
  }
  std::memset(d->front, 0, bytes);  // a fresh Framebuffer is black
  std::memset(d->back, 0, bytes);
  *out = d;
  return MUPSI_OK;
}

void mupsi_gpu_display_destroy(mupsi_display* d) {
  if (!d) return;
  stop_thread(d);
  if (d->st) cudaStreamDestroy(d->st);
  if (d->dev) cudaFree(d->dev);
  if (d->front) cudaFreeHost(d->front);
  if (d->back) cudaFreeHost(d->back);
  delete d;
}

int mupsi_gpu_display_start_progressive(mupsi_display* d, int32_t target_spp, int32_t passes_per_frame) {
  clear_error();
  if (!d) return fail(MUPSI_ERR_INVALID, "null display");
  if (target_spp < 0 || passes_per_frame < 0) return fail(MUPSI_ERR_INVALID, "negative spp");
  stop_thread(d);
  int ppf = passes_per_frame;
  if (ppf == 0) ppf = (int)std::max<int64_t>(1, (int64_t(1) << 20) / std::max<int64_t>(1, (int64_t)d->w * d->h));
  set_cancel(d, 0);
  d->spp_done.store(0);
  d->current.store(0);
  d->status = MUPSI_OK;
  d->error.clear();
  d->running.store(1);
  d->th = std::thread(render_thread, d, (int)target_spp, ppf);
  return MUPSI_OK;
}

int mupsi_gpu_display_start(mupsi_display* d, int32_t spp) {
  return mupsi_gpu_display_start_progressive(d, spp, std::max<int32_t>(1, spp));
}

void mupsi_gpu_display_cancel(mupsi_display* d) {
  if (d) set_cancel(d, 1);
}

int mupsi_gpu_display_stop(mupsi_display* d) {
  clear_error();
  if (!d) return fail(MUPSI_ERR_INVALID, "null display");
  int rc = stop_thread(d);
  if (rc != MUPSI_OK) return fail(rc, d->error);
  return MUPSI_OK;
}

int32_t mupsi_gpu_display_running(const mupsi_display* d) { return d ? d->running.load() : 0; }
int32_t mupsi_gpu_display_spp_pass_done(const mupsi_display* d) { return d ? d->spp_done.load() : 0; }
void mupsi_gpu_display_ack_spp_pass(mupsi_display* d) {
  if (d) d->spp_done.store(0);
}
int32_t mupsi_gpu_display_current_spp(const mupsi_display* d) { return d ? d->current.load() : 0; }

int mupsi_gpu_display_copy_raw(mupsi_display* d, float* dst, int32_t width, int32_t height) {
  return copy_front(d, dst, width, height, false);
}
int mupsi_gpu_display_copy_tonemapped(mupsi_display* d, float* dst, int32_t width, int32_t height) {
  return copy_front(d, dst, width, height, true);
}

}  // extern "C"
