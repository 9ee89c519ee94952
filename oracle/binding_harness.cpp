// Test harness of the reference-side binding (integration/gpu_renderer.*):
// the reference's own Controller::load reads a scene.json, the render context
// is snapshotted as Controller::start does (controller.cpp:279-292), and either
// the reference's Renderer or the GpuRenderer renders it progressively, so a
// test compares the two framebuffers. Test infrastructure: built beside the
// reference sources (oracle/Makefile, target `binding`), never linked by the
// product.
#include <atomic>
#include <cstdint>
#include <iostream>
#include <memory>

#include "controller/controller.h"
#include "geometry/scene.h"
#include "gpu_renderer.h"
#include "primitives/skydrome.h"
#include "rendering/renderer.h"
#include "rendering/trace.h"

using namespace mupsi;

namespace {
template <typename Tag, typename Tag::type M>
struct Reader {
  friend typename Tag::type member(Tag) { return M; }
};
struct ControllerScene {
  using type = std::shared_ptr<Scene> Controller::*;
  friend type member(ControllerScene);
};
template struct Reader<ControllerScene, &Controller::scene_>;

struct Loaded {
  Controller ctrl;
  std::shared_ptr<Scene> scene;
};
}  // namespace

extern "C" {

// Controller::load(json); constant_sky: give the scene Skydrome() (a constant
// sky of 1, as the benchmark scenes use) when the json names no skydrome image.
void* bind_load(const char* json_path, int constant_sky) {
  auto* h = new Loaded();
  if (!h->ctrl.load(json_path)) {
    delete h;
    return nullptr;
  }
  h->scene = h->ctrl.*member(ControllerScene{});
  if (constant_sky && !h->scene->getSkydrome()) h->scene->setSkydrome(std::make_shared<Skydrome>());
  return h;
}

void bind_size(void* hv, int* w, int* hh) {
  auto* h = static_cast<Loaded*>(hv);
  *w = h->scene->cam().width();
  *hh = h->scene->cam().height();
}

// One progressive render of passes 0..spp-1: use_gpu selects GpuRenderer or
// the reference's Renderer. cancel_after > 0 sets the host's cancel flag from
// the progress callback once that many passes are done. out[h*w*3] (row y =
// camera y) receives the framebuffer; *passes_seen the last callback value.
// Returns 0 when the render completed, 1 when cancelled, -1 on failure.
int bind_render(void* hv, int use_gpu, int spp, int cancel_after, float* out, int* passes_seen) {
  auto* h = static_cast<Loaded*>(hv);
  RenderContext ctx(h->scene->cam(), g_pathTracerSettings, g_gpSettings, h->scene);
  std::atomic<bool> cancel{false};
  int seen = 0;
  auto on = [&](int s) {
    seen = s;
    if (cancel_after > 0 && s >= cancel_after) cancel.store(true);
  };
  std::shared_ptr<Framebuffer> fb;
  bool done = false;
  if (use_gpu) {
    GpuRenderer r;
    r.setCancelFlag(&cancel);
    if (!r.prepareRender(ctx)) return -1;
    done = r.startRenderProgressive(ctx, spp, on);
    if (!done && !r.error().empty()) return -1;
    fb = r.getFramebuffer();
  } else {
    Renderer r;
    r.setCancelFlag(&cancel);
    r.prepareRender(ctx);
    done = r.startRenderProgressive(ctx, spp, on);
    fb = r.getFramebuffer();
  }
  if (passes_seen) *passes_seen = seen;
  const int w = fb->width(), hh = fb->height();
  for (int y = 0; y < hh; ++y)
    for (int x = 0; x < w; ++x) {
      const Vec3f& v = (*fb)(x, y).rgb;
      float* o = out + ((size_t)y * w + x) * 3;
      o[0] = v[0];
      o[1] = v[1];
      o[2] = v[2];
    }
  return done ? 0 : 1;
}

void bind_free(void* hv) { delete static_cast<Loaded*>(hv); }

}  // extern "C"
