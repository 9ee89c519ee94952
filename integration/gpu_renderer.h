// GpuRenderer: the reference host's GPU replacement for Renderer
// (rendering/renderer.h:10-45). It takes the same RenderContext snapshot
// (rendering/render_context.h:16-27) that Controller::start/startProgressive
// build on their render thread (controller/controller.cpp:268-345), flattens
// its scene into one mupsi_scene_desc, and renders through libmupsi_gpu.so
// (include/mupsi_gpu.h) instead of the OpenMP pixel loop of
// Renderer::startRenderProgressive (renderer.cpp:22-49). The result lands in a
// Framebuffer of the reference's own type, so the Controller's front/back
// buffer swap and copyDisplayTo/copyDisplayRawTo read it unchanged.
//
// In the reference tree this file sits beside renderer.h; GpuRenderer reads
// private members of Scene, Camera, GPMedium, SDFMedium, ExternalGPMedium,
// SparseGPNoiseGenerator, the mean functions, Mesh, LambertianBsdf and
// BitmapTexture, so those classes declare `friend class GpuRenderer;`
// (gpu_renderer.cpp lists the members it reads).
#pragma once

#include <atomic>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "mupsi_gpu.h"
#include "rendering/framebuffer.h"
#include "rendering/render_context.h"

namespace mupsi {

class GpuRenderer {
 public:
  GpuRenderer() = default;
  ~GpuRenderer();
  GpuRenderer(const GpuRenderer&) = delete;
  GpuRenderer& operator=(const GpuRenderer&) = delete;

  // Renderer::setCancelFlag: the host's flag is polled between the library's
  // waves of passes (the reference polls it per pass and per pixel).
  void setCancelFlag(std::atomic<bool>* flag) { cancel_ = flag; }

  // Renderer::prepareRender: copy the scene to the device (BVHs are built by
  // the library), size the framebuffer. False (message in error()) if the
  // scene holds something the GPU path cannot express.
  bool prepareRender(const RenderContext& ctx);

  // Renderer::startRenderProgressive: passes 0..targetSpp-1, onSpp(passes
  // done) after each wave of passes; false when cancelled or failed.
  bool startRenderProgressive(const RenderContext& ctx, int targetSpp,
                              std::function<void(int currentSpp)> onSpp = {});

  std::shared_ptr<Framebuffer> getFramebuffer() const { return framebuffer_; }
  const std::string& error() const { return error_; }

 private:
  bool fail(const std::string& msg);

  mupsi_scene* scene_ = nullptr;
  std::shared_ptr<Framebuffer> framebuffer_;
  std::atomic<bool>* cancel_ = nullptr;
  std::vector<float> rgb_;  // width * height * 3, row y = camera y
  int width_ = 0, height_ = 0;
  std::string error_;
};

}  // namespace mupsi
