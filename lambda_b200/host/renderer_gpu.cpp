// renderer_gpu.cpp — Renderer::render (include/renderer.hpp:39,
// src/renderer.cpp:14-61) on the B200 through the C ABI of lambda_gpu.h.
//
// Linked into the reference's own `lambda` CLI in place of its CPU render
// (lambda_b200/host/Makefile): the reference's loader, CLI, tone map and
// PNG output are unchanged and call this function exactly where they
// called the OpenMP renderer (src/main.cpp:41).  The render settings are
// the Renderer's public members MAX_SCATTERINGS, SPP and SAMPLE_P
// (include/renderer.hpp:35-37); the environment variable LGPU_SEED selects
// the random streams (default 0).
#include <cstdlib>
#include <stdexcept>
#include <string>

#include "lgpu_flatten.hpp"
#include "renderer.hpp"

namespace {

// one context per process, created on the first render
lgpu_ctx* context() {
  static lgpu_ctx* ctx = nullptr;
  if (!ctx) {
    int const rc = lgpu_create(0, &ctx);
    if (rc != LGPU_OK) throw std::runtime_error("lgpu_create failed (" + std::to_string(rc) + "): no CUDA device");
  }
  return ctx;
}

}  // namespace

void Renderer::render(nl::cg::scene const& scene, rendering& buffer) {
  lgpu_ctx* const ctx = context();
  lgpu_host::flat_scene flat;
  lgpu_host::flatten(scene, flat);
  if (lgpu_upload_scene(ctx, &flat.scene) != LGPU_OK) throw std::runtime_error(lgpu_last_error(ctx));
  uint64_t const w = scene.cam.width, h = scene.cam.height;
  buffer.img.init(w, h);
  lgpu_render_params p{};
  p.spp = uint32_t(SPP);
  p.max_scatterings = uint32_t(MAX_SCATTERINGS);
  p.sample_p = SAMPLE_P;
  const char* seed = std::getenv("LGPU_SEED");
  p.seed = seed ? std::strtoull(seed, nullptr, 10) : 0;
  // linRGB is three packed floats, so the image data is the W*H*3 output
  static_assert(sizeof(nl::cg::linRGB) == 3 * sizeof(float), "linRGB must be three packed floats");
  if (lgpu_render(ctx, &p, reinterpret_cast<float*>(buffer.img.data.data())) != LGPU_OK)
    throw std::runtime_error(lgpu_last_error(ctx));
}
