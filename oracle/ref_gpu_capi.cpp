// Test/baseline-only C-ABI over the reference's own GPU renderer
// (cuda/gpu_render.cu + cuda/wavefront.cu of joelsalzman/beamtrace2007,
// compiled for sm_100a from its sources by oracle/Makefile into
// oracle/_ref/libbtref_gpu.so).  It measures the reference's wavefront
// engine on the same scenes; nothing in the product links it.
#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "cuda/gpu_render.h"
#include "render/render.h"

#define BTRG_API extern "C" __attribute__((visibility("default")))

using namespace bt;

namespace {
struct Ctx {
  Scene scene;
  KdTree tree;
  GpuRenderer* gpu = nullptr;
};
}  // namespace

BTRG_API int btrg_available() { return gpuAvailable(nullptr) ? 1 : 0; }

BTRG_API void* btrg_create(const float* pos, int64_t nv, const uint32_t* tris, int64_t nt, double costIntersect) {
  Ctx* c = new Ctx();
  c->scene.pos.resize(size_t(nv));
  for (int64_t i = 0; i < nv; ++i) c->scene.pos[size_t(i)] = Vec3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  for (int64_t t = 0; t < nt; ++t) c->scene.addTri(tris[3 * t], tris[3 * t + 1], tris[3 * t + 2], 0);
  c->scene.finalize();
  KdBuildParams kp;
  kp.costIntersect = Real(costIntersect);
  c->tree.build(c->scene, kp);
  c->gpu = new GpuRenderer(c->scene, c->tree);
  return c;
}

BTRG_API void btrg_destroy(void* h) {
  Ctx* c = static_cast<Ctx*>(h);
  delete c->gpu;
  delete c;
}

// GpuRenderer::softShadows on a camera (eye fwd right down halfW halfH);
// timing: [primary s, trace s (GPU kernels + CPU fallback), kernel s,
// fallback s, overflow pixels].
BTRG_API void btrg_soft(void* h, const double* cv, int W, int H, const double* l, int exact, int32_t* tri,
                        float* vis, float* E, double* timing) {
  Ctx* c = static_cast<Ctx*>(h);
  Camera cam;
  cam.eye = Vec3(Real(cv[0]), Real(cv[1]), Real(cv[2]));
  cam.fwd = Vec3(Real(cv[3]), Real(cv[4]), Real(cv[5]));
  cam.right = Vec3(Real(cv[6]), Real(cv[7]), Real(cv[8]));
  cam.down = Vec3(Real(cv[9]), Real(cv[10]), Real(cv[11]));
  cam.halfW = Real(cv[12]);
  cam.halfH = Real(cv[13]);
  cam.W = W;
  cam.H = H;
  AreaLight L;
  L.c = Vec3(Real(l[0]), Real(l[1]), Real(l[2]));
  L.U = Vec3(Real(l[3]), Real(l[4]), Real(l[5]));
  L.V = Vec3(Real(l[6]), Real(l[7]), Real(l[8]));
  SoftOptions opt;
  opt.exact = exact != 0;
  SoftResult res;
  c->gpu->softShadows(cam, L, opt, res);
  const size_t n = size_t(W) * size_t(H);
  for (size_t k = 0; k < n; ++k) {
    if (tri) tri[k] = res.tri[k];
    if (vis) vis[k] = res.vis[k];
    if (E) E[k] = res.E[k];
  }
  timing[0] = res.stats.primarySeconds;
  timing[1] = res.stats.traceSeconds;
  timing[2] = c->gpu->lastKernelSeconds;
  timing[3] = c->gpu->lastFallbackSeconds;
  timing[4] = double(c->gpu->lastOverflowPixels);
}

// GpuRenderer::primary (tile roots) and GpuRenderer::pointShadows on its
// hit polygons, each wall-clocked around the synchronous call; out:
// [primary s, point s, hit polygons, shadow polygons, primary kernel s,
// point kernel s, primary overflow, point overflow, primary CPU-fallback s,
// point CPU-fallback s].
BTRG_API void btrg_primary_point(void* h, const double* cv, int W, int H, int tile, const double* light, double* out) {
  Ctx* c = static_cast<Ctx*>(h);
  Camera cam;
  cam.eye = Vec3(Real(cv[0]), Real(cv[1]), Real(cv[2]));
  cam.fwd = Vec3(Real(cv[3]), Real(cv[4]), Real(cv[5]));
  cam.right = Vec3(Real(cv[6]), Real(cv[7]), Real(cv[8]));
  cam.down = Vec3(Real(cv[9]), Real(cv[10]), Real(cv[11]));
  cam.halfW = Real(cv[12]);
  cam.halfH = Real(cv[13]);
  cam.W = W;
  cam.H = H;
  std::vector<OutBeam> hits, shadow;
  RenderStats rs;
  auto t0 = std::chrono::steady_clock::now();
  c->gpu->primary(cam, false, hits, rs, tile);
  auto t1 = std::chrono::steady_clock::now();
  out[4] = c->gpu->lastKernelSeconds;
  out[6] = double(c->gpu->lastOverflowPixels);
  out[8] = c->gpu->lastFallbackSeconds;
  std::vector<OutBeam> visible;
  for (const OutBeam& b : hits)
    if (b.tri >= 0) visible.push_back(b);
  auto t2 = std::chrono::steady_clock::now();
  c->gpu->pointShadows(cam, visible, Vec3(Real(light[0]), Real(light[1]), Real(light[2])), shadow, rs);
  auto t3 = std::chrono::steady_clock::now();
  out[0] = std::chrono::duration<double>(t1 - t0).count();
  out[1] = std::chrono::duration<double>(t3 - t2).count();
  out[2] = double(visible.size());
  out[3] = double(shadow.size());
  out[5] = c->gpu->lastKernelSeconds;
  out[7] = double(c->gpu->lastOverflowPixels);
  out[9] = c->gpu->lastFallbackSeconds;
}
