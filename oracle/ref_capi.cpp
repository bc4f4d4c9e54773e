// Test-only C-ABI over the reference's own CPU beam tracer.
//
// oracle/Makefile compiles this file together with the reference's CPU
// sources (src/util, src/scene, src/accel, src/beam, src/render of
// joelsalzman/beamtrace2007), once with Real = float and once with
// Real = double (BT_REAL_DOUBLE), into oracle/_ref/libbtref_{f,d}.so.
//
// It is the checker, never the thing measured or shipped: only tests/,
// __graft_entry__.smoke() and the cpu_baseline / reference legs of bench.py
// load it (through oracle/ref.py).  Every entry point calls the reference's
// public functions unchanged; the loops here only re-create the callers the
// reference has for them (render.cpp, gpu_render.cu) so that per-root output
// and counters can be read back.
#include <atomic>
#include <string>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "beam/beam_tracer.h"
#include "beam/wavefront.h"
#include "render/point_core.h"
#include "render/render.h"
#include "ray/ray_tracer.h"
#include "util/misc.h"

#define BTR_API extern "C" __attribute__((visibility("default")))

using namespace bt;

namespace {

struct RefCtx {
  Scene scene;
  KdTree tree;
};

// Counter layout shared with oracle/ref.py (TraceStats, stats.h:8-42).
void packStats(const TraceStats& t, uint64_t* s) {
  if (!s) return;
  s[0] = t.kdSteps;
  s[1] = t.leafVisits;
  s[2] = t.triTests;
  s[3] = t.hits;
  s[4] = t.splits;
  s[5] = t.beams;
  s[6] = t.rootBeams;
  s[7] = t.presplitBeams;
  s[8] = t.mailboxSkips;
  s[9] = t.fiveSplits;
  s[10] = t.visibleTris;
  s[11] = t.rays;
  s[12] = t.climbs;
  double d = t.droppedArea;
  std::memcpy(&s[13], &d, sizeof(double));
}

// cam: eye[3] fwd[3] right[3] down[3] halfW halfH (render_types.h:15-39).
Camera makeCam(const double* c, int W, int H) {
  Camera cam;
  cam.eye = Vec3(Real(c[0]), Real(c[1]), Real(c[2]));
  cam.fwd = Vec3(Real(c[3]), Real(c[4]), Real(c[5]));
  cam.right = Vec3(Real(c[6]), Real(c[7]), Real(c[8]));
  cam.down = Vec3(Real(c[9]), Real(c[10]), Real(c[11]));
  cam.halfW = Real(c[12]);
  cam.halfH = Real(c[13]);
  cam.W = W;
  cam.H = H;
  return cam;
}

AreaLight makeLight(const double* l) {
  AreaLight L;
  L.c = Vec3(Real(l[0]), Real(l[1]), Real(l[2]));
  L.U = Vec3(Real(l[3]), Real(l[4]), Real(l[5]));
  L.V = Vec3(Real(l[6]), Real(l[7]), Real(l[8]));
  return L;
}

template <class F>
void parallelFor(int n, int threads, F&& f) {
  threads = threads < 1 ? 1 : threads;
  std::atomic<int> next(0);
  auto worker = [&](int id) {
    for (int i = next++; i < n; i = next++) f(id, i);
  };
  std::vector<std::thread> th;
  for (int t = 1; t < threads; ++t) th.emplace_back(worker, t);
  worker(0);
  for (auto& t : th) t.join();
}

// Polygon sink with the root index of every output piece.
struct PolyOut {
  double* x;
  double* y;
  int32_t* n;
  int32_t* tri;
  double* area;
  int32_t* root;
  int64_t cap;
  int64_t count = 0;
  void push(const OutBeam& ob, int r) {
    if (count < cap) {
      for (int i = 0; i < 4; ++i) {
        x[count * 4 + i] = double(ob.x[i]);
        y[count * 4 + i] = double(ob.y[i]);
      }
      n[count] = ob.n;
      tri[count] = ob.tri;
      area[count] = double(ob.area);
      root[count] = r;
    }
    ++count;
  }
};

}  // namespace

BTR_API int btr_real_size() { return int(sizeof(Real)); }

// Builds Scene (positions, triangles; Scene::finalize drops degenerate
// triangles) and its kd-tree (KdTree::build with the given SAH cost).
BTR_API void* btr_create(const float* pos, int64_t nv, const uint32_t* tris, int64_t nt, double costIntersect,
                         int singleLeaf) {
  RefCtx* c = new RefCtx();
  c->scene.pos.resize(size_t(nv));
  for (int64_t i = 0; i < nv; ++i) c->scene.pos[size_t(i)] = Vec3(Real(pos[3 * i]), Real(pos[3 * i + 1]), Real(pos[3 * i + 2]));
  for (int64_t t = 0; t < nt; ++t) c->scene.addTri(tris[3 * t], tris[3 * t + 1], tris[3 * t + 2], 0);
  c->scene.finalize();
  KdBuildParams kp;
  kp.costIntersect = Real(costIntersect);
  kp.singleLeaf = singleLeaf != 0;
  c->tree.build(c->scene, kp);
  return c;
}

BTR_API void btr_destroy(void* h) { delete static_cast<RefCtx*>(h); }

BTR_API int64_t btr_num_tris(void* h) { return static_cast<RefCtx*>(h)->scene.numTris(); }

BTR_API void btr_scene_export(void* h, uint32_t* tris, double* triN, double* triArea, double* bounds) {
  const Scene& s = static_cast<RefCtx*>(h)->scene;
  for (int t = 0; t < s.numTris(); ++t) {
    for (int k = 0; k < 3; ++k) {
      tris[3 * t + k] = s.tris[size_t(t)][size_t(k)];
      triN[3 * t + k] = double(s.triN[size_t(t)][k]);
    }
    triArea[t] = double(s.triArea[size_t(t)]);
  }
  for (int a = 0; a < 3; ++a) {
    bounds[a] = double(s.bounds.lo[a]);
    bounds[3 + a] = double(s.bounds.hi[a]);
  }
}

// sizes: nodes, leaf refs, leaves, max depth, build ms
BTR_API void btr_kd_sizes(void* h, int64_t* out) {
  const KdTree& t = static_cast<RefCtx*>(h)->tree;
  out[0] = int64_t(t.nodes.size());
  out[1] = int64_t(t.triIndices.size());
  out[2] = t.numLeaves;
  out[3] = t.maxDepthReached;
  out[4] = int64_t(t.buildSeconds * 1e3);
}

BTR_API void btr_kd_export(void* h, double* split, uint32_t* data, uint32_t* offset, uint32_t* triIndices,
                           uint32_t* parent, double* nodeBox, double* bounds) {
  const KdTree& t = static_cast<RefCtx*>(h)->tree;
  for (size_t i = 0; i < t.nodes.size(); ++i) {
    split[i] = double(t.nodes[i].split);
    data[i] = t.nodes[i].data;
    offset[i] = t.nodes[i].offset;
    parent[i] = t.parent[i];
    for (int a = 0; a < 3; ++a) {
      nodeBox[6 * i + a] = double(t.nodeBox[i].lo[a]);
      nodeBox[6 * i + 3 + a] = double(t.nodeBox[i].hi[a]);
    }
  }
  for (size_t i = 0; i < t.triIndices.size(); ++i) triIndices[i] = t.triIndices[i];
  for (int a = 0; a < 3; ++a) {
    bounds[a] = double(t.bounds.lo[a]);
    bounds[3 + a] = double(t.bounds.hi[a]);
  }
}

// Camera::make (render.cpp:14-25) -> eye fwd right down halfW halfH.
BTR_API void btr_camera_make(const double* eye, const double* target, double fov, const double* up, int W, int H,
                             double* out) {
  View v;
  v.eye = Vec3(Real(eye[0]), Real(eye[1]), Real(eye[2]));
  v.target = Vec3(Real(target[0]), Real(target[1]), Real(target[2]));
  v.fovY = Real(fov);
  Camera c = Camera::make(v, Vec3(Real(up[0]), Real(up[1]), Real(up[2])), W, H);
  const Vec3* vs[4] = {&c.eye, &c.fwd, &c.right, &c.down};
  for (int k = 0; k < 4; ++k)
    for (int a = 0; a < 3; ++a) out[3 * k + a] = double((*vs[k])[a]);
  out[12] = double(c.halfW);
  out[13] = double(c.halfH);
}

// The primary-ray pass of softShadows (render.cpp:352-381): tri, X, N per pixel.
BTR_API void btr_primary_rays(void* h, const double* camv, int W, int H, int threads, int32_t* tri, double* X,
                              double* N, uint64_t* stats) {
  RefCtx& c = *static_cast<RefCtx*>(h);
  Camera cam = makeCam(camv, W, H);
  RayTracer rt(c.scene, c.tree);
  std::vector<TraceStats> st(size_t(threads < 1 ? 1 : threads));
  parallelFor(H, threads, [&](int id, int y) {
    for (int x = 0; x < W; ++x) {
      size_t k = size_t(y) * size_t(W) + size_t(x);
      tri[k] = -1;
      for (int a = 0; a < 3; ++a) X[3 * k + a] = N[3 * k + a] = 0;
      Real qx, qy;
      cam.pixelToQ(Real(x) + Real(0.5), Real(y) + Real(0.5), qx, qy);
      Ray r;
      r.o = cam.eye;
      r.d = cam.dir(qx, qy);
      RayHit hit;
      if (!rt.intersect(r, hit, st[size_t(id)])) continue;
      tri[k] = hit.tri;
      Vec3 p = r.o + r.d * hit.t;
      Vec3 n = c.scene.triN[size_t(hit.tri)];
      if (dot(n, r.d) > 0) n = -n;
      for (int a = 0; a < 3; ++a) {
        X[3 * k + a] = double(p[a]);
        N[3 * k + a] = double(n[a]);
      }
    }
  });
  TraceStats tot;
  for (auto& s : st) tot.add(s);
  packStats(tot, stats);
}

// Soft shadows for supplied shading points (the per-pixel loop of
// softShadows, render.cpp:394-414): vis, E, Eunocc.  tri < 0 -> background.
BTR_API void btr_soft_points(void* h, const double* light, double offset, int64_t n, const int32_t* tri,
                             const double* X, const double* N, int exact, int mailbox, int trail, int threads,
                             double* vis, double* E, double* Eu, uint64_t* stats) {
  RefCtx& c = *static_cast<RefCtx*>(h);
  const AreaLight L = makeLight(light);
  const Real A = L.area();
  const int nt = threads < 1 ? 1 : threads;
  std::vector<BeamTracer*> tracers;
  for (int t = 0; t < nt; ++t) {
    BeamTracer* b = new BeamTracer(c.scene, c.tree);
    b->useMailbox = mailbox != 0;
    b->useTrail = trail != 0;
    b->keepOutput = false;
    tracers.push_back(b);
  }
  const int64_t chunk = 64;
  const int nChunks = int((n + chunk - 1) / chunk);
  parallelFor(nChunks, nt, [&](int id, int ci) {
    BeamTracer& btr = *tracers[size_t(id)];
    for (int64_t k = ci * chunk; k < n && k < (ci + 1) * chunk; ++k) {
      const int T = tri[k];
      if (T < 0) {
        vis[k] = -1;
        E[k] = 0;
        Eu[k] = 0;
        continue;
      }
      Vec3 p = Vec3(Real(X[3 * k]), Real(X[3 * k + 1]), Real(X[3 * k + 2]));
      Vec3 nn = Vec3(Real(N[3 * k]), Real(N[3 * k + 1]), Real(N[3 * k + 2]));
      Real G0 = lightCenterG(L, p, nn);
      Real Gx = 0;
      Real V = beamLightVisibility(btr, p, nn, T, L, Real(offset), exact ? &Gx : nullptr);
      vis[k] = double(V);
      Eu[k] = double(float(A * G0));
      E[k] = exact ? double(Gx) : double(A * G0 * V);
    }
  });
  TraceStats tot;
  for (BeamTracer* b : tracers) {
    tot.add(b->stats);
    delete b;
  }
  packStats(tot, stats);
}

// Sampled visibility with `samples` shadow rays (rayLightVisibility,
// render.cpp:305-337), seeded per point as softShadows does per pixel.
BTR_API void btr_soft_points_ray(void* h, const double* light, double offset, int64_t n, const int32_t* tri,
                                 const double* X, const double* N, const int32_t* px, const int32_t* py, int samples,
                                 int jitter, int threads, double* vis) {
  RefCtx& c = *static_cast<RefCtx*>(h);
  const AreaLight L = makeLight(light);
  RayTracer rt(c.scene, c.tree);
  std::vector<TraceStats> st(size_t(threads < 1 ? 1 : threads));
  parallelFor(int(n), threads, [&](int id, int k) {
    const int T = tri[k];
    if (T < 0) {
      vis[k] = -1;
      return;
    }
    Vec3 p = Vec3(Real(X[3 * k]), Real(X[3 * k + 1]), Real(X[3 * k + 2]));
    Vec3 nn = Vec3(Real(N[3 * k]), Real(N[3 * k + 1]), Real(N[3 * k + 2]));
    uint64_t seed = (uint64_t(uint32_t(py[k])) << 32) ^ uint64_t(uint32_t(px[k])) ^ 0x9E3779B97F4A7C15ULL;
    vis[k] = double(rayLightVisibility(rt, p, nn, T, L, Real(offset), samples, jitter != 0, seed, st[size_t(id)]));
  });
}

// The whole CPU soft-shadow pipeline, softShadows (render.cpp:339-424),
// as bt_render --mode softshadow --method beam runs it; timing[0] = primary
// seconds, timing[1] = trace seconds.
BTR_API void btr_soft_image(void* h, const double* camv, int W, int H, const double* light, int exact, int threads,
                            int mailbox, int trail, int32_t* tri, float* vis, float* E, float* Eu, double* timing,
                            uint64_t* stats) {
  RefCtx& c = *static_cast<RefCtx*>(h);
  Camera cam = makeCam(camv, W, H);
  SoftOptions opt;
  opt.useBeams = true;
  opt.exact = exact != 0;
  opt.threads = threads;
  opt.mailbox = mailbox != 0;
  opt.trail = trail != 0;
  SoftResult res;
  softShadows(c.scene, c.tree, cam, makeLight(light), opt, res);
  const size_t np = size_t(W) * size_t(H);
  for (size_t k = 0; k < np; ++k) {
    tri[k] = res.tri[k];
    vis[k] = res.vis[k];
    E[k] = res.E[k];
    Eu[k] = res.Eunocc[k];
  }
  timing[0] = res.stats.primarySeconds;
  timing[1] = res.stats.traceSeconds;
  packStats(res.stats.trace, stats);
}

// Primary visibility with one root per tile x tile pixels, each traced on its
// own (the roots of GpuRenderer::primary, gpu_render.cu:730-742, traced as
// primaryRootsCPU does, render.cpp:487-501).  Every output piece (hit and
// background) is returned with its tile index.  Returns the piece count.
BTR_API int64_t btr_primary_tiles(void* h, const double* camv, int W, int H, int cull, int tile, int mailbox,
                                  int trail, int64_t cap, double* x, double* y, int32_t* n, int32_t* tri,
                                  double* area, int32_t* root, uint64_t* stats) {
  RefCtx& c = *static_cast<RefCtx*>(h);
  Camera cam = makeCam(camv, W, H);
  BeamTracer btr(c.scene, c.tree);
  btr.useMailbox = mailbox != 0;
  btr.useTrail = trail != 0;
  BeamQuery q;
  q.plane = cam.plane();
  q.mode = BeamMode::Nearest;
  q.cullBackfaces = cull != 0;
  const int tilesX = (W + tile - 1) / tile, tilesY = (H + tile - 1) / tile;
  PolyOut po{x, y, n, tri, area, root, cap};
  BeamOutput out;
  for (int i = 0; i < tilesX * tilesY; ++i) {
    int tx = i % tilesX, ty = i / tilesX;
    int x0 = tx * tile, y0 = ty * tile, x1 = std::min(W, x0 + tile), y1 = std::min(H, y0 + tile);
    Real a, b, cc, d;
    cam.pixelToQ(Real(x0), Real(y0), a, b);
    cam.pixelToQ(Real(x1), Real(y1), cc, d);
    Poly2 p;
    p.push(a, b);
    p.push(cc, b);
    p.push(cc, d);
    p.push(a, d);
    btr.trace(q, &p, 1, out);
    for (const OutBeam& ob : out.beams) po.push(ob, i);
  }
  packStats(btr.stats, stats);
  return po.count;
}

// Point-light shadows for the given primary hit beams, one root each
// (beamPointShadows, render.cpp:209-247): the shadowed image-plane polygons
// with the index of the hit beam they came from.  Returns the polygon count.
BTR_API int64_t btr_point_shadows(void* h, const double* camv, int W, int H, const double* light, int64_t nh,
                                  const double* hx, const double* hy, const int32_t* hn, const int32_t* htri,
                                  int mailbox, int trail, int64_t cap, double* x, double* y, int32_t* n, int32_t* tri,
                                  double* area, int32_t* root, uint64_t* stats) {
  RefCtx& c = *static_cast<RefCtx*>(h);
  Camera cam = makeCam(camv, W, H);
  const Vec3 Lp = Vec3(Real(light[0]), Real(light[1]), Real(light[2]));
  BeamTracer btr(c.scene, c.tree);
  btr.useMailbox = mailbox != 0;
  btr.useTrail = trail != 0;
  BeamPlane camPlane = cam.plane();
  PolyOut po{x, y, n, tri, area, root, cap};
  BeamOutput out;
  for (int64_t i = 0; i < nh; ++i) {
    OutBeam pb;
    for (int k = 0; k < 4; ++k) {
      pb.x[k] = Real(hx[4 * i + k]);
      pb.y[k] = Real(hy[4 * i + k]);
    }
    pb.n = hn[i];
    pb.tri = htri[i];
    pb.area = 0;
    if (pb.tri < 0) continue;
    const int T = pb.tri;
    BeamQuery q;
    Poly2 rootPoly;
    if (!pointShadowSetup(cam.eye, cam.fwd, cam.right, cam.down, c.scene.triN[size_t(T)], c.scene.v(T, 0), T, Lp,
                          pb.x, pb.y, pb.n, q, rootPoly)) {
      po.push(pb, int(i));
      continue;
    }
    btr.trace(q, &rootPoly, 1, out);
    for (const OutBeam& sb : out.beams) {
      if (sb.tri < 0) continue;
      OutBeam ip;
      if (pointShadowToImage(camPlane, q.plane, sb.x, sb.y, sb.n, T, ip)) po.push(ip, int(i));
    }
  }
  packStats(btr.stats, stats);
  return po.count;
}

// rasterize (render.cpp:49-95) at one sample per pixel: primary polygons set
// tri ids, shadow polygons set flags.
BTR_API void btr_rasterize(const double* camv, int W, int H, int64_t np, const double* px, const double* py,
                           const int32_t* pn, const int32_t* ptri, int64_t ns, const double* sx, const double* sy,
                           const int32_t* sn, const int32_t* stri, int32_t* triOut, uint8_t* flagOut) {
  Camera cam = makeCam(camv, W, H);
  auto load = [](int64_t m, const double* x, const double* y, const int32_t* n, const int32_t* t) {
    std::vector<OutBeam> v(static_cast<size_t>(m));
    for (int64_t i = 0; i < m; ++i) {
      for (int k = 0; k < 4; ++k) {
        v[size_t(i)].x[k] = Real(x[4 * i + k]);
        v[size_t(i)].y[k] = Real(y[4 * i + k]);
      }
      v[size_t(i)].n = n[i];
      v[size_t(i)].tri = t[i];
      v[size_t(i)].area = 0;
    }
    return v;
  };
  SampleBuffer sb;
  sb.init(W, H, 1);
  rasterize(load(np, px, py, pn, ptri), cam, sb, false);
  if (ns > 0) rasterize(load(ns, sx, sy, sn, stri), cam, sb, true);
  for (size_t k = 0; k < sb.tri.size(); ++k) {
    triOut[k] = sb.tri[k];
    flagOut[k] = sb.flag[k];
  }
}

// Lambert's formula (soft_core.h:18-33) for one polygon, for the exact-E tests.
BTR_API double btr_form_factor(const double* x, const double* n, const double* poly, int count) {
  Vec3 P[8];
  for (int i = 0; i < count && i < 8; ++i) P[i] = Vec3(Real(poly[3 * i]), Real(poly[3 * i + 1]), Real(poly[3 * i + 2]));
  return double(polygonFormFactorG(Vec3(Real(x[0]), Real(x[1]), Real(x[2])), Vec3(Real(n[0]), Real(n[1]), Real(n[2])),
                                   P, count));
}

// The reference's float/double tolerances (real.h:31-39).
BTR_API void btr_tolerances(double* out) {
  out[0] = double(kEpsRel);
  out[1] = double(kKdRel);
  out[2] = double(kDegRel);
}

// ---- scene ingest: the reference's parseConfig + buildScene (scene.cpp) ----
namespace {
struct RefConfig {
  SceneConfig cfg;
  Scene scene;
  std::string err;
};
}  // namespace

// Parses `text` and builds its scene; returns a handle, or null with the
// reason in btr_config_error.  The handle is freed by btr_config_free.
thread_local std::string g_cfgErr;
BTR_API void* btr_config_build(const char* text) {
  auto* r = new RefConfig();
  std::string err;
  if (!parseConfig(text, r->cfg, err) || !buildScene(r->cfg, r->scene, err)) {
    g_cfgErr = err;
    delete r;
    return nullptr;
  }
  return r;
}
BTR_API const char* btr_config_error() { return g_cfgErr.c_str(); }
BTR_API void btr_config_free(void* h) { delete static_cast<RefConfig*>(h); }

// counts: verts, tris, materials, views, cull, has point light, has area light
BTR_API void btr_config_counts(void* h, int64_t* out) {
  const auto* r = static_cast<RefConfig*>(h);
  out[0] = int64_t(r->scene.pos.size());
  out[1] = int64_t(r->scene.tris.size());
  out[2] = int64_t(r->scene.matColor.size());
  out[3] = int64_t(r->cfg.views.size());
  out[4] = r->cfg.cullBackfaces;
  out[5] = r->cfg.hasPointLight;
  out[6] = r->cfg.hasAreaLight;
}

// pos (3/vert), tris (3/tri), triMat, matColor (3/material), views (7/view:
// eye, target, fov), lights (up, point, c, U, V, intensity, background: 22)
BTR_API void btr_config_arrays(void* h, double* pos, uint32_t* tris, uint16_t* mat, double* color, double* views,
                               double* lights) {
  const auto* r = static_cast<RefConfig*>(h);
  const Scene& s = r->scene;
  auto put = [](double* d, const Vec3& v) {
    d[0] = double(v.x);
    d[1] = double(v.y);
    d[2] = double(v.z);
  };
  for (size_t i = 0; i < s.pos.size(); ++i) put(pos + 3 * i, s.pos[i]);
  for (size_t i = 0; i < s.tris.size(); ++i)
    for (int k = 0; k < 3; ++k) tris[3 * i + size_t(k)] = s.tris[i][size_t(k)];
  for (size_t i = 0; i < s.triMat.size(); ++i) mat[i] = s.triMat[i];
  for (size_t i = 0; i < s.matColor.size(); ++i) put(color + 3 * i, s.matColor[i]);
  for (size_t i = 0; i < r->cfg.views.size(); ++i) {
    put(views + 7 * i, r->cfg.views[i].eye);
    put(views + 7 * i + 3, r->cfg.views[i].target);
    views[7 * i + 6] = double(r->cfg.views[i].fovY);
  }
  const SceneConfig& c = r->cfg;
  put(lights, c.up);
  put(lights + 3, c.pointLight);
  put(lights + 6, c.lightC);
  put(lights + 9, c.lightU);
  put(lights + 12, c.lightV);
  lights[15] = double(c.lightIntensity);
  put(lights + 16, c.background);
  lights[19] = lights[20] = lights[21] = 0;
}

// The reference's own fuzzy split and clean-up (beam_geom.h:83-150) of one
// polygon by one line, for the polygon fuzz test; corners as doubles of the
// build's Real.  Returns 0 if its splitter reported an overflow.
BTR_API int btr_split_clean(const double* px, const double* py, int n, const double* line, double eps, double* inx,
                            double* iny, int* nin, double* outx, double* outy, int* nout) {
  PolyN<kMaxPoly> p, in, out;
  for (int i = 0; i < n && i < kMaxPoly; ++i) p.push(Real(px[i]), Real(py[i]));
  Line2 L;
  L.a = Real(line[0]);
  L.b = Real(line[1]);
  L.c = Real(line[2]);
  if (!splitPoly(p, L, Real(eps), in, out)) return 0;
  cleanPoly(in, Real(eps));
  cleanPoly(out, Real(eps));
  *nin = in.n;
  *nout = out.n;
  for (int i = 0; i < in.n; ++i) {
    inx[i] = double(in.x[i]);
    iny[i] = double(in.y[i]);
  }
  for (int i = 0; i < out.n; ++i) {
    outx[i] = double(out.x[i]);
    outy[i] = double(out.y[i]);
  }
  return 1;
}

BTR_API double btr_poly_area(const double* px, const double* py, int n) {
  PolyN<kMaxPoly> p;
  for (int i = 0; i < n && i < kMaxPoly; ++i) p.push(Real(px[i]), Real(py[i]));
  return double(p.area());
}
