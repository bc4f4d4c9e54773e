// bt::GpuRenderer and bt::gpuAvailable (cuda/gpu_render.h of
// joelsalzman/beamtrace2007) on top of the C-ABI of libbt_gpu.so.
//
// Compiled against the reference's own headers (cuda/gpu_render.h,
// render/render_types.h, accel/kdtree.h), so its applications
// (apps/bt_render.cpp as bt_render_cuda, cuda/test_cuda.cpp) link against
// this file and libbt_gpu.so in place of cuda/gpu_render.cu and
// cuda/wavefront.cu.  Every GPU call goes through include/bt_gpu.h.
//
// Differences of contract, all on the side of the caller:
//   * Roots over budget are retried on the GPU with a 16x budget instead of
//     being recomputed on the CPU: lastOverflowPixels counts them (roots over
//     budget in their first pass, as the reference counts the pixels it
//     hands to the CPU) and lastFallbackSeconds stays 0.
//   * A failing call throws std::runtime_error with bt_gpu_last_error()
//     (the reference aborts the process on CUDA errors, gpu_common.cuh:15-22).
//   * useMailbox and useWavefront are accepted and ignored: the engine has
//     one path, without mailboxing (bitwise the reference's trail engine).
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "bt_gpu.h"
#include "cuda/gpu_render.h"
#include "render/render_types.h"
#include "render/soft_core.h"

namespace bt {

namespace {

void check(int code, const char* what) {
  if (code != BT_OK) throw std::runtime_error(std::string(what) + ": " + bt_gpu_last_error());
}

bt_camera toCam(const Camera& c) {
  bt_camera o;
  const Vec3* v[4] = {&c.eye, &c.fwd, &c.right, &c.down};
  float* d[4] = {o.eye, o.fwd, o.right, o.down};
  for (int i = 0; i < 4; ++i) {
    d[i][0] = float(v[i]->x);
    d[i][1] = float(v[i]->y);
    d[i][2] = float(v[i]->z);
  }
  o.half_w = float(c.halfW);
  o.half_h = float(c.halfH);
  o.W = c.W;
  o.H = c.H;
  return o;
}

void toStats(const bt_run_info& in, TraceStats& t) {
  t.kdSteps += in.kd_steps;
  t.leafVisits += in.leaf_visits;
  t.triTests += in.tri_tests;
  t.hits += in.hits;
  t.splits += in.splits;
  t.beams += in.beams;
  t.rootBeams += in.root_beams;
  t.presplitBeams += in.presplit_beams;
  t.fiveSplits += in.five_splits;
  t.climbs += in.climbs;
  t.droppedArea += in.dropped_area;
}

// Host staging of a polygon list in the C-ABI's layout.
struct PolyBuf {
  std::vector<float> x, y, area;
  std::vector<int32_t> n, tri, root;
  void resize(size_t cap) {
    x.assign(4 * cap, 0.f);
    y.assign(4 * cap, 0.f);
    area.assign(cap, 0.f);
    n.assign(cap, 0);
    tri.assign(cap, 0);
    root.assign(cap, 0);
  }
  bt_polys view() {
    bt_polys p;
    p.x = x.data();
    p.y = y.data();
    p.n = n.data();
    p.tri = tri.data();
    p.area = area.data();
    p.root = root.data();
    p.cap = int64_t(n.size());
    return p;
  }
  void append(size_t count, std::vector<OutBeam>& out) const {
    for (size_t k = 0; k < count; ++k) {
      OutBeam b;
      for (int i = 0; i < 4; ++i) {
        b.x[i] = Real(x[4 * k + size_t(i)]);
        b.y[i] = Real(y[4 * k + size_t(i)]);
      }
      b.n = n[k];
      b.tri = tri[k];
      b.area = Real(area[k]);
      out.push_back(b);
    }
  }
};

}  // namespace

struct GpuRenderer::Impl {
  bt_gpu_ctx* ctx = nullptr;
  bt_gpu_config cfg{};
  // host copies of the scene and tree in the C-ABI's structure-of-arrays form
  std::vector<float> pos, triN, split, nodeBox;
  std::vector<uint32_t> tris, data, offset;
  bt_scene_desc sd{};
  bt_kd_desc kd{};
};

bool gpuAvailable(GpuInfo* info) {
  bt_gpu_info gi;
  if (bt_gpu_available(&gi) != BT_OK) return false;
  if (info) {
    info->name = gi.name;
    info->smCount = gi.sm_count;
    info->memGB = gi.mem_gb;
  }
  return true;
}

GpuRenderer::GpuRenderer(const Scene& scene, const KdTree& tree) : impl_(new Impl), scene_(scene), tree_(tree) {
  Impl& m = *impl_;
  const size_t nv = scene.pos.size(), nt = scene.tris.size(), nn = tree.nodes.size();
  m.pos.resize(3 * nv);
  for (size_t i = 0; i < nv; ++i) {
    m.pos[3 * i] = float(scene.pos[i].x);
    m.pos[3 * i + 1] = float(scene.pos[i].y);
    m.pos[3 * i + 2] = float(scene.pos[i].z);
  }
  m.tris.resize(3 * nt);
  m.triN.resize(3 * nt);
  for (size_t t = 0; t < nt; ++t) {
    for (int k = 0; k < 3; ++k) m.tris[3 * t + size_t(k)] = scene.tris[t][size_t(k)];
    m.triN[3 * t] = float(scene.triN[t].x);
    m.triN[3 * t + 1] = float(scene.triN[t].y);
    m.triN[3 * t + 2] = float(scene.triN[t].z);
  }
  m.split.resize(nn);
  m.data.resize(nn);
  m.offset.resize(nn);
  m.nodeBox.resize(6 * nn);
  for (size_t i = 0; i < nn; ++i) {
    m.split[i] = float(tree.nodes[i].split);
    m.data[i] = tree.nodes[i].data;
    m.offset[i] = tree.nodes[i].offset;
    const AABB& b = tree.nodeBox[i];
    const float bx[6] = {float(b.lo.x), float(b.lo.y), float(b.lo.z), float(b.hi.x), float(b.hi.y), float(b.hi.z)};
    for (int k = 0; k < 6; ++k) m.nodeBox[6 * i + size_t(k)] = bx[k];
  }
  m.sd.pos = m.pos.data();
  m.sd.num_verts = int64_t(nv);
  m.sd.tris = m.tris.data();
  m.sd.tri_normals = m.triN.data();
  m.sd.num_tris = int64_t(nt);
  const float sb[6] = {float(scene.bounds.lo.x), float(scene.bounds.lo.y), float(scene.bounds.lo.z),
                       float(scene.bounds.hi.x), float(scene.bounds.hi.y), float(scene.bounds.hi.z)};
  memcpy(m.sd.bounds, sb, sizeof sb);
  m.kd.split = m.split.data();
  m.kd.data = m.data.data();
  m.kd.offset = m.offset.data();
  m.kd.parent = tree.parent.data();
  m.kd.node_box = m.nodeBox.data();
  m.kd.num_nodes = int64_t(nn);
  m.kd.tri_indices = tree.triIndices.data();
  m.kd.num_refs = int64_t(tree.triIndices.size());
  const float kb[6] = {float(tree.bounds.lo.x), float(tree.bounds.lo.y), float(tree.bounds.lo.z),
                       float(tree.bounds.hi.x), float(tree.bounds.hi.y), float(tree.bounds.hi.z)};
  memcpy(m.kd.bounds, kb, sizeof kb);
  bt_gpu_config_default(&m.cfg);
  m.cfg.budget = wfBudget;
  m.cfg.primary_budget = wfPrimaryBudget;
  m.cfg.capacity = int64_t(wfCapacity);
  check(bt_gpu_create(&m.sd, &m.kd, &m.cfg, &m.ctx), "bt_gpu_create");
}

GpuRenderer::~GpuRenderer() {
  if (impl_) bt_gpu_destroy(impl_->ctx);
  delete impl_;
}

namespace {
// The public tunables may change between calls: a new context follows them.
void syncConfig(GpuRenderer::Impl& m, int budget, int primaryBudget, size_t capacity) {
  if (m.cfg.budget == budget && m.cfg.primary_budget == primaryBudget && m.cfg.capacity == int64_t(capacity)) return;
  bt_gpu_destroy(m.ctx);
  m.ctx = nullptr;
  m.cfg.budget = budget;
  m.cfg.primary_budget = primaryBudget;
  m.cfg.capacity = int64_t(capacity);
  check(bt_gpu_create(&m.sd, &m.kd, &m.cfg, &m.ctx), "bt_gpu_create");
}
}  // namespace

void GpuRenderer::softShadows(const Camera& cam, const AreaLight& light, const SoftOptions& opt, SoftResult& res) {
  if (!opt.useBeams) throw std::runtime_error("GpuRenderer::softShadows: only the beam method runs on the GPU");
  syncConfig(*impl_, wfBudget, wfPrimaryBudget, wfCapacity);
  const bt_camera c = toCam(cam);
  bt_area_light L;
  const Vec3* v[3] = {&light.c, &light.U, &light.V};
  float* d[3] = {L.c, L.U, L.V};
  for (int i = 0; i < 3; ++i) {
    d[i][0] = float(v[i]->x);
    d[i][1] = float(v[i]->y);
    d[i][2] = float(v[i]->z);
  }
  bt_soft_opts o;
  o.exact = opt.exact ? 1 : 0;
  o.offset = 0.f;
  const size_t np = size_t(cam.W) * size_t(cam.H);
  res.W = cam.W;
  res.H = cam.H;
  res.vis.assign(np, 0.f);
  res.E.assign(np, 0.f);
  res.Eunocc.assign(np, 0.f);
  res.tri.assign(np, -1);
  std::vector<int32_t> tri(np);
  bt_run_info info;
  check(bt_gpu_soft(impl_->ctx, &c, &L, &o, tri.data(), res.vis.data(), res.E.data(), res.Eunocc.data(), &info),
        "bt_gpu_soft");
  for (size_t k = 0; k < np; ++k) res.tri[k] = tri[k];
  res.stats = RenderStats();
  toStats(info, res.stats.trace);
  res.stats.primarySeconds = info.ms_primary * 1e-3;
  res.stats.traceSeconds = info.ms_trace * 1e-3;
  lastRounds = info.rounds;
  lastMaxQueue = info.max_spill;
  lastOverflowPixels = int(info.overflow_roots);
  lastFallbackSeconds = 0;
  lastKernelSeconds = info.ms_round * 1e-3;
}

void GpuRenderer::primary(const Camera& cam, bool cull, std::vector<OutBeam>& hitBeams, RenderStats& rs, int tile) {
  syncConfig(*impl_, wfBudget, wfPrimaryBudget, wfCapacity);
  const bt_camera c = toCam(cam);
  size_t cap = std::max<size_t>(size_t(1) << 16, 2 * size_t(cam.W) * size_t(cam.H));
  PolyBuf buf;
  bt_run_info info;
  int64_t count = 0;
  buf.resize(cap);
  bt_polys out = buf.view();
  check(bt_gpu_primary(impl_->ctx, &c, cull ? 1 : 0, tile, &out, &count, &info), "bt_gpu_primary");
  if (size_t(count) > cap) {  // more than fit: the polygons are still on the device
    buf.resize(size_t(count));
    out = buf.view();
    check(bt_gpu_last_polys(impl_->ctx, &out, &count), "bt_gpu_last_polys");
  }
  hitBeams.clear();
  buf.append(size_t(count), hitBeams);
  toStats(info, rs.trace);
  rs.traceSeconds += info.ms_total * 1e-3;
  lastRounds = info.rounds;
  lastMaxQueue = info.max_spill;
  lastOverflowPixels = int(info.overflow_roots);
  lastFallbackSeconds = 0;
  lastKernelSeconds = info.ms_round * 1e-3;
}

void GpuRenderer::pointShadows(const Camera& cam, const std::vector<OutBeam>& primaryHits, const Vec3& light,
                               std::vector<OutBeam>& shadowPolys, RenderStats& rs) {
  syncConfig(*impl_, wfBudget, wfPrimaryBudget, wfCapacity);
  const bt_camera c = toCam(cam);
  PolyBuf hits;
  hits.resize(std::max<size_t>(primaryHits.size(), 1));
  for (size_t k = 0; k < primaryHits.size(); ++k) {
    const OutBeam& b = primaryHits[k];
    for (int i = 0; i < 4; ++i) {
      hits.x[4 * k + size_t(i)] = float(b.x[i]);
      hits.y[4 * k + size_t(i)] = float(b.y[i]);
    }
    hits.n[k] = b.n;
    hits.tri[k] = b.tri;
    hits.area[k] = float(b.area);
    hits.root[k] = int32_t(k);
  }
  bt_polys hv = hits.view();
  const float Lp[3] = {float(light.x), float(light.y), float(light.z)};
  size_t cap = std::max<size_t>(size_t(1) << 16, 4 * primaryHits.size());
  PolyBuf buf;
  bt_run_info info;
  int64_t count = 0;
  buf.resize(cap);
  bt_polys out = buf.view();
  check(bt_gpu_point(impl_->ctx, &c, &hv, int64_t(primaryHits.size()), Lp, &out, &count, &info), "bt_gpu_point");
  if (size_t(count) > cap) {  // more than fit: the polygons are still on the device
    buf.resize(size_t(count));
    out = buf.view();
    check(bt_gpu_last_polys(impl_->ctx, &out, &count), "bt_gpu_last_polys");
  }
  buf.append(size_t(count), shadowPolys);
  toStats(info, rs.trace);
  rs.traceSeconds += info.ms_total * 1e-3;
  lastRounds = info.rounds;
  lastMaxQueue = info.max_spill;
  lastOverflowPixels = int(info.overflow_roots);
  lastFallbackSeconds = 0;
  lastKernelSeconds = info.ms_round * 1e-3;
}

}  // namespace bt
