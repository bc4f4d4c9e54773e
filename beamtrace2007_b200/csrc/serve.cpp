// Serving: continuous batching behind bt_gpu_submit / bt_gpu_poll
// (include/bt_gpu.h).  No counterpart in the reference, whose GpuRenderer
// is synchronous and renders one image per call (cuda/gpu_render.h:26-46).
//
// A context that serves owns threads and lanes (engine buffers and a stream
// of their own, viewing the context's scene pool; serve_engine.h):
//   - one soft lane runs streaming engine runs: the soft requests waiting
//     when a run starts, and those that arrive while it is younger than
//     fold_ms, share its rounds; each is handed back when its own roots are
//     done (engine.cu, laneSoftRun);
//   - vis_lanes lanes take primary-id and point-mask requests, one at a
//     time each, so several overlap with each other and with the soft run.
// Admission charges each request an estimate of the device memory its
// pixels need; a request is refused (BT_ERR_BUSY) while the resident scenes,
// the lanes' sub-beam queue high-water mark and the admitted requests would
// exceed the memory budget.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bt_gpu.h"
#include "serve_engine.h"

void btSetError(const char* msg);  // engine.cu: the message bt_gpu_last_error returns

namespace {

using Clock = std::chrono::steady_clock;

double msSince(Clock::time_point t) { return std::chrono::duration<double, std::milli>(Clock::now() - t).count(); }

struct Pending {
  uint64_t ticket = 0;
  bt_request r;
  Clock::time_point submitted, started;
  int64_t bytes = 0;  // what admission charged
};

struct Serving {
  bt_gpu_ctx* ctx = nullptr;
  bt_serve_config cfg;
  std::mutex m;
  std::condition_variable work;  // lanes wait for requests
  std::condition_variable ready; // pollers wait for completions
  std::deque<Pending> soft, vis;
  std::unordered_map<uint64_t, Pending> running;
  std::deque<bt_completion> done;
  uint64_t nextTicket = 1;
  bool stopping = false;
  bt_serve_stats st;
  bt_gpu_ctx* softLane = nullptr;
  std::vector<bt_gpu_ctx*> visLanes;
  std::vector<std::thread> threads;
};

Serving* servingOf(bt_gpu_ctx* c) { return static_cast<Serving*>(btserve::servingState(c)); }

int64_t softRootsOf(const bt_camera& cam) { return int64_t((cam.W + 7) / 8) * ((cam.H + 3) / 4) * 32; }

// Device bytes a request's pixels need, as admission charges them: soft
// 40 B/px of arena (ids, shading point and normal in; vis, E, Eu out) and
// 72 B per root; primary ids and point masks 9 B/px (ids, mask, ids for the
// raster) and about two output polygons of 52 B per pixel.
int64_t chargeOf(const bt_request& r) {
  const int64_t px = int64_t(r.cam.W) * r.cam.H;
  if (r.kind == BT_REQ_SOFT) return px * 40 + softRootsOf(r.cam) * 72;
  return px * (9 + 2 * 52);
}

// Hands a request back (called with S.m held).
void complete(Serving& S, const Pending& p, int status, const char* error) {
  bt_completion c;
  memset(&c, 0, sizeof c);
  c.ticket = p.ticket;
  c.user = p.r.user;
  c.kind = p.r.kind;
  c.status = status;
  c.ms_queued = std::chrono::duration<double, std::milli>(p.started - p.submitted).count();
  c.ms_total = msSince(p.submitted);
  if (status != BT_OK && error) snprintf(c.error, sizeof c.error, "%s", error);
  S.done.push_back(c);
  S.st.admitted_bytes -= p.bytes;
  S.st.completed++;
  S.st.running--;
  S.ready.notify_all();
}

// The soft lane's feed: takes waiting soft requests in arrival order while
// they fit in the run.
class Feed : public btserve::SoftFeed {
 public:
  explicit Feed(Serving& s) : S(s) {}
  bool runOpen = false;  // the run has started launching: further jobs are folded in

  bool next(btserve::StreamJob& j, uint64_t& tag, int64_t pixels, int64_t roots) override {
    std::lock_guard<std::mutex> lk(S.m);
    if (S.soft.empty() || S.stopping) {
      runOpen = true;  // whatever comes from now on joins a running run
      return false;
    }
    Pending& f = S.soft.front();
    const int64_t px = int64_t(f.r.cam.W) * f.r.cam.H;
    if (px > pixels || softRootsOf(f.r.cam) > roots) {
      runOpen = true;
      return false;
    }
    Pending p = f;
    S.soft.pop_front();
    p.started = Clock::now();
    S.st.queued--;
    S.st.running++;
    if (runOpen) S.st.soft_folded++;
    j.cam = p.r.cam;
    j.light = p.r.light;
    j.opts = p.r.opts;
    j.scene = p.r.scene;
    j.tri = p.r.tri;
    j.vis = p.r.vis;
    j.E = p.r.E;
    j.Eu = p.r.Eu;
    tag = p.ticket;
    S.running[p.ticket] = p;
    return true;
  }

  void finished(uint64_t tag, int status, const char* error) override {
    std::lock_guard<std::mutex> lk(S.m);
    auto it = S.running.find(tag);
    if (it == S.running.end()) return;
    const Pending p = it->second;
    S.running.erase(it);
    complete(S, p, status, error);
  }

 private:
  Serving& S;
};

void softLoop(Serving* S) {
  btserve::useDevice(S->ctx);
  Feed feed(*S);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(S->m);
      S->work.wait(lk, [&] { return S->stopping || !S->soft.empty(); });
      if (S->stopping) return;
      S->st.soft_runs++;
    }
    feed.runOpen = false;
    bt_run_info info;
    memset(&info, 0, sizeof info);
    std::shared_lock<std::shared_mutex> scene(btserve::sceneLock(S->ctx));
    btserve::laneView(S->softLane);
    btserve::laneSoftRun(S->softLane, feed, S->cfg.fold_ms, &info);  // failures reach each job's completion
  }
}

void visLoop(Serving* S, bt_gpu_ctx* lane) {
  btserve::useDevice(S->ctx);
  for (;;) {
    Pending p;
    {
      std::unique_lock<std::mutex> lk(S->m);
      S->work.wait(lk, [&] { return S->stopping || !S->vis.empty(); });
      if (S->stopping) return;
      p = S->vis.front();
      S->vis.pop_front();
      p.started = Clock::now();
      S->st.queued--;
      S->st.running++;
    }
    bt_run_info info;
    memset(&info, 0, sizeof info);
    int e;
    std::string why;
    {
      std::shared_lock<std::shared_mutex> scene(btserve::sceneLock(S->ctx));
      btserve::laneView(lane);
      e = btserve::laneVisibility(lane, p.r.kind, p.r.scene, p.r.cam, p.r.cull, p.r.tile, p.r.point_light, p.r.tri,
                                  p.r.mask, &info);
      if (e) why = btserve::lastError();
    }
    std::lock_guard<std::mutex> lk(S->m);
    complete(*S, p, e, why.c_str());
  }
}

}  // namespace

namespace btserve {

void stop(bt_gpu_ctx* c) {
  Serving* S = servingOf(c);
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->m);
    S->stopping = true;
  }
  S->work.notify_all();
  for (std::thread& t : S->threads) t.join();
  if (S->softLane) laneDestroy(S->softLane);
  for (bt_gpu_ctx* l : S->visLanes) laneDestroy(l);
  servingState(c) = nullptr;
  delete S;
}

}  // namespace btserve

extern "C" {

int bt_gpu_serve_start(bt_gpu_ctx* c, const bt_serve_config* cfg) {
  if (!c) {
    btSetError("bt_gpu_serve_start: no context");
    return BT_ERR_INVALID;
  }
  if (servingOf(c)) {
    btSetError("bt_gpu_serve_start: already serving");
    return BT_ERR_INVALID;
  }
  auto* S = new Serving();
  S->ctx = c;
  if (cfg) S->cfg = *cfg;
  else memset(&S->cfg, 0, sizeof S->cfg);
  bt_serve_config& k = S->cfg;
  if (k.vis_lanes <= 0) k.vis_lanes = 4;
  if (k.soft_jobs <= 0) k.soft_jobs = 256;
  if (k.soft_pixels <= 0) k.soft_pixels = int64_t(8) << 20;
  if (k.fold_ms <= 0) k.fold_ms = 100;
  memset(&S->st, 0, sizeof S->st);
  btserve::useDevice(c);
  int e = btserve::laneCreate(c, k.capacity, k.soft_pixels, k.soft_jobs, &S->softLane);
  if (!e && k.soft_blocks_per_sm > 0) btserve::laneBlocksPerSm(S->softLane, k.soft_blocks_per_sm);
  for (int i = 0; !e && i < k.vis_lanes; ++i) {
    bt_gpu_ctx* l = nullptr;
    e = btserve::laneCreate(c, k.capacity, 0, 0, &l);
    if (!e) S->visLanes.push_back(l);
  }
  if (e) {
    if (S->softLane) btserve::laneDestroy(S->softLane);
    for (bt_gpu_ctx* l : S->visLanes) btserve::laneDestroy(l);
    delete S;
    return e;
  }
  btserve::servingState(c) = S;
  S->threads.emplace_back(softLoop, S);
  for (bt_gpu_ctx* l : S->visLanes) S->threads.emplace_back(visLoop, S, l);
  return BT_OK;
}

int bt_gpu_submit(bt_gpu_ctx* c, const bt_request* r, uint64_t* ticket) {
  if (!c || !r) {
    btSetError("bt_gpu_submit: no context or request");
    return BT_ERR_INVALID;
  }
  if (!servingOf(c)) {
    const int e = bt_gpu_serve_start(c, nullptr);
    if (e) return e;
  }
  Serving& S = *servingOf(c);
  if (r->kind < BT_REQ_SOFT || r->kind > BT_REQ_POINT_MASK || r->cam.W <= 0 || r->cam.H <= 0 ||
      r->cam.W > 65536 || r->cam.H > 65536 || r->scene < 0 || r->scene >= btserve::sceneCount(c)) {
    btSetError("bt_gpu_submit: bad request kind, camera or scene");
    return BT_ERR_INVALID;
  }
  const int64_t px = int64_t(r->cam.W) * r->cam.H;
  if (r->kind == BT_REQ_SOFT && (px > S.cfg.soft_pixels || softRootsOf(r->cam) > S.cfg.soft_pixels)) {
    char msg[160];
    snprintf(msg, sizeof msg, "bt_gpu_submit: %lld soft-shadow pixels exceed the %lld one soft run holds",
             (long long)px, (long long)S.cfg.soft_pixels);
    btSetError(msg);
    return BT_ERR_TOO_LARGE;
  }
  Pending p;
  p.r = *r;
  p.bytes = chargeOf(*r);
  p.submitted = p.started = Clock::now();
  // the lanes' queue high-water marks, read outside the lock (they only grow)
  int64_t high = btserve::laneHighWater(S.softLane);
  for (bt_gpu_ctx* l : S.visLanes) high += btserve::laneHighWater(l);
  std::lock_guard<std::mutex> lk(S.m);
  S.st.queue_high_water = high;
  if (S.cfg.memory_budget > 0) {
    const int64_t need = btserve::sceneBytes(c) + high + S.st.admitted_bytes + p.bytes;
    if (need > S.cfg.memory_budget && S.st.admitted_bytes > 0) {  // (alone, any request is admitted)
      S.st.refused++;
      char msg[200];
      snprintf(msg, sizeof msg, "bt_gpu_submit: %lld bytes of scenes, queues and requests would exceed the budget of %lld",
               (long long)need, (long long)S.cfg.memory_budget);
      btSetError(msg);
      return BT_ERR_BUSY;
    }
  }
  p.ticket = S.nextTicket++;
  if (ticket) *ticket = p.ticket;
  S.st.admitted_bytes += p.bytes;
  S.st.submitted++;
  S.st.queued++;
  (r->kind == BT_REQ_SOFT ? S.soft : S.vis).push_back(p);
  S.work.notify_all();
  return BT_OK;
}

int bt_gpu_poll(bt_gpu_ctx* c, bt_completion* out, int32_t cap, int32_t* count, int32_t wait_ms) {
  if (count) *count = 0;
  if (!c || (cap > 0 && !out)) {
    btSetError("bt_gpu_poll: bad arguments");
    return BT_ERR_INVALID;
  }
  Serving* S = servingOf(c);
  if (!S) return BT_OK;
  std::unique_lock<std::mutex> lk(S->m);
  auto some = [&] { return !S->done.empty(); };
  if (wait_ms > 0)
    S->ready.wait_for(lk, std::chrono::milliseconds(wait_ms), some);
  else if (wait_ms < 0)
    S->ready.wait(lk, [&] { return some() || S->st.queued + S->st.running == 0; });
  int n = 0;
  while (n < cap && !S->done.empty()) {
    out[n++] = S->done.front();
    S->done.pop_front();
  }
  if (count) *count = n;
  return BT_OK;
}

int bt_gpu_serve_stats(bt_gpu_ctx* c, bt_serve_stats* st) {
  if (!c || !st) return BT_ERR_INVALID;
  Serving* S = servingOf(c);
  memset(st, 0, sizeof *st);
  st->scene_bytes = btserve::sceneBytes(c);
  if (!S) return BT_OK;
  int64_t lanes = btserve::laneBytes(S->softLane), high = btserve::laneHighWater(S->softLane);
  for (bt_gpu_ctx* l : S->visLanes) {
    lanes += btserve::laneBytes(l);
    high += btserve::laneHighWater(l);
  }
  std::lock_guard<std::mutex> lk(S->m);
  *st = S->st;
  st->scene_bytes = btserve::sceneBytes(c);
  st->lane_bytes = lanes;
  st->queue_high_water = high;
  return BT_OK;
}

}  // extern "C"
