// The B200 beam engine: rounds of persistent-grid kernels over sub-beam
// records, and the C-ABI entry points (include/bt_gpu.h).
//
// Sub-beams are 64-byte self-contained records.  A round is three kernels:
//   admit  roots whose queue reservation fits become pre-split records in the
//          round's trace queue;
//   trace  a persistent grid drains the trace queue: a lane takes a record,
//          traces it leaf by leaf until it finishes or a triangle needs a
//          clip, and takes the next record as soon as it is free (one atomic
//          per warp for all idle lanes, ballot/popc compaction).  Records
//          that need a clip go to the bottom of the clip queue, finished
//          pieces to its top;
//   clip   one lane per clip record (pieces go to the next round's trace
//          queue, siblings in consecutive slots) and per finished piece
//          (the output step: soft-shadow accumulators, polygon lists);
// plus a one-thread bookkeeping kernel.  Every warp works on every root, so
// no lane starves while work exists anywhere on the GPU.
//
// Memory is bounded without waiting: a root is admitted only if `budget`
// queue slots are free for it, and a root that would exceed its budget is
// abandoned and traced again, on the GPU, in a retry pass with a 16x budget
// (the reference recomputed such roots on the CPU, cuda/gpu_render.cu:651-672).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <shared_mutex>
#include <string>
#include <vector>

#include "bt_gpu.h"
#include "engine_core.cuh"
#include "serve_engine.h"

using namespace btg;

namespace {

thread_local char g_err[512] = "";

void setErr(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof g_err, fmt, ap);
  va_end(ap);
}

#define CK(x)                                                                         \
  do {                                                                                \
    cudaError_t e_ = (x);                                                             \
    if (e_ != cudaSuccess) {                                                          \
      setErr("%s: %s (%s:%d)", #x, cudaGetErrorString(e_), __FILE__, __LINE__);     \
      return BT_ERR_CUDA;                                                             \
    }                                                                                 \
  } while (0)

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 4;
constexpr int kThreads = 32 * kWarps;
constexpr double kFixVis = 1099511627776.0;         // 2^40: visible fraction, fixed point
constexpr double kFixG = 1152921504606846976.0;     // 2^60: Lambert integral, fixed point
// Launches per call before BT_ERR_TIMEOUT: a guard against a run that stops
// making progress, far above what long batches need (a 64-job batch of
// 100-200K-triangle scenes with large lights takes thousands of rounds).
constexpr int kMaxLaunches = 1000000;
// Queue slots a root reserves when it is admitted (its budget if smaller);
// it takes more from the pool as it grows.  Roots admitted at once are
// bounded by capacity / this: 128 admits a whole 512^2 soft frame into
// 2^25-record queues, and primary tiles (budget 4096) as many.
constexpr int kInitialReserve = 128;

enum App { kAppSoft = 0, kAppPrimary = 1, kAppPoint = 2 };
enum RootState { kRootNone = 0, kRootTraced = 1, kRootKilled = 2 };
enum Phase { kIdle = 0, kLoaded = 1, kTrace = 2, kSplit = 3 };

// Engine state shared by all warps of a pass.
struct __align__(128) Counters {
  unsigned long long reserved;  // queue slots reserved by roots in flight
  int rootNext;                 // next entry of the root list to admit
  int inflight;                 // admitted roots not finished
  int killed;                   // roots abandoned in this pass
  int error;                    // a queue append found no slot (impossible by the reservation rule)
  int outCount;                 // output polygons
  int maxQueue;                 // largest trace queue
  int done;                     // set by roundEnd: every root of the pass is done
  int rounds;
  int warpsOut;                 // trace warps that have exited in this round
  int yields;                   // records handed on unfinished (all rounds of the pass)
  int pad0[4];
  int count[2];                 // records in trace queue 0 / 1
  int head;                     // fetch cursor of the trace queue being drained
  int pad1[13];
  int clipCount;                // records waiting for a clip (from the bottom of the clip queue)
  int clipHead;                 // fetch cursor of the clip queue (clips, then deferred outputs)
  int outQ;                     // finished pieces waiting for output (from the top of the clip queue)
  int pad2[13];
};

// Per-root query: plane, tolerances, mode (WfRoot, cuda/wavefront.cu:80-86).
struct __align__(16) RootRec {
  float4 a, b, c, d, e, f;  // O.xyz ext | p0.xyz exclude | u.xyz lightArea | v.xyz flags | n.xyz attempt | d.xyz -
};

struct OutPolyDev {
  float* x;
  float* y;
  int32_t* n;
  int32_t* tri;
  float* area;
  int32_t* root;
  int32_t* attempt;
  int cap;
};

struct AppParams {
  // image / camera
  int W, H, tilesX, tile, tilesW, cull, tiled;
  Plane camPlane;
  V3 eye, fwd, right, down;
  float halfW, halfH;
  // soft shadows
  V3 Lc, LU, LV;
  float offset;
  int exact;
  const int32_t* pixTri;
  const float* pixX;
  const float* pixN;
  // fused primary rays: admission traces each pixel's eye ray itself and
  // writes tri, X, N here (instead of reading them from a primary-ray pass)
  int fusedPrimary;
  int32_t* pixTriOut;
  float* pixXOut;
  float* pixNOut;
  float *vis, *E, *Eu;
  unsigned long long* missFx;
  unsigned long long* gFx;
  float4* shade;  // x, ns per root
  // batched soft shadows: per-job parameters (camera, light, pixel and
  // output arrays of each job) in device memory; job j owns the roots
  // [jobStart[j], jobStart[j + 1]).  The accumulators above are indexed by
  // the batch-wide root.
  const AppParams* jobs;
  const int32_t* jobStart;
  int numJobs;
  // a job's scene in the context's scene pool: kd root, its box, first triangle id
  Box rootBox;
  uint32_t rootNode;
  int triBase;
  // point shadows
  V3 pointLight;
  const float* hx;
  const float* hy;
  const int32_t* hn;
  const int32_t* htri;
  OutPolyDev out;
};

struct RoundParams {
  SceneDev s;
  SubBeam* tq[2];  // trace queues: round r drains tq[r & 1], its clips fill tq[(r + 1) & 1]
  SubBeam* cq;     // clip queue of the round
  int cur;
  int capacity;
  int budget;   // live sub-beams a root may hold before it is abandoned (and retried with 16x)
  int reserve;  // queue slots a root reserves when admitted: min(budget, kInitialReserve), at least 32 (its
                // pre-split pieces always fit); it grows from the pool, up to the budget, as the root needs

  int numRoots;
  int rootCap;  // size of the per-root arrays
  int yieldAt;  // exited trace warps at which the rest hand their records on (INT_MAX: never)
  const int32_t* rootList;
  RootRec* roots;  // per-root query records
  int32_t* live;
  int32_t* resv;  // per root: queue slots it holds reserved
  int32_t* state;
  int32_t* attempt;
  Counters* ctr;
  unsigned long long* stats;
  AppParams app;
};

__device__ __forceinline__ int laneId() { return threadIdx.x & 31; }

__device__ __forceinline__ float asF(int i) { return __int_as_float(i); }
__device__ __forceinline__ int asI(float f) { return __float_as_int(f); }

__device__ void storeRoot(RootRec* R, const Query& q, float lightArea, int attempt) {
  RootRec r;
  r.a = make_float4(q.P.O.x, q.P.O.y, q.P.O.z, q.ext);
  r.b = make_float4(q.P.p0.x, q.P.p0.y, q.P.p0.z, asF(q.exclude));
  r.c = make_float4(q.P.u.x, q.P.u.y, q.P.u.z, lightArea);
  r.d = make_float4(q.P.v.x, q.P.v.y, q.P.v.z, asF(q.mode | (q.farIsPlane << 1) | (q.cull << 2)));
  r.e = make_float4(q.P.n.x, q.P.n.y, q.P.n.z, asF(attempt));
  r.f = make_float4(q.P.d.x, q.P.d.y, q.P.d.z, 0.f);
  *R = r;
}

// Per-root records are written during the launch by the admitting SM; they
// are read from L2 (an L1 line could hold a neighbouring root's older copy).
// Soft- and point-shadow queries are always AnyHit with the far plane and
// no culling (lightBeamSetup, pointShadowSetup); stating that at compile
// time drops the Nearest-mode hit-plane state and code from those kernels.
template <int App>
__device__ __forceinline__ void loadRoot(const RootRec* R, Query& q, float& lightArea) {
  const float4 a = __ldcg(&R->a), b = __ldcg(&R->b), c = __ldcg(&R->c), d = __ldcg(&R->d), e = __ldcg(&R->e),
               f = __ldcg(&R->f);
  q.P.O = mk(a.x, a.y, a.z);
  q.P.p0 = mk(b.x, b.y, b.z);
  q.P.u = mk(c.x, c.y, c.z);
  q.P.v = mk(d.x, d.y, d.z);
  q.P.n = mk(e.x, e.y, e.z);
  q.P.d = mk(f.x, f.y, f.z);
  q.exclude = asI(b.w);
  const int fl = asI(d.w);
  q.mode = App == kAppPrimary ? (fl & 1) : int(kModeAnyHit);
  q.farIsPlane = App == kAppPrimary ? (fl >> 1) & 1 : 1;
  q.cull = App == kAppPrimary ? (fl >> 2) & 1 : 0;
  lightArea = c.w;
  querySetup(q, a.w);
}

// A root is finished: its reservation goes back to the pool.
__device__ __forceinline__ void rootDone(const RoundParams& p, int root) {
  atomicAdd(&p.ctr->reserved, (unsigned long long)(-(long long)__ldcg(&p.resv[root])));
  atomicSub(&p.ctr->inflight, 1);
}

__device__ __forceinline__ void liveSub(const RoundParams& p, int root, int n) {
  if (n > 0 && atomicSub(&p.live[root], n) == n) rootDone(p, root);
}

// A root now holds `need` live sub-beams: its reservation covers them, or
// grows from the pool (at least doubling, never past the budget) while the
// queues' capacity allows.  False: the pool cannot cover it (the caller
// abandons the root).  Lanes that grow one root at once may both add;
// rootDone gives back whatever the root holds.
__device__ __forceinline__ bool coverLive(const RoundParams& p, int root, int need) {
  const int have = __ldcg(&p.resv[root]);
  if (need <= have) return true;
  const int grow = min(max(need - have, have), p.budget - have);  // need <= budget: at least need - have
  const unsigned long long old = atomicAdd(&p.ctr->reserved, (unsigned long long)grow);
  if (old + (unsigned long long)grow > (unsigned long long)p.capacity) {
    atomicAdd(&p.ctr->reserved, (unsigned long long)(-(long long)grow));
    return false;
  }
  atomicAdd(&p.resv[root], grow);
  return true;
}

__device__ __forceinline__ void killRoot(const RoundParams& p, int root) {
  if (atomicExch(&p.state[root], int(kRootKilled)) != int(kRootKilled)) atomicAdd(&p.ctr->killed, 1);
}

__device__ void appendPoly(const RoundParams& p, int root, const float* x, const float* y, int n, int tri,
                           float area) {
  const int k = atomicAdd(&p.ctr->outCount, 1);
  if (k >= p.app.out.cap) return;  // counted: the host retries with a larger buffer
  const OutPolyDev& o = p.app.out;
  for (int i = 0; i < 4; ++i) {
    const int j = i < n ? i : n - 1;
    o.x[4 * k + i] = x[j];
    o.y[4 * k + i] = y[j];
  }
  o.n[k] = n;
  o.tri[k] = tri;
  o.area[k] = area;
  o.root[k] = root;
  o.attempt[k] = __ldcg(&p.attempt[root]);
}

// A finished piece handed to the output path in a small temporary: the
// tracing lane's query and beam never leave registers.
struct PieceOut {
  Plane P;
  float qx[4], qy[4];
  int n, root, tri, exclude;
  float lightArea;
};

// Finished pieces.  Soft: unoccluded area (fixed point) and, with exact, the
// FP64 Lambert integral; primary: visible polygons; point shadows: occluded
// pieces projected back into the image (WfOut, cuda/wavefront.cu:193-227).
template <int App>
__device__ __noinline__ void outputPieceCold(const RoundParams& p, const PieceOut* o) {
  Poly<4> poly;
  poly.n = o->n;
  for (int i = 0; i < 4; ++i) {
    poly.x[i] = o->qx[i];
    poly.y[i] = o->qy[i];
  }
  const float area = poly.area();
  const int root = o->root;
  if (App == kAppSoft) {
    const double f = double(area) / double(o->lightArea) * kFixVis;
    if (f > 0) atomicAdd(&p.app.missFx[root], (unsigned long long)llrint(f));
    if (p.app.exact) {
      V3 P[4];
      for (int i = 0; i < poly.n; ++i) P[i] = planePoint(o->P, poly.x[i], poly.y[i]);
      const float4 xs = __ldcg(&p.app.shade[2 * root]), ns = __ldcg(&p.app.shade[2 * root + 1]);
      const double G = formFactorFP64(mk(xs.x, xs.y, xs.z), mk(ns.x, ns.y, ns.z), P, poly.n);
      const double g = G * kFixG;
      if (g > 0) atomicAdd(&p.app.gFx[root], (unsigned long long)llrint(g));
    }
  } else if (App == kAppPrimary) {
    appendPoly(p, root, poly.x, poly.y, poly.n, o->tri, area);
  } else {
    float ox[4], oy[4];
    if (pointShadowToImage(p.app.camPlane, o->P, poly.x, poly.y, poly.n, ox, oy))
      appendPoly(p, root, ox, oy, poly.n, o->exclude, 0.f);
  }
}

template <int App>
__device__ __forceinline__ void outputPiece(const RoundParams& p, const Query& q, float lightArea, int root,
                                            const Beam& b, int tri, Stats& st) {
  if (tri >= 0) st.hits++;
  st.beams++;
  if (App == kAppSoft ? tri >= 0 : tri < 0) return;  // soft keeps the visible light, the others the hits
  PieceOut o;
  o.P = q.P;
  for (int i = 0; i < 4; ++i) {
    o.qx[i] = b.qx[i];
    o.qy[i] = b.qy[i];
  }
  o.n = b.n;
  o.root = root;
  o.tri = tri;
  o.exclude = q.exclude;
  o.lightArea = lightArea;
  outputPieceCold<App>(p, &o);
}

// Appends n records to trace queue `q` (one atomic); returns the first slot
// or -1 (and flags an error) if they do not fit, which the reservation rule
// rules out.
__device__ __forceinline__ int queueAppend(const RoundParams& p, int q, int n) {
  const int at = atomicAdd(&p.ctr->count[q], n);
  if (at + n > p.capacity) {
    atomicExch(&p.ctr->error, 1);
    return -1;
  }
  return at;
}

// ------------------------------------------------------------ primary rays

// Moller-Trumbore (rayHitTri, src/ray/ray_core.h:22-37).
__device__ __forceinline__ float rayHit(V3 o, V3 d, V3 v0, V3 v1, V3 v2) {
  V3 e1 = sub(v1, v0), e2 = sub(v2, v0);
  V3 pv = cross(d, e2);
  float det = dot(e1, pv);
  if (det == 0) return kInf;
  float inv = 1 / det;
  V3 tv = sub(o, v0);
  float u = dot(tv, pv) * inv;
  if (u < 0 || u > 1) return kInf;
  V3 qv = cross(tv, e1);
  float v = dot(d, qv) * inv;
  if (v < 0 || u + v > 1) return kInf;
  return dot(e2, qv) * inv;
}

// The eye ray through the centre of pixel (x, y), nearest hit with coplanar
// ties to the lower id (rayTraverse<false>, src/ray/ray_core.h:42-132):
// returns the triangle (-1: none) and sets X, N (normal facing the eye; 0
// when nothing is hit).
__device__ __noinline__ int eyeRay(const SceneDev& s, V3 o, V3 fwd, V3 right, V3 down, float halfW, float halfH,
                                   int W, int H, int x, int y, V3* Xo, V3* No) {
  const float qx = (2 * (float(x) + 0.5f) / float(W) - 1) * halfW;
  const float qy = (2 * (float(y) + 0.5f) / float(H) - 1) * halfH;
  const V3 d = add(add(fwd, mul(right, qx)), mul(down, qy));
  *Xo = mk(0, 0, 0);
  *No = mk(0, 0, 0);
  float t0 = 0, t1 = kInf;
  float inv[3];
  for (int a = 0; a < 3; ++a) {
    const float da = comp(d, a), oa = comp(o, a);
    inv[a] = 1 / da;
    if (da == 0) {
      if (oa < s.bounds.lo[a] || oa > s.bounds.hi[a]) return -1;
      continue;
    }
    float ta = (s.bounds.lo[a] - oa) * inv[a];
    float tb = (s.bounds.hi[a] - oa) * inv[a];
    if (ta > tb) {
      float tt = ta;
      ta = tb;
      tb = tt;
    }
    t0 = t0 > ta ? t0 : ta;
    t1 = t1 < tb ? t1 : tb;
  }
  if (t0 > t1) return -1;
  struct Entry {
    uint32_t node;
    float t0, t1;
  };
  Entry stk[64];
  int sp = 0;
  uint32_t node = s.rootNode;
  float best = kInf;
  int bestTri = -1;
  const float tieEps = 4 * 1.1920928955078125e-07f;
  for (;;) {
    const uint2 nd = s.node[node];
    if (!isLeaf(nd)) {
      const int a = int(nd.y & 3u);
      const float sp_ = splitOf(nd);
      const float oa = comp(o, a), da = comp(d, a);
      const bool belowFirst = oa < sp_ || (oa == sp_ && da <= 0);
      const uint32_t first = belowFirst ? node + 1 : (nd.y >> 2);
      const uint32_t second = belowFirst ? (nd.y >> 2) : node + 1;
      if (da == 0) {
        node = first;
        continue;
      }
      const float tp = (sp_ - oa) * inv[a];
      if (tp > t1 || tp <= 0) {
        node = first;
      } else if (tp < t0) {
        node = second;
      } else {
        if (sp < 64) stk[sp++] = Entry{second, tp, t1};
        node = first;
        t1 = tp;
      }
      continue;
    }
    const uint32_t cnt = nd.y >> 2;
    for (uint32_t i = 0; i < cnt; ++i) {
      const TriRec t = loadRef(s, nd.x + i);
      const float th = rayHit(o, d, t.v0, t.v1, t.v2);
      if (!(th > 0 && th < kInf)) continue;
      const float tol = bestTri < 0 ? 0.f : best * tieEps;
      if (bestTri < 0 || th < best - tol || (th <= best + tol && t.tri < bestTri)) {
        best = th;
        bestTri = t.tri;
      }
    }
    if (bestTri >= 0 && best <= t1) break;
    if (sp == 0) break;
    --sp;
    node = stk[sp].node;
    t0 = stk[sp].t0;
    t1 = stk[sp].t1;
  }
  if (bestTri < 0) return -1;
  *Xo = add(o, mul(d, best));
  V3 nT, v0;
  triNV(s, bestTri, nT, v0);
  if (dot(nT, d) > 0) nT = neg(nT);
  *No = nT;
  return bestTri;
}

// Admission: every pre-split piece goes to the round's trace queue.
template <int App>
struct AdmitEnv {
  const RoundParams* p;
  const Query* q;
  float lightArea;
  int root;
  Stats* st;
  int queued;
  __device__ bool queue(const SubBeam& r) {
    ++queued;
    const int at = queueAppend(*p, p->cur, 1);
    if (at >= 0) p->tq[p->cur][at] = r;
    return at >= 0;
  }
  __device__ void occluded(const Beam& b, int tri) { outputPiece<App>(*p, *q, lightArea, root, b, tri, *st); }
  __device__ void missed(const Beam& b) { outputPiece<App>(*p, *q, lightArea, root, b, -1, *st); }
  __device__ void dropped(float) {}
};

// Clip emission into the next round's trace queue (wfSplitEmit,
// wavefront_core.h:367-422): the slots pass 1 counted are reserved with one
// atomic and each piece is written straight into its own, so siblings stay
// adjacent; slots left by slivers that beamGeom drops are filled with empty
// records (n = -1), which the trace kernel skips.
template <int App>
struct SplitEnv {
  const RoundParams* p;
  const Query* q;
  float lightArea;
  int root;
  Stats* st;
  SubBeam* dst;   // the reserved slots
  int reserved;
  int filled;
  SubBeam* keep;  // tail rounds: the first piece stays with the clipping lane
  bool kept;
  __device__ void reserve(int n) {
    reserved = 0;
    filled = 0;
    dst = nullptr;
    if (n <= 0) return;
    const int nxt = p->cur ^ 1;
    const int at = queueAppend(*p, nxt, n);
    if (at < 0) return;
    dst = p->tq[nxt] + at;
    reserved = n;
  }
  // empty records in the slots no piece took; returns their number
  __device__ int finish() {
    for (int i = filled; i < reserved; ++i) {
      SubBeam d;
      for (int k = 0; k < 4; ++k) d.qx[k] = d.qy[k] = 0.f;
      d.trail = 0;
      d.node = 0;
      d.root = root;
      d.hit = -1;
      d.cursor = 0;
      d.depth = 0;
      d.n = -1;
      d.neg = 0;
      dst[i] = d;
    }
    return reserved - filled;
  }
  __device__ bool queue(const SubBeam& r) {
    if (keep && !kept) {
      *keep = r;
      kept = true;
      return true;
    }
    if (filled < reserved) dst[filled++] = r;
    return true;
  }
  __device__ void occluded(const Beam& b, int tri) { outputPiece<App>(*p, *q, lightArea, root, b, tri, *st); }
  __device__ void missed(const Beam& b) { outputPiece<App>(*p, *q, lightArea, root, b, -1, *st); }
  __device__ void dropped(float) {}
};

// Root k of an 8x4-pixel tile per warp (cuda/wavefront.cu:245-252).
__device__ __forceinline__ bool softPixel(const AppParams& a, int k, int& pix) {
  if (!a.tiled) {
    pix = k;
    return true;
  }
  const int tile = k >> 5, l = k & 31;
  const int x = (tile % a.tilesX) * 8 + (l & 7), y = (tile / a.tilesX) * 4 + (l >> 3);
  pix = y * a.W + x;
  return x < a.W && y < a.H;
}

// What admission hands back to the lane (a temporary: the lane's own state
// stays in registers).
struct AdmitOut {
  Query q;
  float lightArea;
  Stats st;
};

// Sets up root k and queues its pre-split pieces (admitRoot,
// cuda/wavefront.cu:255-325).
template <int App>
__device__ __noinline__ bool admit(const RoundParams& p, int k, AdmitOut* out) {
  Query& q = out->q;
  float& lightArea = out->lightArea;
  Stats& st = out->st;
  p.live[k] = 0;
  p.resv[k] = p.reserve;  // what the admission claimed for it
  p.state[k] = kRootNone;
  const int att = p.attempt[k] + 1;
  p.attempt[k] = att;
  Poly<8> poly;
  poly.clear();
  lightArea = 0;
  SceneDev sj = p.s;  // the root's scene: the pool's first, or its job's
  if (App == kAppSoft) {
    p.app.missFx[k] = 0;
    p.app.gFx[k] = 0;
    // the root's job (a batch) or the call's parameters
    int kl = k;
    const AppParams* ap = &p.app;
    if (p.app.numJobs > 0) {
      int lo = 0, hi = p.app.numJobs - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.app.jobStart[mid] <= k)
          lo = mid;
        else
          hi = mid - 1;
      }
      ap = &p.app.jobs[lo];
      kl = k - p.app.jobStart[lo];
      sj.bounds = ap->rootBox;
      sj.rootNode = ap->rootNode;
    }
    const AppParams& a = *ap;
    int pix;
    if (!softPixel(a, kl, pix)) {
      rootDone(p, k);
      return false;
    }
    int T;
    V3 x, ns;
    if (a.fusedPrimary) {
      T = eyeRay(sj, a.eye, a.fwd, a.right, a.down, a.halfW, a.halfH, a.W, a.H, pix % a.W, pix / a.W, &x, &ns);
      a.pixTriOut[pix] = T;
      a.pixXOut[3 * pix] = x.x;
      a.pixXOut[3 * pix + 1] = x.y;
      a.pixXOut[3 * pix + 2] = x.z;
      a.pixNOut[3 * pix] = ns.x;
      a.pixNOut[3 * pix + 1] = ns.y;
      a.pixNOut[3 * pix + 2] = ns.z;
    } else {
      T = a.pixTri[pix];
    }
    if (T < 0) {
      if (a.vis) a.vis[pix] = -1;
      if (a.E) a.E[pix] = 0;
      if (a.Eu) a.Eu[pix] = 0;
      rootDone(p, k);
      return false;
    }
    if (!a.fusedPrimary) {
      x = mk(a.pixX[3 * pix], a.pixX[3 * pix + 1], a.pixX[3 * pix + 2]);
      ns = mk(a.pixN[3 * pix], a.pixN[3 * pix + 1], a.pixN[3 * pix + 2]);
    }
    const float A = length(cross(a.LU, a.LV));
    if (a.Eu) a.Eu[pix] = A * lightCenterG(a.Lc, a.LU, a.LV, x, ns);
    if (!lightBeamSetup(a.Lc, a.LU, a.LV, x, ns, T, a.offset, q, poly, lightArea)) {
      if (a.vis) a.vis[pix] = 0;
      if (a.E) a.E[pix] = 0;
      rootDone(p, k);
      return false;
    }
    p.app.shade[2 * k] = make_float4(x.x, x.y, x.z, 0.f);
    p.app.shade[2 * k + 1] = make_float4(ns.x, ns.y, ns.z, 0.f);
  } else if (App == kAppPrimary) {
    const int tx = k % p.app.tilesW, ty = k / p.app.tilesW;
    const int x0 = tx * p.app.tile, y0 = ty * p.app.tile;
    const int x1 = min(p.app.W, x0 + p.app.tile), y1 = min(p.app.H, y0 + p.app.tile);
    const float qx0 = (2 * float(x0) / float(p.app.W) - 1) * p.app.halfW;
    const float qx1 = (2 * float(x1) / float(p.app.W) - 1) * p.app.halfW;
    const float qy0 = (2 * float(y0) / float(p.app.H) - 1) * p.app.halfH;
    const float qy1 = (2 * float(y1) / float(p.app.H) - 1) * p.app.halfH;
    poly.push(qx0, qy0);
    poly.push(qx1, qy0);
    poly.push(qx1, qy1);
    poly.push(qx0, qy1);
    q.P = p.app.camPlane;
    q.mode = kModeNearest;
    q.farIsPlane = 0;
    q.exclude = -1;
    q.cull = p.app.cull;
  } else {
    const int T = p.app.htri[k];
    float px[4], py[4];
    const int n = p.app.hn[k];
    for (int i = 0; i < 4; ++i) {
      px[i] = p.app.hx[4 * k + i];
      py[i] = p.app.hy[4 * k + i];
    }
    if (T < 0) {
      rootDone(p, k);
      return false;
    }
    V3 nT, v0;
    triNV(p.s, T, nT, v0);
    if (!pointShadowSetup(p.app.eye, p.app.fwd, p.app.right, p.app.down, nT, v0, T, p.app.pointLight, px, py, n, q,
                          poly)) {
      appendPoly(p, k, px, py, n, T, 0.f);  // receiver faces away from the light: all in shadow
      p.state[k] = kRootTraced;
      rootDone(p, k);
      return false;
    }
  }
  querySetup(q, poly.extent());
  storeRoot(&p.roots[k], q, lightArea, att);
  p.state[k] = kRootTraced;
  AdmitEnv<App> env{&p, &q, lightArea, k, &st, 0};
  const bool ok = admitRoot(sj, q, poly, k, env, st);
  p.live[k] = env.queued;  // the pieces are traced by a later kernel
  if (!ok || env.queued > p.budget) killRoot(p, k);
  if (env.queued == 0) rootDone(p, k);
  return env.queued > 0;
}

__device__ __forceinline__ void addStats(Stats& a, const Stats& b) {
  a.kdSteps += b.kdSteps;
  a.leafVisits += b.leafVisits;
  a.triTests += b.triTests;
  a.hits += b.hits;
  a.splits += b.splits;
  a.beams += b.beams;
  a.rootBeams += b.rootBeams;
  a.presplitBeams += b.presplitBeams;
  a.fiveSplits += b.fiveSplits;
  a.climbs += b.climbs;
  a.epsBand += b.epsBand;
  a.epsFlip += b.epsFlip;
  a.dropped += b.dropped;
}

__device__ __forceinline__ void flushStats(const RoundParams& p, const Stats& st) {
  unsigned long long v[kStDropped] = {st.kdSteps, st.leafVisits, st.triTests, st.hits, st.splits,
                                      st.beams, st.rootBeams, st.presplitBeams, st.fiveSplits, st.climbs};
  for (int f = 0; f < kStDropped; ++f) {
    unsigned long long s = v[f];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(kFull, s, o);
    if (laneId() == 0 && s) atomicAdd(&p.stats[f], s);
  }
  double d = st.dropped;
  for (int o = 16; o > 0; o >>= 1) d += __shfl_down_sync(kFull, d, o);
  if (laneId() == 0 && d != 0) atomicAdd(reinterpret_cast<double*>(&p.stats[kStDropped]), d);
  if (__any_sync(kFull, st.epsBand != 0)) {  // logging kernels only
    unsigned long long b = st.epsBand, f = st.epsFlip;
    for (int o = 16; o > 0; o >>= 1) {
      b += __shfl_down_sync(kFull, b, o);
      f += __shfl_down_sync(kFull, f, o);
    }
    if (laneId() == 0) {
      atomicAdd(&p.stats[kStEpsBand], b);
      if (f) atomicAdd(&p.stats[kStEpsFlip], f);
    }
  }
}

// Each clipping thread's piece log (clipRecord), in dynamic shared memory
// rather than the thread's local frame: kThreads logs of 10 pieces, 55.8 KB
// a CTA, which still lets 4 clip CTAs share an SM (a log of 8 pieces was
// 0.5 ms a plant frame slower, one of 6 1.5 ms: the clips it cannot hold
// are clipped again).  The clip and fused trace kernels are launched with
// kLogSmem bytes.
extern __shared__ PieceLog s_pieceLog[];
constexpr size_t kLogSmem = sizeof(PieceLog) * kThreads;

// Clips one record of the clip queue (a triangle at its cursor needs it):
// the pieces go to the next round's trace queue in consecutive slots (or,
// in tail rounds, the first one back to the calling lane, `keep`).
// Returns true if nothing
// measurable changed and the record (updated in place) continues at the next
// triangle.  Works on its own query and beam: the caller's stay in registers.
// F64: band corners of the edge lines re-decided in FP64 (eps_fp64).
template <int App, bool F64 = false>
__device__ __noinline__ bool clipRecord(const RoundParams& p, SubBeam* recp, Stats* cs, SubBeam* keep = nullptr,
                                        bool* kept = nullptr) {
  Stats& st = *cs;
  SubBeam rec = *recp;
  const int root = rec.root;
  if (p.state[root] == kRootKilled) {
    liveSub(p, root, 1);
    return false;
  }
  Query q;
  float lightArea;
  Beam b;
  loadRoot<App>(&p.roots[root], q, lightArea);
  expand(p.s, q, rec, b);
  TriInfo ti;
  Line L[5];
  int nl = 0;
  bool commit = false;
  PieceLog& log = s_pieceLog[threadIdx.x];  // shared memory: not in the thread's local frame
  Line64 e64[3];
  const int slots = splitPass1<SplitEnv<App>, F64>(p.s, q, rec, b, st, ti, L, nl, commit, &log, e64);
  if (slots < 0) {
    killRoot(p, root);
    liveSub(p, root, 1);
    return false;
  }
  if (!commit) {
    recp->cursor = rec.cursor + 1;
    return true;
  }
  const int old = atomicAdd(&p.live[root], slots - 1);
  if (old + slots - 1 > p.budget || !coverLive(p, root, old + slots - 1)) {
    killRoot(p, root);
    liveSub(p, root, slots);
    return false;
  }
  if (old + slots - 1 == 0) rootDone(p, root);  // every piece occluded: the root is finished
  SplitEnv<App> env;
  env.p = &p;
  env.q = &q;
  env.lightArea = lightArea;
  env.root = root;
  env.st = &st;
  env.keep = keep;
  env.kept = false;
  // `slots` pieces at most: one may stay with the lane (tail rounds), the
  // rest take reserved queue slots
  env.reserve(keep ? slots - 1 : slots);
  splitPass2<SplitEnv<App>, F64>(q, rec, b, ti, L, nl, env, st, &log, e64);
  // slivers dropped by beamGeom were counted in `slots` but never queued
  // (nor kept); with no piece at all (slots = 0) there was no kept slot to
  // give back: the record itself was already taken off by the add above
  const int unused = env.finish() + (keep && slots > 0 && !env.kept ? 1 : 0);
  if (kept) *kept = env.kept;
  if (unused > 0) liveSub(p, root, unused);
  return false;
}

// ---- round kernels ------------------------------------------------------

// Admission: each lane sets up one root (claimed per warp under the queue
// reservation) and queues its pieces in the round's trace queue.  Roots that
// do not fit wait for a later round.
template <int App>
__global__ void __launch_bounds__(kThreads) admitKernel(const __grid_constant__ RoundParams p) {
  const int lane = laneId();
  Stats st;
  st.clear();
  for (;;) {
    // Stop when the pass is done or every root is claimed (claims may
    // overshoot).  rootNext moves while other warps claim, so lane 0 decides
    // for its warp: the shuffles below need all 32 lanes.
    int stop = 0;
    if (lane == 0) stop = (__ldcv(&p.ctr->done) || __ldcv(&p.ctr->rootNext) >= p.numRoots) ? 1 : 0;
    if (__shfl_sync(kFull, stop, 0)) break;
    int base = -1, fit = 0;
    if (lane == 0) {
      const unsigned long long res = (unsigned long long)p.reserve, cap = (unsigned long long)p.capacity;
      const unsigned long long need = 32ull * res;
      const unsigned long long old = atomicAdd(&p.ctr->reserved, need);
      fit = 32;
      if (old + need > cap) {
        fit = old >= cap ? 0 : int(min(32ull, (cap - old) / res));
        atomicAdd(&p.ctr->reserved, (unsigned long long)(-(long long)(32 - fit)) * res);
      }
      if (fit > 0) {
        base = atomicAdd(&p.ctr->rootNext, fit);
        const int got = max(0, min(fit, p.numRoots - base));
        if (got < fit) atomicAdd(&p.ctr->reserved, (unsigned long long)(-(long long)(fit - got)) * res);
        if (got > 0) atomicAdd(&p.ctr->inflight, got);
        fit = got;
      }
    }
    base = __shfl_sync(kFull, base, 0);
    fit = __shfl_sync(kFull, fit, 0);
    if (fit <= 0) break;  // queues full or every root claimed
    if (lane < fit) {
      const int j = base + lane;
      const int k = p.rootList ? p.rootList[j] : j;
      AdmitOut ao;
      ao.st.clear();
      admit<App>(p, k, &ao);
      addStats(st, ao.st);
    }
  }
  flushStats(p, st);
}

// Trace: persistent warps drain the round's queue.  Each lane traces its
// record leaf by leaf until it finishes or a triangle needs a clip; idle
// lanes are refilled at once (one atomic per warp, ballot/popc ranks).
// Records needing a clip are compacted into the clip queue.
// (At least `Ctas` CTAs per SM.  3 lets the compiler keep the lane's state
// in up to 170 registers; 4 caps it at 128 with a few spills and 16 warps
// per SM, which pays on a scene that sits in L1/L2 and costs on a larger
// one (trace_ctas).  The tail-round variant clips inline with its polygons
// in registers and takes 2 CTAs per SM: tail rounds hold too few records to
// need more warps.)
template <int App, bool Fused, int Mode = kVoteFloat, int Ctas = 3>
__global__ void __launch_bounds__(kThreads, Fused ? 2 : Ctas) traceKernel(const __grid_constant__ RoundParams p) {
  const int lane = laneId();
  const unsigned ltMask = (1u << lane) - 1u;
  const int nCur = min(p.ctr->count[p.cur], p.capacity);
  const SubBeam* queue = p.tq[p.cur];
  bool exhausted = nCur == 0;
  int phase = kIdle;
  SubBeam r;
  Beam b;
  Query q;
  Walk w;
  float lightArea = 0;
  int qRoot = -1;
  bool outPending = false;
  int outTri = -1;
  Stats st;
  st.clear();
  for (;;) {
    // Once the queue is drained and enough warps have exited, the records
    // still in flight go to the next round's queue as they stand (at the top
    // of this loop a lane's position -- node, trail, depth, cursor, hit -- is
    // all in its record), so that the round does not wait on a few long
    // walks with most of the GPU idle.  Tail rounds run to completion.
    int warpsOut = 0;
    if (!Fused && exhausted && lane == 0) warpsOut = *(volatile int*)&p.ctr->warpsOut;
    if (!Fused && exhausted && __shfl_sync(kFull, warpsOut, 0) >= p.yieldAt) {
      const unsigned y = __ballot_sync(kFull, phase == kTrace);
      if (y) {
        int base = 0;
        if (lane == 0) {
          base = atomicAdd(&p.ctr->count[p.cur ^ 1], __popc(y));
          atomicAdd(&p.ctr->yields, __popc(y));
        }
        base = __shfl_sync(kFull, base, 0);
        if (phase == kTrace) {
          const int at = base + __popc(y & ltMask);
          if (at < p.capacity)
            p.tq[p.cur ^ 1][at] = r;
          else
            atomicExch(&p.ctr->error, 1);
          phase = kIdle;
        }
      }
      break;
    }
    const unsigned idle = __ballot_sync(kFull, phase == kIdle);
    if (idle && !exhausted) {
      const int ni = __popc(idle);
      int base = 0;
      if (lane == 0) base = atomicAdd(&p.ctr->head, ni);
      base = __shfl_sync(kFull, base, 0);
      if (base + ni >= nCur) exhausted = true;
      const int i = base + __popc(idle & ltMask);
      if (phase == kIdle && i < nCur) {
        r = queue[i];
        if (uint32_t(r.root) >= uint32_t(p.rootCap) || r.node >= p.s.numNodes || r.n > 4) {
          atomicExch(&p.ctr->error, 2);  // a malformed record: report, never index with it
        } else if (r.n < 0) {
          // an empty slot of a clip's reservation
        } else if (r.n == 0 || p.state[r.root] == kRootKilled) {
          liveSub(p, r.root, 1);  // a dropped sliver or an abandoned root
        } else {
          if (r.root != qRoot) {
            loadRoot<App>(&p.roots[r.root], q, lightArea);
            qRoot = r.root;
          }
          expand(p.s, q, r, b);
          walkBegin(p.s, r, w);
          phase = kTrace;
        }
      }
    }
    if (!__any_sync(kFull, phase == kTrace)) {
      if (exhausted) break;
      continue;
    }
    // Per step a lane moves its record to the next leaf cell that holds a
    // triangle to test (descents, trail pops), then tests that leaf's
    // triangles in order until one needs a clip, the beam is finished, or
    // the leaf is exhausted.
    int res = kStepContinue;
    if (phase == kTrace) {
      res = advance(p.s, q, b, r, w, st);
      int occ = -1;
      if (res == kStepContinue) {
        for (;;) {
          res = testOne<Mode>(p.s, q, r, b, st, occ);
          if (res != kStepContinue || !moreInLeaf(p.s, q, r)) break;
        }
      }
      if (res == kStepFinished) {
        outTri = occ >= 0 ? occ : (q.mode == kModeNearest ? b.hit : -1);
        if (Fused) {
          outputPiece<App>(p, q, lightArea, r.root, b, outTri, st);
        } else {
          if (outTri >= 0) st.hits++;
          st.beams++;
          outPending = App == kAppSoft ? outTri < 0 : outTri >= 0;  // soft keeps the visible light, the others the hits
        }
        liveSub(p, r.root, 1);
        phase = kIdle;
      }
      if (Fused && res == kStepSplit) {
        // Tail rounds: clip here and go on with one of the pieces, so that a
        // chain of splits advances several levels per round.
        SubBeam kept;
        bool hasKept = false;
        Stats cs;
        cs.clear();
        if (clipRecord<App, Mode == kVoteFp64>(p, &r, &cs, &kept, &hasKept)) {
          w.phase = kPhTest;  // nothing changed measurably: the next triangle
        } else if (hasKept) {
          r = kept;
          expand(p.s, q, r, b);
          walkBegin(p.s, r, w);
        } else {
          phase = kIdle;
        }
        addStats(st, cs);
        res = kStepContinue;
      }
    }
    // Finished pieces are output by the clip kernel, all lanes at once
    // (the output step is long and only a few lanes finish per step).
    const unsigned outm = __ballot_sync(kFull, outPending);
    if (outm) {
      int base = 0;
      if (lane == 0) base = atomicAdd(&p.ctr->outQ, __popc(outm));
      base = __shfl_sync(kFull, base, 0);
      if (outPending) {
        SubBeam o;
        for (int k = 0; k < 4; ++k) {
          o.qx[k] = b.qx[k];
          o.qy[k] = b.qy[k];
        }
        o.trail = 0;
        o.node = 0;
        o.root = r.root;
        o.hit = outTri;
        o.cursor = 0;
        o.depth = 0;
        o.n = int8_t(b.n);
        o.neg = 0;
        const int k = base + __popc(outm & ltMask);
        if (k < p.capacity) p.cq[p.capacity - 1 - k] = o;
        outPending = false;
      }
    }
    const unsigned clip = __ballot_sync(kFull, phase == kTrace && res == kStepSplit);
    if (clip) {
      int base = 0;
      if (lane == 0) base = atomicAdd(&p.ctr->clipCount, __popc(clip));
      base = __shfl_sync(kFull, base, 0);
      if (phase == kTrace && res == kStepSplit) {
        p.cq[base + __popc(clip & ltMask)] = r;  // (r's corners are the beam's)
        phase = kIdle;
      }
    }
  }
  if (!Fused && lane == 0) atomicAdd(&p.ctr->warpsOut, 1);
  flushStats(p, st);
}

// Clip: one lane per record of the clip queue; pieces go to the next
// round's trace queue.  A record whose clip changes nothing measurable
// continues at its next triangle in the next round.
template <int App, bool F64 = false>
// (At least 4 CTAs per SM, i.e. at most 128 registers: with its polygons
// in registers the clip step would take 255 and run 2 CTAs per SM; 4 keeps
// enough warps for its latency and spills little -- measured 3 and 6 too.)
__global__ void __launch_bounds__(kThreads, 4) clipKernel(const __grid_constant__ RoundParams p) {
  const int lane = laneId();
  // clip records fill the clip queue from the bottom, deferred outputs from
  // the top; together they are at most the round's trace records
  const int nClip = p.ctr->clipCount, nOut = p.ctr->outQ;
  if (int64_t(nClip) + nOut > p.capacity) {
    if (threadIdx.x == 0 && blockIdx.x == 0) atomicExch(&p.ctr->error, 1);
    return;
  }
  const int n = nClip + nOut;
  Stats st;
  st.clear();
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(&p.ctr->clipHead, 32);
    base = __shfl_sync(kFull, base, 0);
    if (base >= n) break;
    const int i = base + lane;
    if (i < nClip) {
      SubBeam rec = p.cq[i];
      Stats cs;
      cs.clear();
      if (clipRecord<App, F64>(p, &rec, &cs)) {
        const int at = queueAppend(p, p.cur ^ 1, 1);
        if (at >= 0) p.tq[p.cur ^ 1][at] = rec;
      }
      addStats(st, cs);
    } else if (i < n) {
      const SubBeam o = p.cq[p.capacity - 1 - (i - nClip)];
      if (uint32_t(o.root) >= uint32_t(p.rootCap) || o.n < 3 || o.n > 4) {
        atomicExch(&p.ctr->error, 2);
      } else {
        PieceOut po;
        float lightArea;
        Query q;
        loadRoot<App>(&p.roots[o.root], q, lightArea);
        po.P = q.P;
        for (int k = 0; k < 4; ++k) {
          po.qx[k] = o.qx[k];
          po.qy[k] = o.qy[k];
        }
        po.n = o.n;
        po.root = o.root;
        po.tri = o.hit;
        po.exclude = q.exclude;
        po.lightArea = lightArea;
        outputPieceCold<App>(p, &po);
      }
    }
  }
  flushStats(p, st);
}

// Between rounds: the drained queues are emptied, completion is decided
// (scheduleKernel's bookkeeping, cuda/wavefront.cu:327-345).
__global__ void roundEndKernel(Counters* c, int cur, int numRoots) {
  const int nxt = cur ^ 1;
  if (c->count[nxt] > c->maxQueue) c->maxQueue = c->count[nxt];
  c->count[cur] = 0;
  c->head = 0;
  c->clipCount = 0;
  c->clipHead = 0;
  c->outQ = 0;
  c->warpsOut = 0;
  c->rounds++;
  c->done = (c->rootNext >= numRoots && c->inflight == 0 && c->count[nxt] == 0) ? 1 : 0;
}

// Hit polygons of the final attempts (tri >= 0), compacted as point-shadow
// roots (any order: the outputs built from them do not depend on it).
__global__ void compactHitsKernel(const float* ox, const float* oy, const int32_t* on, const int32_t* otri,
                                  const int32_t* oroot, const int32_t* oatt, int64_t n, const int32_t* rootState,
                                  const int32_t* rootAttempt, float* hx, float* hy, int32_t* hn, int32_t* htri,
                                  int* count) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int r = oroot[i];
  if (otri[i] < 0 || rootState[r] != kRootTraced || oatt[i] != rootAttempt[r]) return;
  const int k = atomicAdd(count, 1);
  for (int j = 0; j < 4; ++j) {
    hx[4 * k + j] = ox[4 * i + j];
    hy[4 * k + j] = oy[4 * i + j];
  }
  hn[k] = on[i];
  htri[k] = otri[i];
}

// Polygons of the roots' final attempts, compacted on the device in output
// order for the host-polygon calls: the number each block of kKeepBlock
// records keeps, an exclusive scan of those counts (the total after them),
// then every kept polygon written at its rank.
constexpr int kKeepBlock = 1024;

__device__ __forceinline__ bool finalPoly(const int32_t* oroot, const int32_t* oatt, const int32_t* state,
                                          const int32_t* attempt, int64_t i) {
  const int r = oroot[i];
  return state[r] == kRootTraced && oatt[i] == attempt[r];
}

__global__ void __launch_bounds__(kKeepBlock) keepCountKernel(const int32_t* oroot, const int32_t* oatt, int64_t n,
                                                              const int32_t* state, const int32_t* attempt,
                                                              int* blockCount) {
  __shared__ int warpCount[kKeepBlock / 32];
  const int64_t i = int64_t(blockIdx.x) * kKeepBlock + threadIdx.x;
  const unsigned m = __ballot_sync(kFull, i < n && finalPoly(oroot, oatt, state, attempt, i));
  if ((threadIdx.x & 31) == 0) warpCount[threadIdx.x >> 5] = __popc(m);
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = warpCount[threadIdx.x];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFull, v, o);
    if (threadIdx.x == 0) blockCount[blockIdx.x] = v;
  }
}

// One block: blockCount[0..nb) becomes its exclusive prefix sums and
// blockCount[nb] the total.
__global__ void __launch_bounds__(kKeepBlock) keepScanKernel(int* blockCount, int nb) {
  __shared__ int warpSum[kKeepBlock / 32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += kKeepBlock) {
    const int j = base + threadIdx.x;
    const int v = j < nb ? blockCount[j] : 0;
    int x = v;  // inclusive scan within the warp
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warpSum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      int w = warpSum[lane];
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, w, o);
        if (lane >= o) w += y;
      }
      warpSum[lane] = w;
    }
    __syncthreads();
    const int before = carry + (warp ? warpSum[warp - 1] : 0) + x - v;
    if (j < nb) blockCount[j] = before;
    __syncthreads();
    if (threadIdx.x == kKeepBlock - 1) carry = before + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) blockCount[nb] = carry;
}

struct KeepOut {
  float4 *x, *y;
  float* area;
  int32_t *n, *tri, *root;
};

__global__ void __launch_bounds__(kKeepBlock) keepWriteKernel(const float4* ox, const float4* oy, const float* oarea,
                                                              const int32_t* on, const int32_t* otri,
                                                              const int32_t* oroot, const int32_t* oatt, int64_t n,
                                                              const int32_t* state, const int32_t* attempt,
                                                              const int* blockOff, KeepOut k) {
  __shared__ int warpOff[kKeepBlock / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t i = int64_t(blockIdx.x) * kKeepBlock + threadIdx.x;
  const bool keep = i < n && finalPoly(oroot, oatt, state, attempt, i);
  const unsigned m = __ballot_sync(kFull, keep);
  if (lane == 0) warpOff[warp] = __popc(m);
  __syncthreads();
  if (warp == 0) {
    const int v = warpOff[lane];
    int x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    warpOff[lane] = x - v;
  }
  __syncthreads();
  if (!keep) return;
  const int at = blockOff[blockIdx.x] + warpOff[warp] + __popc(m & ((1u << lane) - 1u));
  k.x[at] = ox[i];
  k.y[at] = oy[i];
  k.area[at] = oarea[i];
  k.n[at] = on[i];
  k.tri[at] = otri[i];
  k.root[at] = oroot[i];
}

// Roots abandoned in a pass, compacted for the retry pass.
__global__ void collectKilledKernel(const int32_t* state, const int32_t* list, int n, int32_t* out, int* count) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int k = list ? list[j] : j;
  if (state[k] == kRootKilled) out[atomicAdd(count, 1)] = k;
}

// vis = missFx / 2^40 (clamped), E = Lambert integral or A G0 V
// (finalizeSoftKernel, cuda/wavefront.cu:539-561).
__global__ void softFinalizeKernel(AppParams a, const int32_t* state, int R) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= R) return;
  int pix;
  if (!softPixel(a, k, pix)) return;
  if (state[k] != kRootTraced) return;
  double V = double(a.missFx[k]) / kFixVis;
  V = V < 0 ? 0 : (V > 1 ? 1 : V);
  const float Vf = float(V);
  if (a.vis) a.vis[pix] = Vf;
  if (a.E) {
    if (a.exact) {
      a.E[pix] = float(double(a.gFx[k]) / kFixG);
    } else {
      const V3 x = mk(a.pixX[3 * pix], a.pixX[3 * pix + 1], a.pixX[3 * pix + 2]);
      const V3 ns = mk(a.pixN[3 * pix], a.pixN[3 * pix + 1], a.pixN[3 * pix + 2]);
      const float A = length(cross(a.LU, a.LV));
      a.E[pix] = A * lightCenterG(a.Lc, a.LU, a.LV, x, ns) * Vf;
    }
  }
}

// ------------------------------------------------------------ primary rays

// One eye ray per pixel centre (primaryKernel, cuda/gpu_render.cu:222-244):
// eyeRay, shared with the fused soft-shadow admission.
__global__ void __launch_bounds__(128) primaryRaysKernel(SceneDev s, bt_camera cam, int32_t* triOut, float* Xout,
                                                         float* Nout) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= cam.W || y >= cam.H) return;
  const size_t k = size_t(y) * size_t(cam.W) + size_t(x);
  V3 X, N;
  const int t = eyeRay(s, mk(cam.eye[0], cam.eye[1], cam.eye[2]), mk(cam.fwd[0], cam.fwd[1], cam.fwd[2]),
                       mk(cam.right[0], cam.right[1], cam.right[2]), mk(cam.down[0], cam.down[1], cam.down[2]),
                       cam.half_w, cam.half_h, cam.W, cam.H, x, y, &X, &N);
  triOut[k] = t;
  Xout[3 * k] = X.x;
  Xout[3 * k + 1] = X.y;
  Xout[3 * k + 2] = X.z;
  Nout[3 * k] = N.x;
  Nout[3 * k + 1] = N.y;
  Nout[3 * k + 2] = N.z;
}

// ---------------------------------------------------------------- raster

// Covers pixel centres with convex image-plane polygons (rasterize,
// src/render/render.cpp:49-95, one sample at the pixel centre): one thread
// per polygon; among polygons covering a centre (shared edges) the higher
// triangle id wins, so the result does not depend on polygon order.
// With `proot`, polygons straight from the engine's output buffers: only
// those of a root's final attempt count (the host-side filter of
// downloadPolys, done here).
__global__ void rasterKernel(bt_camera cam, const float* px_, const float* py_, const int32_t* pn, const int32_t* ptri,
                             int64_t np, int shadow, int32_t* triBuf, uint8_t* flagBuf, const int32_t* proot = nullptr,
                             const int32_t* patt = nullptr, const int32_t* rootState = nullptr,
                             const int32_t* rootAttempt = nullptr) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= np) return;
  if (proot) {
    const int r = proot[i];
    if (rootState[r] != kRootTraced || patt[i] != rootAttempt[r]) return;
  }
  const int n = pn[i], tri = ptri[i];
  if (!shadow && tri < 0) return;
  if (n < 3 || n > 4) return;
  double px[4], py[4], A[4], B[4], C[4];
  double ly = 1e300, hy = -1e300;
  for (int k = 0; k < n; ++k) {
    const float x = (px_[4 * i + k] / cam.half_w + 1) * 0.5f * float(cam.W);
    const float y = (py_[4 * i + k] / cam.half_h + 1) * 0.5f * float(cam.H);
    px[k] = double(x);
    py[k] = double(y);
    ly = ly < py[k] ? ly : py[k];
    hy = hy > py[k] ? hy : py[k];
  }
  for (int k = 0; k < n; ++k) {
    const int j = k + 1 == n ? 0 : k + 1;
    A[k] = -(py[j] - py[k]);
    B[k] = px[j] - px[k];
    C[k] = -(A[k] * px[k] + B[k] * py[k]);
  }
  const double o = 0.5;
  const int y0 = max(0, int(ceil(ly - o))), y1 = min(cam.H - 1, int(floor(hy - o)));
  for (int y = y0; y <= y1; ++y) {
    const double sy = y + o;
    double xl = -1e300, xr = 1e300;
    bool empty = false;
    for (int k = 0; k < n && !empty; ++k) {
      const double rr = B[k] * sy + C[k];
      if (A[k] > 0)
        xl = xl > -rr / A[k] ? xl : -rr / A[k];
      else if (A[k] < 0)
        xr = xr < -rr / A[k] ? xr : -rr / A[k];
      else if (rr < 0)
        empty = true;
    }
    if (empty || xl > xr) continue;
    const int x0 = max(0, int(ceil(xl - o))), x1 = min(cam.W - 1, int(floor(xr - o)));
    for (int x = x0; x <= x1; ++x) {
      const size_t k = size_t(y) * size_t(cam.W) + size_t(x);
      if (shadow)
        flagBuf[k] = 1;
      else
        atomicMax(&triBuf[k], tri);
    }
  }
}

// Pool triangle ids to a scene's own (background -1 stays).
__global__ void rebaseKernel(int32_t* p, int64_t n, int32_t base) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n && p[i] >= 0) p[i] -= base;
}

__global__ void fillKernel(int32_t* p, int64_t n, int32_t v) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

template <class T>
int devAlloc(T** p, size_t n) {
  *p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
  if (e != cudaSuccess) {
    setErr("cudaMalloc(%zu bytes): %s", n * sizeof(T), cudaGetErrorString(e));
    return BT_ERR_NOMEM;
  }
  return BT_OK;
}

}  // namespace

// ------------------------------------------------------------------ context

// One scene of a context's pool.
struct PoolScene {
  uint32_t rootNode;
  int triBase;
  int64_t numTris;
  Box box;
  float offset;
};

struct bt_gpu_ctx {
  int device = 0;
  int sms = 1;
  bt_gpu_config cfg;
  cudaStream_t stream = nullptr;
  // scene
  uint2* dNode = nullptr;
  float4* dBox = nullptr;
  uint32_t* dParent = nullptr;
  float4* dRef = nullptr;
  float4* dTriNV = nullptr;
  SceneDev s;        // the whole scene pool; bounds and rootNode are the first scene's
  float offset = 0;  // |first scene's diagonal| * kEpsRel
  int64_t numTris = 0, numRefs = 0;
  std::vector<PoolScene> pool;
  // engine
  SubBeam* dQ[3] = {nullptr, nullptr, nullptr};  // trace queues 0, 1 and the clip queue
  int capacity = 0;
  Counters* dCtr = nullptr;
  unsigned long long* dStats = nullptr;
  size_t rootCap = 0;
  RootRec* dRoots = nullptr;
  int32_t *dLive = nullptr, *dState = nullptr, *dAttempt = nullptr, *dList[2] = {nullptr, nullptr};
  int32_t* dResv = nullptr;  // queue slots each root holds reserved
  unsigned long long *dMiss = nullptr, *dG = nullptr;
  float4* dShade = nullptr;
  int* dKillCount = nullptr;
  // outputs
  int64_t outCap = 0;
  int64_t lastProduced = -1;  // polygons of the last bt_gpu_primary / bt_gpu_point (bt_gpu_last_polys)
  float *dOx = nullptr, *dOy = nullptr, *dOarea = nullptr;
  int32_t *dOn = nullptr, *dOtri = nullptr, *dOroot = nullptr, *dOatt = nullptr;
  // per-image scratch
  int64_t pixCap = 0;
  int32_t* dPixTri = nullptr;
  float *dPixX = nullptr, *dPixN = nullptr, *dVis = nullptr, *dE = nullptr, *dEu = nullptr;
  int blocksSoft = 0, blocksPrimary = 0, blocksPoint = 0;
  // device-resident primary ids / point masks: compacted hit polygons
  int64_t hitCap = 0;
  float *dHx = nullptr, *dHy = nullptr;
  int32_t *dHn = nullptr, *dHt = nullptr;
  int* dHitCount = nullptr;
  // host-polygon calls: the final attempts' polygons compacted on the device
  int64_t keepCap = 0;
  int keepBlocksCap = 0;
  float *dKx = nullptr, *dKy = nullptr, *dKarea = nullptr;
  int32_t *dKn = nullptr, *dKtri = nullptr, *dKroot = nullptr;
  int* dKeepBlocks = nullptr;
  uint8_t* dFlag = nullptr;  // host-output variants: the mask in device memory
  int64_t flagCap = 0;
  // batched soft shadows: per-job parameter table and root offsets
  AppParams* dJobs = nullptr;
  int32_t* dJobStart = nullptr;
  int jobCap = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t rev[2] = {nullptr, nullptr};
  cudaEvent_t kev[32] = {};  // kernel_timing: 2 per round of a batch, around the trace kernel
  // graph_rounds: the last captured batch of rounds, one for full rounds and
  // one for tail rounds, with the launch parameters it was captured with
  struct RoundGraph {
    cudaGraphExec_t exec = nullptr;
    RoundParams p;
    int app = -1, mode = -1, grids[4] = {0, 0, 0, 0};
    bool admit = true;
  } graphs[2];
  // serving (serve.cpp): a lane views its parent's scene pool and owns only
  // its engine buffers; the parent's scene lock is held shared while a lane
  // works and exclusively while bt_gpu_add_scene replaces the arrays
  bt_gpu_ctx* parent = nullptr;
  bool ownsScene = true;
  std::shared_mutex sceneLock;
  void* serving = nullptr;       // the serving state of bt_gpu_submit / bt_gpu_poll
  int32_t* dRanges = nullptr;    // streaming runs: root ranges of the jobs checked for completion
  int* dJobCounts = nullptr;     // and their live / abandoned root counts
  std::atomic<int64_t> queueHighWater{0};  // largest trace queue a lane has needed (records)
};

// For the host-side modules of the library (ingest.cpp): sets the message
// bt_gpu_last_error returns on this thread.
void btSetError(const char* msg) { setErr("%s", msg); }

extern "C" {

const char* bt_gpu_last_error(void) { return g_err; }

void bt_gpu_config_default(bt_gpu_config* c) {
  c->device = 0;
  c->budget = 2048;
  c->primary_budget = 4096;
  c->capacity = 0;
  c->blocks_per_sm = 0;
  c->kernel_timing = 0;
  c->max_retries = 4;
  c->tail_records = 0;
  c->eps_stats = 0;
  c->yield_pct = 0;
  c->fuse_primary = 0;
  c->eps_fp64 = 0;
  c->graph_rounds = 1;
  c->trace_ctas = 0;
}

int bt_gpu_available(bt_gpu_info* info) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    setErr("no CUDA device");
    return BT_ERR_NODEVICE;
  }
  if (info) {
    cudaDeviceProp pr;
    if (cudaGetDeviceProperties(&pr, 0) != cudaSuccess) return BT_ERR_NODEVICE;
    snprintf(info->name, sizeof info->name, "%s", pr.name);
    info->sm_count = pr.multiProcessorCount;
    info->mem_gb = double(pr.totalGlobalMem) / double(1 << 30);
    info->cc_major = pr.major;
    info->cc_minor = pr.minor;
  }
  return BT_OK;
}

}  // extern "C"

namespace {

int ensureRoots(bt_gpu_ctx* c, size_t R) {
  if (c->rootCap >= R) return BT_OK;
  cudaFree(c->dRoots);
  cudaFree(c->dLive);
  cudaFree(c->dResv);
  cudaFree(c->dState);
  cudaFree(c->dAttempt);
  cudaFree(c->dList[0]);
  cudaFree(c->dList[1]);
  cudaFree(c->dMiss);
  cudaFree(c->dG);
  cudaFree(c->dShade);
  c->rootCap = 0;
  int e;
  if ((e = devAlloc(&c->dRoots, R)) || (e = devAlloc(&c->dLive, R)) || (e = devAlloc(&c->dResv, R)) ||
      (e = devAlloc(&c->dState, R)) ||
      (e = devAlloc(&c->dAttempt, R)) || (e = devAlloc(&c->dList[0], R)) || (e = devAlloc(&c->dList[1], R)) ||
      (e = devAlloc(&c->dMiss, R)) || (e = devAlloc(&c->dG, R)) || (e = devAlloc(&c->dShade, 2 * R)))
    return e;
  c->rootCap = R;
  return BT_OK;
}

int ensureOut(bt_gpu_ctx* c, int64_t cap) {
  if (c->outCap >= cap) return BT_OK;
  cudaFree(c->dOx);
  cudaFree(c->dOy);
  cudaFree(c->dOarea);
  cudaFree(c->dOn);
  cudaFree(c->dOtri);
  cudaFree(c->dOroot);
  cudaFree(c->dOatt);
  c->outCap = 0;
  int e;
  if ((e = devAlloc(&c->dOx, size_t(4 * cap))) || (e = devAlloc(&c->dOy, size_t(4 * cap))) ||
      (e = devAlloc(&c->dOarea, size_t(cap))) || (e = devAlloc(&c->dOn, size_t(cap))) ||
      (e = devAlloc(&c->dOtri, size_t(cap))) || (e = devAlloc(&c->dOroot, size_t(cap))) ||
      (e = devAlloc(&c->dOatt, size_t(cap))))
    return e;
  c->outCap = cap;
  return BT_OK;
}

int ensurePix(bt_gpu_ctx* c, int64_t n) {
  if (c->pixCap >= n) return BT_OK;
  cudaFree(c->dPixTri);
  cudaFree(c->dPixX);
  cudaFree(c->dPixN);
  cudaFree(c->dVis);
  cudaFree(c->dE);
  cudaFree(c->dEu);
  c->pixCap = 0;
  int e;
  if ((e = devAlloc(&c->dPixTri, size_t(n))) || (e = devAlloc(&c->dPixX, size_t(3 * n))) ||
      (e = devAlloc(&c->dPixN, size_t(3 * n))) || (e = devAlloc(&c->dVis, size_t(n))) ||
      (e = devAlloc(&c->dE, size_t(n))) || (e = devAlloc(&c->dEu, size_t(n))))
    return e;
  c->pixCap = n;
  return BT_OK;
}

template <class K>
int gridFor(bt_gpu_ctx* c, K kernel, size_t smem = 0) {
  int perSM = 1;
  if (smem > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, kThreads, smem);
  if (c->cfg.blocks_per_sm > 0) perSM = std::min(perSM, c->cfg.blocks_per_sm);
  return c->sms * std::max(1, perSM);
}

void fillInfo(bt_gpu_ctx* c, const Counters& hc, bt_run_info* info) {
  if (!info) return;
  unsigned long long st[kNumStats];
  cudaMemcpy(st, c->dStats, sizeof st, cudaMemcpyDeviceToHost);
  info->kd_steps = st[kStKd];
  info->leaf_visits = st[kStLeaf];
  info->tri_tests = st[kStTests];
  info->hits = st[kStHits];
  info->splits = st[kStSplits];
  info->beams = st[kStBeams];
  info->root_beams = st[kStRoots];
  info->presplit_beams = st[kStPresplit];
  info->five_splits = st[kStFive];
  info->climbs = st[kStClimbs];
  double d;
  memcpy(&d, &st[kStDropped], sizeof d);
  info->dropped_area = d;
  info->eps_band_corners = st[kStEpsBand];
  info->eps_fp64_flips = st[kStEpsFlip];
  info->max_spill = std::max(info->max_spill, hc.maxQueue);
}

// Runs every root of `R` through the engine.  A round is three kernels --
// admit (new roots, as far as the queue reservation allows), trace (drain
// the round's queue), clip (pieces into the next round's queue) -- plus the
// bookkeeping kernel; rounds are launched in batches of kRoundsPerCheck
// between reads of the completion flag (rounds after completion return at
// once).  Roots abandoned over budget are retried in a further pass with a
// 16x budget.
constexpr int kRoundsPerCheck = 8;
// Scenes up to this many bytes on the device (kd nodes and boxes, leaf
// references, triangle normals) take the 4-CTA round trace kernel.
constexpr int64_t kWideSceneBytes = int64_t(16) << 20;
// The first batch of a pass is this many rounds: a pass whose queue then
// holds at most half a record per root (long walks, few splits: point
// shadows of a sparse scene) goes to tail rounds at once.
constexpr int kFirstRounds = 2;

// The FP64 band re-decision is compiled for soft shadows only; the other
// applications map it to the float votes (their kernels are not built twice).
template <int App>
constexpr int kVoteFp64F = App == kAppSoft ? kVoteFp64 : kVoteFloat;

// The resident scene pool's bytes on the device: kd nodes and boxes, leaf
// references, triangle normals and planes.
int64_t sceneDeviceBytes(const bt_gpu_ctx* c) {
  return int64_t(c->s.numNodes) * (8 + 32 + 4) + c->numRefs * 64 + c->numTris * 32;
}

template <int App>
struct RoundRunner {
  bt_gpu_ctx* c;
  bt_run_info* info;
  RoundParams p;
  int mode = kVoteFloat;
  bool wide = false;  // the 4-CTA round trace kernel
  bool ktime = false;
  int gA = 0, gT = 0, gC = 0, gF = 0, yieldAt = INT_MAX;
  int64_t tailRecords = 0;
  FILE* roundLog = nullptr;  // BT_ROUND_LOG=1: one line per batch of rounds on stderr (diagnostics)
  int launches = 0, passes = 0, retried = 0, roundsRun = 0, tailRounds = 0, pass = -1, round = 0;
  int64_t yieldsRun = 0;
  Counters hc;

  RoundRunner(bt_gpu_ctx* ctx, bt_run_info* inf) : c(ctx), info(inf) { memset(&hc, 0, sizeof hc); }

  // Clears the per-run state of R roots and sets the launch parameters.
  int begin(const AppParams& app0, int R) {
    memset(&p, 0, sizeof p);  // no stray padding: graph_rounds compares launch parameters bytewise
    c->lastProduced = -1;  // a new run overwrites what bt_gpu_last_polys would read
    int e = ensureRoots(c, size_t(R));
    if (e) return e;
    CK(cudaMemsetAsync(c->dAttempt, 0, sizeof(int32_t) * size_t(R), c->stream));
    CK(cudaMemsetAsync(c->dStats, 0, sizeof(unsigned long long) * kNumStats, c->stream));
    CK(cudaMemsetAsync(c->dCtr, 0, sizeof(Counters), c->stream));
    AppParams app = app0;
    app.missFx = c->dMiss;
    app.gFx = c->dG;
    app.shade = c->dShade;
    p.s = c->s;
    p.tq[0] = c->dQ[0];
    p.tq[1] = c->dQ[1];
    p.cq = c->dQ[2];
    p.capacity = c->capacity;
    p.roots = c->dRoots;
    p.rootCap = R;
    p.live = c->dLive;
    p.resv = c->dResv;
    p.state = c->dState;
    p.attempt = c->dAttempt;
    p.ctr = c->dCtr;
    p.stats = c->dStats;
    p.app = app;
    // the edge votes: eps_fp64 (soft shadows) re-decides fuzzy-band corners
    // in FP64, eps_stats logs them, else the reference's float votes
    mode = (App == kAppSoft && c->cfg.eps_fp64) ? kVoteFp64 : (c->cfg.eps_stats ? kVoteLog : kVoteFloat);
    gA = gridFor(c, admitKernel<App>);
    // 4 trace CTAs per SM on a scene small enough to stay in L1/L2
    // (trace_ctas 0), or as configured
    wide = mode == kVoteFloat &&
           (c->cfg.trace_ctas == 4 || (c->cfg.trace_ctas == 0 && sceneDeviceBytes(c) <= kWideSceneBytes));
    gT = mode == kVoteFp64 ? gridFor(c, traceKernel<App, false, kVoteFp64F<App>>)
         : mode == kVoteLog ? gridFor(c, traceKernel<App, false, kVoteLog>)
         : wide             ? gridFor(c, traceKernel<App, false, kVoteFloat, 4>)
                            : gridFor(c, traceKernel<App, false>);
    gC = mode == kVoteFp64 ? gridFor(c, clipKernel<App, App == kAppSoft>, kLogSmem)
                           : gridFor(c, clipKernel<App>, kLogSmem);
    gF = mode == kVoteFp64 ? gridFor(c, traceKernel<App, true, kVoteFp64F<App>>, kLogSmem)
         : mode == kVoteLog ? gridFor(c, traceKernel<App, true, kVoteLog>, kLogSmem)
                            : gridFor(c, traceKernel<App, true>, kLogSmem);
    // tail rounds: every root admitted and fewer queued records than this
    // (default: a sixth of the trace grid's lanes, about two warps' worth per SM -- the fused kernel clips
    // inside the divergent walk, which only pays once the queue no longer fills the GPU)
    tailRecords = c->cfg.tail_records > 0 ? c->cfg.tail_records : int64_t(gT) * kThreads / 6;
    const int yieldPct = c->cfg.yield_pct == 0 ? 50 : std::min(c->cfg.yield_pct, 100);
    yieldAt = yieldPct < 0 ? INT_MAX : std::max(1, int(int64_t(gT) * kWarps * yieldPct / 100));
    static_assert(2 * kRoundsPerCheck <= 32, "kernel_timing events");
    ktime = c->cfg.kernel_timing && c->kev[0] != nullptr;
    roundLog = getenv("BT_ROUND_LOG") ? stderr : nullptr;
    return BT_OK;
  }

  // Starts the next pass over `n` roots (the first `n`, or `list`) with a
  // live sub-beam budget of `budget` per root.
  int startPass(int n, const int32_t* list, int budget) {
    ++pass;
    p.budget = budget;
    // Roots reserve little when admitted and grow (a root over its budget,
    // or one the free capacity cannot cover, is retried in the next pass
    // with 16x the budget); the last retry pass admits roots holding their
    // whole budget, or the whole queue, so that no root is squeezed there:
    // every root that fits a queue finishes.
    const bool strict = pass >= c->cfg.max_retries;
    p.reserve = strict ? int(std::max<int64_t>(std::min<int64_t>(budget, c->capacity), 32))
                       : std::max(std::min(budget, kInitialReserve), 32);
    if (int64_t(p.reserve) > c->capacity) {
      setErr("a root needs more than %d live sub-beams (queue capacity %d)", budget / 16, c->capacity);
      return BT_ERR_CAPACITY;
    }
    p.numRoots = n;
    p.rootList = list;
    p.yieldAt = yieldAt;
    if (pass > 0) {
      // per-pass state; the output count carries over
      Counters z;
      memset(&z, 0, sizeof z);
      z.outCount = hc.outCount;
      z.maxQueue = hc.maxQueue;
      CK(cudaMemcpyAsync(c->dCtr, &z, sizeof z, cudaMemcpyHostToDevice, c->stream));
      hc = z;
    }
    ++passes;
    round = 0;
    return BT_OK;
  }

  // More roots for the running pass (numRoots grew): a pass that had
  // finished goes on.
  int reopen() {
    if (!hc.done) return BT_OK;
    const int zero = 0;
    CK(cudaMemcpyAsync(&c->dCtr->done, &zero, sizeof zero, cudaMemcpyHostToDevice, c->stream));
    hc.done = 0;
    return BT_OK;
  }

  // One batch of kRoundsPerCheck rounds (not the first) as one CUDA graph (graph_rounds):
  // the launches are captured once and replayed while their parameters stay
  // the same (a new frame with the same camera, light and buffers replays
  // the graph of the last one); otherwise captured again and the
  // executable graph updated in place.
  int graphBatch(bool tail, bool admit) {
    auto& g = c->graphs[tail ? 1 : 0];
    RoundParams key = p;
    key.cur = 0;
    const int grids[4] = {gA, gT, gC, gF};
    if (!g.exec || g.app != App || g.mode != mode || g.admit != admit || memcmp(grids, g.grids, sizeof grids) != 0 ||
        memcmp(&key, &g.p, sizeof key) != 0) {
      CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
      const int r0 = round, l0 = launches, t0 = tailRounds;
      launchRounds(tail, admit, false);
      round = r0;
      launches = l0;
      tailRounds = t0;
      cudaGraph_t graph = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
      if (ce != cudaSuccess || !graph) {
        setErr("capturing a batch of rounds: %s", cudaGetErrorString(ce));
        return BT_ERR_CUDA;
      }
      cudaError_t ue = cudaErrorUnknown;
      if (g.exec) {
        cudaGraphExecUpdateResultInfo ui;
        ue = cudaGraphExecUpdate(g.exec, graph, &ui);
        if (ue != cudaSuccess) {
          cudaGetLastError();
          cudaGraphExecDestroy(g.exec);
          g.exec = nullptr;
        }
      }
      if (ue != cudaSuccess) {
        const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
        if (ie != cudaSuccess) {
          cudaGraphDestroy(graph);
          g.exec = nullptr;
          setErr("instantiating a batch of rounds: %s", cudaGetErrorString(ie));
          return BT_ERR_CUDA;
        }
      }
      cudaGraphDestroy(graph);
      g.p = key;
      g.app = App;
      g.mode = mode;
      g.admit = admit;
      memcpy(g.grids, grids, sizeof grids);
    }
    CK(cudaGraphLaunch(g.exec, c->stream));
    for (int k = 0; k < kRoundsPerCheck; ++k, ++round) {
      launches += tail ? 2 : (admit ? 4 : 3);
      if (tail) tailRounds++;
    }
    return BT_OK;
  }

  // The launches of one batch of rounds on the engine's stream
  // (kFirstRounds at the start of a pass, else kRoundsPerCheck; full rounds:
  // admit, trace, clip; tail rounds: the fused kernel; then the bookkeeping
  // kernel), with the kernel_timing events when `events`; returns the rounds.
  // `admit`: some roots are not admitted yet (else the admit kernel, which
  // would find none, is not launched).
  int launchRounds(bool tail, bool admit, bool events) {
    const int n = p.numRoots;
    const int nr = round == 0 ? kFirstRounds : kRoundsPerCheck;
    for (int k = 0; k < nr; ++k, ++round) {
      p.cur = round & 1;
      if (tail) {
        if (events) cudaEventRecord(c->kev[2 * k], c->stream);
        if (mode == kVoteFp64)
          traceKernel<App, true, kVoteFp64F<App>><<<gF, kThreads, kLogSmem, c->stream>>>(p);
        else if (mode == kVoteLog)
          traceKernel<App, true, kVoteLog><<<gF, kThreads, kLogSmem, c->stream>>>(p);
        else
          traceKernel<App, true><<<gF, kThreads, kLogSmem, c->stream>>>(p);
        if (events) cudaEventRecord(c->kev[2 * k + 1], c->stream);
        launches += 2;
        tailRounds++;
      } else {
        if (admit) admitKernel<App><<<gA, kThreads, 0, c->stream>>>(p);
        if (events) cudaEventRecord(c->kev[2 * k], c->stream);
        if (mode == kVoteFp64)
          traceKernel<App, false, kVoteFp64F<App>><<<gT, kThreads, 0, c->stream>>>(p);
        else if (mode == kVoteLog)
          traceKernel<App, false, kVoteLog><<<gT, kThreads, 0, c->stream>>>(p);
        else if (wide)
          traceKernel<App, false, kVoteFloat, 4><<<gT, kThreads, 0, c->stream>>>(p);
        else
          traceKernel<App, false><<<gT, kThreads, 0, c->stream>>>(p);
        if (events) cudaEventRecord(c->kev[2 * k + 1], c->stream);
        if (mode == kVoteFp64)
          clipKernel<App, App == kAppSoft><<<gC, kThreads, kLogSmem, c->stream>>>(p);
        else
          clipKernel<App><<<gC, kThreads, kLogSmem, c->stream>>>(p);
        launches += admit ? 4 : 3;
      }
      roundEndKernel<<<1, 1, 0, c->stream>>>(c->dCtr, p.cur, n);
    }
    return nr;
  }

  // One batch of rounds, then the counters.
  int batch() {
    const int n = p.numRoots;
    CK(cudaEventRecord(c->rev[0], c->stream));
    // the mode of this batch of rounds, from the counters of the last one
    const int64_t queued = hc.count[round & 1];
    const bool tail = round > 0 && hc.rootNext >= n && queued < tailRecords && c->cfg.tail_records >= 0 &&
                      (round > kFirstRounds || 2 * queued <= n);
    // (the legacy default stream, which the allocation-free entry point
    // runs on, cannot be captured)
    const bool admit = hc.rootNext < n;
    int nr = kRoundsPerCheck;
    if (c->cfg.graph_rounds && !ktime && c->stream != nullptr && round > 0) {
      const int e = graphBatch(tail, admit);
      if (e) return e;
    } else {
      nr = launchRounds(tail, admit, ktime);
    }
    CK(cudaEventRecord(c->rev[1], c->stream));
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(&hc, c->dCtr, sizeof hc, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->rev[0], c->rev[1]);
    if (info) {
      info->ms_round += ms;
      info->round_launches += 3 * nr;
      if (ktime)
        for (int k = 0; k < nr; ++k) {
          float t = 0;
          CK(cudaEventElapsedTime(&t, c->kev[2 * k], c->kev[2 * k + 1]));
          info->ms_kernel_trace += t;
        }
    }
    if (roundLog)
      fprintf(roundLog, "pass %d rounds %d inflight %d rootNext %d/%d queue %d yields %d ms %.3f\n", pass, hc.rounds,
              hc.inflight, hc.rootNext, n, hc.count[round & 1], hc.yields, ms);
    if (hc.error) {
      setErr(hc.error == 2 ? "malformed sub-beam record" : "sub-beam queue overflow (capacity %d)", c->capacity);
      return BT_ERR_CAPACITY;
    }
    if (!hc.done && launches > kMaxLaunches) {
      setErr("launch limit reached with %d roots in flight", hc.inflight);
      return BT_ERR_TIMEOUT;
    }
    return BT_OK;
  }

  // After a pass: its roots abandoned over budget, compacted into a retry
  // list (*list, *nk; nk = 0: none).
  int endPass(int n, const int32_t** list, int* nk) {
    if (info) info->max_spill = std::max(info->max_spill, hc.maxQueue);
    roundsRun += hc.rounds;
    yieldsRun += hc.yields;
    *nk = 0;
    if (hc.killed == 0) return BT_OK;
    if (pass >= c->cfg.max_retries) {
      setErr("%d roots still over budget %d after %d retries", hc.killed, p.budget, pass);
      return BT_ERR_CAPACITY;
    }
    int32_t* dst = c->dList[pass & 1];
    CK(cudaMemsetAsync(c->dKillCount, 0, sizeof(int), c->stream));
    collectKilledKernel<<<(n + 255) / 256, 256, 0, c->stream>>>(c->dState, *list, n, dst, c->dKillCount);
    launches++;
    CK(cudaMemcpyAsync(nk, c->dKillCount, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    retried += *nk;
    if (pass == 0 && info) info->overflow_roots += *nk;
    *list = dst;
    return BT_OK;
  }

  void finish(int64_t R) {
    if (!info) return;
    info->rounds += roundsRun;
    info->tail_rounds += tailRounds;
    info->yields += yieldsRun;
    info->launches += launches;
    info->passes += passes;
    info->retried_roots += retried;
    info->roots += R;
    fillInfo(c, hc, info);
  }
};

template <int App>
int runRoots(bt_gpu_ctx* c, AppParams app, int R, int budget, bt_run_info* info) {
  RoundRunner<App> rr(c, info);
  int e = rr.begin(app, R);
  if (e) return e;
  const int32_t* list = nullptr;
  int n = R;
  for (;;) {
    if ((e = rr.startPass(n, list, budget))) return e;
    do {
      if ((e = rr.batch())) return e;
    } while (!rr.hc.done);
    int nk = 0;
    if ((e = rr.endPass(n, &list, &nk))) return e;
    if (nk == 0) break;
    // retry the abandoned roots with a larger budget
    n = nk;
    budget *= 16;
  }
  rr.finish(R);
  return BT_OK;
}

// Grows a device array to n elements, keeping the first `keep` (the pool's
// earlier scenes).
template <class T>
int growArray(T** p, size_t keep, size_t n) {
  T* q = nullptr;
  int e = devAlloc(&q, n);
  if (e) return e;
  if (keep && *p) {
    cudaError_t ce = cudaMemcpy(q, *p, keep * sizeof(T), cudaMemcpyDeviceToDevice);
    if (ce != cudaSuccess) {
      cudaFree(q);
      setErr("cudaMemcpy: %s", cudaGetErrorString(ce));
      return BT_ERR_CUDA;
    }
  }
  cudaFree(*p);
  *p = q;
  return BT_OK;
}

// Appends a scene and its kd-tree to the context's scene pool: nodes,
// references and triangles go after the earlier scenes', with child, leaf,
// parent and triangle indices offset to the pool's numbering, so that one
// SceneDev serves every scene and a root only needs its scene's kd root.
int uploadScene(bt_gpu_ctx* c, const bt_scene_desc* sc, const bt_kd_desc* kd) {
  const int64_t nn = kd->num_nodes, nr = kd->num_refs, nt = sc->num_tris;
  const uint32_t nodeBase = c->s.numNodes, triBase = uint32_t(c->numTris);
  const int64_t refBase = c->numRefs;
  if (int64_t(nodeBase) + nn >= (int64_t(1) << 30) || int64_t(triBase) + nt >= (int64_t(1) << 31) ||
      refBase + nr >= (int64_t(1) << 32)) {
    setErr("the scene pool would exceed 2^30 kd nodes, 2^31 triangles or 2^32 references");
    return BT_ERR_TOO_LARGE;
  }
  std::vector<uint2> node(static_cast<size_t>(nn));
  std::vector<float4> box(static_cast<size_t>(2 * nn));
  std::vector<uint32_t> parent(static_cast<size_t>(nn));
  for (int64_t i = 0; i < nn; ++i) {
    const uint32_t d = kd->data[i];
    uint32_t x, dd = d;
    if ((d & 3u) == 3u) {
      x = kd->offset[i];
      if (int64_t(x) + int64_t(d >> 2) > nr) {
        setErr("kd leaf %lld points past the reference list", (long long)i);
        return BT_ERR_INVALID;
      }
      x += uint32_t(refBase);
    } else {
      memcpy(&x, &kd->split[i], 4);
      if (int64_t(d >> 2) >= nn) {
        setErr("kd node %lld has an invalid child", (long long)i);
        return BT_ERR_INVALID;
      }
      dd = (((d >> 2) + nodeBase) << 2) | (d & 3u);
    }
    node[size_t(i)] = make_uint2(x, dd);
    const float* b = kd->node_box + 6 * i;
    box[size_t(2 * i)] = make_float4(b[0], b[1], b[2], b[3]);
    box[size_t(2 * i + 1)] = make_float4(b[4], b[5], 0.f, 0.f);
    const uint32_t par = kd->parent[i];
    parent[size_t(i)] = par == ~0u ? ~0u : par + nodeBase;
  }
  std::vector<float4> ref(static_cast<size_t>(4 * nr));
  for (int64_t k = 0; k < nr; ++k) {
    const uint32_t t = kd->tri_indices[k];
    if (int64_t(t) >= nt) {
      setErr("kd reference %lld names triangle %u of %lld", (long long)k, t, (long long)nt);
      return BT_ERR_INVALID;
    }
    const uint32_t* vi = sc->tris + 3 * size_t(t);
    const float* p0 = sc->pos + 3 * size_t(vi[0]);
    const float* p1 = sc->pos + 3 * size_t(vi[1]);
    const float* p2 = sc->pos + 3 * size_t(vi[2]);
    const float* n = sc->tri_normals + 3 * size_t(t);
    float w[4];
    uint32_t u[4] = {vi[0], vi[1], vi[2], t + triBase};
    memcpy(w, u, 16);
    ref[size_t(4 * k)] = make_float4(p0[0], p0[1], p0[2], p1[0]);
    ref[size_t(4 * k + 1)] = make_float4(p1[1], p1[2], p2[0], p2[1]);
    ref[size_t(4 * k + 2)] = make_float4(p2[2], n[0], n[1], n[2]);
    ref[size_t(4 * k + 3)] = make_float4(w[0], w[1], w[2], w[3]);
  }
  std::vector<float4> tnv(static_cast<size_t>(2 * nt));
  for (int64_t t = 0; t < nt; ++t) {
    const float* n = sc->tri_normals + 3 * t;
    const float* p0 = sc->pos + 3 * size_t(sc->tris[3 * t]);
    tnv[size_t(2 * t)] = make_float4(n[0], n[1], n[2], 0.f);
    tnv[size_t(2 * t + 1)] = make_float4(p0[0], p0[1], p0[2], 0.f);
  }
  const size_t NN = size_t(nodeBase) + size_t(nn), NR = size_t(refBase) + size_t(nr),
               NT = size_t(triBase) + size_t(nt);
  int e;
  if ((e = growArray(&c->dNode, nodeBase, NN)) || (e = growArray(&c->dBox, 2 * size_t(nodeBase), 2 * NN)) ||
      (e = growArray(&c->dParent, nodeBase, NN)) || (e = growArray(&c->dRef, 4 * size_t(refBase), 4 * NR + 4)) ||
      (e = growArray(&c->dTriNV, 2 * size_t(triBase), 2 * NT)))
    return e;
  CK(cudaMemcpy(c->dNode + nodeBase, node.data(), sizeof(uint2) * node.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->dBox + 2 * size_t(nodeBase), box.data(), sizeof(float4) * box.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->dParent + nodeBase, parent.data(), sizeof(uint32_t) * parent.size(), cudaMemcpyHostToDevice));
  if (nr)
    CK(cudaMemcpy(c->dRef + 4 * size_t(refBase), ref.data(), sizeof(float4) * ref.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->dTriNV + 2 * size_t(triBase), tnv.data(), sizeof(float4) * tnv.size(), cudaMemcpyHostToDevice));
  c->s.node = c->dNode;
  c->s.box = c->dBox;
  c->s.parent = c->dParent;
  c->s.ref = c->dRef;
  c->s.triNV = c->dTriNV;
  PoolScene ps;
  ps.rootNode = nodeBase;
  ps.triBase = int(triBase);
  ps.numTris = nt;
  for (int a = 0; a < 3; ++a) {
    ps.box.lo[a] = kd->bounds[a];
    ps.box.hi[a] = kd->bounds[3 + a];
  }
  // offset = length(scene.bounds.diag()) * kEpsRel (render.cpp:348)
  V3 dg = mk(sc->bounds[3] - sc->bounds[0], sc->bounds[4] - sc->bounds[1], sc->bounds[5] - sc->bounds[2]);
  ps.offset = length(dg) * kEpsRel;
  if (c->pool.empty()) {  // the first scene: what the single-scene entry points trace
    c->s.bounds = ps.box;
    c->s.rootNode = 0;
    c->offset = ps.offset;
  }
  c->pool.push_back(ps);
  c->s.numTris = int(NT);
  c->s.numNodes = uint32_t(NN);
  c->numTris = int64_t(NT);
  c->numRefs = int64_t(NR);
  return BT_OK;
}

AppParams baseApp(const bt_gpu_ctx* c, const bt_camera* cam) {
  AppParams a;
  memset(&a, 0, sizeof a);
  if (cam) {
    a.W = cam->W;
    a.H = cam->H;
    a.eye = mk(cam->eye[0], cam->eye[1], cam->eye[2]);
    a.fwd = mk(cam->fwd[0], cam->fwd[1], cam->fwd[2]);
    a.right = mk(cam->right[0], cam->right[1], cam->right[2]);
    a.down = mk(cam->down[0], cam->down[1], cam->down[2]);
    a.halfW = cam->half_w;
    a.halfH = cam->half_h;
    // Camera::plane (render_types.h:21)
    a.camPlane = makePlane(a.eye, add(a.eye, a.fwd), a.right, a.down);
  }
  a.out.x = c->dOx;
  a.out.y = c->dOy;
  a.out.n = c->dOn;
  a.out.tri = c->dOtri;
  a.out.area = c->dOarea;
  a.out.root = c->dOroot;
  a.out.attempt = c->dOatt;
  a.out.cap = int(std::min<int64_t>(c->outCap, 0x7fffffff));
  return a;
}

bool camOk(const bt_camera* cam) { return cam && cam->W > 0 && cam->H > 0 && cam->W <= 65536 && cam->H <= 65536; }

int softCore(bt_gpu_ctx* c, const bt_area_light* L, const bt_soft_opts* o, int64_t n, const bt_camera* cam,
             const int32_t* dTri, const float* dX, const float* dN, float* dVis, float* dE, float* dEu,
             bt_run_info* info, int32_t* fusedTri = nullptr, float* fusedX = nullptr, float* fusedN = nullptr) {
  AppParams a = baseApp(c, cam);
  if (fusedTri && cam) {
    a.fusedPrimary = 1;
    a.pixTriOut = fusedTri;
    a.pixXOut = fusedX;
    a.pixNOut = fusedN;
  }
  a.Lc = mk(L->c[0], L->c[1], L->c[2]);
  a.LU = mk(L->U[0], L->U[1], L->U[2]);
  a.LV = mk(L->V[0], L->V[1], L->V[2]);
  a.offset = (o && o->offset > 0) ? o->offset : c->offset;
  a.exact = o ? o->exact : 0;
  a.pixTri = dTri;
  a.pixX = dX;
  a.pixN = dN;
  a.vis = dVis;
  a.E = dE;
  a.Eu = dEu;
  int R;
  if (cam) {
    a.tiled = 1;
    a.tilesX = (cam->W + 7) / 8;
    R = a.tilesX * ((cam->H + 3) / 4) * 32;
  } else {
    a.tiled = 0;
    a.W = int(n);
    a.H = 1;
    R = int(n);
  }
  if (R == 0) return BT_OK;
  int e = runRoots<kAppSoft>(c, a, R, c->cfg.budget, info);
  if (e) return e;
  a.missFx = c->dMiss;
  a.gFx = c->dG;
  softFinalizeKernel<<<(R + 255) / 256, 256, 0, c->stream>>>(a, c->dState, R);
  if (info) info->launches++;
  CK(cudaGetLastError());
  return BT_OK;
}

}  // namespace

extern "C" {

int bt_gpu_create(const bt_scene_desc* scene, const bt_kd_desc* kd, const bt_gpu_config* cfg, bt_gpu_ctx** out) {
  if (!scene || !kd || !out || scene->num_tris <= 0 || kd->num_nodes <= 0) {
    setErr("bt_gpu_create: empty scene or tree");
    return BT_ERR_INVALID;
  }
  *out = nullptr;
  bt_gpu_ctx* c = new bt_gpu_ctx();
  if (cfg)
    c->cfg = *cfg;
  else
    bt_gpu_config_default(&c->cfg);
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || c->cfg.device < 0 || c->cfg.device >= ndev) {
    cudaGetLastError();
    delete c;
    setErr("no CUDA device %d", cfg ? cfg->device : 0);
    return BT_ERR_NODEVICE;
  }
  c->device = c->cfg.device;
  int e = BT_OK;
  auto fail = [&](int code) {
    bt_gpu_destroy(c);
    return code;
  };
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(BT_ERR_CUDA);
  cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->device);
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(BT_ERR_CUDA);
  for (auto& ev : c->ev)
    if (cudaEventCreate(&ev) != cudaSuccess) return fail(BT_ERR_CUDA);
  for (auto& ev : c->rev)
    if (cudaEventCreate(&ev) != cudaSuccess) return fail(BT_ERR_CUDA);
  if (c->cfg.kernel_timing)
    for (auto& ev : c->kev)
      if (cudaEventCreate(&ev) != cudaSuccess) return fail(BT_ERR_CUDA);
  if ((e = uploadScene(c, scene, kd))) return fail(e);
  // Sub-beam queues: three of `capacity` 64-byte records.  Default 2^25
  // records (2 GiB each), at most 10% of the free memory.  Admission
  // reserves a root's whole budget of queue slots, so the capacity bounds
  // the roots in flight: primary tiles (budget 4096) over dense meshes need
  // 2^25 to admit 1024^2 at 8 x 8 tiles at once (2^23 left them to four
  // waves of admission and 1.3-1.8x the time; soft roots of budget 128 are
  // not bound by it).
  int64_t cap = c->cfg.capacity;
  if (cap <= 0) {
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    cap = std::min<int64_t>(int64_t(1) << 25, int64_t(fr / 10 / (3 * sizeof(SubBeam))));
  }
  cap = std::max<int64_t>(cap, 1024);
  cap = std::min<int64_t>(cap, int64_t(1) << 30);
  c->capacity = int(cap);
  if ((e = devAlloc(&c->dQ[0], size_t(cap))) || (e = devAlloc(&c->dQ[1], size_t(cap))) ||
      (e = devAlloc(&c->dQ[2], size_t(cap))) || (e = devAlloc(&c->dCtr, 1)) || (e = devAlloc(&c->dStats, kNumStats)) ||
      (e = devAlloc(&c->dKillCount, 1)))
    return fail(e);
  *out = c;
  return BT_OK;
}

int bt_gpu_destroy(bt_gpu_ctx* c) {
  if (!c) return BT_OK;
  if (c->serving) btserve::stop(c);  // the serving threads and their lanes first
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (!c->ownsScene) {  // a serving lane: the scene arrays are its parent's
    c->dNode = nullptr;
    c->dBox = nullptr;
    c->dParent = nullptr;
    c->dRef = nullptr;
    c->dTriNV = nullptr;
  }
  void* ptrs[] = {c->dNode, c->dBox, c->dParent, c->dRef, c->dTriNV, c->dQ[0], c->dQ[1], c->dQ[2], c->dCtr, c->dStats,
                  c->dRoots, c->dLive, c->dResv, c->dState, c->dAttempt, c->dList[0], c->dList[1], c->dMiss, c->dG,
                  c->dShade,
                  c->dKillCount, c->dOx, c->dOy, c->dOarea, c->dOn, c->dOtri, c->dOroot, c->dOatt, c->dPixTri,
                  c->dPixX, c->dPixN, c->dVis, c->dE, c->dEu, c->dJobs, c->dJobStart, c->dHx, c->dHy, c->dHn,
                  c->dHt, c->dHitCount, c->dFlag, c->dRanges, c->dJobCounts, c->dKx, c->dKy, c->dKarea,
                  c->dKn, c->dKtri, c->dKroot, c->dKeepBlocks};
  for (void* q : ptrs)
    if (q) cudaFree(q);
  for (auto& g : c->graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  for (auto& ev : c->ev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : c->rev)
    if (ev) cudaEventDestroy(ev);
  for (auto& ev : c->kev)
    if (ev) cudaEventDestroy(ev);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return BT_OK;
}

int bt_gpu_add_scene(bt_gpu_ctx* c, const bt_scene_desc* scene, const bt_kd_desc* kd, int32_t* scene_id) {
  if (!c || !scene || !kd || scene->num_tris <= 0 || kd->num_nodes <= 0) {
    setErr("bt_gpu_add_scene: empty scene or tree");
    return BT_ERR_INVALID;
  }
  if (!c->ownsScene) {
    setErr("bt_gpu_add_scene: add scenes to the context itself, not to a serving lane");
    return BT_ERR_INVALID;
  }
  // serving lanes read the arrays being replaced: wait until none works
  std::unique_lock<std::shared_mutex> lk(c->sceneLock);
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));  // nothing in flight reads the arrays being replaced
  const int e = uploadScene(c, scene, kd);
  if (e) return e;
  if (scene_id) *scene_id = int32_t(c->pool.size() - 1);
  return BT_OK;
}

int bt_gpu_primary_rays_device(bt_gpu_ctx* c, const bt_camera* cam, int32_t* dTri, float* dX, float* dN) {
  if (!c || !camOk(cam) || !dTri || !dX || !dN) return BT_ERR_INVALID;
  CK(cudaSetDevice(c->device));
  dim3 bs(16, 8), gs((cam->W + 15) / 16, (cam->H + 7) / 8);
  primaryRaysKernel<<<gs, bs, 0, c->stream>>>(c->s, *cam, dTri, dX, dN);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
  return BT_OK;
}

int bt_gpu_soft(bt_gpu_ctx* c, const bt_camera* cam, const bt_area_light* L, const bt_soft_opts* o, int32_t* tri,
                float* vis, float* E, float* Eu, bt_run_info* info) {
  if (!c || !camOk(cam) || !L) {
    setErr("bt_gpu_soft: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  const int64_t np = int64_t(cam->W) * cam->H;
  int e = ensurePix(c, np);
  if (e) return e;
  if (info) memset(info, 0, sizeof *info);
  CK(cudaEventRecord(c->ev[0], c->stream));
  const bool fused = c->cfg.fuse_primary != 0;
  if (!fused) {
    dim3 bs(16, 8), gs((cam->W + 15) / 16, (cam->H + 7) / 8);
    primaryRaysKernel<<<gs, bs, 0, c->stream>>>(c->s, *cam, c->dPixTri, c->dPixX, c->dPixN);
    CK(cudaGetLastError());
    if (info) info->launches++;
  }
  CK(cudaEventRecord(c->ev[1], c->stream));
  e = fused ? softCore(c, L, o, np, cam, c->dPixTri, c->dPixX, c->dPixN, c->dVis, c->dE, c->dEu, info, c->dPixTri,
                       c->dPixX, c->dPixN)
            : softCore(c, L, o, np, cam, c->dPixTri, c->dPixX, c->dPixN, c->dVis, c->dE, c->dEu, info);
  if (e) return e;
  CK(cudaEventRecord(c->ev[2], c->stream));
  if (tri) CK(cudaMemcpyAsync(tri, c->dPixTri, sizeof(int32_t) * np, cudaMemcpyDeviceToHost, c->stream));
  if (vis) CK(cudaMemcpyAsync(vis, c->dVis, sizeof(float) * np, cudaMemcpyDeviceToHost, c->stream));
  if (E) CK(cudaMemcpyAsync(E, c->dE, sizeof(float) * np, cudaMemcpyDeviceToHost, c->stream));
  if (Eu) CK(cudaMemcpyAsync(Eu, c->dEu, sizeof(float) * np, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaEventRecord(c->ev[3], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (info) {
    float a = 0, b = 0, t = 0;
    cudaEventElapsedTime(&a, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&b, c->ev[1], c->ev[2]);
    cudaEventElapsedTime(&t, c->ev[0], c->ev[3]);
    info->ms_primary = a;
    info->ms_trace = b;
    info->ms_total = t;
  }
  return BT_OK;
}

int bt_gpu_soft_device(bt_gpu_ctx* c, const bt_camera* cam, const bt_area_light* L, const bt_soft_opts* o,
                       int32_t* dTri, float* dVis, float* dE, float* dEu, bt_run_info* info) {
  if (!c || !camOk(cam) || !L || !dTri) {
    setErr("bt_gpu_soft_device: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  const int64_t np = int64_t(cam->W) * cam->H;
  int e = ensurePix(c, np);
  if (e) return e;
  if (info) memset(info, 0, sizeof *info);
  CK(cudaEventRecord(c->ev[0], c->stream));
  const bool fused = c->cfg.fuse_primary != 0;
  if (!fused) {
    dim3 bs(16, 8), gs((cam->W + 15) / 16, (cam->H + 7) / 8);
    primaryRaysKernel<<<gs, bs, 0, c->stream>>>(c->s, *cam, dTri, c->dPixX, c->dPixN);
    CK(cudaGetLastError());
    if (info) info->launches++;
  }
  CK(cudaEventRecord(c->ev[1], c->stream));
  e = fused ? softCore(c, L, o, np, cam, dTri, c->dPixX, c->dPixN, dVis, dE, dEu, info, dTri, c->dPixX, c->dPixN)
            : softCore(c, L, o, np, cam, dTri, c->dPixX, c->dPixN, dVis, dE, dEu, info);
  if (e) return e;
  CK(cudaEventRecord(c->ev[2], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (info) {
    float a = 0, b = 0;
    cudaEventElapsedTime(&a, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&b, c->ev[1], c->ev[2]);
    info->ms_primary = a;
    info->ms_trace = b;
    info->ms_total = a + b;
  }
  return BT_OK;
}

int bt_gpu_batch_soft(bt_gpu_ctx* c, int32_t n, const bt_soft_job* jobs, bt_run_info* info) {
  if (!c || n < 0 || (n > 0 && !jobs)) {
    setErr("bt_gpu_batch_soft: bad arguments");
    return BT_ERR_INVALID;
  }
  int64_t totPix = 0;
  for (int j = 0; j < n; ++j) {
    if (!camOk(&jobs[j].cam)) {
      setErr("bt_gpu_batch_soft: job %d has a bad camera", j);
      return BT_ERR_INVALID;
    }
    if (jobs[j].scene < 0 || size_t(jobs[j].scene) >= c->pool.size()) {
      setErr("bt_gpu_batch_soft: job %d names scene %d of %zu", j, jobs[j].scene, c->pool.size());
      return BT_ERR_INVALID;
    }
    totPix += int64_t(jobs[j].cam.W) * jobs[j].cam.H;
  }
  CK(cudaSetDevice(c->device));
  if (info) memset(info, 0, sizeof *info);
  if (n == 0) return BT_OK;
  int e = ensurePix(c, totPix);
  if (e) return e;
  if (c->jobCap < n) {
    cudaFree(c->dJobs);
    cudaFree(c->dJobStart);
    c->jobCap = 0;
    if ((e = devAlloc(&c->dJobs, size_t(n))) || (e = devAlloc(&c->dJobStart, size_t(n) + 1))) return e;
    c->jobCap = n;
  }
  std::vector<AppParams> hj(static_cast<size_t>(n));
  std::vector<int32_t> start(static_cast<size_t>(n) + 1);
  int64_t R = 0, off = 0;
  int anyExact = 0;
  CK(cudaEventRecord(c->ev[0], c->stream));
  for (int j = 0; j < n; ++j) {
    const bt_soft_job& J = jobs[j];
    const bt_camera& cam = J.cam;
    const PoolScene& ps = c->pool[size_t(J.scene)];
    int32_t* tri = J.d_tri ? J.d_tri : c->dPixTri + off;
    SceneDev sj = c->s;
    sj.bounds = ps.box;
    sj.rootNode = ps.rootNode;
    dim3 bs(16, 8), gs((cam.W + 15) / 16, (cam.H + 7) / 8);
    primaryRaysKernel<<<gs, bs, 0, c->stream>>>(sj, cam, tri, c->dPixX + 3 * off, c->dPixN + 3 * off);
    AppParams a = baseApp(c, &cam);
    a.rootBox = ps.box;
    a.rootNode = ps.rootNode;
    a.triBase = ps.triBase;
    a.Lc = mk(J.light.c[0], J.light.c[1], J.light.c[2]);
    a.LU = mk(J.light.U[0], J.light.U[1], J.light.U[2]);
    a.LV = mk(J.light.V[0], J.light.V[1], J.light.V[2]);
    a.offset = J.opts.offset > 0 ? J.opts.offset : ps.offset;
    a.exact = J.opts.exact;
    anyExact |= J.opts.exact;
    a.pixTri = tri;
    a.pixX = c->dPixX + 3 * off;
    a.pixN = c->dPixN + 3 * off;
    a.vis = J.d_vis;
    a.E = J.d_E;
    a.Eu = J.d_Eu;
    a.tiled = 1;
    a.tilesX = (cam.W + 7) / 8;
    a.shade = c->dShade;
    hj[size_t(j)] = a;
    start[size_t(j)] = int32_t(R);
    R += int64_t(a.tilesX) * ((cam.H + 3) / 4) * 32;
    off += int64_t(cam.W) * cam.H;
    if (R > 0x7fffffff) {
      setErr("bt_gpu_batch_soft: more than 2^31 roots in one batch");
      return BT_ERR_TOO_LARGE;
    }
  }
  start[size_t(n)] = int32_t(R);
  CK(cudaGetLastError());
  if (info) info->launches += n;
  CK(cudaMemcpyAsync(c->dJobs, hj.data(), sizeof(AppParams) * size_t(n), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->dJobStart, start.data(), sizeof(int32_t) * (size_t(n) + 1), cudaMemcpyHostToDevice,
                     c->stream));
  CK(cudaEventRecord(c->ev[1], c->stream));
  AppParams batch = baseApp(c, nullptr);
  batch.exact = anyExact;
  batch.jobs = c->dJobs;
  batch.jobStart = c->dJobStart;
  batch.numJobs = n;
  e = runRoots<kAppSoft>(c, batch, int(R), c->cfg.budget, info);
  if (e) return e;
  for (int j = 0; j < n; ++j) {
    AppParams a = hj[size_t(j)];
    a.missFx = c->dMiss + start[size_t(j)];
    a.gFx = c->dG + start[size_t(j)];
    const int Rj = start[size_t(j) + 1] - start[size_t(j)];
    softFinalizeKernel<<<(Rj + 255) / 256, 256, 0, c->stream>>>(a, c->dState + start[size_t(j)], Rj);
    // triangle ids of the pool back to the job's scene
    const int64_t np = int64_t(jobs[j].cam.W) * jobs[j].cam.H;
    if (a.triBase != 0 && jobs[j].d_tri)
      rebaseKernel<<<int((np + 255) / 256), 256, 0, c->stream>>>(jobs[j].d_tri, np, a.triBase);
  }
  CK(cudaGetLastError());
  if (info) info->launches += n;
  CK(cudaEventRecord(c->ev[2], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (info) {
    float ta = 0, tb = 0;
    cudaEventElapsedTime(&ta, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&tb, c->ev[1], c->ev[2]);
    info->ms_primary = ta;
    info->ms_trace = tb;
    info->ms_total = ta + tb;
  }
  return BT_OK;
}

int bt_gpu_primary_rays(bt_gpu_ctx* c, const bt_camera* cam, int32_t* tri, float* X, float* N) {
  if (!c || !camOk(cam) || !tri || !X || !N) {
    setErr("bt_gpu_primary_rays: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  const int64_t np = int64_t(cam->W) * cam->H;
  int e = ensurePix(c, np);
  if (e) return e;
  dim3 bs(16, 8), gs((cam->W + 15) / 16, (cam->H + 7) / 8);
  primaryRaysKernel<<<gs, bs, 0, c->stream>>>(c->s, *cam, c->dPixTri, c->dPixX, c->dPixN);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(tri, c->dPixTri, sizeof(int32_t) * np, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(X, c->dPixX, sizeof(float) * 3 * np, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(N, c->dPixN, sizeof(float) * 3 * np, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BT_OK;
}

int bt_gpu_soft_points_device(bt_gpu_ctx* c, const bt_area_light* L, const bt_soft_opts* o, int64_t n,
                              const int32_t* dTri, const float* dX, const float* dN, float* dVis, float* dE, float* dEu,
                              bt_run_info* info) {
  if (!c || !L || n < 0 || n > 0x7fffffff || (n > 0 && (!dTri || !dX || !dN))) {
    setErr("bt_gpu_soft_points_device: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  if (info) memset(info, 0, sizeof *info);
  CK(cudaEventRecord(c->ev[1], c->stream));
  int e = softCore(c, L, o, n, nullptr, dTri, dX, dN, dVis, dE, dEu, info);
  if (e) return e;
  CK(cudaEventRecord(c->ev[2], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (info) {
    float b = 0;
    cudaEventElapsedTime(&b, c->ev[1], c->ev[2]);
    info->ms_trace = b;
    info->ms_total = b;
  }
  return BT_OK;
}

int bt_gpu_soft_points(bt_gpu_ctx* c, const bt_area_light* L, const bt_soft_opts* o, int64_t n, const int32_t* tri,
                       const float* X, const float* N, float* vis, float* E, float* Eu, bt_run_info* info) {
  if (!c || !L || n < 0 || (n > 0 && (!tri || !X || !N))) {
    setErr("bt_gpu_soft_points: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  int e = ensurePix(c, std::max<int64_t>(n, 1));
  if (e) return e;
  if (n > 0) {
    CK(cudaMemcpyAsync(c->dPixTri, tri, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->dPixX, X, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(c->dPixN, N, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, c->stream));
  }
  e = bt_gpu_soft_points_device(c, L, o, n, c->dPixTri, c->dPixX, c->dPixN, c->dVis, c->dE, c->dEu, info);
  if (e) return e;
  if (n > 0) {
    if (vis) CK(cudaMemcpyAsync(vis, c->dVis, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    if (E) CK(cudaMemcpyAsync(E, c->dE, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    if (Eu) CK(cudaMemcpyAsync(Eu, c->dEu, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
  }
  CK(cudaStreamSynchronize(c->stream));
  return BT_OK;
}

}  // extern "C"

namespace {

// Copies the polygons of roots that finished in their last attempt to the
// host (downloadPolys, cuda/wavefront.cu:766-783).
int ensureKeep(bt_gpu_ctx* c, int64_t n, int blocks) {
  if (c->keepBlocksCap < blocks + 1) {
    cudaFree(c->dKeepBlocks);
    c->keepBlocksCap = 0;
    int e = devAlloc(&c->dKeepBlocks, size_t(blocks + 1));
    if (e) return e;
    c->keepBlocksCap = blocks + 1;
  }
  if (c->keepCap >= n) return BT_OK;
  cudaFree(c->dKx);
  cudaFree(c->dKy);
  cudaFree(c->dKarea);
  cudaFree(c->dKn);
  cudaFree(c->dKtri);
  cudaFree(c->dKroot);
  c->keepCap = 0;
  int e;
  if ((e = devAlloc(&c->dKx, size_t(4 * n))) || (e = devAlloc(&c->dKy, size_t(4 * n))) ||
      (e = devAlloc(&c->dKarea, size_t(n))) || (e = devAlloc(&c->dKn, size_t(n))) ||
      (e = devAlloc(&c->dKtri, size_t(n))) || (e = devAlloc(&c->dKroot, size_t(n))))
    return e;
  c->keepCap = n;
  return BT_OK;
}

// The polygons of the roots' final attempts (of the first `produced` output
// records) into the caller's host buffers, in output order: compacted on
// the device, then copied straight into out (its first out->cap entries);
// *count = all kept polygons.
int downloadPolys(bt_gpu_ctx* c, int64_t produced, bt_polys* out, int64_t* count) {
  const int64_t n = std::min<int64_t>(produced, c->outCap);
  *count = 0;
  if (n <= 0) return BT_OK;
  const int64_t nb64 = (n + kKeepBlock - 1) / kKeepBlock;
  if (nb64 > INT_MAX - 1) {
    setErr("too many output polygons (%lld)", (long long)n);
    return BT_ERR_TOO_LARGE;
  }
  const int nb = int(nb64);
  int e = ensureKeep(c, n, nb);
  if (e) return e;
  keepCountKernel<<<nb, kKeepBlock, 0, c->stream>>>(c->dOroot, c->dOatt, n, c->dState, c->dAttempt,
                                                    c->dKeepBlocks);
  keepScanKernel<<<1, kKeepBlock, 0, c->stream>>>(c->dKeepBlocks, nb);
  KeepOut k{reinterpret_cast<float4*>(c->dKx), reinterpret_cast<float4*>(c->dKy), c->dKarea, c->dKn, c->dKtri,
            c->dKroot};
  keepWriteKernel<<<nb, kKeepBlock, 0, c->stream>>>(reinterpret_cast<const float4*>(c->dOx),
                                                    reinterpret_cast<const float4*>(c->dOy), c->dOarea, c->dOn,
                                                    c->dOtri, c->dOroot, c->dOatt, n, c->dState, c->dAttempt,
                                                    c->dKeepBlocks, k);
  CK(cudaGetLastError());
  int total = 0;
  CK(cudaMemcpyAsync(&total, c->dKeepBlocks + nb, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  const int64_t m = std::min<int64_t>(total, std::max<int64_t>(out->cap, 0));
  if (m > 0) {
    CK(cudaMemcpyAsync(out->x, c->dKx, sizeof(float) * 4 * m, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(out->y, c->dKy, sizeof(float) * 4 * m, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(out->n, c->dKn, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(out->tri, c->dKtri, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(out->area, c->dKarea, sizeof(float) * m, cudaMemcpyDeviceToHost, c->stream));
    if (out->root) CK(cudaMemcpyAsync(out->root, c->dKroot, sizeof(int32_t) * m, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
  *count = total;
  return BT_OK;
}

int ensureHits(bt_gpu_ctx* c, int64_t n) {
  if (!c->dHitCount) {
    int e = devAlloc(&c->dHitCount, 1);
    if (e) return e;
  }
  if (c->hitCap >= n) return BT_OK;
  cudaFree(c->dHx);
  cudaFree(c->dHy);
  cudaFree(c->dHn);
  cudaFree(c->dHt);
  c->hitCap = 0;
  int e;
  if ((e = devAlloc(&c->dHx, size_t(4 * n))) || (e = devAlloc(&c->dHy, size_t(4 * n))) ||
      (e = devAlloc(&c->dHn, size_t(n))) || (e = devAlloc(&c->dHt, size_t(n))))
    return e;
  c->hitCap = n;
  return BT_OK;
}

int ensureFlag(bt_gpu_ctx* c, int64_t n) {
  if (c->flagCap >= n) return BT_OK;
  cudaFree(c->dFlag);
  c->flagCap = 0;
  int e = devAlloc(&c->dFlag, size_t(n));
  if (e) return e;
  c->flagCap = n;
  return BT_OK;
}

void addInfo(bt_run_info* a, const bt_run_info& b) {
  a->kd_steps += b.kd_steps;
  a->leaf_visits += b.leaf_visits;
  a->tri_tests += b.tri_tests;
  a->hits += b.hits;
  a->splits += b.splits;
  a->beams += b.beams;
  a->root_beams += b.root_beams;
  a->presplit_beams += b.presplit_beams;
  a->five_splits += b.five_splits;
  a->climbs += b.climbs;
  a->dropped_area += b.dropped_area;
  a->ms_round += b.ms_round;
  a->launches += b.launches;
  a->round_launches += b.round_launches;
  a->passes += b.passes;
  a->retried_roots += b.retried_roots;
  a->overflow_roots += b.overflow_roots;
  a->yields += b.yields;
  a->max_spill = std::max(a->max_spill, b.max_spill);
  a->roots += b.roots;
  a->rounds += b.rounds;
  a->tail_rounds += b.tail_rounds;
  a->ms_kernel_trace += b.ms_kernel_trace;
}

// Primary visibility roots (tile x tile pixels) through the engine; on
// return the visible polygons are in the output buffers (*produced of them,
// filtered by attempt tags) and the roots' state in dState/dAttempt.
int runPrimary(bt_gpu_ctx* c, const bt_camera* cam, int cull, int tile, bt_run_info* info, int64_t* produced,
               int* Rout) {
  const int tilesW = (cam->W + tile - 1) / tile, tilesH = (cam->H + tile - 1) / tile;
  const int R = tilesW * tilesH;
  int64_t cap = std::max<int64_t>(int64_t(1) << 16, int64_t(cam->W) * cam->H * 2);
  for (;;) {
    int e = ensureOut(c, cap);
    if (e) return e;
    AppParams a = baseApp(c, cam);
    a.tile = tile;
    a.tilesW = tilesW;
    a.cull = cull ? 1 : 0;
    bt_run_info ri;
    memset(&ri, 0, sizeof ri);
    e = runRoots<kAppPrimary>(c, a, R, c->cfg.primary_budget, &ri);
    if (e) return e;
    Counters hc;
    CK(cudaMemcpyAsync(&hc, c->dCtr, sizeof hc, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (hc.outCount > c->outCap) {
      cap = int64_t(hc.outCount) + hc.outCount / 4;
      continue;
    }
    if (info) addInfo(info, ri);
    *produced = hc.outCount;
    *Rout = R;
    return BT_OK;
  }
}

}  // namespace

extern "C" {

int bt_gpu_primary(bt_gpu_ctx* c, const bt_camera* cam, int32_t cull, int32_t tile, bt_polys* out, int64_t* count,
                   bt_run_info* info) {
  if (!c || !camOk(cam) || tile <= 0 || !out || !count) {
    setErr("bt_gpu_primary: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  if (info) memset(info, 0, sizeof *info);
  const int tilesW = (cam->W + tile - 1) / tile, tilesH = (cam->H + tile - 1) / tile;
  const int R = tilesW * tilesH;
  int64_t cap = std::max<int64_t>(int64_t(1) << 16, int64_t(cam->W) * cam->H * 2);
  for (;;) {
    int e = ensureOut(c, cap);
    if (e) return e;
    AppParams a = baseApp(c, cam);
    a.tile = tile;
    a.tilesW = tilesW;
    a.cull = cull ? 1 : 0;
    CK(cudaEventRecord(c->ev[1], c->stream));
    e = runRoots<kAppPrimary>(c, a, R, c->cfg.primary_budget, info);
    if (e) return e;
    CK(cudaEventRecord(c->ev[2], c->stream));
    Counters hc;
    CK(cudaMemcpyAsync(&hc, c->dCtr, sizeof hc, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (hc.outCount > c->outCap) {
      cap = int64_t(hc.outCount) + hc.outCount / 4;
      continue;
    }
    if (info) {
      float b = 0;
      cudaEventElapsedTime(&b, c->ev[1], c->ev[2]);
      info->ms_trace = b;
      info->ms_total = b;
    }
    c->lastProduced = hc.outCount;
    return downloadPolys(c, hc.outCount, out, count);
  }
}

int bt_gpu_point(bt_gpu_ctx* c, const bt_camera* cam, const bt_polys* hits, int64_t nh, const float* light,
                 bt_polys* out, int64_t* count, bt_run_info* info) {
  if (!c || !camOk(cam) || !hits || nh < 0 || nh > 0x7fffffff || !light || !out || !count) {
    setErr("bt_gpu_point: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  if (info) memset(info, 0, sizeof *info);
  *count = 0;
  if (nh == 0) return BT_OK;
  for (int64_t i = 0; i < nh; ++i)
    if (hits->tri[i] >= c->numTris || hits->n[i] < 3 || hits->n[i] > 4) {
      setErr("bt_gpu_point: hit polygon %lld is invalid", (long long)i);
      return BT_ERR_INVALID;
    }
  int e = ensureHits(c, nh);
  if (e) return e;
  float *dhx = c->dHx, *dhy = c->dHy;
  int32_t *dhn = c->dHn, *dht = c->dHt;
  CK(cudaMemcpyAsync(dhx, hits->x, sizeof(float) * 4 * nh, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(dhy, hits->y, sizeof(float) * 4 * nh, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(dhn, hits->n, sizeof(int32_t) * nh, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(dht, hits->tri, sizeof(int32_t) * nh, cudaMemcpyHostToDevice, c->stream));
  int64_t cap = std::max<int64_t>(int64_t(1) << 16, nh * 4);
  for (;;) {
    if ((e = ensureOut(c, cap))) return e;
    AppParams a = baseApp(c, cam);
    a.pointLight = mk(light[0], light[1], light[2]);
    a.hx = dhx;
    a.hy = dhy;
    a.hn = dhn;
    a.htri = dht;
    CK(cudaEventRecord(c->ev[1], c->stream));
    e = runRoots<kAppPoint>(c, a, int(nh), c->cfg.budget, info);
    if (e) return e;
    CK(cudaEventRecord(c->ev[2], c->stream));
    Counters hc;
    CK(cudaMemcpyAsync(&hc, c->dCtr, sizeof hc, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (hc.outCount > c->outCap) {
      cap = int64_t(hc.outCount) + hc.outCount / 4;
      continue;
    }
    if (info) {
      float b = 0;
      cudaEventElapsedTime(&b, c->ev[1], c->ev[2]);
      info->ms_trace = b;
      info->ms_total = b;
    }
    c->lastProduced = hc.outCount;
    return downloadPolys(c, hc.outCount, out, count);
  }
}

int bt_gpu_last_polys(bt_gpu_ctx* c, bt_polys* out, int64_t* count) {
  if (!c || !out || !count) {
    setErr("bt_gpu_last_polys: bad arguments");
    return BT_ERR_INVALID;
  }
  if (c->lastProduced < 0) {
    setErr("bt_gpu_last_polys: no polygons kept (the last engine call was not bt_gpu_primary / bt_gpu_point)");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  return downloadPolys(c, c->lastProduced, out, count);
}

int bt_gpu_raster(bt_gpu_ctx* c, const bt_camera* cam, const bt_polys* prim, int64_t np, const bt_polys* shadow,
                  int64_t ns, int32_t* tri, uint8_t* flag) {
  if (!c || !camOk(cam) || np < 0 || ns < 0 || (np > 0 && !prim) || (ns > 0 && !shadow)) {
    setErr("bt_gpu_raster: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  const int64_t npix = int64_t(cam->W) * cam->H;
  const int64_t m = std::max(np, ns);
  int e;
  if ((e = ensureHits(c, std::max<int64_t>(m, 1))) || (e = ensurePix(c, npix)) || (e = ensureFlag(c, npix))) return e;
  float *dx = c->dHx, *dy = c->dHy;
  int32_t *dn = c->dHn, *dt = c->dHt, *dtri = c->dPixTri;
  uint8_t* dflag = c->dFlag;
  fillKernel<<<(npix + 255) / 256, 256, 0, c->stream>>>(dtri, npix, -1);
  CK(cudaMemsetAsync(dflag, 0, size_t(npix), c->stream));
  for (int pass = 0; pass < 2; ++pass) {
    const bt_polys* P = pass == 0 ? prim : shadow;
    const int64_t n = pass == 0 ? np : ns;
    if (n == 0) continue;
    CK(cudaMemcpyAsync(dx, P->x, sizeof(float) * 4 * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dy, P->y, sizeof(float) * 4 * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dn, P->n, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(dt, P->tri, sizeof(int32_t) * n, cudaMemcpyHostToDevice, c->stream));
    rasterKernel<<<int((n + 127) / 128), 128, 0, c->stream>>>(*cam, dx, dy, dn, dt, n, pass, dtri, dflag);
    CK(cudaGetLastError());
  }
  if (tri) CK(cudaMemcpyAsync(tri, dtri, sizeof(int32_t) * npix, cudaMemcpyDeviceToHost, c->stream));
  if (flag) CK(cudaMemcpyAsync(flag, dflag, size_t(npix), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BT_OK;
}

int bt_gpu_primary_ids_device(bt_gpu_ctx* c, const bt_camera* cam, int32_t cull, int32_t tile, int32_t* d_tri,
                              bt_run_info* info) {
  if (!c || !camOk(cam) || tile <= 0 || !d_tri) {
    setErr("bt_gpu_primary_ids_device: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  if (info) memset(info, 0, sizeof *info);
  const int64_t npix = int64_t(cam->W) * cam->H;
  CK(cudaEventRecord(c->ev[0], c->stream));
  int64_t produced = 0;
  int R = 0;
  int e = runPrimary(c, cam, cull, tile, info, &produced, &R);
  if (e) return e;
  fillKernel<<<int((npix + 255) / 256), 256, 0, c->stream>>>(d_tri, npix, -1);
  if (produced > 0)
    rasterKernel<<<int((produced + 127) / 128), 128, 0, c->stream>>>(*cam, c->dOx, c->dOy, c->dOn, c->dOtri, produced,
                                                                     0, d_tri, nullptr, c->dOroot, c->dOatt,
                                                                     c->dState, c->dAttempt);
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[1], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (info) {
    float t = 0;
    cudaEventElapsedTime(&t, c->ev[0], c->ev[1]);
    info->ms_trace = info->ms_total = t;
    info->launches += 2;
  }
  return BT_OK;
}

int bt_gpu_point_mask_device(bt_gpu_ctx* c, const bt_camera* cam, int32_t cull, int32_t tile, const float* light,
                             int32_t* d_tri, uint8_t* d_mask, bt_run_info* info) {
  if (!c || !camOk(cam) || tile <= 0 || !light || !d_mask) {
    setErr("bt_gpu_point_mask_device: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  if (info) memset(info, 0, sizeof *info);
  const int64_t npix = int64_t(cam->W) * cam->H;
  CK(cudaEventRecord(c->ev[0], c->stream));
  int64_t produced = 0;
  int R = 0;
  int e = runPrimary(c, cam, cull, tile, info, &produced, &R);
  if (e) return e;
  if (d_tri) {
    fillKernel<<<int((npix + 255) / 256), 256, 0, c->stream>>>(d_tri, npix, -1);
    if (produced > 0)
      rasterKernel<<<int((produced + 127) / 128), 128, 0, c->stream>>>(*cam, c->dOx, c->dOy, c->dOn, c->dOtri,
                                                                       produced, 0, d_tri, nullptr, c->dOroot,
                                                                       c->dOatt, c->dState, c->dAttempt);
  }
  // the final hit polygons become the point-shadow roots
  if ((e = ensureHits(c, std::max<int64_t>(produced, 1)))) return e;
  CK(cudaMemsetAsync(c->dHitCount, 0, sizeof(int), c->stream));
  if (produced > 0)
    compactHitsKernel<<<int((produced + 255) / 256), 256, 0, c->stream>>>(
        c->dOx, c->dOy, c->dOn, c->dOtri, c->dOroot, c->dOatt, produced, c->dState, c->dAttempt, c->dHx, c->dHy,
        c->dHn, c->dHt, c->dHitCount);
  CK(cudaMemsetAsync(d_mask, 0, size_t(npix), c->stream));
  int nh = 0;
  CK(cudaMemcpyAsync(&nh, c->dHitCount, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (nh > 0) {
    int64_t cap = std::max<int64_t>(int64_t(1) << 16, int64_t(nh) * 4);
    Counters hc;
    for (;;) {
      if ((e = ensureOut(c, cap))) return e;
      AppParams a = baseApp(c, cam);
      a.pointLight = mk(light[0], light[1], light[2]);
      a.hx = c->dHx;
      a.hy = c->dHy;
      a.hn = c->dHn;
      a.htri = c->dHt;
      bt_run_info ri;
      memset(&ri, 0, sizeof ri);
      e = runRoots<kAppPoint>(c, a, nh, c->cfg.budget, &ri);
      if (e) return e;
      CK(cudaMemcpyAsync(&hc, c->dCtr, sizeof hc, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      if (hc.outCount > c->outCap) {
        cap = int64_t(hc.outCount) + hc.outCount / 4;
        continue;
      }
      if (info) addInfo(info, ri);
      break;
    }
    if (hc.outCount > 0)
      rasterKernel<<<int((hc.outCount + 127) / 128), 128, 0, c->stream>>>(
          *cam, c->dOx, c->dOy, c->dOn, c->dOtri, hc.outCount, 1, nullptr, d_mask, c->dOroot, c->dOatt, c->dState,
          c->dAttempt);
  }
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->ev[1], c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (info) {
    float t = 0;
    cudaEventElapsedTime(&t, c->ev[0], c->ev[1]);
    info->ms_trace = info->ms_total = t;
    info->launches += 4;
  }
  return BT_OK;
}

int bt_gpu_primary_ids(bt_gpu_ctx* c, const bt_camera* cam, int32_t cull, int32_t tile, int32_t* tri,
                       bt_run_info* info) {
  if (!c || !camOk(cam) || !tri) {
    setErr("bt_gpu_primary_ids: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  const int64_t npix = int64_t(cam->W) * cam->H;
  int e = ensurePix(c, npix);
  if (e) return e;
  if ((e = bt_gpu_primary_ids_device(c, cam, cull, tile, c->dPixTri, info))) return e;
  CK(cudaMemcpyAsync(tri, c->dPixTri, sizeof(int32_t) * npix, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BT_OK;
}

int bt_gpu_point_mask(bt_gpu_ctx* c, const bt_camera* cam, int32_t cull, int32_t tile, const float* light, int32_t* tri,
                      uint8_t* mask, bt_run_info* info) {
  if (!c || !camOk(cam) || !light || !mask) {
    setErr("bt_gpu_point_mask: bad arguments");
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  const int64_t npix = int64_t(cam->W) * cam->H;
  int e;
  if ((e = ensurePix(c, npix)) || (e = ensureFlag(c, npix))) return e;
  if ((e = bt_gpu_point_mask_device(c, cam, cull, tile, light, tri ? c->dPixTri : nullptr, c->dFlag, info))) return e;
  if (tri) CK(cudaMemcpyAsync(tri, c->dPixTri, sizeof(int32_t) * npix, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(mask, c->dFlag, size_t(npix), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return BT_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving lanes: the engine side of bt_gpu_submit / bt_gpu_poll (serve.cpp).
//
// A lane is a bt_gpu_ctx that views its parent's scene pool (it owns no
// scene array) and owns a stream, sub-beam queues, root arrays and a pixel
// arena, so that lanes run side by side on the device.  A soft lane runs
// streaming engine runs: the soft-shadow jobs of a run share the rounds as
// in bt_gpu_batch_soft, jobs that arrive while the run goes on are folded
// in between batches of rounds (their roots appended to the root list,
// their parameters to the job table), and a job whose roots are all done is
// finalised and handed back at once while the run goes on.  Jobs with a
// root abandoned over budget wait for the retry passes at the run's end.
// ---------------------------------------------------------------------------

namespace {

// For the jobs named in `ranges` (root ranges [a, b), one pair per
// blockIdx.y): counts[2j] = roots still live, counts[2j + 1] = roots
// abandoned over budget.
__global__ void jobStatusKernel(const int32_t* live, const int32_t* state, const int32_t* ranges, int* counts) {
  const int j = blockIdx.y;
  const int a = ranges[2 * j], b = ranges[2 * j + 1];
  int busy = 0, killed = 0;
  for (int k = a + int(blockIdx.x * blockDim.x + threadIdx.x); k < b; k += int(gridDim.x * blockDim.x)) {
    busy += live[k] != 0;
    killed += state[k] == kRootKilled;
  }
  for (int o = 16; o > 0; o >>= 1) {
    busy += __shfl_down_sync(kFull, busy, o);
    killed += __shfl_down_sync(kFull, killed, o);
  }
  if (laneId() == 0) {
    if (busy) atomicAdd(&counts[2 * j], busy);
    if (killed) atomicAdd(&counts[2 * j + 1], killed);
  }
}

// Soft-shadow roots of a W x H job (8 x 4 pixel tiles of 32 roots).
int64_t softRoots(const bt_camera& cam) { return int64_t((cam.W + 7) / 8) * ((cam.H + 3) / 4) * 32; }

}  // namespace

namespace btserve {

int deviceOf(const bt_gpu_ctx* c) { return c->device; }
void useDevice(const bt_gpu_ctx* c) { cudaSetDevice(c->device); }
std::shared_mutex& sceneLock(bt_gpu_ctx* c) { return c->sceneLock; }
void*& servingState(bt_gpu_ctx* c) { return c->serving; }
const char* lastError() { return g_err; }
int sceneCount(bt_gpu_ctx* c) { return int(c->pool.size()); }

int64_t sceneTris(bt_gpu_ctx* c, int32_t scene) {
  return scene >= 0 && size_t(scene) < c->pool.size() ? c->pool[size_t(scene)].numTris : 0;
}

int64_t sceneBytes(const bt_gpu_ctx* c) { return sceneDeviceBytes(c); }

int64_t laneBytes(const bt_gpu_ctx* c) {
  return 3 * int64_t(c->capacity) * int64_t(sizeof(SubBeam)) + int64_t(c->rootCap) * 68 + c->pixCap * 40 +
         c->outCap * 52 + c->hitCap * 40 + c->flagCap;
}

int64_t laneHighWater(const bt_gpu_ctx* c) { return 3 * c->queueHighWater * int64_t(sizeof(SubBeam)); }

void laneView(bt_gpu_ctx* lane) {
  const bt_gpu_ctx* p = lane->parent;
  lane->dNode = p->dNode;
  lane->dBox = p->dBox;
  lane->dParent = p->dParent;
  lane->dRef = p->dRef;
  lane->dTriNV = p->dTriNV;
  lane->s = p->s;
  lane->offset = p->offset;
  lane->numTris = p->numTris;
  lane->numRefs = p->numRefs;
  lane->pool = p->pool;
}

int laneCreate(bt_gpu_ctx* parent, int64_t capacity, int64_t pixels, int jobs, bt_gpu_ctx** out) {
  *out = nullptr;
  bt_gpu_ctx* c = new bt_gpu_ctx();
  c->cfg = parent->cfg;
  // A lane's launch parameters change with every request (camera, light,
  // folded roots), so a captured batch of rounds would never be replayed.
  c->cfg.graph_rounds = 0;
  c->device = parent->device;
  c->sms = parent->sms;
  c->parent = parent;
  c->ownsScene = false;
  auto fail = [&](int code) {
    bt_gpu_destroy(c);
    return code;
  };
  if (cudaSetDevice(c->device) != cudaSuccess) return fail(BT_ERR_CUDA);
  // Visibility lanes (no pixel arena) take the device's highest stream
  // priority: their CTAs are scheduled ahead of a long soft run's pending
  // ones, so a small primary or point request does not queue behind it.
  int prLeast = 0, prGreatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&prLeast, &prGreatest) != cudaSuccess) return fail(BT_ERR_CUDA);
  if (cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, pixels > 0 ? prLeast : prGreatest) !=
      cudaSuccess)
    return fail(BT_ERR_CUDA);
  for (auto& ev : c->ev)
    if (cudaEventCreate(&ev) != cudaSuccess) return fail(BT_ERR_CUDA);
  for (auto& ev : c->rev)
    if (cudaEventCreate(&ev) != cudaSuccess) return fail(BT_ERR_CUDA);
  {
    std::shared_lock<std::shared_mutex> lk(parent->sceneLock);
    laneView(c);
  }
  const int64_t cap = std::max<int64_t>(1024, std::min<int64_t>(capacity > 0 ? capacity : parent->capacity, 1 << 30));
  c->capacity = int(cap);
  int e;
  if ((e = devAlloc(&c->dQ[0], size_t(cap))) || (e = devAlloc(&c->dQ[1], size_t(cap))) ||
      (e = devAlloc(&c->dQ[2], size_t(cap))) || (e = devAlloc(&c->dCtr, 1)) || (e = devAlloc(&c->dStats, kNumStats)) ||
      (e = devAlloc(&c->dKillCount, 1)))
    return fail(e);
  if (pixels > 0) {
    // a soft lane: the pixel arena, roots for it (tiles round each job up),
    // the job table and the completion-check buffers
    jobs = std::max(jobs, 1);
    const int64_t roots = pixels + int64_t(jobs) * 4096;
    if (roots > 0x7fffffff) return fail(BT_ERR_TOO_LARGE);
    if ((e = ensurePix(c, pixels)) || (e = ensureRoots(c, size_t(roots))) || (e = devAlloc(&c->dJobs, size_t(jobs))) ||
        (e = devAlloc(&c->dJobStart, size_t(jobs) + 1)) || (e = devAlloc(&c->dRanges, 2 * size_t(jobs))) ||
        (e = devAlloc(&c->dJobCounts, 2 * size_t(jobs))))
      return fail(e);
    c->jobCap = jobs;
  }
  *out = c;
  return BT_OK;
}

void laneDestroy(bt_gpu_ctx* lane) { bt_gpu_destroy(lane); }

void laneBlocksPerSm(bt_gpu_ctx* lane, int blocks) { lane->cfg.blocks_per_sm = blocks; }

int laneVisibility(bt_gpu_ctx* c, int kind, int32_t scene, const bt_camera& cam, int32_t cull, int32_t tile,
                   const float* light, int32_t* tri, uint8_t* mask, bt_run_info* info) {
  if (scene < 0 || size_t(scene) >= c->pool.size() || !camOk(&cam)) {
    setErr("serving: bad scene %d or camera", scene);
    return BT_ERR_INVALID;
  }
  CK(cudaSetDevice(c->device));
  // render scene `scene` of the pool: its kd root, box and apex offset
  const PoolScene& ps = c->pool[size_t(scene)];
  c->s.bounds = ps.box;
  c->s.rootNode = ps.rootNode;
  c->offset = ps.offset;
  const int64_t npix = int64_t(cam.W) * cam.H;
  int e;
  if ((e = ensurePix(c, npix)) || (e = ensureFlag(c, npix))) return e;
  if (tile <= 0) tile = 16;
  if (kind == BT_REQ_PRIMARY_IDS)
    e = bt_gpu_primary_ids_device(c, &cam, cull, tile, c->dPixTri, info);
  else
    e = bt_gpu_point_mask_device(c, &cam, cull, tile, light, tri ? c->dPixTri : nullptr, c->dFlag, info);
  if (e) return e;
  if (tri && ps.triBase != 0)
    rebaseKernel<<<int((npix + 255) / 256), 256, 0, c->stream>>>(c->dPixTri, npix, ps.triBase);
  if (tri) CK(cudaMemcpyAsync(tri, c->dPixTri, sizeof(int32_t) * size_t(npix), cudaMemcpyDeviceToHost, c->stream));
  if (mask && kind != BT_REQ_PRIMARY_IDS)
    CK(cudaMemcpyAsync(mask, c->dFlag, size_t(npix), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (info && info->max_spill > c->queueHighWater) c->queueHighWater = info->max_spill;
  return BT_OK;
}

int laneSoftRun(bt_gpu_ctx* c, SoftFeed& feed, double foldMs, bt_run_info* info) {
  struct Job {
    uint64_t tag;
    StreamJob j;
    int64_t off;        // first pixel in the arena
    int32_t a, b;       // its roots
    int state;          // 0 running, 1 waiting for the retry passes, 2 handed back
  };
  std::vector<Job> jobs;
  std::vector<AppParams> hj;
  std::vector<int32_t> start(1, 0);
  int64_t off = 0, R = 0;
  int anyExact = 0;
  CK(cudaSetDevice(c->device));
  const auto t0 = std::chrono::steady_clock::now();
  auto ageMs = [&] { return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count(); };

  // Folds in the jobs the feed has for this run; returns how many, or a
  // negative error code.
  auto fold = [&]() -> int {
    const size_t n0 = jobs.size();
    StreamJob j;
    uint64_t tag = 0;
    while (int(jobs.size()) < c->jobCap && feed.next(j, tag, c->pixCap - off, int64_t(c->rootCap) - R)) {
      const PoolScene& ps = c->pool[size_t(j.scene)];
      const int64_t np = int64_t(j.cam.W) * j.cam.H, Rj = softRoots(j.cam);
      SceneDev sj = c->s;
      sj.bounds = ps.box;
      sj.rootNode = ps.rootNode;
      dim3 bs(16, 8), gs((j.cam.W + 15) / 16, (j.cam.H + 7) / 8);
      primaryRaysKernel<<<gs, bs, 0, c->stream>>>(sj, j.cam, c->dPixTri + off, c->dPixX + 3 * off,
                                                 c->dPixN + 3 * off);
      AppParams a = baseApp(c, &j.cam);
      a.rootBox = ps.box;
      a.rootNode = ps.rootNode;
      a.triBase = ps.triBase;
      a.Lc = mk(j.light.c[0], j.light.c[1], j.light.c[2]);
      a.LU = mk(j.light.U[0], j.light.U[1], j.light.U[2]);
      a.LV = mk(j.light.V[0], j.light.V[1], j.light.V[2]);
      a.offset = j.opts.offset > 0 ? j.opts.offset : ps.offset;
      a.exact = j.opts.exact;
      a.pixTri = c->dPixTri + off;
      a.pixX = c->dPixX + 3 * off;
      a.pixN = c->dPixN + 3 * off;
      a.vis = c->dVis + off;
      a.E = c->dE + off;
      a.Eu = c->dEu + off;
      a.tiled = 1;
      a.tilesX = (j.cam.W + 7) / 8;
      a.shade = c->dShade;
      hj.push_back(a);
      start.push_back(int32_t(R + Rj));
      jobs.push_back(Job{tag, j, off, int32_t(R), int32_t(R + Rj), 0});
      anyExact |= j.opts.exact;
      off += np;
      R += Rj;
    }
    const size_t added = jobs.size() - n0;
    if (added) {
      CK(cudaGetLastError());
      CK(cudaMemcpyAsync(c->dJobs + n0, &hj[n0], sizeof(AppParams) * added, cudaMemcpyHostToDevice, c->stream));
      CK(cudaMemcpyAsync(c->dJobStart + n0, &start[n0], sizeof(int32_t) * (added + 1), cudaMemcpyHostToDevice,
                         c->stream));
    }
    return int(added);
  };

  // Finalises job i into its host buffers and hands it back.
  auto handBack = [&](Job& J) -> int {
    AppParams a = hj[size_t(&J - jobs.data())];
    a.missFx = c->dMiss + J.a;
    a.gFx = c->dG + J.a;
    const int Rj = J.b - J.a;
    softFinalizeKernel<<<(Rj + 255) / 256, 256, 0, c->stream>>>(a, c->dState + J.a, Rj);
    const int64_t np = int64_t(J.j.cam.W) * J.j.cam.H;
    if (a.triBase != 0 && J.j.tri)
      rebaseKernel<<<int((np + 255) / 256), 256, 0, c->stream>>>(c->dPixTri + J.off, np, a.triBase);
    CK(cudaGetLastError());
    const size_t f4 = sizeof(float) * size_t(np);
    if (J.j.tri) CK(cudaMemcpyAsync(J.j.tri, c->dPixTri + J.off, f4, cudaMemcpyDeviceToHost, c->stream));
    if (J.j.vis) CK(cudaMemcpyAsync(J.j.vis, c->dVis + J.off, f4, cudaMemcpyDeviceToHost, c->stream));
    if (J.j.E) CK(cudaMemcpyAsync(J.j.E, c->dE + J.off, f4, cudaMemcpyDeviceToHost, c->stream));
    if (J.j.Eu) CK(cudaMemcpyAsync(J.j.Eu, c->dEu + J.off, f4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    J.state = 2;
    feed.finished(J.tag, BT_OK, "");
    return BT_OK;
  };

  // The running jobs whose roots are all admitted: those with every root
  // done are handed back; those with an abandoned root wait for the retries.
  std::vector<int32_t> ranges;
  std::vector<int> counts;
  std::vector<size_t> cand;
  auto settle = [&](int rootNext) -> int {
    cand.clear();
    ranges.clear();
    int32_t longest = 0;
    for (size_t i = 0; i < jobs.size(); ++i)
      if (jobs[i].state == 0 && jobs[i].b <= rootNext) {
        cand.push_back(i);
        ranges.push_back(jobs[i].a);
        ranges.push_back(jobs[i].b);
        longest = std::max(longest, jobs[i].b - jobs[i].a);
      }
    if (cand.empty()) return BT_OK;
    const size_t nc = cand.size();
    counts.assign(2 * nc, 0);
    CK(cudaMemcpyAsync(c->dRanges, ranges.data(), sizeof(int32_t) * 2 * nc, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemsetAsync(c->dJobCounts, 0, sizeof(int) * 2 * nc, c->stream));
    dim3 g(unsigned(std::min<int64_t>((longest + 255) / 256, 64)), unsigned(nc));
    jobStatusKernel<<<g, 256, 0, c->stream>>>(c->dLive, c->dState, c->dRanges, c->dJobCounts);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(counts.data(), c->dJobCounts, sizeof(int) * 2 * nc, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k < nc; ++k) {
      if (counts[2 * k] != 0) continue;
      Job& J = jobs[cand[k]];
      if (counts[2 * k + 1] != 0) {
        J.state = 1;
        continue;
      }
      const int e = handBack(J);
      if (e) return e;
    }
    return BT_OK;
  };

  auto failAll = [&](int e) {
    const std::string why = g_err;
    for (Job& J : jobs)
      if (J.state != 2) {
        J.state = 2;
        feed.finished(J.tag, e, why.c_str());
      }
    return e;
  };

  const int first = fold();
  if (first < 0) return failAll(first);
  if (first == 0) return BT_OK;
  RoundRunner<kAppSoft> rr(c, info);
  AppParams batch = baseApp(c, nullptr);
  batch.exact = anyExact;
  batch.jobs = c->dJobs;
  batch.jobStart = c->dJobStart;
  batch.numJobs = int(jobs.size());
  int e = rr.begin(batch, int(c->rootCap));
  if (!e) e = rr.startPass(int(R), nullptr, c->cfg.budget);
  if (e) return failAll(e);
  // pass 0, folding arrivals in while the run is young
  for (;;) {
    if ((e = rr.batch()) || (e = settle(rr.hc.rootNext))) return failAll(e);
    const int added = ageMs() < foldMs ? fold() : 0;
    if (added < 0) return failAll(added);
    if (added > 0) {
      // roots [old numRoots, R) join the pass; admission overshoots the
      // end of the root list by up to a warp's claim per warp, so its
      // cursor comes back to the old end first
      if (rr.hc.rootNext > rr.p.numRoots) {
        CK(cudaMemcpyAsync(&c->dCtr->rootNext, &rr.p.numRoots, sizeof(int), cudaMemcpyHostToDevice, c->stream));
        rr.hc.rootNext = rr.p.numRoots;
      }
      rr.p.numRoots = int(R);
      rr.p.app.numJobs = int(jobs.size());
      rr.p.app.exact = anyExact;
      if ((e = rr.reopen())) return failAll(e);
      continue;
    }
    if (rr.hc.done) break;
  }
  if (rr.hc.maxQueue > c->queueHighWater) c->queueHighWater = rr.hc.maxQueue;
  // retry passes for the roots abandoned over budget
  const int32_t* list = nullptr;
  int n = int(R), budget = c->cfg.budget;
  for (;;) {
    int nk = 0;
    if ((e = rr.endPass(n, &list, &nk))) return failAll(e);
    if (nk == 0) break;
    n = nk;
    budget *= 16;
    if ((e = rr.startPass(n, list, budget))) return failAll(e);
    do {
      if ((e = rr.batch())) return failAll(e);
    } while (!rr.hc.done);
  }
  for (Job& J : jobs)
    if (J.state != 2 && (e = handBack(J))) return failAll(e);
  rr.finish(R);
  return BT_OK;
}

}  // namespace btserve

// ---------------------------------------------------------------------------
// Allocation-free soft shadows (bt_gpu_soft_points_noalloc).
//
// Every byte of device scratch this entry point needs -- the scene in the
// engine's layout, the per-point root records and the three sub-beam queues
// -- comes out of one fixed array compiled into this library, so a call
// makes no device allocation.  The array lives at file scope; its name in
// host code is only a host-side stand-in, so the host looks up its device
// address once per device with cudaGetSymbolAddress and passes that
// address on.  All calls on a device share the array: a call clears what
// has to start at zero, and two calls whose work overlaps on the GPU would
// corrupt each other (see the lock below).
// ---------------------------------------------------------------------------

static __device__ __align__(256) unsigned char g_noallocScratch[BT_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int64_t kNoAllocMinQueue = 8192;  // sub-beam records per queue, at least
constexpr int kNoAllocMaxDevices = 64;

struct NoAllocDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noallocScratch on this device
  int sms = 0;
  cudaEvent_t rev[2] = {nullptr, nullptr};
  std::mutex run;  // one call at a time per device in this process
};
NoAllocDevice g_noalloc[kNoAllocMaxDevices];
std::mutex g_noallocSetup;

// Byte offsets of the sections of the scratch array (each 256-aligned).
struct NoAllocLayout {
  size_t err, ctr, stats, kill;
  size_t node, box, parent, ref, triNV;
  size_t roots, live, resv, state, attempt, list0, list1, miss, g, shade;
  size_t queues;
  int64_t cap;  // records per queue
};

// Lays the sections out; false when the fixed part leaves less than
// kNoAllocMinQueue records per queue.  *need = bytes of the fixed part plus
// the smallest queues.
bool noallocLayout(int64_t nn, int64_t nr, int64_t nt, int64_t n, NoAllocLayout* L, size_t* need) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~size_t(255);
    return o;
  };
  const size_t R = size_t(std::max<int64_t>(n, 1));
  L->err = take(2 * sizeof(int));
  L->ctr = take(sizeof(Counters));
  L->stats = take(kNumStats * sizeof(unsigned long long));
  L->kill = take(sizeof(int));
  L->node = take(size_t(nn) * sizeof(uint2));
  L->box = take(size_t(2 * nn) * sizeof(float4));
  L->parent = take(size_t(nn) * sizeof(uint32_t));
  L->ref = take(size_t(4 * nr) * sizeof(float4));
  L->triNV = take(size_t(2 * nt) * sizeof(float4));
  L->roots = take(R * sizeof(RootRec));
  L->live = take(R * sizeof(int32_t));
  L->resv = take(R * sizeof(int32_t));
  L->state = take(R * sizeof(int32_t));
  L->attempt = take(R * sizeof(int32_t));
  L->list0 = take(R * sizeof(int32_t));
  L->list1 = take(R * sizeof(int32_t));
  L->miss = take(R * sizeof(unsigned long long));
  L->g = take(R * sizeof(unsigned long long));
  L->shade = take(2 * R * sizeof(float4));
  L->queues = off;
  *need = off + 3 * size_t(kNoAllocMinQueue) * sizeof(SubBeam);
  if (*need > size_t(BT_NOALLOC_SCRATCH_BYTES)) return false;
  L->cap = int64_t((size_t(BT_NOALLOC_SCRATCH_BYTES) - off) / (3 * sizeof(SubBeam)));
  return true;
}

struct PackArgs {
  const float* pos;
  int64_t nv;
  const uint32_t* tris;
  const float* nrm;
  int64_t nt;
  const float* split;
  const uint32_t* data;
  const uint32_t* offset;
  const uint32_t* parent;
  const float* box;
  int64_t nn;
  const uint32_t* triIdx;
  int64_t nr;
  uint2* oNode;
  float4* oBox;
  uint32_t* oParent;
  float4* oRef;
  float4* oTriNV;
  int* err;  // [0]: first failure (1 node, 2 reference, 3 triangle), [1]: its index
};

__device__ void packFail(int* err, int code, int64_t i) {
  if (atomicCAS(err, 0, code) == 0) atomicExch(err + 1, int(i));
}

// The device-side twin of uploadScene's packing: kd nodes as {split bits or
// leaf offset, data}, node boxes as two float4, parents, 64-byte triangle
// references and per-triangle normal + first vertex.  Every index read from
// the caller's arrays is checked before it is used; a bad one is recorded
// in `err` and its record is skipped.  Interior nodes must have their
// children after them and every node but the root its parent before it,
// which bt_kd_build's trees satisfy and which keeps descents and climbs
// finite.
__global__ void packSceneKernel(PackArgs a) {
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  const int64_t m = max(a.nn, max(a.nr, a.nt));
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += stride) {
    if (i < a.nn) {
      const uint32_t d = a.data[i];
      uint32_t x;
      bool ok;
      if ((d & 3u) == 3u) {
        x = a.offset[i];
        ok = int64_t(x) + int64_t(d >> 2) <= a.nr;
      } else {
        x = __float_as_uint(a.split[i]);
        ok = int64_t(d >> 2) > i + 1 && int64_t(d >> 2) < a.nn;
      }
      const uint32_t par = a.parent[i];
      if (i > 0) ok = ok && int64_t(par) < i;
      if (!ok) {
        packFail(a.err, 1, i);
      } else {
        a.oNode[i] = make_uint2(x, d);
        const float* b = a.box + 6 * i;
        a.oBox[2 * i] = make_float4(b[0], b[1], b[2], b[3]);
        a.oBox[2 * i + 1] = make_float4(b[4], b[5], 0.f, 0.f);
        a.oParent[i] = par;
      }
    }
    if (i < a.nr) {
      const uint32_t t = a.triIdx[i];
      bool ok = int64_t(t) < a.nt;
      uint32_t v0 = 0, v1 = 0, v2 = 0;
      if (ok) {
        v0 = a.tris[3 * size_t(t)];
        v1 = a.tris[3 * size_t(t) + 1];
        v2 = a.tris[3 * size_t(t) + 2];
        ok = int64_t(v0) < a.nv && int64_t(v1) < a.nv && int64_t(v2) < a.nv;
      }
      if (!ok) {
        packFail(a.err, 2, i);
      } else {
        const float* p0 = a.pos + 3 * size_t(v0);
        const float* p1 = a.pos + 3 * size_t(v1);
        const float* p2 = a.pos + 3 * size_t(v2);
        const float* nr = a.nrm + 3 * size_t(t);
        a.oRef[4 * i] = make_float4(p0[0], p0[1], p0[2], p1[0]);
        a.oRef[4 * i + 1] = make_float4(p1[1], p1[2], p2[0], p2[1]);
        a.oRef[4 * i + 2] = make_float4(p2[2], nr[0], nr[1], nr[2]);
        a.oRef[4 * i + 3] = make_float4(__uint_as_float(v0), __uint_as_float(v1), __uint_as_float(v2), __uint_as_float(t));
      }
    }
    if (i < a.nt) {
      const uint32_t v0 = a.tris[3 * size_t(i)];
      if (int64_t(v0) >= a.nv) {
        packFail(a.err, 3, i);
      } else {
        const float* nr = a.nrm + 3 * size_t(i);
        const float* p0 = a.pos + 3 * size_t(v0);
        a.oTriNV[2 * i] = make_float4(nr[0], nr[1], nr[2], 0.f);
        a.oTriNV[2 * i + 1] = make_float4(p0[0], p0[1], p0[2], 0.f);
      }
    }
  }
}

// True when p is a 4-byte-aligned address of device (or managed) memory of
// device `dev`; a host address handed to a kernel would fault.
bool deviceReachable(const void* p, int dev) {
  if ((reinterpret_cast<uintptr_t>(p) & 3u) != 0) return false;
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type == cudaMemoryTypeManaged) return true;
  return at.type == cudaMemoryTypeDevice && at.device == dev;
}

}  // namespace

extern "C" {

int bt_gpu_soft_points_noalloc(const bt_scene_desc* sc, const bt_kd_desc* kd, const bt_area_light* L,
                               const bt_soft_opts* o, int64_t n, const int32_t* dTri, const float* dX, const float* dN,
                               float* dVis, float* dE, float* dEu, bt_run_info* info) {
  const int64_t kMax32 = 0x7fffffff;
  if (!sc || !kd || !L || n < 0 || n > kMax32 || sc->num_tris <= 0 || sc->num_tris > kMax32 || sc->num_verts <= 0 ||
      sc->num_verts > kMax32 || kd->num_nodes <= 0 || kd->num_nodes > kMax32 || kd->num_refs < 0 ||
      kd->num_refs > kMax32 || !sc->pos || !sc->tris || !sc->tri_normals || !kd->split || !kd->data || !kd->offset ||
      !kd->parent || !kd->node_box || (kd->num_refs > 0 && !kd->tri_indices) || (n > 0 && (!dTri || !dX || !dN))) {
    setErr("bt_gpu_soft_points_noalloc: bad arguments");
    return BT_ERR_INVALID;
  }
  NoAllocLayout lay;
  size_t need = 0;
  if (!noallocLayout(kd->num_nodes, kd->num_refs, sc->num_tris, n, &lay, &need)) {
    setErr("bt_gpu_soft_points_noalloc: %lld kd nodes, %lld references, %lld triangles and %lld points need %zu bytes "
           "of scratch; the fixed limit is %lld bytes (BT_NOALLOC_SCRATCH_BYTES)",
           (long long)kd->num_nodes, (long long)kd->num_refs, (long long)sc->num_tris, (long long)n, need,
           (long long)BT_NOALLOC_SCRATCH_BYTES);
    return BT_ERR_TOO_LARGE;
  }
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kNoAllocMaxDevices) {
    setErr("bt_gpu_soft_points_noalloc: device %d is beyond the %d this library serves", dev, kNoAllocMaxDevices);
    return BT_ERR_INVALID;
  }
  NoAllocDevice& D = g_noalloc[dev];
  {
    // One-time set-up per device, with that device current: the device
    // address of the scratch array, the SM count and two timing events.
    std::lock_guard<std::mutex> lk(g_noallocSetup);
    if (!D.ready) {
      void* p = nullptr;
      CK(cudaGetSymbolAddress(&p, g_noallocScratch));
      CK(cudaDeviceGetAttribute(&D.sms, cudaDevAttrMultiProcessorCount, dev));
      for (auto& ev : D.rev)
        if (!ev) CK(cudaEventCreate(&ev));
      D.scratch = static_cast<unsigned char*>(p);
      D.ready = true;
    }
  }
  const void* ins[] = {sc->pos, sc->tris, sc->tri_normals, kd->split, kd->data, kd->offset, kd->parent, kd->node_box};
  for (const void* p : ins)
    if (!deviceReachable(p, dev)) {
      setErr("bt_gpu_soft_points_noalloc: a scene array is not 4-byte-aligned device memory of device %d", dev);
      return BT_ERR_INVALID;
    }
  if ((kd->num_refs > 0 && !deviceReachable(kd->tri_indices, dev)) ||
      (n > 0 && (!deviceReachable(dTri, dev) || !deviceReachable(dX, dev) || !deviceReachable(dN, dev) ||
                 (dVis && !deviceReachable(dVis, dev)) || (dE && !deviceReachable(dE, dev)) ||
                 (dEu && !deviceReachable(dEu, dev))))) {
    setErr("bt_gpu_soft_points_noalloc: a point or output array is not 4-byte-aligned device memory of device %d", dev);
    return BT_ERR_INVALID;
  }
  std::lock_guard<std::mutex> run(D.run);
  unsigned char* S = D.scratch;
  auto at = [&](size_t off) { return static_cast<void*>(S + off); };

  // the scene, packed into the scratch array
  int* dErr = static_cast<int*>(at(lay.err));
  CK(cudaMemsetAsync(dErr, 0, 2 * sizeof(int), 0));
  PackArgs pa;
  pa.pos = sc->pos;
  pa.nv = sc->num_verts;
  pa.tris = sc->tris;
  pa.nrm = sc->tri_normals;
  pa.nt = sc->num_tris;
  pa.split = kd->split;
  pa.data = kd->data;
  pa.offset = kd->offset;
  pa.parent = kd->parent;
  pa.box = kd->node_box;
  pa.nn = kd->num_nodes;
  pa.triIdx = kd->tri_indices;
  pa.nr = kd->num_refs;
  pa.oNode = static_cast<uint2*>(at(lay.node));
  pa.oBox = static_cast<float4*>(at(lay.box));
  pa.oParent = static_cast<uint32_t*>(at(lay.parent));
  pa.oRef = static_cast<float4*>(at(lay.ref));
  pa.oTriNV = static_cast<float4*>(at(lay.triNV));
  pa.err = dErr;
  const int64_t m = std::max(kd->num_nodes, std::max(kd->num_refs, sc->num_tris));
  const int pg = int(std::min<int64_t>((m + 255) / 256, int64_t(D.sms) * 8));
  packSceneKernel<<<pg, 256, 0, 0>>>(pa);
  CK(cudaGetLastError());
  int herr[2] = {0, 0};
  CK(cudaMemcpy(herr, dErr, sizeof herr, cudaMemcpyDeviceToHost));
  if (herr[0]) {
    static const char* what[] = {"", "kd node", "kd reference", "triangle"};
    setErr("bt_gpu_soft_points_noalloc: %s %d is malformed (an index out of range or out of order)",
           what[herr[0] & 3], herr[1]);
    return BT_ERR_INVALID;
  }

  // an engine context that only views the scratch array (it owns nothing
  // and never reaches bt_gpu_destroy); the legacy default stream
  bt_gpu_ctx c;
  bt_gpu_config_default(&c.cfg);
  c.device = dev;
  c.sms = D.sms;
  c.stream = nullptr;
  c.rev[0] = D.rev[0];
  c.rev[1] = D.rev[1];
  c.s.node = pa.oNode;
  c.s.box = pa.oBox;
  c.s.parent = pa.oParent;
  c.s.ref = pa.oRef;
  c.s.triNV = pa.oTriNV;
  for (int a = 0; a < 3; ++a) {
    c.s.bounds.lo[a] = kd->bounds[a];
    c.s.bounds.hi[a] = kd->bounds[3 + a];
  }
  c.s.numTris = int(sc->num_tris);
  c.s.numNodes = uint32_t(kd->num_nodes);
  c.s.rootNode = 0;
  c.numTris = sc->num_tris;
  V3 dg = mk(sc->bounds[3] - sc->bounds[0], sc->bounds[4] - sc->bounds[1], sc->bounds[5] - sc->bounds[2]);
  c.offset = length(dg) * kEpsRel;
  c.capacity = int(std::min<int64_t>(lay.cap, kMax32));
  SubBeam* q = static_cast<SubBeam*>(at(lay.queues));
  c.dQ[0] = q;
  c.dQ[1] = q + lay.cap;
  c.dQ[2] = q + 2 * lay.cap;
  c.dCtr = static_cast<Counters*>(at(lay.ctr));
  c.dStats = static_cast<unsigned long long*>(at(lay.stats));
  c.dKillCount = static_cast<int*>(at(lay.kill));
  c.rootCap = size_t(std::max<int64_t>(n, 1));
  c.dRoots = static_cast<RootRec*>(at(lay.roots));
  c.dLive = static_cast<int32_t*>(at(lay.live));
  c.dResv = static_cast<int32_t*>(at(lay.resv));
  c.dState = static_cast<int32_t*>(at(lay.state));
  c.dAttempt = static_cast<int32_t*>(at(lay.attempt));
  c.dList[0] = static_cast<int32_t*>(at(lay.list0));
  c.dList[1] = static_cast<int32_t*>(at(lay.list1));
  c.dMiss = static_cast<unsigned long long*>(at(lay.miss));
  c.dG = static_cast<unsigned long long*>(at(lay.g));
  c.dShade = static_cast<float4*>(at(lay.shade));

  if (info) memset(info, 0, sizeof *info);
  const auto t0 = std::chrono::steady_clock::now();
  // The engine clears the counters, statistics and attempt tags at the start
  // of every pass and writes each root's state when it admits the root, so
  // nothing a previous call left in the array is read.
  int e = softCore(&c, L, o, n, nullptr, dTri, dX, dN, dVis, dE, dEu, info);
  if (e == BT_ERR_CAPACITY) {
    const std::string why = g_err;
    setErr("%s (the allocation-free call's queues hold %lld sub-beams each, out of its fixed scratch array)",
           why.c_str(), (long long)lay.cap);
  }
  if (e) return e;
  CK(cudaStreamSynchronize(0));
  if (info)
    info->ms_total = info->ms_trace =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return BT_OK;
}

}  // extern "C"
