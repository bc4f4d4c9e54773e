// Beam arithmetic of the tracer: beam-kd slab decisions, triangle setup,
// fuzzy four-corner edge votes, clipping into convex pieces, pre-split by
// direction sign.  Written once as __host__ __device__ code: the CUDA engine
// runs it per lane, and a host build of the same header lets the CPU tests
// check every step against the reference's float build bit for bit.
//
// Bit-exactness with the reference's float build (bt_render) requires the
// same IEEE single-precision operations in the same order: no contraction
// into FMA (nvcc -fmad=false; g++ -ffp-contract=off), IEEE division and
// square root (no --use_fast_math), and left-to-right evaluation of every
// sum exactly as the reference writes it.  Each function cites the
// reference code whose arithmetic it keeps; the data layout around it
// (corner arrays, packed records, per-lane state) is this engine's own.
#pragma once

#include <stdint.h>

#include <cmath>

// BT_HD: small helpers, always inlined.  BT_COLD: clipping, pre-split,
// set-up and output paths, kept out of line as one copy each: the hot
// traversal loop then fits the instruction caches (inlining everything made
// instruction fetch the dominant stall).
#if defined(__CUDACC__)
#define BT_HD __host__ __device__ __forceinline__
#define BT_COLD __host__ __device__ __noinline__
#define BT_UNROLL _Pragma("unroll")
// the polygon steps of a clip: inlined into the one out-of-line clip
// routine, so that its polygons can stay in registers
#define BT_CLIP __host__ __device__ __forceinline__
#else
#define BT_HD inline
#define BT_COLD __attribute__((noinline))
#define BT_UNROLL
#define BT_CLIP inline
#endif

// Vertices of a clip polygon.  The reference sizes its lists for 8
// (kMaxPoly, beam_geom.h:12), but the clip only ever splits polygons of at
// most 4 corners (beams, and pentagons are split into 4 + 3 before the next
// line), so a piece has at most 5; 6 keeps the splitter's overflow check
// unreachable and the clip's local arrays small.
constexpr int kPolyMax = 6;

namespace btg {

// Tolerances of the float build (src/core/real.h:35-37, src/beam/beam_core.h:26-27).
constexpr float kEpsRel = 2e-5f;       // fuzzy split epsilon, relative to the root's extent
constexpr float kKdRel = 1e-5f;        // kd decision margin
constexpr float kDegRel = 2e-6f;       // edge-on triangle rejection
constexpr float kCoplanarCos = 2e-6f;  // coplanar depth tie
constexpr float kCoplanarRel = 2e-5f;
constexpr float kInf = __builtin_huge_valf();

enum { kNear = 0, kFar = 1, kBoth = 2 };                 // kd decisions
enum { kTriKeep = 0, kTriAllIn = 1, kTriClip = 2 };      // beam-triangle outcome
enum { kModeNearest = 0, kModeAnyHit = 1 };

// |x| as the FP unit's operand modifier.  It differs from x < 0 ? -x : x only
// in the sign of a zero, and every use here is compared or feeds a tolerance
// that is compared, where -0 and +0 are equal.
BT_HD float fabs_(float x) { return fabsf(x); }

struct V3 {
  float x, y, z;
};
BT_HD V3 mk(float x, float y, float z) { return V3{x, y, z}; }
BT_HD V3 sub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
BT_HD V3 add(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
BT_HD V3 neg(V3 a) { return V3{-a.x, -a.y, -a.z}; }
BT_HD V3 mul(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
BT_HD V3 divs(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
// dot and cross as src/core/vec.h:27-30 evaluates them.
BT_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
BT_HD V3 cross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
BT_HD float length(V3 a) { return sqrtf(dot(a, a)); }
BT_HD V3 normalize(V3 a) {
  float l = length(a);
  return l > 0 ? divs(a, l) : a;
}
BT_HD float comp(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
// Any unit vector orthogonal to unit n (vec.h:39-42).
BT_HD V3 anyOrthogonal(V3 n) {
  V3 a = fabs_(n.x) < 0.6f ? mk(1, 0, 0) : (fabs_(n.y) < 0.6f ? mk(0, 1, 0) : mk(0, 0, 1));
  return normalize(cross(n, a));
}

// ------------------------------------------------------------------ planes

// The plane carrying a beam tree's corner directions (beam_types.h:14-52):
// corner ray k is O + t * (d + u qx + v qy); t = 1 on the plane.
struct Plane {
  V3 O, p0, u, v, n, d;
};

BT_HD Plane makePlane(V3 O, V3 p0, V3 u_, V3 v_) {  // BeamPlane::make
  Plane P;
  P.O = O;
  P.p0 = p0;
  V3 n = normalize(cross(u_, v_));
  if (dot(n, sub(p0, O)) < 0) n = neg(n);
  P.u = normalize(u_);
  P.v = cross(n, P.u);
  P.n = n;
  P.d = sub(p0, O);
  return P;
}
BT_HD V3 planePoint(const Plane& P, float qx, float qy) { return add(add(P.p0, mul(P.u, qx)), mul(P.v, qy)); }
BT_HD void planeCoords(const Plane& P, V3 p, float& qx, float& qy) {
  V3 r = sub(p, P.p0);
  qx = dot(r, P.u);
  qy = dot(r, P.v);
}
// Central projection through O onto the plane (BeamPlane::project).
BT_HD bool planeProject(const Plane& P, V3 p, float& qx, float& qy) {
  V3 r = sub(p, P.O);
  float den = dot(P.n, r);
  if (!(den > 0)) return false;
  V3 x = add(P.O, mul(r, dot(P.n, P.d) / den));
  planeCoords(P, x, qx, qy);
  return true;
}

// ------------------------------------------------------------ 2D polygons

// A convex polygon of at most N vertices.  Every element access is either
// at a compile-time index (loops unrolled to N, guarded by i < n) or a
// select chain over the N slots, so that a polygon held in a local variable
// stays in registers: a run-time array index would put it in local memory,
// which the clip step otherwise reads and writes hundreds of times per
// record.  The arithmetic is the same operations in the same order.
template <int N>
struct Poly {
  float x[N], y[N];
  int n;
  BT_HD float X(int i) const {
    float v = x[0];
    BT_UNROLL for (int k = 1; k < N; ++k) v = i == k ? x[k] : v;
    return v;
  }
  BT_HD float Y(int i) const {
    float v = y[0];
    BT_UNROLL for (int k = 1; k < N; ++k) v = i == k ? y[k] : v;
    return v;
  }
  BT_HD void set(int i, float px, float py) {
    BT_UNROLL for (int k = 0; k < N; ++k) {
      x[k] = i == k ? px : x[k];
      y[k] = i == k ? py : y[k];
    }
  }
  // vertex after i (i < n): i + 1, or 0 at the end
  BT_HD float nextX(int i) const { return i + 1 == n ? x[0] : x[i + 1 < N ? i + 1 : 0]; }
  BT_HD float nextY(int i) const { return i + 1 == n ? y[0] : y[i + 1 < N ? i + 1 : 0]; }
  BT_HD void clear() { n = 0; }
  BT_HD void push(float px, float py) {
    if (n < N) {
      set(n, px, py);
      ++n;
    }
  }
  // Signed area, accumulated as beam_geom.h:27-34 does.
  BT_HD float area() const {
    float a = 0;
    BT_UNROLL for (int i = 0; i < N; ++i) {
      if (i < n) a += x[i] * nextY(i) - nextX(i) * y[i];
    }
    return a * 0.5f;
  }
  BT_HD void reverse() {
    float rx[N], ry[N];
    BT_UNROLL for (int k = 0; k < N; ++k) {
      rx[k] = k < n ? X(n - 1 - k) : x[k];
      ry[k] = k < n ? Y(n - 1 - k) : y[k];
    }
    BT_UNROLL for (int k = 0; k < N; ++k) {
      x[k] = rx[k];
      y[k] = ry[k];
    }
  }
  BT_HD float extent() const {
    float lx = kInf, hx = -kInf, ly = kInf, hy = -kInf;
    BT_UNROLL for (int i = 0; i < N; ++i) {
      if (i < n) {
        lx = x[i] < lx ? x[i] : lx;
        hx = x[i] > hx ? x[i] : hx;
        ly = y[i] < ly ? y[i] : ly;
        hy = y[i] > hy ? y[i] : hy;
      }
    }
    float ex = hx - lx, ey = hy - ly;
    return ex > ey ? ex : ey;
  }
  template <int M>
  BT_HD void copyFrom(const Poly<M>& o) {
    n = o.n < N ? o.n : N;
    BT_UNROLL for (int i = 0; i < (N < M ? N : M); ++i) {
      if (i < n) {
        x[i] = o.x[i];
        y[i] = o.y[i];
      }
    }
  }
};

struct Line {
  float a, b, c;
  BT_HD float eval(float x, float y) const { return a * x + b * y + c; }
};

// Normalised line; a line ~1e9 extents away (or parallel) becomes the
// constant sign(c) (beam_geom.h:65-76).
// |D| > kDegRel * length(m) * length(r), computed in float exactly as the
// triangle setup computes it (beam_core.h:260-286).  The square roots are
// needed only when the two sides lie within 1e-4 of each other: comparing
// squares (relative error below 1e-6) decides every other case the same way.
BT_HD bool notEdgeOn(float D, V3 m, V3 r) {
  const float mm = dot(m, m), rr = dot(r, r);
  const float D2 = D * D;
  const float T = (kDegRel * kDegRel) * mm * rr;
  if (T > 1e-30f && T < 1e30f && D2 < 1e30f) {
    if (D2 > T * 1.0001f) return true;
    if (D2 < T * 0.9999f) return false;
  }
  const float scale = sqrtf(mm) * sqrtf(rr);
  return (D < 0 ? -D : D) > kDegRel * scale;
}

BT_HD Line makeLine(float a, float b, float c, float ext) {
  Line L{0, 0, 0};
  float nrm = sqrtf(a * a + b * b);
  if (!(nrm > 0) || nrm * ext * 1e9f < fabs_(c)) {
    L.c = c > 0 ? 1.f : (c < 0 ? -1.f : 0.f);
    return L;
  }
  L.a = a / nrm;
  L.b = b / nrm;
  L.c = c / nrm;
  return L;
}

// An edge line in FP64 (the opt-in band re-decision, eps_fp64): the same
// line as the float one -- from the same float vertices and apex, in the
// same canonical orientation -- with every operation in double, normalised
// to unit (a, b).  ok = 0 where the float line is not a plain edge (a
// constant line) or the FP64 one is degenerate: no re-decision then.
struct Line64 {
  double a, b, c;
  int ok;
  BT_HD double eval(float x, float y) const { return double(x) * a + double(y) * b + c; }
};

// Side of a point at float distance d from line L: +1 / -1 outside the
// fuzzy band, 0 inside it; with l64 (F64), a point inside the float band
// takes the side of its FP64 distance when that lies outside the band, and
// *dq carries that distance (as float) for crossing interpolation.
template <bool F64>
BT_HD int bandSide(float d, float x, float y, float eps, const Line64* l64, float* dq) {
  const int s = d > eps ? 1 : (d < -eps ? -1 : 0);
  if (!F64 || s != 0 || !l64 || !l64->ok) return s;
  const double d64 = l64->eval(x, y);
  if (d64 > double(eps)) {
    *dq = float(d64);
    return 1;
  }
  if (d64 < -double(eps)) {
    *dq = float(d64);
    return -1;
  }
  return 0;
}

// Fuzzy split of convex p by L; crossings computed from the
// lexicographically smaller endpoint (beam_geom.h:83-114).  F64: band
// vertices re-decided by l64 (bandSide).
template <int N, bool F64 = false>
BT_CLIP bool splitPoly(const Poly<N>& p, const Line& L, float eps, Poly<N>& in, Poly<N>& out,
                       const Line64* l64 = nullptr) {
  in.clear();
  out.clear();
  float d[N];
  int side[N];
  int keptIn = 0, keptOut = 0;
  BT_UNROLL for (int i = 0; i < N; ++i) {
    d[i] = 0.f;
    side[i] = 0;
    if (i < p.n) {
      d[i] = L.eval(p.x[i], p.y[i]);
      side[i] = bandSide<F64>(d[i], p.x[i], p.y[i], eps, l64, &d[i]);
    }
  }
  BT_UNROLL for (int i = 0; i < N; ++i) {
    if (i < p.n) {
      const int sideNext = i + 1 == p.n ? side[0] : side[i + 1 < N ? i + 1 : 0];
      keptIn += (side[i] >= 0) + (side[i] * sideNext < 0);
      keptOut += (side[i] <= 0) + (side[i] * sideNext < 0);
    }
  }
  if (keptIn > N || keptOut > N) return false;
  BT_UNROLL for (int i = 0; i < N; ++i) {
    if (i < p.n) {
      const bool wrap = i + 1 == p.n;
      const int next = i + 1 < N ? i + 1 : 0;
      const int sideNext = wrap ? side[0] : side[next];
      const float dNext = wrap ? d[0] : d[next];
      const float xj = wrap ? p.x[0] : p.x[next], yj = wrap ? p.y[0] : p.y[next];
      if (side[i] >= 0) in.push(p.x[i], p.y[i]);
      if (side[i] <= 0) out.push(p.x[i], p.y[i]);
      if (side[i] * sideNext < 0) {
        const bool fromHere = p.x[i] < xj || (p.x[i] == xj && p.y[i] < yj);
        const float da = fromHere ? d[i] : dNext, db = fromHere ? dNext : d[i];
        const float xa = fromHere ? p.x[i] : xj, xb = fromHere ? xj : p.x[i];
        const float ya = fromHere ? p.y[i] : yj, yb = fromHere ? yj : p.y[i];
        float t = da / (da - db);
        float X = xa + t * (xb - xa);
        float Y = ya + t * (yb - ya);
        in.push(X, Y);
        out.push(X, Y);
      }
    }
  }
  return true;
}

// Welds duplicate / collinear vertices within 1e-3 of the split epsilon
// (beam_geom.h:122-150); n = 0 if the polygon collapses.
template <int N>
BT_CLIP void cleanPoly(Poly<N>& p, float epsSplit) {
  const float eps = epsSplit * 1e-3f;
  bool changed = true;
  while (changed && p.n >= 3) {
    changed = false;
    for (int i = 0; i < p.n && p.n >= 3; ++i) {
      int h = i == 0 ? p.n - 1 : i - 1;
      int j = i + 1 == p.n ? 0 : i + 1;
      const float xh = p.X(h), yh = p.Y(h), xi = p.X(i), yi = p.Y(i), xj = p.X(j), yj = p.Y(j);
      float ex = xj - xh, ey = yj - yh;
      float dx = xi - xh, dy = yi - yh;
      float len = sqrtf(ex * ex + ey * ey);
      float gapSq = dx * dx + dy * dy;
      float offLine = fabs_(ex * dy - ey * dx);
      bool dup = gapSq <= eps * eps;
      bool collinear = offLine <= eps * len;
      if (dup || collinear) {
        // drop vertex i: the later ones move down one slot
        BT_UNROLL for (int k = 0; k + 1 < N; ++k) {
          if (k >= i && k + 1 < p.n) {
            p.x[k] = p.x[k + 1];
            p.y[k] = p.y[k + 1];
          }
        }
        --p.n;
        changed = true;
        --i;
      }
    }
  }
  if (p.n < 3) p.n = 0;
}

// Bit 0: some vertex strictly inside; bit 1: some vertex strictly outside
// (beam_core.h:69-78).
template <int N, bool F64 = false>
BT_HD int classifyPoly(const Poly<N>& p, const Line& L, float eps, const Line64* l64 = nullptr) {
  int c = 0;
  BT_UNROLL for (int i = 0; i < N; ++i) {
    if (i < p.n) {
      float d = L.eval(p.x[i], p.y[i]);
      const int s = bandSide<F64>(d, p.x[i], p.y[i], eps, l64, &d);
      if (s > 0)
        c |= 1;
      else if (s < 0)
        c |= 2;
    }
  }
  return c;
}

// Pentagon -> quad (0,1,2,3) + triangle (0,3,4) (beam_core.h:81-89).
template <int N, int M>
BT_HD void splitFive(const Poly<N>& p, Poly<M>& a, Poly<M>& b) {
  a.clear();
  b.clear();
  for (int i = 0; i < 4; ++i) a.push(p.x[i], p.y[i]);
  b.push(p.x[0], p.y[0]);
  b.push(p.x[3], p.y[3]);
  b.push(p.x[4], p.y[4]);
}

// ------------------------------------------------------------------ beams

// Per-root constants: the query plane, mode and tolerances (BeamCtx::setup,
// beam_core.h:123-132).
struct Query {
  Plane P;
  int mode;
  int farIsPlane;
  int exclude;
  int cull;
  float ext, eps, minArea, farCq;
};

BT_HD void querySetup(Query& q, float extent) {
  q.ext = extent > 0 ? extent : 1.f;
  q.eps = kEpsRel * q.ext;
  q.minArea = q.eps * q.eps;
  q.farCq = dot(q.P.n, q.P.d);
}

// A sub-beam in working form: corners (lanes past n repeat the last corner),
// |w_axis| at the corners, far plane, hit status (CoreBeam, beam_core.h:30-40,
// plus the hit plane WfWork caches, wavefront_core.h:58-61).
struct Beam {
  float qx[4], qy[4];
  float aw[3][4];
  float farA[4];
  float farC;
  int n;
  int hit;
  int neg;  // bit a: rays move toward -a
  int hasFar;
  float hitA[3], hitC;
  V3 hitN;
};

BT_HD float sgnOf(const Beam& b, int a) { return ((b.neg >> a) & 1) ? -1.f : 1.f; }
BT_HD float awAt(const Beam& b, int c, int i) { return c == 0 ? b.aw[0][i] : (c == 1 ? b.aw[1][i] : b.aw[2][i]); }

// |w_a| at the corners (beamGeom / wfExpand, beam_core.h:214-219).
BT_HD void beamAxes(const Query& q, Beam& b) {
  for (int a = 0; a < 3; ++a) {
    const float s = sgnOf(b, a), ua = comp(q.P.u, a), va = comp(q.P.v, a), da = comp(q.P.d, a);
    for (int k = 0; k < 4; ++k) {
      float w = b.qx[k] * ua + b.qy[k] * va + da;
      float ws = w * s;
      b.aw[a][k] = 0.f > ws ? 0.f : ws;
    }
  }
}

// Hit status and far plane (BeamCtx::setStatus, beam_core.h:225-240).
BT_HD void setStatus(const Query& q, Beam& b, int hit, const float* A, float C) {
  b.hit = hit;
  if (hit >= 0) {
    for (int k = 0; k < 4; ++k) b.farA[k] = fabs_(b.qx[k] * A[0] + b.qy[k] * A[1] + A[2]);
    b.farC = C < 0 ? -C : C;
    b.hasFar = 1;
  } else if (q.farIsPlane) {
    float c0 = q.farCq < 0 ? -q.farCq : q.farCq;
    for (int k = 0; k < 4; ++k) b.farA[k] = c0;
    b.farC = c0;
    b.hasFar = 1;
  } else {
    b.farC = 0;
    b.hasFar = 0;
  }
}

// Loads corners of a convex polygon with <= 4 vertices into the beam
// (lanes past n repeat corner n-1, as beamGeom's l3 rule does).
template <int N>
BT_HD void beamCorners(const Poly<N>& c, Beam& b) {
  const bool four = c.n > 3;
  b.qx[0] = c.x[0];
  b.qx[1] = c.x[1];
  b.qx[2] = c.x[2];
  b.qx[3] = four ? c.x[3] : c.x[2];
  b.qy[0] = c.y[0];
  b.qy[1] = c.y[1];
  b.qy[2] = c.y[2];
  b.qy[3] = four ? c.y[3] : c.y[2];
  b.n = c.n;
}

// Cleaned corners and axes of a piece; false (and `dropped` = |area|) for
// slivers below minArea (BeamCtx::beamGeom, beam_core.h:200-221).
// `clean`: p is already a cleanPoly result, whose cleaning would change
// nothing (cleanPoly returns only after a pass without a change).
template <int N>
BT_CLIP bool beamGeom(const Query& q, const Poly<N>& p, int negBits, Beam& b, float& dropped, bool clean = false) {
  Poly<N> c = p;
  if (!clean) cleanPoly(c, q.eps);
  float A = c.n >= 3 ? c.area() : 0.f;
  if (c.n < 3 || A < q.minArea) {
    float a0 = p.area();
    dropped = a0 < 0 ? -a0 : a0;
    return false;
  }
  beamCorners(c, b);
  b.neg = negBits;
  beamAxes(q, b);
  return true;
}

BT_HD bool all4lt(const float* l, const float* r) { return l[0] < r[0] && l[1] < r[1] && l[2] < r[2] && l[3] < r[3]; }
BT_HD bool all4gt(const float* l, const float* r) { return l[0] > r[0] && l[1] > r[1] && l[2] > r[2] && l[3] > r[3]; }

struct Box {
  float lo[3], hi[3];
};
// Component access with a run-time axis, as selects (an indexed array would
// live in local memory).
BT_HD float boxLo(const Box& b, int c) { return c == 0 ? b.lo[0] : (c == 1 ? b.lo[1] : b.lo[2]); }
BT_HD float boxHi(const Box& b, int c) { return c == 0 ? b.hi[0] : (c == 1 ? b.hi[1] : b.hi[2]); }
BT_HD void boxSetLo(Box& b, int c, float v) {
  b.lo[0] = c == 0 ? v : b.lo[0];
  b.lo[1] = c == 1 ? v : b.lo[1];
  b.lo[2] = c == 2 ? v : b.lo[2];
}
BT_HD void boxSetHi(Box& b, int c, float v) {
  b.hi[0] = c == 0 ? v : b.hi[0];
  b.hi[1] = c == 1 ? v : b.hi[1];
  b.hi[2] = c == 2 ? v : b.hi[2];
}

// kd decision at an inner node (BeamCtx::decide, beam_core.h:139-164).
BT_HD int decide(const Query& q, const Beam& b, int a, float Ns, const Box& box) {
  for (int k = 1; k <= 2; ++k) {
    int c = a + k >= 3 ? a + k - 3 : a + k;
    const bool pos = !((b.neg >> c) & 1);
    const float s = pos ? 1.f : -1.f;
    const float Oc = comp(q.P.O, c);
    float entry = pos ? boxLo(box, c) : boxHi(box, c);
    float exit = pos ? boxHi(box, c) : boxLo(box, c);
    float Nmin = s * (entry - Oc);
    float Nmax = s * (exit - Oc);
    float lhs[4], tl[4];
    for (int i = 0; i < 4; ++i) {
      lhs[i] = awAt(b, c, i) * Ns;
      float r = awAt(b, a, i) * Nmin;
      float tol = (fabs_(lhs[i]) + fabs_(r)) * kKdRel;
      tl[i] = r - tol;
    }
    if (all4lt(lhs, tl)) return kFar;
    for (int i = 0; i < 4; ++i) {
      float r = awAt(b, a, i) * Nmax;
      float tol = (fabs_(lhs[i]) + fabs_(r)) * kKdRel;
      tl[i] = r + tol;
    }
    if (all4gt(lhs, tl)) return kNear;
  }
  if (b.hasFar) {
    float lhs[4], tl[4];
    for (int i = 0; i < 4; ++i) {
      lhs[i] = b.farA[i] * Ns;
      float r = awAt(b, a, i) * b.farC;
      float tol = (fabs_(lhs[i]) + fabs_(r)) * kKdRel;
      tl[i] = r + tol;
    }
    if (all4gt(lhs, tl)) return kNear;
  }
  return kBoth;
}

// Conservative beam-box overlap (BeamCtx::overlaps, beam_core.h:166-195).
BT_HD bool overlaps(const Query& q, const Beam& b, const Box& box) {
  float Nmin[3], Nmax[3];
  for (int c = 0; c < 3; ++c) {
    const bool pos = !((b.neg >> c) & 1);
    const float s = pos ? 1.f : -1.f;
    const float Oc = comp(q.P.O, c);
    Nmin[c] = s * ((pos ? box.lo[c] : box.hi[c]) - Oc);
    Nmax[c] = s * ((pos ? box.hi[c] : box.lo[c]) - Oc);
    if (Nmax[c] < 0) return false;
  }
  for (int c = 0; c < 3; ++c) {
    for (int e = 0; e < 3; ++e) {
      if (c == e) continue;
      float lhs[4], tl[4];
      for (int i = 0; i < 4; ++i) {
        lhs[i] = b.aw[e][i] * Nmax[c];
        float r = b.aw[c][i] * Nmin[e];
        float tol = (fabs_(lhs[i]) + fabs_(r)) * kKdRel;
        tl[i] = r - tol;
      }
      if (all4lt(lhs, tl)) return false;
    }
  }
  if (b.hasFar) {
    for (int c = 0; c < 3; ++c) {
      float lhs[4], tl[4];
      for (int i = 0; i < 4; ++i) {
        lhs[i] = b.farA[i] * Nmin[c];
        float r = b.aw[c][i] * b.farC;
        float tol = (fabs_(lhs[i]) + fabs_(r)) * kKdRel;
        tl[i] = r + tol;
      }
      if (all4gt(lhs, tl)) return false;
    }
  }
  return true;
}

// ---------------------------------------------------------- triangle tests

// Per-test triangle setup (CoreTriInfo, beam_core.h:42-51).
struct TriInfo {
  int tri;
  int ok;
  Line edge[3];
  float A[3];
  float C;
  V3 r[3];
  V3 n;
};

// Edge planes through O in canonical vertex order (shared edges come out
// exactly negated), orientation, degeneracy and back-face rejection, edge
// lines and the hit plane (BeamCtx::triSetup, beam_core.h:260-286).
BT_HD void triSetup(const Query& q, V3 v0, V3 v1, V3 v2, V3 nT, const uint32_t* T, int tri, TriInfo& ti) {
  ti.tri = tri;
  ti.ok = 0;
  ti.r[0] = sub(v0, q.P.O);
  ti.r[1] = sub(v1, q.P.O);
  ti.r[2] = sub(v2, q.P.O);
  ti.n = nT;
  V3 m[3];
  for (int k = 0; k < 3; ++k) {
    int i = k, j = k == 2 ? 0 : k + 1;
    m[k] = T[i] < T[j] ? cross(ti.r[i], ti.r[j]) : neg(cross(ti.r[j], ti.r[i]));
  }
  float D = dot(ti.r[2], m[0]);
  float scale = length(m[0]) * length(ti.r[2]);
  if (!((D < 0 ? -D : D) > kDegRel * scale)) return;
  if (q.cull && D > 0) return;
  float s = D > 0 ? 1.f : -1.f;
  for (int k = 0; k < 3; ++k)
    ti.edge[k] = makeLine(s * dot(m[k], q.P.u), s * dot(m[k], q.P.v), s * dot(m[k], q.P.d), q.ext);
  ti.A[0] = dot(nT, q.P.u);
  ti.A[1] = dot(nT, q.P.v);
  ti.A[2] = dot(nT, q.P.d);
  ti.C = dot(nT, ti.r[0]);
  ti.ok = 1;
}

// An edge line of a triangle in FP64 (Line64), oriented as triSetup orients
// the float one: the plane through the apex and the edge's vertices vi, vj
// taken in canonical vertex order (fwd: vi's index is the smaller), times
// the sign sg of the orientation test.  fl: the float line (a constant one
// gets no FP64 twin).
BT_HD Line64 edgeLine64(const Query& q, V3 vi, V3 vj, bool fwd, float sg, const Line& fl) {
  double ri[3], rj[3];
  for (int a = 0; a < 3; ++a) {
    ri[a] = double(comp(vi, a)) - double(comp(q.P.O, a));
    rj[a] = double(comp(vj, a)) - double(comp(q.P.O, a));
  }
  const double* p0 = fwd ? ri : rj;
  const double* p1 = fwd ? rj : ri;
  const double m[3] = {p0[1] * p1[2] - p0[2] * p1[1], p0[2] * p1[0] - p0[0] * p1[2], p0[0] * p1[1] - p0[1] * p1[0]};
  const double f = fwd ? double(sg) : -double(sg);
  const double a = f * (m[0] * double(q.P.u.x) + m[1] * double(q.P.u.y) + m[2] * double(q.P.u.z));
  const double b = f * (m[0] * double(q.P.v.x) + m[1] * double(q.P.v.y) + m[2] * double(q.P.v.z));
  const double c = f * (m[0] * double(q.P.d.x) + m[1] * double(q.P.d.y) + m[2] * double(q.P.d.z));
  const double nrm = sqrt(a * a + b * b);
  Line64 e;
  e.ok = (fl.a != 0.f || fl.b != 0.f) && nrm > 0;
  e.a = e.ok ? a / nrm : 0;
  e.b = e.ok ? b / nrm : 0;
  e.c = e.ok ? c / nrm : 0;
  return e;
}

// The three edge lines of a triangle (vertices v0..v2 with indices T) in
// FP64, edge k from vertex k to k + 1; fl: the float edge lines.
BT_HD void edgeLines64(const Query& q, V3 v0, V3 v1, V3 v2, const uint32_t* T, float sg, const Line* fl,
                       Line64* e) {
  e[0] = edgeLine64(q, v0, v1, T[0] < T[1], sg, fl[0]);
  e[1] = edgeLine64(q, v1, v2, T[1] < T[2], sg, fl[1]);
  e[2] = edgeLine64(q, v2, v0, T[2] < T[0], sg, fl[2]);
}

// Hit plane of triangle t (BeamCtx::hitPlane, beam_core.h:290-297).
BT_HD void hitPlane(const Query& q, V3 nT, V3 v0, float* A, float& C) {
  A[0] = dot(nT, q.P.u);
  A[1] = dot(nT, q.P.v);
  A[2] = dot(nT, q.P.d);
  C = dot(nT, sub(v0, q.P.O));
}

// Positive where triangle T is strictly closer to O than plane F
// (BeamCtx::closerLine, beam_core.h:302-317).
BT_HD Line closerLine(const Query& q, const TriInfo& T, const float* AF, float CF, V3 nF, int fId) {
  float cosang = dot(T.n, nF);
  float aC = T.C < 0 ? -T.C : T.C, aF = CF < 0 ? -CF : CF;
  float scaleC = aC > aF ? aC : aF;
  float ca = cosang < 0 ? -cosang : cosang;
  float diff = T.C - cosang * CF;
  if (ca > 1 - kCoplanarCos && (diff < 0 ? -diff : diff) <= kCoplanarRel * scaleC) {
    Line L{0, 0, (fId >= 0 && T.tri < fId) ? 1.f : -1.f};
    return L;
  }
  float sg = T.C * CF > 0 ? 1.f : -1.f;
  return makeLine(sg * (CF * T.A[0] - T.C * AF[0]), sg * (CF * T.A[1] - T.C * AF[1]),
                  sg * (CF * T.A[2] - T.C * AF[2]), q.ext);
}

// Trivial case (b): a beam side plane has all three vertices strictly
// outside it (BeamCtx::separated, beam_core.h:321-342).
BT_HD bool separated(const Query& q, const Beam& b, const TriInfo& ti) {
  float wx[4], wy[4], wz[4];
  for (int k = 0; k < 4; ++k) {
    wx[k] = b.qx[k] * q.P.u.x + b.qy[k] * q.P.v.x + q.P.d.x;
    wy[k] = b.qx[k] * q.P.u.y + b.qy[k] * q.P.v.y + q.P.d.y;
    wz[k] = b.qx[k] * q.P.u.z + b.qy[k] * q.P.v.z + q.P.d.z;
  }
  float nx[4], ny[4], nz[4], nlen[4];
  for (int k = 0; k < 4; ++k) {
    int k1 = (k + 1) & 3;
    nx[k] = wy[k] * wz[k1] - wz[k] * wy[k1];
    ny[k] = wz[k] * wx[k1] - wx[k] * wz[k1];
    nz[k] = wx[k] * wy[k1] - wy[k] * wx[k1];
    nlen[k] = sqrtf(nx[k] * nx[k] + ny[k] * ny[k] + nz[k] * nz[k]);
  }
  int outAll = b.n == 4 ? 0xF : 0xB;
  for (int v = 0; v < 3 && outAll; ++v) {
    const V3 r = ti.r[v];
    const float lr = length(r) * kEpsRel;
    int m = 0;
    for (int k = 0; k < 4; ++k) {
      float s = nx[k] * r.x + ny[k] * r.y + nz[k] * r.z;
      float tol = nlen[k] * lr;
      m |= (s < -tol) ? (1 << k) : 0;
    }
    outAll &= m;
  }
  return outAll != 0;
}

// Fuzzy 4-corner vote (BeamCtx::testLine, beam_core.h:356-362); F64: band
// corners re-decided by l64.
template <bool F64 = false>
BT_HD bool testLine(const Query& q, const Beam& B, const Line& line, Line* L, int& nl, bool& allIn,
                    const Line64* l64 = nullptr) {
  bool anyIn = false, anyOut = false;
  for (int k = 0; k < 4; ++k) {
    float dv = B.qx[k] * line.a + B.qy[k] * line.b + line.c;
    const int sd = bandSide<F64>(dv, B.qx[k], B.qy[k], q.eps, l64, &dv);
    anyIn |= sd > 0;
    anyOut |= sd < 0;
  }
  if (!anyIn) return false;
  if (anyOut) allIn = false;
  L[nl++] = line;
  return true;
}

// The cheap beam-triangle tests: trivial cases, depth line, far plane
// (BeamCtx::classifyTri, beam_core.h:374-409).  The current hit's plane
// comes from the beam (hitA, hitC, hitN).  F64: the edge votes re-decide
// band corners with the FP64 edge lines e64.  Without `separation`, the
// last test (the beam's side planes, case (b)) is left out: a clip, whose
// triangle the trace step already classified, needs only the lines L.
template <bool F64 = false>
BT_CLIP int classifyTri(const Query& q, const Beam& B, const TriInfo& ti, Line* L, int& nl,
                        const Line64* e64 = nullptr, bool separation = true) {
  nl = 0;
  bool allIn = true;
  for (int k = 0; k < 3; ++k)
    if (!testLine<F64>(q, B, ti.edge[k], L, nl, allIn, F64 ? &e64[k] : nullptr)) return kTriKeep;
  if (q.mode == kModeNearest && B.hit >= 0) {
    if (!testLine(q, B, closerLine(q, ti, B.hitA, B.hitC, B.hitN, B.hit), L, nl, allIn)) return kTriKeep;
  }
  if (q.farIsPlane) {
    const float farA[3] = {0.f, 0.f, q.farCq};
    if (!testLine(q, B, closerLine(q, ti, farA, q.farCq, q.P.n, -1), L, nl, allIn)) return kTriKeep;
  }
  if (allIn) return kTriAllIn;
  if (separation && separated(q, B, ti)) return kTriKeep;
  return kTriClip;
}

// Clips B by L[0..nl) one line at a time, most-cutting edge first; pieces
// outside some line go to sink.push(0, p, clean), pieces inside every line
// to sink.push(1, p, clean) (BeamCtx::clipTri with orderEdges,
// beam_core.h:420-479).  `clean` says the piece is a cleanPoly result: the
// beam's own corners (every beam is made from a cleaned polygon) and the
// halves of a split, but not the halves of a pentagon.
// Line li (run-time, < 5) of five held in registers.
BT_HD Line lineAt(const Line* L, int li) {
  Line r = L[0];
  BT_UNROLL for (int k = 1; k < 5; ++k) {
    r.a = li == k ? L[k].a : r.a;
    r.b = li == k ? L[k].b : r.b;
    r.c = li == k ? L[k].c : r.c;
  }
  return r;
}

template <int N, class Sink, bool F64 = false>
BT_CLIP bool clipTri(const Query& q, const Beam& B, const Line* Lin, int nl, Sink& sink, uint32_t& fiveSplits,
                     const Line64* e64in = nullptr) {
  Line L[5];
  BT_UNROLL for (int k = 0; k < 5; ++k) L[k] = Lin[k];
  Line64 E[3];  // F64: the edge lines' FP64 twins, kept in the order of L[0..2]
  if (F64) {
    E[0] = e64in[0];
    E[1] = e64in[1];
    E[2] = e64in[2];
  }
  {
    float score[3];
    BT_UNROLL for (int k = 0; k < 3; ++k) {
      float pos[4];
      BT_UNROLL for (int i = 0; i < 4; ++i) {
        float dv = B.qx[i] * L[k].a + B.qy[i] * L[k].b + L[k].c;
        pos[i] = dv > 0.f ? dv : 0.f;
      }
      score[k] = pos[0] + pos[1] + pos[2] + (B.n == 4 ? pos[3] : 0.f);
    }
    // insertion sort of the three edge lines by score (stable)
    if (score[1] < score[0]) {
      float ts = score[0];
      score[0] = score[1];
      score[1] = ts;
      Line tl = L[0];
      L[0] = L[1];
      L[1] = tl;
      if (F64) {
        const Line64 te = E[0];
        E[0] = E[1];
        E[1] = te;
      }
    }
    if (score[2] < score[1]) {
      float ts = score[1];
      score[1] = score[2];
      score[2] = ts;
      Line tl = L[1];
      L[1] = L[2];
      L[2] = tl;
      if (F64) {
        const Line64 te = E[1];
        E[1] = E[2];
        E[2] = te;
      }
      if (score[1] < score[0]) {
        ts = score[0];
        score[0] = score[1];
        score[1] = ts;
        tl = L[0];
        L[0] = L[1];
        L[1] = tl;
        if (F64) {
          const Line64 te = E[0];
          E[0] = E[1];
          E[1] = te;
        }
      }
    }
  }
  bool ok = true;
  // pending pentagon halves (LIFO), with the line each resumes at.  A half
  // pushed at line li resumes at li + 1 and everything pushed above it
  // resumes later still, so the lines on the stack rise strictly from
  // bottom to top: at most one entry per line, five at most.
  Poly<N> stack[5];
  int stackLine[5];
  int sp = 0;
  Poly<N> p;
  p.n = B.n;
  BT_UNROLL for (int i = 0; i < 4; ++i) {
    p.x[i] = B.qx[i];
    p.y[i] = B.qy[i];
  }
  bool pClean = true;
  int li = 0;
  for (;;) {
    bool inside = true;
    for (; li < nl; ++li) {
      const Line Lk = lineAt(L, li);
      // F64: the edge lines (the first three) re-decide band vertices
      Line64 Ek;
      Ek.ok = 0;
      if (F64 && li < 3) Ek = li == 0 ? E[0] : (li == 1 ? E[1] : E[2]);
      int c = classifyPoly<N, F64>(p, Lk, q.eps, &Ek);
      if (!(c & 2)) continue;
      if (!(c & 1)) {
        if (!sink.push(0, p, pClean)) ok = false;
        inside = false;
        break;
      }
      Poly<N> in, out;
      if (!splitPoly<N, F64>(p, Lk, q.eps, in, out, &Ek)) return false;
      cleanPoly(out, q.eps);
      if (out.n >= 3 && !sink.push(0, out, true)) ok = false;
      cleanPoly(in, q.eps);
      if (in.n < 3) {
        inside = false;
        break;
      }
      if (in.n == 5) {
        Poly<N> a, b;
        splitFive(in, a, b);
        fiveSplits++;
        if (sp >= 5) return false;
        stack[sp] = b;
        stackLine[sp] = li + 1;
        ++sp;
        p = a;
        pClean = false;
      } else {
        p = in;
        pClean = true;
      }
    }
    if (inside && !sink.push(1, p, pClean)) ok = false;
    if (sp == 0) break;
    --sp;
    p = stack[sp];
    pClean = false;
    li = stackLine[sp];
  }
  return ok;
}

// Pre-split of a root polygon by the lines where a direction component is
// zero, then fan into pieces of <= 4 vertices (BeamCtx::presplit,
// beam_core.h:488-546).  emit.piece(poly, negBits) per piece (false aborts),
// emit.presplit() per extra split, emit.dropped(area) per sign-line sliver.
template <class Emit>
BT_COLD bool presplit(const Query& q, const Poly<8>& root, Emit& emit) {
  struct Item {
    Poly<8> p;
    int axis;
    int neg;
  };
  Item stack[16];
  int sp = 0;
  stack[0].p = root;
  stack[0].axis = 0;
  stack[0].neg = 0;
  sp = 1;
  while (sp > 0) {
    Item it = stack[--sp];
    const Poly<8>& p = it.p;
    if (p.n < 3) continue;
    if (it.axis == 3) {
      for (int k = 1; k + 1 < p.n; k += 2) {
        Poly<8> qd;
        qd.clear();
        qd.push(p.x[0], p.y[0]);
        qd.push(p.x[k], p.y[k]);
        qd.push(p.x[k + 1], p.y[k + 1]);
        if (k + 2 < p.n) qd.push(p.x[k + 2], p.y[k + 2]);
        if (!emit.piece(qd, it.neg)) return false;
      }
      continue;
    }
    const int axis = it.axis;
    Line L = makeLine(comp(q.P.u, axis), comp(q.P.v, axis), comp(q.P.d, axis), q.ext);
    int c = classifyPoly(p, L, q.eps);
    if (c == 3) {
      if (sp + 2 > 16) return false;
      Poly<8> in, out;
      splitPoly(p, L, q.eps, in, out);
      cleanPoly(in, q.eps);
      cleanPoly(out, q.eps);
      Item a = it, b = it;
      a.p = in;
      a.axis = axis + 1;
      a.neg &= ~(1 << axis);
      b.p = out;
      b.axis = axis + 1;
      b.neg |= 1 << axis;
      stack[sp++] = b;
      stack[sp++] = a;
      emit.presplit();
    } else if (c != 0) {
      it.axis = axis + 1;
      if (c & 1)
        it.neg &= ~(1 << axis);
      else
        it.neg |= 1 << axis;
      stack[sp++] = it;
    } else {
      float a0 = p.area();
      a0 = a0 < 0 ? -a0 : a0;
      emit.dropped(a0);
    }
  }
  return true;
}

// ------------------------------------------------------- application setup

// Light-quad shadow beam from shading point x (normal ns), clipped by the
// horizon (lightBeamSetup, src/render/soft_core.h:38-73).
BT_COLD bool lightBeamSetup(V3 Lc, V3 LU, V3 LV, V3 x, V3 ns, int tri, float offset, Query& q, Poly<8>& root,
                          float& lightArea) {
  V3 nL = normalize(cross(LU, LV));
  if (!(dot(sub(x, Lc), nL) > 0)) return false;
  V3 apex = add(x, mul(ns, offset));
  q.P = makePlane(apex, Lc, LU, LV);
  q.mode = kModeAnyHit;
  q.farIsPlane = 1;
  q.exclude = tri;
  q.cull = 0;
  V3 corners[4] = {sub(sub(Lc, mul(LU, 0.5f)), mul(LV, 0.5f)), sub(add(Lc, mul(LU, 0.5f)), mul(LV, 0.5f)),
                   add(add(Lc, mul(LU, 0.5f)), mul(LV, 0.5f)), add(sub(Lc, mul(LU, 0.5f)), mul(LV, 0.5f))};
  Poly<8> quad;
  quad.clear();
  for (int i = 0; i < 4; ++i) {
    float qx, qy;
    planeCoords(q.P, corners[i], qx, qy);
    quad.push(qx, qy);
  }
  if (quad.area() < 0) quad.reverse();
  lightArea = quad.area();
  Line hz;
  hz.a = dot(ns, q.P.u);
  hz.b = dot(ns, q.P.v);
  hz.c = dot(ns, sub(Lc, x));
  int above = 0;
  for (int i = 0; i < quad.n; ++i) above += hz.eval(quad.x[i], quad.y[i]) > 0;
  if (above == 0) return false;
  if (above == quad.n) {
    root = quad;
  } else {
    Poly<8> out;
    splitPoly(quad, hz, 0.f, root, out);
  }
  return root.n >= 3 && root.area() > 0;
}

// Light-centre geometry term of eq. 2 (lightCenterG, soft_core.h:76-84).
BT_COLD float lightCenterG(V3 Lc, V3 LU, V3 LV, V3 x, V3 ns) {
  V3 nL = normalize(cross(LU, LV));
  if (!(dot(sub(x, Lc), nL) > 0)) return 0;
  V3 w = sub(Lc, x);
  float r2 = dot(w, w);
  V3 wn = divs(w, sqrtf(r2));
  float ci = dot(ns, wn), cl = -dot(nL, wn);
  return (ci > 0 ? ci : 0) * (cl > 0 ? cl : 0) / r2;
}

// Shadow beam of a primary hit beam: corners back-projected onto the
// receiver plane, traced from the light (pointShadowSetup,
// src/render/point_core.h:15-36).  `cam` holds eye, fwd, right, down.
BT_COLD bool pointShadowSetup(V3 eye, V3 fwd, V3 right, V3 down, V3 nT, V3 P0, int T, V3 light, const float* px,
                            const float* py, int n, Query& q, Poly<8>& root) {
  float sideCam = dot(nT, sub(eye, P0)), sideL = dot(nT, sub(light, P0));
  if (!(sideCam * sideL > 0)) return false;
  V3 tu = anyOrthogonal(nT);
  q.P = makePlane(light, P0, tu, cross(nT, tu));
  q.mode = kModeAnyHit;
  q.farIsPlane = 1;
  q.exclude = T;
  q.cull = 0;
  root.clear();
  for (int i = 0; i < n; ++i) {
    V3 d = add(add(fwd, mul(right, px[i])), mul(down, py[i]));
    V3 X = add(eye, mul(d, dot(nT, sub(P0, eye)) / dot(nT, d)));
    float qx, qy;
    planeCoords(q.P, X, qx, qy);
    root.push(qx, qy);
  }
  return true;
}

// Occluded piece back to the image plane, counter-clockwise
// (pointShadowToImage, point_core.h:41-64).
BT_COLD bool pointShadowToImage(const Plane& camPlane, const Plane& shadowPlane, const float* sx, const float* sy, int n,
                              float* ox, float* oy) {
  for (int i = 0; i < n; ++i)
    if (!planeProject(camPlane, planePoint(shadowPlane, sx[i], sy[i]), ox[i], oy[i])) return false;
  Poly<8> p;
  p.clear();
  for (int i = 0; i < n; ++i) p.push(ox[i], oy[i]);
  float a = p.area();
  if (!(a > 0 || a < 0)) return false;
  if (a < 0) {
    p.reverse();
    for (int i = 0; i < n; ++i) {
      ox[i] = p.x[i];
      oy[i] = p.y[i];
    }
  }
  for (int i = n; i < 4; ++i) {
    ox[i] = ox[n - 1];
    oy[i] = oy[n - 1];
  }
  return true;
}

}  // namespace btg
