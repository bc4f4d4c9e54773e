// Per-sub-beam steps of the engine: expand a queued record, advance it
// through the kd-tree to its next triangle, test triangles, clip and emit
// pieces, admit a root.  Host/device code: the CUDA kernels (engine.cu) run
// these per lane; a host emulator in the tests runs them one record at a time.
//
// A sub-beam visits the same kd cells and triangles in the same order as the
// reference's BeamCore with the restart trail and no mailboxing
// (src/beam/wavefront_core.h:17-19), so its pieces are bitwise the same.
//
// Scene layout in device memory (SceneView of beam_types.h:86-97, re-laid
// for 128-bit loads):
//   node[i]    uint2  {split bits | leaf offset, data}: low 2 bits of data are
//              the axis (3 = leaf), the high bits the right child / count
//   box[i]     2 x float4 {lo.xyz, hi.x}, {hi.yz, -, -}: node boxes for the
//              restart-trail climb
//   parent[i]  uint32
//   ref[k]     4 x float4 per leaf reference, in leaf order (area-sorted):
//              {v0.xyz, v1.x} {v1.yz, v2.xy} {v2.z, n.xyz} {vi0, vi1, vi2, tri}
//   triNV[t]   2 x float4 {n.xyz, -}, {v0.xyz, -}: hit planes by triangle id
#pragma once

#include <string.h>

#if !defined(__CUDACC__)
#include <vector_functions.h>
#include <vector_types.h>
#endif

#include "beam_math.cuh"

namespace btg {

struct SceneDev {
  const uint2* node;
  const float4* box;
  const uint32_t* parent;
  const float4* ref;
  const float4* triNV;
  Box bounds;         // the kd root's box
  int numTris;
  uint32_t numNodes;
  uint32_t rootNode;  // where traversal starts (scenes after the first of a pool start further on)
};

// A queued sub-beam: 64 bytes, self-contained (corners on the root's plane,
// restart trail, kd position, root, hit, cursor in the leaf).
struct __align__(16) SubBeam {
  float qx[4], qy[4];
  unsigned long long trail;
  uint32_t node;
  int32_t root;
  int32_t hit;
  int32_t cursor;  // next triangle in the leaf; -1: descend from `node`
  int16_t depth;
  int8_t n;
  int8_t neg;
};

// Per-lane counters (TraceStats, src/util/stats.h:8-42).
struct Stats {
  uint32_t kdSteps, leafVisits, triTests, hits, splits, beams, rootBeams, presplitBeams, fiveSplits, climbs;
  uint32_t epsBand, epsFlip;  // edge votes in the fuzzy band; of those, outside it in FP64 (logging only)
  double dropped;
  BT_HD void clear() {
    kdSteps = leafVisits = triTests = hits = splits = beams = rootBeams = presplitBeams = fiveSplits = climbs = 0;
    epsBand = epsFlip = 0;
    dropped = 0;
  }
};
enum { kStKd, kStLeaf, kStTests, kStHits, kStSplits, kStBeams, kStRoots, kStPresplit, kStFive, kStClimbs,
       kStDropped, kStEpsBand, kStEpsFlip, kNumStats };

BT_HD bool isLeaf(uint2 nd) { return (nd.y & 3u) == 3u; }

BT_HD Box loadBox(const SceneDev& s, uint32_t i) {
  float4 a = s.box[2 * i], b = s.box[2 * i + 1];
  Box B;
  B.lo[0] = a.x;
  B.lo[1] = a.y;
  B.lo[2] = a.z;
  B.hi[0] = a.w;
  B.hi[1] = b.x;
  B.hi[2] = b.y;
  return B;
}

struct TriRec {
  V3 v0, v1, v2, n;
  uint32_t vi[3];
  int tri;
};

BT_HD TriRec loadRef(const SceneDev& s, uint32_t k) {
#if defined(__CUDA_ARCH__)
  const float4 a = __ldg(&s.ref[4 * k]), b = __ldg(&s.ref[4 * k + 1]), c = __ldg(&s.ref[4 * k + 2]),
               d = __ldg(&s.ref[4 * k + 3]);
#else
  const float4 a = s.ref[4 * k], b = s.ref[4 * k + 1], c = s.ref[4 * k + 2], d = s.ref[4 * k + 3];
#endif
  TriRec t;
  t.v0 = mk(a.x, a.y, a.z);
  t.v1 = mk(a.w, b.x, b.y);
  t.v2 = mk(b.z, b.w, c.x);
  t.n = mk(c.y, c.z, c.w);
  float fv[4] = {d.x, d.y, d.z, d.w};
  uint32_t u[4];
  for (int i = 0; i < 4; ++i) memcpy(&u[i], &fv[i], 4);
  t.vi[0] = u[0];
  t.vi[1] = u[1];
  t.vi[2] = u[2];
  t.tri = int(u[3]);
  return t;
}

BT_HD int refTri(const SceneDev& s, uint32_t k) {
#if defined(__CUDA_ARCH__)
  return __float_as_int(__ldg(&s.ref[4 * k + 3].w));
#else
  float f = s.ref[4 * k + 3].w;
  int t;
  memcpy(&t, &f, 4);
  return t;
#endif
}

BT_HD void triNV(const SceneDev& s, int t, V3& n, V3& v0) {
  float4 a = s.triNV[2 * t], b = s.triNV[2 * t + 1];
  n = mk(a.x, a.y, a.z);
  v0 = mk(b.x, b.y, b.z);
}

BT_HD float splitOf(uint2 nd) {
  float f;
  memcpy(&f, &nd.x, 4);
  return f;
}

// Record -> working beam (wfExpand, wavefront_core.h:92-112).
BT_HD void expand(const SceneDev& s, const Query& q, const SubBeam& r, Beam& b) {
  const int n = r.n, l3 = n > 3 ? 3 : 2;
  for (int i = 0; i < 3; ++i) {
    b.qx[i] = r.qx[i];
    b.qy[i] = r.qy[i];
  }
  b.qx[3] = l3 == 3 ? r.qx[3] : r.qx[2];
  b.qy[3] = l3 == 3 ? r.qy[3] : r.qy[2];
  b.n = n;
  b.neg = r.neg;
  beamAxes(q, b);
  if (r.hit >= 0) {
    V3 nT, v0;
    triNV(s, r.hit, nT, v0);
    hitPlane(q, nT, v0, b.hitA, b.hitC);
    b.hitN = nT;
    setStatus(q, b, r.hit, b.hitA, b.hitC);
  } else {
    b.hitA[0] = b.hitA[1] = b.hitA[2] = b.hitC = 0;
    b.hitN = mk(0, 0, 0);
    setStatus(q, b, -1, nullptr, 0);
  }
}

BT_HD void storeGeom(const Beam& b, SubBeam& r) {
  r.n = int8_t(b.n);
  for (int i = 0; i < 4; ++i) {
    r.qx[i] = b.qx[i];
    r.qy[i] = b.qy[i];
  }
  r.neg = int8_t(b.neg);
}

enum { kStepFinished = 0, kStepSplit = 1, kStepContinue = 2 };
enum { kPhDescend = 0, kPhTest = 1, kPhClimb = 2 };

// Where a record is in the per-lane state machine (WfStepState).
struct Walk {
  int phase;
  Box box;
};

BT_HD void walkBegin(const SceneDev& s, const SubBeam& r, Walk& w) {
  if (r.cursor < 0) {
    w.phase = kPhDescend;
    w.box = loadBox(s, r.node);
  } else {
    w.phase = kPhTest;
  }
}

BT_HD int highestBit64(unsigned long long x) {
#if defined(__CUDA_ARCH__)
  return 63 - __clzll((long long)x);
#else
  return 63 - __builtin_clzll(x);
#endif
}

// Ancestors of the current kd node for the restart-trail climb: parent
// links one level at a time, as the reference walks them.  (The step
// functions take the walk as a parameter so that a cache of the current
// path can stand in for it; the climb counter counts levels either way.)
struct ParentClimb {
  BT_HD void begin(int) {}
  BT_HD void descend(int, uint32_t) {}
  BT_HD uint32_t ancestor(const SceneDev& s, uint32_t node, int depth, int d) {
    for (; depth > d; --depth) node = s.parent[node];
    return node;
  }
};

// One node visit of the descent (the inner loop of wfAdvance,
// wavefront_core.h:163-189): a kd step into the child the beam enters
// (false), or the leaf is reached (true: cursor 0, leaf counted).  `nd`
// holds the current node's record on entry and the entered child's on
// return: both children are loaded while the slab test runs, so the next
// step does not wait for its load.
template <class Anc>
BT_HD bool descendStep(const SceneDev& s, const Query& q, const Beam& B, SubBeam& r, Walk& w, Stats& st, Anc& anc,
                       uint2& nd) {
  if (isLeaf(nd)) {
    r.cursor = 0;
    st.leafVisits++;
    return true;
  }
  st.kdSteps++;
  const int d = r.depth++;
  anc.descend(d, r.node);
  const int a = int(nd.y & 3u);
  const float sp = splitOf(nd);
  const bool pos = !((B.neg >> a) & 1);
  const float Ns = (pos ? 1.f : -1.f) * (sp - comp(q.P.O, a));
  const uint32_t left = r.node + 1, right = nd.y >> 2;
  const uint2 ndLeft = s.node[left], ndRight = s.node[right];
  const uint32_t cs = pos ? right : left, co = pos ? left : right;
  int dec = kFar;
  if (Ns > 0) dec = decide(q, B, a, Ns, w.box);
  // the child entered is the right one (lo[a] = split) or the left one (hi[a] = split)
  const bool goRight = dec == kFar ? pos : !pos;
  if (dec == kBoth) r.trail |= 1ull << d;
  r.node = dec == kFar ? cs : co;
  nd = goRight ? ndRight : ndLeft;
  if (goRight)
    boxSetLo(w.box, a, sp);
  else
    boxSetHi(w.box, a, sp);
  return false;
}

// One pop of the restart trail (wfAdvance's climb, wavefront_core.h:
// 204-229): the deepest pending far child is entered if the beam overlaps
// its box (kClimbDescend, w.box set), skipped (kClimbNext), or nothing is
// pending (kClimbFinished).
enum { kClimbFinished = 0, kClimbDescend = 1, kClimbNext = 2 };
template <class Anc>
BT_HD int climbStep(const SceneDev& s, const Query& q, const Beam& B, SubBeam& r, Walk& w, Stats& st, Anc& anc) {
  if (r.trail == 0) return kClimbFinished;
  const int d = highestBit64(r.trail);
  const uint32_t node = anc.ancestor(s, r.node, r.depth, d);
  st.climbs += uint32_t(r.depth - d);
  r.trail &= (1ull << d) - 1;
  const uint2 nd = s.node[node];
  const uint32_t cs = ((B.neg >> (nd.y & 3u)) & 1) ? node + 1 : (nd.y >> 2);
  r.node = node;
  r.depth = int16_t(d);
  const Box cb = loadBox(s, cs);
  if (!overlaps(q, B, cb)) return kClimbNext;
  r.node = cs;
  r.depth = int16_t(d + 1);
  r.cursor = -1;
  w.box = cb;
  return kClimbDescend;
}

// True if the leaf has another triangle to test (skipping the excluded one)
// (wfMoreInLeaf, wavefront_core.h:272-279).
BT_HD bool moreInLeaf(const SceneDev& s, const Query& q, SubBeam& r) {
  const uint2 leaf = s.node[r.node];
  const uint32_t cnt = leaf.y >> 2;
  uint32_t i = uint32_t(r.cursor);
  while (i < cnt && refTri(s, leaf.x + i) == q.exclude) ++i;
  r.cursor = int32_t(i);
  return i < cnt;
}

// Descends to the next leaf / climbs to the next pending far child until a
// triangle is pending (kStepContinue, phase kPhTest) or no cell is left
// (kStepFinished: the caller outputs the beam) (wfAdvance,
// wavefront_core.h:157-231).
template <class Anc>
BT_HD int advance(const SceneDev& s, const Query& q, const Beam& B, SubBeam& r, Walk& w, Stats& st, Anc& anc) {
  for (;;) {
    if (w.phase == kPhDescend) {
      uint2 nd = s.node[r.node];
      while (!descendStep(s, q, B, r, w, st, anc, nd)) {
      }
      w.phase = kPhTest;
    }
    if (w.phase == kPhTest) {
      if (moreInLeaf(s, q, r)) return kStepContinue;
      w.phase = kPhClimb;
    }
    for (;;) {
      const int c = climbStep(s, q, B, r, w, st, anc);
      if (c == kClimbFinished) return kStepFinished;
      if (c == kClimbDescend) {
        w.phase = kPhDescend;
        break;
      }
    }
  }
}

BT_HD int advance(const SceneDev& s, const Query& q, const Beam& B, SubBeam& r, Walk& w, Stats& st) {
  ParentClimb anc;
  return advance(s, q, B, r, w, st, anc);
}


BT_HD V3 edgePlane(const V3* r, const uint32_t* T, int i, int j) {
  return T[i] < T[j] ? cross(r[i], r[j]) : neg(cross(r[j], r[i]));
}

BT_CLIP void setupRef(const SceneDev& s, const Query& q, uint32_t k, TriInfo& ti) {
  TriRec t = loadRef(s, k);
  triSetup(q, t.v0, t.v1, t.v2, t.n, t.vi, t.tri, ti);
}

// setupRef and the FP64 twins of the edge lines (the eps_fp64 clip).
BT_COLD void setupRef64(const SceneDev& s, const Query& q, uint32_t k, TriInfo& ti, Line64* e64) {
  TriRec t = loadRef(s, k);
  triSetup(q, t.v0, t.v1, t.v2, t.n, t.vi, t.tri, ti);
  e64[0].ok = e64[1].ok = e64[2].ok = 0;
  if (!ti.ok) return;
  const V3 m0 = edgePlane(ti.r, t.vi, 0, 1);
  const float sg = dot(ti.r[2], m0) > 0 ? 1.f : -1.f;  // triSetup's orientation sign
  edgeLines64(q, t.v0, t.v1, t.v2, t.vi, sg, ti.edge, e64);
}

// How an edge vote treats beam corners inside the fuzzy band: as the
// reference does (float); the same, counting the band corners and their
// FP64 re-evaluation (eps_stats); re-deciding them in FP64 (eps_fp64).
enum VoteMode { kVoteFloat = 0, kVoteLog = 1, kVoteFp64 = 2 };

// Tests the pending triangle (wfTestOne, wavefront_core.h:236-268).
// kStepFinished: AnyHit beam fully occluded by `occluder` (caller outputs
// it); kStepSplit: triangle `cursor` needs a clip.
BT_HD bool voteLine(const Query& q, const Beam& B, const Line& line, bool& allIn) {
  bool anyIn = false, anyOut = false;
  for (int k = 0; k < 4; ++k) {
    float dv = B.qx[k] * line.a + B.qy[k] * line.b + line.c;
    anyIn |= dv > q.eps;
    anyOut |= dv < -q.eps;
  }
  if (anyOut) allIn = false;
  return anyIn;
}

// The tests after the three edges (depth line, far plane, inside, beam side)
// of BeamCtx::classifyTri (beam_core.h:386-408); ti holds the full setup.
BT_HD int classifyAfterEdges(const Query& q, const Beam& B, const TriInfo& ti, bool allIn) {
  if (q.mode == kModeNearest && B.hit >= 0) {
    if (!voteLine(q, B, closerLine(q, ti, B.hitA, B.hitC, B.hitN, B.hit), allIn)) return kTriKeep;
  }
  if (q.farIsPlane) {
    const float farA[3] = {0.f, 0.f, q.farCq};
    if (!voteLine(q, B, closerLine(q, ti, farA, q.farCq, q.P.n, -1), allIn)) return kTriKeep;
  }
  if (allIn) return kTriAllIn;
  if (separated(q, B, ti)) return kTriKeep;
  return kTriClip;
}

// Disagreement logging for one edge vote: corners whose float distance to
// the edge line falls inside the fuzzy band (+-eps, where the vote counts
// neither side) and, of those, corners that the same line evaluated in
// FP64 -- from the float vertices and apex, in the same canonical
// orientation -- places outside the band.  Decisions stay the float ones;
// the FP64 line is computed only when a corner is in the band.
BT_HD void logBand(const Query& q, const Beam& B, const Line& L, const TriRec& t, int i, int j, float sg, Stats& st) {
  int band = 0;
  bool in[4];
  for (int k = 0; k < 4; ++k) {
    const float dv = B.qx[k] * L.a + B.qy[k] * L.b + L.c;
    in[k] = k < B.n && !(dv > q.eps) && !(dv < -q.eps);
    band += in[k];
  }
  if (!band) return;
  st.epsBand += uint32_t(band);
  const V3 vf[3] = {t.v0, t.v1, t.v2};
  double ri[3], rj[3];
  for (int a = 0; a < 3; ++a) {
    ri[a] = double(comp(vf[i], a)) - double(comp(q.P.O, a));
    rj[a] = double(comp(vf[j], a)) - double(comp(q.P.O, a));
  }
  const bool fwd = t.vi[i] < t.vi[j];
  const double* p0 = fwd ? ri : rj;
  const double* p1 = fwd ? rj : ri;
  double m[3] = {p0[1] * p1[2] - p0[2] * p1[1], p0[2] * p1[0] - p0[0] * p1[2], p0[0] * p1[1] - p0[1] * p1[0]};
  if (!fwd)
    for (int a = 0; a < 3; ++a) m[a] = -m[a];
  const double a = sg * (m[0] * q.P.u.x + m[1] * q.P.u.y + m[2] * q.P.u.z);
  const double b = sg * (m[0] * q.P.v.x + m[1] * q.P.v.y + m[2] * q.P.v.z);
  const double c = sg * (m[0] * q.P.d.x + m[1] * q.P.d.y + m[2] * q.P.d.z);
  const double nrm = sqrt(a * a + b * b);
  if (!(nrm > 0)) return;
  for (int k = 0; k < 4; ++k) {
    if (!in[k]) continue;
    const double dv = (double(B.qx[k]) * a + double(B.qy[k]) * b + c) / nrm;
    if (dv > double(q.eps) || dv < -double(q.eps)) st.epsFlip++;
  }
}

// voteLine with the corners inside the float band re-decided by the FP64
// edge line from vertex i to j of t (computed only when a corner is in the
// band); counts the band corners and those the FP64 line re-decides.
BT_HD bool voteLine64(const Query& q, const Beam& B, const Line& L, const TriRec& t, int i, int j, float sg,
                      bool& allIn, Stats& st) {
  bool anyIn = false, anyOut = false;
  bool in[4];
  int band = 0;
  for (int k = 0; k < 4; ++k) {
    const float dv = B.qx[k] * L.a + B.qy[k] * L.b + L.c;
    in[k] = !(dv > q.eps) && !(dv < -q.eps);
    anyIn |= dv > q.eps;
    anyOut |= dv < -q.eps;
    band += in[k];
  }
  if (band) {
    const V3 vf[3] = {t.v0, t.v1, t.v2};
    const Line64 e = edgeLine64(q, vf[i], vf[j], t.vi[i] < t.vi[j], sg, L);
    st.epsBand += uint32_t(band);
    if (e.ok)
      for (int k = 0; k < 4; ++k) {
        if (!in[k]) continue;
        const double d = e.eval(B.qx[k], B.qy[k]);
        if (d > double(q.eps)) {
          anyIn = true;
          st.epsFlip++;
        } else if (d < -double(q.eps)) {
          anyOut = true;
          st.epsFlip++;
        }
      }
  }
  if (anyOut) allIn = false;
  return anyIn;
}

template <int Mode = kVoteFloat>
BT_HD int testOne(const SceneDev& s, const Query& q, SubBeam& r, Beam& B, Stats& st, int& occluder) {
  constexpr bool EpsLog = Mode == kVoteLog, F64 = Mode == kVoteFp64;
  const uint2 leaf = s.node[r.node];
  const uint32_t i = uint32_t(r.cursor);
  r.cursor = int32_t(i + 1);
  // Triangle setup as BeamCtx::triSetup (beam_core.h:260-286) computes it,
  // but the edge lines one at a time: the test stops at the first edge that
  // separates (trivial case (a), the usual outcome).  Every value is
  // computed exactly as in the full setup, so outcomes are identical.
  const TriRec t = loadRef(s, leaf.x + i);
  TriInfo ti;
  ti.tri = t.tri;
  ti.r[0] = sub(t.v0, q.P.O);
  ti.r[1] = sub(t.v1, q.P.O);
  ti.r[2] = sub(t.v2, q.P.O);
  const V3 m0 = edgePlane(ti.r, t.vi, 0, 1);
  const float D = dot(ti.r[2], m0);
  if (!notEdgeOn(D, m0, ti.r[2])) return kStepContinue;  // edge-on: not a test
  if (q.cull && D > 0) return kStepContinue;                        // back-facing
  st.triTests++;
  if (B.hit == t.tri) return kStepContinue;
  const float sg = D > 0 ? 1.f : -1.f;
  bool allIn = true;
  ti.edge[0] = makeLine(sg * dot(m0, q.P.u), sg * dot(m0, q.P.v), sg * dot(m0, q.P.d), q.ext);
  if (EpsLog) logBand(q, B, ti.edge[0], t, 0, 1, sg, st);
  if (F64 ? !voteLine64(q, B, ti.edge[0], t, 0, 1, sg, allIn, st) : !voteLine(q, B, ti.edge[0], allIn))
    return kStepContinue;
  const V3 m1 = edgePlane(ti.r, t.vi, 1, 2);
  ti.edge[1] = makeLine(sg * dot(m1, q.P.u), sg * dot(m1, q.P.v), sg * dot(m1, q.P.d), q.ext);
  if (EpsLog) logBand(q, B, ti.edge[1], t, 1, 2, sg, st);
  if (F64 ? !voteLine64(q, B, ti.edge[1], t, 1, 2, sg, allIn, st) : !voteLine(q, B, ti.edge[1], allIn))
    return kStepContinue;
  const V3 m2 = edgePlane(ti.r, t.vi, 2, 0);
  ti.edge[2] = makeLine(sg * dot(m2, q.P.u), sg * dot(m2, q.P.v), sg * dot(m2, q.P.d), q.ext);
  if (EpsLog) logBand(q, B, ti.edge[2], t, 2, 0, sg, st);
  if (F64 ? !voteLine64(q, B, ti.edge[2], t, 2, 0, sg, allIn, st) : !voteLine(q, B, ti.edge[2], allIn))
    return kStepContinue;
  ti.n = t.n;
  ti.A[0] = dot(t.n, q.P.u);
  ti.A[1] = dot(t.n, q.P.v);
  ti.A[2] = dot(t.n, q.P.d);
  ti.C = dot(t.n, ti.r[0]);
  ti.ok = 1;
  const int res = classifyAfterEdges(q, B, ti, allIn);
  if (res == kTriKeep) return kStepContinue;
  if (res == kTriAllIn) {
    if (q.mode == kModeAnyHit) {
      occluder = t.tri;
      return kStepFinished;
    }
    setStatus(q, B, t.tri, ti.A, ti.C);
    B.hitA[0] = ti.A[0];
    B.hitA[1] = ti.A[1];
    B.hitA[2] = ti.A[2];
    B.hitC = ti.C;
    B.hitN = ti.n;
    r.hit = t.tri;
    return kStepContinue;
  }
  r.cursor = int32_t(i);
  return kStepSplit;
}

// Sink of clipTri's first pass: the area of the pieces that take the new
// status (wfSplitClip's commit rule, wavefront_core.h:350-363), and the
// number of queue slots the pieces would take.
struct AreaSink {
  float newArea;
  int slots0, slots1;
  BT_HD bool push(int l, const Poly<kPolyMax>& p, bool) {
    if (p.n > 5) return false;
    if (l == 1)
      newArea += p.area();
    if (l == 0)
      slots0 += p.n == 5 ? 2 : 1;
    else
      slots1 += p.n == 5 ? 2 : 1;
    return true;
  }
};

// Sink of the second pass: each piece (pentagons split into quad and
// triangle) becomes a beam; queued pieces continue at the next triangle of
// the leaf with their new status, AnyHit occluded pieces are output
// (wfSplitEmit, wavefront_core.h:370-422).  Env provides
//   queue(const SubBeam&)                a continuing piece
//   occluded(const Beam&, int tri)       an AnyHit piece hidden by tri
//   dropped(float area)                  a sliver below minArea
template <class Env>
struct EmitSink {
  const Query* q;
  const SubBeam* base;
  const Beam* parent;
  int t;
  Env* env;
  Stats* st;
  BT_HD void one(bool hitNow, bool queued, const Poly<kPolyMax>& piece, bool clean) {
    Beam nb;
    float dropped = 0;
    if (!beamGeom(*q, piece, parent->neg, nb, dropped, clean)) {
      st->dropped += double(dropped);
      env->dropped(dropped);
      return;
    }
    if (!queued) {
      env->occluded(nb, t);
      return;
    }
    SubBeam pr = *base;
    storeGeom(nb, pr);
    pr.hit = hitNow ? t : parent->hit;
    env->queue(pr);
  }
  BT_HD bool push(int l, const Poly<kPolyMax>& p0, bool clean) {
    const bool hitNow = l == 1;
    const bool queued = !(hitNow && q->mode == kModeAnyHit);
    if (p0.n == 5) {
      Poly<kPolyMax> a, b;
      splitFive(p0, a, b);
      st->fiveSplits++;
      one(hitNow, queued, a, false);
      one(hitNow, queued, b, false);
    } else {
      one(hitNow, queued, p0, clean);
    }
    return true;
  }
};

// The pieces of pass 1 in push order, so that pass 2 can emit them without
// clipping again (pieces have at most 5 corners; a clip with more than
// kPieceLog pieces is replayed instead).  The engine keeps one per clipping
// thread in shared memory, 436 bytes each.
constexpr int kPieceLog = 10;
struct PieceLog {
  int count;
  int8_t level[kPieceLog], n[kPieceLog], clean[kPieceLog];
  float x[kPieceLog][5], y[kPieceLog][5];
  BT_HD void add(int l, const Poly<kPolyMax>& p, bool isClean) {
    if (count < kPieceLog) {
      level[count] = int8_t(l);
      n[count] = int8_t(p.n);
      clean[count] = int8_t(isClean);
      BT_UNROLL for (int i = 0; i < 5; ++i) {
        x[count][i] = i < p.n ? p.x[i] : 0.f;
        y[count][i] = i < p.n ? p.y[i] : 0.f;
      }
    }
    ++count;
  }
};

// One clipper instance per environment: measure (pass 1, optionally
// logging the pieces) or emit (pass 2).
template <class Env>
struct ClipSink {
  int emitting;
  AreaSink area;
  EmitSink<Env> emit;
  PieceLog* log;
  BT_HD bool push(int l, const Poly<kPolyMax>& p, bool clean) {
    if (emitting) return emit.push(l, p, clean);
    if (!area.push(l, p, clean)) return false;
    if (log) log->add(l, p, clean);
    return true;
  }
};

// Clip of a record whose pending triangle needs it (after testOne returned
// kStepSplit).  Pass 1 decides whether any piece measurably changes status
// and counts queue slots; pass 2 (only if it does) replays the same clip and
// streams the pieces to env.  Returns -1 if the clip overflowed its fixed
// lists (the root must be abandoned), else the slots pass 2 will use
// (0 if nothing changes: the record continues unchanged at cursor + 1).
template <class Env, bool F64 = false>
BT_CLIP int splitPass1(const SceneDev& s, const Query& q, const SubBeam& r, const Beam& B, Stats& st, TriInfo& ti,
                       Line* L, int& nl, bool& commit, PieceLog* log = nullptr, Line64* e64 = nullptr) {
  const uint2 leaf = s.node[r.node];
  if (F64)
    setupRef64(s, q, leaf.x + uint32_t(r.cursor), ti, e64);
  else
    setupRef(s, q, leaf.x + uint32_t(r.cursor), ti);
  classifyTri<F64>(q, B, ti, L, nl, e64, false);  // the lines only: the trace step classified it
  ClipSink<Env> sink;
  sink.emitting = 0;
  sink.area = AreaSink{0.f, 0, 0};
  sink.log = log;
  if (log) log->count = 0;
  uint32_t five = 0;
  if (!clipTri<kPolyMax, ClipSink<Env>, F64>(q, B, L, nl, sink, five, e64)) return -1;
  st.fiveSplits += five;
  commit = sink.area.newArea >= q.minArea;
  if (!commit) return 0;
  return sink.area.slots0 + (q.mode == kModeAnyHit ? 0 : sink.area.slots1);
}

// Pass 2 of a clip whose pieces overflowed the log: the clip again, out of
// line (rare), with the pieces streamed to emit.
template <class Env, bool F64>
BT_COLD void replayClip(const Query& q, const Beam& B, Line* L, int nl, const EmitSink<Env>& emit,
                        const Line64* e64) {
  ClipSink<Env> sink;
  sink.emitting = 1;
  sink.emit = emit;
  sink.log = nullptr;
  uint32_t five = 0;  // counted in pass 1
  clipTri<kPolyMax, ClipSink<Env>, F64>(q, B, L, nl, sink, five, e64);
}

template <class Env, bool F64 = false>
BT_CLIP void splitPass2(const Query& q, const SubBeam& r, const Beam& B, const TriInfo& ti, Line* L, int nl, Env& env,
                        Stats& st, const PieceLog* log = nullptr, const Line64* e64 = nullptr) {
  st.splits++;
  SubBeam base = r;
  base.cursor = r.cursor + 1;
  EmitSink<Env> emit{&q, &base, &B, ti.tri, &env, &st};
  if (log && log->count <= kPieceLog) {
    // the same pieces in the same order as a replayed clip would push them
    for (int k = 0; k < log->count; ++k) {
      Poly<kPolyMax> p;
      p.n = log->n[k];
      BT_UNROLL for (int i = 0; i < kPolyMax; ++i) {
        p.x[i] = i < 5 ? log->x[k][i] : 0.f;
        p.y[i] = i < 5 ? log->y[k][i] : 0.f;
      }
      emit.push(log->level[k], p, log->clean[k] != 0);
    }
    return;
  }
  replayClip<Env, F64>(q, B, L, nl, emit, e64);
}

// Root admission: pre-split pieces become records at the kd root; pieces
// missing the scene box are output at once (wfAdmit, wavefront_core.h:428-471).
// Env provides queue / missed(const Beam&) / dropped.
template <class Env>
struct AdmitEmit {
  const SceneDev* s;
  const Query* q;
  int root;
  Env* env;
  Stats* st;
  BT_HD bool piece(const Poly<8>& p, int negBits) {
    Beam b;
    float dropped = 0;
    if (!beamGeom(*q, p, negBits, b, dropped)) {
      st->dropped += double(dropped);
      env->dropped(dropped);
      return true;
    }
    b.hitA[0] = b.hitA[1] = b.hitA[2] = b.hitC = 0;
    b.hitN = mk(0, 0, 0);
    setStatus(*q, b, -1, nullptr, 0);
    st->rootBeams++;
    if (!overlaps(*q, b, s->bounds)) {
      env->missed(b);
      return true;
    }
    SubBeam r;
    storeGeom(b, r);
    r.trail = 0;
    r.node = s->rootNode;
    r.root = root;
    r.hit = -1;
    r.cursor = -1;
    r.depth = 0;
    return env->queue(r);
  }
  BT_HD void presplit() { st->presplitBeams++; }
  BT_HD void dropped(float a) {
    st->dropped += double(a);
    env->dropped(a);
  }
};

template <class Env>
BT_COLD bool admitRoot(const SceneDev& s, const Query& q, const Poly<8>& rootPoly, int root, Env& env, Stats& st) {
  Poly<8> p = rootPoly;
  if (p.n < 3) return true;
  if (p.area() < 0) p.reverse();
  AdmitEmit<Env> e{&s, &q, root, &env, &st};
  return presplit(q, p, e);
}

// Final piece polygon and area (wfOutput, wavefront_core.h:125-132).
BT_HD float beamPoly(const Beam& b, Poly<4>& p) {
  p.n = b.n;
  for (int i = 0; i < b.n; ++i) {
    p.x[i] = b.qx[i];
    p.y[i] = b.qy[i];
  }
  return p.area();
}

// Lambert's formula over a visible light piece, in FP64 from the piece's
// float corners on the light plane (the exact term of soft_core.h:18-33).
BT_COLD double formFactorFP64(V3 x, V3 n, const V3* P, int count) {
  double sum = 0;
  for (int i = 0; i < count; ++i) {
    V3 pa = P[i], pb = P[i + 1 == count ? 0 : i + 1];
    double ax = double(pa.x) - double(x.x), ay = double(pa.y) - double(x.y), az = double(pa.z) - double(x.z);
    double bx = double(pb.x) - double(x.x), by = double(pb.y) - double(x.y), bz = double(pb.z) - double(x.z);
    double la = sqrt(ax * ax + ay * ay + az * az), lb = sqrt(bx * bx + by * by + bz * bz);
    if (la == 0 || lb == 0) continue;
    double c = (ax * bx + ay * by + az * bz) / (la * lb);
    c = c < -1 ? -1 : (c > 1 ? 1 : c);
    double theta = acos(c);
    double gx = ay * bz - az * by, gy = az * bx - ax * bz, gz = ax * by - ay * bx;
    double lg = sqrt(gx * gx + gy * gy + gz * gz);
    if (lg == 0) continue;
    sum += theta * (gx * double(n.x) + gy * double(n.y) + gz * double(n.z)) / lg;
  }
  return (sum < 0 ? -sum : sum) * 0.5;
}

}  // namespace btg
