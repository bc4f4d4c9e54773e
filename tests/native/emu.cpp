// Host emulator of the engine's per-lane steps (test infrastructure only).
//
// Compiles beamtrace2007_b200/csrc/engine_core.cuh for the CPU and runs every
// root sequentially: admission, trace to the next clip, two-pass clip, with a
// FIFO of records instead of the GPU's warps and queues.  The pieces it
// produces must equal the reference BeamCore's (trail, no mailbox) bit for
// bit; the CUDA kernels run the same functions per lane.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <vector>

#include "bt_gpu.h"
#include "engine_core.cuh"

using namespace btg;

#define EMU_API extern "C" __attribute__((visibility("default")))

namespace {

struct Emu {
  std::vector<uint2> node;
  std::vector<float4> box, ref, triNV;
  std::vector<uint32_t> parent;
  SceneDev s;
};

struct Counters {
  Stats st;
  void add(uint64_t* out) const {
    uint64_t v[10] = {st.kdSteps, st.leafVisits, st.triTests, st.hits, st.splits,
                      st.beams, st.rootBeams, st.presplitBeams, st.fiveSplits, st.climbs};
    for (int i = 0; i < 10; ++i) out[i] += v[i];
    double d;
    memcpy(&d, &out[10], 8);
    d += st.dropped;
    memcpy(&out[10], &d, 8);
  }
};

// Output of one root: pieces (x, y, n, tri, area).
struct Piece {
  float x[4], y[4];
  int n, tri;
  float area;
};

struct RootEnv {
  std::deque<SubBeam>* q;
  std::vector<Piece>* out;
  const Query* qq;
  int app;  // 0 soft, 1 primary, 2 point
  int queued = 0;
  bool queue(const SubBeam& r) {
    q->push_back(r);
    ++queued;
    return true;
  }
  void put(const Beam& b, int tri, Stats& st) {
    Poly<4> p;
    float a = beamPoly(b, p);
    if (tri >= 0) st.hits++;
    st.beams++;
    Piece pc;
    for (int i = 0; i < 4; ++i) {
      int k = i < p.n ? i : p.n - 1;
      pc.x[i] = p.x[k];
      pc.y[i] = p.y[k];
    }
    pc.n = p.n;
    pc.tri = tri;
    pc.area = a;
    out->push_back(pc);
  }
  Stats* st;
  void occluded(const Beam& b, int tri) { put(b, tri, *st); }
  void missed(const Beam& b) { put(b, -1, *st); }
  void dropped(float) {}
};

// Traces one root to completion; appends all output pieces.
void traceRoot(const SceneDev& s, const Query& q, const Poly<8>& poly, std::vector<Piece>& out, Stats& st) {
  std::deque<SubBeam> fifo;
  RootEnv env;
  env.q = &fifo;
  env.out = &out;
  env.qq = &q;
  env.st = &st;
  admitRoot(s, q, poly, 0, env, st);
  while (!fifo.empty()) {
    SubBeam r = fifo.front();
    fifo.pop_front();
    if (r.n == 0) continue;
    Beam b;
    expand(s, q, r, b);
    Walk w;
    walkBegin(s, r, w);
    for (;;) {
      int res = advance(s, q, b, r, w, st);
      int occ = -1;
      if (res == kStepContinue) {
        for (;;) {
          res = testOne(s, q, r, b, st, occ);
          if (res != kStepContinue || !moreInLeaf(s, q, r)) break;
        }
      }
      if (res == kStepFinished) {
        env.put(b, occ >= 0 ? occ : (q.mode == kModeNearest ? b.hit : -1), st);
        break;
      }
      if (res == kStepSplit) {
        TriInfo ti;
        Line L[5];
        int nl = 0;
        bool commit = false;
        PieceLog log;
        int slots = splitPass1<RootEnv>(s, q, r, b, st, ti, L, nl, commit, &log);
        if (slots < 0) {
          out.clear();
          return;
        }
        if (!commit) {
          r.cursor += 1;
          w.phase = kPhTest;
          continue;
        }
        splitPass2(q, r, b, ti, L, nl, env, st, &log);
        break;
      }
    }
  }
}

void writePieces(const std::vector<Piece>& ps, int root, int64_t& k, int64_t cap, float* x, float* y, int32_t* n,
                 int32_t* tri, float* area, int32_t* rootOut) {
  for (const Piece& p : ps) {
    if (k < cap) {
      for (int i = 0; i < 4; ++i) {
        x[4 * k + i] = p.x[i];
        y[4 * k + i] = p.y[i];
      }
      n[k] = p.n;
      tri[k] = p.tri;
      area[k] = p.area;
      rootOut[k] = root;
    }
    ++k;
  }
}

}  // namespace

EMU_API void* emu_create(const bt_scene_desc* sc, const bt_kd_desc* kd) {
  Emu* e = new Emu();
  const int64_t nn = kd->num_nodes, nr = kd->num_refs, nt = sc->num_tris;
  e->node.resize(size_t(nn));
  e->box.resize(size_t(2 * nn));
  e->parent.assign(kd->parent, kd->parent + nn);
  for (int64_t i = 0; i < nn; ++i) {
    uint32_t d = kd->data[i], x;
    if ((d & 3u) == 3u)
      x = kd->offset[i];
    else
      memcpy(&x, &kd->split[i], 4);
    e->node[size_t(i)] = make_uint2(x, d);
    const float* b = kd->node_box + 6 * i;
    e->box[size_t(2 * i)] = make_float4(b[0], b[1], b[2], b[3]);
    e->box[size_t(2 * i + 1)] = make_float4(b[4], b[5], 0.f, 0.f);
  }
  e->ref.resize(size_t(4 * nr));
  for (int64_t k = 0; k < nr; ++k) {
    uint32_t t = kd->tri_indices[k];
    const uint32_t* vi = sc->tris + 3 * size_t(t);
    const float* p0 = sc->pos + 3 * size_t(vi[0]);
    const float* p1 = sc->pos + 3 * size_t(vi[1]);
    const float* p2 = sc->pos + 3 * size_t(vi[2]);
    const float* n = sc->tri_normals + 3 * size_t(t);
    uint32_t u[4] = {vi[0], vi[1], vi[2], t};
    float w[4];
    memcpy(w, u, 16);
    e->ref[size_t(4 * k)] = make_float4(p0[0], p0[1], p0[2], p1[0]);
    e->ref[size_t(4 * k + 1)] = make_float4(p1[1], p1[2], p2[0], p2[1]);
    e->ref[size_t(4 * k + 2)] = make_float4(p2[2], n[0], n[1], n[2]);
    e->ref[size_t(4 * k + 3)] = make_float4(w[0], w[1], w[2], w[3]);
  }
  e->triNV.resize(size_t(2 * nt));
  for (int64_t t = 0; t < nt; ++t) {
    const float* n = sc->tri_normals + 3 * t;
    const float* p0 = sc->pos + 3 * size_t(sc->tris[3 * t]);
    e->triNV[size_t(2 * t)] = make_float4(n[0], n[1], n[2], 0.f);
    e->triNV[size_t(2 * t + 1)] = make_float4(p0[0], p0[1], p0[2], 0.f);
  }
  e->s.node = e->node.data();
  e->s.box = e->box.data();
  e->s.parent = e->parent.data();
  e->s.ref = e->ref.data();
  e->s.triNV = e->triNV.data();
  for (int a = 0; a < 3; ++a) {
    e->s.bounds.lo[a] = kd->bounds[a];
    e->s.bounds.hi[a] = kd->bounds[3 + a];
  }
  e->s.numTris = int(nt);
  e->s.numNodes = uint32_t(nn);
  e->s.rootNode = 0;
  return e;
}

EMU_API void emu_destroy(void* h) { delete static_cast<Emu*>(h); }

// Soft shadows for supplied shading points: vis = miss area / light area in
// double (sum in piece order), exact G in FP64; stats accumulate.
EMU_API void emu_soft_points(void* h, const float* light, float offset, int64_t n, const int32_t* tri, const float* X,
                             const float* N, int exact, double* vis, double* G, uint64_t* stats) {
  Emu& e = *static_cast<Emu*>(h);
  V3 Lc = mk(light[0], light[1], light[2]), LU = mk(light[3], light[4], light[5]), LV = mk(light[6], light[7], light[8]);
  Counters c;
  c.st.clear();
  std::vector<Piece> out;
  for (int64_t k = 0; k < n; ++k) {
    vis[k] = -1;
    G[k] = 0;
    if (tri[k] < 0) continue;
    V3 x = mk(X[3 * k], X[3 * k + 1], X[3 * k + 2]), ns = mk(N[3 * k], N[3 * k + 1], N[3 * k + 2]);
    Query q;
    Poly<8> root;
    float lightArea;
    if (!lightBeamSetup(Lc, LU, LV, x, ns, tri[k], offset, q, root, lightArea)) {
      vis[k] = 0;
      continue;
    }
    querySetup(q, root.extent());
    out.clear();
    traceRoot(e.s, q, root, out, c.st);
    double miss = 0, g = 0;
    for (const Piece& p : out) {
      if (p.tri >= 0) continue;
      miss += double(p.area);
      if (exact) {
        V3 P[4];
        for (int i = 0; i < p.n; ++i) P[i] = planePoint(q.P, p.x[i], p.y[i]);
        g += formFactorFP64(x, ns, P, p.n);
      }
    }
    double V = miss / double(lightArea);
    vis[k] = V < 0 ? 0 : (V > 1 ? 1 : V);
    G[k] = g;
  }
  c.add(stats);
}

// Primary visibility, one root per tile: all pieces (hit and background).
EMU_API int64_t emu_primary_tiles(void* h, const bt_camera* cam, int cull, int tile, int64_t cap, float* x, float* y,
                                  int32_t* n, int32_t* tri, float* area, int32_t* root, uint64_t* stats) {
  Emu& e = *static_cast<Emu*>(h);
  V3 eye = mk(cam->eye[0], cam->eye[1], cam->eye[2]), fwd = mk(cam->fwd[0], cam->fwd[1], cam->fwd[2]);
  V3 right = mk(cam->right[0], cam->right[1], cam->right[2]), down = mk(cam->down[0], cam->down[1], cam->down[2]);
  Plane camPlane = makePlane(eye, add(eye, fwd), right, down);
  const int tilesW = (cam->W + tile - 1) / tile, tilesH = (cam->H + tile - 1) / tile;
  Counters c;
  c.st.clear();
  int64_t k = 0;
  std::vector<Piece> out;
  for (int i = 0; i < tilesW * tilesH; ++i) {
    int tx = i % tilesW, ty = i / tilesW;
    int x0 = tx * tile, y0 = ty * tile, x1 = std::min(cam->W, x0 + tile), y1 = std::min(cam->H, y0 + tile);
    float qx0 = (2 * float(x0) / float(cam->W) - 1) * cam->half_w, qx1 = (2 * float(x1) / float(cam->W) - 1) * cam->half_w;
    float qy0 = (2 * float(y0) / float(cam->H) - 1) * cam->half_h, qy1 = (2 * float(y1) / float(cam->H) - 1) * cam->half_h;
    Poly<8> p;
    p.clear();
    p.push(qx0, qy0);
    p.push(qx1, qy0);
    p.push(qx1, qy1);
    p.push(qx0, qy1);
    Query q;
    q.P = camPlane;
    q.mode = kModeNearest;
    q.farIsPlane = 0;
    q.exclude = -1;
    q.cull = cull;
    querySetup(q, p.extent());
    out.clear();
    traceRoot(e.s, q, p, out, c.st);
    writePieces(out, i, k, cap, x, y, n, tri, area, root);
  }
  c.add(stats);
  return k;
}

// Point shadows for hit polygons: the occluded pieces on each shadow plane,
// projected to the image (tri = receiver), as beamPointShadows outputs them.
EMU_API int64_t emu_point(void* h, const bt_camera* cam, const float* light, int64_t nh, const float* hx,
                          const float* hy, const int32_t* hn, const int32_t* htri, int64_t cap, float* x, float* y,
                          int32_t* n, int32_t* tri, float* area, int32_t* root, uint64_t* stats) {
  Emu& e = *static_cast<Emu*>(h);
  V3 eye = mk(cam->eye[0], cam->eye[1], cam->eye[2]), fwd = mk(cam->fwd[0], cam->fwd[1], cam->fwd[2]);
  V3 right = mk(cam->right[0], cam->right[1], cam->right[2]), down = mk(cam->down[0], cam->down[1], cam->down[2]);
  Plane camPlane = makePlane(eye, add(eye, fwd), right, down);
  V3 Lp = mk(light[0], light[1], light[2]);
  Counters c;
  c.st.clear();
  int64_t k = 0;
  std::vector<Piece> out, img;
  for (int64_t i = 0; i < nh; ++i) {
    const int T = htri[i];
    if (T < 0) continue;
    V3 nT, v0;
    triNV(e.s, T, nT, v0);
    Query q;
    Poly<8> p;
    if (!pointShadowSetup(eye, fwd, right, down, nT, v0, T, Lp, hx + 4 * i, hy + 4 * i, hn[i], q, p)) {
      Piece pc;
      for (int j = 0; j < 4; ++j) {
        pc.x[j] = hx[4 * i + j];
        pc.y[j] = hy[4 * i + j];
      }
      pc.n = hn[i];
      pc.tri = T;
      pc.area = 0;
      img.assign(1, pc);
      writePieces(img, int(i), k, cap, x, y, n, tri, area, root);
      continue;
    }
    querySetup(q, p.extent());
    out.clear();
    traceRoot(e.s, q, p, out, c.st);
    img.clear();
    for (const Piece& pc : out) {
      if (pc.tri < 0) continue;
      Piece ip;
      if (!pointShadowToImage(camPlane, q.P, pc.x, pc.y, pc.n, ip.x, ip.y)) continue;
      ip.n = pc.n;
      ip.tri = T;
      ip.area = 0;
      img.push_back(ip);
    }
    writePieces(img, int(i), k, cap, x, y, n, tri, area, root);
  }
  c.add(stats);
  return k;
}

// Round structure of the wavefront for soft-shadow points: records of round
// r run until they finish or need a clip; pieces form round r + 1.  For each
// round: records, summed work and the largest single-record work, in units of
// (kd steps + leaf visits + climbs + 4 * triangle tests).  Returns rounds.
EMU_API int emu_soft_rounds(void* h, const float* light, float offset, int64_t n, const int32_t* tri, const float* X,
                            const float* N, int maxRounds, int64_t* recs, double* work, double* maxWork,
                            double* chain) {
  Emu& e = *static_cast<Emu*>(h);
  V3 Lc = mk(light[0], light[1], light[2]), LU = mk(light[3], light[4], light[5]), LV = mk(light[6], light[7], light[8]);
  struct Rec {
    SubBeam r;
    Query q;
    double pathWork;
  };
  std::vector<Rec> cur, nxt;
  std::vector<Piece> sink;
  double longest = 0;
  for (int64_t k = 0; k < n; ++k) {
    if (tri[k] < 0) continue;
    V3 x = mk(X[3 * k], X[3 * k + 1], X[3 * k + 2]), ns = mk(N[3 * k], N[3 * k + 1], N[3 * k + 2]);
    Query q;
    Poly<8> root;
    float la;
    if (!lightBeamSetup(Lc, LU, LV, x, ns, tri[k], offset, q, root, la)) continue;
    querySetup(q, root.extent());
    std::deque<SubBeam> fifo;
    Stats st;
    st.clear();
    RootEnv env;
    env.q = &fifo;
    env.out = &sink;
    env.qq = &q;
    env.st = &st;
    admitRoot(e.s, q, root, int(k), env, st);
    for (const SubBeam& r : fifo) cur.push_back(Rec{r, q, 0});
  }
  int round = 0;
  while (!cur.empty() && round < maxRounds) {
    nxt.clear();
    double tot = 0, mx = 0;
    for (Rec& rc : cur) {
      SubBeam r = rc.r;
      const Query& q = rc.q;
      Beam b;
      expand(e.s, q, r, b);
      Walk w;
      walkBegin(e.s, r, w);
      Stats st;
      st.clear();
      std::deque<SubBeam> fifo;
      RootEnv env;
      env.q = &fifo;
      env.out = &sink;
      env.qq = &q;
      env.st = &st;
      bool split = false;
      for (;;) {
        int res = advance(e.s, q, b, r, w, st);
        int occ = -1;
        if (res == kStepContinue) {
          for (;;) {
            res = testOne(e.s, q, r, b, st, occ);
            if (res != kStepContinue || !moreInLeaf(e.s, q, r)) break;
          }
        }
        if (res == kStepFinished) break;
        if (res == kStepSplit) {
          TriInfo ti;
          Line L[5];
          int nl = 0;
          bool commit = false;
          splitPass1<RootEnv>(e.s, q, r, b, st, ti, L, nl, commit);
          if (!commit) {
            r.cursor += 1;
            w.phase = kPhTest;
            continue;
          }
          splitPass2(q, r, b, ti, L, nl, env, st);
          split = true;
          break;
        }
      }
      double wk = double(st.kdSteps + st.leafVisits + st.climbs) + 4.0 * st.triTests + (split ? 20.0 : 0.0);
      tot += wk;
      mx = wk > mx ? wk : mx;
      const double pw = rc.pathWork + wk;
      longest = pw > longest ? pw : longest;
      for (const SubBeam& c : fifo) nxt.push_back(Rec{c, q, pw});
      sink.clear();
    }
    recs[round] = int64_t(cur.size());
    work[round] = tot;
    maxWork[round] = mx;
    ++round;
    cur.swap(nxt);
  }
  *chain = longest;
  return round;
}

// One fuzzy split of a polygon (n <= 4 corners) by a line, then the
// clean-up of both pieces, with this package's polygon code (splitPoly,
// cleanPoly of beam_math.cuh): the pieces' corners and counts, and 0 if
// the splitter reported an overflow.  For the polygon fuzz test.
EMU_API int emu_split_clean(const float* px, const float* py, int n, const float* line, float eps, float* inx,
                            float* iny, int* nin, float* outx, float* outy, int* nout) {
  Poly<kPolyMax> p, in, out;
  p.n = n;
  for (int i = 0; i < n && i < kPolyMax; ++i) {
    p.x[i] = px[i];
    p.y[i] = py[i];
  }
  Line L{line[0], line[1], line[2]};
  if (!splitPoly(p, L, eps, in, out)) return 0;
  cleanPoly(in, eps);
  cleanPoly(out, eps);
  *nin = in.n;
  *nout = out.n;
  for (int i = 0; i < in.n; ++i) {
    inx[i] = in.x[i];
    iny[i] = in.y[i];
  }
  for (int i = 0; i < out.n; ++i) {
    outx[i] = out.x[i];
    outy[i] = out.y[i];
  }
  return 1;
}

// Signed area of a polygon with this package's Poly::area.
EMU_API float emu_poly_area(const float* px, const float* py, int n) {
  Poly<kPolyMax> p;
  p.n = n;
  for (int i = 0; i < n && i < kPolyMax; ++i) {
    p.x[i] = px[i];
    p.y[i] = py[i];
  }
  return p.area();
}

// The kd slab decision (decide, beam_math.cuh) for one beam -- apex O, plane
// through p0 spanned by u and v, corners (qx, qy) -- against a box and a
// split plane on `axis`: kNear 0, kFar 1, kBoth 2; -1 if the corner rays
// mix direction signs on an axis (not a pre-split piece), -2 if the split
// lies behind the apex.  Returns the plane's u, v, d (the ray at (x, y) is
// O + t (d + x u + y v)) as the decision used them.  For the kd fuzz test.
EMU_API int emu_decide(const float* O, const float* p0, const float* u, const float* v, const float* qx,
                       const float* qy, int n, int axis, float split, const float* box6, float* uvd) {
  Query q;
  memset(&q, 0, sizeof q);
  q.P = makePlane(mk(O[0], O[1], O[2]), mk(p0[0], p0[1], p0[2]), mk(u[0], u[1], u[2]), mk(v[0], v[1], v[2]));
  q.mode = kModeAnyHit;
  q.exclude = -1;
  querySetup(q, 1.f);
  const V3 vv[3] = {q.P.u, q.P.v, q.P.d};
  for (int k = 0; k < 3; ++k) {
    uvd[3 * k] = vv[k].x;
    uvd[3 * k + 1] = vv[k].y;
    uvd[3 * k + 2] = vv[k].z;
  }
  Beam b;
  memset(&b, 0, sizeof b);
  for (int i = 0; i < 4; ++i) {
    const int j = i < n ? i : n - 1;
    b.qx[i] = qx[j];
    b.qy[i] = qy[j];
  }
  b.n = n;
  int neg = 0;
  for (int c = 0; c < 3; ++c) {
    int pos = 0, negs = 0;
    for (int i = 0; i < n; ++i) {
      const float w = qx[i] * comp(q.P.u, c) + qy[i] * comp(q.P.v, c) + comp(q.P.d, c);
      pos += w > 0;
      negs += w < 0;
    }
    if (pos && negs) return -1;
    if (negs) neg |= 1 << c;
  }
  b.neg = neg;
  beamAxes(q, b);
  setStatus(q, b, -1, nullptr, 0);
  Box box;
  for (int c = 0; c < 3; ++c) {
    box.lo[c] = box6[c];
    box.hi[c] = box6[3 + c];
  }
  const bool posA = !((neg >> axis) & 1);
  const float Ns = (posA ? 1.f : -1.f) * (split - comp(q.P.O, axis));
  if (!(Ns > 0)) return -2;
  return decide(q, b, axis, Ns, box);
}
