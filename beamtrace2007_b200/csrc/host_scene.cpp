// Host side of the scene: triangle finalisation, the SAH kd-tree and the
// camera, exported through the C-ABI (include/bt_gpu.h).
//
// The beam tracer's output depends on the kd-tree (cells are visited in tree
// order) and on the per-triangle normals, so these reproduce the reference's
// host code exactly: Scene::finalize (src/scene/scene.cpp:89-118),
// KdTree::build with perfect splits and area-sorted leaves
// (src/accel/kdtree.cpp:77-338) and Camera::make (src/render/render.cpp:14-25).
// Compiled with -ffp-contract=off like the reference (CMakeLists.txt:21).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <new>
#include <vector>

#include "bt_gpu.h"
#include "kd_rules.h"
#include "kd_tree.h"

namespace {

struct F3 {
  float x, y, z;
  float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
F3 f3(float x, float y, float z) { return F3{x, y, z}; }
F3 operator-(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
F3 operator+(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
F3 operator*(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
F3 cross(F3 a, F3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
F3 normalize(F3 a) {
  float l = std::sqrt(dot(a, a));
  return l > 0 ? f3(a.x / l, a.y / l, a.z / l) : a;
}

struct Aabb {
  F3 lo{std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(),
        std::numeric_limits<float>::infinity()};
  F3 hi{-std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(),
        -std::numeric_limits<float>::infinity()};
  void expand(F3 p) {
    for (int a = 0; a < 3; ++a) {
      lo[a] = lo[a] < p[a] ? lo[a] : p[a];
      hi[a] = hi[a] > p[a] ? hi[a] : p[a];
    }
  }
  float surfaceArea() const {
    F3 d = hi - lo;
    return 2 * (d.x * d.y + d.y * d.z + d.z * d.x);
  }
};

struct TriBox {
  uint32_t tri;
  Aabb b;
};

struct KdBuild {
  const float* pos;
  const uint32_t* tris;
  const float* area;
  float costTraverse, costIntersect, emptyBonus;
  int binThreshold, bins;
  bool clipBounds, singleLeaf;
  int maxDepth;
  std::vector<float> split;
  std::vector<uint32_t> data, offset, triIndices;
  int numLeaves = 0, maxDepthReached = 0;

  F3 v(uint32_t t, int k) const {
    const float* p = pos + 3 * size_t(tris[3 * size_t(t) + size_t(k)]);
    return f3(p[0], p[1], p[2]);
  }

  // Bounds of triangle t clipped to `box`, never beyond `box` or `fallback`
  // (clippedTriangleBounds, kdtree.cpp:77-134; kd_rules.h).
  Aabb clipped(uint32_t t, const Aabb& box, const Aabb& fallback) const {
    const float* v[3];
    for (int k = 0; k < 3; ++k) v[k] = pos + 3 * size_t(tris[3 * size_t(t) + size_t(k)]);
    const kdr::Box r = kdr::clippedBounds(v[0], v[1], v[2], toBox(box), toBox(fallback));
    Aabb a;
    for (int c = 0; c < 3; ++c) {
      a.lo[c] = r.lo[c];
      a.hi[c] = r.hi[c];
    }
    return a;
  }

  static kdr::Box toBox(const Aabb& b) {
    kdr::Box r;
    for (int c = 0; c < 3; ++c) {
      r.lo[c] = b.lo[c];
      r.hi[c] = b.hi[c];
    }
    return r;
  }

  float sahCost(const Aabb& box, int axis, float s, size_t nl, size_t nr) const {
    return kdr::sahCost(kdr::Costs{costTraverse, costIntersect, emptyBonus}, toBox(box), axis, s, nl, nr);
  }

  // The cheapest split plane of `box` for `refs` (SAH, kd_rules.h): per
  // axis with extent, binned candidates above binThreshold references, else
  // every face of the references' extents (kdtree.cpp:215-285 makes the same
  // choices; a candidate replaces the best only when strictly cheaper, so
  // among equal costs the first in axis order, then plane order, stays).
  void findSplit(const std::vector<TriBox>& refs, const Aabb& box, int& bestAxis, float& bestSplit,
                 float& bestCost) const {
    if (!(box.surfaceArea() > 0)) return;
    auto offer = [&](int axis, float plane, size_t below, size_t above) {
      const float c = sahCost(box, axis, plane, below, above);
      if (c < bestCost) {
        bestCost = c;
        bestAxis = axis;
        bestSplit = plane;
      }
    };
    for (int axis = 0; axis < 3; ++axis) {
      if (!(box.hi[axis] > box.lo[axis])) continue;
      if (refs.size() > size_t(binThreshold))
        offerBinned(refs, box, axis, offer);
      else
        offerFaces(refs, box, axis, offer);
    }
  }

  // Planes between `bins` equal bins: a reference counts below a plane once
  // the bin of its low end lies below it, above while the bin of its high
  // end does not.
  template <class Offer>
  void offerBinned(const std::vector<TriBox>& refs, const Aabb& box, int axis, Offer& offer) const {
    const float lo = box.lo[axis], hi = box.hi[axis];
    const float perUnit = float(bins) / (hi - lo);
    std::vector<size_t> lowEnds(size_t(bins), 0), highEnds(size_t(bins), 0);
    for (const TriBox& r : refs) {
      ++lowEnds[size_t(kdr::binOf(r.b.lo[axis], lo, perUnit, bins))];
      ++highEnds[size_t(kdr::binOf(r.b.hi[axis], lo, perUnit, bins))];
    }
    size_t below = 0, above = refs.size();
    for (int k = 1; k < bins; ++k) {
      below += lowEnds[size_t(k - 1)];
      above -= highEnds[size_t(k - 1)];
      offer(axis, kdr::binPlane(lo, hi, k, bins), below, above);
    }
  }

  // Planes at every distinct face position strictly inside the box.  Faces
  // sort by position, and at one position closing faces before flat ones
  // (references of no extent) before opening ones; a flat reference at the
  // plane counts on both sides.
  template <class Offer>
  void offerFaces(const std::vector<TriBox>& refs, const Aabb& box, int axis, Offer& offer) const {
    enum : uint8_t { kClosing = 0, kFlat = 1, kOpening = 2 };
    struct Face {
      float at;
      uint8_t kind;
    };
    std::vector<Face> faces;
    faces.reserve(2 * refs.size());
    for (const TriBox& r : refs) {
      const float a = r.b.lo[axis], b = r.b.hi[axis];
      if (a == b) {
        faces.push_back({a, kFlat});
      } else {
        faces.push_back({a, kOpening});
        faces.push_back({b, kClosing});
      }
    }
    std::sort(faces.begin(), faces.end(),
              [](const Face& x, const Face& y) { return x.at != y.at ? x.at < y.at : x.kind < y.kind; });
    const float lo = box.lo[axis], hi = box.hi[axis];
    size_t below = 0, above = refs.size();
    for (size_t i = 0; i < faces.size();) {
      const float at = faces[i].at;
      size_t n[3] = {0, 0, 0};
      do ++n[faces[i++].kind];
      while (i < faces.size() && faces[i].at == at);
      above -= n[kClosing] + n[kFlat];
      if (at > lo && at < hi) offer(axis, at, below + n[kFlat], above + n[kFlat]);
      below += n[kOpening] + n[kFlat];
    }
  }

  void makeLeaf(size_t node, std::vector<TriBox>& refs) {
    std::sort(refs.begin(), refs.end(), [&](const TriBox& a, const TriBox& b) {
      float aa = area[a.tri], ab = area[b.tri];
      return aa != ab ? aa > ab : a.tri < b.tri;
    });
    offset[node] = uint32_t(triIndices.size());
    data[node] = (uint32_t(refs.size()) << 2) | 3u;
    for (const TriBox& r : refs) triIndices.push_back(r.tri);
    numLeaves++;
  }

  // Depth-first build: left subtree at node + 1, right child recorded in the
  // node (kdtree.cpp:142-187).
  void build(std::vector<TriBox>& refs, const Aabb& box, int depth) {
    const size_t node = split.size();
    split.push_back(0.f);
    data.push_back(3u);
    offset.push_back(0u);
    maxDepthReached = std::max(maxDepthReached, depth);
    const size_t N = refs.size();
    int bestAxis = -1;
    float bestSplit = 0, bestCost = std::numeric_limits<float>::infinity();
    if (!singleLeaf && N > 1 && depth < maxDepth) findSplit(refs, box, bestAxis, bestSplit, bestCost);
    const float leafCost = costIntersect * float(N);
    if (bestAxis < 0 || !(bestCost < leafCost)) {
      makeLeaf(node, refs);
      return;
    }
    Aabb lbox = box, rbox = box;
    lbox.hi[bestAxis] = bestSplit;
    rbox.lo[bestAxis] = bestSplit;
    std::vector<TriBox> left, right;
    left.reserve(N / 2 + 1);
    right.reserve(N / 2 + 1);
    for (const TriBox& r : refs) {
      bool goLeft, goRight, planar;
      kdr::sides(r.b.lo[bestAxis], r.b.hi[bestAxis], bestSplit, goLeft, goRight, planar);
      if (goLeft && goRight && !planar && clipBounds) {
        left.push_back({r.tri, clipped(r.tri, lbox, r.b)});
        right.push_back({r.tri, clipped(r.tri, rbox, r.b)});
      } else {
        if (goLeft) left.push_back(r);
        if (goRight) right.push_back(r);
      }
    }
    std::vector<TriBox>().swap(refs);
    build(left, lbox, depth + 1);
    std::vector<TriBox>().swap(left);
    const size_t rightIndex = split.size();
    build(right, rbox, depth + 1);
    split[node] = bestSplit;
    data[node] = (uint32_t(rightIndex) << 2) | uint32_t(bestAxis);
  }
};

}  // namespace

void kdRootAndDepth(const float* sceneBounds, const bt_kd_params& p, int64_t numTris, kdr::Box& root, int& maxDepth) {
  for (int a = 0; a < 3; ++a) {
    const float lo = sceneBounds[a], hi = sceneBounds[3 + a];
    const float pad = (hi - lo) * 1e-4f + 1e-6f;
    root.lo[a] = lo - pad;
    root.hi[a] = hi + pad;
  }
  const int N = numTris > 1 ? int(numTris) : 1;
  maxDepth = p.max_depth >= 0 ? p.max_depth : int(8 + 1.3 * std::log2(double(N)));
  maxDepth = std::min(maxDepth, 63);
}

void kdFinish(bt_kd_tree* t) {
  const size_t nn = t->split.size();
  t->parent.assign(nn, ~0u);
  t->nodeBox.assign(6 * nn, 0.f);
  if (!nn) return;
  for (int a = 0; a < 6; ++a) t->nodeBox[size_t(a)] = t->bounds[a];
  std::vector<uint32_t> stack(1, 0u);
  while (!stack.empty()) {
    const uint32_t i = stack.back();
    stack.pop_back();
    const uint32_t d = t->data[i];
    if ((d & 3u) == 3u) continue;
    const int a = int(d & 3u);
    const uint32_t l = i + 1, r = d >> 2;
    for (int k = 0; k < 6; ++k) {
      t->nodeBox[6 * size_t(l) + size_t(k)] = t->nodeBox[6 * size_t(i) + size_t(k)];
      t->nodeBox[6 * size_t(r) + size_t(k)] = t->nodeBox[6 * size_t(i) + size_t(k)];
    }
    t->nodeBox[6 * size_t(l) + 3 + size_t(a)] = t->split[i];
    t->nodeBox[6 * size_t(r) + size_t(a)] = t->split[i];
    t->parent[l] = t->parent[r] = i;
    stack.push_back(l);
    stack.push_back(r);
  }
}

extern "C" {

// Scene::finalize: drops degenerate triangles (tested in double), computes
// unit normals, areas and bounds.  Returns the number of triangles kept.
int64_t bt_scene_finalize(const float* pos, int64_t numVerts, const uint32_t* trisIn, int64_t numTrisIn,
                          uint32_t* trisOut, float* triN, float* triArea, float* bounds) {
  float lo[3] = {std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(),
                 std::numeric_limits<float>::infinity()};
  float hi[3] = {-lo[0], -lo[1], -lo[2]};
  int64_t kept = 0;
  for (int64_t i = 0; i < numTrisIn; ++i) {
    const uint32_t* t = trisIn + 3 * i;
    if (int64_t(t[0]) >= numVerts || int64_t(t[1]) >= numVerts || int64_t(t[2]) >= numVerts) return -1;
    const float* a = pos + 3 * size_t(t[0]);
    const float* b = pos + 3 * size_t(t[1]);
    const float* c = pos + 3 * size_t(t[2]);
    double e1x = double(b[0]) - a[0], e1y = double(b[1]) - a[1], e1z = double(b[2]) - a[2];
    double e2x = double(c[0]) - a[0], e2y = double(c[1]) - a[1], e2z = double(c[2]) - a[2];
    double nx = e1y * e2z - e1z * e2y, ny = e1z * e2x - e1x * e2z, nz = e1x * e2y - e1y * e2x;
    double l = std::sqrt(nx * nx + ny * ny + nz * nz);
    double scale = std::sqrt(e1x * e1x + e1y * e1y + e1z * e1z) * std::sqrt(e2x * e2x + e2y * e2y + e2z * e2z);
    if (!(l > 1e-7 * scale) || t[0] == t[1] || t[1] == t[2] || t[0] == t[2]) continue;
    for (int k = 0; k < 3; ++k) trisOut[3 * kept + k] = t[k];
    triN[3 * kept] = float(nx / l);
    triN[3 * kept + 1] = float(ny / l);
    triN[3 * kept + 2] = float(nz / l);
    triArea[kept] = float(0.5 * l);
    for (const float* p : {a, b, c})
      for (int k = 0; k < 3; ++k) {
        lo[k] = lo[k] < p[k] ? lo[k] : p[k];
        hi[k] = hi[k] > p[k] ? hi[k] : p[k];
      }
    ++kept;
  }
  for (int k = 0; k < 3; ++k) {
    bounds[k] = lo[k];
    bounds[3 + k] = hi[k];
  }
  return kept;
}

int bt_kd_build(const float* pos, const uint32_t* tris, const float* triArea, int64_t numTris, const float* sceneBounds,
                const bt_kd_params* params, bt_kd_tree** out) {
  if (!out || !pos || !tris || !triArea || numTris < 0) return BT_ERR_INVALID;
  bt_kd_params p;
  if (params) {
    p = *params;
  } else {
    bt_kd_params_default(&p);
  }
  KdBuild b;
  b.pos = pos;
  b.tris = tris;
  b.area = triArea;
  b.costTraverse = p.cost_traverse;
  b.costIntersect = p.cost_intersect;
  b.emptyBonus = p.empty_bonus;
  b.binThreshold = p.bin_threshold;
  b.bins = p.bins;
  b.clipBounds = p.clip_bounds != 0;
  b.singleLeaf = p.single_leaf != 0;
  kdr::Box rb;
  int maxDepth;
  kdRootAndDepth(sceneBounds, p, numTris, rb, maxDepth);
  Aabb root;
  for (int a = 0; a < 3; ++a) {
    root.lo[a] = rb.lo[a];
    root.hi[a] = rb.hi[a];
  }
  std::vector<TriBox> refs(static_cast<size_t>(numTris));
  for (int64_t t = 0; t < numTris; ++t) {
    Aabb bb;
    for (int k = 0; k < 3; ++k) bb.expand(b.v(uint32_t(t), k));
    refs[size_t(t)] = {uint32_t(t), bb};
  }
  b.maxDepth = maxDepth;
  try {
    b.build(refs, root, 0);
  } catch (const std::bad_alloc&) {
    return BT_ERR_NOMEM;
  }
  bt_kd_tree* t = new (std::nothrow) bt_kd_tree();
  if (!t) return BT_ERR_NOMEM;
  t->split.swap(b.split);
  t->data.swap(b.data);
  t->offset.swap(b.offset);
  t->triIndices.swap(b.triIndices);
  t->numLeaves = b.numLeaves;
  t->maxDepth = b.maxDepthReached;
  for (int a = 0; a < 3; ++a) {
    t->bounds[a] = root.lo[a];
    t->bounds[3 + a] = root.hi[a];
  }
  kdFinish(t);
  *out = t;
  return BT_OK;
}

void bt_kd_params_default(bt_kd_params* p) {
  p->cost_traverse = 1.f;
  p->cost_intersect = 0.4f;  // the beam setting of apps/bt_render.cpp:172
  p->empty_bonus = 0.8f;
  p->max_depth = -1;
  p->bin_threshold = 2048;
  p->bins = 64;
  p->clip_bounds = 1;
  p->single_leaf = 0;
}

void bt_kd_sizes(const bt_kd_tree* t, int64_t* numNodes, int64_t* numRefs, int32_t* numLeaves, int32_t* maxDepth) {
  if (numNodes) *numNodes = int64_t(t->split.size());
  if (numRefs) *numRefs = int64_t(t->triIndices.size());
  if (numLeaves) *numLeaves = t->numLeaves;
  if (maxDepth) *maxDepth = t->maxDepth;
}

void bt_kd_view(const bt_kd_tree* t, bt_kd_desc* d) {
  d->split = t->split.data();
  d->data = t->data.data();
  d->offset = t->offset.data();
  d->parent = t->parent.data();
  d->node_box = t->nodeBox.data();
  d->num_nodes = int64_t(t->split.size());
  d->tri_indices = t->triIndices.data();
  d->num_refs = int64_t(t->triIndices.size());
  for (int a = 0; a < 6; ++a) d->bounds[a] = t->bounds[a];
}

void bt_kd_free(bt_kd_tree* t) { delete t; }

// Camera::make: fwd, right, down and the half extents of the image plane at
// distance 1.
void bt_camera_make(const float* eye, const float* target, float fovY, const float* up, int32_t W, int32_t H,
                    bt_camera* c) {
  F3 e = f3(eye[0], eye[1], eye[2]), t = f3(target[0], target[1], target[2]), u = f3(up[0], up[1], up[2]);
  F3 fwd = normalize(t - e);
  F3 right = normalize(cross(fwd, u));
  F3 down = cross(fwd, right);
  for (int a = 0; a < 3; ++a) {
    c->eye[a] = e[a];
    c->fwd[a] = fwd[a];
    c->right[a] = right[a];
    c->down[a] = down[a];
  }
  c->W = W;
  c->H = H;
  c->half_h = float(std::tan(double(fovY) * M_PI / 360.0));
  c->half_w = c->half_h * float(W) / float(H);
}

}  // extern "C"
