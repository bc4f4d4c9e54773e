// The per-node arithmetic of the SAH kd-tree build, shared by the host
// build (host_scene.cpp) and the GPU build (kd_build.cu) so that both make
// the same decisions bit for bit:
//   the SAH cost of a split            KdTree::sahCost   src/accel/kdtree.cpp:189-198
//   the bin of a bound (binned SAH)     findSplit         src/accel/kdtree.cpp:222-236
//   a triangle's bounds clipped to a    clippedTriangleBounds
//   node box (perfect splits)                             src/accel/kdtree.cpp:77-134
// Host code is compiled with -ffp-contract=off and device code with
// -fmad=false, IEEE division and square root, so every operation below is
// one rounded IEEE operation in the order written.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define KD_HD __host__ __device__ __forceinline__
#else
#define KD_HD inline
#endif

namespace kdr {

struct Box {
  float lo[3], hi[3];
};

KD_HD float surfaceArea(const Box& b) {
  const float dx = b.hi[0] - b.lo[0], dy = b.hi[1] - b.lo[1], dz = b.hi[2] - b.lo[2];
  return 2 * (dx * dy + dy * dz + dz * dx);
}

struct Costs {
  float traverse, intersect, emptyBonus;
};

// Cost of splitting `box` at s on `axis` with nl / nr references each side.
KD_HD float sahCost(const Costs& k, const Box& box, int axis, float s, uint64_t nl, uint64_t nr) {
  Box l = box, r = box;
  l.hi[axis] = s;
  r.lo[axis] = s;
  const float inv = 1 / surfaceArea(box);
  float cost = k.traverse + k.intersect * (surfaceArea(l) * inv * float(nl) + surfaceArea(r) * inv * float(nr));
  if (nl == 0 || nr == 0) cost *= k.emptyBonus;
  return cost;
}

// Bin of coordinate x among B bins over [lo, hi) with scale B / (hi - lo),
// clamped to [0, B - 1].
KD_HD int binOf(float x, float lo, float scale, int B) {
  int b = int((x - lo) * scale);
  return b < 0 ? 0 : (b > B - 1 ? B - 1 : b);
}

// Candidate plane k (1 .. B-1) of the binned SAH.
KD_HD float binPlane(float lo, float hi, int k, int B) { return lo + (hi - lo) * float(k) / float(B); }

KD_HD double dmin(double a, double b) { return b < a ? b : a; }
KD_HD double dmax(double a, double b) { return a < b ? b : a; }
KD_HD double dabs(double a) { return a < 0 ? -a : a; }

// Bounds of the triangle (v0, v1, v2) clipped to `box` (Sutherland-Hodgman
// in double against the six planes), padded outward by 4 float ulps of the
// magnitudes involved, never beyond `box` or `fallback`; `fallback` when
// nothing is left.
KD_HD Box clippedBounds(const float* v0, const float* v1, const float* v2, const Box& box, const Box& fallback) {
  double poly[2][12][3];
  const float* v[3] = {v0, v1, v2};
  for (int k = 0; k < 3; ++k)
    for (int c = 0; c < 3; ++c) poly[0][k][c] = v[k][c];
  int n = 3, cur = 0;
  for (int axis = 0; axis < 3 && n > 0; ++axis) {
    for (int side = 0; side < 2 && n > 0; ++side) {
      const double plane = side == 0 ? double(box.lo[axis]) : double(box.hi[axis]);
      const double sign = side == 0 ? 1.0 : -1.0;
      int m = 0;
      for (int i = 0; i < n; ++i) {
        const double* a = poly[cur][i];
        const double* b = poly[cur][(i + 1) % n];
        const double da = sign * (a[axis] - plane), db = sign * (b[axis] - plane);
        if (da >= 0) {
          for (int c = 0; c < 3; ++c) poly[1 - cur][m][c] = a[c];
          ++m;
        }
        if ((da >= 0) != (db >= 0)) {
          const double tt = da / (da - db);
          for (int c = 0; c < 3; ++c) poly[1 - cur][m][c] = a[c] + tt * (b[c] - a[c]);
          poly[1 - cur][m][axis] = plane;
          ++m;
        }
      }
      n = m;
      cur = 1 - cur;
    }
  }
  if (n == 0) return fallback;
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      lo[c] = dmin(lo[c], poly[cur][i][c]);
      hi[c] = dmax(hi[c], poly[cur][i][c]);
    }
  Box r;
  const double ulp = 1.1920928955078125e-07;  // float epsilon, 2^-23
  for (int c = 0; c < 3; ++c) {
    const double pad = 4 * ulp * (dabs(lo[c]) + dabs(hi[c]) + double(box.hi[c] - box.lo[c]));
    r.lo[c] = float(lo[c] - pad);
    r.hi[c] = float(hi[c] + pad);
  }
  for (int a = 0; a < 3; ++a) {
    const float blo = box.lo[a] > fallback.lo[a] ? box.lo[a] : fallback.lo[a];
    const float bhi = box.hi[a] < fallback.hi[a] ? box.hi[a] : fallback.hi[a];
    r.lo[a] = r.lo[a] > blo ? r.lo[a] : blo;
    r.hi[a] = r.hi[a] < bhi ? r.hi[a] : bhi;
    if (r.lo[a] > r.hi[a]) r.lo[a] = r.hi[a];
  }
  return r;
}

// Which children a reference with bounds [lo, hi] on the split axis goes
// to (planar references at the split go to both).
KD_HD void sides(float lo, float hi, float split, bool& left, bool& right, bool& planar) {
  planar = lo == hi && lo == split;
  left = planar || lo < split;
  right = planar || hi > split;
  if (!left && !right) left = right = true;
}

}  // namespace kdr
