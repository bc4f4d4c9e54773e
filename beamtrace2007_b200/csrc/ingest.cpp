// Scene ingest: scene configs, OBJ and PLY meshes and the procedural
// scenes, exported through the C-ABI (include/bt_gpu.h, bt_scene_file_*).
//
// A config names meshes and views; the scene built from it must be the one
// the reference builds from the same file, vertex for vertex, since the kd
// tree and every beam depend on the float coordinates.  So the parser, the
// loaders and the generators follow the reference's arithmetic in its
// order and in single precision (its float build):
//   parseConfig / loadConfig / buildScene   src/scene/scene.cpp:127-262
//   loadOBJ / loadPLY                       src/scene/loaders.cpp:29-240
//   buildProcedural and its scenes          src/scene/procedural.cpp:17-226
//   addQuad / addBox / addSphere            src/scene/scene.cpp:44-87
//   Scene::finalize                         src/scene/scene.cpp:8-42
//   Rng (PCG32), splitWS, trim              src/util/misc.h:24-46, misc.cpp
// Compiled with -ffp-contract=off like the reference.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "bt_gpu.h"

void btSetError(const char* msg);  // engine.cu: the message bt_gpu_last_error returns

namespace {

struct V {
  float x = 0, y = 0, z = 0;
  V() {}
  V(float a, float b, float c) : x(a), y(b), z(c) {}
};
V operator+(V a, V b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
V operator-(V a, V b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
V operator*(V a, float s) { return V(a.x * s, a.y * s, a.z * s); }
float dot(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V cross(V a, V b) { return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
V unit(V a) {
  const float l = std::sqrt(dot(a, a));
  return l > 0 ? V(a.x / l, a.y / l, a.z / l) : a;
}
// a unit vector orthogonal to the unit vector n (anyOrthogonal, src/core/vec.h)
V orthogonalTo(V n) {
  const V a = std::fabs(n.x) < 0.6f ? V(1, 0, 0) : (std::fabs(n.y) < 0.6f ? V(0, 1, 0) : V(0, 0, 1));
  return unit(cross(n, a));
}

// PCG32 (O'Neill 2014): the published generator, with the reference's seeding
// and its 27-bit [0, 1) mapping.
class Pcg32 {
 public:
  explicit Pcg32(uint64_t seed) {
    inc_ = (0xda3e39cb94b95bdbULL << 1u) | 1u;
    step();
    state_ += seed;
    step();
  }
  double uniform() { return (step() >> 5) * (1.0 / 134217728.0); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }

 private:
  uint32_t step() {
    const uint64_t s = state_;
    state_ = s * 6364136223846793005ULL + inc_;
    const uint32_t x = uint32_t(((s >> 18u) ^ s) >> 27u);
    const uint32_t r = uint32_t(s >> 59u);
    return (x >> r) | (x << ((-r) & 31));
  }
  uint64_t state_ = 0, inc_ = 0;
};

std::vector<std::string> words(const std::string& s) {
  std::vector<std::string> out;
  std::istringstream is(s);
  std::string t;
  while (is >> t) out.push_back(t);
  return out;
}

std::string stripped(const std::string& s) {
  const size_t a = s.find_first_not_of(" \t\r\n");
  if (a == std::string::npos) return "";
  return s.substr(a, s.find_last_not_of(" \t\r\n") - a + 1);
}

struct Mesh {
  std::vector<V> pos;
  std::vector<uint32_t> tris;  // 3 per triangle
  std::vector<uint16_t> mat;
  std::vector<V> colors;

  uint32_t vert(V p) {
    pos.push_back(p);
    return uint32_t(pos.size() - 1);
  }
  void tri(uint32_t a, uint32_t b, uint32_t c, uint16_t m) {
    tris.insert(tris.end(), {a, b, c});
    mat.push_back(m);
  }
  uint16_t material(V c) {
    colors.push_back(c);
    return uint16_t(colors.size() - 1);
  }

  void quad(V a, V b, V c, V d, uint16_t m) {
    const uint32_t i = vert(a), j = vert(b), k = vert(c), l = vert(d);
    tri(i, j, k, m);
    tri(i, k, l, m);
  }

  // Axis box on 8 shared corners (corner k takes hi on the axes of its set
  // bits); faces counter-clockwise seen from outside, or from inside.
  void box(V lo, V hi, uint16_t m, bool inward = false) {
    static const int kFaces[6][4] = {{0, 4, 6, 2}, {1, 3, 7, 5}, {0, 1, 5, 4},
                                     {2, 6, 7, 3}, {0, 2, 3, 1}, {4, 5, 7, 6}};
    uint32_t c[8];
    for (int k = 0; k < 8; ++k) c[k] = vert(V(k & 1 ? hi.x : lo.x, k & 2 ? hi.y : lo.y, k & 4 ? hi.z : lo.z));
    for (const auto& f : kFaces) {
      if (inward) {
        tri(c[f[0]], c[f[2]], c[f[1]], m);
        tri(c[f[0]], c[f[3]], c[f[2]], m);
      } else {
        tri(c[f[0]], c[f[1]], c[f[2]], m);
        tri(c[f[0]], c[f[2]], c[f[3]], m);
      }
    }
  }

  // UV sphere: poles, then (stacks - 1) rings of `slices` vertices; pole
  // fans interleaved per slice, then the bands.
  void sphere(V c, float r, int stacks, int slices, uint16_t m) {
    stacks = std::max(stacks, 2);
    slices = std::max(slices, 3);
    const uint32_t north = vert(c + V(0, r, 0));
    const uint32_t south = vert(c - V(0, r, 0));
    const uint32_t first = uint32_t(pos.size());
    for (int i = 1; i < stacks; ++i) {
      const double th = M_PI * i / stacks;
      for (int j = 0; j < slices; ++j) {
        const double ph = 2 * M_PI * j / slices;
        const V u(float(std::sin(th) * std::cos(ph)), float(std::cos(th)), float(std::sin(th) * std::sin(ph)));
        vert(c + u * r);
      }
    }
    auto ring = [&](int i, int j) { return first + uint32_t((i - 1) * slices + j % slices); };
    for (int j = 0; j < slices; ++j) {
      tri(north, ring(1, j + 1), ring(1, j), m);
      tri(south, ring(stacks - 1, j), ring(stacks - 1, j + 1), m);
    }
    for (int i = 1; i + 1 < stacks; ++i)
      for (int j = 0; j < slices; ++j) {
        tri(ring(i, j), ring(i, j + 1), ring(i + 1, j + 1), m);
        tri(ring(i, j), ring(i + 1, j + 1), ring(i + 1, j), m);
      }
  }

  // Open cylinder with a bottom fan: (bottom, top) per segment, then the
  // centre of the base.
  void cylinder(V base, float r, float h, int seg, uint16_t m) {
    std::vector<uint32_t> lo(static_cast<size_t>(seg)), hi(static_cast<size_t>(seg));
    for (int i = 0; i < seg; ++i) {
      const double a = 2 * M_PI * i / seg;
      const V d(float(std::cos(a)) * r, 0, float(std::sin(a)) * r);
      lo[size_t(i)] = vert(base + d);
      hi[size_t(i)] = vert(base + d + V(0, h, 0));
    }
    const uint32_t centre = vert(base);
    for (int i = 0; i < seg; ++i) {
      const size_t a = size_t(i), b = size_t((i + 1) % seg);
      tri(lo[a], hi[a], hi[b], m);
      tri(lo[a], hi[b], lo[b], m);
      tri(centre, lo[a], lo[b], m);
    }
  }

  void chair(V p, float size, uint16_t m) {
    const float leg = 0.05f * size, seat = 0.45f * size, w = 0.45f * size;
    for (int k = 0; k < 4; ++k) {
      const float x = k & 1 ? w - leg : 0, z = k & 2 ? w - leg : 0;
      box(p + V(x, 0, z), p + V(x + leg, seat, z + leg), m);
    }
    box(p + V(0, seat, 0), p + V(w, seat + 0.05f * size, w), m);
    box(p + V(0, seat, w - leg), p + V(w, seat + 0.5f * size, w), m);
  }

  void table(V p, float wx, float wz, float h, uint16_t m) {
    const float leg = 0.06f;
    box(p + V(0, h - 0.05f, 0), p + V(wx, h, wz), m);
    for (int k = 0; k < 4; ++k) {
      const float x = k & 1 ? wx - leg : 0, z = k & 2 ? wz - leg : 0;
      box(p + V(x, 0, z), p + V(x + leg, h - 0.05f, z + leg), m);
    }
  }

  // Wall slab along x (axis 0) or z (axis 2), with a 1.2 x 2.2 m door gap
  // in the middle when `door`.
  void wall(V o, int axis, float len, float height, float thick, bool door, uint16_t m) {
    auto slab = [&](float a0, float a1, float y0, float y1) {
      if (axis == 0)
        box(o + V(a0, y0, 0), o + V(a1, y1, thick), m);
      else
        box(o + V(0, y0, a0), o + V(thick, y1, a1), m);
    };
    if (!door) {
      slab(0, len, 0, height);
      return;
    }
    const float dw = 1.2f, dh = 2.2f, a = (len - dw) / 2;
    slab(0, a, 0, height);
    slab(a + dw, len, 0, height);
    slab(a, a + dw, dh, height);
  }
};

// ---- the procedural scenes (buildProcedural, procedural.cpp:175-226) ----

void sceneRoom(Mesh& s) {
  const uint16_t wall = s.material(V(0.8f, 0.78f, 0.72f)), wood = s.material(V(0.6f, 0.42f, 0.28f));
  const uint16_t blue = s.material(V(0.35f, 0.45f, 0.75f)), red = s.material(V(0.75f, 0.3f, 0.25f));
  s.box(V(0, 0, 0), V(8, 3, 8), wall, true);
  s.table(V(3, 0, 3), 2, 1.2f, 0.75f, wood);
  s.table(V(0.5f, 0, 6), 1.5f, 1.5f, 0.75f, wood);
  for (int i = 0; i < 4; ++i) s.chair(V(float(2.6 + 0.8 * i), 0, 4.4f), 1, blue);
  for (int i = 0; i < 2; ++i) s.chair(V(float(2.8 + 1.0 * i), 0, 2.2f), 1, blue);
  s.box(V(7.3f, 0, 1), V(7.9f, 2, 3.5f), wood);
  for (int i = 0; i < 8; ++i)
    s.box(V(7.2f, 1.2f, float(1.1 + 0.28 * i)), V(7.3f, float(1.45 + 0.04 * (i % 3)), float(1.3 + 0.28 * i)), red);
  s.sphere(V(4, 0.95f, 3.6f), 0.2f, 6, 10, red);
  s.sphere(V(1.2f, 1.0f, 6.7f), 0.25f, 6, 10, blue);
}

// Three draws for one vector, in the order the reference's compiled
// generator makes them (its arguments are evaluated last to first).
V draw3(Pcg32& g, double a0, double b0, double a1, double b1, double a2, double b2) {
  const float z = float(g.uniform(a2, b2));
  const float y = float(g.uniform(a1, b1));
  const float x = float(g.uniform(a0, b0));
  return V(x, y, z);
}

void scenePlant(Mesh& s, uint64_t seed) {
  const uint16_t floorM = s.material(V(0.75f, 0.72f, 0.68f)), potM = s.material(V(0.7f, 0.4f, 0.25f));
  const uint16_t stemM = s.material(V(0.35f, 0.5f, 0.2f)), leafM = s.material(V(0.3f, 0.65f, 0.25f));
  s.quad(V(-4, 0, -4), V(-4, 0, 4), V(4, 0, 4), V(4, 0, -4), floorM);
  s.quad(V(-4, 0, -1.5f), V(4, 0, -1.5f), V(4, 4, -1.5f), V(-4, 4, -1.5f), floorM);
  s.cylinder(V(0, 0, 0), 0.3f, 0.45f, 24, potM);
  Pcg32 g(seed);
  const int branches = 7, leaves = 180;
  for (int b = 0; b < branches; ++b) {
    const double az = 2 * M_PI * (b + g.uniform() * 0.5) / branches;
    const double el = 0.9 + 0.5 * g.uniform();
    const V dir(float(std::cos(az) * std::cos(el)), float(std::sin(el)), float(std::sin(az) * std::cos(el)));
    const V start(0, 0.4f, 0);
    const float len = float(0.9 + 0.5 * g.uniform());
    const V end = start + dir * len;
    for (int k = 0; k < 4; ++k) {
      const V c = start + (end - start) * (float(k) / 3);
      s.box(c - V(0.015f, 0.015f, 0.015f), c + V(0.015f, 0.015f, 0.015f), stemM);
    }
    for (int l = 0; l < leaves; ++l) {
      const float t = float(0.25 + 0.75 * g.uniform());
      const V jitter = draw3(g, -0.3, 0.3, -0.2, 0.3, -0.3, 0.3);
      const V c = start + dir * (t * len) + jitter;
      const V axis = unit(draw3(g, -1, 1, -0.3, 1, -1, 1));
      const V n = orthogonalTo(axis);
      const V side = unit(cross(axis, n) + n * float(g.uniform(-0.5, 0.5)));
      const V up = unit(cross(axis, side));
      const float L = float(0.07 + 0.06 * g.uniform()), W = L * 0.45f;
      // a folded diamond: four triangles around a raised midrib point
      const uint32_t ic = s.vert(c + up * (L * 0.15f));
      const uint32_t i0 = s.vert(c - axis * L), i1 = s.vert(c + side * W), i2 = s.vert(c + axis * L),
                     i3 = s.vert(c - side * W);
      s.tri(ic, i0, i1, leafM);
      s.tri(ic, i1, i2, leafM);
      s.tri(ic, i2, i3, leafM);
      s.tri(ic, i3, i0, leafM);
    }
  }
}

void sceneBuilding(Mesh& s, int floors, int rooms, int detail) {
  const uint16_t wallM = s.material(V(0.78f, 0.76f, 0.7f)), floorM = s.material(V(0.55f, 0.5f, 0.45f));
  const uint16_t woodM = s.material(V(0.6f, 0.42f, 0.28f)), chairM = s.material(V(0.35f, 0.45f, 0.75f));
  const uint16_t ballM = s.material(V(0.75f, 0.35f, 0.3f)), bookM = s.material(V(0.4f, 0.6f, 0.4f));
  const float W = 5, H = 3, T = 0.15f;
  for (int f = 0; f < floors; ++f)
    for (int i = 0; i < rooms; ++i)
      for (int j = 0; j < rooms; ++j) {
        const V o(float(i) * W, float(f) * H, float(j) * W);
        s.quad(o, o + V(0, 0, W), o + V(W, 0, W), o + V(W, 0, 0), floorM);
        s.quad(o + V(0, H - T, 0), o + V(W, H - T, 0), o + V(W, H - T, W), o + V(0, H - T, W), wallM);
        s.wall(o, 2, W, H - T, T, true, wallM);
        s.wall(o, 0, W, H - T, T, true, wallM);
        if (i == rooms - 1) s.wall(o + V(W - T, 0, 0), 2, W, H - T, T, false, wallM);
        if (j == rooms - 1) s.wall(o + V(0, 0, W - T), 0, W, H - T, T, false, wallM);
        s.table(o + V(0.6f, 0, 3.2f), 1.6f, 0.8f, 0.75f, woodM);
        s.chair(o + V(1.1f, 0, 2.5f), 1, chairM);
        s.box(o + V(3.9f, 0, 3.3f), o + V(4.7f, 1.8f, 4.7f), woodM);
        for (int b = 0; b < 16; ++b)
          s.box(o + V(3.8f, float(0.3 + 0.35 * (b / 8)), float(3.4 + 0.16 * (b % 8))),
                o + V(3.9f, float(0.58 + 0.35 * (b / 8)), float(3.52 + 0.16 * (b % 8))), bookM);
        s.sphere(o + V(1.4f, 1.05f, 3.6f), 0.28f, detail, 2 * detail, ballM);
      }
}

using Params = std::map<std::string, std::string>;

double param(const Params& p, const char* k, double def) {
  const auto it = p.find(k);
  return it == p.end() ? def : std::stod(it->second);
}

bool procedural(const std::string& name, const Params& p, Mesh& s, std::string& err) {
  if (name == "room") {
    sceneRoom(s);
  } else if (name == "plant") {
    scenePlant(s, uint64_t(param(p, "seed", 7)));
  } else if (name == "building") {
    sceneBuilding(s, int(param(p, "floors", 7)), int(param(p, "rooms", 8)), int(param(p, "detail", 33)));
  } else if (name == "tess_sweep") {
    const int stacks = int(param(p, "stacks", 16));
    const uint16_t floorM = s.material(V(0.75f, 0.75f, 0.75f)), ballM = s.material(V(0.8f, 0.5f, 0.35f));
    s.quad(V(-6, 0, -6), V(-6, 0, 6), V(6, 0, 6), V(6, 0, -6), floorM);
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) s.sphere(V(float(-4 + 2 * i), 0.8f, float(-4 + 2 * j)), 0.75f, stacks, 2 * stacks, ballM);
  } else if (name == "analytic") {
    const float h = float(param(p, "h", 1)), occ = float(param(p, "occ", 1)), F = float(param(p, "floor", 10));
    const float ox = float(param(p, "ox", 0)), oz = float(param(p, "oz", 0));
    const uint16_t floorM = s.material(V(0.8f, 0.8f, 0.8f)), occM = s.material(V(0.8f, 0.4f, 0.3f));
    s.quad(V(-F, 0, -F), V(-F, 0, F), V(F, 0, F), V(F, 0, -F), floorM);
    const float a = occ / 2;
    s.quad(V(ox - a, h, oz - a), V(ox - a, h, oz + a), V(ox + a, h, oz + a), V(ox + a, h, oz - a), occM);
  } else if (name == "random_tris") {
    const int n = int(param(p, "n", 50));
    Pcg32 g(uint64_t(param(p, "seed", 1)));
    const float size = float(param(p, "size", 0.3));
    const uint16_t m = s.material(V(0.7f, 0.7f, 0.7f));
    for (int i = 0; i < n; ++i) {
      const V c = draw3(g, 0, 1, 0, 1, 0, 1);
      uint32_t idx[3];
      for (int k = 0; k < 3; ++k) idx[k] = s.vert(c + draw3(g, -size, size, -size, size, -size, size));
      s.tri(idx[0], idx[1], idx[2], m);
    }
  } else if (name == "floorquad") {
    const float y = float(param(p, "y", 0)), F = float(param(p, "size", 10)) / 2;
    const uint16_t m = s.material(V(0.75f, 0.75f, 0.72f));
    s.quad(V(-F, y, -F), V(-F, y, F), V(F, y, F), V(F, y, -F), m);
  } else if (name == "sphere") {
    const uint16_t m = s.material(V(0.7f, 0.7f, 0.7f));
    const int st = int(param(p, "stacks", 24));
    s.sphere(V(0, 0, 0), float(param(p, "r", 1)), st, 2 * st, m);
  } else {
    err = "unknown procedural scene '" + name + "'";
    return false;
  }
  return true;
}

// ---- mesh files (loaders.cpp) ----

bool slurp(const std::string& path, std::string& out) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) return false;
  fseek(f, 0, SEEK_END);
  const long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  out.resize(size_t(n > 0 ? n : 0));
  const size_t got = n > 0 ? fread(&out[0], 1, size_t(n), f) : 0;
  fclose(f);
  return n >= 0 && got == size_t(n);
}

// Polygon (i0, i1, ..., ik) as the fan (i0, i[k-1], i[k]); indices outside
// [0, nv) drop that triangle only.
void fan(Mesh& s, uint32_t base, const std::vector<long>& idx, long nv, uint16_t m) {
  for (size_t k = 2; k < idx.size(); ++k) {
    const long a = idx[0], b = idx[k - 1], c = idx[k];
    if (a < 0 || b < 0 || c < 0 || a >= nv || b >= nv || c >= nv) continue;
    s.tri(base + uint32_t(a), base + uint32_t(b), base + uint32_t(c), m);
  }
}

// Wavefront OBJ: `v x y z` and `f a b c ...` (a/vt/vn accepted, negative
// indices count back from the last vertex); other lines are ignored.
bool loadObj(const std::string& path, Mesh& s, uint16_t m, std::string& err) {
  std::string text;
  if (!slurp(path, text)) {
    err = "cannot read " + path;
    return false;
  }
  const uint32_t base = uint32_t(s.pos.size());
  long nv = 0;
  std::vector<long> face;
  const char* p = text.c_str();
  const char* const end = p + text.size();
  while (p < end) {
    const char* eol = static_cast<const char*>(memchr(p, '\n', size_t(end - p)));
    if (!eol) eol = end;
    while (p < eol && (*p == ' ' || *p == '\t')) ++p;
    const bool tag = p + 1 < eol && (p[1] == ' ' || p[1] == '\t');
    if (tag && p[0] == 'v') {
      char* q;
      const double x = strtod(p + 1, &q);
      const double y = strtod(q, &q);
      const double z = strtod(q, &q);
      s.vert(V(float(x), float(y), float(z)));
      ++nv;
    } else if (tag && p[0] == 'f') {
      face.clear();
      const char* q = p + 1;
      while (q < eol) {
        while (q < eol && (*q == ' ' || *q == '\t' || *q == '\r')) ++q;
        if (q >= eol) break;
        char* r;
        const long i = strtol(q, &r, 10);
        if (r == q) break;
        face.push_back(i > 0 ? i - 1 : nv + i);
        q = r;
        while (q < eol && *q != ' ' && *q != '\t') ++q;
      }
      fan(s, base, face, nv, m);
    }
    p = eol + 1;
  }
  if (nv == 0) {
    err = "no vertices in " + path;
    return false;
  }
  return true;
}

enum class Ply { I8, U8, I16, U16, I32, U32, F32, F64, Bad };

Ply plyType(const std::string& t) {
  static const std::pair<const char*, Ply> kNames[] = {
      {"char", Ply::I8},   {"int8", Ply::I8},     {"uchar", Ply::U8},   {"uint8", Ply::U8},
      {"short", Ply::I16}, {"int16", Ply::I16},   {"ushort", Ply::U16}, {"uint16", Ply::U16},
      {"int", Ply::I32},   {"int32", Ply::I32},   {"uint", Ply::U32},   {"uint32", Ply::U32},
      {"float", Ply::F32}, {"float32", Ply::F32}, {"double", Ply::F64}, {"float64", Ply::F64}};
  for (const auto& kv : kNames)
    if (t == kv.first) return kv.second;
  return Ply::Bad;
}

int plyBytes(Ply t) {
  switch (t) {
    case Ply::I8: case Ply::U8: return 1;
    case Ply::I16: case Ply::U16: return 2;
    case Ply::I32: case Ply::U32: case Ply::F32: return 4;
    case Ply::F64: return 8;
    default: return 0;
  }
}

double plyBinary(const char*& p, Ply t, bool big) {
  unsigned char b[8] = {0};
  const int n = plyBytes(t);
  for (int i = 0; i < n; ++i) b[i] = static_cast<unsigned char>(p[big ? n - 1 - i : i]);
  p += n;
  switch (t) {
    case Ply::I8: return double(int8_t(b[0]));
    case Ply::U8: return double(b[0]);
    case Ply::I16: { int16_t v; memcpy(&v, b, 2); return v; }
    case Ply::U16: { uint16_t v; memcpy(&v, b, 2); return v; }
    case Ply::I32: { int32_t v; memcpy(&v, b, 4); return v; }
    case Ply::U32: { uint32_t v; memcpy(&v, b, 4); return v; }
    case Ply::F32: { float v; memcpy(&v, b, 4); return v; }
    case Ply::F64: { double v; memcpy(&v, b, 8); return v; }
    default: return 0;
  }
}

struct PlyProperty {
  std::string name;
  Ply type = Ply::Bad, countType = Ply::Bad;
  bool list = false;
};
struct PlyElement {
  std::string name;
  size_t count = 0;
  std::vector<PlyProperty> props;
};

// PLY in ascii, binary_little_endian or binary_big_endian: x, y, z of the
// `vertex` element and vertex_indices / vertex_index lists of `face`.
bool loadPly(const std::string& path, Mesh& s, uint16_t m, std::string& err) {
  std::string data;
  if (!slurp(path, data)) {
    err = "cannot read " + path;
    return false;
  }
  const size_t hdrEnd = data.find("end_header");
  if (data.compare(0, 3, "ply") != 0 || hdrEnd == std::string::npos) {
    err = path + ": not a PLY file";
    return false;
  }
  size_t body = data.find('\n', hdrEnd);
  if (body == std::string::npos) {
    err = path + ": truncated header";
    return false;
  }
  ++body;
  std::istringstream hs(data.substr(0, hdrEnd));
  std::string line, format;
  std::vector<PlyElement> elems;
  while (std::getline(hs, line)) {
    const auto t = words(line);
    if (t.empty()) continue;
    if (t[0] == "format" && t.size() > 1) {
      format = t[1];
    } else if (t[0] == "element" && t.size() > 2) {
      PlyElement e;
      e.name = t[1];
      e.count = size_t(std::stoull(t[2]));
      elems.push_back(e);
    } else if (t[0] == "property" && !elems.empty()) {
      PlyProperty pr;
      if (t.size() > 4 && t[1] == "list") {
        pr.list = true;
        pr.countType = plyType(t[2]);
        pr.type = plyType(t[3]);
        pr.name = t[4];
      } else if (t.size() > 2) {
        pr.type = plyType(t[1]);
        pr.name = t[2];
      }
      elems.back().props.push_back(pr);
    }
  }
  const bool ascii = format == "ascii", big = format == "binary_big_endian";
  if (!ascii && !big && format != "binary_little_endian") {
    err = path + ": unsupported PLY format " + format;
    return false;
  }
  const uint32_t base = uint32_t(s.pos.size());
  long nv = 0;
  const char* p = data.c_str() + body;
  const char* const end = data.c_str() + data.size();
  auto value = [&](Ply t) -> double {
    if (ascii) {
      char* q;
      const double v = strtod(p, &q);
      p = q;
      return v;
    }
    if (p + plyBytes(t) > end) return 0;
    return plyBinary(p, t, big);
  };
  std::vector<long> idx;
  for (const PlyElement& e : elems)
    for (size_t i = 0; i < e.count; ++i) {
      double xyz[3] = {0, 0, 0};
      idx.clear();
      for (const PlyProperty& pr : e.props) {
        if (pr.list) {
          const long n = long(value(pr.countType));
          for (long k = 0; k < n; ++k) {
            const double v = value(pr.type);
            if (pr.name == "vertex_indices" || pr.name == "vertex_index") idx.push_back(long(v));
          }
        } else {
          const double v = value(pr.type);
          if (pr.name == "x") xyz[0] = v;
          else if (pr.name == "y") xyz[1] = v;
          else if (pr.name == "z") xyz[2] = v;
        }
      }
      if (e.name == "vertex") {
        s.vert(V(float(xyz[0]), float(xyz[1]), float(xyz[2])));
        ++nv;
      } else if (e.name == "face") {
        fan(s, base, idx, nv, m);
      }
    }
  if (nv == 0) {
    err = path + ": no vertices";
    return false;
  }
  return true;
}

}  // namespace

// ---- configs (scene.cpp:127-262) ----

struct bt_scene_file {
  bt_scene_file_info info;
  std::vector<std::string> meshLines;
  std::vector<float> views;  // eye, target, fov per view
  Mesh mesh;
};

namespace {

bool numbers(const std::vector<std::string>& t, size_t n, float* out, std::string& err) {
  if (t.size() < 1 + n) {
    err = "expected " + std::to_string(n) + " numbers after '" + t[0] + "'";
    return false;
  }
  for (size_t i = 0; i < n; ++i) out[i] = float(std::stod(t[1 + i]));
  return true;
}

void setV(float* dst, V v) {
  dst[0] = v.x;
  dst[1] = v.y;
  dst[2] = v.z;
}
V getV(const float* s) { return V(s[0], s[1], s[2]); }

void addView(bt_scene_file& f, V eye, V target, float fov) {
  f.views.insert(f.views.end(), {eye.x, eye.y, eye.z, target.x, target.y, target.z, fov});
}

bool parse(const std::string& text, bt_scene_file& f, std::string& err) {
  std::istringstream is(text);
  std::string line;
  int lineNo = 0;
  try {
    while (std::getline(is, line)) {
      ++lineNo;
      const size_t hash = line.find('#');
      if (hash != std::string::npos) line = line.substr(0, hash);
      const auto t = words(line);
      if (t.empty()) continue;
      const std::string& k = t[0];
      float v[9];
      bt_scene_file_info& in = f.info;
      if (k == "name") {
        snprintf(in.name, sizeof in.name, "%s", t.size() > 1 ? t[1].c_str() : "");
      } else if (k == "mesh") {
        f.meshLines.push_back(stripped(line.substr(line.find("mesh") + 4)));
      } else if (k == "cull_backfaces") {
        in.cull_backfaces = t.size() > 1 && t[1] != "0";
      } else if (k == "up") {
        if (!numbers(t, 3, v, err)) return false;
        setV(in.up, V(v[0], v[1], v[2]));
      } else if (k == "view") {
        if (!numbers(t, 7, v, err)) return false;
        addView(f, V(v[0], v[1], v[2]), V(v[3], v[4], v[5]), v[6]);
      } else if (k == "orbit") {
        // orbit cx cy cz radius height count fov: views on a circle about c
        if (!numbers(t, 7, v, err)) return false;
        const int n = int(v[5]);
        const V c(v[0], v[1], v[2]), up = unit(getV(in.up));
        const V a = orthogonalTo(up), b = cross(up, a);
        for (int i = 0; i < n; ++i) {
          const double ang = 2 * M_PI * (i + 0.125) / n;
          const V eye = c + a * float(v[3] * std::cos(ang)) + b * float(v[3] * std::sin(ang)) + up * v[4];
          addView(f, eye, c, v[6]);
        }
      } else if (k == "walk") {
        // walk x0 y0 z0 x1 y1 z1 count fov: views along a segment, looking
        // ahead with a small left-right swing
        if (!numbers(t, 8, v, err)) return false;
        const V p0(v[0], v[1], v[2]), p1(v[3], v[4], v[5]);
        const int n = int(v[6]);
        const V dir = unit(p1 - p0);
        for (int i = 0; i < n; ++i) {
          const float s = n > 1 ? float(i) / float(n - 1) : 0;
          const V eye = p0 + (p1 - p0) * (s * 0.85f);
          const V side = unit(cross(dir, unit(getV(in.up))));
          const float swing = float(0.6 * std::sin(2.3 * i));
          addView(f, eye, eye + dir + side * swing, v[7]);
        }
      } else if (k == "point_light") {
        if (!numbers(t, 3, v, err)) return false;
        in.has_point_light = 1;
        setV(in.point_light, V(v[0], v[1], v[2]));
      } else if (k == "area_light") {
        if (!numbers(t, 9, v, err)) return false;
        in.has_area_light = 1;
        setV(in.light_c, V(v[0], v[1], v[2]));
        setV(in.light_u, V(v[3], v[4], v[5]));
        setV(in.light_v, V(v[6], v[7], v[8]));
      } else if (k == "light_intensity") {
        if (!numbers(t, 1, v, err)) return false;
        in.light_intensity = v[0];
      } else if (k == "background") {
        if (!numbers(t, 3, v, err)) return false;
        setV(in.background, V(v[0], v[1], v[2]));
      } else {
        err = "unknown key '" + k + "'";
        return false;
      }
    }
  } catch (const std::exception& e) {
    err = "line " + std::to_string(lineNo) + ": " + e.what();
    return false;
  }
  return true;
}

// The meshes of the config, in order; each may carry `scale s`,
// `translate x y z`, `color r g b` (file meshes) or key=value parameters
// (procedural scenes).  Then Scene::finalize's degeneracy rule, keeping
// each surviving triangle's material.
bool build(bt_scene_file& f, std::string& err) {
  static const V kPalette[6] = {V(0.75f, 0.75f, 0.75f), V(0.8f, 0.55f, 0.4f), V(0.45f, 0.65f, 0.8f),
                                V(0.6f, 0.8f, 0.45f),   V(0.85f, 0.8f, 0.5f), V(0.7f, 0.5f, 0.75f)};
  Mesh& s = f.mesh;
  int index = 0;
  try {
    for (const std::string& ml : f.meshLines) {
      const auto t = words(ml);
      if (t.size() < 2) {
        err = "bad mesh line: " + ml;
        return false;
      }
      float scale = 1;
      V translate, color = kPalette[index % 6];
      Params params;
      for (size_t i = 2; i < t.size(); ++i) {
        if (t[i] == "scale" && i + 1 < t.size()) {
          scale = float(std::stod(t[++i]));
        } else if (t[i] == "translate" && i + 3 < t.size()) {
          translate = V(float(std::stod(t[i + 1])), float(std::stod(t[i + 2])), float(std::stod(t[i + 3])));
          i += 3;
        } else if (t[i] == "color" && i + 3 < t.size()) {
          color = V(float(std::stod(t[i + 1])), float(std::stod(t[i + 2])), float(std::stod(t[i + 3])));
          i += 3;
        } else if (t[i].find('=') != std::string::npos) {
          const size_t e = t[i].find('=');
          params[t[i].substr(0, e)] = t[i].substr(e + 1);
        }
      }
      const size_t first = s.pos.size();
      bool ok;
      if (t[0] == "obj") {
        ok = loadObj(t[1], s, s.material(color), err);
      } else if (t[0] == "ply") {
        ok = loadPly(t[1], s, s.material(color), err);
      } else if (t[0] == "procedural") {
        ok = procedural(t[1], params, s, err);
      } else {
        err = "unknown mesh type " + t[0];
        return false;
      }
      if (!ok) return false;
      for (size_t i = first; i < s.pos.size(); ++i) s.pos[i] = s.pos[i] * scale + translate;
      ++index;
    }
  } catch (const std::exception& e) {
    err = std::string("mesh parameters: ") + e.what();
    return false;
  }
  // degenerate triangles out (bt_scene_finalize's rule; it keeps the order,
  // so the kept triangles are matched back to their materials in one walk)
  const int64_t nt = int64_t(s.mat.size());
  std::vector<uint32_t> kept(size_t(3 * std::max<int64_t>(nt, 1)));
  std::vector<float> nrm(kept.size()), area(size_t(std::max<int64_t>(nt, 1)));
  float bounds[6];
  const int64_t nk = nt ? bt_scene_finalize(&s.pos[0].x, int64_t(s.pos.size()), s.tris.data(), nt, kept.data(),
                                            nrm.data(), area.data(), bounds)
                        : 0;
  if (nk < 0) {
    err = "triangle index out of range";
    return false;
  }
  std::vector<uint16_t> mat;
  mat.reserve(size_t(nk));
  for (int64_t i = 0, j = 0; i < nt && j < nk; ++i)
    if (std::equal(&s.tris[size_t(3 * i)], &s.tris[size_t(3 * i + 3)], &kept[size_t(3 * j)])) {
      mat.push_back(s.mat[size_t(i)]);
      ++j;
    }
  kept.resize(size_t(3 * nk));
  s.tris.swap(kept);
  s.mat.swap(mat);
  if (s.colors.empty()) s.material(V(0.75f, 0.75f, 0.75f));
  if (nk == 0) {
    err = "scene has no triangles";
    return false;
  }
  return true;
}

bt_scene_file* fresh() {
  auto* f = new bt_scene_file();
  memset(&f->info, 0, sizeof f->info);
  f->info.up[1] = 1;
  f->info.light_intensity = 1;
  return f;
}

int make(const std::string& text, const std::string& path, bt_scene_file** out) {
  *out = nullptr;
  bt_scene_file* f = fresh();
  std::string err;
  if (!parse(text, *f, err)) {
    btSetError((path.empty() ? err : path + ": " + err).c_str());
    delete f;
    return BT_ERR_INVALID;
  }
  if (!build(*f, err)) {
    btSetError(err.c_str());
    delete f;
    return BT_ERR_INVALID;
  }
  f->info.num_verts = int64_t(f->mesh.pos.size());
  f->info.num_tris = int64_t(f->mesh.mat.size());
  f->info.num_materials = int64_t(f->mesh.colors.size());
  f->info.num_views = int64_t(f->views.size() / 7);
  *out = f;
  return BT_OK;
}

}  // namespace

int bt_scene_parse_config(const char* text, bt_scene_file** out) {
  if (!text || !out) return BT_ERR_INVALID;
  return make(text, "", out);
}

int bt_scene_load_config(const char* path, bt_scene_file** out) {
  if (!path || !out) return BT_ERR_INVALID;
  *out = nullptr;
  std::string text;
  if (!slurp(path, text)) {
    btSetError((std::string("cannot open config ") + path).c_str());
    return BT_ERR_INVALID;
  }
  return make(text, path, out);
}

void bt_scene_file_info_get(const bt_scene_file* f, bt_scene_file_info* info) {
  if (f && info) *info = f->info;
}

void bt_scene_file_arrays(const bt_scene_file* f, float* pos, uint32_t* tris, uint16_t* tri_mat, float* mat_color,
                          float* views) {
  if (!f) return;
  const Mesh& m = f->mesh;
  if (pos)
    for (size_t i = 0; i < m.pos.size(); ++i) setV(pos + 3 * i, m.pos[i]);
  if (tris && !m.tris.empty()) memcpy(tris, m.tris.data(), m.tris.size() * sizeof(uint32_t));
  if (tri_mat && !m.mat.empty()) memcpy(tri_mat, m.mat.data(), m.mat.size() * sizeof(uint16_t));
  if (mat_color)
    for (size_t i = 0; i < m.colors.size(); ++i) setV(mat_color + 3 * i, m.colors[i]);
  if (views && !f->views.empty()) memcpy(views, f->views.data(), f->views.size() * sizeof(float));
}

void bt_scene_file_free(bt_scene_file* f) { delete f; }
