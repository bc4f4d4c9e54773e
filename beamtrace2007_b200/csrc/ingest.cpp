// Scene ingest: scene configs, OBJ and PLY meshes and the procedural
// scenes, exported through the C-ABI (include/bt_gpu.h, bt_scene_file_*).
//
// A config names meshes and views; the scene built from it must be the one
// the reference builds from the same file, vertex for vertex, since the kd
// tree and every beam depend on the float coordinates.  What that fixes is
// the arithmetic, not the code: decimal text to double (correctly rounded)
// to float, polygons cut into fans around their first corner, the index
// rules of the two mesh formats, the view formulas of `orbit` and `walk`,
// and the generators' float operations and random draws in their order.
// The file readers and the config parser here are written from the formats'
// own descriptions (Wavefront OBJ, Stanford PLY, and the config keys of
// src/scene/scene.h:13-61); the generators restate the reference's scenes:
//   buildProcedural and its scenes          src/scene/procedural.cpp:17-226
//   addQuad / addBox / addSphere            src/scene/scene.cpp:44-87
//   Scene::finalize                         src/scene/scene.cpp:8-42
//   PCG32 and its [0, 1) mapping            src/util/misc.h:24-46
// Compiled with -ffp-contract=off like the reference.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <charconv>
#include <map>
#include <stdexcept>
#include <string>
#include <string_view>
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

  // The box lo..hi on its eight corners (bit a of a corner's number picks
  // hi on axis a), so neighbouring faces share vertices; each face is two
  // triangles wound counter-clockwise when looked at from outside (with
  // `inward`, from inside).
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

  // A wall: a box `thick` deep running `len` from o along x (axis 0) or z
  // (axis 2); with `door`, two side slabs and a lintel leave a 1.2 m wide,
  // 2.2 m high opening at the middle.
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
      // the leaf: a centre vertex lifted off the blade plane, joined to the
      // tip, the two side points and the base (four triangles, a shallow tent)
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


// ---- text fields and numbers ----

constexpr bool isBlank(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\f' || c == '\v'; }

// Walks the blank-separated fields of a piece of text.
class Fields {
 public:
  explicit Fields(std::string_view text) : rest_(text) {}
  bool next(std::string_view& field) {
    size_t a = 0;
    while (a < rest_.size() && isBlank(rest_[a])) ++a;
    size_t b = a;
    while (b < rest_.size() && !isBlank(rest_[b])) ++b;
    field = rest_.substr(a, b - a);
    rest_.remove_prefix(b);
    return !field.empty();
  }
  std::vector<std::string_view> all() {
    std::vector<std::string_view> out;
    std::string_view f;
    while (next(f)) out.push_back(f);
    return out;
  }

 private:
  std::string_view rest_;
};

// Calls fn(line number from 1, line) for every line of `text` (LF ends a line).
template <class Fn>
void eachLine(std::string_view text, Fn&& fn) {
  int number = 0;
  while (!text.empty()) {
    const size_t lf = text.find('\n');
    fn(++number, text.substr(0, lf));
    if (lf == std::string_view::npos) break;
    text.remove_prefix(lf + 1);
  }
}

// Reads a number at the start of `s` as strtod does, without its leading
// blanks: optional sign, then decimal digits with an optional exponent, a
// 0x-prefixed hexadecimal float, inf or nan.  The double is the correctly
// rounded value of the digits.  Returns the characters used, 0 when `s`
// does not start with a number.
size_t numberPrefix(std::string_view s, double& v) {
  size_t i = 0;
  const bool neg = !s.empty() && s[0] == '-';
  if (!s.empty() && (s[0] == '+' || s[0] == '-')) i = 1;
  if (i < s.size() && (s[i] == '+' || s[i] == '-')) return 0;
  const bool hex = i + 1 < s.size() && s[i] == '0' && (s[i + 1] == 'x' || s[i + 1] == 'X');
  const char* from = s.data() + i + (hex ? 2 : 0);
  const auto r = std::from_chars(from, s.data() + s.size(), v, hex ? std::chars_format::hex : std::chars_format::general);
  if (r.ec == std::errc::invalid_argument) {
    if (!hex) return 0;
    v = neg ? -0.0 : 0.0;  // "0x" with no hexadecimal digits: the "0"
    return i + 1;
  }
  const size_t used = size_t(r.ptr - s.data());
  if (r.ec == std::errc::result_out_of_range) {
    v = std::strtod(std::string(s.substr(0, used)).c_str(), nullptr);  // saturated: +-HUGE_VAL or a zero
    return used;
  }
  if (neg) v = -v;
  return used;
}

// The whole field as a number.
bool wholeNumber(std::string_view s, double& v) { return !s.empty() && numberPrefix(s, v) == s.size(); }

// An integer at the start of `s` (a leading '+' allowed); values beyond
// int64 saturate.  False when `s` does not start with one.
bool integerPrefix(std::string_view s, int64_t& v) {
  const size_t skip = (s.size() > 1 && s[0] == '+' && s[1] != '-') ? 1 : 0;
  const auto r = std::from_chars(s.data() + skip, s.data() + s.size(), v);
  if (r.ec == std::errc::invalid_argument) return false;
  if (r.ec == std::errc::result_out_of_range) v = s[skip] == '-' ? INT64_MIN : INT64_MAX;
  return true;
}

std::string quoted(std::string_view s) { return "'" + std::string(s) + "'"; }

// ---- procedural scenes by name ----

// key=value parameters of a procedural mesh line.
class SceneParams {
 public:
  void set(std::string_view kv) {
    const size_t e = kv.find('=');
    values_[std::string(kv.substr(0, e))] = std::string(kv.substr(e + 1));
  }
  double get(const char* key, double fallback) const {
    const auto it = values_.find(key);
    if (it == values_.end()) return fallback;
    double v;
    if (!wholeNumber(it->second, v))
      throw std::invalid_argument(std::string("procedural parameter ") + key + "=" + it->second + " is not a number");
    return v;
  }

 private:
  std::map<std::string, std::string, std::less<>> values_;
};

bool procedural(std::string_view name, const SceneParams& p, Mesh& s, std::string& why) {
  if (name == "room") {
    sceneRoom(s);
  } else if (name == "plant") {
    scenePlant(s, uint64_t(p.get("seed", 7)));
  } else if (name == "building") {
    sceneBuilding(s, int(p.get("floors", 7)), int(p.get("rooms", 8)), int(p.get("detail", 33)));
  } else if (name == "tess_sweep") {
    const int stacks = int(p.get("stacks", 16));
    const uint16_t floorM = s.material(V(0.75f, 0.75f, 0.75f)), ballM = s.material(V(0.8f, 0.5f, 0.35f));
    s.quad(V(-6, 0, -6), V(-6, 0, 6), V(6, 0, 6), V(6, 0, -6), floorM);
    for (int i = 0; i < 5; ++i)
      for (int j = 0; j < 5; ++j) s.sphere(V(float(-4 + 2 * i), 0.8f, float(-4 + 2 * j)), 0.75f, stacks, 2 * stacks, ballM);
  } else if (name == "analytic") {
    const float h = float(p.get("h", 1)), occ = float(p.get("occ", 1)), F = float(p.get("floor", 10));
    const float ox = float(p.get("ox", 0)), oz = float(p.get("oz", 0));
    const uint16_t floorM = s.material(V(0.8f, 0.8f, 0.8f)), occM = s.material(V(0.8f, 0.4f, 0.3f));
    s.quad(V(-F, 0, -F), V(-F, 0, F), V(F, 0, F), V(F, 0, -F), floorM);
    const float a = occ / 2;
    s.quad(V(ox - a, h, oz - a), V(ox - a, h, oz + a), V(ox + a, h, oz + a), V(ox + a, h, oz - a), occM);
  } else if (name == "random_tris") {
    const int n = int(p.get("n", 50));
    Pcg32 g(uint64_t(p.get("seed", 1)));
    const float size = float(p.get("size", 0.3));
    const uint16_t m = s.material(V(0.7f, 0.7f, 0.7f));
    for (int i = 0; i < n; ++i) {
      const V c = draw3(g, 0, 1, 0, 1, 0, 1);
      uint32_t idx[3];
      for (int k = 0; k < 3; ++k) idx[k] = s.vert(c + draw3(g, -size, size, -size, size, -size, size));
      s.tri(idx[0], idx[1], idx[2], m);
    }
  } else if (name == "floorquad") {
    const float y = float(p.get("y", 0)), F = float(p.get("size", 10)) / 2;
    const uint16_t m = s.material(V(0.75f, 0.75f, 0.72f));
    s.quad(V(-F, y, -F), V(-F, y, F), V(F, y, F), V(F, y, -F), m);
  } else if (name == "sphere") {
    const uint16_t m = s.material(V(0.7f, 0.7f, 0.7f));
    const int st = int(p.get("stacks", 24));
    s.sphere(V(0, 0, 0), float(p.get("r", 1)), st, 2 * st, m);
  } else {
    why = "no procedural scene named " + quoted(name);
    return false;
  }
  return true;
}

// ---- mesh files ----

bool readWholeFile(const std::string& path, std::string& bytes) {
  std::FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  bytes.clear();
  char chunk[1 << 16];
  size_t got;
  while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) bytes.append(chunk, got);
  const bool ok = !std::ferror(f);
  std::fclose(f);
  return ok;
}

// Adds polygon `corners` (indices into the positions [first, first + count)
// of one file) as the triangles (c0, c[k-1], c[k]); a triangle with a corner
// outside that range is left out, the rest of the polygon is kept.
void addPolygon(Mesh& m, uint32_t first, const std::vector<int64_t>& corners, int64_t count, uint16_t mat) {
  auto valid = [count](int64_t c) { return c >= 0 && c < count; };
  for (size_t k = 2; k < corners.size(); ++k) {
    const int64_t a = corners[0], b = corners[k - 1], c = corners[k];
    if (valid(a) && valid(b) && valid(c)) m.tri(first + uint32_t(a), first + uint32_t(b), first + uint32_t(c), mat);
  }
}

// Wavefront OBJ geometry.  A `v` record adds a position; coordinates that
// are missing or not numbers read as 0.  An `f` record is a polygon whose
// corners name positions of this file: 1-based, or negative to count back
// from the newest position, each possibly followed by /texture/normal
// references, which are ignored; a field that does not start with an
// integer ends the corner list.  Every other record (vt, vn, o, g, usemtl,
// l, ...) is skipped.
bool readObj(const std::string& path, Mesh& m, uint16_t mat, std::string& why) {
  std::string bytes;
  if (!readWholeFile(path, bytes)) {
    why = "could not open mesh file " + path;
    return false;
  }
  const uint32_t first = uint32_t(m.pos.size());
  int64_t count = 0;
  std::vector<int64_t> corners;
  eachLine(bytes, [&](int, std::string_view line) {
    Fields f(line);
    std::string_view record, field;
    if (!f.next(record)) return;
    if (record == "v") {
      float xyz[3] = {0, 0, 0};
      for (float& c : xyz) {
        double d;
        if (!f.next(field) || numberPrefix(field, d) == 0) break;
        c = float(d);
      }
      m.vert(V(xyz[0], xyz[1], xyz[2]));
      ++count;
    } else if (record == "f") {
      corners.clear();
      int64_t ref;
      while (f.next(field) && integerPrefix(field, ref))
        corners.push_back(ref > 0 ? ref - 1 : (ref < -count ? -1 : count + ref));
      addPolygon(m, first, corners, count, mat);
    }
  });
  if (count == 0) {
    why = path + " holds no vertex positions";
    return false;
  }
  return true;
}

// PLY (ascii, binary_little_endian, binary_big_endian).  The header lists
// groups of records ("element NAME COUNT"), each with its columns
// ("property TYPE NAME" or "property list LENGTHTYPE TYPE NAME"); the body
// holds the records group after group.  Positions come from the x, y, z
// columns of group `vertex`, polygons from the vertex_indices (or
// vertex_index) list of group `face`; everything else is read and dropped.
enum class PlyType : uint8_t { None, I8, U8, I16, U16, I32, U32, F32, F64 };

PlyType plyTypeNamed(std::string_view n) {
  struct Name { const char* text; PlyType type; };
  static const Name kNames[] = {{"char", PlyType::I8},    {"int8", PlyType::I8},     {"uchar", PlyType::U8},
                                {"uint8", PlyType::U8},   {"short", PlyType::I16},   {"int16", PlyType::I16},
                                {"ushort", PlyType::U16}, {"uint16", PlyType::U16},  {"int", PlyType::I32},
                                {"int32", PlyType::I32},  {"uint", PlyType::U32},    {"uint32", PlyType::U32},
                                {"float", PlyType::F32},  {"float32", PlyType::F32}, {"double", PlyType::F64},
                                {"float64", PlyType::F64}};
  for (const Name& x : kNames)
    if (n == x.text) return x.type;
  return PlyType::None;
}

size_t plySize(PlyType t) {
  static const size_t kSize[] = {0, 1, 1, 2, 2, 4, 4, 4, 8};
  return kSize[size_t(t)];
}

struct PlyColumn {
  std::string name;
  PlyType type = PlyType::None;
  PlyType lengthType = PlyType::None;  // set for list columns
};

struct PlyGroup {
  std::string name;
  uint64_t rows = 0;
  std::vector<PlyColumn> columns;
};

enum class PlyEncoding { Ascii, Little, Big };

// Reads the header; `body` = offset of the first byte after end_header's line.
bool plyHeader(const std::string& bytes, const std::string& path, PlyEncoding& enc, std::vector<PlyGroup>& groups,
               size_t& body, std::string& why) {
  size_t at = 0;
  bool sawMagic = false, sawFormat = false;
  while (at < bytes.size()) {
    const size_t lf = bytes.find('\n', at);
    const size_t end = lf == std::string::npos ? bytes.size() : lf;
    const std::vector<std::string_view> t = Fields(std::string_view(bytes).substr(at, end - at)).all();
    at = lf == std::string::npos ? bytes.size() : lf + 1;
    if (!sawMagic) {
      if (t.size() != 1 || t[0] != "ply") break;
      sawMagic = true;
      continue;
    }
    if (t.empty() || t[0] == "comment" || t[0] == "obj_info") continue;
    if (t[0] == "end_header") {
      if (!sawFormat) {
        why = path + ": PLY header names no format";
        return false;
      }
      if (lf == std::string::npos) {
        why = path + ": PLY file ends inside its header";
        return false;
      }
      body = at;
      return true;
    }
    if (t[0] == "format" && t.size() >= 2) {
      sawFormat = true;
      if (t[1] == "ascii") {
        enc = PlyEncoding::Ascii;
      } else if (t[1] == "binary_little_endian") {
        enc = PlyEncoding::Little;
      } else if (t[1] == "binary_big_endian") {
        enc = PlyEncoding::Big;
      } else {
        why = path + ": PLY encoding " + quoted(t[1]) + " is not supported";
        return false;
      }
    } else if (t[0] == "element" && t.size() >= 3) {
      PlyGroup g;
      g.name = std::string(t[1]);
      const auto r = std::from_chars(t[2].data(), t[2].data() + t[2].size(), g.rows);
      if (r.ec != std::errc() || r.ptr != t[2].data() + t[2].size()) {
        why = path + ": PLY record count " + quoted(t[2]) + " is not a count";
        return false;
      }
      groups.push_back(std::move(g));
    } else if (t[0] == "property" && !groups.empty()) {
      PlyColumn c;
      const bool list = t.size() >= 5 && t[1] == "list";
      if (list) {
        c.lengthType = plyTypeNamed(t[2]);
        c.type = plyTypeNamed(t[3]);
        c.name = std::string(t[4]);
      } else if (t.size() >= 3) {
        c.type = plyTypeNamed(t[1]);
        c.name = std::string(t[2]);
      }
      if (c.type == PlyType::None || (list && c.lengthType == PlyType::None)) {
        why = path + ": PLY column with an unknown type";
        return false;
      }
      groups.back().columns.push_back(std::move(c));
    } else {
      why = path + ": PLY header line " + quoted(t[0]) + " not understood";
      return false;
    }
  }
  why = sawMagic ? path + ": PLY header has no end_header line" : path + ": not a PLY file (no 'ply' line)";
  return false;
}

// Values of a PLY body, one at a time.
class PlyBody {
 public:
  PlyBody(std::string_view bytes, PlyEncoding enc) : rest_(bytes), fields_(bytes), enc_(enc) {}

  bool value(PlyType t, double& v) {
    if (enc_ == PlyEncoding::Ascii) {
      std::string_view f;
      return fields_.next(f) && wholeNumber(f, v);
    }
    const size_t n = plySize(t);
    if (rest_.size() < n) return false;
    unsigned char b[8];
    std::memcpy(b, rest_.data(), n);
    rest_.remove_prefix(n);
    if (enc_ == PlyEncoding::Big) std::reverse(b, b + n);  // this library runs on little-endian hosts
    switch (t) {
      case PlyType::I8: v = double(int8_t(b[0])); break;
      case PlyType::U8: v = double(b[0]); break;
      case PlyType::I16: v = double(bitsAs<int16_t>(b)); break;
      case PlyType::U16: v = double(bitsAs<uint16_t>(b)); break;
      case PlyType::I32: v = double(bitsAs<int32_t>(b)); break;
      case PlyType::U32: v = double(bitsAs<uint32_t>(b)); break;
      case PlyType::F32: v = double(bitsAs<float>(b)); break;
      case PlyType::F64: v = bitsAs<double>(b); break;
      default: return false;
    }
    return true;
  }

 private:
  template <class T>
  static T bitsAs(const unsigned char* b) {
    T x;
    std::memcpy(&x, b, sizeof x);
    return x;
  }
  std::string_view rest_;
  Fields fields_;
  PlyEncoding enc_;
};
static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "the PLY reader assumes a little-endian host");

bool readPly(const std::string& path, Mesh& m, uint16_t mat, std::string& why) {
  std::string bytes;
  if (!readWholeFile(path, bytes)) {
    why = "could not open mesh file " + path;
    return false;
  }
  PlyEncoding enc = PlyEncoding::Ascii;
  std::vector<PlyGroup> groups;
  size_t body = 0;
  if (!plyHeader(bytes, path, enc, groups, body, why)) return false;
  PlyBody in(std::string_view(bytes).substr(body), enc);
  const uint32_t first = uint32_t(m.pos.size());
  int64_t count = 0;
  std::vector<int64_t> corners;
  auto readGroup = [&](const PlyGroup& g) {
    const bool positions = g.name == "vertex", polygons = g.name == "face";
    for (uint64_t row = 0; row < g.rows; ++row) {
      double xyz[3] = {0, 0, 0};
      corners.clear();
      for (const PlyColumn& c : g.columns) {
        double v;
        if (c.lengthType == PlyType::None) {
          if (!in.value(c.type, v)) return false;
          if (c.name.size() == 1 && c.name[0] >= 'x' && c.name[0] <= 'z') xyz[c.name[0] - 'x'] = v;
          continue;
        }
        if (!in.value(c.lengthType, v)) return false;
        const bool keep = polygons && (c.name == "vertex_indices" || c.name == "vertex_index");
        for (int64_t k = 0, n = int64_t(v); k < n; ++k) {
          if (!in.value(c.type, v)) return false;
          if (keep) corners.push_back(int64_t(v));
        }
      }
      if (positions) {
        m.vert(V(float(xyz[0]), float(xyz[1]), float(xyz[2])));
        ++count;
      } else if (polygons) {
        addPolygon(m, first, corners, count, mat);
      }
    }
    return true;
  };
  for (const PlyGroup& g : groups)
    if (!readGroup(g)) {
      why = path + ": PLY body ends early or holds a value that is not a number";
      return false;
    }
  if (count == 0) {
    why = path + " holds no vertex positions";
    return false;
  }
  return true;
}

}  // namespace

// ---- configs ----

struct bt_scene_file {
  bt_scene_file_info info;
  std::vector<std::vector<std::string>> meshes;  // the fields after `mesh`, per mesh line
  std::vector<float> views;                      // eye, target, fov per view
  Mesh mesh;
};

namespace {

void setV(float* dst, V v) {
  dst[0] = v.x;
  dst[1] = v.y;
  dst[2] = v.z;
}
V getV(const float* s) { return V(s[0], s[1], s[2]); }

void addView(bt_scene_file& f, V eye, V target, float fov) {
  f.views.insert(f.views.end(), {eye.x, eye.y, eye.z, target.x, target.y, target.z, fov});
}

// orbit cx cy cz radius height count fov: `count` views on a circle of
// `radius` about c, raised by `height` along up, looking at c; the first at
// an eighth of the spacing past the first axis orthogonal to up.
void addOrbit(bt_scene_file& f, const float* a) {
  const int n = int(a[5]);
  const V c(a[0], a[1], a[2]), up = unit(getV(f.info.up));
  const V e0 = orthogonalTo(up), e1 = cross(up, e0);
  for (int i = 0; i < n; ++i) {
    const double phi = 2 * M_PI * (i + 0.125) / n;
    addView(f, c + e0 * float(a[3] * std::cos(phi)) + e1 * float(a[3] * std::sin(phi)) + up * a[4], c, a[6]);
  }
}

// walk x0 y0 z0 x1 y1 z1 count fov: `count` views spread over the first 85%
// of the segment p0 -> p1, each looking one unit ahead, turned sideways by
// 0.6 sin(2.3 i) units.
void addWalk(bt_scene_file& f, const float* a) {
  const V p0(a[0], a[1], a[2]), p1(a[3], a[4], a[5]);
  const int n = int(a[6]);
  const V dir = unit(p1 - p0);
  for (int i = 0; i < n; ++i) {
    const float s = n > 1 ? float(i) / float(n - 1) : 0;
    const V eye = p0 + (p1 - p0) * (s * 0.85f);
    const V side = unit(cross(dir, unit(getV(f.info.up))));
    addView(f, eye, eye + dir + side * float(0.6 * std::sin(2.3 * i)), a[7]);
  }
}

// Keys that take a fixed number of numbers.
struct NumericKey {
  const char* key;
  int count;
  void (*apply)(bt_scene_file& f, const float* a);
};

const NumericKey kNumericKeys[] = {
    {"up", 3, [](bt_scene_file& f, const float* a) { setV(f.info.up, getV(a)); }},
    {"view", 7, [](bt_scene_file& f, const float* a) { addView(f, getV(a), getV(a + 3), a[6]); }},
    {"orbit", 7, addOrbit},
    {"walk", 8, addWalk},
    {"point_light", 3,
     [](bt_scene_file& f, const float* a) {
       f.info.has_point_light = 1;
       setV(f.info.point_light, getV(a));
     }},
    {"area_light", 9,
     [](bt_scene_file& f, const float* a) {
       f.info.has_area_light = 1;
       setV(f.info.light_c, getV(a));
       setV(f.info.light_u, getV(a + 3));
       setV(f.info.light_v, getV(a + 6));
     }},
    {"light_intensity", 1, [](bt_scene_file& f, const float* a) { f.info.light_intensity = a[0]; }},
    {"background", 3, [](bt_scene_file& f, const float* a) { setV(f.info.background, getV(a)); }},
};

// One `key values...` line (the text after '#' dropped); false with `why`.
bool configLine(bt_scene_file& f, const std::vector<std::string_view>& t, std::string& why) {
  const std::string_view key = t[0];
  if (key == "name") {
    snprintf(f.info.name, sizeof f.info.name, "%s", t.size() > 1 ? std::string(t[1]).c_str() : "");
    return true;
  }
  if (key == "mesh") {
    f.meshes.emplace_back(t.begin() + 1, t.end());
    return true;
  }
  if (key == "cull_backfaces") {
    f.info.cull_backfaces = t.size() > 1 && t[1] != "0";
    return true;
  }
  for (const NumericKey& k : kNumericKeys) {
    if (key != k.key) continue;
    if (int(t.size()) - 1 < k.count) {
      why = quoted(key) + " takes " + std::to_string(k.count) + " numbers, got " + std::to_string(t.size() - 1);
      return false;
    }
    float a[9];
    for (int i = 0; i < k.count; ++i) {
      double d;
      if (!wholeNumber(t[size_t(1 + i)], d)) {
        why = quoted(t[size_t(1 + i)]) + " is not a number";
        return false;
      }
      a[i] = float(d);
    }
    k.apply(f, a);
    return true;
  }
  why = quoted(key) + " is not a config key";
  return false;
}

bool parse(std::string_view text, bt_scene_file& f, std::string& why) {
  bool ok = true;
  eachLine(text, [&](int number, std::string_view line) {
    if (!ok) return;
    const std::vector<std::string_view> t = Fields(line.substr(0, line.find('#'))).all();
    if (t.empty() || configLine(f, t, why)) return;
    why = "line " + std::to_string(number) + ": " + why;
    ok = false;
  });
  return ok;
}

// A mesh line: `obj PATH` or `ply PATH` with optional `scale s`,
// `translate x y z` and `color r g b` (placed as p * s + t, in that order),
// or `procedural NAME` with key=value parameters.  A file mesh without a
// colour takes the next of six palette colours by its place among the
// config's meshes.
bool addMesh(Mesh& s, const std::vector<std::string>& t, int place, std::string& why) {
  static const V kPalette[6] = {V(0.75f, 0.75f, 0.75f), V(0.8f, 0.55f, 0.4f), V(0.45f, 0.65f, 0.8f),
                                V(0.6f, 0.8f, 0.45f),   V(0.85f, 0.8f, 0.5f), V(0.7f, 0.5f, 0.75f)};
  if (t.size() < 2) {
    why = "mesh line " + quoted(t.empty() ? "" : t[0]) + " names no file or scene";
    return false;
  }
  float scale = 1;
  V shift, color = kPalette[place % 6];
  SceneParams params;
  auto numbersAt = [&](size_t i, int k, float* out) {
    for (int j = 0; j < k; ++j) {
      double d;
      if (!wholeNumber(t[i + size_t(j)], d)) throw std::invalid_argument(quoted(t[i + size_t(j)]) + " is not a number");
      out[j] = float(d);
    }
  };
  for (size_t i = 2; i < t.size(); ++i) {
    const std::string& w = t[i];
    float a[3];
    if (w == "scale" && i + 1 < t.size()) {
      numbersAt(i + 1, 1, &scale);
      i += 1;
    } else if ((w == "translate" || w == "color") && i + 3 < t.size()) {
      numbersAt(i + 1, 3, a);
      (w == "translate" ? shift : color) = V(a[0], a[1], a[2]);
      i += 3;
    } else if (w.find('=') != std::string::npos) {
      params.set(w);
    }
  }
  const size_t before = s.pos.size();
  bool ok;
  if (t[0] == "obj") {
    ok = readObj(t[1], s, s.material(color), why);
  } else if (t[0] == "ply") {
    ok = readPly(t[1], s, s.material(color), why);
  } else if (t[0] == "procedural") {
    ok = procedural(t[1], params, s, why);
  } else {
    why = "mesh kind " + quoted(t[0]) + " is not obj, ply or procedural";
    return false;
  }
  if (!ok) return false;
  for (size_t i = before; i < s.pos.size(); ++i) s.pos[i] = s.pos[i] * scale + shift;
  return true;
}

// The meshes in config order, then bt_scene_finalize's degeneracy rule;
// each surviving triangle keeps its material.
bool build(bt_scene_file& f, std::string& why) {
  Mesh& s = f.mesh;
  try {
    for (size_t i = 0; i < f.meshes.size(); ++i)
      if (!addMesh(s, f.meshes[i], int(i), why)) return false;
  } catch (const std::exception& e) {
    why = e.what();
    return false;
  }
  // bt_scene_finalize keeps the order of the triangles it keeps, so one walk
  // matches them back to their materials
  const int64_t nt = int64_t(s.mat.size());
  std::vector<uint32_t> kept(size_t(3 * std::max<int64_t>(nt, 1)));
  std::vector<float> nrm(kept.size()), area(size_t(std::max<int64_t>(nt, 1)));
  float bounds[6];
  const int64_t nk = nt ? bt_scene_finalize(&s.pos[0].x, int64_t(s.pos.size()), s.tris.data(), nt, kept.data(),
                                            nrm.data(), area.data(), bounds)
                        : 0;
  if (nk < 0) {
    why = "triangle index out of range";
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
    why = "the config yields no triangles";
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

int make(std::string_view text, const std::string& path, bt_scene_file** out) {
  *out = nullptr;
  bt_scene_file* f = fresh();
  std::string why;
  if (!parse(text, *f, why)) {
    btSetError((path.empty() ? why : path + ": " + why).c_str());
    delete f;
    return BT_ERR_INVALID;
  }
  if (!build(*f, why)) {
    btSetError(why.c_str());
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
  if (!readWholeFile(path, text)) {
    btSetError((std::string("could not read config file ") + path).c_str());
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
