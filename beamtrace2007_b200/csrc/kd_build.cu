// GPU build of the SAH kd-tree: the tree bt_kd_build makes on the host
// (KdTree::build, src/accel/kdtree.cpp:142-338), node for node, built one
// level at a time on the device.
//
// Level d holds the nodes at depth d, each with its references (triangle id
// and bounds, 32 B) in one array.  Per level:
//   1. split selection.  Nodes over bin_threshold references: binned SAH --
//      start/end bin histograms of each node (shared-memory histograms per
//      chunk of references, added into the node's), then one thread per
//      node scans the bins in the host build's order.  The others: the exact
//      event sweep, one CTA per node -- the events of an axis sorted in
//      shared memory (bitonic), then swept in order by one thread, so ties
//      resolve as in the host build;
//   2. the host compares the best cost with the leaf cost (the same float
//      comparison) and lays out the next level: the children of the split
//      nodes in order, their reference ranges by prefix sums of the counts;
//   3. partition: each reference goes to the side(s) of its node's plane
//      (straddling ones clipped to each child box in double); leaf nodes copy
//      their triangle ids to the leaf store.
// Then each leaf's triangles are sorted (area descending, id ascending), and
// the host numbers the nodes depth first (left child at node + 1) and
// concatenates the leaves in that order: the layout of the recursive build.
//
// The order of a node's references does not enter any decision (counts,
// sorted events, per-reference clipping), so the partition writes them in
// any order.  Positions are compared as floats, so -0 and +0 are one event
// position; the split plane takes the zero sign of its group's first event
// (+0 sorts before -0 among events of one type), which is the host build's
// value whenever a position's events have one sign.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "bt_gpu.h"
#include "kd_rules.h"
#include "kd_tree.h"

void btSetError(const char* msg);

namespace {

constexpr int kThreads = 256;
constexpr int kWarpChunk = 512;     // references per warp in the count and partition kernels
constexpr int kHistChunk = 8192;    // references per CTA in the histogram kernel
constexpr int kLeafThread = 16;     // leaves up to this size are sorted by one thread
constexpr int kLeafBlock = 4096;    // up to this size by one CTA; larger ones on the host

struct __align__(16) Ref {
  float4 lo;  // w: triangle id (bits)
  float4 hi;
};

struct Best {
  int axis;
  float split, cost;
};

struct Chunk {
  uint32_t node, start, len, slot;  // slot: the node's histogram (binned nodes)
};

__device__ __forceinline__ float comp(const float4& v, int a) { return a == 0 ? v.x : (a == 1 ? v.y : v.z); }

// Float -> unsigned key with the same order; -0 and +0 map to one key.
__device__ __forceinline__ uint32_t orderedBits(float f) {
  const uint32_t u = __float_as_uint(f == 0.f ? 0.f : f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fromOrdered(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}
// Sweep event key: position, then type, then 1 for -0.
__device__ __forceinline__ unsigned long long eventKey(float pos, int type) {
  const bool negZero = pos == 0.f && (__float_as_uint(pos) >> 31);
  return (static_cast<unsigned long long>(orderedBits(pos)) << 3) | (unsigned long long)(type << 1) |
         (negZero ? 1ull : 0ull);
}

__global__ void initRefs(const float* __restrict__ pos, const uint32_t* __restrict__ tris, int64_t n, Ref* refs) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float inf = __int_as_float(0x7f800000);
  float lo[3] = {inf, inf, inf}, hi[3] = {-inf, -inf, -inf};
  for (int k = 0; k < 3; ++k) {
    const float* p = pos + 3 * size_t(tris[3 * i + k]);
    for (int a = 0; a < 3; ++a) {
      lo[a] = lo[a] < p[a] ? lo[a] : p[a];
      hi[a] = hi[a] > p[a] ? hi[a] : p[a];
    }
  }
  refs[i].lo = make_float4(lo[0], lo[1], lo[2], __uint_as_float(uint32_t(i)));
  refs[i].hi = make_float4(hi[0], hi[1], hi[2], 0.f);
}

// Binned SAH, step 1: per chunk of one node, start and end bin counts per
// axis in shared memory, added into the node's histogram.
__global__ void __launch_bounds__(kThreads) binHist(const Ref* __restrict__ refs, const kdr::Box* __restrict__ box,
                                                    const Chunk* __restrict__ chunks, int bins, uint32_t* hist) {
  extern __shared__ uint32_t h[];  // [axis][start | end][bin]
  const Chunk c = chunks[blockIdx.x];
  for (int i = threadIdx.x; i < 6 * bins; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const kdr::Box b = box[c.node];
  float scale[3];
  bool ok[3];
  for (int a = 0; a < 3; ++a) {
    ok[a] = b.hi[a] > b.lo[a];
    scale[a] = ok[a] ? float(bins) / (b.hi[a] - b.lo[a]) : 0.f;
  }
  for (uint32_t i = threadIdx.x; i < c.len; i += blockDim.x) {
    const Ref r = refs[c.start + i];
    for (int a = 0; a < 3; ++a) {
      if (!ok[a]) continue;
      atomicAdd(&h[(2 * a) * bins + kdr::binOf(comp(r.lo, a), b.lo[a], scale[a], bins)], 1u);
      atomicAdd(&h[(2 * a + 1) * bins + kdr::binOf(comp(r.hi, a), b.lo[a], scale[a], bins)], 1u);
    }
  }
  __syncthreads();
  uint32_t* out = hist + size_t(c.slot) * 6 * bins;
  for (int i = threadIdx.x; i < 6 * bins; i += blockDim.x)
    if (h[i]) atomicAdd(&out[i], h[i]);
}

// Binned SAH, step 2: one thread per node, candidates in the host build's
// order (axis, then plane), the first of equal costs kept.
__global__ void binSelect(const kdr::Box* __restrict__ box, const uint32_t* __restrict__ count,
                          const uint32_t* __restrict__ nodes, int n, int bins, const uint32_t* __restrict__ hist,
                          kdr::Costs k, Best* best) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t node = nodes[j];
  const kdr::Box b = box[node];
  const uint64_t N = count[node];
  Best r{-1, 0.f, __int_as_float(0x7f800000)};
  for (int axis = 0; axis < 3; ++axis) {
    const float lo = b.lo[axis], hi = b.hi[axis];
    if (!(hi > lo)) continue;
    const uint32_t* st = hist + (size_t(j) * 6 + 2 * axis) * bins;
    const uint32_t* en = st + bins;
    uint64_t nl = 0, nr = N;
    for (int q = 1; q < bins; ++q) {
      nl += st[q - 1];
      nr -= en[q - 1];
      const float s = kdr::binPlane(lo, hi, q, bins);
      const float c = kdr::sahCost(k, b, axis, s, nl, nr);
      if (c < r.cost) r = Best{axis, s, c};
    }
  }
  best[node] = r;
}

__device__ void bitonicSort(unsigned long long* keys, int n) {
  for (int k = 2; k <= n; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long a = keys[i], c = keys[ixj];
          if ((a > c) == ((i & k) == 0)) {
            keys[i] = c;
            keys[ixj] = a;
          }
        }
      }
      __syncthreads();
    }
}

// Exact event sweep: one CTA per node.  Events (end 0, planar 1, start 2)
// keyed by (position, type); the sweep is the host build's loop.
__global__ void __launch_bounds__(kThreads) sweepSelect(const Ref* __restrict__ refs, const kdr::Box* __restrict__ box,
                                                        const uint32_t* __restrict__ start,
                                                        const uint32_t* __restrict__ count,
                                                        const uint32_t* __restrict__ nodes, kdr::Costs k, Best* best) {
  extern __shared__ unsigned long long keys[];
  __shared__ int nev;
  const uint32_t node = nodes[blockIdx.x];
  const kdr::Box b = box[node];
  const uint32_t N = count[node], s0 = start[node];
  Best r{-1, 0.f, __int_as_float(0x7f800000)};
  for (int axis = 0; axis < 3; ++axis) {
    const float lo = b.lo[axis], hi = b.hi[axis];
    if (!(hi > lo)) continue;
    if (threadIdx.x == 0) nev = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
      const Ref rf = refs[s0 + i];
      const float a = comp(rf.lo, axis), e = comp(rf.hi, axis);
      // key: position (ordered bits), type (end 0, planar 1, start 2), -0 marker
      if (a == e) {
        keys[atomicAdd(&nev, 1)] = eventKey(a, 1);
      } else {
        const int at = atomicAdd(&nev, 2);
        keys[at] = eventKey(a, 2);
        keys[at + 1] = eventKey(e, 0);
      }
    }
    __syncthreads();
    const int n = nev;
    int P = 1;
    while (P < n) P <<= 1;
    for (int i = n + threadIdx.x; i < P; i += blockDim.x) keys[i] = ~0ull;
    __syncthreads();
    bitonicSort(keys, P);
    if (threadIdx.x == 0) {
      uint64_t nl = 0, nr = N;
      for (int i = 0; i < n;) {
        const uint32_t pk = uint32_t(keys[i] >> 3);
        const float p = (keys[i] & 1) ? -0.f : fromOrdered(pk);
        uint64_t pe = 0, pp = 0, ps = 0;
        while (i < n && uint32_t(keys[i] >> 3) == pk && ((keys[i] >> 1) & 3) == 0) ++pe, ++i;
        while (i < n && uint32_t(keys[i] >> 3) == pk && ((keys[i] >> 1) & 3) == 1) ++pp, ++i;
        while (i < n && uint32_t(keys[i] >> 3) == pk && ((keys[i] >> 1) & 3) == 2) ++ps, ++i;
        nr -= pe + pp;
        if (p > lo && p < hi) {
          const float c = kdr::sahCost(k, b, axis, p, nl + pp, nr + pp);
          if (c < r.cost) r = Best{axis, p, c};
        }
        nl += ps + pp;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) best[node] = r;
}

// Children counts of the split nodes: a warp per chunk of one node.
__global__ void __launch_bounds__(kThreads) countSides(const Ref* __restrict__ refs, const Chunk* __restrict__ chunks,
                                                       int nChunks, const int32_t* __restrict__ axis,
                                                       const float* __restrict__ split, uint32_t* sideCount) {
  const int w = blockIdx.x * (kThreads / 32) + int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
  if (w >= nChunks) return;
  const Chunk c = chunks[w];
  const int a = axis[c.node];
  if (a < 0) return;
  const float s = split[c.node];
  uint32_t nl = 0, nr = 0;
  for (uint32_t i = uint32_t(lane); i < c.len; i += 32) {
    const Ref r = refs[c.start + i];
    bool left, right, planar;
    kdr::sides(comp(r.lo, a), comp(r.hi, a), s, left, right, planar);
    nl += left;
    nr += right;
  }
  nl = __reduce_add_sync(0xffffffffu, nl);
  nr = __reduce_add_sync(0xffffffffu, nr);
  if (lane == 0) {
    if (nl) atomicAdd(&sideCount[2 * c.node], nl);
    if (nr) atomicAdd(&sideCount[2 * c.node + 1], nr);
  }
}

struct PartitionArgs {
  const Ref* refs;
  Ref* next;
  const Chunk* chunks;
  int nChunks;
  const kdr::Box* box;
  const uint32_t* start;
  const int32_t* axis;
  const float* split;
  const uint32_t* childStart;  // 2 per node: left and right ranges in `next`
  uint32_t* cursor;            // 2 per node
  const uint32_t* leafStart;   // per node: first slot in the leaf store (leaves)
  uint32_t* leafStore;
  const float* pos;
  const uint32_t* tris;
  int clip;
};

__device__ void clipTo(const PartitionArgs& p, const Ref& r, const kdr::Box& box, Ref& out) {
  const uint32_t t = __float_as_uint(r.lo.w);
  const float* v0 = p.pos + 3 * size_t(p.tris[3 * size_t(t)]);
  const float* v1 = p.pos + 3 * size_t(p.tris[3 * size_t(t) + 1]);
  const float* v2 = p.pos + 3 * size_t(p.tris[3 * size_t(t) + 2]);
  const kdr::Box fb{{r.lo.x, r.lo.y, r.lo.z}, {r.hi.x, r.hi.y, r.hi.z}};
  const kdr::Box c = kdr::clippedBounds(v0, v1, v2, box, fb);
  out.lo = make_float4(c.lo[0], c.lo[1], c.lo[2], r.lo.w);
  out.hi = make_float4(c.hi[0], c.hi[1], c.hi[2], 0.f);
}

// Partition: a warp per chunk of one node; slots in each child's range by
// one atomic per warp and side.
__global__ void __launch_bounds__(kThreads) partition(const PartitionArgs p) {
  const int w = blockIdx.x * (kThreads / 32) + int(threadIdx.x >> 5), lane = int(threadIdx.x & 31);
  if (w >= p.nChunks) return;
  const Chunk c = p.chunks[w];
  const int a = p.axis[c.node];
  if (a < 0) {
    const uint32_t base = p.leafStart[c.node] + (c.start - p.start[c.node]);
    for (uint32_t i = uint32_t(lane); i < c.len; i += 32) p.leafStore[base + i] = __float_as_uint(p.refs[c.start + i].lo.w);
    return;
  }
  const float s = p.split[c.node];
  kdr::Box lb = p.box[c.node], rb = lb;
  lb.hi[a] = s;
  rb.lo[a] = s;
  for (uint32_t i0 = 0; i0 < c.len; i0 += 32) {
    const uint32_t i = i0 + uint32_t(lane);
    const bool live = i < c.len;
    Ref r;
    bool left = false, right = false, planar = false;
    if (live) {
      r = p.refs[c.start + i];
      kdr::sides(comp(r.lo, a), comp(r.hi, a), s, left, right, planar);
    }
    const unsigned ml = __ballot_sync(0xffffffffu, left), mr = __ballot_sync(0xffffffffu, right);
    uint32_t bl = 0, br = 0;
    if (lane == 0) {
      if (ml) bl = atomicAdd(&p.cursor[2 * c.node], uint32_t(__popc(ml)));
      if (mr) br = atomicAdd(&p.cursor[2 * c.node + 1], uint32_t(__popc(mr)));
    }
    bl = __shfl_sync(0xffffffffu, bl, 0);
    br = __shfl_sync(0xffffffffu, br, 0);
    const unsigned below = (1u << lane) - 1u;
    const bool clip = left && right && !planar && p.clip;
    if (left) {
      Ref o = r;
      if (clip) clipTo(p, r, lb, o);
      p.next[p.childStart[2 * c.node] + bl + uint32_t(__popc(ml & below))] = o;
    }
    if (right) {
      Ref o = r;
      if (clip) clipTo(p, r, rb, o);
      p.next[p.childStart[2 * c.node + 1] + br + uint32_t(__popc(mr & below))] = o;
    }
  }
}

// Leaf order: area descending, then triangle id ascending.
__device__ __forceinline__ unsigned long long leafKey(const float* area, uint32_t t) {
  return (static_cast<unsigned long long>(~__float_as_uint(area[t])) << 32) | t;
}

__global__ void sortSmallLeaves(uint32_t* store, const uint32_t* __restrict__ begin, const uint32_t* __restrict__ len,
                                int n, const float* __restrict__ area) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  unsigned long long k[kLeafThread];
  const uint32_t b = begin[j], m = len[j];
  for (uint32_t i = 0; i < m; ++i) {
    const unsigned long long x = leafKey(area, store[b + i]);
    uint32_t q = i;
    while (q > 0 && k[q - 1] > x) {
      k[q] = k[q - 1];
      --q;
    }
    k[q] = x;
  }
  for (uint32_t i = 0; i < m; ++i) store[b + i] = uint32_t(k[i]);
}

__global__ void __launch_bounds__(kThreads) sortLeaves(uint32_t* store, const uint32_t* __restrict__ begin,
                                                       const uint32_t* __restrict__ len,
                                                       const float* __restrict__ area) {
  extern __shared__ unsigned long long keys[];
  const uint32_t b = begin[blockIdx.x], m = len[blockIdx.x];
  int P = 1;
  while (P < int(m)) P <<= 1;
  for (int i = threadIdx.x; i < P; i += blockDim.x) keys[i] = i < int(m) ? leafKey(area, store[b + i]) : ~0ull;
  __syncthreads();
  bitonicSort(keys, P);
  for (int i = threadIdx.x; i < int(m); i += blockDim.x) store[b + i] = uint32_t(keys[i]);
}

// ---- host side ----

struct Err {
  int code = BT_OK;
  std::string msg;
};

template <class T>
struct Dev {
  T* p = nullptr;
  size_t n = 0;
  ~Dev() {
    if (p) cudaFree(p);
  }
  bool reserve(size_t m, Err& e) {
    if (m <= n) return true;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    const cudaError_t ce = cudaMalloc(&p, std::max<size_t>(m, 1) * sizeof(T));
    if (ce != cudaSuccess) {
      e.code = ce == cudaErrorMemoryAllocation ? BT_ERR_NOMEM : BT_ERR_CUDA;
      e.msg = std::string("cudaMalloc: ") + cudaGetErrorString(ce);
      return false;
    }
    n = std::max<size_t>(m, 1);
    return true;
  }
  // grows to at least m elements keeping the first `keep` (stream-ordered copy)
  bool grow(size_t m, size_t keep, cudaStream_t st, Err& e) {
    if (m <= n) return true;
    Dev<T> q;
    if (!q.reserve(std::max(m, n + n / 2), e)) return false;
    if (keep && cudaMemcpyAsync(q.p, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st) != cudaSuccess) {
      e.code = BT_ERR_CUDA;
      e.msg = "leaf store copy";
      return false;
    }
    std::swap(p, q.p);
    std::swap(n, q.n);
    return true;
  }
};

bool ck(cudaError_t ce, Err& e, const char* what) {
  if (ce == cudaSuccess) return true;
  e.code = BT_ERR_CUDA;
  e.msg = std::string(what) + ": " + cudaGetErrorString(ce);
  return false;
}

// One node of a finished level, as the host keeps it for the layout.
struct NodeRec {
  int32_t axis;      // -1: leaf
  float split;
  uint32_t child;    // split: left child's index in the next level (right = child + 1)
  uint32_t leaf;     // leaf: first slot in the leaf store
  uint32_t count;    // leaf: triangles
};

template <class T>
bool upload(Dev<T>& d, const std::vector<T>& h, cudaStream_t st, Err& e) {
  if (!d.reserve(h.size(), e)) return false;
  return h.empty() || ck(cudaMemcpyAsync(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, st), e, "upload");
}

template <class T>
bool download(std::vector<T>& h, const Dev<T>& d, size_t n, cudaStream_t st, Err& e) {
  h.resize(n);
  if (!n) return true;
  return ck(cudaMemcpyAsync(h.data(), d.p, n * sizeof(T), cudaMemcpyDeviceToHost, st), e, "download") &&
         ck(cudaStreamSynchronize(st), e, "build step");
}

int buildOnDevice(const float* pos, int64_t numVerts, const uint32_t* tris, const float* area, int64_t numTris,
                  const float* sceneBounds, const bt_kd_params& prm, cudaStream_t st, bt_kd_tree* t, Err& e) {
  kdr::Box root;
  int maxDepth;
  kdRootAndDepth(sceneBounds, prm, numTris, root, maxDepth);
  const kdr::Costs costs{prm.cost_traverse, prm.cost_intersect, prm.empty_bonus};
  const int bins = prm.bins;
  const uint32_t binThreshold = uint32_t(std::max(prm.bin_threshold, 0));
  int P = 1;
  while (P < int(2 * binThreshold)) P <<= 1;
  const size_t sweepShared = size_t(P) * sizeof(unsigned long long);
  if (bins < 1 || bins > 4096 || sweepShared > 200 * 1024) {
    e.code = BT_ERR_INVALID;
    e.msg = "bt_kd_build_gpu: bins must be 1..4096 and bin_threshold at most 12800";
    return e.code;
  }
  if (sweepShared > 48 * 1024 &&
      !ck(cudaFuncSetAttribute(sweepSelect, cudaFuncAttributeMaxDynamicSharedMemorySize, int(sweepShared)), e,
          "sweep shared memory"))
    return e.code;
  if (!ck(cudaFuncSetAttribute(sortLeaves, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kLeafBlock * sizeof(unsigned long long))),
          e, "leaf sort shared memory"))
    return e.code;

  Dev<float> dPos, dArea;
  Dev<uint32_t> dTris;
  if (!dPos.reserve(size_t(3 * numVerts), e) || !dTris.reserve(size_t(3 * numTris), e) ||
      !dArea.reserve(size_t(numTris), e))
    return e.code;
  if (!ck(cudaMemcpyAsync(dPos.p, pos, size_t(3 * numVerts) * 4, cudaMemcpyHostToDevice, st), e, "upload") ||
      !ck(cudaMemcpyAsync(dTris.p, tris, size_t(3 * numTris) * 4, cudaMemcpyHostToDevice, st), e, "upload") ||
      !ck(cudaMemcpyAsync(dArea.p, area, size_t(numTris) * 4, cudaMemcpyHostToDevice, st), e, "upload"))
    return e.code;
  Dev<Ref> refs[2];
  if (!refs[0].reserve(size_t(numTris), e)) return e.code;
  if (numTris) initRefs<<<unsigned((numTris + kThreads - 1) / kThreads), kThreads, 0, st>>>(dPos.p, dTris.p, numTris,
                                                                                             refs[0].p);

  // the current level
  std::vector<kdr::Box> box(1, root);
  std::vector<uint32_t> start(1, 0u), count(1, uint32_t(numTris));
  std::vector<std::vector<NodeRec>> levels;
  Dev<kdr::Box> dBox;
  Dev<uint32_t> dStart, dCount, dNodes, dHist, dSide, dChild, dCursor, dLeafStart, dStore;
  Dev<Best> dBest;
  Dev<Chunk> dChunks;
  Dev<int32_t> dAxis;
  Dev<float> dSplit;
  uint64_t storeUsed = 0;
  int cur = 0;
  for (int depth = 0; !box.empty(); ++depth) {
    const size_t n = box.size();
    if (!upload(dBox, box, st, e) || !upload(dStart, start, st, e) || !upload(dCount, count, st, e)) return e.code;
    std::vector<uint32_t> large, small;
    std::vector<Chunk> histChunks;
    for (size_t j = 0; j < n; ++j) {
      const bool cand = !prm.single_leaf && count[j] > 1 && depth < maxDepth && kdr::surfaceArea(box[j]) > 0;
      if (!cand) continue;
      if (count[j] > binThreshold) {
        for (uint32_t s = 0; s < count[j]; s += kHistChunk)
          histChunks.push_back(Chunk{uint32_t(j), start[j] + s, std::min<uint32_t>(kHistChunk, count[j] - s),
                                     uint32_t(large.size())});
        large.push_back(uint32_t(j));
      } else {
        small.push_back(uint32_t(j));
      }
    }
    if (!dBest.reserve(n, e)) return e.code;
    if (!large.empty()) {
      if (!upload(dNodes, large, st, e) || !upload(dChunks, histChunks, st, e) ||
          !dHist.reserve(large.size() * 6 * size_t(bins), e) ||
          !ck(cudaMemsetAsync(dHist.p, 0, large.size() * 6 * size_t(bins) * 4, st), e, "memset"))
        return e.code;
      binHist<<<unsigned(histChunks.size()), kThreads, 6 * size_t(bins) * 4, st>>>(refs[cur].p, dBox.p, dChunks.p,
                                                                                   bins, dHist.p);
      binSelect<<<unsigned((large.size() + 127) / 128), 128, 0, st>>>(dBox.p, dCount.p, dNodes.p, int(large.size()),
                                                                     bins, dHist.p, costs, dBest.p);
    }
    Dev<uint32_t> dSmall;
    if (!small.empty()) {
      if (!upload(dSmall, small, st, e)) return e.code;
      sweepSelect<<<unsigned(small.size()), kThreads, sweepShared, st>>>(refs[cur].p, dBox.p, dStart.p, dCount.p,
                                                                        dSmall.p, costs, dBest.p);
    }
    if (!ck(cudaGetLastError(), e, "split selection")) return e.code;
    std::vector<Best> best;
    if (!download(best, dBest, n, st, e)) return e.code;
    // split or leaf (KdTree::build's test), and the next level's layout
    std::vector<int32_t> axis(n, -1);
    std::vector<float> split(n, 0.f);
    std::vector<char> cand(n, 0);
    for (uint32_t j : large) cand[j] = 1;
    for (uint32_t j : small) cand[j] = 1;
    bool anySplit = false;
    for (size_t j = 0; j < n; ++j) {
      if (!cand[j]) continue;
      const float leafCost = prm.cost_intersect * float(count[j]);
      if (best[j].axis >= 0 && best[j].cost < leafCost) {
        axis[j] = best[j].axis;
        split[j] = best[j].split;
        anySplit = true;
      }
    }
    std::vector<Chunk> chunks;
    for (size_t j = 0; j < n; ++j)
      for (uint32_t s = 0; s < count[j]; s += kWarpChunk)
        chunks.push_back(Chunk{uint32_t(j), start[j] + s, std::min<uint32_t>(kWarpChunk, count[j] - s), 0});
    if (!upload(dAxis, axis, st, e) || !upload(dSplit, split, st, e) || !upload(dChunks, chunks, st, e)) return e.code;
    const unsigned warpBlocks = unsigned((chunks.size() + kThreads / 32 - 1) / (kThreads / 32));
    std::vector<uint32_t> side(2 * n, 0u);
    if (anySplit) {
      if (!dSide.reserve(2 * n, e) || !ck(cudaMemsetAsync(dSide.p, 0, 2 * n * 4, st), e, "memset")) return e.code;
      if (warpBlocks)
        countSides<<<warpBlocks, kThreads, 0, st>>>(refs[cur].p, dChunks.p, int(chunks.size()), dAxis.p, dSplit.p,
                                                   dSide.p);
      if (!ck(cudaGetLastError(), e, "count") || !download(side, dSide, 2 * n, st, e)) return e.code;
    }
    std::vector<NodeRec> rec(n);
    const uint64_t storeBefore = storeUsed;
    std::vector<kdr::Box> nbox;
    std::vector<uint32_t> nstart, ncount, childStart(2 * n, 0u), leafStart(n, 0u);
    uint64_t nextRefs = 0;
    for (size_t j = 0; j < n; ++j) {
      rec[j].axis = axis[j];
      rec[j].split = split[j];
      if (axis[j] < 0) {
        rec[j].leaf = uint32_t(storeUsed);
        rec[j].count = count[j];
        leafStart[j] = uint32_t(storeUsed);
        storeUsed += count[j];
        continue;
      }
      rec[j].child = uint32_t(nbox.size());
      kdr::Box lb = box[j], rb = box[j];
      lb.hi[axis[j]] = split[j];
      rb.lo[axis[j]] = split[j];
      for (int s = 0; s < 2; ++s) {
        childStart[2 * j + size_t(s)] = uint32_t(nextRefs);
        nbox.push_back(s ? rb : lb);
        nstart.push_back(uint32_t(nextRefs));
        ncount.push_back(side[2 * j + size_t(s)]);
        nextRefs += side[2 * j + size_t(s)];
      }
    }
    if (nextRefs > 0xffffffffull || storeUsed > 0xffffffffull) {
      e.code = BT_ERR_NOMEM;
      e.msg = "bt_kd_build_gpu: more than 2^32 triangle references";
      return e.code;
    }
    // (the leaf store keeps the earlier levels' leaves)
    if (!refs[cur ^ 1].reserve(size_t(nextRefs), e) || !dStore.grow(size_t(storeUsed), size_t(storeBefore), st, e))
      return e.code;
    levels.push_back(std::move(rec));
    if (!upload(dChild, childStart, st, e) || !upload(dLeafStart, leafStart, st, e) || !dCursor.reserve(2 * n, e) ||
        !ck(cudaMemsetAsync(dCursor.p, 0, 2 * n * 4, st), e, "memset"))
      return e.code;
    PartitionArgs pa;
    pa.refs = refs[cur].p;
    pa.next = refs[cur ^ 1].p;
    pa.chunks = dChunks.p;
    pa.nChunks = int(chunks.size());
    pa.box = dBox.p;
    pa.start = dStart.p;
    pa.axis = dAxis.p;
    pa.split = dSplit.p;
    pa.childStart = dChild.p;
    pa.cursor = dCursor.p;
    pa.leafStart = dLeafStart.p;
    pa.leafStore = dStore.p;
    pa.pos = dPos.p;
    pa.tris = dTris.p;
    pa.clip = prm.clip_bounds;
    if (warpBlocks) partition<<<warpBlocks, kThreads, 0, st>>>(pa);
    if (!ck(cudaGetLastError(), e, "partition")) return e.code;
    box.swap(nbox);
    start.swap(nstart);
    count.swap(ncount);
    cur ^= 1;
  }
  // leaf order
  std::vector<uint32_t> sb, sl, bb, bl, hb, hl;
  for (const auto& lv : levels)
    for (const NodeRec& r : lv) {
      if (r.axis >= 0 || r.count < 2) continue;
      if (r.count <= uint32_t(kLeafThread)) {
        sb.push_back(r.leaf);
        sl.push_back(r.count);
      } else if (r.count <= uint32_t(kLeafBlock)) {
        bb.push_back(r.leaf);
        bl.push_back(r.count);
      } else {
        hb.push_back(r.leaf);
        hl.push_back(r.count);
      }
    }
  Dev<uint32_t> dB0, dL0, dB1, dL1;
  if (!upload(dB0, sb, st, e) || !upload(dL0, sl, st, e) || !upload(dB1, bb, st, e) || !upload(dL1, bl, st, e))
    return e.code;
  if (!sb.empty())
    sortSmallLeaves<<<unsigned((sb.size() + 127) / 128), 128, 0, st>>>(dStore.p, dB0.p, dL0.p, int(sb.size()),
                                                                        dArea.p);
  if (!bb.empty())
    sortLeaves<<<unsigned(bb.size()), kThreads, kLeafBlock * sizeof(unsigned long long), st>>>(dStore.p, dB1.p, dL1.p,
                                                                                               dArea.p);
  if (!ck(cudaGetLastError(), e, "leaf sort")) return e.code;
  std::vector<uint32_t> store;
  if (!download(store, dStore, size_t(storeUsed), st, e)) return e.code;
  for (size_t i = 0; i < hb.size(); ++i)
    std::sort(store.begin() + hb[i], store.begin() + hb[i] + hl[i], [&](uint32_t a, uint32_t b) {
      return area[a] != area[b] ? area[a] > area[b] : a < b;
    });
  // depth-first numbering: a node, its left subtree, then its right subtree
  struct Item {
    uint32_t level, index, parent;  // parent: the split node whose right child this is (~0u: none)
  };
  std::vector<Item> stack{{0u, 0u, ~0u}};
  int leaves = 0;
  while (!stack.empty()) {
    const Item it = stack.back();
    stack.pop_back();
    const NodeRec& r = levels[it.level][it.index];
    const uint32_t id = uint32_t(t->split.size());
    if (it.parent != ~0u) t->data[it.parent] |= id << 2;
    if (r.axis < 0) {
      t->split.push_back(0.f);
      t->data.push_back((r.count << 2) | 3u);
      t->offset.push_back(uint32_t(t->triIndices.size()));
      t->triIndices.insert(t->triIndices.end(), store.begin() + r.leaf, store.begin() + r.leaf + r.count);
      ++leaves;
      continue;
    }
    t->split.push_back(r.split);
    t->data.push_back(uint32_t(r.axis));
    t->offset.push_back(0u);
    stack.push_back(Item{it.level + 1, r.child + 1, id});
    stack.push_back(Item{it.level + 1, r.child, ~0u});
  }
  t->numLeaves = leaves;
  t->maxDepth = int(levels.size()) - 1;
  for (int a = 0; a < 3; ++a) {
    t->bounds[a] = root.lo[a];
    t->bounds[3 + a] = root.hi[a];
  }
  kdFinish(t);
  return BT_OK;
}

}  // namespace

extern "C" int bt_kd_build_gpu(const float* pos, int64_t numVerts, const uint32_t* tris, const float* triArea,
                               int64_t numTris, const float* sceneBounds, const bt_kd_params* params, int32_t device,
                               bt_kd_tree** out, double* ms) {
  if (!out || !pos || !tris || !triArea || !sceneBounds || numTris < 0 || numVerts < 0 || numTris >= (1ll << 31)) {
    btSetError("bt_kd_build_gpu: bad arguments");
    return BT_ERR_INVALID;
  }
  *out = nullptr;
  for (int64_t i = 0; i < 3 * numTris; ++i)
    if (int64_t(tris[i]) >= numVerts) {
      btSetError("bt_kd_build_gpu: triangle index out of range");
      return BT_ERR_INVALID;
    }
  bt_kd_params p;
  if (params)
    p = *params;
  else
    bt_kd_params_default(&p);
  const auto t0 = std::chrono::steady_clock::now();
  int prev = 0, ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    btSetError("bt_kd_build_gpu: no such CUDA device");
    return BT_ERR_NODEVICE;
  }
  cudaGetDevice(&prev);
  Err e;
  bt_kd_tree* t = new bt_kd_tree();
  cudaStream_t st = nullptr;
  if (ck(cudaSetDevice(device), e, "cudaSetDevice") && ck(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), e, "stream"))
    buildOnDevice(pos, numVerts, tris, triArea, numTris, sceneBounds, p, st, t, e);
  if (st) {
    if (e.code == BT_OK) ck(cudaStreamSynchronize(st), e, "build");
    cudaStreamDestroy(st);
  }
  cudaSetDevice(prev);
  if (e.code != BT_OK) {
    delete t;
    btSetError(e.msg.c_str());
    return e.code;
  }
  if (ms) *ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *out = t;
  return BT_OK;
}
