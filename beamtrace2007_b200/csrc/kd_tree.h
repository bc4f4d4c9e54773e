// The kd-tree as bt_kd_build and bt_kd_build_gpu return it (bt_kd_tree of
// include/bt_gpu.h), and the steps both builds share.
#pragma once

#include <cstdint>
#include <vector>

#include "bt_gpu.h"
#include "kd_rules.h"

struct bt_kd_tree {
  std::vector<float> split;
  std::vector<uint32_t> data, offset, parent, triIndices;
  std::vector<float> nodeBox;  // 6 per node: lo xyz, hi xyz
  float bounds[6];
  int numLeaves, maxDepth;
};

// Root box (scene bounds padded by 1e-4 of the diagonal + 1e-6) and the
// depth limit (8 + 1.3 log2 N unless set, at most 63) (kdtree.cpp:296-310).
void kdRootAndDepth(const float* sceneBounds, const bt_kd_params& p, int64_t numTris, kdr::Box& root, int& maxDepth);

// Parents and node boxes as a descent from the root computes them, from
// split / data and the root box in `bounds` (kdtree.cpp:318-336).
void kdFinish(bt_kd_tree* t);
