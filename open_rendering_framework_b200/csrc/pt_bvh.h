// Host BVH builder interface (implementation in pt_bvh.cu; layout documented in pt_scene.cuh).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "pt_scene.cuh"

namespace pt {

struct BvhHost {
  std::vector<float4> nodes;                 // 4 float4 per node, root = node 0
  std::vector<float4> tri_v0, tri_e1, tri_e2;  // leaf order
  std::vector<uint32_t> order;               // leaf position -> original triangle index
  int depth = 0;                             // levels including the leaves
};

// Binned-SAH parameters: the cost of a node step relative to one triangle test, and the largest leaf
// the SAH may choose (1..15; a leaf is forced only where no split separates the centroids).
struct BvhParams {
  float trav_cost = 1.2f;
  int max_leaf = 8;
  int collapse = 1;         // 4-wide collapse: 0 greedy (largest area opened first), 1 SAH-optimal
  float wide_cost = 1.5f;   // SAH cost of a wide node visit relative to one triangle test (collapse 1)
  int treelet_rounds = 3;   // device builder: rounds of treelet restructuring after the LBVH (0 = none)
  int treelet_min = 8;      // device builder: treelets only at nodes of at least this many triangles
};

// tri_pos: 9 floats per triangle (v0, v1, v2).  Returns false if the scene is too large for the
// node encoding (2^27 triangles) or the tree is deeper than the traversal trail allows.
bool build_bvh(const float* tri_pos, uint32_t n_tris, BvhHost& out, const BvhParams& params = BvhParams());

// The BVH2 collapsed into a wide BVH of kWide children per node over the same leaves (kWideStride
// float4 per node, root = node 0; layout in pt_scene.cuh).  Returns false (and leaves nodes4 empty)
// when the wide tree would be deeper than kMaxDepthWide levels, whose pending children the traversal
// stack could not hold.
constexpr int kMaxDepth4 = kMaxDepthWide;
bool build_bvh4(const BvhHost& bvh2, std::vector<float4>& nodes4, int& depth4, const BvhParams& params = BvhParams());

// The diagonal of the bounding box of n triangles (9 floats each): the scale of the box tests' margin
// (SceneDev::trav_scale).
float scene_diagonal(const float* tri_pos, uint32_t n);

}  // namespace pt
