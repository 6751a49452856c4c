// BVH construction (host): binned-SAH BVH2 flattened into child-pair nodes with parent links, and
// triangles reordered into leaf order as Moller-Trumbore records (see pt_scene.cuh for the layout).
//
// The reference relies on OptiX's Trbvh/Sbvh builders (OptixSceneLoader.cpp:136,
// ObjLoader.cpp:387-399), which are not available; this builder only has to produce a valid BVH,
// because hit results are decided by the triangle test alone (closest t, ties to the lower
// triangle index), so any valid tree gives the same hits as a brute-force loop.
//
// Build: 32 centroid bins per axis, SAH with traversal cost 1.2 and intersection cost 1 per
// triangle, leaves of at most 8 triangles (15 when forced), object-median splits below depth 48 so
// the depth stays below the traversal's 64-level trail.  Subtrees with more than 32k triangles are
// built on separate host threads.
#include <algorithm>
#include <array>
#include <limits>
#include <atomic>
#include <cmath>
#include <cstring>
#include <functional>
#include <future>
#include <memory>
#include <thread>
#include <vector>

#include "pt_bvh.h"

namespace pt {
namespace {

struct Box {
  float lo[3] = {INFINITY, INFINITY, INFINITY};
  float hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  void grow(const float* p)
  {
    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], p[k]); hi[k] = std::max(hi[k], p[k]); }
  }
  void grow(const Box& b)
  {
    for (int k = 0; k < 3; ++k) { lo[k] = std::min(lo[k], b.lo[k]); hi[k] = std::max(hi[k], b.hi[k]); }
  }
  float area() const
  {
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = std::max(0.0f, hi[k] - lo[k]);
    return 2.0f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
  }
};

struct TriRef {
  Box box;
  float c[3];
};

struct TmpNode {
  Box box[2];
  int child_kind[2];  // 0 = internal (node ptr), 1 = leaf
  std::unique_ptr<TmpNode> node[2];
  uint32_t first[2], count[2];
};

constexpr int kBins = 32;
constexpr int kForcedMaxLeaf = 15;
constexpr int kMedianDepth = 48;

struct Builder {
  const std::vector<TriRef>& refs;
  std::vector<uint32_t>& idx;
  std::atomic<int> max_depth{0};
  const int kMaxLeaf;      // largest leaf the SAH may choose
  const float kTravCost;   // SAH cost of a node step relative to one triangle test
  Builder(const std::vector<TriRef>& r, std::vector<uint32_t>& i, const BvhParams& p)
      : refs(r), idx(i), kMaxLeaf(p.max_leaf), kTravCost(p.trav_cost) {}

  Box bounds(uint32_t b, uint32_t e, Box* cbox) const
  {
    Box bb, cb;
    for (uint32_t i = b; i < e; ++i) {
      const TriRef& t = refs[idx[i]];
      bb.grow(t.box);
      cb.grow(t.c);
    }
    if (cbox) *cbox = cb;
    return bb;
  }

  // Returns the split position (b < mid < e) for [b, e).
  uint32_t split(uint32_t b, uint32_t e, const Box& cb, int depth, bool& make_leaf)
  {
    uint32_t n = e - b;
    make_leaf = false;
    int axis = 0;
    float ext[3];
    for (int k = 0; k < 3; ++k) ext[k] = cb.hi[k] - cb.lo[k];
    if (ext[1] > ext[axis]) axis = 1;
    if (ext[2] > ext[axis]) axis = 2;
    if (!(ext[axis] > 0.0f)) {  // all centroids coincide: any partition is as good
      if (n <= (uint32_t)kForcedMaxLeaf) { make_leaf = true; return e; }
      return b + n / 2;
    }
    if (depth >= kMedianDepth) {
      uint32_t mid = b + n / 2;
      std::nth_element(idx.begin() + b, idx.begin() + mid, idx.begin() + e,
                       [&](uint32_t x, uint32_t y) { return refs[x].c[axis] < refs[y].c[axis]; });
      return mid;
    }
    float best_cost = INFINITY;
    int best_axis = -1, best_bin = -1;
    for (int a = 0; a < 3; ++a) {
      if (!(ext[a] > 0.0f)) continue;
      Box bin_box[kBins];
      uint32_t bin_cnt[kBins] = {0};
      float scale = (float)kBins / ext[a];
      for (uint32_t i = b; i < e; ++i) {
        const TriRef& t = refs[idx[i]];
        int bi = std::min(kBins - 1, std::max(0, (int)((t.c[a] - cb.lo[a]) * scale)));
        bin_cnt[bi]++;
        bin_box[bi].grow(t.box);
      }
      float right_area[kBins];
      uint32_t right_cnt[kBins];
      Box acc;
      uint32_t cnt = 0;
      for (int i = kBins - 1; i > 0; --i) {
        acc.grow(bin_box[i]);
        cnt += bin_cnt[i];
        right_area[i] = acc.area();
        right_cnt[i] = cnt;
      }
      acc = Box();
      cnt = 0;
      for (int i = 0; i < kBins - 1; ++i) {
        acc.grow(bin_box[i]);
        cnt += bin_cnt[i];
        if (cnt == 0 || right_cnt[i + 1] == 0) continue;
        float cost = acc.area() * (float)cnt + right_area[i + 1] * (float)right_cnt[i + 1];
        if (cost < best_cost) { best_cost = cost; best_axis = a; best_bin = i; }
      }
    }
    Box all;
    for (uint32_t i = b; i < e; ++i) all.grow(refs[idx[i]].box);
    float parent_area = all.area();
    float leaf_cost = (float)n;
    float split_cost = parent_area > 0.0f ? kTravCost + best_cost / parent_area : INFINITY;
    if (best_axis < 0) {
      if (n <= (uint32_t)kForcedMaxLeaf) { make_leaf = true; return e; }
      return b + n / 2;
    }
    if (n <= (uint32_t)kMaxLeaf && split_cost >= leaf_cost) { make_leaf = true; return e; }
    float scale = (float)kBins / ext[best_axis];
    auto it = std::partition(idx.begin() + b, idx.begin() + e, [&](uint32_t x) {
      int bi = std::min(kBins - 1, std::max(0, (int)((refs[x].c[best_axis] - cb.lo[best_axis]) * scale)));
      return bi <= best_bin;
    });
    uint32_t mid = (uint32_t)(it - idx.begin());
    if (mid == b || mid == e) mid = b + n / 2;
    return mid;
  }

  // Builds the subtree over [b, e) into `slot` of `parent` (child k).
  void build_child(TmpNode* parent, int k, uint32_t b, uint32_t e, int depth)
  {
    Box cb;
    parent->box[k] = bounds(b, e, &cb);
    int d = depth;
    int cur = max_depth.load();
    while (d > cur && !max_depth.compare_exchange_weak(cur, d)) {}
    uint32_t n = e - b;
    bool leaf = false;
    uint32_t mid = e;
    if (n <= 1) leaf = true;
    else mid = split(b, e, cb, depth, leaf);
    if (leaf) {
      parent->child_kind[k] = 1;
      parent->first[k] = b;
      parent->count[k] = n;
      return;
    }
    parent->child_kind[k] = 0;
    parent->node[k].reset(new TmpNode());
    TmpNode* node = parent->node[k].get();
    if (n > 32768 && depth < 8) {
      auto fut = std::async(std::launch::async, [=] { build_child(node, 0, b, mid, depth + 1); });
      build_child(node, 1, mid, e, depth + 1);
      fut.get();
    } else {
      build_child(node, 0, b, mid, depth + 1);
      build_child(node, 1, mid, e, depth + 1);
    }
  }
};

void flatten(const TmpNode* n, int parent, std::vector<float4>& out, int& index_out)
{
  int me = (int)(out.size() / 4);
  index_out = me;
  out.resize(out.size() + 4);
  int child_ref[2];
  for (int k = 0; k < 2; ++k) {
    if (n->child_kind[k] == 1) {
      child_ref[k] = (int)(0x80000000u | (n->first[k] << 4) | n->count[k]);
    } else {
      int ci;
      flatten(n->node[k].get(), me, out, ci);
      child_ref[k] = ci;
    }
  }
  float4* nd = out.data() + 4 * me;
  auto box_or_far = [](const Box& b, int k, bool lo) {
    if (!(b.lo[0] <= b.hi[0])) return 1e30f;  // empty child: a point far outside any ray's reach
    return lo ? b.lo[k] : b.hi[k];
  };
  nd[0] = make_float4(box_or_far(n->box[0], 0, true), box_or_far(n->box[0], 0, false), box_or_far(n->box[0], 1, true),
                      box_or_far(n->box[0], 1, false));
  nd[1] = make_float4(box_or_far(n->box[1], 0, true), box_or_far(n->box[1], 0, false), box_or_far(n->box[1], 1, true),
                      box_or_far(n->box[1], 1, false));
  nd[2] = make_float4(box_or_far(n->box[0], 2, true), box_or_far(n->box[0], 2, false), box_or_far(n->box[1], 2, true),
                      box_or_far(n->box[1], 2, false));
  int4 n3 = make_int4(child_ref[0], child_ref[1], parent, 0);
  memcpy(&nd[3], &n3, sizeof(n3));
}

}  // namespace

bool build_bvh(const float* tri_pos, uint32_t n_tris, BvhHost& out, const BvhParams& params)
{
  out = BvhHost();
  if (n_tris >= (1u << 27)) return false;
  std::vector<TriRef> refs(n_tris);
  for (uint32_t i = 0; i < n_tris; ++i) {
    const float* p = tri_pos + 9 * (size_t)i;
    TriRef& r = refs[i];
    r.box.grow(p);
    r.box.grow(p + 3);
    r.box.grow(p + 6);
    for (int k = 0; k < 3; ++k) r.c[k] = 0.5f * (r.box.lo[k] + r.box.hi[k]);
  }
  std::vector<uint32_t> idx(n_tris);
  for (uint32_t i = 0; i < n_tris; ++i) idx[i] = i;
  Builder B(refs, idx, params);
  // Root: an internal node whose two children split the triangles; with fewer than two triangles
  // the second child is an empty leaf.
  TmpNode root;
  if (n_tris <= 1) {
    root.child_kind[0] = 1;
    root.first[0] = 0;
    root.count[0] = n_tris;
    if (n_tris) root.box[0] = B.bounds(0, n_tris, nullptr);
    root.child_kind[1] = 1;
    root.first[1] = 0;
    root.count[1] = 0;
  } else {
    Box cb;
    B.bounds(0, n_tris, &cb);
    bool leaf = false;
    uint32_t mid = B.split(0, n_tris, cb, 0, leaf);
    if (leaf || mid == 0 || mid >= n_tris) mid = n_tris / 2;
    B.build_child(&root, 0, 0, mid, 1);
    B.build_child(&root, 1, mid, n_tris, 1);
  }
  int root_index = 0;
  flatten(&root, -1, out.nodes, root_index);
  out.depth = B.max_depth.load() + 1;
  out.tri_v0.resize(n_tris);
  out.tri_e1.resize(n_tris);
  out.tri_e2.resize(n_tris);
  out.order = idx;
  for (uint32_t j = 0; j < n_tris; ++j) {
    uint32_t i = idx[j];
    const float* p = tri_pos + 9 * (size_t)i;
    int orig = (int)i;
    float w;
    memcpy(&w, &orig, 4);
    out.tri_v0[j] = make_float4(p[0], p[1], p[2], w);
    out.tri_e1[j] = make_float4(p[3] - p[0], p[4] - p[1], p[5] - p[2], 0.0f);
    out.tri_e2[j] = make_float4(p[6] - p[0], p[7] - p[1], p[8] - p[2], 0.0f);
  }
  return out.depth < 64;
}

float scene_diagonal(const float* tri_pos, uint32_t n)
{
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (size_t i = 0; i < (size_t)n * 3; ++i)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], tri_pos[3 * i + k]);
      hi[k] = std::max(hi[k], tri_pos[3 * i + k]);
    }
  double d2 = 0.0;
  for (int k = 0; k < 3; ++k) d2 += (double)(hi[k] - lo[k]) * (hi[k] - lo[k]);
  return n ? (float)std::sqrt(d2) : 0.0f;
}

// Collapse of the BVH2 into the wide layout over the same leaves.
//  * collapse 0 (greedy): starting from a BVH2 node's two children, the internal child of largest
//    surface area is replaced by its own two children until there are four or no internal child is
//    left (the usual greedy collapse of a binary SAH tree into a wide one).
//  * collapse 1 (SAH-optimal over the given BVH2): a dynamic program over the BVH2 picks, for every wide
//    node, which BVH2 nodes below it become its up to four children, minimising the SAH cost
//    sum(wide nodes) wide_cost * A + sum(leaves) A * triangles, the BVH2's leaves kept as they are (the
//    cost model of H. Ylitie, T. Karras, S. Laine, "Efficient Incoherent Ray Traversal on GPUs Through
//    Compressed Wide BVHs", HPG 2017, for 4 children and fixed leaves):
//      W(x)    = wide_cost * A(x) + D(x, 4)                   x as the root of a wide node
//      D(x, j) = min_{k=1..j-1} S(left(x), k) + S(right(x), j - k)   x's children in at most j slots
//      S(y, 1) = leaf cost, or W(y);  S(y, i >= 2) = min(S(y, 1), D(y, i))   y in at most i slots
bool build_bvh4(const BvhHost& b2, std::vector<float4>& out4, int& depth4, const BvhParams& params)
{
  out4.clear();
  depth4 = 0;
  struct Kid {
    int code;          // BVH2 node index (>= 0) or leaf code (< 0)
    float lo[3], hi[3];
  };
  auto kid = [&](int node, int k) {
    const float4* nd = b2.nodes.data() + 4 * (size_t)node;
    Kid c;
    int4 n3;
    memcpy(&n3, &nd[3], sizeof(n3));
    c.code = k == 0 ? n3.x : n3.y;
    const float4& a = nd[k];
    c.lo[0] = a.x; c.hi[0] = a.y; c.lo[1] = a.z; c.hi[1] = a.w;
    c.lo[2] = k == 0 ? nd[2].x : nd[2].z;
    c.hi[2] = k == 0 ? nd[2].y : nd[2].w;
    return c;
  };
  auto area = [](const Kid& c) {
    float d[3];
    for (int k = 0; k < 3; ++k) d[k] = std::max(0.0f, c.hi[k] - c.lo[k]);
    return d[0] * d[1] + d[1] * d[2] + d[2] * d[0];
  };
  const size_t n_nodes = b2.nodes.size() / 4;
  // SAH-optimal choices: per BVH2 node y and slot budget i (1..4), choice[y][i] = 0 for "y in one slot
  // (its own wide node)", else the slots k given to y's first child when y is opened (i - k to the
  // second); wsplit[x] the split of W(x)'s four slots.
  std::vector<std::array<uint8_t, kWide + 1>> choice;
  std::vector<uint8_t> wsplit;
  if (params.collapse == 1 && n_nodes > 0) {
    choice.assign(n_nodes, {});
    wsplit.assign(n_nodes, 1);
    std::vector<std::array<double, kWide + 1>> S(n_nodes);
    std::vector<double> A(n_nodes, 0.0);
    const double inf = std::numeric_limits<double>::infinity();
    // children before parents: a reverse pre-order of the BVH2
    std::vector<int> order;
    order.reserve(n_nodes);
    std::vector<int> todo{0};
    while (!todo.empty()) {
      const int x = todo.back();
      todo.pop_back();
      order.push_back(x);
      for (int k = 0; k < 2; ++k) {
        const Kid c = kid(x, k);
        if (c.code >= 0) {
          A[c.code] = area(c);
          todo.push_back(c.code);
        }
      }
    }
    {
      const Kid a = kid(0, 0), b = kid(0, 1);
      Kid u = a;
      for (int k = 0; k < 3; ++k) {
        u.lo[k] = std::min(a.lo[k], b.lo[k]);
        u.hi[k] = std::max(a.hi[k], b.hi[k]);
      }
      A[0] = area(u);
    }
    auto slot_cost = [&](const Kid& c, int i) -> double {  // S(c, i)
      if (c.code >= 0) return S[c.code][i];
      const double count = (double)((uint32_t)c.code & 15u);
      return (double)area(c) * count;
    };
    auto dist = [&](int x, int j, int& best_k) -> double {  // D(x, j)
      const Kid l = kid(x, 0), r = kid(x, 1);
      double best = inf;
      best_k = 1;
      for (int k = 1; k < j; ++k) {
        const double c = slot_cost(l, k) + slot_cost(r, j - k);
        if (c < best) {
          best = c;
          best_k = k;
        }
      }
      return best;
    };
    for (auto it = order.rbegin(); it != order.rend(); ++it) {
      const int x = *it;
      int k4 = 1;
      const double w = (double)params.wide_cost * A[x] + dist(x, kWide, k4);
      wsplit[x] = (uint8_t)k4;
      S[x][1] = w;
      choice[x][1] = 0;
      for (int i = 2; i <= kWide; ++i) {
        int k = 1;
        const double d = dist(x, i, k);
        if (d < w) {
          S[x][i] = d;
          choice[x][i] = (uint8_t)k;
        } else {
          S[x][i] = w;
          choice[x][i] = 0;
        }
      }
    }
  }
  // the children (BVH2 nodes or leaves) of the wide node rooted at BVH2 node n2
  auto children = [&](int n2, Kid* kids) -> int {
    int nk = 0;
    if (params.collapse == 1) {
      std::function<void(const Kid&, int)> place = [&](const Kid& c, int slots) {
        if (c.code < 0 || choice[c.code][slots] == 0) {
          kids[nk++] = c;
          return;
        }
        const int k = choice[c.code][slots];
        place(kid(c.code, 0), k);
        place(kid(c.code, 1), slots - k);
      };
      const int k = wsplit[n2];
      place(kid(n2, 0), k);
      place(kid(n2, 1), kWide - k);
      return nk;
    }
    kids[nk++] = kid(n2, 0);
    kids[nk++] = kid(n2, 1);
    while (nk < kWide) {  // open the internal child of largest surface area
      int best = -1;
      float ba = -1.0f;
      for (int j = 0; j < nk; ++j)
        if (kids[j].code >= 0 && area(kids[j]) > ba) { ba = area(kids[j]); best = j; }
      if (best < 0) break;
      const int inner = kids[best].code;
      kids[best] = kid(inner, 0);
      kids[nk++] = kid(inner, 1);
    }
    return nk;
  };
  bool ok = true;
  std::function<int(int, int)> build = [&](int n2, int depth) -> int {
    depth4 = std::max(depth4, depth);
    if (depth >= kMaxDepth4) ok = false;
    Kid kids[kWide];
    const int nk = children(n2, kids);
    const int me = (int)(out4.size() / kWideStride);
    out4.resize(out4.size() + kWideStride, make_float4(0.0f, 0.0f, 0.0f, 0.0f));
    int codes[kWide];
    for (int j = 0; j < kWide; ++j) {
      if (j >= nk) codes[j] = (int)0x80000000u;  // empty slot: a leaf of no triangles behind a far box
      else if (kids[j].code >= 0) codes[j] = ok ? build(kids[j].code, depth + 1) : 0;
      else codes[j] = kids[j].code;
    }
    float4* nd = out4.data() + kWideStride * (size_t)me;
    auto comp = [&](int j, int axis, bool lo) { return j < nk ? (lo ? kids[j].lo[axis] : kids[j].hi[axis]) : 1e30f; };
    for (int axis = 0; axis < 3; ++axis)
      for (int r = 0; r < kWideRow; ++r) {
        nd[(2 * axis) * kWideRow + r] = make_float4(comp(4 * r, axis, true), comp(4 * r + 1, axis, true), comp(4 * r + 2, axis, true),
                                                    comp(4 * r + 3, axis, true));
        nd[(2 * axis + 1) * kWideRow + r] = make_float4(comp(4 * r, axis, false), comp(4 * r + 1, axis, false),
                                                        comp(4 * r + 2, axis, false), comp(4 * r + 3, axis, false));
      }
    for (int r = 0; r < kWideRow; ++r) {
      int4 c4 = make_int4(codes[4 * r], codes[4 * r + 1], codes[4 * r + 2], codes[4 * r + 3]);
      memcpy(&nd[6 * kWideRow + r], &c4, sizeof(c4));
    }
    if (kWideStride > 7 * kWideRow) nd[7 * kWideRow] = make_float4((float)nk, 0.0f, 0.0f, 0.0f);
    return me;
  };
  build(0, 1);
  if (!ok) out4.clear();
  return ok;
}

}  // namespace pt
