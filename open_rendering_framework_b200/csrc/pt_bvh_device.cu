// BVH construction on the device: a linear BVH over Morton codes (T. Karras, "Maximizing Parallelism
// in the Construction of BVHs, Octrees, and k-d Trees", HPG 2012) with SAH-chosen leaves, written in
// the child-pair BVH2 layout of pt_scene.cuh, then collapsed level by level into the 4-wide layout.
//
// The reference builds its acceleration structure on the device through OptiX (Trbvh / Sbvh,
// OptixSceneLoader.cpp:136, ObjLoader.cpp:387-399).  Hits are decided by the triangle test alone
// (closest t, ties to the lower triangle index), so this tree gives the same hits as the host SAH
// tree and as a brute-force loop; it trades a little traversal speed for a build that takes
// milliseconds instead of a host pass over the triangles.
//
// Passes (all on the context's stream):
//   1. triangle boxes and the centroids' bounds (ordered-integer atomics);
//   2. 30-bit Morton codes of the centroids in those bounds;
//   3. a stable least-significant-digit radix sort of (code, triangle) in four 8-bit passes: per-block
//      digit counts stored digit-major, a scan of each digit's row by its own block (the rows' totals
//      scanned again by every scatter block), a scatter ranked within each warp by __match_any_sync;
//   4. the Karras hierarchy: internal node i covers a contiguous range of the sorted triangles and
//      splits it at the highest differing bit (equal codes are ordered by index);
//   5. bottom-up boxes and SAH costs (the second of a node's two children to finish computes it); a node
//      of at most `max_leaf` triangles whose leaf cost (one per triangle) does not exceed its split cost
//      (trav_cost + the children's costs weighted by their areas) becomes a leaf;
//   5b. rounds of treelet restructuring (option bvh_treelets), then pass 5 again over the new topology;
//   5c. each leaf's position in the tree's left-to-right order and each node's range of positions;
//   6. the BVH2 nodes, the triangles in leaf order, and the tree depth (every leaf walks to the root);
//   7. the 4-wide collapse: one launch per level, each wide node taking the children the SAH-optimal
//      dynamic program chose (bvh_collapse = 1, the host builder's rule; a bottom-up pass computes it)
//      or opening its BVH2 node's internal child of largest area until it has four (bvh_collapse = 0),
//      its internal children appended to the next level's work list.
// The wide tree's depth is bounded by the traversal stack; a deeper tree leaves the 4-wide BVH unset.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "pt_common.cuh"
#include "pt_context.h"

namespace pt {
namespace {

constexpr int kBlock = 256;
constexpr int kRadix = 256;
constexpr int kWarpsPerBlock = kBlock / 32;
constexpr uint32_t kEmptyLeaf = 0x80000000u;

__device__ __forceinline__ uint32_t f2ord(float f)
{
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u); }

__device__ __forceinline__ float area_of(const float4& lo, const float4& hi)
{
  const float dx = fmaxf(0.0f, hi.x - lo.x), dy = fmaxf(0.0f, hi.y - lo.y), dz = fmaxf(0.0f, hi.z - lo.z);
  return dx * dy + dy * dz + dz * dx;
}

// Pass 1: per triangle its box (sorted later), and the bounds of the centroids (box midpoints, as
// the host builder takes them).
__global__ void __launch_bounds__(kBlock) k_tri_boxes(const float* __restrict__ tri, uint32_t n, float4* __restrict__ box_lo,
                                                      float4* __restrict__ box_hi, uint32_t* __restrict__ cbounds)
{
  float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float* p = tri + 9 * (size_t)i;
    float bl[3], bh[3], c[3];
    for (int k = 0; k < 3; ++k) {
      bl[k] = fminf(fminf(p[k], p[3 + k]), p[6 + k]);
      bh[k] = fmaxf(fmaxf(p[k], p[3 + k]), p[6 + k]);
      c[k] = 0.5f * (bl[k] + bh[k]);
      lo[k] = fminf(lo[k], c[k]);
      hi[k] = fmaxf(hi[k], c[k]);
    }
    box_lo[i] = make_float4(bl[0], bl[1], bl[2], 0.0f);
    box_hi[i] = make_float4(bh[0], bh[1], bh[2], 0.0f);
  }
  // warp, then block reduction: one atomic per bound and block
  __shared__ uint32_t red[6];
  if (threadIdx.x < 6) red[threadIdx.x] = threadIdx.x < 3 ? 0xffffffffu : 0u;
  __syncthreads();
  for (int k = 0; k < 3; ++k) {
    for (int off = 16; off > 0; off >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int k = 0; k < 3; ++k) {
      atomicMin(red + k, f2ord(lo[k]));
      atomicMax(red + 3 + k, f2ord(hi[k]));
    }
  }
  __syncthreads();
  if (threadIdx.x < 3) atomicMin(cbounds + threadIdx.x, red[threadIdx.x]);
  else if (threadIdx.x < 6) atomicMax(cbounds + threadIdx.x, red[threadIdx.x]);
}

// 10 bits of x spread to every third bit.
__device__ __forceinline__ uint32_t spread10(uint32_t x)
{
  x &= 0x3ffu;
  x = (x | (x << 16)) & 0x030000ffu;
  x = (x | (x << 8)) & 0x0300f00fu;
  x = (x | (x << 4)) & 0x030c30c3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

// Pass 2: Morton code of each centroid in the centroid bounds; idx = the triangle.
__global__ void __launch_bounds__(kBlock) k_morton(const float4* __restrict__ box_lo, const float4* __restrict__ box_hi, uint32_t n,
                                                   const uint32_t* __restrict__ cbounds, uint32_t* __restrict__ keys, uint32_t* __restrict__ idx)
{
  float lo[3], inv[3];
  for (int k = 0; k < 3; ++k) {
    lo[k] = ord2f(cbounds[k]);
    const float ext = ord2f(cbounds[3 + k]) - lo[k];
    inv[k] = ext > 0.0f ? 1024.0f / ext : 0.0f;
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4 a = box_lo[i], b = box_hi[i];
    const float c[3] = {0.5f * (a.x + b.x), 0.5f * (a.y + b.y), 0.5f * (a.z + b.z)};
    uint32_t q[3];
    for (int k = 0; k < 3; ++k) {
      const float t = (c[k] - lo[k]) * inv[k];
      q[k] = t <= 0.0f ? 0u : (t >= 1023.0f ? 1023u : (uint32_t)t);
    }
    keys[i] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    idx[i] = i;
  }
}

// Pass 3a: digit counts of one block of kBlock keys, stored digit-major: hist[digit * nblocks + block].
__global__ void __launch_bounds__(kBlock) k_radix_hist(const uint32_t* __restrict__ keys, uint32_t n, int shift, uint32_t* __restrict__ hist)
{
  __shared__ uint32_t cnt[kRadix];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & (kRadix - 1)], 1u);
  __syncthreads();
  hist[threadIdx.x * gridDim.x + blockIdx.x] = cnt[threadIdx.x];
}

// Exclusive scan of one value per thread over the block (kBlock threads): warp shuffles, then the
// warps' totals from shared memory; *total receives the block's sum.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_tot, uint32_t& total)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) warp_tot[warp] = x;
  __syncthreads();
  uint32_t before = 0, all = 0;
#pragma unroll
  for (int w = 0; w < kWarpsPerBlock; ++w) {
    const uint32_t t = warp_tot[w];
    before += w < warp ? t : 0u;
    all += t;
  }
  __syncthreads();  // warp_tot may be reused
  total = all;
  return before + x - v;
}

// Pass 3b: the digit-major counts scanned row by row: block d turns row d (the counts of digit d in
// blocks 0 .. nb - 1) into its exclusive prefix sums and stores the row's total in row_tot[d].  The
// scatter adds the exclusive scan of the 256 row totals (the digit's start in the output).
__global__ void __launch_bounds__(kBlock) k_radix_row_scan(uint32_t* __restrict__ hist, uint32_t nb, uint32_t* __restrict__ row_tot)
{
  __shared__ uint32_t wt[kWarpsPerBlock];
  uint32_t* row = hist + (size_t)blockIdx.x * nb;
  uint32_t carry = 0;
  for (uint32_t b = 0; b < nb; b += kBlock) {
    const uint32_t i = b + threadIdx.x;
    const uint32_t v = i < nb ? row[i] : 0u;
    uint32_t tot;
    const uint32_t ex = block_exclusive_scan(v, wt, tot);
    if (i < nb) row[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) row_tot[blockIdx.x] = carry;
}

// Pass 3c: stable scatter.  A key's destination is its digit's start (the exclusive scan of the row
// totals), plus the keys of that digit in earlier blocks (the row scan), in earlier warps of the block
// and in earlier lanes of its warp.
static_assert(kBlock == kRadix, "the scatter scans the kRadix row totals with one value per thread");
__global__ void __launch_bounds__(kBlock) k_radix_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t n,
                                                          int shift, const uint32_t* __restrict__ offs, const uint32_t* __restrict__ row_tot,
                                                          uint32_t* __restrict__ kout, uint32_t* __restrict__ vout)
{
  __shared__ uint32_t wcnt[kWarpsPerBlock][kRadix];
  __shared__ uint32_t base[kRadix];
  __shared__ uint32_t wt[kWarpsPerBlock];
  uint32_t all;
  base[threadIdx.x] = block_exclusive_scan(row_tot[threadIdx.x], wt, all);
  for (int j = threadIdx.x; j < kWarpsPerBlock * kRadix; j += kBlock) (&wcnt[0][0])[j] = 0;
  __syncthreads();
  const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
  const bool valid = i < n;
  const uint32_t key = valid ? kin[i] : 0u;
  const uint32_t digit = valid ? (key >> shift) & (kRadix - 1) : (uint32_t)kRadix;  // kRadix matches no real digit
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t peers = __match_any_sync(0xffffffffu, digit);
  const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
  if (valid && rank == 0) wcnt[warp][digit] = __popc(peers);
  __syncthreads();
  if (!valid) return;
  uint32_t pos = base[digit] + offs[digit * gridDim.x + blockIdx.x] + rank;
  for (int w = 0; w < warp; ++w) pos += wcnt[w][digit];
  kout[pos] = key;
  vout[pos] = vin[i];
}

// Karras' delta: length of the common prefix of keys i and j, extended by the indices for equal keys;
// -1 outside [0, n).
__device__ __forceinline__ int kdelta(const uint32_t* __restrict__ keys, int n, int i, int j)
{
  if (j < 0 || j >= n) return -1;
  const uint32_t a = keys[i], b = keys[j];
  return a == b ? 32 + __clz((uint32_t)(i ^ j)) : __clz(a ^ b);
}

// Pass 4: internal node i of n - 1.  Children >= 0 are internal nodes, < 0 are leaves ~j (sorted
// position j).  first / last: the sorted range the node covers.
__global__ void __launch_bounds__(kBlock) k_karras(const uint32_t* __restrict__ keys, int n, int2* __restrict__ child,
                                                   int* __restrict__ iparent, int* __restrict__ lparent, int2* __restrict__ range)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  const int dmin = kdelta(keys, n, i, i - d);
  int lmax = 2;
  while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  const int j = i + l * d;
  const int dnode = kdelta(keys, n, i, j);
  int s = 0, t = l;
  do {
    t = (t + 1) >> 1;
    if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
  } while (t > 1);
  const int gamma = i + s * d + min(d, 0);
  const int first = min(i, j), last = max(i, j);
  const int left = first == gamma ? ~gamma : gamma;
  const int right = last == gamma + 1 ? ~(gamma + 1) : gamma + 1;
  child[i] = make_int2(left, right);
  range[i] = make_int2(first, last);
  if (left >= 0) iparent[left] = i; else lparent[~left] = i;
  if (right >= 0) iparent[right] = i; else lparent[~right] = i;
  if (i == 0) iparent[0] = -1;
}

struct NodeRec {
  float4 lo, hi;  // box; lo.w = SAH cost, hi.w = triangle count (as float)
};

// Every walk from a leaf to the root is bounded: a walk longer than kMaxWalk levels means a broken tree
// (the BVH2 may not reach depth 64 anyway); the kernel then raises *err and stops, and the host
// discards the build.
constexpr int kMaxWalk = 256;

// Pass 5: bottom-up boxes and SAH costs.  One thread per leaf walks up; at each internal node the
// first arriving child stops, the second computes the node (its sibling's record is then complete:
// every record is written before the __threadfence that precedes the arrival counter).
__global__ void __launch_bounds__(kBlock) k_bottom_up(int n, const uint32_t* __restrict__ order, const float4* __restrict__ box_lo,
                                                      const float4* __restrict__ box_hi, const int2* __restrict__ child,
                                                      const int* __restrict__ iparent, const int* __restrict__ lparent,
                                                      NodeRec* leafrec, NodeRec* noderec, uint32_t* visits, uint8_t* collapse,
                                                      float trav_cost, int max_leaf, int* err)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t tri = order[j];
  NodeRec r;
  r.lo = box_lo[tri];
  r.hi = box_hi[tri];
  r.lo.w = 1.0f;
  r.hi.w = 1.0f;
  leafrec[j] = r;
  __threadfence();
  int p = lparent[j], steps = 0;
  while (p >= 0) {
    if (p >= n - 1 || ++steps > kMaxWalk) {
      atomicExch(err, 1);
      return;
    }
    if (atomicAdd(visits + p, 1u) == 0u) return;
    __threadfence();
    const int2 c = child[p];
    NodeRec a, b;
    const NodeRec* pa = c.x >= 0 ? noderec + c.x : leafrec + ~c.x;
    const NodeRec* pb = c.y >= 0 ? noderec + c.y : leafrec + ~c.y;
    a.lo = __ldcg(&pa->lo);
    a.hi = __ldcg(&pa->hi);
    b.lo = __ldcg(&pb->lo);
    b.hi = __ldcg(&pb->hi);
    NodeRec m;
    m.lo = make_float4(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z), 0.0f);
    m.hi = make_float4(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z), 0.0f);
    const float count = a.hi.w + b.hi.w;
    const float A = area_of(m.lo, m.hi);
    const float wa = A > 0.0f ? area_of(a.lo, a.hi) / A : 0.5f, wb = A > 0.0f ? area_of(b.lo, b.hi) / A : 0.5f;
    const float split_cost = trav_cost + wa * a.lo.w + wb * b.lo.w;
    const bool leaf = count <= (float)max_leaf && count <= split_cost;
    m.lo.w = leaf ? count : split_cost;
    m.hi.w = count;
    collapse[p] = leaf ? 1 : 0;
    __stcg(&noderec[p].lo, m.lo);
    __stcg(&noderec[p].hi, m.hi);
    __threadfence();
    p = iparent[p];
  }
}

// Pass 5b (option bvh_treelets, rounds of it): treelet restructuring (T. Karras, T. Aila, "Fast
// Parallel Construction of High-Quality Bounding Volume Hierarchies", HPG 2013; the "Trbvh" builder the
// reference requests from OptiX, OptixSceneLoader.cpp:136).  Bottom-up as pass 5: at each internal node
// of at least `treelet_min` triangles (option bvh_treelet_min) whose subtrees are complete, the node and its descendants form a
// treelet of up to 7 leaves (the treelet leaf of largest area is opened while there are fewer than 7),
// and a dynamic program over the 127 subsets of those leaves finds the topology of least SAH cost
//   c(S) = min( trav_cost * A(S) + min over splits P of S of c(P) + c(S \ P),  A(S) * N(S) if N(S) <= max_leaf )
// (a treelet leaf's c is A x its subtree's cost per area, noderec lo.w).  The warp that finds such nodes
// processes them one after the other, all lanes sharing each dynamic program; the treelet's internal
// nodes are reused for the new topology, and their boxes, counts and costs rewritten.  Only the nodes
// below the treelet's root change, and nothing else touches them once both of the root's subtrees are
// complete, so each treelet depends on its own subtree only: the result does not depend on the order
// in which warps arrive.
constexpr int kTreeletLeaves = 7;
constexpr int kTreeletSets = 1 << kTreeletLeaves;

struct TreeletShared {
  float area[kTreeletSets];
  float cost[kTreeletSets];
  uint8_t part[kTreeletSets];
  NodeRec leaf_rec[kTreeletLeaves];
  float leaf_area[kTreeletLeaves];
  int leaves[kTreeletLeaves], inner[kTreeletLeaves - 1], node_set[kTreeletLeaves - 1];
  int nl, used;
};

__device__ __forceinline__ NodeRec load_rec(const NodeRec* r)
{
  NodeRec a;
  a.lo = __ldcg(&r->lo);
  a.hi = __ldcg(&r->hi);
  return a;
}

// The bits of i deposited, lowest first, into the set bits of mask.
__device__ __forceinline__ int deposit_bits(int i, int mask)
{
  int r = 0;
  for (int b = 0; mask; ++b) {
    const int low = mask & -mask;
    r |= ((i >> b) & 1) ? low : 0;
    mask ^= low;
  }
  return r;
}

// The 127 nonempty subsets of seven leaves ordered by size (then value); subsets of k leaves sit at
// [set_start(k), set_start(k + 1)).  A treelet of fewer leaves uses the entries that fit in it.
__constant__ uint8_t kSetsBySize[kTreeletSets - 1] = {
    1, 2, 4, 8, 16, 32, 64, 3, 5, 6, 9, 10, 12, 17, 18, 20,
    24, 33, 34, 36, 40, 48, 65, 66, 68, 72, 80, 96, 7, 11, 13, 14,
    19, 21, 22, 25, 26, 28, 35, 37, 38, 41, 42, 44, 49, 50, 52, 56,
    67, 69, 70, 73, 74, 76, 81, 82, 84, 88, 97, 98, 100, 104, 112, 15,
    23, 27, 29, 30, 39, 43, 45, 46, 51, 53, 54, 57, 58, 60, 71, 75,
    77, 78, 83, 85, 86, 89, 90, 92, 99, 101, 102, 105, 106, 108, 113, 114,
    116, 120, 31, 47, 55, 59, 61, 62, 79, 87, 91, 93, 94, 103, 107, 109,
    110, 115, 117, 118, 121, 122, 124, 63, 95, 111, 119, 123, 125, 126, 127};
__host__ __device__ constexpr int set_start(int k)
{
  return k <= 1 ? 0 : k == 2 ? 7 : k == 3 ? 28 : k == 4 ? 63 : k == 5 ? 98 : k == 6 ? 119 : k == 7 ? 126 : 127;
}
static_assert(kTreeletLeaves == 7, "the subset table is written for seven leaves");

// The cost and the chosen split of subset `set` from its best split cost.
__device__ __forceinline__ void treelet_finish(TreeletShared& sh, int set, float best, int bp, float trav_cost, int max_leaf)
{
  float n_tris = 0.0f;
  for (int k = 0; k < sh.nl; ++k) n_tris += ((set >> k) & 1) ? sh.leaf_rec[k].hi.w : 0.0f;
  const float split = trav_cost * sh.area[set] + best;
  const float leaf = n_tris <= (float)max_leaf ? sh.area[set] * n_tris : INFINITY;
  sh.cost[set] = fminf(split, leaf);
  sh.part[set] = (uint8_t)bp;
}

// One treelet at `root`, processed by the whole warp (root uniform across the warp).  Each split of a
// subset is counted once, by the part that holds the subset's lowest leaf.  Subsets of up to five leaves
// take one lane each; those of six and seven (31 and 63 splits) are shared by the warp and reduced to
// the least cost (ties to the smaller part).
__device__ void treelet_optimize(int root, int2* child, int* iparent, int* lparent, const NodeRec* leafrec, NodeRec* noderec,
                                 TreeletShared& sh, float trav_cost, int max_leaf)
{
  const int lane = threadIdx.x & 31;
  if (lane == 0) {  // form the treelet: open the treelet leaf of largest area while there are fewer than 7
    int nl = 0, ni = 0;
    auto put = [&](int k, int code) {
      const NodeRec r = load_rec(code >= 0 ? noderec + code : leafrec + ~code);
      sh.leaves[k] = code;
      sh.leaf_rec[k] = r;
      sh.leaf_area[k] = code >= 0 ? area_of(r.lo, r.hi) : -1.0f;  // -1: a triangle, never opened
    };
    sh.inner[ni++] = root;
    const int2 c = __ldcg(&child[root]);
    put(nl++, c.x);
    put(nl++, c.y);
    while (nl < kTreeletLeaves) {
      int best = -1;
      float ba = -1.0f;
      for (int k = 0; k < nl; ++k)
        if (sh.leaf_area[k] > ba) { ba = sh.leaf_area[k]; best = k; }
      if (best < 0) break;
      const int x = sh.leaves[best];
      sh.inner[ni++] = x;
      const int2 g = __ldcg(&child[x]);
      put(best, g.x);
      put(nl++, g.y);
    }
    sh.nl = nl;
  }
  __syncwarp();
  const int nl = sh.nl;
  const int full = (1 << nl) - 1;
  // subset areas and the treelet leaves' own costs
  for (int set = lane + 1; set <= full; set += 32) {
    float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int k = 0; k < nl; ++k) {
      if (!((set >> k) & 1)) continue;
      const NodeRec& r = sh.leaf_rec[k];
      lo[0] = fminf(lo[0], r.lo.x); lo[1] = fminf(lo[1], r.lo.y); lo[2] = fminf(lo[2], r.lo.z);
      hi[0] = fmaxf(hi[0], r.hi.x); hi[1] = fmaxf(hi[1], r.hi.y); hi[2] = fmaxf(hi[2], r.hi.z);
    }
    const float dx = fmaxf(0.0f, hi[0] - lo[0]), dy = fmaxf(0.0f, hi[1] - lo[1]), dz = fmaxf(0.0f, hi[2] - lo[2]);
    sh.area[set] = dx * dy + dy * dz + dz * dx;
    if (__popc(set) == 1) {
      sh.cost[set] = sh.area[set] * sh.leaf_rec[__ffs(set) - 1].lo.w;
      sh.part[set] = 0;
    }
  }
  __syncwarp();
  // subsets by increasing size (every split of a subset is into smaller ones): up to five leaves one
  // subset per lane, six and seven leaves (8 subsets, 31 or 63 splits) shared by the warp
  for (int size = 2; size <= nl && size <= 5; ++size) {
    for (int e = set_start(size) + lane; e < set_start(size + 1); e += 32) {
      const int set = kSetsBySize[e];
      if (set > full) continue;
      const int low = set & -set, rest = set ^ low;
      float best = INFINITY;
      int bp = low;
      for (int sub = (rest - 1) & rest;; sub = (sub - 1) & rest) {  // the proper subsets of rest
        const int part = low | sub;
        const float c = sh.cost[part] + sh.cost[set ^ part];
        if (c < best) { best = c; bp = part; }
        if (sub == 0) break;
      }
      treelet_finish(sh, set, best, bp, trav_cost, max_leaf);
    }
    __syncwarp();
  }
  for (int size = 6; size <= nl; ++size) {
    for (int e = set_start(size); e < set_start(size + 1); ++e) {
      const int set = kSetsBySize[e];
      if (set > full) continue;
      const int low = set & -set, rest = set ^ low;
      const int n_split = (1 << (size - 1)) - 1;
      float best = INFINITY;
      int bp = low;
      for (int i = lane; i < n_split; i += 32) {
        const int part = low | deposit_bits(i, rest);
        const float c = sh.cost[part] + sh.cost[set ^ part];
        if (c < best || (c == best && part < bp)) { best = c; bp = part; }
      }
      for (int off = 16; off > 0; off >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, off);
        const int op = __shfl_xor_sync(0xffffffffu, bp, off);
        if (ob < best || (ob == best && op < bp)) { best = ob; bp = op; }
      }
      if (lane == 0) treelet_finish(sh, set, best, bp, trav_cost, max_leaf);
    }
    __syncwarp();
  }
  // rebuild the treelet on its internal nodes: the pre-order assignment (lane 0), then each rewired
  // node's record from the treelet leaves it covers (one lane per node)
  if (lane == 0) {
    int* node_set = sh.node_set;
    int used = 1;
    node_set[0] = full;
    for (int q = 0; q < used; ++q) {
      const int set = node_set[q];
      const int a = sh.part[set], b = set ^ a;
      int code[2];
      const int sides[2] = {a, b};
      for (int h = 0; h < 2; ++h) {
        if (__popc(sides[h]) == 1) {
          code[h] = sh.leaves[__ffs(sides[h]) - 1];
        } else {
          node_set[used] = sides[h];
          code[h] = sh.inner[used++];
        }
        if (code[h] >= 0) iparent[code[h]] = sh.inner[q];
        else lparent[~code[h]] = sh.inner[q];
      }
      __stcg(&child[sh.inner[q]], make_int2(code[0], code[1]));
    }
    sh.used = used;
  }
  __syncwarp();
  {
    const int q = lane;
    if (q < sh.used) {
      const int set = sh.node_set[q];
      NodeRec m;
      m.lo = make_float4(INFINITY, INFINITY, INFINITY, 0.0f);
      m.hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.0f);
      float cost_sum = 0.0f;
      for (int k = 0; k < nl; ++k) {
        if (!((set >> k) & 1)) continue;
        const NodeRec& r = sh.leaf_rec[k];
        m.lo.x = fminf(m.lo.x, r.lo.x); m.lo.y = fminf(m.lo.y, r.lo.y); m.lo.z = fminf(m.lo.z, r.lo.z);
        m.hi.x = fmaxf(m.hi.x, r.hi.x); m.hi.y = fmaxf(m.hi.y, r.hi.y); m.hi.z = fmaxf(m.hi.z, r.hi.z);
        m.hi.w += r.hi.w;
        cost_sum += r.lo.w;
      }
      const float A = area_of(m.lo, m.hi);
      m.lo.w = A > 0.0f ? sh.cost[set] / A : cost_sum;  // cost per area, as pass 5 keeps it
      __stcg(&noderec[sh.inner[q]].lo, m.lo);
      __stcg(&noderec[sh.inner[q]].hi, m.hi);
    }
  }
  __syncwarp();
}

__global__ void __launch_bounds__(kBlock) k_treelets(int n, int2* child, int* iparent, int* lparent, const NodeRec* leafrec, NodeRec* noderec,
                                                     uint32_t* visits, float trav_cost, int max_leaf, int treelet_min, int* err)
{
  __shared__ TreeletShared sh[kWarpsPerBlock];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = j < n;
  int p = active ? lparent[j] : -1, steps = 0;
  for (;;) {
    bool ready = false;
    if (active) {
      if (p < 0 || p >= n - 1 || ++steps > kMaxWalk) {
        if (p >= n - 1 || steps > kMaxWalk) atomicExch(err, 1);
        active = false;
      } else if (atomicAdd(visits + p, 1u) == 0u) {
        active = false;
      } else {
        ready = true;
      }
    }
    __threadfence();
    unsigned m = __ballot_sync(0xffffffffu, ready);
    if (!__any_sync(0xffffffffu, active) && m == 0) break;
    while (m) {
      const int src = __ffs(m) - 1;
      m &= m - 1;
      const int node = __shfl_sync(0xffffffffu, p, src);
      if (__ldcg(&noderec[node].hi.w) >= (float)treelet_min)
        treelet_optimize(node, child, iparent, lparent, leafrec, noderec, sh[threadIdx.x >> 5], trav_cost, max_leaf);
    }
    __threadfence();
    if (ready) p = __ldcg(&iparent[p]);
  }
}

// Pass 5c: each leaf's position in the tree's left-to-right leaf order (the triangles are written in that
// order, so every subtree covers a contiguous range): the triangle counts of the left siblings on the
// way up; and for each internal node the range of its subtree, set by its leftmost leaf.
__global__ void __launch_bounds__(kBlock) k_leaf_positions(int n, const int2* __restrict__ child, const int* __restrict__ iparent,
                                                           const int* __restrict__ lparent, const NodeRec* __restrict__ noderec,
                                                           uint32_t* __restrict__ pos_of, int2* __restrict__ range, int* __restrict__ err)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  uint32_t pos = 0;
  int c = ~j, steps = 0;
  for (int q = lparent[j]; q >= 0; q = iparent[q]) {
    if (q >= n - 1 || ++steps > kMaxWalk) {
      atomicExch(err, 1);
      pos_of[j] = 0;
      return;
    }
    const int2 k = child[q];
    if (k.y == c) pos += k.x >= 0 ? (uint32_t)noderec[k.x].hi.w : 1u;
    c = q;
  }
  if (pos >= (uint32_t)n) {
    atomicExch(err, 1);
    pos = 0;
  }
  pos_of[j] = pos;
  c = ~j;
  steps = 0;
  for (int q = lparent[j]; q >= 0 && q < n - 1 && child[q].x == c && ++steps <= kMaxWalk; q = iparent[q]) {
    const int last = (int)pos + (int)noderec[q].hi.w - 1;
    if (last >= n) atomicExch(err, 1);
    range[q] = make_int2((int)pos, last < n ? last : n - 1);
    c = q;
  }
}

// The code of child c (>= 0 internal, < 0 leaf ~j) as the BVH2 stores it, and its record.
__device__ __forceinline__ int child_code(int c, const int2* range, const uint8_t* collapse, const uint32_t* pos_of)
{
  if (c < 0) return (int)(kEmptyLeaf | (pos_of[~c] << 4) | 1u);
  if (collapse[c]) {
    const int2 r = range[c];
    return (int)(kEmptyLeaf | ((uint32_t)r.x << 4) | (uint32_t)(r.y - r.x + 1));
  }
  return c;
}

// Pass 6a: the BVH2 nodes (internal node p at index p; nodes inside a leaf subtree are written too
// and never reached).  The root of a tree that is a single leaf holds that leaf and an empty one.
__global__ void __launch_bounds__(kBlock) k_write_bvh2(int n, const int2* __restrict__ child, const int* __restrict__ iparent,
                                                       const int2* __restrict__ range, const uint8_t* __restrict__ collapse,
                                                       const uint32_t* __restrict__ pos_of, const NodeRec* __restrict__ leafrec,
                                                       const NodeRec* __restrict__ noderec, float4* __restrict__ nodes)
{
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n - 1) return;
  int c0, c1;
  NodeRec r0, r1;
  if (p == 0 && collapse[0]) {
    c0 = (int)(kEmptyLeaf | (uint32_t)n);  // first 0, count n (<= 15)
    c1 = (int)kEmptyLeaf;
    r0 = noderec[0];
    r1.lo = make_float4(1e30f, 1e30f, 1e30f, 0.0f);
    r1.hi = r1.lo;
  } else {
    const int2 c = child[p];
    c0 = child_code(c.x, range, collapse, pos_of);
    c1 = child_code(c.y, range, collapse, pos_of);
    r0 = c.x >= 0 ? noderec[c.x] : leafrec[~c.x];
    r1 = c.y >= 0 ? noderec[c.y] : leafrec[~c.y];
  }
  float4* nd = nodes + 4 * (size_t)p;
  nd[0] = make_float4(r0.lo.x, r0.hi.x, r0.lo.y, r0.hi.y);
  nd[1] = make_float4(r1.lo.x, r1.hi.x, r1.lo.y, r1.hi.y);
  nd[2] = make_float4(r0.lo.z, r0.hi.z, r1.lo.z, r1.hi.z);
  nd[3] = make_float4(__int_as_float(c0), __int_as_float(c1), __int_as_float(iparent[p]), 0.0f);
}

// Pass 6b: triangles in leaf order (pass 5c) as Moller-Trumbore records, and the BVH2 depth (levels
// including the leaves): each triangle counts the internal nodes above it that the tree keeps (those
// inside a leaf's subtree are not nodes of the tree), plus its leaf.
__global__ void __launch_bounds__(kBlock) k_write_tris(int n, const float* __restrict__ tri, const uint32_t* __restrict__ order,
                                                       const uint32_t* __restrict__ pos_of, const int* __restrict__ lparent,
                                                       const int* __restrict__ iparent, const uint8_t* __restrict__ collapse,
                                                       float4* __restrict__ v0, float4* __restrict__ e1, float4* __restrict__ e2,
                                                       int* __restrict__ max_depth)  // max_depth[0] depth, [1] error
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint32_t i = order[j], at = pos_of[j];
  if (at >= (uint32_t)n) return;  // k_leaf_positions raised the error
  const float* p = tri + 9 * (size_t)i;
  v0[at] = make_float4(p[0], p[1], p[2], __int_as_float((int)i));
  e1[at] = make_float4(p[3] - p[0], p[4] - p[1], p[5] - p[2], 0.0f);
  e2[at] = make_float4(p[6] - p[0], p[7] - p[1], p[8] - p[2], 0.0f);
  int d = 1, steps = 0;
  for (int q = lparent[j]; q >= 0; q = iparent[q]) {
    if (q >= n - 1 || ++steps > kMaxWalk) {
      atomicExch(max_depth + 1, 1);  // the error word after the depth
      return;
    }
    d += collapse[q] ? 0 : 1;
  }
  if (collapse[0]) d = 2;  // a single-leaf tree: the root and its leaf
  atomicMax(max_depth, d);
}

struct Kid {
  int code;
  float lo[3], hi[3];
};
__device__ __forceinline__ Kid kid_of(const float4* __restrict__ nodes, int node, int k)
{
  const float4* nd = nodes + 4 * (size_t)node;
  const float4 a = nd[k], z = nd[2], c = nd[3];
  Kid r;
  r.code = __float_as_int(k == 0 ? c.x : c.y);
  r.lo[0] = a.x; r.hi[0] = a.y; r.lo[1] = a.z; r.hi[1] = a.w;
  r.lo[2] = k == 0 ? z.x : z.z;
  r.hi[2] = k == 0 ? z.y : z.w;
  return r;
}
__device__ __forceinline__ float kid_area(const Kid& c)
{
  float d[3];
  for (int k = 0; k < 3; ++k) d[k] = fmaxf(0.0f, c.hi[k] - c.lo[k]);
  return d[0] * d[1] + d[1] * d[2] + d[2] * d[0];
}

// Pass 6c (bvh_collapse = 1): the SAH-optimal 4-wide collapse's dynamic program over the BVH2 as
// written (the host builder's rule, pt_bvh.cu): per internal node x, S(x, i) = the least SAH cost of x's
// subtree placed in at most i slots of its parent's wide node (i = 1: x becomes a wide node of its own,
// W(x) = wide_cost A(x) + D(x, 4); i >= 2: min(W(x), D(x, i)), D(x, i) = min over k of
// S(child 0, k) + S(child 1, i - k); a leaf costs A x its triangles in any number of slots).  Bottom-up
// with arrival counters like pass 5; nodes inside a leaf (collapsed) are passed through.  choice[x]:
// byte 0 the split k of W(x)'s four slots, bytes 1..3 the split k for i = 2..4 (0: x stays whole).
__device__ __forceinline__ float dp_slot_cost(const Kid& c, int i, const float4* __restrict__ dp_cost)
{
  if (c.code < 0) return kid_area(c) * (float)((uint32_t)c.code & 15u);
  const float4 s = __ldcg(dp_cost + c.code);
  return i == 1 ? s.x : (i == 2 ? s.y : (i == 3 ? s.z : s.w));
}
__global__ void __launch_bounds__(kBlock) k_collapse_dp(int n, const float4* __restrict__ nodes, const int* __restrict__ iparent,
                                                        const int* __restrict__ lparent, const uint8_t* __restrict__ collapse,
                                                        uint32_t* visits, float wide_cost, float4* dp_cost, uint32_t* dp_choice, int* err)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int p = lparent[j], steps = 0;
  while (p >= 0) {
    if (p >= n - 1 || ++steps > kMaxWalk) {
      atomicExch(err, 1);
      return;
    }
    if (atomicAdd(visits + p, 1u) == 0u) return;
    __threadfence();
    if (!collapse[p]) {
      const Kid a = kid_of(nodes, p, 0), b = kid_of(nodes, p, 1);
      float D[5];
      int K[5];
      for (int i = 2; i <= 4; ++i) {
        D[i] = INFINITY;
        K[i] = 1;
        for (int k = 1; k < i; ++k) {
          const float c = dp_slot_cost(a, k, dp_cost) + dp_slot_cost(b, i - k, dp_cost);
          if (c < D[i]) { D[i] = c; K[i] = k; }
        }
      }
      Kid u = a;
      for (int k = 0; k < 3; ++k) {
        u.lo[k] = fminf(a.lo[k], b.lo[k]);
        u.hi[k] = fmaxf(a.hi[k], b.hi[k]);
      }
      const float W = wide_cost * kid_area(u) + D[4];
      float S[5];
      uint32_t ch = (uint32_t)K[4];
      S[1] = W;
      for (int i = 2; i <= 4; ++i) {
        const bool open = D[i] < W;
        S[i] = open ? D[i] : W;
        ch |= (uint32_t)(open ? K[i] : 0) << (8 * (i - 1));
      }
      __stcg(dp_cost + p, make_float4(S[1], S[2], S[3], S[4]));
      __stcg(dp_choice + p, ch);
    }
    __threadfence();
    p = iparent[p];
  }
}

// Pass 7: one level of the 4-wide collapse.  Work item (BVH2 node, wide node index); each internal
// child gets the next wide index from *wide_count and becomes a work item of the next level.  The
// level's item count is read on the device (*n_in_ptr), so the levels launch back to back; the grid
// of level L covers min(4^L, n - 1) items, the most that level can hold, up to 8 blocks per SM (the
// threads stride over the rest).
__global__ void __launch_bounds__(128) k_collapse_level(const float4* __restrict__ nodes, const int2* __restrict__ work_in,
                                                        const uint32_t* __restrict__ n_in_ptr, int2* __restrict__ work_out,
                                                        uint32_t* __restrict__ n_out, uint32_t* __restrict__ wide_count, uint32_t wide_cap,
                                                        float4* __restrict__ nodes4, uint32_t* __restrict__ overflow,
                                                        const uint32_t* __restrict__ dp_choice)
{
  const uint32_t n_in = *n_in_ptr;
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < n_in; w += gridDim.x * blockDim.x) {
    const int2 item = work_in[w];
    Kid kids[kWide];
    int nk = 0;
    if (dp_choice) {
      // the children the dynamic program chose: each (BVH2 child, slots) is kept whole or split again
      struct Open {
        Kid c;
        int slots;
      } todo[kWide];
      int nt = 0;
      const int k0 = min(max((int)(dp_choice[item.x] & 0xffu), 1), kWide - 1);
      todo[nt++] = {kid_of(nodes, item.x, 1), kWide - k0};
      todo[nt++] = {kid_of(nodes, item.x, 0), k0};
      while (nt > 0 && nk < kWide) {
        const Open o = todo[--nt];
        const int k = o.c.code >= 0 && o.slots >= 2 ? (int)((dp_choice[o.c.code] >> (8 * (o.slots - 1))) & 0xffu) : 0;
        if (k <= 0 || k >= o.slots || nt + 2 > kWide) {
          kids[nk++] = o.c;
        } else {
          todo[nt++] = {kid_of(nodes, o.c.code, 1), o.slots - k};
          todo[nt++] = {kid_of(nodes, o.c.code, 0), k};
        }
      }
    } else {
      kids[nk++] = kid_of(nodes, item.x, 0);
      kids[nk++] = kid_of(nodes, item.x, 1);
      while (nk < kWide) {
        int best = -1;
        float ba = -1.0f;
        for (int j = 0; j < nk; ++j)
          if (kids[j].code >= 0 && kid_area(kids[j]) > ba) { ba = kid_area(kids[j]); best = j; }
        if (best < 0) break;
        const int inner = kids[best].code;
        kids[best] = kid_of(nodes, inner, 0);
        kids[nk++] = kid_of(nodes, inner, 1);
      }
    }
    int codes[kWide];
    for (int j = 0; j < kWide; ++j) {
      if (j >= nk) {
        codes[j] = (int)kEmptyLeaf;
      } else if (kids[j].code >= 0) {
        const uint32_t slot = atomicAdd(wide_count, 1u);
        if (slot >= wide_cap) {
          atomicAdd(overflow, 1u);
          codes[j] = (int)kEmptyLeaf;
        } else {
          codes[j] = (int)slot;
          work_out[atomicAdd(n_out, 1u)] = make_int2(kids[j].code, (int)slot);
        }
      } else {
        codes[j] = kids[j].code;
      }
    }
    float4* nd = nodes4 + kWideStride * (size_t)item.y;
    for (int axis = 0; axis < 3; ++axis)
      for (int r = 0; r < kWideRow; ++r) {
        float l[4], h[4];
        for (int q = 0; q < 4; ++q) {
          const int j = 4 * r + q;
          l[q] = j < nk ? kids[j].lo[axis] : 1e30f;
          h[q] = j < nk ? kids[j].hi[axis] : 1e30f;
        }
        nd[(2 * axis) * kWideRow + r] = make_float4(l[0], l[1], l[2], l[3]);
        nd[(2 * axis + 1) * kWideRow + r] = make_float4(h[0], h[1], h[2], h[3]);
      }
    for (int r = 0; r < kWideRow; ++r)
      nd[6 * kWideRow + r] = make_float4(__int_as_float(codes[4 * r]), __int_as_float(codes[4 * r + 1]), __int_as_float(codes[4 * r + 2]),
                                         __int_as_float(codes[4 * r + 3]));
    if (kWideStride > 7 * kWideRow) nd[7 * kWideRow] = make_float4((float)nk, 0.0f, 0.0f, 0.0f);
  }
}

// Offsets of the build's temporaries in one scratch allocation (256-byte aligned), kept by the context
// for later rebuilds.
struct BuildLayout {
  size_t tri, blo, bhi, keys_a, keys_b, idx_a, idx_b, hist, rowtot, posof, dpcost, dpchoice, cb, child, range, ipar, lpar, leafrec, noderec, visits, collapse, depth, work_a,
      work_b, counters, total;
  BuildLayout(uint32_t n, uint32_t nb)
  {
    size_t at = 0;
    auto take = [&](size_t bytes) {
      const size_t here = at;
      at += (bytes + 255) & ~(size_t)255;
      return here;
    };
    tri = take((size_t)n * 9 * sizeof(float));
    blo = take((size_t)n * sizeof(float4));
    bhi = take((size_t)n * sizeof(float4));
    keys_a = take((size_t)n * 4);
    keys_b = take((size_t)n * 4);
    idx_a = take((size_t)n * 4);
    idx_b = take((size_t)n * 4);
    hist = take((size_t)kRadix * nb * 4);
    rowtot = take((size_t)kRadix * 4);
    posof = take((size_t)n * 4);
    dpcost = take((size_t)(n - 1) * sizeof(float4));
    dpchoice = take((size_t)(n - 1) * 4);
    cb = take(6 * 4);
    child = take((size_t)(n - 1) * sizeof(int2));
    range = take((size_t)(n - 1) * sizeof(int2));
    ipar = take((size_t)(n - 1) * 4);
    lpar = take((size_t)n * 4);
    leafrec = take((size_t)n * sizeof(NodeRec));
    noderec = take((size_t)(n - 1) * sizeof(NodeRec));
    visits = take((size_t)(n - 1) * 4);
    collapse = take((size_t)(n - 1));
    depth = take(8);  // [0] BVH2 depth, [1] error raised by the treelet / position passes
    work_a = take((size_t)n * sizeof(int2));
    work_b = take((size_t)n * sizeof(int2));
    counters = take((size_t)(kMaxDepth4 + 4) * 4);
    total = at;
  }
};

}  // namespace

pt_status build_bvh_device(Context& c)
{
  const uint32_t n = c.n_tris;
  if (n < 2) return fail(PT_INVALID_ARG, "device BVH build: needs at least two triangles");
  if (n >= (1u << 27)) return fail(PT_CAP_EXCEEDED, "device BVH build: more than 2^27 triangles");
  cudaStream_t st = c.stream;
  const uint32_t nb = (n + kBlock - 1) / kBlock;
  const BuildLayout Lo(n, nb);
  pt_status s = c.d_build_scratch.reserve(Lo.total, "device BVH build scratch");
  if (s == PT_OK) s = c.d_nodes.reserve((size_t)(n - 1) * 4 * sizeof(float4), "BVH nodes");
  if (s == PT_OK) s = c.d_nodes4.reserve((size_t)(n - 1) * kWideStride * sizeof(float4), "4-wide BVH nodes");
  if (s == PT_OK) s = c.d_v0.reserve((size_t)n * sizeof(float4), "triangles");
  if (s == PT_OK) s = c.d_e1.reserve((size_t)n * sizeof(float4), "triangles");
  if (s == PT_OK) s = c.d_e2.reserve((size_t)n * sizeof(float4), "triangles");
  if (s != PT_OK) return s;
  char* base = c.d_build_scratch.as<char>();
  float* tri = (float*)(base + Lo.tri);
  float4 *blo = (float4*)(base + Lo.blo), *bhi = (float4*)(base + Lo.bhi);
  uint32_t *keys_a = (uint32_t*)(base + Lo.keys_a), *keys_b = (uint32_t*)(base + Lo.keys_b);
  uint32_t *idx_a = (uint32_t*)(base + Lo.idx_a), *idx_b = (uint32_t*)(base + Lo.idx_b);
  uint32_t *hist = (uint32_t*)(base + Lo.hist), *rowtot = (uint32_t*)(base + Lo.rowtot), *cb = (uint32_t*)(base + Lo.cb);
  uint32_t* pos_of = (uint32_t*)(base + Lo.posof);
  float4* dp_cost = (float4*)(base + Lo.dpcost);
  uint32_t* dp_choice = (uint32_t*)(base + Lo.dpchoice);
  int2 *child = (int2*)(base + Lo.child), *range = (int2*)(base + Lo.range);
  int *ipar = (int*)(base + Lo.ipar), *lpar = (int*)(base + Lo.lpar);
  NodeRec *leafrec = (NodeRec*)(base + Lo.leafrec), *noderec = (NodeRec*)(base + Lo.noderec);
  uint32_t* visits = (uint32_t*)(base + Lo.visits);
  uint8_t* collapse = (uint8_t*)(base + Lo.collapse);
  int* depth = (int*)(base + Lo.depth);
  int2 *work_a = (int2*)(base + Lo.work_a), *work_b = (int2*)(base + Lo.work_b);
  // counters: [0] wide nodes allocated, [1] overflow, [2 + L] items of collapse level L
  uint32_t* cnt = (uint32_t*)(base + Lo.counters);
  PT_CHECK_CUDA(cudaEventRecord(c.ev0, st), "device BVH build");
  PT_CHECK_CUDA(cudaMemcpyAsync(tri, c.tri_pos.data(), (size_t)n * 9 * sizeof(float), cudaMemcpyHostToDevice, st), "device BVH build H2D");
  const uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
  PT_CHECK_CUDA(cudaMemcpyAsync(cb, init, sizeof(init), cudaMemcpyHostToDevice, st), "device BVH build H2D");
  PT_CHECK_CUDA(cudaMemsetAsync(visits, 0, (size_t)(n - 1) * 4, st), "device BVH build");
  PT_CHECK_CUDA(cudaMemsetAsync(depth, 0, 8, st), "device BVH build");
  // the root: BVH2 node 0 becomes wide node 0, the one item of level 0
  std::vector<uint32_t> cinit(kMaxDepth4 + 4, 0u);
  cinit[0] = 1;
  cinit[2] = 1;
  PT_CHECK_CUDA(cudaMemcpyAsync(cnt, cinit.data(), cinit.size() * 4, cudaMemcpyHostToDevice, st), "device BVH build H2D");
  const int2 root = make_int2(0, 0);
  PT_CHECK_CUDA(cudaMemcpyAsync(work_a, &root, sizeof(root), cudaMemcpyHostToDevice, st), "device BVH build H2D");
  const int g = grid_for(n, kBlock, 8);
  k_tri_boxes<<<g, kBlock, 0, st>>>(tri, n, blo, bhi, cb);
  k_morton<<<g, kBlock, 0, st>>>(blo, bhi, n, cb, keys_a, idx_a);
  count_launch(2);
  uint32_t *kin = keys_a, *kout = keys_b, *vin = idx_a, *vout = idx_b;
  for (int shift = 0; shift < 32; shift += 8) {  // four passes: the sorted keys end in keys_a
    k_radix_hist<<<nb, kBlock, 0, st>>>(kin, n, shift, hist);
    k_radix_row_scan<<<kRadix, kBlock, 0, st>>>(hist, nb, rowtot);
    k_radix_scatter<<<nb, kBlock, 0, st>>>(kin, vin, n, shift, hist, rowtot, kout, vout);
    count_launch(3);
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  const int gi = (int)((n - 1 + kBlock - 1) / kBlock), gl = (int)nb;
  k_karras<<<gi, kBlock, 0, st>>>(kin, (int)n, child, ipar, lpar, range);
  k_bottom_up<<<gl, kBlock, 0, st>>>((int)n, vin, blo, bhi, child, ipar, lpar, leafrec, noderec, visits, collapse, c.bvh_params.trav_cost,
                                     c.bvh_params.max_leaf, depth + 1);
  count_launch(2);
  for (int r = 0; r < c.bvh_params.treelet_rounds; ++r) {
    PT_CHECK_CUDA(cudaMemsetAsync(visits, 0, (size_t)(n - 1) * 4, st), "device BVH build");
    k_treelets<<<gl, kBlock, 0, st>>>((int)n, child, ipar, lpar, leafrec, noderec, visits, c.bvh_params.trav_cost, c.bvh_params.max_leaf,
                                      c.bvh_params.treelet_min, depth + 1);
    count_launch();
  }
  if (c.bvh_params.treelet_rounds > 0) {  // the leaf collapse and costs over the final topology
    PT_CHECK_CUDA(cudaMemsetAsync(visits, 0, (size_t)(n - 1) * 4, st), "device BVH build");
    k_bottom_up<<<gl, kBlock, 0, st>>>((int)n, vin, blo, bhi, child, ipar, lpar, leafrec, noderec, visits, collapse, c.bvh_params.trav_cost,
                                       c.bvh_params.max_leaf, depth + 1);
    count_launch();
  }
  k_leaf_positions<<<gl, kBlock, 0, st>>>((int)n, child, ipar, lpar, noderec, pos_of, range, depth + 1);
  k_write_bvh2<<<gi, kBlock, 0, st>>>((int)n, child, ipar, range, collapse, pos_of, leafrec, noderec, c.d_nodes.as<float4>());
  k_write_tris<<<gl, kBlock, 0, st>>>((int)n, tri, vin, pos_of, lpar, ipar, collapse, c.d_v0.as<float4>(), c.d_e1.as<float4>(),
                                      c.d_e2.as<float4>(), depth);
  count_launch(3);
  const bool dp = c.bvh_params.collapse == 1;
  if (dp) {
    PT_CHECK_CUDA(cudaMemsetAsync(visits, 0, (size_t)(n - 1) * 4, st), "device BVH build");
    PT_CHECK_CUDA(cudaMemsetAsync(dp_choice, 0, (size_t)(n - 1) * 4, st), "device BVH build");
    k_collapse_dp<<<gl, kBlock, 0, st>>>((int)n, c.d_nodes.as<float4>(), ipar, lpar, collapse, visits, c.bvh_params.wide_cost, dp_cost,
                                         dp_choice, depth + 1);
    count_launch();
  }
  // 4-wide collapse: levels 0 .. kMaxDepth4 - 2 (wide depth, root = 1, below kMaxDepth4)
  int2 *win = work_a, *wout = work_b;
  uint64_t cap_items = 1;
  for (int L = 0; L + 1 < kMaxDepth4; ++L) {
    const int grid = grid_for(std::min<uint64_t>(cap_items, n - 1), 128, 8);
    k_collapse_level<<<grid, 128, 0, st>>>(c.d_nodes.as<float4>(), win, cnt + 2 + L, wout, cnt + 3 + L, cnt, n - 1, c.d_nodes4.as<float4>(),
                                           cnt + 1, dp ? dp_choice : nullptr);
    count_launch();
    std::swap(win, wout);
    cap_items = std::min<uint64_t>(cap_items * 4, (uint64_t)n);
  }
  PT_CHECK_CUDA(cudaGetLastError(), "device BVH build launch");
  std::vector<uint32_t> host_cnt(kMaxDepth4 + 4, 0u);
  int d2e[2] = {0, 0};
  PT_CHECK_CUDA(cudaMemcpyAsync(host_cnt.data(), cnt, host_cnt.size() * 4, cudaMemcpyDeviceToHost, st), "device BVH build");
  PT_CHECK_CUDA(cudaMemcpyAsync(d2e, depth, 8, cudaMemcpyDeviceToHost, st), "device BVH build");
  PT_CHECK_CUDA(cudaEventRecord(c.ev1, st), "device BVH build");
  PT_CHECK_CUDA(cudaStreamSynchronize(st), "device BVH build");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, c.ev0, c.ev1);
  const int d2 = d2e[0];
  if (d2e[1]) return fail(PT_CAP_EXCEEDED, "device BVH build: inconsistent tree after restructuring");
  if (d2 >= 64) return fail(PT_CAP_EXCEEDED, "device BVH build: the tree is deeper than the traversal trail allows");
  int levels = 0;
  while (levels + 1 < kMaxDepth4 && host_cnt[2 + levels] > 0) ++levels;
  const bool too_deep = host_cnt[2 + kMaxDepth4 - 1] > 0;  // items left for a level the traversal stack cannot hold
  c.bvh_depth = d2;
  c.has_bvh4 = !too_deep && host_cnt[1] == 0;
  c.build_info.builder = 1;
  c.build_info.device_ms = ms;
  c.build_info.bvh2_nodes = n - 1;
  c.build_info.bvh2_depth = (uint32_t)d2;
  c.build_info.wide_nodes = c.has_bvh4 ? host_cnt[0] : 0u;
  c.build_info.wide_depth = c.has_bvh4 ? (uint32_t)levels : 0u;
  return PT_OK;
}

}  // namespace pt
