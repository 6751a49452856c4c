// Test-only library: the product's BVH builder (pt_bvh.cu) and stackless traversal (pt_scene.cuh)
// compiled for the HOST, so the traversal logic can be checked against brute force without a GPU.
// Built by tests/conftest.py into tests/native/_build/libhost_trace.so; never part of the product.
#include <vector>

#include "../../open_rendering_framework_b200/csrc/pt_bvh.h"
#include "../../open_rendering_framework_b200/csrc/pt_scene.cuh"

using namespace pt;

struct HostScene {
  BvhHost bvh;
  std::vector<float4> nodes4;
  SceneDev S;
};

static void host_scene_views(HostScene* h, unsigned n, const BvhParams& params = BvhParams())
{
  memset(&h->S, 0, sizeof(h->S));
  h->S.nodes = h->bvh.nodes.data();
  h->S.tri_v0 = h->bvh.tri_v0.data();
  h->S.tri_e1 = h->bvh.tri_e1.data();
  h->S.tri_e2 = h->bvh.tri_e2.data();
  h->S.n_tris = n;
  int depth4 = 0;
  if (build_bvh4(h->bvh, h->nodes4, depth4, params)) h->S.nodes4 = h->nodes4.data();
}

extern "C" __attribute__((visibility("default"))) void* ht_build(const float* tri_pos, unsigned n, int* depth_out)
{
  HostScene* h = new HostScene();
  if (!build_bvh(tri_pos, n, h->bvh)) { delete h; return nullptr; }
  host_scene_views(h, n);
  h->S.trav_scale = scene_diagonal(tri_pos, n);
  if (depth_out) *depth_out = h->bvh.depth;
  return h;
}
// The same with the 4-wide collapse chosen (0 greedy, 1 SAH-optimal) and its wide-node cost.
extern "C" __attribute__((visibility("default"))) void* ht_build_collapse(const float* tri_pos, unsigned n, int collapse, float wide_cost,
                                                                          unsigned* wide_nodes)
{
  HostScene* h = new HostScene();
  BvhParams params;
  params.collapse = collapse;
  params.wide_cost = wide_cost;
  if (!build_bvh(tri_pos, n, h->bvh, params)) { delete h; return nullptr; }
  host_scene_views(h, n, params);
  h->S.trav_scale = scene_diagonal(tri_pos, n);
  if (wide_nodes) *wide_nodes = (unsigned)(h->nodes4.size() / kWideStride);
  return h;
}
// A tree given as child-pair BVH2 nodes and leaf-order triangle records (the device builder's layout,
// restated on the host by tests/lbvh_host.py), with its 4-wide collapse (greedy, as on the device).
extern "C" __attribute__((visibility("default"))) void* ht_from_arrays(const float* nodes, unsigned n_nodes, const float* v0, const float* e1,
                                                                       const float* e2, unsigned n, const float* tri_pos)
{
  HostScene* h = new HostScene();
  h->bvh.nodes.assign((const float4*)nodes, (const float4*)nodes + 4 * (size_t)n_nodes);
  h->bvh.tri_v0.assign((const float4*)v0, (const float4*)v0 + n);
  h->bvh.tri_e1.assign((const float4*)e1, (const float4*)e1 + n);
  h->bvh.tri_e2.assign((const float4*)e2, (const float4*)e2 + n);
  BvhParams greedy;  // the device builder's collapse rule
  greedy.collapse = 0;
  host_scene_views(h, n, greedy);
  h->S.trav_scale = scene_diagonal(tri_pos, n);
  return h;
}
extern "C" __attribute__((visibility("default"))) void ht_free(void* h) { delete (HostScene*)h; }
extern "C" __attribute__((visibility("default"))) unsigned ht_nodes(void* h) { return (unsigned)(((HostScene*)h)->bvh.nodes.size() / 4); }
// The same traversal with a kShortStack-entry stack of pending far children (as the persistent kernels
// use it), stride 1.
extern "C" __attribute__((visibility("default"))) void ht_trace_stack(void* hp, const float* rays, long n, int* prim, float* t, float* bary, int* any)
{
  HostScene* h = (HostScene*)hp;
  for (long i = 0; i < n; ++i) {
    const float* r = rays + 8 * i;
    float3 o = make_float3(r[0], r[1], r[2]), d = make_float3(r[4], r[5], r[6]);
    uint2 stk[kShortStack];
    RayPre rp = ray_pre(o, d, h->S.trav_scale);
    Hit hh;
    hh.t = r[7];
    hh.u = hh.v = 0.0f;
    hh.prim = -1;
    TravState st;
    trav_init(st, stk, 1);
    while (!trav_step_closest(h->S, o, d, rp, r[3], hh, st)) {}
    prim[i] = hh.prim;
    t[i] = hh.prim >= 0 ? hh.t : -1.0f;
    bary[2 * i] = hh.u;
    bary[2 * i + 1] = hh.v;
    trav_init(st, stk, 1);
    int res;
    while ((res = trav_step_any(h->S, o, d, rp, r[3], r[7], st)) == 0) {}
    any[i] = res > 0 ? 1 : 0;
  }
}
// The 4-wide BVH walked as the persistent kernels walk it (the next target a node, a leaf or kDone4;
// a kRing4-entry ring spilling to a local array).  max_sp: the deepest stack seen (above kRing4, the
// spill path ran).  Returns 0, or -1 when the scene has no 4-wide BVH.
extern "C" __attribute__((visibility("default"))) int ht_trace4(void* hp, const float* rays, long n, int* prim, float* t, float* bary, int* any, int* max_sp)
{
  HostScene* h = (HostScene*)hp;
  if (!h->S.nodes4) return -1;
  *max_sp = 0;
  for (long i = 0; i < n; ++i) {
    const float* r = rays + 8 * i;
    float3 o = make_float3(r[0], r[1], r[2]), d = make_float3(r[4], r[5], r[6]);
    uint2 ring[kRing4], spill[kSpill4];
    const int stride = 1;
    RayPre4 rp = ray_pre4(o, d, h->S.trav_scale);
    Hit hh;
    hh.t = r[7];
    hh.u = hh.v = 0.0f;
    hh.prim = -1;
    Stack4 s4;
    stack4_init(s4, ring, stride, spill);
    int cur = 0;
    while (cur != kDone4) {
      if (cur < 0) {
        leaf_closest(h->S, (uint32_t)cur, o, d, r[3], hh);
        cur = stack4_next(s4, hh.t, true);
      } else {
        cur = trav4_node_closest(h->S, cur, rp, r[3], hh, s4);
      }
      *max_sp = s4.sp > *max_sp ? s4.sp : *max_sp;
    }
    prim[i] = hh.prim;
    t[i] = hh.prim >= 0 ? hh.t : -1.0f;
    bary[2 * i] = hh.u;
    bary[2 * i + 1] = hh.v;
    stack4_init(s4, ring, stride, spill);
    cur = 0;
    int res = 0;
    while (res == 0) {
      if (cur == kDone4) res = -1;
      else if (cur < 0) {
        if (leaf_any(h->S, (uint32_t)cur, o, d, r[3], r[7])) res = 1;
        else cur = stack4_next(s4, r[7], false);
      } else {
        cur = trav4_node_any(h->S, cur, rp, r[3], r[7], s4);
      }
      *max_sp = s4.sp > *max_sp ? s4.sp : *max_sp;
    }
    any[i] = res > 0 ? 1 : 0;
  }
  return 0;
}
// rays: n x 8 floats (origin, tmin, dir, tmax)
extern "C" __attribute__((visibility("default"))) void ht_trace(void* hp, const float* rays, long n, int* prim, float* t, float* bary, int* any)
{
  HostScene* h = (HostScene*)hp;
  for (long i = 0; i < n; ++i) {
    const float* r = rays + 8 * i;
    float3 o = make_float3(r[0], r[1], r[2]), d = make_float3(r[4], r[5], r[6]);
    Hit hh = trace_closest(h->S, o, d, r[3], r[7]);
    prim[i] = hh.prim;
    t[i] = hh.prim >= 0 ? hh.t : -1.0f;
    bary[2 * i] = hh.u;
    bary[2 * i + 1] = hh.v;
    any[i] = trace_any(h->S, o, d, r[3], r[7]) ? 1 : 0;
  }
}
