// Wavefront path tracer: the sm_100a replacement for the recursive OptiX launch of
// OptixScene::renderScene (OptixScene.cpp:159) running path_tracer.cu and the material programs.
//
// One call of pt_render_frames traces every (pixel, frame) camera sample of a group of frames at
// once.  Per bounce:
//   extend   closest hit through the stackless BVH; each path id is appended to the queue of its
//            hit's material class (miss, emitter, diffuse, conductor, rough dielectric) -- the sort
//            by material key -- with block-aggregated appends (warp ballots + shared-memory prefix,
//            one global atomic per block and class)
//   shade    one kernel per material class, following diffuse_shader.cu, metallic_shader.cu,
//            rough_transparent_shader.cu, arealight_shader.cu, constantbg.cu; continuing paths are
//            appended to the next active queue and diffuse next-event estimation to the shadow queue
//   shadow   any-hit through the same BVH; unoccluded contributions are added to the path radiance
// and finally `accumulate` folds the frames into the float4 running mean in frame order
// (path_tracer.cu:64-68).  Each path keeps one tea stream and one MD5 stream exactly as the
// reference's recursion passes prd.seed down the path, so paths consume identical random numbers.
//
// The reference's recursion result is result = own + child * weight; here the equivalent iterative
// form is used: radiance += throughput * own, throughput *= weight.
//
// All queue counts live in device memory and every kernel reads its count there, so a whole render
// is a fixed sequence of launches with no host synchronisation (CUDA-graph capturable).
#include <algorithm>
#include <cstring>

#include "pt_context.h"

namespace pt {

constexpr int kBlock = 128;
constexpr int kWarps = kBlock / 32;

// Per-path metadata in rng.w
constexpr uint32_t META_DEPTH = 0xffffu;
constexpr uint32_t META_EMIT = 1u << 16;
constexpr uint32_t META_OUTSIDE = 1u << 17;

struct WfDev {
  float4* ray_o;
  float4* ray_d;
  float4* thr;
  float4* rad;
  uint4* rng;
  float4* hit;
  uint32_t* q_in;
  uint32_t* q_out;
  uint32_t* q_mat;  // kQueues * cap
  float4* sh_o;
  float4* sh_d;
  float4* sh_c;
  uint32_t* sh_pid;
  uint32_t* cnt;
  uint64_t cap;
  int in_slot, out_slot;
};

__device__ __forceinline__ unsigned lanemask_lt() { return (1u << (threadIdx.x & 31)) - 1u; }
__device__ __forceinline__ unsigned long long* cnt64(uint32_t* cnt, int slot) { return reinterpret_cast<unsigned long long*>(cnt + slot); }

// Block-aggregated append: every thread of the block calls this (uniform control flow); threads
// with want == true receive a distinct slot in [0, *counter).  One global atomic per block.
__device__ __forceinline__ uint32_t block_slot(bool want, uint32_t* counter, uint32_t* smem /* kWarps + 1 */)
{
  unsigned m = __ballot_sync(0xffffffffu, want);
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) smem[warp] = __popc(m);
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t total = 0;
    for (int w = 0; w < kWarps; ++w) {
      uint32_t c = smem[w];
      smem[w] = total;
      total += c;
    }
    smem[kWarps] = total ? atomicAdd(counter, total) : 0u;
  }
  __syncthreads();
  uint32_t slot = smem[kWarps] + smem[warp] + __popc(m & lanemask_lt());
  __syncthreads();
  return slot;
}

// Multi-queue variant: cls in [0, kQueues) or -1.
__device__ __forceinline__ uint32_t block_slot_multi(int cls, uint32_t* counters /* kQueues consecutive */, uint32_t* smem /* kWarps*kQueues + kQueues */)
{
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t rank = 0;
#pragma unroll
  for (int q = 0; q < kQueues; ++q) {
    unsigned m = __ballot_sync(0xffffffffu, cls == q);
    if (lane == 0) smem[warp * kQueues + q] = __popc(m);
    if (cls == q) rank = __popc(m & lanemask_lt());
  }
  __syncthreads();
  if (threadIdx.x < kQueues) {
    int q = threadIdx.x;
    uint32_t total = 0;
    for (int w = 0; w < kWarps; ++w) {
      uint32_t c = smem[w * kQueues + q];
      smem[w * kQueues + q] = total;
      total += c;
    }
    smem[kWarps * kQueues + q] = total ? atomicAdd(counters + q, total) : 0u;
  }
  __syncthreads();
  uint32_t slot = cls >= 0 ? smem[kWarps * kQueues + cls] + smem[warp * kQueues + cls] + rank : 0u;
  __syncthreads();
  return slot;
}

// Shading normal of a hit: normalize(rtTransformNormal(normalize(n))) with the identity transform,
// where n is the interpolated vertex normal or the geometric normal (triangle_mesh.cu:63-70,
// diffuse_shader.cu:48).
__device__ __forceinline__ float3 shading_normal(const SceneDev& S, const float4* geo, const int4& info, float u, float v, int prim)
{
  float3 n;
  if (info.x >= 0) {
    float3 n0 = ld3(__ldg(S.normals + info.x)), n1 = ld3(__ldg(S.normals + info.y)), n2 = ld3(__ldg(S.normals + info.z));
    n = normalize(n1 * u + n2 * v + n0 * (1.0f - u - v));
  } else {
    n = normalize(ld3(__ldg(geo + prim)));
  }
  return normalize(n);
}

// ------------------------------------------------------------------ lights (LightSampler.h)
__device__ __forceinline__ float3 ldf3(const float* p) { return f3(p[0], p[1], p[2]); }

// evaluate_direct_illumination, LightSampler.h:143-166 (all five light types).  Out-of-range
// triangle indices (a draw that rounds to 1.0) are clamped and counted.
__device__ void eval_direct(const SceneDev& S, const float3& pos, const LightRaw& ls, float3& dir, float3& L, float& dist, uint32_t& seed,
                            uint32_t& clamped)
{
  const float3 em = ldf3(ls.emitted);
  switch (ls.type) {
    case POINT_LIGHT: {  // :20-28
      dir = ldf3(ls.p) - pos;
      float r2 = dot(dir, dir);
      dist = sqrtf(r2);
      dir = dir / dist;
      L = em / r2;
      break;
    }
    case DIRECTIONAL_LIGHT: {  // :31-37
      dir = normalize(-ldf3(ls.p));
      dist = kDefaultMax;
      L = em;
      break;
    }
    case TRIANGLES_AREA_LIGHT: {  // :40-71
      float cnt_f = ls.p[0], start_f = ls.p[1];
      uint32_t tris = (uint32_t)cnt_f;
      uint32_t tid = (uint32_t)((float)(uint32_t)(rnd_tea(seed) * (float)tris) + start_f);
      if (tid >= (uint32_t)S.n_tri_lights) { tid = (uint32_t)S.n_tri_lights - 1; ++clamped; }
      const TriLightRaw& tl = S.tri_lights[tid];
      float3 uvw = sample_barycentric(seed);
      float3 v0 = ldf3(tl.v0), v1 = ldf3(tl.v1), v2 = ldf3(tl.v2);
      float3 lp = v0 * uvw.x + v1 * uvw.y + v2 * uvw.z;
      float3 n = tl.has_normals ? normalize(ldf3(tl.n0) * uvw.x + ldf3(tl.n1) * uvw.y + ldf3(tl.n2) * uvw.z) : normalize(cross(v1 - v0, v2 - v0));
      dir = lp - pos;
      float sq = dot(dir, dir);
      dist = sqrtf(sq);
      dir = normalize(dir);
      float cp = fmaxf(dot(n, -dir), 0.0f);
      L = em * (tl.area * cp / sq * (float)tris);
      break;
    }
    case DISK_LIGHT: {  // :73-101
      float3 lp = ldf3(ls.p);
      float radius = ls.pad[0];
      float theta = ls.pad[2] * kPi / 180.0f, phi = ls.pad[1] * kPi / 180.0f;
      float area = kPi * radius * radius;
      float pdf = 1.0f / area;
      float3 nrm = f3(sinf(theta) * sinf(phi), cosf(theta), sinf(theta) * cosf(phi));
      float3 U, V;
      create_onb(nrm, U, V);
      float u1 = rnd_tea(seed), u2 = rnd_tea(seed);
      float r = sqrtf(u1) * radius;
      float t = 2.0f * kPi * u2;
      float3 dp = f3(r * cosf(t), r * sinf(t), 0.0f);
      dp = dp.x * U + dp.y * V + dp.z * nrm;
      lp = lp + dp;
      dir = lp - pos;
      float sq = dot(dir, dir);
      dist = sqrtf(sq);
      dir = normalize(dir);
      float cp = fmaxf(dot(nrm, -dir), 0.0f);
      L = em * (cp / sq) / pdf;
      break;
    }
    case SPHERICAL_LIGHT: {  // :103-141
      float3 lp = ldf3(ls.p);
      float radius = ls.pad[0];
      float3 vn = normalize(pos - lp);
      float3 U, V;
      create_onb(vn, U, V);
      float area = 4.0f * kPi * radius * radius;
      float pdf = 1.0f / area;
      float u1 = rnd_tea(seed), u2 = rnd_tea(seed);
      float z = u1;
      float3 sp = radius * f3(cosf(2.0f * kPi * u2) * sqrtf(1.0f - z * z), sinf(2.0f * kPi * u2) * sqrtf(1.0f - z * z), z);
      sp = sp.x * U + sp.y * V + sp.z * vn + lp;
      float3 nrm = normalize(sp - lp);
      dir = sp - pos;
      float sq = dot(dir, dir);
      dist = sqrtf(sq);
      dir = normalize(dir);
      float cp = fmaxf(dot(nrm, -dir), 0.0f);
      L = em * (cp / sq) / pdf;
      break;
    }
    case ENVMAP_LIGHT: {  // the environment map as a light: sample_environment (Envmap.h:66-98)
      sample_environment(S.env, dir, L, seed);
      dist = kDefaultMax;
      break;
    }
    default:
      dir = f3s(0.0f);
      L = f3s(0.0f);
      dist = 0.0f;
      break;
  }
}

// ------------------------------------------------------------------ kernels
// path_tracer.cu:32-60: seed, jitter, pinhole direction; paths outside the patch are flagged.
__global__ void __launch_bounds__(kBlock) k_raygen(SceneDev S, WfDev w, uint32_t first_frame, uint64_t n_paths, uint32_t pixels)
{
  __shared__ uint32_t sm[kWarps + 1];
  const CameraDev& C = S.cam;
  for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < n_paths; base += (uint64_t)gridDim.x * kBlock) {
    uint64_t pid = base + threadIdx.x;
    bool valid = pid < n_paths;
    bool inside = false;
    if (valid) {
      uint32_t fl = (uint32_t)(pid / pixels), p = (uint32_t)(pid % pixels);
      uint32_t x = p % C.width, y = p / C.width;
      uint32_t frame = first_frame + fl;
      inside = !(x < C.patch_origin.x || x > C.patch_origin.x + C.patch_dims.x || y < C.patch_origin.y || y > C.patch_origin.y + C.patch_dims.y);
      if (inside) {
        uint32_t seed = tea16(C.width * y + x, frame);
        uint2 s64 = make_uint2(seed, seed);
        float jx = rnd_tea(seed);
        float jy = rnd_tea(seed);
        float ipx = ((float)x + jx) / (float)C.width * 2.0f - 1.0f;
        float ipy = ((float)y + jy) / (float)C.height * 2.0f - 1.0f;
        float3 dir = normalize(ipx * C.U + ipy * C.V + C.W);
        w.ray_o[pid] = make_float4(C.eye.x, C.eye.y, C.eye.z, 0.0f);
        w.ray_d[pid] = make_float4(dir.x, dir.y, dir.z, 0.0f);
        w.thr[pid] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        w.rad[pid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w.rng[pid] = make_uint4(seed, s64.x, s64.y, META_EMIT);
      } else {
        w.rad[pid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w.rng[pid] = make_uint4(0, 0, 0, META_OUTSIDE);
      }
    }
    uint32_t slot = block_slot(inside, w.cnt + w.in_slot, sm);
    if (inside) w.q_in[slot] = (uint32_t)pid;
  }
}

__device__ __forceinline__ int class_of(uint32_t type)
{
  switch (type) {
    case MAT_DIFFUSE: return QC_DIFFUSE;
    case MAT_METAL: return QC_METAL;
    case MAT_ROUGH_GLASS: return QC_GLASS;
    case MAT_LIGHT: return QC_LIGHT;
    default: return -1;
  }
}

__global__ void __launch_bounds__(kBlock) k_extend(SceneDev S, WfDev w)
{
  __shared__ uint32_t sm[kWarps * kQueues + kQueues];
  const uint32_t n = w.cnt[w.in_slot];
  const float eps = S.integ.scene_epsilon;
  uint32_t traced = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    uint32_t i = base + threadIdx.x;
    int cls = -1;
    uint32_t pid = 0;
    if (i < n) {
      pid = w.q_in[i];
      float4 o = w.ray_o[pid], d = w.ray_d[pid];
      Hit h = trace_closest(S, ld3(o), ld3(d), eps, kDefaultMax);
      w.hit[pid] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
      if (h.prim < 0) cls = QC_MISS;
      else cls = class_of(__ldg(&S.mats[__ldg(&S.tri_info[h.prim].w)].type));
      ++traced;
    }
    uint32_t slot = block_slot_multi(cls, w.cnt + CNT_Q_MISS, sm);
    if (cls >= 0) w.q_mat[(size_t)cls * w.cap + slot] = pid;
  }
  if (traced) atomicAdd(cnt64(w.cnt, CNT_SEGMENTS_LO), (unsigned long long)traced);
}

// Warp-aggregated multi-queue append (no block barrier): lanes with cls in [0, kQueues) get distinct
// slots; one atomic per warp and class.  All lanes of the warp must call it.
__device__ __forceinline__ uint32_t warp_slot_multi(int cls, uint32_t* counters)
{
  const unsigned lane = threadIdx.x & 31;
  uint32_t slot = 0;
#pragma unroll
  for (int q = 0; q < kQueues; ++q) {
    unsigned m = __ballot_sync(0xffffffffu, cls == q);
    if (m) {
      int leader = __ffs(m) - 1;
      uint32_t base = 0;
      if ((int)lane == leader) base = atomicAdd(counters + q, (uint32_t)__popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (cls == q) slot = base + __popc(m & lanemask_lt());
    }
  }
  return slot;
}

// Persistent closest-hit kernel with dynamic ray fetch: every warp keeps 32 rays in flight and,
// whenever at least `refill` of its lanes have finished (or the queue is drained and all have),
// hands the finished ones to the material queues and fetches new rays for the idle lanes with one
// atomic.  Traversal state (pt_scene.cuh TravState) is resumable, so lanes never wait for the
// slowest ray of a whole block (T. Aila, S. Laine, "Understanding the efficiency of ray traversal
// on GPUs", HPG 2009: persistent threads with ray replacement).
__global__ void __launch_bounds__(kBlock) k_extend_persistent(SceneDev S, WfDev w, int refill)
{
  const uint32_t n = w.cnt[w.in_slot];
  uint32_t* fetch = w.cnt + CNT_FETCH_EXT;
  const float eps = S.integ.scene_epsilon;
  const unsigned lane = threadIdx.x & 31;
  bool has = false, done = false, drained = false;
  uint32_t pid = 0, traced = 0;
  float3 o = f3s(0.0f), d = f3s(0.0f);
  RayPre rp;
  rp.inv = f3s(0.0f);
  Hit h;
  h.t = 0.0f; h.u = h.v = 0.0f; h.prim = -1;
  TravState st;
  trav_init(st);
  for (;;) {
    unsigned idle = __ballot_sync(0xffffffffu, !has);
    if (!drained && (__popc(idle) >= refill || idle == 0xffffffffu)) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(fetch, (uint32_t)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base + __popc(idle) >= n) drained = true;
      if (!has) {
        uint32_t i = base + __popc(idle & lanemask_lt());
        if (i < n) {
          pid = w.q_in[i];
          float4 o4 = w.ray_o[pid], d4 = w.ray_d[pid];
          o = ld3(o4);
          d = ld3(d4);
          rp = ray_pre(o, d);
          h.t = kDefaultMax;
          h.u = h.v = 0.0f;
          h.prim = -1;
          trav_init(st);
          has = true;
          done = false;
          ++traced;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, has) == 0) break;
    for (;;) {
      if (has && !done) done = trav_step_closest(S, o, d, rp, eps, h, st);
      unsigned fin = __ballot_sync(0xffffffffu, !has || done);
      if (fin == 0xffffffffu || (!drained && __popc(fin) >= refill)) break;
    }
    int cls = -1;
    if (has && done) {
      w.hit[pid] = make_float4(h.t, h.u, h.v, as_float(h.prim));
      cls = h.prim < 0 ? QC_MISS : class_of(__ldg(&S.mats[__ldg(&S.tri_info[h.prim].w)].type));
    }
    uint32_t slot = warp_slot_multi(cls, w.cnt + CNT_Q_MISS);
    if (cls >= 0) w.q_mat[(size_t)cls * w.cap + slot] = pid;
    if (has && done) has = false;
  }
  traced += __shfl_xor_sync(0xffffffffu, traced, 16);
  traced += __shfl_xor_sync(0xffffffffu, traced, 8);
  traced += __shfl_xor_sync(0xffffffffu, traced, 4);
  traced += __shfl_xor_sync(0xffffffffu, traced, 2);
  traced += __shfl_xor_sync(0xffffffffu, traced, 1);
  if (lane == 0 && traced) atomicAdd(cnt64(w.cnt, CNT_SEGMENTS_LO), (unsigned long long)traced);
}

// Persistent any-hit kernel for the shadow queue (same ray replacement).
__global__ void __launch_bounds__(kBlock) k_shadow_persistent(SceneDev S, WfDev w, int refill)
{
  const uint32_t n = w.cnt[CNT_SHADOW];
  uint32_t* fetch = w.cnt + CNT_FETCH_SH;
  const unsigned lane = threadIdx.x & 31;
  bool has = false, drained = false;
  int res = 0;
  uint32_t slot = 0;
  float3 o = f3s(0.0f), d = f3s(0.0f);
  float tmin = 0.0f, tmax = 0.0f;
  RayPre rp;
  rp.inv = f3s(0.0f);
  TravState st;
  trav_init(st);
  for (;;) {
    unsigned idle = __ballot_sync(0xffffffffu, !has);
    if (!drained && (__popc(idle) >= refill || idle == 0xffffffffu)) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(fetch, (uint32_t)__popc(idle));
      base = __shfl_sync(0xffffffffu, base, 0);
      if (base + __popc(idle) >= n) drained = true;
      if (!has) {
        uint32_t i = base + __popc(idle & lanemask_lt());
        if (i < n) {
          slot = i;
          float4 o4 = w.sh_o[i], d4 = w.sh_d[i];
          o = ld3(o4);
          d = ld3(d4);
          tmin = o4.w;
          tmax = d4.w;
          rp = ray_pre(o, d);
          trav_init(st);
          has = true;
          res = 0;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, has) == 0) break;
    for (;;) {
      if (has && res == 0) res = trav_step_any(S, o, d, rp, tmin, tmax, st);
      unsigned fin = __ballot_sync(0xffffffffu, !has || res != 0);
      if (fin == 0xffffffffu || (!drained && __popc(fin) >= refill)) break;
    }
    if (has && res != 0) {
      if (res < 0) {
        uint32_t p = w.sh_pid[slot];
        float4 c = w.sh_c[slot], r = w.rad[p];
        w.rad[p] = make_float4(r.x + c.x, r.y + c.y, r.z + c.z, 0.0f);
      }
      has = false;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && n) atomicAdd(cnt64(w.cnt, CNT_SHADOW_TOTAL), (unsigned long long)n);
}

// constantbg.cu:16-19 / envmap_background.cu:20-23.  With the environment map registered as a light,
// a miss after next-event estimation (emission disabled) adds nothing, as for area lights.
__global__ void __launch_bounds__(kBlock) k_shade_miss(SceneDev S, WfDev w)
{
  const uint32_t n = w.cnt[CNT_Q_MISS];
  const uint32_t* q = w.q_mat + (size_t)QC_MISS * w.cap;
  for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
    uint32_t pid = q[i];
    float3 bg = S.bg_color;
    if (S.env.present) {
      if (S.env.is_light && !(w.rng[pid].w & META_EMIT)) continue;
      bg = env_lookup(S.env, ld3(w.ray_d[pid]));
    }
    float4 t = w.thr[pid], r = w.rad[pid];
    float3 L = ld3(r) + ld3(t) * bg;
    w.rad[pid] = make_float4(L.x, L.y, L.z, 0.0f);
  }
}

// arealight_shader.cu:36-50: emitted radiance if the hit is front-facing and emission is enabled.
__global__ void __launch_bounds__(kBlock) k_shade_light(SceneDev S, WfDev w, const float4* geo)
{
  const uint32_t n = w.cnt[CNT_Q_LIGHT];
  const uint32_t* q = w.q_mat + (size_t)QC_LIGHT * w.cap;
  for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
    uint32_t pid = q[i];
    if (!(w.rng[pid].w & META_EMIT)) continue;
    float4 h = w.hit[pid], d = w.ray_d[pid];
    int prim = __float_as_int(h.w);
    int4 info = __ldg(S.tri_info + prim);
    float3 normal = shading_normal(S, geo, info, h.y, h.z, prim);
    if (dot(normal, -ld3(d)) > 0.0f) {
      const MatDev& m = S.mats[info.w];
      float4 t = w.thr[pid], r = w.rad[pid];
      float3 L = ld3(r) + ld3(t) * f3(m.a.x, m.a.y, m.a.z);
      w.rad[pid] = make_float4(L.x, L.y, L.z, 0.0f);
    }
  }
}

// diffuse_shader.cu:122-187
__global__ void __launch_bounds__(kBlock) k_shade_diffuse(SceneDev S, WfDev w, const float4* geo)
{
  __shared__ uint32_t sm[kWarps + 1];
  const uint32_t n = w.cnt[CNT_Q_DIFFUSE];
  const uint32_t* q = w.q_mat + (size_t)QC_DIFFUSE * w.cap;
  const float eps = S.integ.scene_epsilon;
  uint32_t clamped = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    uint32_t i = base + threadIdx.x;
    bool shadow = false, cont = false;
    uint32_t pid = 0;
    float3 hit_pos, w_l, sh_contrib;
    float sh_tmax = 0.0f;
    if (i < n) {
      pid = q[i];
      uint4 rg = w.rng[pid];
      int depth = (int)(rg.w & META_DEPTH);
      if (depth <= S.integ.max_depth) {
        float4 h = w.hit[pid], o = w.ray_o[pid], d4 = w.ray_d[pid], t4 = w.thr[pid];
        int prim = __float_as_int(h.w);
        int4 info = __ldg(S.tri_info + prim);
        const MatDev& m = S.mats[info.w];
        const float3 dc = f3(m.a.x, m.a.y, m.a.z);
        float3 d = ld3(d4);
        hit_pos = ld3(o) + h.x * d;
        float3 normal = shading_normal(S, geo, info, h.y, h.z, prim);
        float3 ffnormal = faceforward(normal, -d, normal);
        uint32_t t = rg.x;
        bool emit = (rg.w & META_EMIT) != 0;
        // uniform light pick and next-event estimation (:135-161)
        float draw = rnd_tea(t);
        if (S.n_lights > 0) {
          uint32_t li = (uint32_t)((float)S.n_lights * draw);
          if (li >= (uint32_t)S.n_lights) { li = (uint32_t)S.n_lights - 1; ++clamped; }
          float light_pdf = 1.0f / (float)S.n_lights;
          LightRaw ls = S.lights[li];
          float3 radiance;
          float dist;
          eval_direct(S, hit_pos, ls, w_l, radiance, dist, t, clamped);
          radiance = radiance / light_pdf;
          float cos_theta = dot(ffnormal, w_l);
          if (cos_theta > 0.0f) {
            shadow = true;
            sh_tmax = dist - eps;
            sh_contrib = ld3(t4) * (radiance * kInvPi * cos_theta * dc);
            emit = false;
          }
        }
        // Russian roulette on the mean albedo (:165-184)
        float prob = (dc.x + dc.y + dc.z) / 3.0f;
        float xi = rnd_tea(t);
        if (depth < S.integ.rr_start) prob = 1.0f;
        if (xi < prob || depth < S.integ.rr_start) {
          float3 nd = sample_cosine_weighted(ffnormal, t);
          float3 nt = ld3(t4) * (dc / prob);
          w.ray_o[pid] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, 0.0f);
          w.ray_d[pid] = make_float4(nd.x, nd.y, nd.z, 0.0f);
          w.thr[pid] = make_float4(nt.x, nt.y, nt.z, 0.0f);
          cont = true;
        }
        w.rng[pid] = make_uint4(t, rg.y, rg.z, (uint32_t)(depth + 1) | (emit ? META_EMIT : 0u));
      }
    }
    uint32_t s_slot = block_slot(shadow, w.cnt + CNT_SHADOW, sm);
    if (shadow) {
      w.sh_o[s_slot] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, eps);
      w.sh_d[s_slot] = make_float4(w_l.x, w_l.y, w_l.z, sh_tmax);
      w.sh_c[s_slot] = make_float4(sh_contrib.x, sh_contrib.y, sh_contrib.z, 0.0f);
      w.sh_pid[s_slot] = pid;
    }
    uint32_t c_slot = block_slot(cont, w.cnt + w.out_slot, sm);
    if (cont) w.q_out[c_slot] = pid;
  }
  if (clamped) atomicAdd(cnt64(w.cnt, CNT_CLAMPED), (unsigned long long)clamped);
}

// metallic_shader.cu:232-348
__global__ void __launch_bounds__(kBlock) k_shade_metal(SceneDev S, WfDev w, const float4* geo)
{
  __shared__ uint32_t sm[kWarps + 1];
  const uint32_t n = w.cnt[CNT_Q_METAL];
  const uint32_t* q = w.q_mat + (size_t)QC_METAL * w.cap;
  uint32_t capped_total = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    uint32_t i = base + threadIdx.x;
    bool cont = false;
    uint32_t pid = 0;
    if (i < n) {
      pid = q[i];
      uint4 rg = w.rng[pid];
      int depth = (int)(rg.w & META_DEPTH);
      if (depth < S.integ.max_depth) {
        float4 h = w.hit[pid], o = w.ray_o[pid], d4 = w.ray_d[pid];
        int prim = __float_as_int(h.w);
        int4 info = __ldg(S.tri_info + prim);
        const MatDev& m = S.mats[info.w];
        float3 d = ld3(d4);
        float3 hit_point = ld3(o) + h.x * d;
        float3 normal = shading_normal(S, geo, info, h.y, h.z, prim);
        float3 ffnormal = faceforward(normal, -d, normal);
        float3 w_i = -d;
        uint32_t seed = rg.x;
        float a_x = m.a.x, a_y = m.a.y;
        int capped = 0;
        float3 w_o, weight;
        bool go = true;
        if (m.model == MULTISCATTERING) {
          uint32_t order = 0;
          float3 lwo = ms_conductor_sample(m.dist, to_local(w_i, normal), m.eta, m.inv_eta, a_x, a_y, seed, order, weight, &capped);
          w_o = to_world(lwo, normal);
        } else {
          float z1 = rnd_tea(seed), z2 = rnd_tea(seed);
          float3 mn;
          float G_i_m, G_o_m;
          if (m.model == WALTER) {
            mn = sample_normal(m.dist, ffnormal, z1, z2, a_x);
            G_i_m = masking_G1(m.dist, w_i, mn, ffnormal, a_x);
          } else {
            mn = sample_visible_normal(m.dist, w_i, ffnormal, a_x, a_y, z1, z2, &capped);
            G_i_m = masking_G1_aniso(m.dist, w_i, mn, ffnormal, a_x, a_y);
          }
          go = G_i_m > 0.0f;
          if (go) {
            float3 F = fresnel_complex(w_i, mn, m.eta);
            w_o = -w_i + 2.0f * mn * dot(w_i, mn);
            float abs_i_m = fabsf(dot(w_i, mn)), abs_i_n = fabsf(dot(w_i, ffnormal)), abs_n_m = fabsf(dot(normal, mn));
            G_o_m = (m.model == WALTER) ? masking_G1(m.dist, w_o, mn, ffnormal, a_x) : masking_G1_aniso(m.dist, w_o, mn, ffnormal, a_x, a_y);
            go = G_o_m > 0.0f;
            weight = (m.model == WALTER) ? F * (abs_i_m * G_i_m * G_o_m / (abs_i_n * abs_n_m)) : F * G_o_m;
          }
        }
        capped_total += capped;
        if (go) {
          float4 t4 = w.thr[pid];
          float3 nt = ld3(t4) * weight;
          w.ray_o[pid] = make_float4(hit_point.x, hit_point.y, hit_point.z, 0.0f);
          w.ray_d[pid] = make_float4(w_o.x, w_o.y, w_o.z, 0.0f);
          w.thr[pid] = make_float4(nt.x, nt.y, nt.z, 0.0f);
          cont = true;
        }
        w.rng[pid] = make_uint4(seed, rg.y, rg.z, (uint32_t)(depth + 1) | META_EMIT);
      }
    }
    uint32_t c_slot = block_slot(cont, w.cnt + w.out_slot, sm);
    if (cont) w.q_out[c_slot] = pid;
  }
  if (capped_total) atomicAdd(cnt64(w.cnt, CNT_CAPPED), (unsigned long long)capped_total);
}

// rough_transparent_shader.cu:66-225
__global__ void __launch_bounds__(kBlock) k_shade_glass(SceneDev S, WfDev w, const float4* geo)
{
  __shared__ uint32_t sm[kWarps + 1];
  const uint32_t n = w.cnt[CNT_Q_GLASS];
  const uint32_t* q = w.q_mat + (size_t)QC_GLASS * w.cap;
  uint32_t capped_total = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    uint32_t i = base + threadIdx.x;
    bool cont = false;
    uint32_t pid = 0;
    if (i < n) {
      pid = q[i];
      uint4 rg = w.rng[pid];
      int depth = (int)(rg.w & META_DEPTH);
      if (depth < S.integ.max_depth) {
        float4 h = w.hit[pid], o = w.ray_o[pid], d4 = w.ray_d[pid];
        int prim = __float_as_int(h.w);
        int4 info = __ldg(S.tri_info + prim);
        const MatDev& m = S.mats[info.w];
        const float ior = m.a.x, rough = m.a.y;
        float3 d = ld3(d4);
        float3 hit_point = ld3(o) + h.x * d;
        float3 normal = shading_normal(S, geo, info, h.y, h.z, prim);
        float3 ffnormal = faceforward(normal, -d, normal);
        float3 w_i = -d;
        uint32_t t = rg.x;
        float3 beam_T = f3s(1.0f);
        bool go = true;
        float cos_theta = dot(-d, normal);
        if (cos_theta < 0.0f) {  // Beer absorption with Russian roulette inside (:84-91)
          beam_T = expf3((-h.x) * f3(m.b.x, m.b.y, m.b.z));
          float prob = (beam_T.x + beam_T.y + beam_T.z) / 3.0f;
          if (rnd_tea(t) >= prob) go = false;
          else beam_T = beam_T / prob;
        }
        int capped = 0;
        float3 w_o;
        float3 weight = f3s(1.0f);
        if (go) {
          float z1 = rnd_tea(t), z2 = rnd_tea(t);
          if (m.model == MULTISCATTERING) {  // :100-120
            uint32_t order = 0;
            float3 lwo = ms_dielectric_sample(m.dist, to_local(w_i, normal), 1.0f / ior, rough, rough, t, order, &capped);
            w_o = to_world(lwo, normal);
          } else {
            float3 mn = (m.model == WALTER) ? sample_normal(m.dist, ffnormal, z1, z2, rough)
                                            : sample_visible_normal(m.dist, w_i, ffnormal, rough, rough, z1, z2, &capped);
            float cos_in = dot(normal, w_i);
            float eta = cos_in < 0.0f ? ior : 1.0f / ior;
            float G_i_m = (m.model == WALTER) ? masking_G1(m.dist, w_i, mn, ffnormal, rough) : masking_G1_aniso(m.dist, w_i, mn, ffnormal, rough, rough);
            go = G_i_m > 0.0f;
            if (go) {
              // get_rough_glass_rays (:39-55)
              float ct = fabsf(dot(mn, -d));
              float st2 = eta * eta * (1.0f - ct * ct);
              float ctt = sqrtf(1.0f - st2);
              float R = st2 < 1.0f ? fresnel_R(ct, ctt, eta) : 1.0f;
              float3 refr = eta * d + mn * (eta * ct - ctt);
              float3 refl = reflect(d, mn);
              float abs_i_m = fabsf(dot(w_i, mn)), abs_i_n = fabsf(dot(w_i, ffnormal)), abs_n_m = fabsf(dot(normal, mn));
              float rr = rnd_tea(t);
              w_o = rr > R ? refr : refl;
              float G_o_m = (m.model == WALTER) ? masking_G1(m.dist, w_o, mn, ffnormal, rough) : masking_G1_aniso(m.dist, w_o, mn, ffnormal, rough, rough);
              go = G_o_m > 0.0f;
              float wgt = (m.model == WALTER) ? abs_i_m * G_i_m * G_o_m / (abs_i_n * abs_n_m) : G_o_m;
              weight = f3s(wgt);
            }
          }
        }
        capped_total += capped;
        if (go) {
          float4 t4 = w.thr[pid];
          float3 nt = ld3(t4) * weight * beam_T;
          w.ray_o[pid] = make_float4(hit_point.x, hit_point.y, hit_point.z, 0.0f);
          w.ray_d[pid] = make_float4(w_o.x, w_o.y, w_o.z, 0.0f);
          w.thr[pid] = make_float4(nt.x, nt.y, nt.z, 0.0f);
          cont = true;
        }
        w.rng[pid] = make_uint4(t, rg.y, rg.z, (uint32_t)(depth + 1) | META_EMIT);
      }
    }
    uint32_t c_slot = block_slot(cont, w.cnt + w.out_slot, sm);
    if (cont) w.q_out[c_slot] = pid;
  }
  if (capped_total) atomicAdd(cnt64(w.cnt, CNT_CAPPED), (unsigned long long)capped_total);
}

// Shadow rays of diffuse_shader.cu:149-161 (every material's any-hit program is opaque).
__global__ void __launch_bounds__(kBlock) k_shadow(SceneDev S, WfDev w)
{
  const uint32_t n = w.cnt[CNT_SHADOW];
  for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
    float4 o = w.sh_o[i], d = w.sh_d[i];
    if (!trace_any(S, ld3(o), ld3(d), o.w, d.w)) {
      uint32_t pid = w.sh_pid[i];
      float4 c = w.sh_c[i], r = w.rad[pid];
      w.rad[pid] = make_float4(r.x + c.x, r.y + c.y, r.z + c.z, 0.0f);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && n) atomicAdd(cnt64(w.cnt, CNT_SHADOW_TOTAL), (unsigned long long)n);
}

// path_tracer.cu:36-43 and :64-68, frame by frame in order.
__global__ void __launch_bounds__(kBlock) k_accumulate(SceneDev S, WfDev w, float4* accum, uint32_t first_frame, uint32_t n_frames, uint32_t pixels)
{
  for (uint32_t p = blockIdx.x * kBlock + threadIdx.x; p < pixels; p += gridDim.x * kBlock) {
    float4 out = accum[p];
    for (uint32_t fl = 0; fl < n_frames; ++fl) {
      uint64_t pid = (uint64_t)fl * pixels + p;
      uint32_t frame = first_frame + fl;
      if (w.rng[pid].w & META_OUTSIDE) {
        out = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        continue;
      }
      float4 r = w.rad[pid];
      if (isfinite(r.x) && isfinite(r.y) && isfinite(r.z)) {
        float4 cur = frame != 0 ? make_float4(out.x * (float)frame, out.y * (float)frame, out.z * (float)frame, out.w * (float)frame)
                                : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        float den = (float)(frame + 1);
        out = make_float4((r.x + cur.x) / den, (r.y + cur.y) / den, (r.z + cur.z) / den, (1.0f + cur.w) / den);
      }
    }
    accum[p] = out;
  }
}

// Geometric normals (unnormalised cross(v1-v0, v2-v0)) per original triangle, for meshes without
// vertex normals and for the emitter test.
__global__ void k_geo_normals(SceneDev S, float4* geo)
{
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < S.n_tris; j += gridDim.x * blockDim.x) {
    float4 a = S.tri_v0[j], b = S.tri_e1[j], c = S.tri_e2[j];
    float3 n = cross(ld3(b), ld3(c));
    geo[__float_as_int(a.w)] = make_float4(n.x, n.y, n.z, 0.0f);
  }
}

static pt_status ensure_wavefront(Context& c, uint64_t cap)
{
  Wavefront& wf = c.wf;
  if (wf.cap >= cap && wf.counters.p) return PT_OK;
  pt_status st = PT_OK;
  const size_t f4 = sizeof(float4), u4 = sizeof(uint4);
  if (st == PT_OK) st = wf.ray_o.reserve(cap * f4, "wavefront ray origins");
  if (st == PT_OK) st = wf.ray_d.reserve(cap * f4, "wavefront ray directions");
  if (st == PT_OK) st = wf.thr.reserve(cap * f4, "wavefront throughput");
  if (st == PT_OK) st = wf.rad.reserve(cap * f4, "wavefront radiance");
  if (st == PT_OK) st = wf.rng.reserve(cap * u4, "wavefront rng");
  if (st == PT_OK) st = wf.hit.reserve(cap * f4, "wavefront hits");
  if (st == PT_OK) st = wf.q_a.reserve(cap * 4, "queue");
  if (st == PT_OK) st = wf.q_b.reserve(cap * 4, "queue");
  if (st == PT_OK) st = wf.q_mat.reserve(cap * 4 * kQueues, "material queues");
  if (st == PT_OK) st = wf.sh_o.reserve(cap * f4, "shadow queue");
  if (st == PT_OK) st = wf.sh_d.reserve(cap * f4, "shadow queue");
  if (st == PT_OK) st = wf.sh_c.reserve(cap * f4, "shadow queue");
  if (st == PT_OK) st = wf.sh_pid.reserve(cap * 4, "shadow queue");
  if (st == PT_OK) st = wf.counters.reserve(kCounters * 4, "counters");
  if (st != PT_OK) {
    wf.cap = 0;
    return st;
  }
  wf.cap = cap;
  return PT_OK;
}

}  // namespace pt

using namespace pt;

extern "C" {

pt_status pt_render_frames(pt_ctx* ctx, uint32_t first_frame, uint32_t n_frames)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  Context& c = ctx->c;
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  if (!c.built) return fail(PT_NOT_READY, "pt_render_frames: call pt_build first");
  if (!c.camera_set) return fail(PT_NOT_READY, "pt_render_frames: camera not set");
  if (n_frames == 0) return PT_OK;
  for (const LightRaw& l : c.lights)
    if (l.type == ENVMAP_LIGHT && !c.env_present)
      return fail(PT_NOT_READY, "pt_render_frames: an environment-map light needs pt_set_envmap");
  for (const MatDev& m : c.mats)
    if (m.type == MAT_DIFFUSE && c.lights.empty())
      return fail(PT_NOT_READY, "pt_render_frames: diffuse materials need at least one light (light_buffer is indexed unguarded by the diffuse shader)");
  if (c.dirty_materials) {
    PT_CHECK_CUDA(cudaMemcpyAsync(c.d_mats.p, c.mats.data(), c.mats.size() * sizeof(MatDev), cudaMemcpyHostToDevice, c.stream), "material upload");
    c.dirty_materials = false;
  }
  const uint32_t pixels = c.cam.width * c.cam.height;
  uint32_t frames_per_pass = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(n_frames, c.max_paths / pixels));
  uint64_t cap = (uint64_t)frames_per_pass * pixels;
  pt_status st = ensure_wavefront(c, cap);
  if (st != PT_OK) return st;
  // per-context geometric normals (computed once per build)
  DevBuf& geo = c.d_normals_geo;
  if (!geo.p || geo.bytes < (size_t)c.n_tris * sizeof(float4) || c.geo_stale) {
    st = geo.reserve((size_t)c.n_tris * sizeof(float4), "geometric normals");
    if (st != PT_OK) return st;
    k_geo_normals<<<grid_for(c.n_tris, 256, 8), 256, 0, c.stream>>>(c.view(), geo.as<float4>());
    count_launch();
    c.geo_stale = false;
  }
  uint64_t launches0 = pt_kernel_launch_count();
  SceneDev S = c.view();
  WfDev w;
  Wavefront& wf = c.wf;
  w.ray_o = wf.ray_o.as<float4>();
  w.ray_d = wf.ray_d.as<float4>();
  w.thr = wf.thr.as<float4>();
  w.rad = wf.rad.as<float4>();
  w.rng = wf.rng.as<uint4>();
  w.hit = wf.hit.as<float4>();
  w.q_mat = wf.q_mat.as<uint32_t>();
  w.sh_o = wf.sh_o.as<float4>();
  w.sh_d = wf.sh_d.as<float4>();
  w.sh_c = wf.sh_c.as<float4>();
  w.sh_pid = wf.sh_pid.as<uint32_t>();
  w.cnt = wf.counters.as<uint32_t>();
  w.cap = wf.cap;
  const float4* geo_p = geo.as<float4>();
  const int grid_trace = sm_count() * 8, grid_shade = sm_count() * 8;
  int occ_ext = 0, occ_sh = 0;
  PT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_ext, k_extend_persistent, kBlock, 0), "occupancy");
  PT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sh, k_shadow_persistent, kBlock, 0), "occupancy");
  const int grid_persist = sm_count() * std::max(1, std::min(occ_ext, occ_sh));
  PT_CHECK_CUDA(cudaMemsetAsync(w.cnt, 0, kCounters * 4, c.stream), "reset counters");
  c.prof_pairs = 0;
  PT_CHECK_CUDA(cudaEventRecord(c.ev0, c.stream), "event");
  float extend_ms = 0.0f;
  uint32_t extend_launches = 0;
  for (uint32_t f0 = 0; f0 < n_frames; f0 += frames_per_pass) {
    uint32_t nf = std::min(frames_per_pass, n_frames - f0);
    uint64_t n_paths = (uint64_t)nf * pixels;
    w.q_in = wf.q_a.as<uint32_t>();
    w.q_out = wf.q_b.as<uint32_t>();
    w.in_slot = CNT_ACTIVE_A;
    w.out_slot = CNT_ACTIVE_B;
    PT_CHECK_CUDA(cudaMemsetAsync(w.cnt, 0, 8 * 4, c.stream), "reset queues");
    k_raygen<<<grid_for(n_paths, kBlock, 16), kBlock, 0, c.stream>>>(S, w, first_frame + f0, n_paths, pixels);
    count_launch();
    const int passes = c.integ.max_depth + 2;
    for (int b = 0; b < passes; ++b) {
      PT_CHECK_CUDA(cudaMemsetAsync(w.cnt + CNT_Q_MISS, 0, 6 * 4, c.stream), "reset queues");
      PT_CHECK_CUDA(cudaMemsetAsync(w.cnt + CNT_FETCH_EXT, 0, 2 * 4, c.stream), "reset fetch counters");
      PT_CHECK_CUDA(cudaMemsetAsync(w.cnt + w.out_slot, 0, 4, c.stream), "reset queues");
      if (c.profile) {
        while (c.prof_events.size() < 2 * (size_t)(c.prof_pairs + 1)) {
          cudaEvent_t ev;
          PT_CHECK_CUDA(cudaEventCreate(&ev), "profiling event");
          c.prof_events.push_back(ev);
        }
        PT_CHECK_CUDA(cudaEventRecord(c.prof_events[2 * c.prof_pairs], c.stream), "profiling event");
      }
      if (c.opt.extend_mode == 1)
        k_extend_persistent<<<grid_persist, kBlock, 0, c.stream>>>(S, w, c.opt.refill);
      else
        k_extend<<<grid_trace, kBlock, 0, c.stream>>>(S, w);
      if (c.profile) {
        PT_CHECK_CUDA(cudaEventRecord(c.prof_events[2 * c.prof_pairs + 1], c.stream), "profiling event");
        ++c.prof_pairs;
      }
      k_shade_miss<<<grid_shade, kBlock, 0, c.stream>>>(S, w);
      k_shade_light<<<grid_shade, kBlock, 0, c.stream>>>(S, w, geo_p);
      k_shade_diffuse<<<grid_shade, kBlock, 0, c.stream>>>(S, w, geo_p);
      k_shade_metal<<<grid_shade, kBlock, 0, c.stream>>>(S, w, geo_p);
      k_shade_glass<<<grid_shade, kBlock, 0, c.stream>>>(S, w, geo_p);
      if (c.opt.extend_mode == 1)
        k_shadow_persistent<<<grid_persist, kBlock, 0, c.stream>>>(S, w, c.opt.refill);
      else
        k_shadow<<<grid_trace, kBlock, 0, c.stream>>>(S, w);
      count_launch(7);
      ++extend_launches;
      std::swap(w.q_in, w.q_out);
      std::swap(w.in_slot, w.out_slot);
    }
    k_accumulate<<<grid_for(pixels, kBlock, 16), kBlock, 0, c.stream>>>(S, w, c.d_accum.as<float4>(), first_frame + f0, nf, pixels);
    count_launch();
  }
  PT_CHECK_CUDA(cudaEventRecord(c.ev1, c.stream), "event");
  PT_CHECK_CUDA(cudaGetLastError(), "pt_render_frames launch");
  memset(&c.stats, 0, sizeof(c.stats));
  c.stats.path_samples = 0;
  {
    uint64_t inside_w = (uint64_t)std::min<uint32_t>(c.cam.width, c.cam.patch_origin.x + c.cam.patch_dims.x + 1) -
                        std::min<uint32_t>(c.cam.width, c.cam.patch_origin.x);
    uint64_t inside_h = (uint64_t)std::min<uint32_t>(c.cam.height, c.cam.patch_origin.y + c.cam.patch_dims.y + 1) -
                        std::min<uint32_t>(c.cam.height, c.cam.patch_origin.y);
    c.stats.path_samples = inside_w * inside_h * n_frames;
  }
  c.stats.extend_launches = extend_launches;
  c.stats.kernel_launches = (uint32_t)(pt_kernel_launch_count() - launches0);
  c.stats.extend_ms = extend_ms;
  c.stats_pending = true;
  return PT_OK;
}

pt_status pt_get_render_stats(pt_ctx* ctx, pt_render_stats* out)
{
  if (!ctx || !out) return fail(PT_INVALID_ARG, "pt_get_render_stats: null argument");
  Context& c = ctx->c;
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_get_render_stats");
  if (c.stats_pending && c.wf.counters.p) {
    uint32_t h[kCounters];
    PT_CHECK_CUDA(cudaMemcpy(h, c.wf.counters.p, sizeof(h), cudaMemcpyDeviceToHost), "read counters");
    auto rd64 = [&](int slot) { unsigned long long v; memcpy(&v, h + slot, 8); return (uint64_t)v; };
    c.stats.segments = rd64(CNT_SEGMENTS_LO);
    c.stats.shadow_rays = rd64(CNT_SHADOW_TOTAL);
    c.stats.capped_walks = rd64(CNT_CAPPED);
    c.stats.clamped_indices = rd64(CNT_CLAMPED);
    float ms = 0.0f;
    PT_CHECK_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1), "event time");
    c.stats.gpu_ms = ms;
    float ext = 0.0f;
    for (uint32_t k = 0; k < c.prof_pairs; ++k) {
      float e = 0.0f;
      PT_CHECK_CUDA(cudaEventElapsedTime(&e, c.prof_events[2 * k], c.prof_events[2 * k + 1]), "event time");
      ext += e;
    }
    c.stats.extend_ms = ext;
    c.stats_pending = false;
  }
  *out = c.stats;
  return PT_OK;
}

}  // extern "C"
