// Wavefront path tracer: the sm_100a replacement for the recursive OptiX launch of
// OptixScene::renderScene (OptixScene.cpp:159) running path_tracer.cu and the material programs.
//
// One call of pt_render_frames traces every (pixel, frame) camera sample of a group of frames at
// once.  Per bounce:
//   extend   closest hit through the BVH; the class of each ray's hit (miss, emitter, diffuse, conductor,
//            rough dielectric, translucent, layered) is recorded by queue position
//   bin      a stable partition of the queue by class into the material queues -- the sort by material
//            key -- (warp ballots + shared-memory prefix per block, a scan over the blocks)
//   shade    one kernel per material class, following diffuse_shader.cu, metallic_shader.cu,
//            rough_transparent_shader.cu, arealight_shader.cu, constantbg.cu; continuing paths are
//            appended to the next active queue and diffuse next-event estimation to the shadow queue
//   shadow   any-hit through the same BVH; unoccluded contributions are added to the path radiance
// and finally `accumulate` folds the frames into the float4 running mean in frame order
// (path_tracer.cu:64-68).
//
// Scenes with translucent objects first run the probe pass of every frame (sample_camera.cu): one
// PositionSample per (object, sample), lit by a shadowed light sample or by an indirect path that
// goes through the same wavefront.  The probes with L != 0 are compacted in order, and the dipole
// gathers that camera paths owe on entering a translucent object are evaluated after the paths end
// (see k_shade_translucent).  Each path keeps one tea stream and one MD5 stream exactly as the
// reference's recursion passes prd.seed down the path, so paths consume identical random numbers.
//
// The reference's recursion result is result = own + child * weight; here the equivalent iterative
// form is used: radiance += throughput * own, throughput *= weight.
//
// All queue counts live in device memory and every kernel reads its count there, so a whole render
// is a fixed sequence of launches with no host synchronisation (CUDA-graph capturable).
#include <algorithm>
#include <cstring>
#include <type_traits>

#include "pt_context.h"
#include "pt_dipole.cuh"

namespace pt {

constexpr int kBlock = 128;
constexpr int kWarps = kBlock / 32;
// Threads per block of the persistent traversal kernels, and the resident blocks per SM they are
// compiled for (register budget: 1,024 threads per SM at 64 registers).
#ifndef PT_TRACE_BLOCK
#define PT_TRACE_BLOCK 128
#endif
#ifndef PT_TRACE_MIN_BLOCKS
#define PT_TRACE_MIN_BLOCKS (1024 / PT_TRACE_BLOCK)
#endif
constexpr int kTraceBlock = PT_TRACE_BLOCK;
// The 4-wide persistent kernels alternate warp-wide phases of leaf tests and node steps.  Closest hit:
// a leaf phase once the lanes holding a leaf are at least twice those that can take a node step
// (leaf tests wait for more company); any hit: once they are at least half of them (an occluder found
// early ends the ray).  Measured against "at least as many" on the single-scene render: +0.5 %.
constexpr int kLeafVsNodeClosest = 2;
constexpr int kLeafVsNodeAny = 2;
// Per-path metadata in rng.w
constexpr uint32_t META_DEPTH = 0xffffu;
constexpr uint32_t META_EMIT = 1u << 16;
constexpr uint32_t META_OUTSIDE = 1u << 17;
constexpr uint32_t META_PROBE = 1u << 18;  // a probe's indirect path (sample_camera.cu:168-206)
constexpr int META_GSHIFT = 24;            // pending dipole gathers on the path's stack (8 bits)
constexpr uint32_t META_KEEP = ~(META_DEPTH | META_EMIT);

// One 16-byte field of a per-path pair record: field k of path i sits at rec[2 i + k].  The ray (origin,
// direction) and the path state (throughput, rng state) are two 32-byte records per path, each one
// whole sector: a shading kernel reading and rewriting a path at a random id touches two whole sectors
// instead of four half sectors of four arrays, and the extend kernel reads exactly the ray's sector
// (consecutive paths' rays are contiguous).
template <class T> struct Field2 {
  T* p;
  __device__ __forceinline__ T& operator[](uint64_t i) const { return p[2 * i]; }
};

struct WfDev {
  Field2<float4> ray_o;
  Field2<float4> ray_d;
  Field2<float4> thr;
  float4* rad;
  Field2<uint4> rng;
  float4* hit;
  uint32_t* q_in;
  uint32_t* q_out;
  uint32_t* q_mat;  // kQueues * cap
  uint8_t* cls_of;  // material class of the ray at each position of q_in (written by extend, binned by k_bin_*)
  uint32_t* bin;    // per chunk of kBinChunk queue positions: kQueues class counts, then starts in the queues
  float4* sh_o;
  float4* sh_d;
  float4* sh_c;
  uint32_t* sh_pid;
  uint32_t* cnt;
  uint64_t cap;
  int in_slot, out_slot;
  // pending dipole gathers, [slot * cap + path]: (xo, throughput.x), (no, throughput.y), (throughput.z, material)
  float4* g_a;
  float4* g_b;
  float2* g_c;
  float4* g_d;  // the gather's weight (rough boundary) and 1, or (1, 1, 1, 0) for a smooth boundary
  uint32_t g_slots;
  // adjoint renders: per path (image gradient of the path, pending kind) and (pending d w / w, index)
  float4* adj_a;
  float4* adj_b;
  // the scenes and items of the pass; each path's item
  const SceneDev* scenes;
  const ItemDev* items;
  uint32_t n_items;
  uint32_t multi;   // 0: every path of the chunk renders scenes[scene0]
  uint32_t scene0;
  uint16_t* path_item;
};

// Probe storage of a pass, indexed by probe id (item after item, then frame, object, sample).
struct SssDev {
  float4* probes;      // 5 float4 per PositionSample
  float4* pc_pos;      // compacted probes with L != 0 per (frame, object) set, at the set's first probe id: pos
  float4* pc_wl;       //   weight * L
  float4* pc_nrm;      //   normal
  float4* pc_tr;       //   transmitted
  uint32_t* pc_cnt;    //   count per set
};

// Index of the last item whose begin field is <= key (every begin field increases item after item).
template <class F>
__device__ __forceinline__ uint32_t find_item(const ItemDev* items, uint32_t n, uint64_t key, F begin)
{
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if ((uint64_t)begin(items[mid]) <= key) lo = mid;
    else hi = mid;
  }
  return lo;
}
__device__ __forceinline__ const SceneDev& scene_of(const WfDev& w, uint32_t pid)
{
  const uint32_t k = w.multi ? w.items[w.path_item[pid]].scene : w.scene0;
  return w.scenes[k];
}

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


// Shading normal of a hit: normalize(rtTransformNormal(normalize(n))) with the identity transform,
// where n is the interpolated vertex normal or the geometric normal (triangle_mesh.cu:63-70,
// diffuse_shader.cu:48).
__device__ __forceinline__ float3 shading_normal(const SceneDev& S, const int4& info, float u, float v, int prim)
{
  float3 n;
  if (info.x >= 0) {
    float3 n0 = ld3(__ldg(S.normals + info.x)), n1 = ld3(__ldg(S.normals + info.y)), n2 = ld3(__ldg(S.normals + info.z));
    n = normalize(n1 * u + n2 * v + n0 * (1.0f - u - v));
  } else {
    n = normalize(ld3(__ldg(S.geo + prim)));
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


// ------------------------------------------------------------------ MD5 stream across vertices
// The diffuse, conductor, rough-dielectric and layered shaders hand their child ray only the tea seed
// (diffuse_shader.cu:92-101, metallic_shader.cu:76-156, rough_transparent_shader.cu:114-220,
// lambertian_interface_shader.cu:143-147, rough_diffuse_shader.cu:207-211): their own
// MD5 state is never updated from the child, so after such a vertex returns, the dipole gathers of the
// translucent vertices above it draw from the MD5 state the vertex was entered with (the oracle passes
// that state down to the child, which the reference leaves uninitialised).  The wavefront keeps one
// running MD5 state per path and evaluates the gathers at the end, newest first; a vertex of those
// shaders with gathers pending above it therefore pushes a reset marker holding its entry state,
// which the gather evaluation restores when it reaches the marker.  The smooth transparent shader
// traces its child with its own payload (transparent_shader.cu:110-112), so the MD5 state simply
// runs on through it and it pushes no marker.
__device__ __forceinline__ uint32_t push_md5_reset(const WfDev& w, uint32_t pid, uint32_t meta, uint32_t s64x, uint32_t s64y, uint32_t& overflow)
{
  if (!(meta & META_PROBE) && (meta >> META_GSHIFT) != 0) {
    const uint32_t slot = meta >> META_GSHIFT;
    if (slot < w.g_slots) {
      size_t at = (size_t)slot * w.cap + pid;
      w.g_a[at] = make_float4(__uint_as_float(s64x), __uint_as_float(s64y), 0.0f, 0.0f);
      w.g_b[at] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      w.g_c[at] = make_float2(0.0f, __int_as_float(-1));
      meta += 1u << META_GSHIFT;
    } else {
      ++overflow;
    }
  }
  return meta;
}

// ------------------------------------------------------------------ path replay backprop
// The adjoint render replays every camera path with the same random numbers (same kernels, same
// decisions) and differentiates the path's contribution with respect to the scene parameters,
// with sampling detached: directions, Russian-roulette and acceptance decisions and their
// probabilities are those of the forward render; only the weights and emissions that the parameters
// enter are differentiated (M. Vicini, S. Speierer, W. Jakob, "Path replay backpropagation",
// SIGGRAPH 2021).  With T_k the throughput at vertex k, w_k its weight and E_k what vertex k adds
// to the path radiance L = sum_k T_k E_k:
//   dL/dtheta = sum_k T_k dE_k/dtheta + (dw_k/dtheta / w_k) R_{k+1},   R_{k+1} = sum_{m>k} T_m E_m.
// R starts as the forward render's L of the path and loses T_k E_k as the replay passes vertex k, so
// nothing of the path is stored: a vertex leaves (dw/w, parameter) pending in the path state, and the
// next kernel that handles the path -- after the shadow ray of the vertex has been resolved -- adds it
// times the current R.  Each gradient is weighted by the path's image gradient dLoss/dL.
enum PendingKind : uint32_t { PEND_NONE = 0, PEND_ALBEDO = 1, PEND_ROUGH = 2, PEND_SIGMA = 3 };
constexpr uint32_t kNoTexel = 0xffffffffu;

__device__ __forceinline__ void set_pending(const WfDev& w, uint32_t pid, uint32_t kind, uint32_t id, uint32_t index, const float3& d)
{
  float4 a = w.adj_a[pid];
  w.adj_a[pid] = make_float4(a.x, a.y, a.z, __uint_as_float(kind | (id << 8)));
  w.adj_b[pid] = make_float4(d.x, d.y, d.z, __uint_as_float(index));
}

// Adds the pending gradient of the path's previous vertex (R is the radiance collected beyond it).
__device__ __forceinline__ void apply_pending(const SceneDev& S, const WfDev& w, uint32_t pid)
{
  float4 a = w.adj_a[pid];
  const uint32_t kind = __float_as_uint(a.w);
  if ((kind & 0xffu) == PEND_NONE) return;
  const float4 b = w.adj_b[pid];
  const float3 R = ld3(w.rad[pid]);
  const uint32_t id = kind >> 8, idx = __float_as_uint(b.w);
  switch (kind & 0xffu) {
    case PEND_ALBEDO: {
      float* g = S.tex[id].grad;
      if (g) {
        atomicAdd(g + 3 * idx, a.x * b.x * R.x);
        atomicAdd(g + 3 * idx + 1, a.y * b.y * R.y);
        atomicAdd(g + 3 * idx + 2, a.z * b.z * R.z);
      }
      break;
    }
    case PEND_ROUGH: {
      float* g = S.tex[id].grad;
      if (g) atomicAdd(g + idx, (a.x * R.x + a.y * R.y + a.z * R.z) * b.x);
      break;
    }
    case PEND_SIGMA: {
      float* g = S.mat_grad[id];
      if (g) {
        // b = d w / d sigma_a / w per channel; sigma_s' enters the extinction divided by (1 - g)
        // (standard dipole) or times (1 + g) (delta-Eddington, directional dipole)
        const float3 mc = S.scat[id].meancosine;
        const bool dir = S.mats[id].model == DIRECTIONAL_DIPOLE;
        const float3 k = dir ? f3(1.0f + mc.x, 1.0f + mc.y, 1.0f + mc.z) : f3(1.0f / (1.0f - mc.x), 1.0f / (1.0f - mc.y), 1.0f / (1.0f - mc.z));
        const float3 ga = f3(a.x * b.x * R.x, a.y * b.y * R.y, a.z * b.z * R.z);
        atomicAdd(g + 0, ga.x);
        atomicAdd(g + 1, ga.y);
        atomicAdd(g + 2, ga.z);
        atomicAdd(g + 3, ga.x * k.x);
        atomicAdd(g + 4, ga.y * k.y);
        atomicAdd(g + 5, ga.z * k.z);
      }
      break;
    }
    default:
      break;
  }
  w.adj_a[pid] = make_float4(a.x, a.y, a.z, __uint_as_float(PEND_NONE));
}

// d ln D / d alpha of the GGX distribution at microfacet normal m (ggx_distribution):
// D = alpha^2 / (pi cos^4 (alpha^2 + tan^2)^2).
__device__ __forceinline__ float ggx_dlnD(const float3& m, const float3& n, float alpha)
{
  float c = dot(m, n);
  if (!(c > 0.0f)) return 0.0f;
  float c2 = c * c, t2 = (1.0f - c2) / c2, a2 = alpha * alpha;
  return 2.0f / alpha - 4.0f * alpha / (a2 + t2);
}
// d ln G1 / d alpha of the GGX Smith masking (ggx_G1_cos): G1 = 2 / (1 + sqrt(1 + alpha^2 tan^2)).
__device__ __forceinline__ float ggx_dlnG1(const float3& v, const float3& n, float alpha)
{
  float c = dot(v, n);
  float c2 = c * c, t2 = (1.0f - c2) / c2;
  float q = sqrtf(1.0f + alpha * alpha * t2);
  return -(alpha * t2 / q) / (1.0f + q);
}

// A value with its derivatives with respect to (sigma_a, sigma_s') of one channel.
struct Dual2 {
  float v, da, ds;
};
// The standard dipole of one channel (standard_dipole.h:8-29) and its derivatives with respect to the
// channel's sigma_a and sigma_s' (before the material's scale; A depends on the ior only):
// ln S_r = ln 3D + ln(1 + tr d_r) - tr d_r - 3 ln d_r, and likewise for the virtual source.
__device__ __forceinline__ Dual2 dipole_channel_grad(float dist, float sa, float red_ext, float A, float scale)
{
  const float x = red_ext;             // sigma_t' (scaled)
  const float D = 1.0f / (3.0f * x);
  const float dD = -D / x * scale;     // d D / d sigma (either), sigma_t' = (sigma_s' + sigma_a) * scale
  const float three_D = 3.0f * D, d3D = 3.0f * dD;
  const float tr = sqrtf(sa / D);      // sqrt(3 sigma_a sigma_t')
  const float dtr_a = 3.0f * scale * (x + sa) / (2.0f * tr), dtr_s = 3.0f * sa * scale / (2.0f * tr);
  const float ext = 4.0f * A * D, dext = 4.0f * A * dD;
  const float r2 = dist * dist;
  const float dr2 = r2 + three_D * three_D, dr = sqrtf(dr2), ddr = three_D * d3D / dr;
  const float dv2 = r2 + ext * ext, dv = sqrtf(dv2), ddv = ext * dext / dv;
  const float cmf = three_D + ext, dcmf = d3D + dext;
  const float trr = tr * dr, trv = tr * dv;
  const float Sr = three_D * (1.0f + trr) / (dr2 * dr) * expf(-trr);
  const float Sv = cmf * (1.0f + trv) / (dv2 * dv) * expf(-trv);
  // d(tr d) for each of the two parameters
  const float dtrr_a = dtr_a * dr + tr * ddr, dtrr_s = dtr_s * dr + tr * ddr;
  const float dtrv_a = dtr_a * dv + tr * ddv, dtrv_s = dtr_s * dv + tr * ddv;
  const float kr_a = d3D / three_D + dtrr_a / (1.0f + trr) - dtrr_a - 3.0f * ddr / dr;
  const float kr_s = d3D / three_D + dtrr_s / (1.0f + trr) - dtrr_s - 3.0f * ddr / dr;
  const float kv_a = dcmf / cmf + dtrv_a / (1.0f + trv) - dtrv_a - 3.0f * ddv / dv;
  const float kv_s = dcmf / cmf + dtrv_s / (1.0f + trv) - dtrv_s - 3.0f * ddv / dv;
  return Dual2{Sr + Sv, Sr * kr_a + Sv * kv_a, Sr * kr_s + Sv * kv_s};
}

// ------------------------------------------------------------------ kernels
// path_tracer.cu:32-60: seed, jitter, pinhole direction; paths outside the patch are flagged.
// kAdj: the adjoint replay; the path's radiance slot carries R (the forward radiance of the path, not
// yet passed by the replay) and adj_a its image gradient.
template <bool kAdj>
__global__ void __launch_bounds__(kBlock) k_raygen(WfDev w, uint64_t n_paths)
{
  __shared__ uint32_t sm[kWarps + 1];
  for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < n_paths; base += (uint64_t)gridDim.x * kBlock) {
    uint64_t pid = base + threadIdx.x;
    bool valid = pid < n_paths;
    bool inside = false;
    if (valid) {
      uint32_t k = find_item(w.items, w.n_items, pid, [](const ItemDev& it) { return it.path_begin; });
      const ItemDev& it = w.items[k];
      const SceneDev& S = w.scenes[it.scene];
      const CameraDev& C = S.cam;
      w.path_item[pid] = (uint16_t)k;
      uint64_t local = pid - it.path_begin;
      uint32_t fl = (uint32_t)(local / it.pixels), p = (uint32_t)(local % it.pixels);
      uint32_t x = p % C.width, y = p / C.width;
      uint32_t frame = it.first_frame + fl;
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
        if constexpr (kAdj) {
          const uint64_t gp = (uint64_t)(frame - S.adj_first) * it.pixels + p;
          const float4 L = S.adj_L[gp];
          const float4 di = S.adj_dimg[p];
          // the running mean skips non-finite samples (path_tracer.cu:64-68): no gradient through them
          const bool fin = isfinite(L.x) && isfinite(L.y) && isfinite(L.z);
          const float sc = fin ? S.adj_dscale : 0.0f;
          w.rad[pid] = make_float4(L.x, L.y, L.z, 0.0f);
          w.adj_a[pid] = make_float4(di.x * sc, di.y * sc, di.z * sc, __uint_as_float(PEND_NONE));
        } else {
          w.rad[pid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
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
    case MAT_LAMBERTIAN_INTERFACE: return QC_LAYERED;
    case MAT_ROUGH_DIFFUSE: return QC_LAYERED;
    case MAT_METAL: return QC_METAL;
    case MAT_ROUGH_GLASS: return QC_GLASS;
    case MAT_TRANSPARENT: return QC_GLASS;
    case MAT_TRANSLUCENT: return QC_TRANS;
    case MAT_ROUGH_TRANSLUCENT: return QC_TRANS;
    case MAT_LIGHT: return QC_LIGHT;
    default: return -1;
  }
}

__global__ void __launch_bounds__(kBlock) k_extend(WfDev w)
{
  const uint32_t n = w.cnt[w.in_slot];
  uint32_t traced = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    uint32_t i = base + threadIdx.x;
    int cls = -1;
    uint32_t pid = 0;
    if (i < n) {
      pid = w.q_in[i];
      const SceneDev& S = scene_of(w, pid);
      float4 o = w.ray_o[pid], d = w.ray_d[pid];
      Hit h = scene_closest(S, ld3(o), ld3(d), S.integ.scene_epsilon, kDefaultMax);
      w.hit[pid] = make_float4(h.t, h.u, h.v, __int_as_float(h.prim));
      if (h.prim < 0) cls = QC_MISS;
      else if ((uint32_t)h.prim >= S.n_tris) cls = QC_LIGHT;  // a disk or sphere emitter
      else cls = class_of(__ldg(&S.mats[__ldg(&S.tri_info[h.prim].w)].type));
      w.cls_of[i] = (uint8_t)cls;
      ++traced;
    }
  }
  if (traced) atomicAdd(cnt64(w.cnt, CNT_SEGMENTS_LO), (unsigned long long)traced);
}


// Persistent closest-hit kernel with dynamic ray fetch: every warp keeps 32 rays in flight and,
// whenever at least `refill` of its lanes have finished (or the queue is drained and all have),
// hands the finished ones to the material queues and fetches new rays for the idle lanes with one
// atomic.  Traversal state (pt_scene.cuh TravState) is resumable, so lanes never wait for the
// slowest ray of a whole block (T. Aila, S. Laine, "Understanding the efficiency of ray traversal
// on GPUs", HPG 2009: persistent threads with ray replacement).
// kMulti: the rays belong to several scenes (a batch); each lane keeps its ray's scene view in
// registers.  Otherwise the single scene is the kernel parameter S0.
// kW4: the 4-wide BVH (node steps of pt_scene.cuh trav4_*, the next target `cur` a node, a leaf or
// kDone4); otherwise the BVH2 with the postponed-leaf pair (leafA, leafB).
template <bool kMulti, bool kW4>
__global__ void __launch_bounds__(kTraceBlock, PT_TRACE_MIN_BLOCKS) k_extend_persistent(SceneDev S0, WfDev w, int refill)
{
  __shared__ uint2 stk[(kW4 ? kRing4 : kShortStack) * kTraceBlock];
  const uint32_t n = w.cnt[w.in_slot];
  uint32_t* fetch = w.cnt + CNT_FETCH_EXT;
  TravGeom g = trav_geom(S0);
  float eps = S0.integ.scene_epsilon;
  const MatDev* mats = S0.mats;
  const int4* tinfo = S0.tri_info;
  const unsigned lane = threadIdx.x & 31;
  bool has = false, done = false, drained = false;
  uint32_t pid = 0, qi = 0, traced = 0;
  float3 o = f3s(0.0f), d = f3s(0.0f);
  std::conditional_t<kW4, RayPre4, RayPre> rp{};
  Hit h;
  h.t = 0.0f; h.u = h.v = 0.0f; h.prim = -1;
  TravState st;
  trav_init(st, stk + threadIdx.x, kTraceBlock);
  uint32_t leafA = 0, leafB = 0;
  uint2 spill4[kW4 ? kSpill4 : 1];
  Stack4 s4;
  stack4_init(s4, stk + threadIdx.x, kTraceBlock, spill4);
  int cur = kDone4;
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
          qi = i;
          if constexpr (kMulti) {
            const SceneDev& S = scene_of(w, pid);
            g = trav_geom(S);
            eps = S.integ.scene_epsilon;
            mats = S.mats;
            tinfo = S.tri_info;
          }
          float4 o4 = w.ray_o[pid], d4 = w.ray_d[pid];
          o = ld3(o4);
          d = ld3(d4);
          if constexpr (kW4) rp = ray_pre4(o, d, g.trav_scale);
          else rp = ray_pre(o, d, g.trav_scale);
          h.t = kDefaultMax;
          h.u = h.v = 0.0f;
          h.prim = -1;
          if constexpr (kW4) {
            stack4_init(s4, stk + threadIdx.x, kTraceBlock, spill4);
            cur = 0;
          } else {
            trav_init(st, stk + threadIdx.x, kTraceBlock);
          }
          has = true;
          done = false;
          ++traced;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, has) == 0) break;
    for (;;) {
      // a warp-wide phase: intersect the postponed leaves (4-wide: when the lanes holding leaves are at
      // least kLeafVsNodeClosest times those that can take a node step; BVH2: at least as many), else
      // advance the lanes without leaves by one node
      if constexpr (kW4) {
        const bool lp = has && cur < 0;
        const bool np = has && cur >= 0 && cur != kDone4;
        const unsigned lmask = __ballot_sync(0xffffffffu, lp);
        const unsigned nmask = __ballot_sync(0xffffffffu, np);
        if (lmask && (nmask == 0 || __popc(lmask) >= kLeafVsNodeClosest * __popc(nmask))) {
          if (lp) {
            leaf_closest(g, (uint32_t)cur, o, d, eps, h);
            cur = stack4_next(s4, h.t, true);
          }
        } else if (np) {
          cur = trav4_node_closest(g, cur, rp, eps, h, s4);
        }
        done = cur == kDone4;
      } else {
        const bool lp = has && leafA != 0;
        const unsigned lmask = __ballot_sync(0xffffffffu, lp);
        const unsigned nmask = __ballot_sync(0xffffffffu, has && !done && !lp);
        if (lmask && (nmask == 0 || __popc(lmask) >= __popc(nmask))) {
          if (lp) {
            leaf_closest(g, leafA, o, d, eps, h);
            if (leafB) leaf_closest(g, leafB, o, d, eps, h);
            leafA = leafB = 0;
          }
        } else if (has && !done && !lp) {
          done = trav_node_closest(g, o, rp, eps, h, st, leafA, leafB);
        }
      }
      unsigned fin = __ballot_sync(0xffffffffu, !has || (done && leafA == 0));
      if (fin == 0xffffffffu || (!drained && __popc(fin) >= refill)) break;
    }
    int cls = -1;
    if (has && done && leafA == 0) {
      // the analytic emitters (disk and sphere lights) after the triangles
      uint32_t n_tris;
      if constexpr (kMulti) {
        const SceneDev& S = scene_of(w, pid);
        n_tris = S.n_tris;
        if (S.n_ana) ana_closest(S, o, d, eps, h);
      } else {
        n_tris = S0.n_tris;
        if (S0.n_ana) ana_closest(S0, o, d, eps, h);
      }
      w.hit[pid] = make_float4(h.t, h.u, h.v, as_float(h.prim));
      cls = h.prim < 0 ? QC_MISS : (uint32_t)h.prim >= n_tris ? QC_LIGHT : class_of(__ldg(&mats[__ldg(&tinfo[h.prim].w)].type));
      w.cls_of[qi] = (uint8_t)cls;
    }
    if (has && done && leafA == 0) has = false;
  }
  traced += __shfl_xor_sync(0xffffffffu, traced, 16);
  traced += __shfl_xor_sync(0xffffffffu, traced, 8);
  traced += __shfl_xor_sync(0xffffffffu, traced, 4);
  traced += __shfl_xor_sync(0xffffffffu, traced, 2);
  traced += __shfl_xor_sync(0xffffffffu, traced, 1);
  if (lane == 0 && traced) atomicAdd(cnt64(w.cnt, CNT_SEGMENTS_LO), (unsigned long long)traced);
}

// ------------------------------------------------------------------ binning by material (the sort by material key)
// The extend kernels record the class of the ray at each queue position (cls_of); these three kernels
// partition the queue stably by class into the material queues, so that each queue keeps the order of
// the rays it came from: camera rays in pixel order, later bounces in the order the shading kernels
// appended them.  Neighbouring entries of a material queue then address neighbouring path records
// (coalesced state reads and writes in the shading kernels) and emit spatially coherent shadow rays.
// The queue is cut into chunks of kBinThreads * kItems positions (kItems consecutive positions per
// thread; kItems = 4, 8 or 16, the launch option "bin_items" that the autotuner sets -- the sort
// granularity); k_bin_count counts every chunk's classes, k_bin_scan turns the counts into each
// chunk's start in every material queue (one block, chunk order), and k_bin_scatter writes every
// chunk's entries there.
constexpr int kBinThreads = 256;
constexpr int kBinItemsMin = 4;
constexpr int kBinWarps = kBinThreads / 32;
__host__ __device__ constexpr uint32_t bin_chunk(int items) { return (uint32_t)kBinThreads * (uint32_t)items; }

// The classes of the kItems positions of this thread in chunk k (-1 past the end of the queue); a full
// run is one aligned vector load of kItems bytes.
template <int kItems>
__device__ __forceinline__ void bin_load(const WfDev& w, uint32_t n, uint32_t k, int c[kItems])
{
  const uint32_t i0 = k * bin_chunk(kItems) + threadIdx.x * kItems;
  if (i0 + kItems <= n) {
    uint32_t v[kItems / 4];
    if constexpr (kItems == 4) {
      v[0] = *reinterpret_cast<const uint32_t*>(w.cls_of + i0);
    } else if constexpr (kItems == 8) {
      const uint2 u = *reinterpret_cast<const uint2*>(w.cls_of + i0);
      v[0] = u.x;
      v[1] = u.y;
    } else {
      const uint4 u = *reinterpret_cast<const uint4*>(w.cls_of + i0);
      v[0] = u.x;
      v[1] = u.y;
      v[2] = u.z;
      v[3] = u.w;
    }
#pragma unroll
    for (int j = 0; j < kItems; ++j) c[j] = (int)((v[j >> 2] >> (8 * (j & 3))) & 0xffu);
  } else {
#pragma unroll
    for (int j = 0; j < kItems; ++j) c[j] = i0 + j < n ? (int)w.cls_of[i0 + j] : -1;
  }
}

template <int kItems>
__global__ void __launch_bounds__(kBinThreads) k_bin_count(WfDev w)
{
  __shared__ uint32_t cnt[kQueues];
  const uint32_t n = w.cnt[w.in_slot];
  const uint32_t chunks = (n + bin_chunk(kItems) - 1) / bin_chunk(kItems);
  for (uint32_t k = blockIdx.x; k < chunks; k += gridDim.x) {
    if (threadIdx.x < kQueues) cnt[threadIdx.x] = 0;
    __syncthreads();
    int c[kItems];
    bin_load<kItems>(w, n, k, c);
#pragma unroll
    for (int q = 0; q < kQueues; ++q) {
      uint32_t v = 0;
#pragma unroll
      for (int j = 0; j < kItems; ++j) v += c[j] == q;
      for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
      if ((threadIdx.x & 31) == 0 && v) atomicAdd(&cnt[q], v);
    }
    __syncthreads();
    if (threadIdx.x < kQueues) w.bin[(size_t)k * kQueues + threadIdx.x] = cnt[threadIdx.x];
  }
}

// One block of 1024 threads per class q (blockIdx.x): the exclusive scan of the class's chunk counts
// (in place, chunk order) and its total (the material queue count).
__global__ void __launch_bounds__(1024) k_bin_scan(WfDev w, uint32_t chunk)
{
  __shared__ uint32_t warp_sum[32];
  const uint32_t n = w.cnt[w.in_slot];
  const uint32_t chunks = (n + chunk - 1) / chunk;
  const uint32_t per = (chunks + 1023) / 1024;  // consecutive chunks per thread
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  {
    const int q = blockIdx.x;
    uint32_t v = 0;
    for (uint32_t j = 0; j < per; ++j) {
      const uint32_t k = t * per + j;
      if (k < chunks) v += w.bin[(size_t)k * kQueues + q];
    }
    uint32_t x = v;  // inclusive warp scan of the per-thread sums
    for (int off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
      if (lane >= off) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
      uint32_t s = warp_sum[lane];
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, s, off);
        if (lane >= off) s += y;
      }
      warp_sum[lane] = s;
    }
    __syncthreads();
    uint32_t run = x - v + (wid ? warp_sum[wid - 1] : 0u);
    for (uint32_t j = 0; j < per; ++j) {
      const uint32_t k = t * per + j;
      if (k < chunks) {
        const uint32_t c = w.bin[(size_t)k * kQueues + q];
        w.bin[(size_t)k * kQueues + q] = run;
        run += c;
      }
    }
    if (t == 0) w.cnt[CNT_Q_MISS + q] = warp_sum[31];
  }
}

template <int kItems>
__global__ void __launch_bounds__(kBinThreads) k_bin_scatter(WfDev w)
{
  __shared__ uint32_t wtot[kBinWarps][kQueues];
  const uint32_t n = w.cnt[w.in_slot];
  const uint32_t chunks = (n + bin_chunk(kItems) - 1) / bin_chunk(kItems);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint32_t k = blockIdx.x; k < chunks; k += gridDim.x) {
    int c[kItems];
    bin_load<kItems>(w, n, k, c);
    uint32_t pos[kQueues];
#pragma unroll
    for (int q = 0; q < kQueues; ++q) {  // exclusive prefix of this thread's count over the warp
      uint32_t v = 0;
#pragma unroll
      for (int j = 0; j < kItems; ++j) v += c[j] == q;
      uint32_t x = v;
      for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
      }
      pos[q] = x - v;
      if (lane == 31) wtot[wid][q] = x;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < kQueues; ++q) {
      uint32_t base = w.bin[(size_t)k * kQueues + q];
      for (int ww = 0; ww < wid; ++ww) base += wtot[ww][q];
      pos[q] += base;
    }
    const uint32_t i0 = k * bin_chunk(kItems) + threadIdx.x * kItems;
#pragma unroll
    for (int j = 0; j < kItems; ++j) {
      if (c[j] < 0) continue;
      uint32_t at = 0;
#pragma unroll
      for (int q = 0; q < kQueues; ++q)
        if (c[j] == q) at = pos[q]++;
      w.q_mat[(size_t)c[j] * w.cap + at] = w.q_in[i0 + j];
    }
    __syncthreads();
  }
}

// The three binning launches at kItems positions per thread.
template <int kItems>
static void launch_binning(const WfDev& w, int grid, cudaStream_t st)
{
  k_bin_count<kItems><<<grid, kBinThreads, 0, st>>>(w);
  k_bin_scan<<<kQueues, 1024, 0, st>>>(w, bin_chunk(kItems));
  k_bin_scatter<kItems><<<grid, kBinThreads, 0, st>>>(w);
}

// Adds an unoccluded next-event estimate to the path (kAdj: takes it off R, and adds the albedo
// texel's gradient: the estimate is linear in the albedo).
template <bool kAdj>
__device__ __forceinline__ void shadow_unoccluded(const SceneDev& S, const WfDev& w, uint32_t slot)
{
  const uint32_t p = w.sh_pid[slot];
  const float4 c = w.sh_c[slot], r = w.rad[p];
  if constexpr (kAdj) {
    w.rad[p] = make_float4(r.x - c.x, r.y - c.y, r.z - c.z, 0.0f);
    const uint32_t code = __float_as_uint(c.w);
    if (code != kNoTexel) {
      const TexDev& T = S.tex[code >> 24];
      const uint32_t tx = code & 0xffffffu;
      if (T.grad) {
        const float4 a = w.adj_a[p];
        atomicAdd(T.grad + 3 * tx, a.x * c.x / __ldg(T.data + 3 * tx));
        atomicAdd(T.grad + 3 * tx + 1, a.y * c.y / __ldg(T.data + 3 * tx + 1));
        atomicAdd(T.grad + 3 * tx + 2, a.z * c.z / __ldg(T.data + 3 * tx + 2));
      }
    }
  } else {
    w.rad[p] = make_float4(r.x + c.x, r.y + c.y, r.z + c.z, 0.0f);
  }
}

// Persistent any-hit kernel for the shadow queue (same ray replacement and BVH choice).
template <bool kMulti, bool kAdj, bool kW4>
__global__ void __launch_bounds__(kTraceBlock, PT_TRACE_MIN_BLOCKS) k_shadow_persistent(SceneDev S0, WfDev w, int refill)
{
  __shared__ uint2 stk[(kW4 ? kRing4 : kShortStack) * kTraceBlock];
  const uint32_t n = w.cnt[CNT_SHADOW];
  uint32_t* fetch = w.cnt + CNT_FETCH_SH;
  TravGeom g = trav_geom(S0);
  const unsigned lane = threadIdx.x & 31;
  bool has = false, drained = false, nodes_done = false;
  int res = 0;
  uint32_t slot = 0, leafA = 0, leafB = 0;
  float3 o = f3s(0.0f), d = f3s(0.0f);
  float tmin = 0.0f, tmax = 0.0f;
  std::conditional_t<kW4, RayPre4, RayPre> rp{};
  TravState st;
  trav_init(st, stk + threadIdx.x, kTraceBlock);
  uint2 spill4[kW4 ? kSpill4 : 1];
  Stack4 s4;
  stack4_init(s4, stk + threadIdx.x, kTraceBlock, spill4);
  int cur = kDone4;
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
          if constexpr (kMulti) g = trav_geom(scene_of(w, w.sh_pid[i]));
          float4 o4 = w.sh_o[i], d4 = w.sh_d[i];
          o = ld3(o4);
          d = ld3(d4);
          tmin = o4.w;
          tmax = d4.w;
          if constexpr (kW4) rp = ray_pre4(o, d, g.trav_scale);
          else rp = ray_pre(o, d, g.trav_scale);
          if constexpr (kW4) {
            stack4_init(s4, stk + threadIdx.x, kTraceBlock, spill4);
            cur = 0;
          } else {
            trav_init(st, stk + threadIdx.x, kTraceBlock);
          }
          has = true;
          res = 0;
          nodes_done = false;
          leafA = leafB = 0;
        }
      }
    }
    if (__ballot_sync(0xffffffffu, has) == 0) break;
    for (;;) {
      if constexpr (kW4) {
        const bool lp = has && res == 0 && cur < 0;
        const bool np = has && res == 0 && cur >= 0 && cur != kDone4;
        const unsigned lmask = __ballot_sync(0xffffffffu, lp);
        const unsigned nmask = __ballot_sync(0xffffffffu, np);
        if (lmask && (nmask == 0 || kLeafVsNodeAny * __popc(lmask) >= __popc(nmask))) {
          if (lp) {
            if (leaf_any(g, (uint32_t)cur, o, d, tmin, tmax)) res = 1;
            else cur = stack4_next(s4, tmax, false);
          }
        } else if (np) {
          cur = trav4_node_any(g, cur, rp, tmin, tmax, s4);
        }
        if (has && res == 0 && cur == kDone4) res = -1;
      } else {
        const bool lp = has && res == 0 && leafA != 0;
        const unsigned lmask = __ballot_sync(0xffffffffu, lp);
        const unsigned nmask = __ballot_sync(0xffffffffu, has && res == 0 && !nodes_done && !lp);
        if (lmask && (nmask == 0 || __popc(lmask) >= __popc(nmask))) {
          if (lp) {
            if (leaf_any(g, leafA, o, d, tmin, tmax) || (leafB && leaf_any(g, leafB, o, d, tmin, tmax))) res = 1;
            leafA = leafB = 0;
          }
        } else if (has && res == 0 && !nodes_done && !lp) {
          nodes_done = trav_node_any(g, o, rp, tmin, tmax, st, leafA, leafB);
        }
        if (has && res == 0 && nodes_done && leafA == 0) res = -1;
      }
      unsigned fin = __ballot_sync(0xffffffffu, !has || res != 0);
      if (fin == 0xffffffffu || (!drained && __popc(fin) >= refill)) break;
    }
    if (has && res != 0) {
      if (res < 0) {
        if constexpr (kMulti) {
          const SceneDev& S = scene_of(w, w.sh_pid[slot]);
          if (!(S.n_ana && ana_any(S, o, d, tmin, tmax))) shadow_unoccluded<kAdj>(S, w, slot);
        } else {
          if (!(S0.n_ana && ana_any(S0, o, d, tmin, tmax))) shadow_unoccluded<kAdj>(S0, w, slot);
        }
      }
      has = false;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && n) atomicAdd(cnt64(w.cnt, CNT_SHADOW_TOTAL), (unsigned long long)n);
}

// constantbg.cu:16-19 / envmap_background.cu:20-23.  With the environment map registered as a light,
// a miss after next-event estimation (emission disabled) adds nothing, as for area lights.
// kAdj (all shade kernels): the adjoint replay; the first thing done for a path is adding the pending
// gradient of its previous vertex, and what the forward adds to the path radiance is taken off R.
template <bool kAdj>
__global__ void __launch_bounds__(kBlock) k_shade_miss(WfDev w)
{
  const uint32_t n = w.cnt[CNT_Q_MISS];
  const uint32_t* q = w.q_mat + (size_t)QC_MISS * w.cap;
  for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
    uint32_t pid = q[i];
    const SceneDev& S = scene_of(w, pid);
    if constexpr (kAdj) apply_pending(S, w, pid);
    float3 bg = S.bg_color;
    if (S.env.present) {
      if (S.env.is_light && !(w.rng[pid].w & META_EMIT)) continue;
      bg = env_lookup(S.env, ld3(w.ray_d[pid]));
    }
    float4 t = w.thr[pid], r = w.rad[pid];
    float3 L = kAdj ? ld3(r) - ld3(t) * bg : ld3(r) + ld3(t) * bg;
    w.rad[pid] = make_float4(L.x, L.y, L.z, 0.0f);
  }
}

// arealight_shader.cu:36-50: emitted radiance if the hit is front-facing and emission is enabled.
template <bool kAdj>
__global__ void __launch_bounds__(kBlock) k_shade_light(WfDev w)
{
  const uint32_t n = w.cnt[CNT_Q_LIGHT];
  const uint32_t* q = w.q_mat + (size_t)QC_LIGHT * w.cap;
  for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
    uint32_t pid = q[i];
    const SceneDev& S = scene_of(w, pid);
    if constexpr (kAdj) apply_pending(S, w, pid);
    if (!(w.rng[pid].w & META_EMIT)) continue;
    float4 h = w.hit[pid], d = w.ray_d[pid];
    int prim = __float_as_int(h.w);
    float3 normal, Le;
    if ((uint32_t)prim >= S.n_tris) {  // a disk or sphere light's geometry with the same emitter program
      const uint32_t k = (uint32_t)prim - S.n_tris;
      normal = ana_normal(S, k, ld3(w.ray_o[pid]), ld3(d), h.x);
      Le = ld3(__ldg(S.ana + 3 * k + 2));
    } else {
      int4 info = __ldg(S.tri_info + prim);
      normal = shading_normal(S, info, h.y, h.z, prim);
      const MatDev& m = S.mats[info.w];
      Le = f3(m.a.x, m.a.y, m.a.z);
    }
    if (dot(normal, -ld3(d)) > 0.0f) {
      float4 t = w.thr[pid], r = w.rad[pid];
      float3 L = kAdj ? ld3(r) - ld3(t) * Le : ld3(r) + ld3(t) * Le;
      w.rad[pid] = make_float4(L.x, L.y, L.z, 0.0f);
    }
  }
}

// rough_diffuse_shader.cu:55-292, one vertex of a Lambertian base under a rough dielectric interface:
// a visible microfacet normal from two tea draws and its Fresnel reflectance R_i; a light sample whose
// shadow ray is traced here, because the reference evaluates the multiscattering BSDFs (which draw tea
// randoms) and clears emit_light only when the light is visible; then, with probability 1 - R_i, the
// base (cosine-weighted about the microfacet normal, or the multiscattering diffuse walk) and otherwise
// the mirror reflection about the microfacet normal (or the multiscattering conductor walk with
// eta = 1 / ior, whose weight the reference does not apply).  Adds the light estimate to the path
// radiance, writes the continuation ray and throughput, and returns whether the path continues.
__device__ __forceinline__ bool rough_diffuse_vertex(const SceneDev& S, const WfDev& w, uint32_t pid, const float3& hit_pos, const float3& d,
                                                  const float3& normal, const float3& ffnormal, const MatDev& m, uint32_t& t, bool& emit,
                                                  uint32_t& clamped, int& capped)
{
  const float3 w_i = -d;
  const float3 dc = f3(m.a.x, m.a.y, m.a.z);
  const float n1_over_n2 = 1.0f / m.a.w;
  const float r_10 = m.b.x;
  const float a_x = m.b.y, a_y = m.b.z;
  const uint32_t dist = m.dist;
  const bool ms = m.model == MULTISCATTERING;
  const float z1 = rnd_tea(t);
  const float z2 = rnd_tea(t);
  const float3 mn = sample_visible_normal(dist, w_i, ffnormal, a_x, a_y, z1, z2, &capped);
  const float R_i = fresnel_interface(dot(w_i, mn), n1_over_n2);
  const float T_01_i = 1.0f - R_i;
  const float4 t4 = w.thr[pid];
  // direct illumination (:100-178)
  uint32_t li = (uint32_t)((float)S.n_lights * rnd_tea(t));
  if (li >= (uint32_t)S.n_lights) { li = (uint32_t)S.n_lights - 1; ++clamped; }
  const float light_pdf = 1.0f / (float)S.n_lights;
  const LightRaw ls = S.lights[li];
  float3 w_l, radiance;
  float ldist;
  eval_direct(S, hit_pos, ls, w_l, radiance, ldist, t, clamped);
  radiance = radiance / light_pdf;
  const float cos_theta_l = dot(ffnormal, w_l);
  if (cos_theta_l > 0.0f && !scene_any(S, hit_pos, w_l, S.integ.scene_epsilon, ldist)) {
    const float3 Li = radiance;  // V * radiance with V = 1
    float3 add;
    if (ms) {  // :126-139
      const float3 lwi = to_local(w_i, ffnormal), lwl = to_local(w_l, ffnormal);
      add = Li * ms_diffuse_eval(dist, lwi, lwl, a_x, a_y, t, dc, 0u, &capped);
      add = add + Li * ms_conductor_eval(dist, lwi, lwl, m.eta, m.inv_eta, a_x, a_y, t, 0u, &capped);
    } else {  // :140-176
      const float3 refl_normal = normalize(w_i + w_l);
      const float R_refl = fresnel_interface(dot(refl_normal, w_l), n1_over_n2);
      const float T_01_diff = 1.0f - fresnel_interface(dot(mn, w_l), n1_over_n2);
      const float G_i_m_refl = masking_G1_aniso(dist, w_i, refl_normal, ffnormal, a_x, a_y);
      const float G_o_m_refl = masking_G1_aniso(dist, w_l, refl_normal, ffnormal, a_x, a_y);
      const float G_o_m_diff = masking_G1_aniso(dist, w_l, mn, ffnormal, a_x, a_y);
      const float D_refl = eval_visible_normal(dist, w_i, refl_normal, ffnormal, a_x, a_y);
      const float weight_refl = G_i_m_refl * G_o_m_refl * D_refl / (4.0f * fabsf(dot(w_i, ffnormal) * dot(w_l, ffnormal)));
      add = Li * kInvPi * cos_theta_l * dc * n1_over_n2 * n1_over_n2 * T_01_i * T_01_diff / (1.0f - dc * r_10) * G_o_m_diff;
      add = add + Li * R_refl * weight_refl;
    }
    emit = false;
    const float4 r = w.rad[pid];
    w.rad[pid] = make_float4(r.x + t4.x * add.x, r.y + t4.y * add.y, r.z + t4.z * add.z, 0.0f);
  }
  // indirect illumination (:181-289)
  const float xi = rnd_tea(t);
  float3 nd, weight;
  if (xi > R_i) {
    if (ms) {  // :187-218
      uint32_t order = 0;
      float3 wgt, lwm;
      nd = to_world(ms_diffuse_sample(dist, to_local(w_i, ffnormal), a_x, a_y, t, order, wgt, dc, lwm, &capped), ffnormal);
      const float T_01_r = 1.0f - fresnel_interface(dot(nd, to_world(lwm, ffnormal)), n1_over_n2);
      weight = f3s(n1_over_n2 * n1_over_n2 * T_01_r) / (1.0f - dc * r_10) * wgt;
    } else {  // :219-248
      nd = sample_cosine_weighted(mn, t);
      const float cos_theta_r = dot(nd, mn);
      const float G_o_m = masking_G1_aniso(dist, nd, mn, ffnormal, a_x, a_y);
      if (G_o_m < 0.0f) return false;
      const float T_01_r = 1.0f - fresnel_interface(cos_theta_r, n1_over_n2);
      weight = dc * n1_over_n2 * n1_over_n2 * T_01_r / (1.0f - dc * r_10) * G_o_m;
    }
  } else {
    if (ms) {  // :252-269 (the walk's Fresnel weight is not applied)
      uint32_t order = 10;
      float3 wgt;
      nd = to_world(ms_conductor_sample(dist, to_local(w_i, normal), m.eta, m.inv_eta, a_x, a_y, t, order, wgt, &capped), normal);
      weight = f3s(1.0f);
    } else {  // :270-287
      nd = reflect(d, mn);
      const float G_o_m = masking_G1_aniso(dist, nd, mn, ffnormal, a_x, a_y);
      if (G_o_m < 0.0f) return false;
      weight = f3s(G_o_m);
    }
  }
  const float3 nt = ld3(t4) * weight;
  w.ray_o[pid] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, 0.0f);
  w.ray_d[pid] = make_float4(nd.x, nd.y, nd.z, 0.0f);
  w.thr[pid] = make_float4(nt.x, nt.y, nt.z, 0.0f);
  return true;
}

// Layered materials: a Lambertian base under a dielectric interface.
//  * lambertian_interface_shader.cu:51-173 (smooth interface): the light sample's estimate carries the
//    interface's Fresnel transmittance in (T_01_i) and out (T_01_l) and the base's internal reflection
//    1 / (1 - rho r_10); its shadow ray (over [scene_epsilon, dist]) goes to the shadow queue.  With
//    probability 1 - R_i the path enters the base (cosine-weighted about the shading normal, weight
//    rho n^2 T_01_r / (1 - rho r_10)), otherwise it is mirrored about the shading normal with emission on.
//  * rough_diffuse_shader.cu:55-292 (rough interface): rough_diffuse_vertex, shadow ray inline.
// Neither is differentiable (pt_render_adjoint rejects them); the adjoint variant only settles the
// pending gradient of the previous vertex and replays the path.
template <bool kAdj>
__global__ void __launch_bounds__(kBlock) k_shade_layered(WfDev w)
{
  __shared__ uint32_t sm[kWarps + 1];
  const uint32_t n = w.cnt[CNT_Q_LAYERED];
  const uint32_t* q = w.q_mat + (size_t)QC_LAYERED * w.cap;
  uint32_t clamped = 0, overflow = 0, capped_total = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    const uint32_t i = base + threadIdx.x;
    bool shadow = false, cont = false;
    uint32_t pid = 0;
    float3 hit_pos, w_l, sh_contrib;
    float sh_tmax = 0.0f, eps = 0.0f;
    if (i < n) {
      pid = q[i];
      const SceneDev& S = scene_of(w, pid);
      if constexpr (kAdj) apply_pending(S, w, pid);
      eps = S.integ.scene_epsilon;
      const uint4 rg = w.rng[pid];
      const float4 h = w.hit[pid], o = w.ray_o[pid], d4 = w.ray_d[pid], t4 = w.thr[pid];
      const int depth = (int)(rg.w & META_DEPTH);
      if (depth <= S.integ.max_depth) {  // both shaders end the path at depth > max_depth
        const int prim = __float_as_int(h.w);
        const int4 info = __ldg(S.tri_info + prim);
        const MatDev& m = S.mats[info.w];
        const float3 d = ld3(d4);
        hit_pos = ld3(o) + h.x * d;
        const float3 normal = shading_normal(S, info, h.y, h.z, prim);
        const float3 ffnormal = faceforward(normal, -d, normal);
        uint32_t t = rg.x;
        bool emit = (rg.w & META_EMIT) != 0;
        if (m.type == MAT_ROUGH_DIFFUSE) {
          int capped = 0;
          cont = rough_diffuse_vertex(S, w, pid, hit_pos, d, normal, ffnormal, m, t, emit, clamped, capped);
          capped_total += capped;
        } else {
          const float3 dc = f3(m.a.x, m.a.y, m.a.z);
          const float n1_over_n2 = 1.0f / m.a.w, r_10 = m.b.x;
          const float R_i = fresnel_interface(dot(-d, ffnormal), n1_over_n2);
          const float T_01_i = 1.0f - R_i;
          const float draw = rnd_tea(t);
          uint32_t li = (uint32_t)((float)S.n_lights * draw);
          if (li >= (uint32_t)S.n_lights) { li = (uint32_t)S.n_lights - 1; ++clamped; }
          const float light_pdf = 1.0f / (float)S.n_lights;
          const LightRaw ls = S.lights[li];
          float3 radiance;
          float dist;
          eval_direct(S, hit_pos, ls, w_l, radiance, dist, t, clamped);
          radiance = radiance / light_pdf;
          const float cos_theta_l = dot(ffnormal, w_l);
          if (cos_theta_l > 0.0f) {  // :95-118
            const float T_01_l = 1.0f - fresnel_interface(cos_theta_l, n1_over_n2);
            shadow = true;
            sh_tmax = dist;
            sh_contrib = ld3(t4) * (radiance * kInvPi * cos_theta_l * dc * n1_over_n2 * n1_over_n2 * T_01_l * T_01_i / (1.0f - dc * r_10));
            emit = false;
          }
          const float xi = rnd_tea(t);
          float3 nd, wgt;
          if (xi > R_i) {  // :127-153
            nd = sample_cosine_weighted(ffnormal, t);
            const float T_01_r = 1.0f - fresnel_interface(dot(nd, ffnormal), n1_over_n2);
            wgt = dc * n1_over_n2 * n1_over_n2 * T_01_r / (1.0f - dc * r_10);
          } else {  // :154-170
            nd = reflect(d, normal);
            wgt = f3s(1.0f);
            emit = true;
          }
          const float3 nt = ld3(t4) * wgt;
          w.ray_o[pid] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, 0.0f);
          w.ray_d[pid] = make_float4(nd.x, nd.y, nd.z, 0.0f);
          w.thr[pid] = make_float4(nt.x, nt.y, nt.z, 0.0f);
          cont = true;
        }
        const uint32_t meta = push_md5_reset(w, pid, rg.w & META_KEEP, rg.y, rg.z, overflow);
        w.rng[pid] = make_uint4(t, rg.y, rg.z, meta | (uint32_t)(depth + 1) | (emit ? META_EMIT : 0u));
      }
    }
    const uint32_t s_slot = block_slot(shadow, w.cnt + CNT_SHADOW, sm);
    if (shadow) {
      w.sh_o[s_slot] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, eps);
      w.sh_d[s_slot] = make_float4(w_l.x, w_l.y, w_l.z, sh_tmax);
      w.sh_c[s_slot] = make_float4(sh_contrib.x, sh_contrib.y, sh_contrib.z, __uint_as_float(kNoTexel));
      w.sh_pid[s_slot] = pid;
    }
    const uint32_t c_slot = block_slot(cont, w.cnt + w.out_slot, sm);
    if (cont) w.q_out[c_slot] = pid;
  }
  if (clamped) atomicAdd(cnt64(w.cnt, CNT_CLAMPED), (unsigned long long)clamped);
  if (overflow) atomicAdd(cnt64(w.cnt, CNT_ERROR), (unsigned long long)overflow);
  if (capped_total) atomicAdd(cnt64(w.cnt, CNT_CAPPED), (unsigned long long)capped_total);
}

// diffuse_shader.cu:42-107.  Adjoint: an albedo texel's gradient through the next-event estimate
// (resolved with the shadow ray) and through the bounce weight albedo / p (pending).
template <bool kAdj>
__global__ void __launch_bounds__(kBlock) k_shade_diffuse(WfDev w)
{
  __shared__ uint32_t sm[kWarps + 1];
  const uint32_t n = w.cnt[CNT_Q_DIFFUSE];
  const uint32_t* q = w.q_mat + (size_t)QC_DIFFUSE * w.cap;
  uint32_t clamped = 0;
  uint32_t overflow = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    uint32_t i = base + threadIdx.x;
    bool shadow = false, cont = false;
    uint32_t pid = 0;
    float3 hit_pos, w_l, sh_contrib;
    float sh_tmax = 0.0f, eps = 0.0f;
    uint32_t texel_code = kNoTexel;
    if (i < n) {
      pid = q[i];
      const SceneDev& S = scene_of(w, pid);
      if constexpr (kAdj) apply_pending(S, w, pid);
      eps = S.integ.scene_epsilon;
      // the path's records are loaded before the depth test (every queued id has them), so that their
      // latency overlaps the scene lookup
      uint4 rg = w.rng[pid];
      float4 h = w.hit[pid], o = w.ray_o[pid], d4 = w.ray_d[pid], t4 = w.thr[pid];
      int depth = (int)(rg.w & META_DEPTH);
      if (depth <= S.integ.max_depth) {
        int prim = __float_as_int(h.w);
        int4 info = __ldg(S.tri_info + prim);
        const MatDev& m = S.mats[info.w];
        float3 d = ld3(d4);
        hit_pos = ld3(o) + h.x * d;
        float3 dc = f3(m.a.x, m.a.y, m.a.z);
        const int tid = __float_as_int(m.tmap.w);
        if (tid >= 0) {  // albedo texture (nearest texel of the cube map)
          const TexDev& T = S.tex[tid];
          const uint32_t tx = cube_texel(hit_pos, ld3(m.tmap), T.w, T.h);
          dc = f3(__ldg(T.data + 3 * tx), __ldg(T.data + 3 * tx + 1), __ldg(T.data + 3 * tx + 2));
          texel_code = ((uint32_t)tid << 24) | tx;
        }
        float3 normal = shading_normal(S, info, h.y, h.z, prim);
        float3 ffnormal = faceforward(normal, -d, normal);
        uint32_t t = rg.x;
        bool emit = (rg.w & META_EMIT) != 0;
        // uniform light pick and next-event estimation (:55-81)
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
        // Russian roulette on the mean albedo (:85-104)
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
          // weight albedo / p with p detached: d w / w = 1 / albedo per channel
          if (kAdj && texel_code != kNoTexel)
            set_pending(w, pid, PEND_ALBEDO, (uint32_t)tid, texel_code & 0xffffffu, f3(1.0f / dc.x, 1.0f / dc.y, 1.0f / dc.z));
        }
        const uint32_t meta = push_md5_reset(w, pid, rg.w & META_KEEP, rg.y, rg.z, overflow);
        w.rng[pid] = make_uint4(t, rg.y, rg.z, meta | (uint32_t)(depth + 1) | (emit ? META_EMIT : 0u));
      }
    }
    uint32_t s_slot = block_slot(shadow, w.cnt + CNT_SHADOW, sm);
    if (shadow) {
      w.sh_o[s_slot] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, eps);
      w.sh_d[s_slot] = make_float4(w_l.x, w_l.y, w_l.z, sh_tmax);
      w.sh_c[s_slot] = make_float4(sh_contrib.x, sh_contrib.y, sh_contrib.z, __uint_as_float(texel_code));
      w.sh_pid[s_slot] = pid;
    }
    uint32_t c_slot = block_slot(cont, w.cnt + w.out_slot, sm);
    if (cont) w.q_out[c_slot] = pid;
  }
  if (clamped) atomicAdd(cnt64(w.cnt, CNT_CLAMPED), (unsigned long long)clamped);
  if (overflow) atomicAdd(cnt64(w.cnt, CNT_ERROR), (unsigned long long)overflow);
}

// metallic_shader.cu:45-161.  Adjoint: a GGX roughness texel's gradient through the weight, with
// the microfacet normal's sampling detached: d ln w / d alpha = d ln D(m) + d ln G1(wi) + d ln G1(wo)
// for the Walter and the visible-normal models alike.
// kMS: some conductor of the pass uses the multiple-scattering model (else that code is left out,
// which keeps the kernel's instruction footprint small).
template <bool kAdj, bool kMS>
__global__ void __launch_bounds__(kBlock) k_shade_metal(WfDev w)
{
  __shared__ uint32_t sm[kWarps + 1];
  const uint32_t n = w.cnt[CNT_Q_METAL];
  const uint32_t* q = w.q_mat + (size_t)QC_METAL * w.cap;
  uint32_t capped_total = 0;
  uint32_t overflow = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    uint32_t i = base + threadIdx.x;
    bool cont = false;
    uint32_t pid = 0;
    if (i < n) {
      pid = q[i];
      const SceneDev& S = scene_of(w, pid);
      if constexpr (kAdj) apply_pending(S, w, pid);
      uint4 rg = w.rng[pid];
      float4 h = w.hit[pid], o = w.ray_o[pid], d4 = w.ray_d[pid];
      int depth = (int)(rg.w & META_DEPTH);
      if (depth < S.integ.max_depth) {
        int prim = __float_as_int(h.w);
        int4 info = __ldg(S.tri_info + prim);
        const MatDev& m = S.mats[info.w];
        float3 d = ld3(d4);
        float3 hit_point = ld3(o) + h.x * d;
        uint32_t rtexel = kNoTexel;
        float3 mn_used = f3s(0.0f);
        float3 normal = shading_normal(S, info, h.y, h.z, prim);
        float3 ffnormal = faceforward(normal, -d, normal);
        float3 w_i = -d;
        uint32_t seed = rg.x;
        float a_x = m.a.x, a_y = m.a.y;
        const int tid = __float_as_int(m.tmap.w);
        if (tid >= 0) {  // isotropic roughness texture (nearest texel of the cube map)
          const TexDev& T = S.tex[tid];
          rtexel = cube_texel(hit_point, ld3(m.tmap), T.w, T.h);
          a_x = a_y = __ldg(T.data + rtexel);
        }
        int capped = 0;
        float3 w_o, weight;
        bool go = true;
        if (kMS && m.model == MULTISCATTERING) {
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
            mn_used = mn;
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
          if (kAdj && rtexel != kNoTexel && m.model != MULTISCATTERING && m.dist == GGX) {
            const float dl = ggx_dlnD(mn_used, ffnormal, a_x) + ggx_dlnG1(w_i, ffnormal, a_x) + ggx_dlnG1(w_o, ffnormal, a_x);
            set_pending(w, pid, PEND_ROUGH, (uint32_t)tid, rtexel, f3s(dl));
          }
        }
        const uint32_t meta = push_md5_reset(w, pid, rg.w & META_KEEP, rg.y, rg.z, overflow);
        w.rng[pid] = make_uint4(seed, rg.y, rg.z, meta | (uint32_t)(depth + 1) | META_EMIT);
      }
    }
    uint32_t c_slot = block_slot(cont, w.cnt + w.out_slot, sm);
    if (cont) w.q_out[c_slot] = pid;
  }
  if (capped_total) atomicAdd(cnt64(w.cnt, CNT_CAPPED), (unsigned long long)capped_total);
  if (overflow) atomicAdd(cnt64(w.cnt, CNT_ERROR), (unsigned long long)overflow);
}

struct DirSeed {
  float3 dir;
  uint32_t seed;
};
// transparent_shader.cu:90-108: Fresnel reflectance about the shading normal (flipped, with the
// relative index inverted, when the ray is inside), one tea draw choosing the mirror or the refracted
// direction.
__device__ __forceinline__ DirSeed smooth_glass_dir(float3 d, float3 normal, float ior, float cos_theta, uint32_t t)
{
  const bool inside = cos_theta < 0.0f;
  const float n1_over_n2 = inside ? ior : 1.0f / ior;
  const float3 nn = inside ? -normal : normal;
  const float ci = inside ? -cos_theta : cos_theta;
  float R = 1.0f, ctt = 0.0f;
  const float st2 = n1_over_n2 * n1_over_n2 * (1.0f - ci * ci);
  if (st2 < 1.0f) {
    ctt = sqrtf(1.0f - st2);
    R = fresnel_R(ci, ctt, n1_over_n2);
  }
  const float reflect_xi = rnd_tea(t);
  DirSeed r;
  r.dir = reflect_xi < R ? reflect(d, nn) : n1_over_n2 * d + nn * (n1_over_n2 * ci - ctt);
  r.seed = t;
  return r;
}

// rough_transparent_shader.cu:66-225, and transparent_shader.cu:47-115 for smooth glass (Beer roulette
// inside, then the Fresnel choice between the mirror and the refracted direction about the shading
// normal).  No parameters to differentiate: the adjoint only settles the pending gradient of the
// previous vertex.
// kMS: some rough dielectric of the pass uses the multiple-scattering model (as for k_shade_metal).
template <bool kAdj, bool kMS>
__global__ void __launch_bounds__(kBlock) k_shade_glass(WfDev w)
{
  __shared__ uint32_t sm[kWarps + 1];
  const uint32_t n = w.cnt[CNT_Q_GLASS];
  const uint32_t* q = w.q_mat + (size_t)QC_GLASS * w.cap;
  uint32_t capped_total = 0;
  uint32_t overflow = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    uint32_t i = base + threadIdx.x;
    bool cont = false;
    uint32_t pid = 0;
    if (i < n) {
      pid = q[i];
      const SceneDev& S = scene_of(w, pid);
      if constexpr (kAdj) apply_pending(S, w, pid);
      uint4 rg = w.rng[pid];
      float4 h = w.hit[pid], o = w.ray_o[pid], d4 = w.ray_d[pid];
      int depth = (int)(rg.w & META_DEPTH);
      // rough_transparent_shader.cu:68 ends paths at depth >= max_depth, transparent_shader.cu:50 at depth > max_depth
      if (depth < S.integ.max_depth ||
          (depth == S.integ.max_depth && S.mats[__ldg(&S.tri_info[__float_as_int(h.w)].w)].type == MAT_TRANSPARENT)) {
        int prim = __float_as_int(h.w);
        int4 info = __ldg(S.tri_info + prim);
        const MatDev& m = S.mats[info.w];
        const bool smooth = m.type == MAT_TRANSPARENT;
        const float ior = m.a.x, rough = m.a.y;
        float3 d = ld3(d4);
        float3 hit_point = ld3(o) + h.x * d;
        float3 normal = shading_normal(S, info, h.y, h.z, prim);
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
        if (go && smooth) {
          const DirSeed ds = smooth_glass_dir(d, normal, ior, cos_theta, t);
          w_o = ds.dir;
          t = ds.seed;
        } else if (go) {
          float z1 = rnd_tea(t), z2 = rnd_tea(t);
          if (kMS && m.model == MULTISCATTERING) {  // :100-120
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
        const uint32_t meta = smooth ? (rg.w & META_KEEP) : push_md5_reset(w, pid, rg.w & META_KEEP, rg.y, rg.z, overflow);
        w.rng[pid] = make_uint4(t, rg.y, rg.z, meta | (uint32_t)(depth + 1) | META_EMIT);
      }
    }
    uint32_t c_slot = block_slot(cont, w.cnt + w.out_slot, sm);
    if (cont) w.q_out[c_slot] = pid;
  }
  if (capped_total) atomicAdd(cnt64(w.cnt, CNT_CAPPED), (unsigned long long)capped_total);
  if (overflow) atomicAdd(cnt64(w.cnt, CNT_ERROR), (unsigned long long)overflow);
}

// ------------------------------------------------------------------ translucent objects
// rough_subsurface_scattering_shader.cu:56-455 (REFLECT, TRANSMIT, DIRECTLIGHT and RND_64 defined),
// one vertex: the microfacet normal from two MD5 draws; a light picked with an MD5 draw and its
// reflection-only estimate (the multiscatter model: the multiscatter dielectric BSDF), with the shadow
// ray traced here because the multiscatter evaluation draws tea randoms only when the light is
// visible; then the smooth shader's Beer roulette and Fresnel choice on the microfacet normal, the
// refraction / reflection weight on the child, and on a refraction from outside the dipole gather
// (pushed with that weight; its draws must also exceed 0.001).  Returns whether the path continues.
__device__ bool rough_translucent_vertex(const SceneDev& S, const WfDev& w, uint32_t pid, const uint4& rg, int depth, const float4& h,
                                         const float4& o, const float4& d4, const int4& info, const MatDev& m, const ScatDev& P,
                                         uint32_t& overflow, uint32_t& clamped, int& capped)
{
  const float3 d = ld3(d4);
  float3 normal = shading_normal(S, info, h.y, h.z, __float_as_int(h.w));
  const float3 ffnormal = faceforward(normal, -d, normal);
  const float3 hit_pos = ld3(o) + h.x * d;
  const float3 w_i = -d;
  float recip_ior = 1.0f / P.relative_ior;
  float3 beam_T = f3s(1.0f);
  uint32_t t = rg.x;
  uint2 t64 = make_uint2(rg.y, rg.z);
  const float reflect_xi = rnd_md5(t64);
  const float z1 = rnd_md5(t64);
  const float z2 = rnd_md5(t64);
  const float a_x = m.a.y, a_y = m.a.z;
  const uint32_t model = __float_as_uint(m.a.w), dist = m.dist;
  const float3 mn = model == WALTER ? sample_normal(dist, ffnormal, z1, z2, a_x) : sample_visible_normal(dist, w_i, ffnormal, a_x, a_y, z1, z2, &capped);
  const float cos_theta_i = dot(w_i, mn);
  const bool inside = dot(w_i, normal) < 0.0f;
  bool emit = (rg.w & META_EMIT) != 0;
  const float4 t4 = w.thr[pid];
  // light sample (:93-152)
  uint32_t li = (uint32_t)((float)S.n_lights * rnd_md5(t64));
  if (li >= (uint32_t)S.n_lights) { li = (uint32_t)S.n_lights - 1; ++clamped; }
  const float light_pdf = 1.0f / (float)S.n_lights;
  const LightRaw ls = S.lights[li];
  float3 w_l, light_radiance;
  float ldist;
  eval_direct(S, hit_pos, ls, w_l, light_radiance, ldist, t, clamped);
  light_radiance = light_radiance / light_pdf;
  const float cos_l = dot(ffnormal, w_l);
  if (!inside && cos_l > 0.0f) {
    const float V = scene_any(S, hit_pos, w_l, S.integ.scene_epsilon, ldist) ? 0.0f : 1.0f;
    if (V > 0.0f) {
      const float3 Li = V * light_radiance;
      float3 add;
      if (model == MULTISCATTERING) {
        const float brdf = ms_dielectric_eval(dist, to_local(w_i, ffnormal), to_local(w_l, ffnormal), recip_ior, a_x, a_y, t, 0u, &capped);
        add = Li * brdf;
        emit = false;
      } else {
        const float3 rn = normalize(w_i + w_l);
        const float cr = dot(rn, w_l);
        float Rr = 1.0f;
        const float st2 = recip_ior * recip_ior * (1.0f - cr * cr);
        if (st2 < 1.0f) Rr = fresnel_R(cr, sqrtf(1.0f - st2), recip_ior);
        const float Gi = masking_G1_aniso(dist, w_i, rn, ffnormal, a_x, a_y);
        const float Go = masking_G1_aniso(dist, w_l, rn, ffnormal, a_x, a_y);
        const float D = eval_visible_normal(dist, w_i, rn, ffnormal, a_x, a_y);
        const float wr = Gi * Go * D / (4.0f * fabsf(dot(w_i, ffnormal) * dot(w_l, ffnormal)));
        add = Li * Rr * wr;
        emit = true;
      }
      const float4 r = w.rad[pid];
      w.rad[pid] = make_float4(r.x + t4.x * add.x, r.y + t4.y * add.y, r.z + t4.z * add.z, 0.0f);
    }
  }
  uint32_t meta = rg.w & META_KEEP;
  bool cont = false, gather = false, child_emit = true;
  float3 nd = f3s(0.0f), weight = f3s(1.0f);
  auto roulette_inside = [&]() -> bool {  // Beer transmittance inside, as the smooth shader
    const float3 ext = m.model == DIRECTIONAL_DIPOLE ? P.deltaEddExtinction : P.extinction;
    beam_T = expf3((-h.x) * ext);
    const float prob = (beam_T.x + beam_T.y + beam_T.z) / 3.0f;
    if (rnd_md5(t64) >= prob) return false;
    beam_T = beam_T / prob;
    recip_ior = P.relative_ior;
    normal = -normal;
    return true;
  };
  if (model == WALTER || model == VISIBLE_NORMALS) {
    if (!inside || roulette_inside()) {
      const float st2 = recip_ior * recip_ior * (1.0f - cos_theta_i * cos_theta_i);
      float cos_t = 1.0f, R = 1.0f;
      if (st2 < 1.0f) {
        cos_t = sqrtf(1.0f - st2);
        R = fresnel_R(cos_theta_i, cos_t, recip_ior);
      }
      if (reflect_xi >= R) {
        nd = recip_ior * (cos_theta_i * mn - w_i) - mn * cos_t;
        gather = !inside;
      } else {
        nd = 2.0f * cos_theta_i * mn - w_i;
        child_emit = emit;
      }
      if (model == WALTER) {
        const float G_i_m = masking_G1(dist, w_i, mn, ffnormal, a_x);
        const float abs_i_m = fabsf(dot(w_i, mn)), abs_i_n = fabsf(dot(w_i, ffnormal)), abs_n_m = fabsf(dot(ffnormal, mn));
        const float G_o_m = masking_G1(dist, nd, mn, ffnormal, a_x);
        weight = f3s(1.0f) * (abs_i_m * G_i_m * G_o_m / (abs_i_n * abs_n_m));
      } else {
        weight = f3s(1.0f) * masking_G1_aniso(dist, nd, mn, ffnormal, a_x, a_y);
      }
      cont = true;
    }
  } else {  // MULTISCATTERING_MODEL (:287-452)
    uint32_t order = 0;
    const float3 w_o = to_world(ms_dielectric_sample(dist, to_local(w_i, normal), 1.0f / P.relative_ior, a_x, a_y, t, order, &capped), normal);
    const bool is_refraction = dot(w_o, ffnormal) < 0.0f;
    if (!inside || roulette_inside()) {
      nd = w_o;
      gather = is_refraction && !inside;
      cont = true;
    }
  }
  if (cont) {
    if (gather && !(rg.w & META_PROBE)) {
      const uint32_t slot = meta >> META_GSHIFT;
      if (slot < w.g_slots) {
        size_t at = (size_t)slot * w.cap + pid;
        w.g_a[at] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, t4.x);
        w.g_b[at] = make_float4(normal.x, normal.y, normal.z, t4.y);
        w.g_c[at] = make_float2(t4.z, __int_as_float(info.w));
        w.g_d[at] = make_float4(weight.x, weight.y, weight.z, 1.0f);
        meta += 1u << META_GSHIFT;
      } else {
        ++overflow;
      }
    }
    const float3 nt = ld3(t4) * weight * beam_T;
    w.ray_o[pid] = make_float4(hit_pos.x, hit_pos.y, hit_pos.z, 0.0f);
    w.ray_d[pid] = make_float4(nd.x, nd.y, nd.z, 0.0f);
    w.thr[pid] = make_float4(nt.x, nt.y, nt.z, 0.0f);
  }
  w.rng[pid] = make_uint4(t, t64.x, t64.y, meta | (uint32_t)(depth + 1) | (child_emit ? META_EMIT : 0u));
  return cont;
}

// subsurface_scattering_shader.cu:55-201 with REFLECT, TRANSMIT and RND_64 defined: the Fresnel
// choice between the reflected and the refracted ray (one MD5 draw), and inside the object Beer
// transmittance over the segment with Russian roulette on its mean (extinction, or the
// delta-Eddington extinction for the directional dipole).  A camera path refracted into the object
// from outside also owes the dipole gather over the frame's probes (:126-173).  The reference
// evaluates it after the refracted subtree has returned, so its MD5 draws follow every draw of that
// subtree; the vertex (position, normal, throughput, material) is therefore pushed on the path's
// gather stack and evaluated in last-in first-out order when the path has ended (k_gather).  A
// probe's indirect path does not gather: in the reference it would read the probe buffer that its
// own launch is writing.
//
// Adjoint: the gather a camera path owes at an entry vertex is taken off R there (its forward value
// was stored with the path); its gradient is added at the end (k_gather_adj).  Inside, the weight
// beam_T / p has p detached: d w / d sigma_a / w = -t * scale per channel.
template <bool kAdj>
__global__ void __launch_bounds__(kBlock) k_shade_translucent(WfDev w)
{
  __shared__ uint32_t sm[kWarps + 1];
  const uint32_t n = w.cnt[CNT_Q_TRANS];
  const uint32_t* q = w.q_mat + (size_t)QC_TRANS * w.cap;
  uint32_t overflow = 0, clamped = 0;
  int capped = 0;
  for (uint32_t base = blockIdx.x * kBlock; base < n; base += gridDim.x * kBlock) {
    uint32_t i = base + threadIdx.x;
    bool cont = false;
    uint32_t pid = 0;
    if (i < n) {
      pid = q[i];
      const SceneDev& S = scene_of(w, pid);
      if constexpr (kAdj) apply_pending(S, w, pid);
      uint4 rg = w.rng[pid];
      float4 h = w.hit[pid], o = w.ray_o[pid], d4 = w.ray_d[pid];
      int depth = (int)(rg.w & META_DEPTH);
      if (depth <= S.integ.max_depth) {
        int prim = __float_as_int(h.w);
        int4 info = __ldg(S.tri_info + prim);
        const MatDev& m = S.mats[info.w];
        const ScatDev& P = S.scat[info.w];
        if (m.type == MAT_ROUGH_TRANSLUCENT) {
          cont = rough_translucent_vertex(S, w, pid, rg, depth, h, o, d4, info, m, P, overflow, clamped, capped);
        } else {
        float3 d = ld3(d4);
        float3 no = shading_normal(S, info, h.y, h.z, prim);
        float3 xo = ld3(o) + h.x * d;
        float3 wo = -d;
        float recip_ior = 1.0f / P.relative_ior;
        float3 beam_T = f3s(1.0f);
        uint2 t64 = make_uint2(rg.y, rg.z);
        float reflect_xi = rnd_md5(t64);
        float cos_o = dot(wo, no);
        bool inside = cos_o < 0.0f;
        bool alive = true;
        if (inside) {
          float3 ext = m.model == DIRECTIONAL_DIPOLE ? P.deltaEddExtinction : P.extinction;
          beam_T = expf3((-h.x) * ext);
          float prob = (beam_T.x + beam_T.y + beam_T.z) / 3.0f;
          if (rnd_md5(t64) >= prob) {
            alive = false;
          } else {
            beam_T = beam_T / prob;
            recip_ior = P.relative_ior;
            no = -no;
            cos_o = -cos_o;
          }
        }
        uint32_t meta = rg.w & META_KEEP;
        if (alive) {
          float st2 = recip_ior * recip_ior * (1.0f - cos_o * cos_o);
          float cos_t = 1.0f, R = 1.0f;
          if (st2 < 1.0f) {
            cos_t = sqrtf(1.0f - st2);
            R = fresnel_R(cos_o, cos_t, recip_ior);
          }
          float4 t4 = w.thr[pid];
          float3 nd;
          if (reflect_xi >= R) {
            nd = recip_ior * (cos_o * no - wo) - no * cos_t;
            if (!inside && !(rg.w & META_PROBE)) {
              uint32_t slot = meta >> META_GSHIFT;
              if (slot < w.g_slots) {
                size_t at = (size_t)slot * w.cap + pid;
                w.g_a[at] = make_float4(xo.x, xo.y, xo.z, t4.x);
                w.g_b[at] = make_float4(no.x, no.y, no.z, t4.y);
                w.g_c[at] = make_float2(t4.z, __int_as_float(info.w));
                w.g_d[at] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
                if constexpr (kAdj) {
                  const ItemDev& it = w.items[w.path_item[pid]];
                  const uint64_t local = pid - it.path_begin;
                  const uint64_t gp = (uint64_t)(it.first_frame + (uint32_t)(local / it.pixels) - S.adj_first) * it.pixels + local % it.pixels;
                  const float4 G = S.adj_G[gp * S.adj_slots + slot];
                  const float4 r = w.rad[pid];
                  w.rad[pid] = make_float4(r.x - t4.x * G.x, r.y - t4.y * G.y, r.z - t4.z * G.z, 0.0f);
                }
                meta += 1u << META_GSHIFT;
              } else {
                ++overflow;
              }
            }
          } else {
            nd = 2.0f * cos_o * no - wo;
          }
          float3 nt = ld3(t4) * beam_T;
          w.ray_o[pid] = make_float4(xo.x, xo.y, xo.z, 0.0f);
          w.ray_d[pid] = make_float4(nd.x, nd.y, nd.z, 0.0f);
          w.thr[pid] = make_float4(nt.x, nt.y, nt.z, 0.0f);
          cont = true;
          if (kAdj && inside) set_pending(w, pid, PEND_SIGMA, (uint32_t)info.w, 0u, f3s(-h.x * m.a.x));
        }
        w.rng[pid] = make_uint4(rg.x, t64.x, t64.y, meta | (uint32_t)(depth + 1) | META_EMIT);
        }
      }
    }
    uint32_t c_slot = block_slot(cont, w.cnt + w.out_slot, sm);
    if (cont) w.q_out[c_slot] = pid;
  }
  if (overflow) atomicAdd(cnt64(w.cnt, CNT_ERROR), (unsigned long long)overflow);
  if (clamped) atomicAdd(cnt64(w.cnt, CNT_CLAMPED), (unsigned long long)clamped);
  if (capped) atomicAdd(cnt64(w.cnt, CNT_CAPPED), (unsigned long long)capped);
}

// Paths with pending dipole gathers, appended to `out` (warp-aggregated).
__global__ void __launch_bounds__(kBlock) k_gather_collect(WfDev w, uint64_t n_paths, uint32_t* out)
{
  for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < n_paths; base += (uint64_t)gridDim.x * kBlock) {
    uint64_t pid = base + threadIdx.x;
    bool want = pid < n_paths && (w.rng[pid].w >> META_GSHIFT) != 0;
    unsigned m = __ballot_sync(0xffffffffu, want);
    if (m) {
      int leader = __ffs(m) - 1;
      uint32_t b = 0;
      if ((int)(threadIdx.x & 31) == leader) b = atomicAdd(w.cnt + CNT_GATHER, (uint32_t)__popc(m));
      b = __shfl_sync(0xffffffffu, b, leader);
      if (want) out[b + __popc(m & lanemask_lt())] = (uint32_t)pid;
    }
  }
}

// The dipole gathers of subsurface_scattering_shader.cu:126-173, evaluated for each path in the
// reverse order of their vertices (the post-order of the reference's recursion).  Per probe with
// L != 0 of the path's frame and object: distance Russian roulette with p = exp(-dist * min sigma_tr)
// on one MD5 draw, and on acceptance T12 * L * S(probe, xo) / p with the standard or directional
// dipole.  The sum times global_coeff / samples is added to the path's radiance, weighted by the
// throughput at the vertex.  One thread per path: the MD5 stream is one sequential chain.
//
// A differentiable forward render also stores each gather's value with the path (adj_G); the adjoint
// replays the same gathers in k_gather_adjoint.
__global__ void __launch_bounds__(kBlock) k_gather(WfDev w, SssDev g, const uint32_t* list)
{
  const uint32_t n = w.cnt[CNT_GATHER];
  unsigned long long pairs = 0, gathers = 0;
  for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
    uint32_t pid = list[i];
    const ItemDev& it = w.items[w.path_item[pid]];
    const SceneDev& S = w.scenes[it.scene];
    uint4 rg = w.rng[pid];
    uint2 t64 = make_uint2(rg.y, rg.z);
    uint32_t fl = (uint32_t)((pid - it.path_begin) / it.pixels);
    float4 r4 = w.rad[pid];
    float3 L = ld3(r4);
    const uint64_t gp = S.adj_G ? (uint64_t)(it.first_frame + fl - S.adj_first) * it.pixels + (pid - it.path_begin) % it.pixels : 0;
    for (int slot = (int)(rg.w >> META_GSHIFT) - 1; slot >= 0; --slot) {
      size_t at = (size_t)slot * w.cap + pid;
      float4 a = w.g_a[at], b = w.g_b[at];
      float2 c = w.g_c[at];
      const int mat = __float_as_int(c.y);
      if (mat < 0) {  // reset marker: the MD5 state the vertex below was entered with
        t64 = make_uint2(__float_as_uint(a.x), __float_as_uint(a.y));
        continue;
      }
      const float3 xo = ld3(a), no = ld3(b), thr = f3(a.w, b.w, c.x);
      const float4 gd = w.g_d[at];
      const bool rough = gd.w != 0.0f;  // rough boundary: draws must exceed 0.001, terms carry the weight
      const float3 gw = ld3(gd);
      const MatDev& m = S.mats[mat];
      const ScatDev& P = S.scat[mat];
      const uint32_t set_in_item = fl * S.n_trans + m.aux;
      const size_t pb = it.probe_begin + (size_t)set_in_item * S.probe_samples;
      const uint32_t nc = g.pc_cnt[it.set_begin + set_in_item];
      const float chosen = fminf(P.transport.x, fminf(P.transport.y, P.transport.z));
      float3 acc = f3s(0.0f);
      if (m.model == DIRECTIONAL_DIPOLE) {
        for (uint32_t k = 0; k < nc; ++k) {
          float3 pos = ld3(__ldg(g.pc_pos + pb + k));
          float dist = length(xo - pos);
          float exp_term = expf(-dist * chosen);
          const float rn = rnd_md5(t64);
          if (rn < exp_term && (!rough || rn > 0.001f)) {
            float3 wl = ld3(__ldg(g.pc_wl + pb + k));
            float3 pn = ld3(__ldg(g.pc_nrm + pb + k)), pt = ld3(__ldg(g.pc_tr + pb + k));
            float3 term = wl * dirpole_bssrdf(pos, pn, pt, xo, no, P) / exp_term;
            acc = acc + (rough ? term * gw : term);
          }
        }
      } else {
        const StdDipole sd = std_dipole_terms(P);
        for (uint32_t k = 0; k < nc; ++k) {
          float3 pos = ld3(__ldg(g.pc_pos + pb + k));
          float dist = length(xo - pos);
          float exp_term = expf(-dist * chosen);
          const float rn = rnd_md5(t64);
          if (rn < exp_term && (!rough || rn > 0.001f)) {
            float3 wl = ld3(__ldg(g.pc_wl + pb + k));
            float3 term = wl * dipole_bssrdf(dist, sd) / exp_term;
            acc = acc + (rough ? term * gw : term);
          }
        }
      }
      const float3 contrib = acc * P.global_coeff / (float)S.probe_samples;
      L = L + thr * contrib;
      if (S.adj_G) S.adj_G[gp * S.adj_slots + slot] = make_float4(contrib.x, contrib.y, contrib.z, 0.0f);
      pairs += nc;
      ++gathers;
    }
    w.rad[pid] = make_float4(L.x, L.y, L.z, r4.w);
    w.rng[pid] = make_uint4(rg.x, t64.x, t64.y, rg.w);
  }
  if (pairs) atomicAdd(cnt64(w.cnt, CNT_PAIRS), pairs);
  if (gathers) atomicAdd(cnt64(w.cnt, CNT_GATHERS), gathers);
}

// The adjoint gathers, warp by warp: lanes walk their paths' gathers and probes (one probe or one gather
// set-up per step: distance, the detached acceptance test on one MD5 draw -- the same chain as the
// forward gather), and every accepted pair of a differentiated material goes to the warp's queue in
// shared memory; whenever 32 pairs are queued, the whole warp evaluates them, one pair per lane, the
// standard dipole's derivatives with respect to sigma_a and sigma_s' per channel (dipole_channel_grad)
// times the pair's weight * L / p and its gather's factor (image gradient x throughput x global_coeff /
// samples), and adds them to the material's gradient buffer (one warp reduction and six atomics when
// the 32 pairs share a material).  The derivative, the costly part, thus runs on full warps instead of
// on the lanes that happened to accept a pair.
struct AdjPair {
  float dist, p;    // distance to the probe, acceptance probability exp_term
  uint32_t wl;      // index of the probe's weight * L in pc_wl
  uint32_t scene;   // the pair's scene in the pass
  float3 f;         // factor of its gather
  int mat;
};
constexpr int kAdjQueue = 64;  // per warp; at most 31 + 32 entries are held

__device__ __forceinline__ void adj_pairs_eval(const WfDev& w, const SssDev& g, const AdjPair* q, int count, int lane)
{
  float3 ga = f3s(0.0f), gs = f3s(0.0f);
  float* gr = nullptr;
  if (lane < count) {
    const AdjPair e = q[lane];
    const SceneDev& S = w.scenes[e.scene];
    const ScatDev& P = S.scat[e.mat];
    const float scale = S.mats[e.mat].a.x;
    gr = S.mat_grad[e.mat];
    const float3 wl = ld3(__ldg(g.pc_wl + e.wl));
    const Dual2 sx = dipole_channel_grad(e.dist, P.absorption.x, P.reducedExtinction.x, P.A.x, scale);
    const Dual2 sy = dipole_channel_grad(e.dist, P.absorption.y, P.reducedExtinction.y, P.A.y, scale);
    const Dual2 sz = dipole_channel_grad(e.dist, P.absorption.z, P.reducedExtinction.z, P.A.z, scale);
    const float3 k = e.f * wl / e.p;
    ga = k * f3(sx.da, sy.da, sz.da);
    gs = k * f3(sx.ds, sy.ds, sz.ds);
  }
  const unsigned long long g0 = __shfl_sync(0xffffffffu, (unsigned long long)gr, 0);
  if (__all_sync(0xffffffffu, lane >= count || (unsigned long long)gr == g0)) {
    float v[6] = {ga.x, ga.y, ga.z, gs.x, gs.y, gs.z};
#pragma unroll
    for (int j = 0; j < 6; ++j)
      for (int off = 16; off; off >>= 1) v[j] += __shfl_xor_sync(0xffffffffu, v[j], off);
    if (lane == 0 && g0) {
      float* d = (float*)g0;
#pragma unroll
      for (int j = 0; j < 6; ++j) atomicAdd(d + j, v[j]);
    }
  } else if (gr) {
    atomicAdd(gr + 0, ga.x);
    atomicAdd(gr + 1, ga.y);
    atomicAdd(gr + 2, ga.z);
    atomicAdd(gr + 3, gs.x);
    atomicAdd(gr + 4, gs.y);
    atomicAdd(gr + 5, gs.z);
  }
}

__global__ void __launch_bounds__(kBlock) k_gather_adjoint(WfDev w, SssDev g, const uint32_t* list)
{
  __shared__ AdjPair queue[kWarps][kAdjQueue];
  const uint32_t n = w.cnt[CNT_GATHER];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  AdjPair* q = queue[wid];
  int qn = 0;  // warp-uniform
  unsigned long long pairs = 0, gathers = 0;
  for (uint32_t base = (blockIdx.x * kWarps + wid) * 32u; base < n; base += gridDim.x * kBlock) {
    const uint32_t i = base + lane;
    bool active = i < n;
    uint32_t pid = 0, scene = 0, fl = 0, pb = 0, nc = 0, k = 0;
    int slot = -1, mat = 0;
    const ItemDev* it = nullptr;
    const SceneDev* S = nullptr;
    uint4 rg = make_uint4(0, 0, 0, 0);
    uint2 t64 = make_uint2(0, 0);
    float3 dl = f3s(0.0f), xo = f3s(0.0f), f = f3s(0.0f);
    float chosen = 0.0f;
    bool diff = false;
    if (active) {
      pid = list[i];
      it = &w.items[w.path_item[pid]];
      scene = it->scene;
      S = &w.scenes[scene];
      rg = w.rng[pid];
      t64 = make_uint2(rg.y, rg.z);
      fl = (uint32_t)((pid - it->path_begin) / it->pixels);
      dl = ld3(w.adj_a[pid]);
      slot = (int)(rg.w >> META_GSHIFT) - 1;
    }
    while (__any_sync(0xffffffffu, active)) {
      bool want = false;
      AdjPair e;
      if (active) {
        if (k >= nc) {  // the next gather of the path (or its end)
          if (slot < 0) {
            w.rng[pid] = make_uint4(rg.x, t64.x, t64.y, rg.w);
            active = false;
          } else {
            const size_t at = (size_t)slot * w.cap + pid;
            const float4 a = w.g_a[at], b = w.g_b[at];
            const float2 c = w.g_c[at];
            --slot;
            mat = __float_as_int(c.y);
            if (mat < 0) {  // reset marker: the MD5 state the vertex below was entered with
              t64 = make_uint2(__float_as_uint(a.x), __float_as_uint(a.y));
            } else {
              xo = ld3(a);
              const float3 thr = f3(a.w, b.w, c.x);
              const MatDev& m = S->mats[mat];
              const ScatDev& P = S->scat[mat];
              const uint32_t set_in_item = fl * S->n_trans + m.aux;
              pb = (uint32_t)(it->probe_begin + (size_t)set_in_item * S->probe_samples);
              nc = g.pc_cnt[it->set_begin + set_in_item];
              k = 0;
              chosen = fminf(P.transport.x, fminf(P.transport.y, P.transport.z));
              f = dl * thr * P.global_coeff / (float)S->probe_samples;
              diff = S->mat_grad[mat] != nullptr;
              pairs += nc;
              ++gathers;
            }
          }
        } else {  // one probe of the gather
          const float3 pos = ld3(__ldg(g.pc_pos + pb + k));
          const float dist = length(xo - pos);
          const float exp_term = expf(-dist * chosen);
          if (rnd_md5(t64) < exp_term && diff) {
            want = true;
            e.dist = dist;
            e.p = exp_term;
            e.wl = pb + k;
            e.scene = scene;
            e.f = f;
            e.mat = mat;
          }
          ++k;
        }
      }
      const unsigned m = __ballot_sync(0xffffffffu, want);
      if (want) q[qn + __popc(m & lanemask_lt())] = e;
      qn += __popc(m);
      __syncwarp();
      if (qn >= 32) {
        adj_pairs_eval(w, g, q, 32, lane);
        __syncwarp();
        const int rest = qn - 32;
        AdjPair moved;
        if (lane < rest) moved = q[32 + lane];
        __syncwarp();
        if (lane < rest) q[lane] = moved;
        qn = rest;
        __syncwarp();
      }
    }
  }
  if (qn > 0) adj_pairs_eval(w, g, q, qn, lane);
  if (pairs) atomicAdd(cnt64(w.cnt, CNT_PAIRS), pairs);
  if (gathers) atomicAdd(cnt64(w.cnt, CNT_GATHERS), gathers);
}

// sample_camera.cu:48-268 for a smooth translucent object, with GLOBAL and RND_64 defined: probe j of
// the group (frame-major, then object, then sample; path id j - j0).  The triangle is picked with an
// MD5 draw, the point uniformly on it, and with probability 1/2 (one LCG draw) the probe is lit by a
// light sample with a shadow ray (written to the path's radiance here), else by an indirect path
// started into the wavefront from the point (depth 0, emission on).  The record keeps pos, dir (of the
// light sample), normal, transmitted direction and T12; pad = (triangles * area, indirect flag) until
// k_probe_finish forms L.
__global__ void __launch_bounds__(kBlock) k_probe_gen(WfDev w, SssDev g, uint64_t j0, uint64_t n)
{
  __shared__ uint32_t sm[kWarps + 1];
  uint32_t clamped = 0;
  for (uint64_t base = (uint64_t)blockIdx.x * kBlock; base < n; base += (uint64_t)gridDim.x * kBlock) {
    uint64_t pid = base + threadIdx.x;
    bool indirect = false;
    if (pid < n) {
      uint64_t j = j0 + pid;
      uint32_t item = find_item(w.items, w.n_items, j, [](const ItemDev& x) { return x.probe_begin; });
      const ItemDev& it = w.items[item];
      const SceneDev& S = w.scenes[it.scene];
      const uint64_t per_frame = (uint64_t)S.n_trans * S.probe_samples;
      uint32_t fl = (uint32_t)((j - it.probe_begin) / per_frame);
      uint32_t idx = (uint32_t)((j - it.probe_begin) % per_frame);  // launch_index + current_translucent_obj * samples
      uint32_t k = idx / S.probe_samples;
      uint32_t frame = it.first_frame + fl;
      uint4 ob = S.trans_objs[k];
      const uint32_t triangles = ob.z;
      const ScatDev& P = S.scat[ob.x];
      uint32_t t = tea16(idx, frame);
      uint32_t s2 = tea16(idx, frame);
      uint2 t64 = make_uint2(s2, s2);
      uint32_t tid = (uint32_t)(int)(rnd_md5(t64) * (float)triangles);
      if (tid >= triangles) { tid = triangles - 1; ++clamped; }
      const float* v = S.trans_pos + 9 * ((size_t)ob.w + tid);
      float3 v0 = f3(v[0], v[1], v[2]), v1 = f3(v[3], v[4], v[5]), v2 = f3(v[6], v[7], v[8]);
      float3 perp = cross(v1 - v0, v2 - v0);
      float area = 0.5f * length(perp);
      float xi1 = sqrtf(rnd_md5(t64));
      float xi2 = rnd_md5(t64);
      float u = 1.0f - xi1, vv = (1.0f - xi2) * xi1, ww = xi1 * xi2;
      float3 pos = u * v0 + vv * v1 + ww * v2;
      int4 info = __ldg(S.tri_info + ob.y + tid);
      float3 nrm;
      if (info.x >= 0) {
        float3 n0 = ld3(__ldg(S.normals + info.x)), n1 = ld3(__ldg(S.normals + info.y)), n2 = ld3(__ldg(S.normals + info.z));
        nrm = normalize(u * n0 + vv * n1 + ww * n2);
        nrm = normalize(nrm);
      } else {
        nrm = normalize(perp);
      }
      const float recip_ior = 1.0f / P.relative_ior;
      // rough objects: the probe's normal is a microfacet normal sampled with two MD5 draws (:130-151)
      const MatDev& om = S.mats[ob.x];
      const bool rough = om.type == MAT_ROUGH_TRANSLUCENT;
      const float r_ax = om.a.y, r_ay = om.a.z;
      const uint32_t r_model = __float_as_uint(om.a.w), r_dist = om.dist;
      float3 mnorm = nrm;
      int capped = 0;
      auto microfacet = [&](const float3& wdir) {
        const float z1 = rnd_md5(t64);
        const float z2 = rnd_md5(t64);
        mnorm = r_model == WALTER ? sample_normal(r_dist, nrm, z1, z2, r_ax) : sample_visible_normal(r_dist, wdir, nrm, r_ax, r_ay, z1, z2, &capped);
      };
      float3 Le, w_i, dir = f3s(0.0f);
      if (rnd_lcg(t) < 0.5f) {
        uint32_t li = (uint32_t)((float)S.n_lights * rnd_md5(t64));
        if (li >= (uint32_t)S.n_lights) { li = (uint32_t)S.n_lights - 1; ++clamped; }
        float light_pdf = 1.0f / (float)S.n_lights;
        LightRaw ls = S.lights[li];
        float r = 0.0f;
        eval_direct(S, pos, ls, w_i, Le, r, t, clamped);
        dir = w_i;
        if (rough) microfacet(w_i);
        float cos_i = fmaxf(dot(w_i, nrm), 0.0f);
        if (cos_i > 0.0f) {
          float att = scene_any(S, pos, w_i, S.integ.scene_epsilon, r) ? 0.0f : 1.0f;
          Le = Le * (att * cos_i / light_pdf);
        } else {
          Le = f3s(0.0f);
        }
        w.rad[pid] = make_float4(Le.x, Le.y, Le.z, 0.0f);
      } else {
        w_i = sample_cosine_weighted(nrm, t);
        if (rough) microfacet(w_i);
        w.ray_o[pid] = make_float4(pos.x, pos.y, pos.z, 0.0f);
        w.ray_d[pid] = make_float4(w_i.x, w_i.y, w_i.z, 0.0f);
        w.thr[pid] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        w.rad[pid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        w.rng[pid] = make_uint4(t, t64.x, t64.y, META_EMIT | META_PROBE);
        w.path_item[pid] = (uint16_t)item;
        indirect = true;
      }
      float cos_i = fmaxf(dot(w_i, mnorm), 0.0f);
      float cos_i2 = cos_i * cos_i;
      float st2 = recip_ior * recip_ior * (1.0f - cos_i2);
      float cos_t = sqrtf(1.0f - st2);
      float3 tr = recip_ior * (cos_i * mnorm - w_i) - mnorm * cos_t;
      float T12 = 1.0f - fresnel_R(cos_i, cos_t, recip_ior);
      float wgt = T12;  // 1 * T12
      if (rough) {  // :232-266
        if (r_model == WALTER) {
          const float G_i_m = masking_G1_aniso(r_dist, w_i, mnorm, nrm, r_ax, r_ay);
          const float abs_i_m = fabsf(dot(w_i, mnorm)), abs_i_n = fabsf(dot(w_i, nrm)), abs_n_m = fabsf(dot(nrm, mnorm));
          const float G_o_m = masking_G1_aniso(r_dist, tr, mnorm, nrm, r_ax, r_ay);
          wgt = (1.0f * (abs_i_m * G_i_m / (abs_i_n * abs_n_m) * G_o_m)) * T12;
        } else if (r_model == VISIBLE_NORMALS) {
          wgt = (1.0f * masking_G1_aniso(r_dist, tr, mnorm, nrm, r_ax, r_ay)) * T12;
        }
      }
      if (capped) atomicAdd(cnt64(w.cnt, CNT_CAPPED), 1ull);
      float4* rec = g.probes + 5 * j;
      rec[0] = make_float4(pos.x, pos.y, pos.z, dir.x);
      rec[1] = make_float4(dir.y, dir.z, mnorm.x, mnorm.y);
      rec[2] = make_float4(mnorm.z, 0.0f, 0.0f, 0.0f);
      rec[3] = make_float4(tr.x, tr.y, tr.z, wgt);
      rec[4] = make_float4(wgt, wgt, (float)triangles * area, indirect ? 1.0f : 0.0f);
    }
    uint32_t slot = block_slot(indirect, w.cnt + w.in_slot, sm);
    if (indirect) w.q_in[slot] = (uint32_t)pid;
  }
  if (clamped) atomicAdd(cnt64(w.cnt, CNT_CLAMPED), (unsigned long long)clamped);
}

// sample_camera.cu:207 and :230: Le = (light sample, or the indirect path's radiance times pi) / 0.5,
// L = Le * (triangles * area).
__global__ void __launch_bounds__(kBlock) k_probe_finish(WfDev w, SssDev g, uint64_t j0, uint64_t n)
{
  for (uint64_t pid = (uint64_t)blockIdx.x * kBlock + threadIdx.x; pid < n; pid += (uint64_t)gridDim.x * kBlock) {
    float4* rec = g.probes + 5 * (j0 + pid);
    float4 r4 = rec[4];
    float3 Le = ld3(w.rad[pid]);
    if (r4.w != 0.0f) Le = Le * kPi;
    Le = Le / 0.5f;
    float3 L = Le * r4.z;
    float4 r2 = rec[2];
    rec[2] = make_float4(r2.x, L.x, L.y, L.z);
    rec[4] = make_float4(r4.x, r4.y, 0.0f, 0.0f);
  }
}

// The probes with dot(L, L) > 0 of one (frame, object) set, compacted in order: one block per set.
__global__ void __launch_bounds__(256) k_probe_compact(WfDev w, SssDev g)
{
  __shared__ uint32_t warp_off[8];
  __shared__ uint32_t total;
  const uint32_t set = blockIdx.x;
  const ItemDev& it = w.items[find_item(w.items, w.n_items, set, [](const ItemDev& x) { return x.set_begin; })];
  const uint32_t samples = w.scenes[it.scene].probe_samples;
  const size_t b = it.probe_begin + (size_t)(set - it.set_begin) * samples;
  if (threadIdx.x == 0) total = 0;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint32_t c0 = 0; c0 < samples; c0 += 256) {
    uint32_t i = c0 + threadIdx.x;
    bool keep = false;
    float3 pos, nrm, L, tr, wt;
    if (i < samples) {
      const float4* rec = g.probes + 5 * (b + i);
      float4 r0 = rec[0], r1 = rec[1], r2 = rec[2], r3 = rec[3], r4 = rec[4];
      pos = ld3(r0);
      nrm = f3(r1.z, r1.w, r2.x);
      L = f3(r2.y, r2.z, r2.w);
      tr = ld3(r3);
      wt = f3(r3.w, r4.x, r4.y);
      keep = dot(L, L) > 0.0f;
    }
    unsigned m = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_off[warp] = __popc(m);
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t run = total;
      for (int k = 0; k < 8; ++k) {
        uint32_t cnt = warp_off[k];
        warp_off[k] = run;
        run += cnt;
      }
      total = run;
    }
    __syncthreads();
    if (keep) {
      size_t o = b + warp_off[warp] + __popc(m & lanemask_lt());
      float3 wl = wt * L;
      g.pc_pos[o] = make_float4(pos.x, pos.y, pos.z, 0.0f);
      g.pc_wl[o] = make_float4(wl.x, wl.y, wl.z, 0.0f);
      g.pc_nrm[o] = make_float4(nrm.x, nrm.y, nrm.z, 0.0f);
      g.pc_tr[o] = make_float4(tr.x, tr.y, tr.z, 0.0f);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) g.pc_cnt[set] = total;
}

// Shadow rays of diffuse_shader.cu:69-81 (every material's any-hit program is opaque).
template <bool kAdj>
__global__ void __launch_bounds__(kBlock) k_shadow(WfDev w)
{
  const uint32_t n = w.cnt[CNT_SHADOW];
  for (uint32_t i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
    float4 o = w.sh_o[i], d = w.sh_d[i];
    uint32_t pid = w.sh_pid[i];
    const SceneDev& S = scene_of(w, pid);
    if (!scene_any(S, ld3(o), ld3(d), o.w, d.w)) shadow_unoccluded<kAdj>(S, w, i);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && n) atomicAdd(cnt64(w.cnt, CNT_SHADOW_TOTAL), (unsigned long long)n);
}

// path_tracer.cu:36-43 and :64-68, frame by frame in order.
// One thread per (item, pixel): the item's frames are folded into the scene's running mean in order.
__global__ void __launch_bounds__(kBlock) k_accumulate(WfDev w, uint64_t n_pix)
{
  for (uint64_t q = (uint64_t)blockIdx.x * kBlock + threadIdx.x; q < n_pix; q += (uint64_t)gridDim.x * kBlock) {
    const ItemDev& it = w.items[find_item(w.items, w.n_items, q, [](const ItemDev& x) { return x.pix_begin; })];
    const uint32_t p = (uint32_t)(q - it.pix_begin);
    const SceneDev& S = w.scenes[it.scene];
    float4* accum = S.accum;
    float4 out = accum[p];
    for (uint32_t fl = 0; fl < it.n_frames; ++fl) {
      uint64_t pid = it.path_begin + (uint64_t)fl * it.pixels + p;
      uint32_t frame = it.first_frame + fl;
      if (S.adj_L) S.adj_L[(uint64_t)(frame - S.adj_first) * it.pixels + p] = w.rad[pid];
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

static pt_status ensure_wavefront(Wavefront& wf, uint64_t cap)
{
  if (wf.cap >= cap && wf.counters.p) return PT_OK;
  pt_status st = PT_OK;
  const size_t f4 = sizeof(float4), u4 = sizeof(uint4);
  if (st == PT_OK) st = wf.rays.reserve(cap * 2 * f4, "wavefront ray records");
  if (st == PT_OK) st = wf.state.reserve(cap * (f4 + u4), "wavefront path-state records");
  if (st == PT_OK) st = wf.rad.reserve(cap * f4, "wavefront radiance");
  if (st == PT_OK) st = wf.hit.reserve(cap * f4, "wavefront hits");
  if (st == PT_OK) st = wf.path_item.reserve(cap * 2, "wavefront path items");
  if (st == PT_OK) st = wf.q_a.reserve(cap * 4, "queue");
  if (st == PT_OK) st = wf.q_b.reserve(cap * 4, "queue");
  if (st == PT_OK) st = wf.q_mat.reserve(cap * 4 * kQueues, "material queues");
  if (st == PT_OK) st = wf.cls_of.reserve(cap, "material classes of the queue");
  if (st == PT_OK) st = wf.bin.reserve(((cap + bin_chunk(kBinItemsMin) - 1) / bin_chunk(kBinItemsMin)) * kQueues * 4, "material binning counts");
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

// Gather stacks for `cap` paths with `slots` entries each, and probe storage for `records` probes.
static pt_status ensure_sss(Context& c, uint64_t cap, uint32_t slots, uint64_t records, uint64_t sets)
{
  Wavefront& wf = c.wf;
  pt_status st = PT_OK;
  if (wf.gather_cap < cap || wf.gather_slots < slots || !wf.g_a.p) {
    const size_t n = (size_t)cap * slots;
    st = wf.g_a.reserve(n * sizeof(float4), "dipole gather stack");
    if (st == PT_OK) st = wf.g_b.reserve(n * sizeof(float4), "dipole gather stack");
    if (st == PT_OK) st = wf.g_c.reserve(n * sizeof(float2), "dipole gather stack");
    if (st == PT_OK) st = wf.g_d.reserve(n * sizeof(float4), "dipole gather stack");
    if (st != PT_OK) {
      wf.gather_cap = 0;
      wf.gather_slots = 0;
      return st;
    }
    wf.gather_cap = cap;
    wf.gather_slots = slots;
  }
  if (wf.probe_cap < records || !wf.probes.p) {
    st = wf.probes.reserve(records * 80, "probe records");
    if (st == PT_OK) st = wf.pc_pos.reserve(records * sizeof(float4), "compacted probes");
    if (st == PT_OK) st = wf.pc_wl.reserve(records * sizeof(float4), "compacted probes");
    if (st == PT_OK) st = wf.pc_nrm.reserve(records * sizeof(float4), "compacted probes");
    if (st == PT_OK) st = wf.pc_tr.reserve(records * sizeof(float4), "compacted probes");
    if (st != PT_OK) {
      wf.probe_cap = 0;
      return st;
    }
    wf.probe_cap = records;
  }
  return wf.pc_cnt.reserve(std::max<uint64_t>(sets, 1) * 4, "probe counts");
}

static int __float_as_int_host(float f)
{
  int i;
  memcpy(&i, &f, 4);
  return i;
}

// Checks a scene before it is rendered and brings its device state up to date on its own stream:
// changed materials, and the geometric normals (once per build).
pt_status prepare_scene(Context& c, const char* who)
{
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  if (!c.built) return fail(PT_NOT_READY, std::string(who) + ": call pt_build first");
  if (!c.camera_set) return fail(PT_NOT_READY, std::string(who) + ": camera not set");
  for (const LightRaw& l : c.lights)
    if (l.type == ENVMAP_LIGHT && !c.env_present) return fail(PT_NOT_READY, std::string(who) + ": an environment-map light needs pt_set_envmap");
  for (const MatDev& m : c.mats)
    if ((m.type == MAT_DIFFUSE || m.type == MAT_LAMBERTIAN_INTERFACE || m.type == MAT_ROUGH_DIFFUSE) && c.lights.empty())
      return fail(PT_NOT_READY, std::string(who) +
                                    ": diffuse materials need at least one light (light_buffer is indexed unguarded by the diffuse, "
                                    "lambertian-interface and rough-diffuse shaders)");
  const bool sss = !c.trans_objs.empty();
  if (sss && c.lights.empty())
    return fail(PT_NOT_READY, std::string(who) + ": translucent objects need at least one light (the probe pass samples light_buffer)");
  if (sss && c.integ.max_depth > 254)
    return fail(PT_CAP_EXCEEDED, std::string(who) + ": translucent objects support max_depth <= 254 (the gather stack holds 255 entries)");
  if (c.dirty_mat_grad || c.mat_grad.size() != c.mats.size()) {
    c.mat_grad.resize(c.mats.size(), nullptr);
    pt_status st = c.d_mat_grad.reserve(std::max<size_t>(c.mats.size(), 1) * sizeof(float*), "gradient table");
    if (st != PT_OK) return st;
    if (!c.mat_grad.empty())
      PT_CHECK_CUDA(cudaMemcpyAsync(c.d_mat_grad.p, c.mat_grad.data(), c.mat_grad.size() * sizeof(float*), cudaMemcpyHostToDevice, c.stream),
                    "gradient table");
    c.dirty_mat_grad = false;
  }
  if (c.dirty_textures) {
    pt_status st = c.d_tex.reserve(std::max<size_t>(c.textures.size(), 1) * sizeof(TexDev), "texture table");
    if (st != PT_OK) return st;
    if (!c.textures.empty())
      PT_CHECK_CUDA(cudaMemcpyAsync(c.d_tex.p, c.textures.data(), c.textures.size() * sizeof(TexDev), cudaMemcpyHostToDevice, c.stream),
                    "texture table");
    c.dirty_textures = false;
  }
  if (c.dirty_materials) {
    PT_CHECK_CUDA(cudaMemcpyAsync(c.d_mats.p, c.mats.data(), c.mats.size() * sizeof(MatDev), cudaMemcpyHostToDevice, c.stream), "material upload");
    PT_CHECK_CUDA(cudaMemcpyAsync(c.d_scat.p, c.scat.data(), c.scat.size() * sizeof(ScatDev), cudaMemcpyHostToDevice, c.stream),
                  "scattering properties upload");
    c.dirty_materials = false;
  }
  DevBuf& geo = c.d_normals_geo;
  if (!geo.p || geo.bytes < (size_t)c.n_tris * sizeof(float4) || c.geo_stale) {
    pt_status st = geo.reserve((size_t)c.n_tris * sizeof(float4), "geometric normals");
    if (st != PT_OK) return st;
    k_geo_normals<<<grid_for(c.n_tris, 256, 8), 256, 0, c.stream>>>(c.view(), geo.as<float4>());
    count_launch();
    c.geo_stale = false;
  }
  return PT_OK;
}

// Camera samples a render of `n_frames` frames of this scene traces (pixels inside the patch).
uint64_t scene_path_samples(const Context& c, uint32_t n_frames)
{
  uint64_t inside_w = (uint64_t)std::min<uint32_t>(c.cam.width, c.cam.patch_origin.x + c.cam.patch_dims.x + 1) -
                      std::min<uint32_t>(c.cam.width, c.cam.patch_origin.x);
  uint64_t inside_h = (uint64_t)std::min<uint32_t>(c.cam.height, c.cam.patch_origin.y + c.cam.patch_dims.y + 1) -
                      std::min<uint32_t>(c.cam.height, c.cam.patch_origin.y);
  return inside_w * inside_h * n_frames;
}

SceneFacts scene_facts(const Context& c)
{
  SceneFacts f;
  f.pixels = c.cam.width * c.cam.height;
  f.n_trans = (uint32_t)c.trans_objs.size();
  f.samples = c.probe_samples;
  f.max_depth = c.integ.max_depth;
  for (const MatDev& m : c.mats)
    if (m.type == MAT_LAMBERTIAN_INTERFACE || m.type == MAT_ROUGH_DIFFUSE) f.layered = true;
    else if ((m.type == MAT_METAL || m.type == MAT_ROUGH_GLASS) && m.model == MULTISCATTERING) f.ms = true;
  return f;
}

PassLayout plan_pass(const std::vector<SceneFacts>& facts, const std::vector<ItemReq>& reqs, uint64_t max_paths, bool dual)
{
  PassLayout L;
  uint32_t max_pixels = 1;
  for (const SceneFacts& f : facts) {
    L.passes = std::max(L.passes, f.max_depth + 2);
    L.layered = L.layered || f.layered;
    L.ms = L.ms || f.ms;
    max_pixels = std::max(max_pixels, f.pixels);
    if (f.n_trans) {
      L.sss = true;
      L.g_slots = std::max<uint32_t>(L.g_slots, (uint32_t)f.max_depth + 1);
    }
  }
  if (L.sss) max_paths = std::min<uint64_t>(max_paths, std::max<uint64_t>(max_pixels, (4ull << 30) / ((uint64_t)L.g_slots * 40)));
  if (dual && !L.sss) {
    L.dual = true;
    max_paths = std::max<uint64_t>(1, max_paths / 2);
  }
  uint64_t paths = 0, probes = 0, pix = 0;
  uint32_t sets = 0;
  auto close_chunk = [&]() {
    if (L.chunk_item_begin.size() && L.chunk_item_begin.back() == (uint32_t)L.items.size()) return;
    L.chunk_paths.push_back(paths);
    L.chunk_probes.push_back(probes);
    L.chunk_pixels.push_back(pix);
    L.chunk_sets.push_back(sets);
    L.cap_paths = std::max(L.cap_paths, paths);
    L.cap_probes = std::max(L.cap_probes, probes);
    L.cap_sets = std::max<uint64_t>(L.cap_sets, sets);
    L.chunk_item_begin.push_back((uint32_t)L.items.size());
    paths = probes = pix = 0;
    sets = 0;
  };
  L.chunk_item_begin.push_back(0);
  for (const ItemReq& r : reqs) {
    const SceneFacts& f = facts[r.scene];
    uint32_t done = 0;
    while (done < r.n_frames) {
      uint64_t room = max_paths > paths ? max_paths - paths : 0;
      uint64_t fit = room / f.pixels;
      if ((fit == 0 && paths > 0) || L.items.size() - L.chunk_item_begin.back() >= 65535) {
        close_chunk();
        continue;
      }
      uint32_t take = (uint32_t)std::min<uint64_t>(r.n_frames - done, std::max<uint64_t>(1, fit));
      ItemDev it;
      it.scene = r.scene;
      it.first_frame = r.first_frame + done;
      it.n_frames = take;
      it.pixels = f.pixels;
      it.path_begin = paths;
      it.probe_begin = probes;
      it.pix_begin = pix;
      it.set_begin = sets;
      it.pad = 0;
      L.items.push_back(it);
      paths += (uint64_t)take * f.pixels;
      probes += (uint64_t)take * f.n_trans * f.samples;
      pix += f.pixels;
      sets += take * f.n_trans;
      done += take;
    }
  }
  close_chunk();
  L.chunk_item_begin.pop_back();  // one begin per chunk
  return L;
}

// Allocates what a pass needs in the engine context E and uploads its scene and item tables (on
// E's stream).  Nothing here may run while E's stream is being captured.
pt_status pass_resources(Context& E, const PassLayout& L, const std::vector<SceneDev>& scenes)
{
  pt_status st = ensure_wavefront(E.wf, L.cap_paths);
  if (st == PT_OK && L.dual) st = ensure_wavefront(E.wf2, L.cap_paths);
  if (st == PT_OK && L.sss) st = ensure_sss(E, E.wf.cap, L.g_slots, L.cap_probes, L.cap_sets);
  if (st == PT_OK) st = E.d_scene_tab.reserve(scenes.size() * sizeof(SceneDev), "scene table");
  if (st == PT_OK) st = E.d_item_tab.reserve(std::max<size_t>(L.items.size(), 1) * sizeof(ItemDev), "item table");
  if (st != PT_OK) return st;
  E.pass_w4 = true;
  for (const SceneDev& s : scenes) E.pass_w4 = E.pass_w4 && s.nodes4 != nullptr;
  // the overlapped schedule's streams and events (created here, outside any graph capture)
  for (cudaStream_t& sd : E.side)
    if (!sd) PT_CHECK_CUDA(cudaStreamCreateWithFlags(&sd, cudaStreamNonBlocking), "side stream");
  for (cudaEvent_t* ev : {&E.ev_fork, &E.ev_join, &E.ev_shade, &E.ev_shadow})
    if (!*ev) PT_CHECK_CUDA(cudaEventCreateWithFlags(ev, cudaEventDisableTiming), "stream event");
  if (L.dual) {
    for (cudaStream_t* sd : {&E.stream2, &E.side2[0], &E.side2[1]})
      if (!*sd) PT_CHECK_CUDA(cudaStreamCreateWithFlags(sd, cudaStreamNonBlocking), "second pipeline stream");
    for (cudaEvent_t* ev : {&E.ev2_fork, &E.ev2_join, &E.ev2_shade, &E.ev2_shadow, &E.ev_start, &E.ev_acc, &E.ev_end2})
      if (!*ev) PT_CHECK_CUDA(cudaEventCreateWithFlags(ev, cudaEventDisableTiming), "stream event");
  }
  PT_CHECK_CUDA(cudaMemcpyAsync(E.d_scene_tab.p, scenes.data(), scenes.size() * sizeof(SceneDev), cudaMemcpyHostToDevice, E.stream), "scene table");
  PT_CHECK_CUDA(cudaMemcpyAsync(E.d_item_tab.p, L.items.data(), L.items.size() * sizeof(ItemDev), cudaMemcpyHostToDevice, E.stream), "item table");
  return PT_OK;
}

// Launches a planned pass on E's stream: per chunk, the probe pass (chunks with translucent objects),
// the camera paths, the deferred gathers and the accumulation.  Only kernel launches and memsets of
// device state: the whole sequence can be captured into a CUDA graph.  multi: the pass spans
// several scenes (the traversal kernels then read each ray's scene from the table; otherwise S0).
// One full wave of a grid-stride kernel: the SM count times the blocks of kBlock threads that fit on an
// SM at the kernel's register and shared-memory use (cached per kernel and thread).
template <class K> int full_wave(K kernel)
{
  static thread_local std::vector<std::pair<const void*, int>> cache;
  const void* key = reinterpret_cast<const void*>(kernel);
  for (const auto& e : cache)
    if (e.first == key) return e.second;
  int blocks = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, kBlock, 0) != cudaSuccess || blocks < 1) blocks = 8;
  const int grid = sm_count() * blocks;
  cache.emplace_back(key, grid);
  return grid;
}

pt_status launch_pass(Context& E, const PassLayout& L, const std::vector<SceneDev>& tab, bool multi_pass, bool allow_events, bool adjoint)
{
  // per chunk: a chunk whose paths all render one scene runs the single-scene kernels on that scene
  // (its record as a kernel parameter, no per-ray scene lookup), else the multi-scene kernels
  SceneDev S0 = tab[0];
  bool multi = multi_pass;
  Context& c = E;
  // the device view of one wavefront (dual passes: one per pipeline)
  auto make_w = [&](Wavefront& wf) {
    WfDev v;
    float4* rays = wf.rays.as<float4>();
    float4* state = wf.state.as<float4>();
    v.ray_o = Field2<float4>{rays};
    v.ray_d = Field2<float4>{rays + 1};
    v.thr = Field2<float4>{state};
    v.rad = wf.rad.as<float4>();
    v.rng = Field2<uint4>{reinterpret_cast<uint4*>(state + 1)};
    v.hit = wf.hit.as<float4>();
    v.q_mat = wf.q_mat.as<uint32_t>();
    v.cls_of = wf.cls_of.as<uint8_t>();
    v.bin = wf.bin.as<uint32_t>();
    v.sh_o = wf.sh_o.as<float4>();
    v.sh_d = wf.sh_d.as<float4>();
    v.sh_c = wf.sh_c.as<float4>();
    v.sh_pid = wf.sh_pid.as<uint32_t>();
    v.cnt = wf.counters.as<uint32_t>();
    v.cap = wf.cap;
    v.g_a = L.sss ? wf.g_a.as<float4>() : nullptr;
    v.g_b = L.sss ? wf.g_b.as<float4>() : nullptr;
    v.g_c = L.sss ? wf.g_c.as<float2>() : nullptr;
    v.g_d = L.sss ? wf.g_d.as<float4>() : nullptr;
    v.g_slots = L.sss ? wf.gather_slots : 0;
    v.scenes = c.d_scene_tab.as<SceneDev>();
    v.multi = multi ? 1u : 0u;
    v.scene0 = 0;
    v.path_item = wf.path_item.as<uint16_t>();
    v.adj_a = adjoint ? wf.adj_a.as<float4>() : nullptr;
    v.adj_b = adjoint ? wf.adj_b.as<float4>() : nullptr;
    return v;
  };
  const size_t n_chunks = L.chunk_paths.size();
  const bool prof = c.profile && allow_events;
  // two pipelines: chunk k runs on wavefront k % 2 with that pipeline's streams; the accumulations
  // (each chunk's frames folded into its scenes' running means) stay in chunk order
  const bool dual = L.dual && !adjoint && !prof && n_chunks >= 2 && c.stream2 && c.wf2.cap >= L.cap_paths;
  const WfDev w_of[2] = {make_w(c.wf), dual ? make_w(c.wf2) : make_w(c.wf)};
  Wavefront* const wf_of[2] = {&c.wf, dual ? &c.wf2 : &c.wf};
  WfDev w = w_of[0];
  Wavefront* wf = wf_of[0];
  c.pass_dual = dual;
  Wavefront& wf0 = c.wf;
  SssDev g;
  memset(&g, 0, sizeof(g));
  if (L.sss) {
    g.probes = wf0.probes.as<float4>();
    g.pc_pos = wf0.pc_pos.as<float4>();
    g.pc_wl = wf0.pc_wl.as<float4>();
    g.pc_nrm = wf0.pc_nrm.as<float4>();
    g.pc_tr = wf0.pc_tr.as<float4>();
    g.pc_cnt = wf0.pc_cnt.as<uint32_t>();
  }
  const int grid_trace = sm_count() * 8, grid_shade = sm_count() * 8;
  // the 4-wide BVH when every scene of the pass has one (pass_resources)
  const bool w4 = E.pass_w4;
  // persistent grids: the SM count times the resident blocks of the single- and multi-scene kernels
  int grid_persist_of[2] = {0, 0};
  auto occupancy = [&](auto ext, auto sh, int& grid) -> pt_status {
    int occ_ext = 0, occ_sh = 0;
    PT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_ext, ext, kTraceBlock, 0), "occupancy");
    PT_CHECK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_sh, sh, kTraceBlock, 0), "occupancy");
    grid = sm_count() * std::max(1, std::min(occ_ext, occ_sh));
    return PT_OK;
  };
  pt_status ost;
  if (w4) ost = occupancy(k_extend_persistent<false, true>, k_shadow_persistent<false, false, true>, grid_persist_of[0]);
  else ost = occupancy(k_extend_persistent<false, false>, k_shadow_persistent<false, false, false>, grid_persist_of[0]);
  if (ost == PT_OK && multi_pass) {
    if (w4) ost = occupancy(k_extend_persistent<true, true>, k_shadow_persistent<true, false, true>, grid_persist_of[1]);
    else ost = occupancy(k_extend_persistent<true, false>, k_shadow_persistent<true, false, false>, grid_persist_of[1]);
  }
  if (ost != PT_OK) return ost;
  int grid_persist = grid_persist_of[0];
  const int grid_bin = sm_count() * 8;
  PT_CHECK_CUDA(cudaMemsetAsync(w_of[0].cnt, 0, kCounters * 4, c.stream), "reset counters");
  if (dual) {  // the second pipeline starts after everything queued on the context stream so far
    PT_CHECK_CUDA(cudaEventRecord(c.ev_start, c.stream), "second pipeline start");
    PT_CHECK_CUDA(cudaStreamWaitEvent(c.stream2, c.ev_start, 0), "second pipeline start");
    PT_CHECK_CUDA(cudaMemsetAsync(w_of[1].cnt, 0, kCounters * 4, c.stream2), "reset counters");
  }
  c.prof_pairs = 0;
  pt_status st = PT_OK;
  // CUDA events around the launches whose device time the stats report (when profiling is on)
  auto prof_begin = [&](int kind) -> pt_status {
    if (!prof) return PT_OK;
    while (c.prof_events.size() < 2 * (size_t)(c.prof_pairs + 1)) {
      cudaEvent_t ev;
      PT_CHECK_CUDA(cudaEventCreate(&ev), "profiling event");
      c.prof_events.push_back(ev);
    }
    if (c.prof_kind.size() < (size_t)c.prof_pairs + 1) c.prof_kind.resize(c.prof_pairs + 1);
    c.prof_kind[c.prof_pairs] = kind;
    PT_CHECK_CUDA(cudaEventRecord(c.prof_events[2 * c.prof_pairs], c.stream), "profiling event");
    return PT_OK;
  };
  auto prof_end = [&]() -> pt_status {
    if (!prof) return PT_OK;
    PT_CHECK_CUDA(cudaEventRecord(c.prof_events[2 * c.prof_pairs + 1], c.stream), "profiling event");
    ++c.prof_pairs;
    return PT_OK;
  };
  // the current chunk's pipeline: its stream, side streams and events (pipeline 0: the context's)
  cudaStream_t s_main = c.stream;
  cudaEvent_t e_fork = c.ev_fork, e_join = c.ev_join, e_shade = c.ev_shade, e_shadow = c.ev_shadow;
  auto reset_queues = [&]() -> pt_status {
    w.q_in = wf->q_a.as<uint32_t>();
    w.q_out = wf->q_b.as<uint32_t>();
    w.in_slot = CNT_ACTIVE_A;
    w.out_slot = CNT_ACTIVE_B;
    PT_CHECK_CUDA(cudaMemsetAsync(w.cnt, 0, (CNT_FETCH_SH + 1) * 4, s_main), "reset queues");
    return PT_OK;
  };
  // The overlapped schedule (option "overlap", off while profiling so that the extend events time the
  // extend kernel alone).  A bounce's shading kernels work on disjoint paths and only append to the
  // next-ray and shadow-ray queues through atomics, so the smaller classes (miss, light, conductor,
  // dielectric) run on side[0] beside the diffuse, layered and translucent kernels on the context
  // stream.  The shadow rays of bounce b touch only the shadow queue, the path radiance (and, in the
  // adjoint, the adjoint state and gradients); the extend and binning of bounce b + 1 touch neither,
  // so the shadow kernel runs on side[1] beside them, and bounce b + 1's shading, which rewrites the
  // shadow queue and adds to the radiance, waits for it.  Every path's arithmetic is its own, so the
  // images do not depend on the schedule.
  const bool overlap = c.opt.overlap && !prof && c.side[0] && c.side[1] && (!dual || (c.side2[0] && c.side2[1]));
  cudaStream_t s_small = overlap ? c.side[0] : c.stream;
  cudaStream_t s_shadow = overlap ? c.side[1] : c.stream;
  auto wait_on = [&](cudaStream_t waiter, cudaStream_t from, cudaEvent_t ev) -> pt_status {
    PT_CHECK_CUDA(cudaEventRecord(ev, from), "stream fork / join");
    PT_CHECK_CUDA(cudaStreamWaitEvent(waiter, ev, 0), "stream fork / join");
    return PT_OK;
  };
  // L.passes = max_depth + 2 bounces: every path has ended by then (each shader stops at max_depth).
  auto bounces = [&](bool adj_pass) -> pt_status {
    const bool adjoint = adj_pass;
    for (int b = 0; b < L.passes; ++b) {
      PT_CHECK_CUDA(cudaMemsetAsync(w.cnt + CNT_Q_MISS, 0, (CNT_FETCH_EXT - CNT_Q_MISS + 1) * 4, s_main), "reset queues");
      PT_CHECK_CUDA(cudaMemsetAsync(w.cnt + w.out_slot, 0, 4, s_main), "reset queues");
      if ((st = prof_begin(PROF_EXTEND)) != PT_OK) return st;
      if (c.opt.extend_mode == 1) {
        if (w4) {
          if (multi) k_extend_persistent<true, true><<<grid_persist, kTraceBlock, 0, s_main>>>(S0, w, c.opt.refill);
          else k_extend_persistent<false, true><<<grid_persist, kTraceBlock, 0, s_main>>>(S0, w, c.opt.refill);
        } else {
          if (multi) k_extend_persistent<true, false><<<grid_persist, kTraceBlock, 0, s_main>>>(S0, w, c.opt.refill);
          else k_extend_persistent<false, false><<<grid_persist, kTraceBlock, 0, s_main>>>(S0, w, c.opt.refill);
        }
      } else {
        k_extend<<<grid_trace, kBlock, 0, s_main>>>(w);
      }
      if ((st = prof_end()) != PT_OK) return st;
      if (c.opt.bin_items == 4) launch_binning<4>(w, grid_bin, s_main);
      else if (c.opt.bin_items == 16) launch_binning<16>(w, grid_bin, s_main);
      else launch_binning<8>(w, grid_bin, s_main);
      count_launch(3);
      // the previous bounce's shadow rays are done before this bounce's shading refills their queue
      if (overlap && b > 0 && (st = wait_on(s_main, s_shadow, e_shadow)) != PT_OK) return st;
      PT_CHECK_CUDA(cudaMemsetAsync(w.cnt + CNT_SHADOW, 0, (CNT_FETCH_SH - CNT_SHADOW + 1) * 4, s_main), "reset queues");
      if (overlap && (st = wait_on(s_small, s_main, e_fork)) != PT_OK) return st;
      if (adjoint) {
        k_shade_diffuse<true><<<full_wave(k_shade_diffuse<true>), kBlock, 0, s_main>>>(w);
        k_shade_miss<true><<<full_wave(k_shade_miss<true>), kBlock, 0, s_small>>>(w);
        k_shade_light<true><<<full_wave(k_shade_light<true>), kBlock, 0, s_small>>>(w);
        if (L.ms) {
          k_shade_metal<true, true><<<full_wave(k_shade_metal<true, true>), kBlock, 0, s_small>>>(w);
          k_shade_glass<true, true><<<full_wave(k_shade_glass<true, true>), kBlock, 0, s_small>>>(w);
        } else {
          k_shade_metal<true, false><<<full_wave(k_shade_metal<true, false>), kBlock, 0, s_small>>>(w);
          k_shade_glass<true, false><<<full_wave(k_shade_glass<true, false>), kBlock, 0, s_small>>>(w);
        }
      } else {
        k_shade_diffuse<false><<<full_wave(k_shade_diffuse<false>), kBlock, 0, s_main>>>(w);
        k_shade_miss<false><<<full_wave(k_shade_miss<false>), kBlock, 0, s_small>>>(w);
        k_shade_light<false><<<full_wave(k_shade_light<false>), kBlock, 0, s_small>>>(w);
        if (L.ms) {
          k_shade_metal<false, true><<<full_wave(k_shade_metal<false, true>), kBlock, 0, s_small>>>(w);
          k_shade_glass<false, true><<<full_wave(k_shade_glass<false, true>), kBlock, 0, s_small>>>(w);
        } else {
          k_shade_metal<false, false><<<full_wave(k_shade_metal<false, false>), kBlock, 0, s_small>>>(w);
          k_shade_glass<false, false><<<full_wave(k_shade_glass<false, false>), kBlock, 0, s_small>>>(w);
        }
      }
      count_launch(6);
      if (L.layered) {
        if (adjoint) k_shade_layered<true><<<full_wave(k_shade_layered<true>), kBlock, 0, s_main>>>(w);
        else k_shade_layered<false><<<full_wave(k_shade_layered<false>), kBlock, 0, s_main>>>(w);
        count_launch();
      }
      if (L.sss) {
        if (adjoint) k_shade_translucent<true><<<full_wave(k_shade_translucent<true>), kBlock, 0, s_main>>>(w);
        else k_shade_translucent<false><<<full_wave(k_shade_translucent<false>), kBlock, 0, s_main>>>(w);
        count_launch();
      }
      if (overlap) {
        // join the smaller classes, then fork the shadow rays off the joined stream
        if ((st = wait_on(s_main, s_small, e_join)) != PT_OK) return st;
        if ((st = wait_on(s_shadow, s_main, e_shade)) != PT_OK) return st;
      }
      if (c.opt.extend_mode == 1) {
        if (w4) {
          if (multi && adjoint) k_shadow_persistent<true, true, true><<<grid_persist, kTraceBlock, 0, s_shadow>>>(S0, w, c.opt.refill);
          else if (multi) k_shadow_persistent<true, false, true><<<grid_persist, kTraceBlock, 0, s_shadow>>>(S0, w, c.opt.refill);
          else if (adjoint) k_shadow_persistent<false, true, true><<<grid_persist, kTraceBlock, 0, s_shadow>>>(S0, w, c.opt.refill);
          else k_shadow_persistent<false, false, true><<<grid_persist, kTraceBlock, 0, s_shadow>>>(S0, w, c.opt.refill);
        } else {
          if (multi && adjoint) k_shadow_persistent<true, true, false><<<grid_persist, kTraceBlock, 0, s_shadow>>>(S0, w, c.opt.refill);
          else if (multi) k_shadow_persistent<true, false, false><<<grid_persist, kTraceBlock, 0, s_shadow>>>(S0, w, c.opt.refill);
          else if (adjoint) k_shadow_persistent<false, true, false><<<grid_persist, kTraceBlock, 0, s_shadow>>>(S0, w, c.opt.refill);
          else k_shadow_persistent<false, false, false><<<grid_persist, kTraceBlock, 0, s_shadow>>>(S0, w, c.opt.refill);
        }
      } else {
        if (adjoint) k_shadow<true><<<grid_trace, kBlock, 0, s_shadow>>>(w);
        else k_shadow<false><<<grid_trace, kBlock, 0, s_shadow>>>(w);
      }
      count_launch();
      ++c.stats.extend_launches;
      std::swap(w.q_in, w.q_out);
      std::swap(w.in_slot, w.out_slot);
    }
    // the last bounce's shadow rays join the context stream before anything reads the radiance
    if (overlap && (st = wait_on(s_main, s_shadow, e_shadow)) != PT_OK) return st;
    return PT_OK;
  };
  const ItemDev* items = c.d_item_tab.as<ItemDev>();
  for (size_t k = 0; k < n_chunks; ++k) {
    const int pl = dual ? (int)(k & 1) : 0;
    w = w_of[pl];
    wf = wf_of[pl];
    s_main = pl ? c.stream2 : c.stream;
    s_small = overlap ? (pl ? c.side2[0] : c.side[0]) : s_main;
    s_shadow = overlap ? (pl ? c.side2[1] : c.side[1]) : s_main;
    e_fork = pl ? c.ev2_fork : c.ev_fork;
    e_join = pl ? c.ev2_join : c.ev_join;
    e_shade = pl ? c.ev2_shade : c.ev_shade;
    e_shadow = pl ? c.ev2_shadow : c.ev_shadow;
    const uint32_t ib = L.chunk_item_begin[k];
    const uint32_t ie = k + 1 < n_chunks ? L.chunk_item_begin[k + 1] : (uint32_t)L.items.size();
    w.items = items + ib;
    w.n_items = ie - ib;
    bool one_scene = true;
    for (uint32_t i = ib + 1; i < ie; ++i) one_scene = one_scene && L.items[i].scene == L.items[ib].scene;
    multi = multi_pass && !one_scene;
    w.multi = multi ? 1u : 0u;
    w.scene0 = multi ? 0u : L.items[ib].scene;
    S0 = tab[w.scene0];
    grid_persist = grid_persist_of[multi ? 1 : 0];
    const uint64_t n_paths = L.chunk_paths[k], n_probes = L.chunk_probes[k];
    if (n_probes) {
      for (uint64_t j0 = 0; j0 < n_probes; j0 += w.cap) {
        uint64_t nj = std::min<uint64_t>(w.cap, n_probes - j0);
        if ((st = reset_queues()) != PT_OK) return st;
        k_probe_gen<<<grid_for(nj, kBlock, 16), kBlock, 0, s_main>>>(w, g, j0, nj);
        count_launch();
        if ((st = bounces(false)) != PT_OK) return st;
        k_probe_finish<<<grid_for(nj, kBlock, 16), kBlock, 0, s_main>>>(w, g, j0, nj);
        count_launch();
      }
      k_probe_compact<<<L.chunk_sets[k], 256, 0, s_main>>>(w, g);
      count_launch();
    }
    if ((st = reset_queues()) != PT_OK) return st;
    if (adjoint) k_raygen<true><<<grid_for(n_paths, kBlock, 16), kBlock, 0, s_main>>>(w, n_paths);
    else k_raygen<false><<<grid_for(n_paths, kBlock, 16), kBlock, 0, s_main>>>(w, n_paths);
    count_launch();
    if ((st = bounces(adjoint)) != PT_OK) return st;
    if (n_probes) {
      PT_CHECK_CUDA(cudaMemsetAsync(w.cnt + CNT_GATHER, 0, 4, s_main), "reset gather list");
      uint32_t* list = wf->q_a.as<uint32_t>();
      k_gather_collect<<<grid_for(n_paths, kBlock, 16), kBlock, 0, s_main>>>(w, n_paths, list);
      if ((st = prof_begin(PROF_GATHER)) != PT_OK) return st;
      if (adjoint) k_gather_adjoint<<<grid_shade, kBlock, 0, s_main>>>(w, g, list);
      else k_gather<<<grid_shade, kBlock, 0, s_main>>>(w, g, list);
      if ((st = prof_end()) != PT_OK) return st;
      count_launch(2);
    }
    if (!adjoint) {
      // the running means take the chunks' frames in chunk order
      if (dual && k > 0) PT_CHECK_CUDA(cudaStreamWaitEvent(s_main, c.ev_acc, 0), "accumulation order");
      k_accumulate<<<grid_for(L.chunk_pixels[k], kBlock, 16), kBlock, 0, s_main>>>(w, L.chunk_pixels[k]);
      count_launch();
      if (dual) PT_CHECK_CUDA(cudaEventRecord(c.ev_acc, s_main), "accumulation order");
    }
  }
  if (dual) {  // the second pipeline joins the context stream
    PT_CHECK_CUDA(cudaEventRecord(c.ev_end2, c.stream2), "second pipeline join");
    PT_CHECK_CUDA(cudaStreamWaitEvent(c.stream, c.ev_end2, 0), "second pipeline join");
  }
  PT_CHECK_CUDA(cudaGetLastError(), "render launch");
  return PT_OK;
}

}  // namespace pt

using namespace pt;

extern "C" {

pt_status pt_render_frames(pt_ctx* ctx, uint32_t first_frame, uint32_t n_frames)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  Context& c = ctx->c;
  pt_status st = prepare_scene(c, "pt_render_frames");
  if (st != PT_OK) return st;
  if (n_frames == 0) return PT_OK;
  SceneFacts f = scene_facts(c);
  if (c.differentiable) {
    // keep what the adjoint needs: each path's radiance and the value of each of its gathers
    const uint64_t n = (uint64_t)n_frames * f.pixels;
    const uint32_t slots = f.n_trans ? (uint32_t)f.max_depth + 1 : 0;
    if (n * (1 + slots) * sizeof(float4) > (16ull << 30)) return fail(PT_CAP_EXCEEDED, "pt_render_frames: differentiable state above 16 GiB");
    if ((st = c.d_adj_L.reserve(n * sizeof(float4), "adjoint path radiance")) != PT_OK) return st;
    if (slots && (st = c.d_adj_G.reserve(n * slots * sizeof(float4), "adjoint gather values")) != PT_OK) return st;
    c.adj_first = first_frame;
    c.adj_frames = n_frames;
    c.adj_slots = slots;
    c.adj_valid = true;
  }
  // profiled renders time the kernels of one wavefront (the extend events are on the context stream)
  PassLayout L = plan_pass({f}, {ItemReq{0, first_frame, n_frames}}, c.max_paths, c.opt.dual && !c.differentiable && !c.profile);
  std::vector<SceneDev> scenes{c.view()};
  if ((st = pass_resources(c, L, scenes)) != PT_OK) return st;
  uint64_t launches0 = pt_kernel_launch_count();
  memset(&c.stats, 0, sizeof(c.stats));
  PT_CHECK_CUDA(cudaEventRecord(c.ev0, c.stream), "event");
  if ((st = launch_pass(c, L, scenes, false, true)) != PT_OK) return st;
  PT_CHECK_CUDA(cudaEventRecord(c.ev1, c.stream), "event");
  c.stats.path_samples = scene_path_samples(c, n_frames);
  c.stats.kernel_launches = (uint32_t)(pt_kernel_launch_count() - launches0);
  c.stats_pending = true;
  // the probe buffer of the last chunk holds the last frames of this scene
  c.probe_last_frames = L.items.empty() ? 0 : L.items.back().n_frames;
  c.next_frame = first_frame + n_frames;
  return PT_OK;
}

pt_status pt_render_adjoint(pt_ctx* ctx, uint32_t first_frame, uint32_t n_frames, const float* d_dimage)
{
  if (!ctx || !d_dimage) return fail(PT_INVALID_ARG, "pt_render_adjoint: null argument");
  Context& c = ctx->c;
  if (!c.differentiable || !c.adj_valid) return fail(PT_NOT_READY, "pt_render_adjoint: needs a forward pt_render_frames with the differentiable option on");
  if (first_frame != c.adj_first || n_frames != c.adj_frames)
    return fail(PT_INVALID_ARG, "pt_render_adjoint: frames differ from the last differentiable forward render");
  for (const MatDev& m : c.mats) {
    if (m.type == PT_METALLIC_SHADER && __float_as_int_host(m.tmap.w) >= 0 && m.dist != PT_GGX_DISTRIBUTION)
      return fail(PT_INVALID_ARG, "pt_render_adjoint: roughness gradients are implemented for the GGX distribution");
    if (m.type == PT_ROUGH_TRANSLUCENT_SHADER)
      return fail(PT_INVALID_ARG, "pt_render_adjoint: rough translucent materials are not differentiable");
    if (m.type == PT_TRANSPARENT_SHADER || m.type == PT_LAMBERTIAN_INTERFACE_SHADER || m.type == PT_ROUGH_DIFFUSE_SHADER)
      return fail(PT_INVALID_ARG, "pt_render_adjoint: transparent, lambertian-interface and rough-diffuse materials are not differentiable");
  }
  pt_status st = prepare_scene(c, "pt_render_adjoint");
  if (st != PT_OK) return st;
  SceneFacts f = scene_facts(c);
  PassLayout L = plan_pass({f}, {ItemReq{0, first_frame, n_frames}}, c.max_paths);
  c.adj_dimg = (const float4*)d_dimage;
  c.adj_dscale = 1.0f / (float)((uint64_t)first_frame + n_frames);
  std::vector<SceneDev> scenes{c.view()};
  c.adj_dimg = nullptr;
  c.adj_dscale = 0.0f;
  if ((st = pass_resources(c, L, scenes)) != PT_OK) return st;
  if ((st = c.wf.adj_a.reserve(c.wf.cap * sizeof(float4), "adjoint path state")) != PT_OK) return st;
  if ((st = c.wf.adj_b.reserve(c.wf.cap * sizeof(float4), "adjoint path state")) != PT_OK) return st;
  uint64_t launches0 = pt_kernel_launch_count();
  memset(&c.stats, 0, sizeof(c.stats));
  PT_CHECK_CUDA(cudaEventRecord(c.ev0, c.stream), "event");
  if ((st = launch_pass(c, L, scenes, false, true, true)) != PT_OK) return st;
  PT_CHECK_CUDA(cudaEventRecord(c.ev1, c.stream), "event");
  c.stats.path_samples = scene_path_samples(c, n_frames);
  c.stats.kernel_launches = (uint32_t)(pt_kernel_launch_count() - launches0);
  c.stats_pending = true;
  return PT_OK;
}

pt_status pt_get_probes(pt_ctx* ctx, void* out, uint64_t capacity, uint64_t* n_out)
{
  if (!ctx || !n_out) return fail(PT_INVALID_ARG, "pt_get_probes: null argument");
  Context& c = ctx->c;
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  const uint64_t per_frame = (uint64_t)c.trans_objs.size() * c.probe_samples;
  if (c.probe_last_frames == 0 || per_frame == 0 || !c.wf.probes.p) {
    *n_out = 0;
    return PT_OK;
  }
  *n_out = per_frame;
  uint64_t n = std::min(capacity, per_frame);
  if (n && !out) return fail(PT_INVALID_ARG, "pt_get_probes: null output buffer");
  const char* src = (const char*)c.wf.probes.p + (size_t)(c.probe_last_frames - 1) * per_frame * 80;
  if (n) PT_CHECK_CUDA(cudaMemcpyAsync(out, src, (size_t)n * 80, cudaMemcpyDeviceToHost, c.stream), "pt_get_probes");
  PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_get_probes");
  return PT_OK;
}

pt_status pt_get_render_stats(pt_ctx* ctx, pt_render_stats* out)
{
  if (!ctx || !out) return fail(PT_INVALID_ARG, "pt_get_render_stats: null argument");
  Context& c = ctx->c;
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_get_render_stats");
  if (c.stats_pending && c.wf.counters.p) {
    uint32_t h[kCounters], h2[kCounters];
    PT_CHECK_CUDA(cudaMemcpy(h, c.wf.counters.p, sizeof(h), cudaMemcpyDeviceToHost), "read counters");
    const bool two = c.pass_dual && c.wf2.counters.p;  // a dual pass counts in both wavefronts
    if (two) PT_CHECK_CUDA(cudaMemcpy(h2, c.wf2.counters.p, sizeof(h2), cudaMemcpyDeviceToHost), "read counters");
    auto rd64 = [&](int slot) {
      unsigned long long v, v2 = 0;
      memcpy(&v, h + slot, 8);
      if (two) memcpy(&v2, h2 + slot, 8);
      return (uint64_t)(v + v2);
    };
    c.stats.segments = rd64(CNT_SEGMENTS_LO);
    c.stats.shadow_rays = rd64(CNT_SHADOW_TOTAL);
    c.stats.capped_walks = rd64(CNT_CAPPED);
    c.stats.clamped_indices = rd64(CNT_CLAMPED);
    c.stats.dipole_gathers = rd64(CNT_GATHERS);
    c.stats.dipole_pairs = rd64(CNT_PAIRS);
    c.stats.gather_overflows = rd64(CNT_ERROR);
    float ms = 0.0f;
    PT_CHECK_CUDA(cudaEventElapsedTime(&ms, c.ev0, c.ev1), "event time");
    c.stats.gpu_ms = ms;
    float ext = 0.0f, gat = 0.0f;
    for (uint32_t k = 0; k < c.prof_pairs; ++k) {
      float e = 0.0f;
      PT_CHECK_CUDA(cudaEventElapsedTime(&e, c.prof_events[2 * k], c.prof_events[2 * k + 1]), "event time");
      (c.prof_kind[k] == PROF_GATHER ? gat : ext) += e;
    }
    c.stats.extend_ms = ext;
    c.stats.gather_ms = gat;
    c.stats_pending = false;
  }
  *out = c.stats;
  return PT_OK;
}

}  // extern "C"
