// Host-side context behind the opaque pt_ctx handle of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <vector>

#include "pt_bvh.h"
#include "pt_common.cuh"
#include "pt_scene.cuh"

namespace pt {

// The boundary polynomials of Fresnel.h:93-124 (two_C1, three_C2, C_phi, C_E) on the host, in the
// scalar type R with the reference's float coefficients (R = float is the reference's arithmetic).
template <class R> inline R two_C1_t(R n)
{
  if (n >= R(1)) return R(-9.23372f) + n * (R(22.2272f) + n * (R(-20.9292f) + n * (R(10.2291f) + n * (R(-2.54396f) + n * R(0.254913f)))));
  return R(0.919317f) + n * (R(-3.4793f) + n * (R(6.75335f) + n * (R(-7.80989f) + n * (R(4.98554f) - n * R(1.36881f)))));
}
template <class R> inline R three_C2_t(R n)
{
  R r;
  if (n >= R(1)) {
    r = R(-1641.1f) + n * (R(1213.67f) + n * (R(-568.556f) + n * (R(164.798f) + n * (R(-27.0181f) + n * R(1.91826f)))));
    r += (((R(135.926f) / n) - R(656.175f)) / n + R(1376.53f)) / n;
  } else {
    r = R(0.828421f) + n * (R(-2.62051f) + n * (R(3.36231f) + n * (R(-1.95284f) + n * (R(0.236494f) + n * R(0.145787f)))));
  }
  return r;
}
template <class R> inline R C_phi_t(R n) { return R(0.25f) * (R(1) - two_C1_t<R>(n)); }
template <class R> inline R C_E_t(R n) { return R(0.5f) * (R(1) - three_C2_t<R>(n)); }

// 1.0f / MyComplex in the reference's arithmetic (MyComplex.h:155-160), evaluated on the host.
Cx host_recip(const Cx& b);
// TranslucentMaterial::computeCoefficients (TranslucentMaterial.cpp:303-330), FP32 on the host.
ScatDev compute_coefficients(const pt_translucent_params& q);

// Owning device allocation (cudaMalloc / cudaFree), reused when large enough.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release()
  {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
  }
  // Ensures capacity >= n bytes (contents are not preserved when it grows).
  pt_status reserve(size_t n, const char* what)
  {
    if (n <= bytes && p) return PT_OK;
    release();
    if (n == 0) return PT_OK;
    cudaError_t e = cudaMalloc(&p, n);
    if (e != cudaSuccess) {
      p = nullptr;
      return cuda_status(e, what);
    }
    bytes = n;
    return PT_OK;
  }
  template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

// Wavefront buffers, sized for `cap` paths in flight.
struct Wavefront {
  uint64_t cap = 0;
  DevBuf rays, state;                         // per path, 32-byte records: (ray origin, direction), (throughput, rng)
  DevBuf rad, hit;                            // per path
  DevBuf path_item;                           // per path: its item of the pass (uint16)
  DevBuf adj_a, adj_b;                        // adjoint renders: per path image gradient and pending gradient
  DevBuf q_a, q_b;                            // active queues (path ids)
  DevBuf q_mat;                               // per-material-class queues, kQueues x cap
  DevBuf cls_of, bin;                         // class per queue position (bytes) and binning block counts
  DevBuf sh_o, sh_d, sh_c, sh_pid;            // shadow-ray queue
  DevBuf counters;                            // kCounters uint32
  // translucent objects: the per-path stack of pending dipole gathers ([slot][path]) and the probes
  uint32_t gather_slots = 0;
  uint64_t gather_cap = 0;
  DevBuf g_a, g_b, g_c, g_d;
  uint64_t probe_cap = 0;                     // PositionSample records held
  DevBuf probes;                              // PositionSample (80 B) per probe, [frame][object][sample]
  DevBuf pc_pos, pc_wl, pc_nrm, pc_tr, pc_cnt;// probes with L != 0, compacted in order per (frame, object)
};

// Counter slots in Wavefront::counters.
enum CounterSlot {
  CNT_ACTIVE_A = 0,
  CNT_ACTIVE_B = 1,
  CNT_Q_MISS = 2,        // kQueues consecutive material-queue counts
  CNT_Q_LIGHT = 3,
  CNT_Q_DIFFUSE = 4,
  CNT_Q_METAL = 5,
  CNT_Q_GLASS = 6,
  CNT_Q_TRANS = 7,
  CNT_Q_LAYERED = 8,
  CNT_FETCH_EXT = 9,     // slots 2..9 are reset at the start of each bounce,
  CNT_SHADOW = 10,       // 10..11 before its shading (the previous bounce's shadow rays may still run)
  CNT_FETCH_SH = 11,
  CNT_GATHER = 12,
  CNT_SEGMENTS_LO = 14,  // 64-bit totals as two words each at even slots (8-byte aligned atomicAdd on unsigned long long)
  CNT_SHADOW_TOTAL = 16,
  CNT_CAPPED = 18,
  CNT_CLAMPED = 20,
  CNT_ERROR = 22,
  CNT_PAIRS = 24,        // probe evaluations of the dipole gathers
  CNT_GATHERS = 26,      // dipole gathers evaluated
  kCounters = 32
};
static_assert(CNT_SEGMENTS_LO % 2 == 0 && CNT_SHADOW_TOTAL % 2 == 0 && CNT_CAPPED % 2 == 0 && CNT_CLAMPED % 2 == 0 &&
                  CNT_ERROR % 2 == 0 && CNT_PAIRS % 2 == 0 && CNT_GATHERS % 2 == 0 && CNT_GATHERS + 2 <= kCounters,
              "64-bit counters sit at even slots inside the counter block");
// Material classes of the extend kernel's binning; QC_LAYERED: a Lambertian base under a smooth or rough
// dielectric interface (lambertian_interface_shader.cu, rough_diffuse_shader.cu).
enum QueueClass { QC_MISS = 0, QC_LIGHT = 1, QC_DIFFUSE = 2, QC_METAL = 3, QC_GLASS = 4, QC_TRANS = 5, QC_LAYERED = 6, kQueues = 7 };
static_assert(CNT_Q_MISS + kQueues - 1 == CNT_Q_LAYERED, "one consecutive count per material class");

// One (scene, frame range) of a wavefront pass.  The camera paths, probes, accumulated pixels and probe
// sets of a pass are numbered item after item; every path records its item.
struct ItemDev {
  uint32_t scene;        // index into the pass's scene table
  uint32_t first_frame;
  uint32_t n_frames;
  uint32_t pixels;       // width * height of the scene
  uint64_t path_begin;   // first camera path id: path = path_begin + frame_in_item * pixels + pixel
  uint64_t probe_begin;  // first probe id: probe = probe_begin + (frame_in_item * n_trans + object) * samples + sample
  uint64_t pix_begin;    // first accumulation id: pix_begin + pixel
  uint32_t set_begin;    // first probe set: set_begin + frame_in_item * n_trans + object
  uint32_t pad;
};

// What the pass planner needs to know of a scene.
struct SceneFacts {
  uint32_t pixels = 1, n_trans = 0, samples = 0;
  int max_depth = 0;
  bool layered = false;  // has a material of queue class QC_LAYERED
  bool ms = false;       // has a conductor or rough dielectric of the multiple-scattering model
};
// A request: frames [first_frame, first_frame + n_frames) of scene `scene`.
struct ItemReq {
  uint32_t scene, first_frame, n_frames;
};
// A planned pass: chunks of whole frames, each at most max_paths camera paths, items chunk after chunk.
struct PassLayout {
  std::vector<ItemDev> items;
  std::vector<uint32_t> chunk_item_begin;
  std::vector<uint64_t> chunk_paths, chunk_probes, chunk_pixels;
  std::vector<uint32_t> chunk_sets;
  uint64_t cap_paths = 0, cap_probes = 0, cap_sets = 0;
  int passes = 0;
  bool sss = false;
  bool dual = false;     // chunks alternate between two wavefronts that run at once (two pipelines)
  bool layered = false;  // some scene of the pass has layered materials (k_shade_layered is launched)
  bool ms = false;       // some scene of the pass has multiple-scattering conductors or dielectrics
  uint32_t g_slots = 0;
};

enum ProfKind { PROF_EXTEND = 0, PROF_GATHER = 1 };

// Tunable launch options (pt_set_option); the autotuner searches over these.
struct Options {
  int extend_mode = 1;  // 0: one ray per thread, block-aggregated appends; 1: persistent warps with ray refill
  int refill = 20;      // persistent kernels: refill when at least this many lanes of a warp are idle (1..32)
  int bin_items = 8;    // material binning: queue positions per thread (4, 8 or 16; 256 threads per chunk)
  int overlap = 1;      // 1: a bounce's shading classes on two streams and its shadow rays beside the next
                        // bounce's extend and binning; 0: every launch in order on the context stream
  int dual = 1;         // 1: passes without translucent materials split their paths into chunks of half the
                        // wavefront that run two at a time on two wavefronts (two pipelines); 0: one wavefront
};

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ext0 = nullptr, ext1 = nullptr;

  IntegratorDev integ{50, 1e-4f, 0, {1.0f, 0.0f, 0.0f}};  // PathTracer defaults (Integrator.cpp:6-24)
  CameraDev cam{};
  bool camera_set = false;
  float3 bg_color{1.0f, 1.0f, 1.0f};                      // ConstantBackground default (Background.cpp:10)

  std::vector<MatDev> mats;
  std::vector<ScatDev> scat;        // per material; the scattering properties of translucent ones
  // translucent objects (OptixSceneLoader::computeTranslucentGeometries, OptixSceneLoader.cpp:482-524):
  // (material, first triangle, triangle count, offset into trans_pos) per translucent mesh
  std::vector<uint4> trans_objs;
  std::vector<float> trans_pos;     // their vertex positions, 9 floats per triangle, as given
  uint32_t probe_samples = 500;     // context["samples"] (OptixSceneLoader.cpp:11-17)
  uint32_t probe_last_frames = 0;   // frames whose probes the probe buffer holds (the last one is read back)
  // meshes as added (host copies until pt_build)
  std::vector<float> tri_pos;       // 9 floats per triangle
  std::vector<int4> tri_info;       // (n0, n1, n2, material)
  std::vector<float4> normals;
  std::vector<LightRaw> lights;
  std::vector<TriLightRaw> tri_lights;
  bool built = false;
  bool dirty_materials = true;
  int bvh_depth = 0;
  uint32_t n_tris = 0;

  DevBuf d_nodes, d_nodes4, d_v0, d_e1, d_e2, d_info, d_normals, d_mats, d_lights, d_tri_lights;
  std::vector<float4> ana;  // analytic emitters of the disk and sphere lights (3 float4 each)
  DevBuf d_ana;
  BvhParams bvh_params;    // options "bvh_trav_cost_milli" and "bvh_max_leaf", applied by pt_build
  bool has_bvh4 = false;
  bool use_bvh4 = true;  // option "bvh4": the persistent traversal kernels walk the 4-wide BVH
  int bvh_builder = 0;   // option "bvh_builder": 0 host binned SAH, 1 device LBVH
  float trav_scale = 0.0f;  // diagonal of the triangles' bounding box (the box tests' margin), set by pt_build
  pt_build_info build_info{};
  DevBuf d_build_scratch;  // the device builder's temporaries, kept for rebuilds
  DevBuf d_scat, d_trans_objs, d_trans_pos;
  DevBuf d_scene_tab, d_item_tab;  // scene and item tables of the current pass (this context as the engine)
  bool pass_w4 = false;            // every scene of the current pass has a 4-wide BVH
  // differentiable renders: the forward state of the last render of frames [adj_first, +adj_frames)
  bool differentiable = false;
  DevBuf d_adj_L, d_adj_G;
  uint32_t adj_first = 0, adj_frames = 0, adj_slots = 0;
  bool adj_valid = false;
  const float4* adj_dimg = nullptr;  // set while an adjoint render is being launched
  float adj_dscale = 0.0f;
  std::vector<float*> mat_grad;     // per material: sigma gradient buffer (6 floats) or null
  DevBuf d_mat_grad;
  bool dirty_mat_grad = true;
  std::vector<TexDev> textures;     // bound textures (data in tex_own or caller-owned device memory)
  std::vector<std::unique_ptr<DevBuf>> tex_own;
  DevBuf d_tex;
  bool dirty_textures = false;
  uint32_t next_frame = 0;         // first frame of the next render that does not name one (batches)
  DevBuf d_accum;  // float4 per pixel
  DevBuf d_env_tex, d_env_mpdf, d_env_mcdf, d_env_cpdf, d_env_ccdf, d_env_lum, d_env_mf;
  int env_w = 0, env_h = 0;
  bool env_present = false;
  DevBuf d_normals_geo;  // float4 per original triangle: cross(v1-v0, v2-v0)
  bool geo_stale = true;
  Wavefront wf;
  uint64_t max_paths = 1ull << 24;

  Options opt;
  // the overlapped schedule: side[0] runs the shading kernels of the smaller classes, side[1] the
  // shadow rays; events fork from and join into `stream` (created by pass_resources, before any
  // graph capture)
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_shade = nullptr, ev_shadow = nullptr;
  // the second pipeline of dual passes: its wavefront, its three streams and events, and the events
  // that start it after the context stream, order the chunks' accumulations and join it back
  Wavefront wf2;
  cudaStream_t stream2 = nullptr, side2[2] = {nullptr, nullptr};
  cudaEvent_t ev2_fork = nullptr, ev2_join = nullptr, ev2_shade = nullptr, ev2_shadow = nullptr;
  cudaEvent_t ev_start = nullptr, ev_acc = nullptr, ev_end2 = nullptr;
  bool pass_dual = false;  // the last pass ran two pipelines (its counters are in wf and wf2)
  bool profile = false;
  std::vector<cudaEvent_t> prof_events;  // pairs around each extend and gather launch when profiling
  std::vector<int> prof_kind;            // PROF_EXTEND or PROF_GATHER per pair
  uint32_t prof_pairs = 0;
  pt_render_stats stats{};
  bool stats_pending = false;
  uint64_t launches_at_start = 0;

  SceneDev view() const;
};

// The LBVH of pt_bvh_device.cu built on the device from tri_pos into d_nodes, d_nodes4, d_v0/e1/e2
// (sets bvh_depth, has_bvh4 and build_info); PT_CAP_EXCEEDED when the tree is too deep for the
// traversal trail.
pt_status build_bvh_device(Context& c);

struct Context;
pt_status prepare_scene(Context& c, const char* who);
uint64_t scene_path_samples(const Context& c, uint32_t n_frames);
// Environment map: device buffers for a width x height texture and its tables, and the CDF build over
// the texels in d_env_tex (env_cameras.cu:23-75), queued on the context's stream.
pt_status env_reserve(Context& c, uint32_t width, uint32_t height);
pt_status env_build_tables(Context& c, uint32_t width, uint32_t height);
// What the pass planner needs to know of a scene (its size, translucent objects, layered materials).
SceneFacts scene_facts(const Context& c);
// dual: a pass without translucent materials is planned in chunks of at most max_paths / 2 paths that
// launch_pass runs two at a time (PassLayout::dual).
PassLayout plan_pass(const std::vector<SceneFacts>& facts, const std::vector<ItemReq>& reqs, uint64_t max_paths, bool dual = false);
pt_status pass_resources(Context& E, const PassLayout& L, const std::vector<SceneDev>& scenes);
pt_status launch_pass(Context& E, const PassLayout& L, const std::vector<SceneDev>& tab, bool multi, bool allow_events, bool adjoint = false);

}  // namespace pt

struct pt_ctx {
  pt::Context c;
};
