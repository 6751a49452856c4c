// C ABI: context lifetime, scene objects (integrator, camera, background, materials, meshes,
// lights), BVH build and upload, readback, and the closest/any-hit query kernels.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <new>
#include <string>

#include "pt_bvh.h"
#include "pt_context.h"

namespace pt {

SceneDev Context::view() const
{
  SceneDev s;
  memset(&s, 0, sizeof(s));  // padding included: captured passes key on the record's bytes
  s.nodes = d_nodes.as<float4>();
  s.nodes4 = has_bvh4 && use_bvh4 ? d_nodes4.as<float4>() : nullptr;
  s.trav_scale = trav_scale;
  s.tri_v0 = d_v0.as<float4>();
  s.tri_e1 = d_e1.as<float4>();
  s.tri_e2 = d_e2.as<float4>();
  s.tri_info = d_info.as<int4>();
  s.normals = d_normals.as<float4>();
  s.mats = d_mats.as<MatDev>();
  s.scat = d_scat.as<ScatDev>();
  s.tex = d_tex.as<TexDev>();
  s.geo = d_normals_geo.as<float4>();
  s.accum = d_accum.as<float4>();
  s.trans_objs = d_trans_objs.as<uint4>();
  s.trans_pos = d_trans_pos.as<float>();
  s.n_trans = (uint32_t)trans_objs.size();
  s.probe_samples = probe_samples;
  const bool adj = differentiable && d_adj_L.p;
  s.adj_L = adj ? d_adj_L.as<float4>() : nullptr;
  s.adj_G = adj && adj_slots ? d_adj_G.as<float4>() : nullptr;
  s.adj_first = adj_first;
  s.adj_frames = adj_frames;
  s.adj_slots = adj_slots;
  s.adj_dimg = adj_dimg;
  s.adj_dscale = adj_dscale;
  s.mat_grad = d_mat_grad.as<float*>();
  s.lights = d_lights.as<LightRaw>();
  s.tri_lights = d_tri_lights.as<TriLightRaw>();
  s.n_lights = (int)lights.size();
  s.n_tri_lights = (int)tri_lights.size();
  s.n_tris = n_tris;
  s.ana = d_ana.as<float4>();
  s.n_ana = (uint32_t)(ana.size() / 3);
  s.bg_color = bg_color;
  s.env.tex = d_env_tex.as<float4>();
  s.env.marginal_pdf = d_env_mpdf.as<float>();
  s.env.marginal_cdf = d_env_mcdf.as<float>();
  s.env.conditional_pdf = d_env_cpdf.as<float>();
  s.env.conditional_cdf = d_env_ccdf.as<float>();
  s.env.w = env_w;
  s.env.h = env_h;
  s.env.present = env_present ? 1 : 0;
  s.env.is_light = 0;
  for (const LightRaw& l : lights)
    if (l.type == ENVMAP_LIGHT) s.env.is_light = 1;
  s.cam = cam;
  s.integ = integ;
  return s;
}

// 1.0f / MyComplex in the reference's arithmetic (MyComplex.h:155-160 with :18-23): the squared
// magnitude is powf(float |c|, 2) and the quotient is formed in double.
Cx host_recip(const Cx& b)
{
  float r = (float)b.re, i = (float)b.im;
  float ab = sqrtf(r * r + i * i);
  double den = (double)powf(ab, 2.0f);
  double s = 1.0 / den;
  return Cx{((double)1.0f * b.re) * s, ((double)1.0f * -b.im) * s};
}

static bool finite_nonneg3(const float* v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]) && v[0] >= 0 && v[1] >= 0 && v[2] >= 0; }

static float __int_as_float_host(int i)
{
  float f;
  memcpy(&f, &i, 4);
  return f;
}

static float two_C1(float n) { return two_C1_t<float>(n); }
static float C_phi(float n) { return C_phi_t<float>(n); }
static float C_E(float n) { return C_E_t<float>(n); }

// TranslucentMaterial::computeCoefficients (TranslucentMaterial.cpp:303-330) with ior_outside = 1,
// evaluated in FP32 on the host in the same order.
ScatDev compute_coefficients(const pt_translucent_params& q)
{
  ScatDev p;
  memset(&p, 0, sizeof(p));
  const float3 one = f3s(1.0f);
  const float3 ior_outside = one;
  p.absorption = f3(q.absorption[0], q.absorption[1], q.absorption[2]) * q.scale;
  p.scattering = f3(q.scattering[0], q.scattering[1], q.scattering[2]) * q.scale;
  p.meancosine = f3(q.meancosine[0], q.meancosine[1], q.meancosine[2]);
  p.relative_ior = q.ior;
  p.ior_real = f3s(q.ior);
  float3 ior_rgb = p.ior_real / ior_outside;
  float3 reducedScattering = p.scattering * (1.0f - p.meancosine);
  p.relative_ior /= (ior_outside.x + ior_outside.y + ior_outside.z) / 3.0f;
  p.ior_real = ior_rgb;
  p.extinction = p.scattering + p.absorption;
  p.reducedExtinction = reducedScattering + p.absorption;
  p.deltaEddExtinction = p.scattering * (1.0f - p.meancosine * p.meancosine) + p.absorption;
  p.D = one / (3.0f * p.reducedExtinction);
  float3 aD = p.absorption / p.D;
  p.transport = f3(sqrtf(aD.x), sqrtf(aD.y), sqrtf(aD.z));
  p.C_phi = f3(C_phi(ior_rgb.x), C_phi(ior_rgb.y), C_phi(ior_rgb.z));
  p.C_phi_inv = f3(C_phi(1.0f / ior_rgb.x), C_phi(1.0f / ior_rgb.y), C_phi(1.0f / ior_rgb.z));
  p.C_E = f3(C_E(ior_rgb.x), C_E(ior_rgb.y), C_E(ior_rgb.z));
  p.albedo = p.scattering / p.extinction;
  p.reducedAlbedo = reducedScattering / p.reducedExtinction;
  p.de = 2.131f * p.D / f3(sqrtf(p.reducedAlbedo.x), sqrtf(p.reducedAlbedo.y), sqrtf(p.reducedAlbedo.z));
  p.A = (1.0f - p.C_E) / (2.0f * p.C_phi);
  p.three_D = 3.0f * p.D;
  p.two_A_de = 2.0f * p.A * p.de;
  p.global_coeff = one / (4.0f * p.C_phi_inv) * 1.0f / (4.0f * kPi * kPi);
  p.one_over_three_ext = one / (3.0f * p.extinction);
  p.mean_transport = (p.transport.x + p.transport.y + p.transport.z) / 3.0f;
  return p;
}

static pt_status make_material(uint32_t type, const void* params, size_t size, MatDev& m, ScatDev& sc)
{
  memset(&m, 0, sizeof(m));
  memset(&sc, 0, sizeof(sc));
  m.type = type;
  m.tmap = make_float4(0.0f, 0.0f, 0.0f, __int_as_float_host(-1));
  if (!params) return fail(PT_INVALID_ARG, "material: null parameters");
  switch (type) {
    case PT_DIFFUSE_SHADER: {
      if (size != sizeof(pt_diffuse_params)) return fail(PT_INVALID_ARG, "diffuse material: wrong parameter size");
      const pt_diffuse_params* p = (const pt_diffuse_params*)params;
      if (!finite_nonneg3(p->diffuse_color)) return fail(PT_INVALID_ARG, "diffuse material: diffuse_color must be finite and >= 0");
      m.a = make_float4(p->diffuse_color[0], p->diffuse_color[1], p->diffuse_color[2], 0.0f);
      return PT_OK;
    }
    case PT_METALLIC_SHADER: {
      if (size != sizeof(pt_metallic_params)) return fail(PT_INVALID_ARG, "metallic material: wrong parameter size");
      const pt_metallic_params* p = (const pt_metallic_params*)params;
      if (!(p->roughness[0] > 0.0f && p->roughness[1] > 0.0f && std::isfinite(p->roughness[0]) && std::isfinite(p->roughness[1])))
        return fail(PT_INVALID_ARG, "metallic material: roughness must be finite and > 0");
      if (p->microfacet_model > PT_MULTISCATTERING_MODEL || p->normal_distribution > PT_GGX_DISTRIBUTION)
        return fail(PT_INVALID_ARG, "metallic material: bad microfacet_model or normal_distribution");
      for (int k = 0; k < 6; ++k)
        if (!std::isfinite(p->ior[k])) return fail(PT_INVALID_ARG, "metallic material: ior must be finite");
      m.model = p->microfacet_model;
      m.dist = p->normal_distribution;
      m.a = make_float4(p->roughness[0], p->roughness[1], 0.0f, 0.0f);
      for (int c = 0; c < 3; ++c) {
        Cx ior{p->ior[2 * c], p->ior[2 * c + 1]};
        if (ior.re == 0.0 && ior.im == 0.0) return fail(PT_INVALID_ARG, "metallic material: ior must be non-zero");
        m.eta.c[c] = host_recip(ior);
        m.inv_eta.c[c] = host_recip(m.eta.c[c]);
      }
      return PT_OK;
    }
    case PT_ROUGH_TRANSPARENT_SHADER: {
      if (size != sizeof(pt_rough_transparent_params)) return fail(PT_INVALID_ARG, "rough transparent material: wrong parameter size");
      const pt_rough_transparent_params* p = (const pt_rough_transparent_params*)params;
      if (!(p->ior > 0.0f && std::isfinite(p->ior))) return fail(PT_INVALID_ARG, "rough transparent material: ior must be > 0");
      if (!(p->roughness > 0.0f && std::isfinite(p->roughness))) return fail(PT_INVALID_ARG, "rough transparent material: roughness must be > 0");
      if (!finite_nonneg3(p->glass_absorption)) return fail(PT_INVALID_ARG, "rough transparent material: glass_absorption must be finite and >= 0");
      if (p->microfacet_model > PT_MULTISCATTERING_MODEL || p->normal_distribution > PT_GGX_DISTRIBUTION)
        return fail(PT_INVALID_ARG, "rough transparent material: bad microfacet_model or normal_distribution");
      m.model = p->microfacet_model;
      m.dist = p->normal_distribution;
      m.a = make_float4(p->ior, p->roughness, 0.0f, 0.0f);
      m.b = make_float4(p->glass_absorption[0], p->glass_absorption[1], p->glass_absorption[2], 0.0f);
      return PT_OK;
    }
    case PT_TRANSPARENT_SHADER: {
      if (size != sizeof(pt_transparent_params)) return fail(PT_INVALID_ARG, "transparent material: wrong parameter size");
      const pt_transparent_params* p = (const pt_transparent_params*)params;
      if (!(p->ior > 0.0f && std::isfinite(p->ior))) return fail(PT_INVALID_ARG, "transparent material: ior must be > 0");
      if (!finite_nonneg3(p->glass_absorption)) return fail(PT_INVALID_ARG, "transparent material: glass_absorption must be finite and >= 0");
      m.a = make_float4(p->ior, 0.0f, 0.0f, 0.0f);
      m.b = make_float4(p->glass_absorption[0], p->glass_absorption[1], p->glass_absorption[2], 0.0f);
      return PT_OK;
    }
    case PT_LAMBERTIAN_INTERFACE_SHADER: {
      if (size != sizeof(pt_lambertian_interface_params)) return fail(PT_INVALID_ARG, "lambertian interface material: wrong parameter size");
      const pt_lambertian_interface_params* p = (const pt_lambertian_interface_params*)params;
      if (!finite_nonneg3(p->diffuse_color)) return fail(PT_INVALID_ARG, "lambertian interface material: diffuse_color must be finite and >= 0");
      if (!(p->ior > 0.0f && std::isfinite(p->ior))) return fail(PT_INVALID_ARG, "lambertian interface material: ior must be > 0");
      m.a = make_float4(p->diffuse_color[0], p->diffuse_color[1], p->diffuse_color[2], p->ior);
      m.b = make_float4(two_C1(p->ior), 0.0f, 0.0f, 0.0f);  // r_10 (lambertian_interface_shader.cu:63)
      return PT_OK;
    }
    case PT_ROUGH_DIFFUSE_SHADER: {
      if (size != sizeof(pt_rough_diffuse_params)) return fail(PT_INVALID_ARG, "rough diffuse material: wrong parameter size");
      const pt_rough_diffuse_params* p = (const pt_rough_diffuse_params*)params;
      if (!finite_nonneg3(p->diffuse_color)) return fail(PT_INVALID_ARG, "rough diffuse material: diffuse_color must be finite and >= 0");
      if (!(p->ior > 0.0f && std::isfinite(p->ior))) return fail(PT_INVALID_ARG, "rough diffuse material: ior must be > 0");
      if (!(p->roughness[0] > 0.0f && p->roughness[1] > 0.0f && std::isfinite(p->roughness[0]) && std::isfinite(p->roughness[1])))
        return fail(PT_INVALID_ARG, "rough diffuse material: roughness must be finite and > 0");
      if (p->microfacet_model > PT_MULTISCATTERING_MODEL || p->normal_distribution > PT_GGX_DISTRIBUTION)
        return fail(PT_INVALID_ARG, "rough diffuse material: bad microfacet_model or normal_distribution");
      m.model = p->microfacet_model;
      m.dist = p->normal_distribution;
      m.a = make_float4(p->diffuse_color[0], p->diffuse_color[1], p->diffuse_color[2], p->ior);
      m.b = make_float4(two_C1(p->ior), p->roughness[0], p->roughness[1], 0.0f);  // r_10 (rough_diffuse_shader.cu:70)
      // the multiscattering conductor walks' eta = MyComplex{1 / ior, 0} per channel (:132-133, :254-255)
      const float n1_over_n2 = 1.0f / p->ior;
      for (int c = 0; c < 3; ++c) {
        m.eta.c[c] = Cx{(double)n1_over_n2, 0.0};
        m.inv_eta.c[c] = host_recip(m.eta.c[c]);
      }
      return PT_OK;
    }
    case PT_ROUGH_TRANSLUCENT_SHADER: {
      if (size != sizeof(pt_rough_translucent_params)) return fail(PT_INVALID_ARG, "rough translucent material: wrong parameter size");
      const pt_rough_translucent_params* r = (const pt_rough_translucent_params*)params;
      if (!(r->roughness[0] > 0.0f && r->roughness[1] > 0.0f && std::isfinite(r->roughness[0]) && std::isfinite(r->roughness[1])))
        return fail(PT_INVALID_ARG, "rough translucent material: roughness must be finite and > 0");
      if (r->microfacet_model > PT_MULTISCATTERING_MODEL || r->normal_distribution > PT_GGX_DISTRIBUTION)
        return fail(PT_INVALID_ARG, "rough translucent material: bad microfacet_model or normal_distribution");
      pt_translucent_params t;
      memcpy(t.scattering, r->scattering, sizeof t.scattering);
      memcpy(t.absorption, r->absorption, sizeof t.absorption);
      memcpy(t.meancosine, r->meancosine, sizeof t.meancosine);
      t.ior = r->ior;
      t.scale = r->scale;
      t.dipole_model = r->dipole_model;
      pt_status st = make_material(PT_TRANSLUCENT_SHADER, &t, sizeof t, m, sc);
      if (st != PT_OK) return st;
      m.type = PT_ROUGH_TRANSLUCENT_SHADER;
      m.dist = r->normal_distribution;
      m.a = make_float4(r->scale, r->roughness[0], r->roughness[1], __int_as_float_host((int)r->microfacet_model));
      return PT_OK;
    }
    case PT_TRANSLUCENT_SHADER: {
      if (size != sizeof(pt_translucent_params)) return fail(PT_INVALID_ARG, "translucent material: wrong parameter size");
      const pt_translucent_params* p = (const pt_translucent_params*)params;
      if (!finite_nonneg3(p->absorption) || !finite_nonneg3(p->scattering))
        return fail(PT_INVALID_ARG, "translucent material: absorption and scattering must be finite and >= 0");
      for (int k = 0; k < 3; ++k) {
        if (!(p->meancosine[k] > -1.0f && p->meancosine[k] < 1.0f)) return fail(PT_INVALID_ARG, "translucent material: meancosine must be in (-1, 1)");
        if (!(p->absorption[k] + p->scattering[k] * (1.0f - p->meancosine[k]) > 0.0f))
          return fail(PT_INVALID_ARG, "translucent material: the reduced extinction must be > 0");
      }
      if (!(p->ior > 0.0f && std::isfinite(p->ior))) return fail(PT_INVALID_ARG, "translucent material: ior must be > 0");
      if (!(p->scale > 0.0f && std::isfinite(p->scale))) return fail(PT_INVALID_ARG, "translucent material: scale must be > 0");
      if (p->dipole_model > PT_DIRECTIONAL_DIPOLE) return fail(PT_INVALID_ARG, "translucent material: bad dipole_model");
      m.model = p->dipole_model;
      m.a = make_float4(p->scale, 0.0f, 0.0f, 0.0f);  // scale: d extinction / d sigma (adjoint renders)
      sc = compute_coefficients(*p);
      return PT_OK;
    }
    case PT_AREA_LIGHT_MATERIAL: {
      if (size != sizeof(pt_area_light_params)) return fail(PT_INVALID_ARG, "area light material: wrong parameter size");
      const pt_area_light_params* p = (const pt_area_light_params*)params;
      if (!finite_nonneg3(p->radiance)) return fail(PT_INVALID_ARG, "area light material: radiance must be finite and >= 0");
      m.a = make_float4(p->radiance[0], p->radiance[1], p->radiance[2], 0.0f);
      return PT_OK;
    }
    default:
      return fail(PT_INVALID_ARG, "material: unsupported type " + std::to_string(type));
  }
}

template <class T> static pt_status upload(DevBuf& buf, const std::vector<T>& v, cudaStream_t s, const char* what)
{
  size_t bytes = v.size() * sizeof(T);
  pt_status st = buf.reserve(bytes ? bytes : 16, what);
  if (st != PT_OK) return st;
  if (bytes) PT_CHECK_CUDA(cudaMemcpyAsync(buf.p, v.data(), bytes, cudaMemcpyHostToDevice, s), what);
  return PT_OK;
}

// ------------------------------------------------------------------ query kernels
__global__ void k_trace_closest(SceneDev S, const float4* ot, const float4* dt, uint32_t n, int32_t* prim, float* tout, float* bary)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 a = ot[i], b = dt[i];
    Hit h = scene_closest(S, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), a.w, b.w);
    prim[i] = h.prim;
    tout[i] = h.prim >= 0 ? h.t : -1.0f;
    bary[2 * i] = h.u;
    bary[2 * i + 1] = h.v;
  }
}
__global__ void k_trace_any(SceneDev S, const float4* ot, const float4* dt, uint32_t n, int32_t* hit)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 a = ot[i], b = dt[i];
    hit[i] = scene_any(S, f3(a.x, a.y, a.z), f3(b.x, b.y, b.z), a.w, b.w) ? 1 : 0;
  }
}

// ------------------------------------------------------------------ environment CDFs (env_cameras.cu:23-75)
// env_luminance_camera: luminance_NTSC(texel at the texel centre) * sin(theta).
__global__ void k_env_luminance(EnvDev E, float* lum)
{
  size_t n = (size_t)E.w * E.h;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    int i = (int)(k % E.w), j = (int)(k / E.w);
    float u = ((float)i + 0.5f) / (float)E.w, v = ((float)j + 0.5f) / (float)E.h;
    float theta = (1.0f - v) * kPi;
    float3 t = env_tex(E, u, v);
    lum[k] = (t.x * 0.2989f + t.y * 0.5866f + t.z * 0.1145f) * sinf(theta);
  }
}
// env_marginal_camera and the conditional half of env_pdf_camera: per row, the sequential float sum
// in the reference's order (every prefix is the sum the reference recomputes per texel).
__global__ void k_env_rows(EnvDev E, const float* lum, float* mf, float* cpdf, float* ccdf)
{
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < E.h; j += gridDim.x * blockDim.x) {
    const float* row = lum + (size_t)j * E.w;
    float s = 0.0f;
    for (int i = 0; i < E.w; ++i) s += row[i];
    float m = s / (float)E.w;
    mf[j] = m;
    float c = 0.0f;
    for (int i = 0; i < E.w; ++i) {
      c += row[i];
      cpdf[(size_t)j * E.w + i] = row[i] / m;
      ccdf[(size_t)j * E.w + i] = (c / (float)E.w) / m;
    }
  }
}
// The marginal half of env_pdf_camera (one sequential pass) and the two entries forced to 1.
__global__ void k_env_marginal(EnvDev E, const float* mf, float* mpdf, float* mcdf, float* ccdf)
{
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  float total = 0.0f;
  for (int j = 0; j < E.h; ++j) total += mf[j];
  float m = total / (float)E.h;
  float c = 0.0f;
  for (int j = 0; j < E.h; ++j) {
    c += mf[j];
    mpdf[j] = mf[j] / m;
    mcdf[j] = (c / (float)E.h) / m;
  }
  mcdf[E.h - 1] = 1.0f;
  ccdf[(size_t)(E.h - 1) * E.w + (E.w - 1)] = 1.0f;
}

__global__ void k_env_query(EnvDev E, const float* dirs, uint32_t n_dirs, float* looked, uint32_t* seeds, uint32_t n_samples, float* sdir, float* sL)
{
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n_dirs + n_samples; i += gridDim.x * blockDim.x) {
    if (i < n_dirs) {
      float3 r = env_lookup(E, f3(dirs[3 * i], dirs[3 * i + 1], dirs[3 * i + 2]));
      looked[3 * i] = r.x;
      looked[3 * i + 1] = r.y;
      looked[3 * i + 2] = r.z;
    } else {
      uint32_t k = i - n_dirs;
      uint32_t t = seeds[k];
      float3 d, L;
      sample_environment(E, d, L, t);
      seeds[k] = t;
      sdir[3 * k] = d.x; sdir[3 * k + 1] = d.y; sdir[3 * k + 2] = d.z;
      sL[3 * k] = L.x; sL[3 * k + 1] = L.y; sL[3 * k + 2] = L.z;
    }
  }
}

}  // namespace pt

using namespace pt;

#define CTX_CHECK(ctx)                                                          \
  do {                                                                          \
    if (!(ctx)) return fail(PT_INVALID_ARG, "null context");                    \
    PT_CHECK_CUDA(cudaSetDevice((ctx)->c.device), "cudaSetDevice");             \
  } while (0)

extern "C" {

pt_status pt_context_create(int device, pt_ctx** out)
{
  if (!out) return fail(PT_INVALID_ARG, "pt_context_create: null output");
  *out = nullptr;
  int n = 0;
  PT_CHECK_CUDA(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
  if (device < 0 || device >= n) return fail(PT_INVALID_ARG, "pt_context_create: no such device");
  PT_CHECK_CUDA(cudaSetDevice(device), "cudaSetDevice");
  pt_ctx* ctx = new (std::nothrow) pt_ctx();
  if (!ctx) return fail(PT_OOM, "pt_context_create: host allocation");
  ctx->c.device = device;
  cudaError_t e = cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->c.ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->c.ev1);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->c.ext0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->c.ext1);
  if (e != cudaSuccess) {
    pt_context_destroy(ctx);
    return cuda_status(e, "pt_context_create");
  }
  *out = ctx;
  return PT_OK;
}

pt_status pt_context_destroy(pt_ctx* ctx)
{
  if (!ctx) return PT_OK;
  cudaSetDevice(ctx->c.device);
  if (ctx->c.stream) cudaStreamSynchronize(ctx->c.stream);
  Context& c = ctx->c;
  for (cudaEvent_t ev : {c.ev0, c.ev1, c.ext0, c.ext1})
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : c.prof_events)
    if (ev) cudaEventDestroy(ev);
  for (cudaEvent_t ev : {c.ev_fork, c.ev_join, c.ev_shade, c.ev_shadow, c.ev2_fork, c.ev2_join, c.ev2_shade, c.ev2_shadow, c.ev_start,
                         c.ev_acc, c.ev_end2})
    if (ev) cudaEventDestroy(ev);
  for (cudaStream_t sd : {c.side[0], c.side[1], c.side2[0], c.side2[1], c.stream2})
    if (sd) cudaStreamDestroy(sd);
  cudaStream_t s = c.stream;
  delete ctx;  // frees device buffers
  if (s) cudaStreamDestroy(s);
  return PT_OK;
}

void* pt_context_stream(pt_ctx* ctx) { return ctx ? (void*)ctx->c.stream : nullptr; }

pt_status pt_set_integrator(pt_ctx* ctx, uint32_t max_depth, float scene_epsilon, const float exception_color[3], uint32_t rr_start_depth)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  if (max_depth > 1000) return fail(PT_INVALID_ARG, "pt_set_integrator: max_depth must be <= 1000");
  if (!(scene_epsilon >= 0.0f) || !std::isfinite(scene_epsilon)) return fail(PT_INVALID_ARG, "pt_set_integrator: scene_epsilon must be finite and >= 0");
  ctx->c.integ.max_depth = (int)max_depth;
  ctx->c.integ.scene_epsilon = scene_epsilon;
  ctx->c.integ.rr_start = (int)rr_start_depth;
  if (exception_color) ctx->c.integ.exception_color = make_float3(exception_color[0], exception_color[1], exception_color[2]);
  return PT_OK;
}

pt_status pt_set_camera(pt_ctx* ctx, const float eye[3], const float U[3], const float V[3], const float W[3], uint32_t width,
                        uint32_t height, const uint32_t patch_origin[2], const uint32_t patch_dims[2])
{
  CTX_CHECK(ctx);
  if (!eye || !U || !V || !W) return fail(PT_INVALID_ARG, "pt_set_camera: null vector");
  if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 28)) return fail(PT_INVALID_ARG, "pt_set_camera: bad image size");
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(eye[k]) || !std::isfinite(U[k]) || !std::isfinite(V[k]) || !std::isfinite(W[k]))
      return fail(PT_INVALID_ARG, "pt_set_camera: non-finite camera vector");
  Context& c = ctx->c;
  c.cam.eye = make_float3(eye[0], eye[1], eye[2]);
  c.cam.U = make_float3(U[0], U[1], U[2]);
  c.cam.V = make_float3(V[0], V[1], V[2]);
  c.cam.W = make_float3(W[0], W[1], W[2]);
  c.cam.patch_origin = patch_origin ? make_uint2(patch_origin[0], patch_origin[1]) : make_uint2(0, 0);
  c.cam.patch_dims = patch_dims ? make_uint2(patch_dims[0], patch_dims[1]) : make_uint2(width, height);
  bool resized = c.cam.width != width || c.cam.height != height || !c.d_accum.p;
  c.cam.width = width;
  c.cam.height = height;
  c.camera_set = true;
  c.next_frame = 0;
  if (resized) {
    pt_status st = c.d_accum.reserve((size_t)width * height * sizeof(float4), "accumulation buffer");
    if (st != PT_OK) return st;
    PT_CHECK_CUDA(cudaMemsetAsync(c.d_accum.p, 0, (size_t)width * height * sizeof(float4), c.stream), "clear accumulation");
  }
  return PT_OK;
}

pt_status pt_set_background_constant(pt_ctx* ctx, const float color[3])
{
  if (!ctx || !color) return fail(PT_INVALID_ARG, "pt_set_background_constant: null argument");
  if (!std::isfinite(color[0]) || !std::isfinite(color[1]) || !std::isfinite(color[2]))
    return fail(PT_INVALID_ARG, "pt_set_background_constant: non-finite color");
  ctx->c.bg_color = make_float3(color[0], color[1], color[2]);
  return PT_OK;
}

pt_status pt_set_envmap(pt_ctx* ctx, const float* rgba, uint32_t width, uint32_t height)
{
  CTX_CHECK(ctx);
  Context& c = ctx->c;
  if (!rgba) return fail(PT_INVALID_ARG, "pt_set_envmap: null texels");
  if (width < 2 || height < 2 || (uint64_t)width * height > (1ull << 26)) return fail(PT_INVALID_ARG, "pt_set_envmap: bad size");
  for (uint64_t k = 0; k < 4ull * width * height; ++k)
    if (!std::isfinite(rgba[k]) || rgba[k] < 0.0f) return fail(PT_INVALID_ARG, "pt_set_envmap: texels must be finite and >= 0");
  size_t n = (size_t)width * height;
  pt_status st = env_reserve(c, width, height);
  if (st != PT_OK) return st;
  PT_CHECK_CUDA(cudaMemcpyAsync(c.d_env_tex.p, rgba, n * sizeof(float4), cudaMemcpyHostToDevice, c.stream), "env upload");
  if ((st = env_build_tables(c, width, height)) != PT_OK) return st;
  PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_set_envmap");
  return PT_OK;
}

}  // extern "C"

namespace pt {
pt_status env_reserve(Context& c, uint32_t width, uint32_t height)
{
  size_t n = (size_t)width * height;
  pt_status st = c.d_env_tex.reserve(n * sizeof(float4), "env texture");
  if (st == PT_OK) st = c.d_env_lum.reserve(n * 4, "env luminance");
  if (st == PT_OK) st = c.d_env_cpdf.reserve(n * 4, "env conditional pdf");
  if (st == PT_OK) st = c.d_env_ccdf.reserve(n * 4, "env conditional cdf");
  if (st == PT_OK) st = c.d_env_mf.reserve((size_t)height * 4, "env marginal");
  if (st == PT_OK) st = c.d_env_mpdf.reserve((size_t)height * 4, "env marginal pdf");
  if (st == PT_OK) st = c.d_env_mcdf.reserve((size_t)height * 4, "env marginal cdf");
  return st;
}

pt_status env_build_tables(Context& c, uint32_t width, uint32_t height)
{
  size_t n = (size_t)width * height;
  c.env_w = (int)width;
  c.env_h = (int)height;
  c.env_present = true;
  EnvDev E = c.view().env;
  k_env_luminance<<<grid_for(n, 256, 8), 256, 0, c.stream>>>(E, c.d_env_lum.as<float>());
  k_env_rows<<<(height + 127) / 128, 128, 0, c.stream>>>(E, c.d_env_lum.as<float>(), c.d_env_mf.as<float>(), c.d_env_cpdf.as<float>(),
                                                         c.d_env_ccdf.as<float>());
  k_env_marginal<<<1, 32, 0, c.stream>>>(E, c.d_env_mf.as<float>(), c.d_env_mpdf.as<float>(), c.d_env_mcdf.as<float>(), c.d_env_ccdf.as<float>());
  count_launch(3);
  PT_CHECK_CUDA(cudaGetLastError(), "environment CDF build");
  return PT_OK;
}
}  // namespace pt

extern "C" {

pt_status pt_get_envmap_tables(pt_ctx* ctx, float* marginal_pdf, float* marginal_cdf, float* conditional_pdf, float* conditional_cdf)
{
  CTX_CHECK(ctx);
  Context& c = ctx->c;
  if (!c.env_present) return fail(PT_NOT_READY, "pt_get_envmap_tables: no environment map");
  size_t n = (size_t)c.env_w * c.env_h;
  if (marginal_pdf) PT_CHECK_CUDA(cudaMemcpy(marginal_pdf, c.d_env_mpdf.p, (size_t)c.env_h * 4, cudaMemcpyDeviceToHost), "env tables");
  if (marginal_cdf) PT_CHECK_CUDA(cudaMemcpy(marginal_cdf, c.d_env_mcdf.p, (size_t)c.env_h * 4, cudaMemcpyDeviceToHost), "env tables");
  if (conditional_pdf) PT_CHECK_CUDA(cudaMemcpy(conditional_pdf, c.d_env_cpdf.p, n * 4, cudaMemcpyDeviceToHost), "env tables");
  if (conditional_cdf) PT_CHECK_CUDA(cudaMemcpy(conditional_cdf, c.d_env_ccdf.p, n * 4, cudaMemcpyDeviceToHost), "env tables");
  return PT_OK;
}

pt_status pt_env_query(pt_ctx* ctx, const float* d_dirs, uint32_t n_dirs, float* d_looked, uint32_t* d_seeds, uint32_t n_samples,
                       float* d_sample_dirs, float* d_sample_L)
{
  CTX_CHECK(ctx);
  Context& c = ctx->c;
  if (!c.env_present) return fail(PT_NOT_READY, "pt_env_query: no environment map");
  if ((n_dirs && (!d_dirs || !d_looked)) || (n_samples && (!d_seeds || !d_sample_dirs || !d_sample_L)))
    return fail(PT_INVALID_ARG, "pt_env_query: null pointer");
  if (n_dirs + (uint64_t)n_samples == 0) return PT_OK;
  k_env_query<<<grid_for(n_dirs + (uint64_t)n_samples, 128, 8), 128, 0, c.stream>>>(c.view().env, d_dirs, n_dirs, d_looked, d_seeds, n_samples,
                                                                                    d_sample_dirs, d_sample_L);
  count_launch();
  PT_CHECK_CUDA(cudaGetLastError(), "pt_env_query launch");
  return PT_OK;
}

pt_status pt_material_create(pt_ctx* ctx, uint32_t type, const void* params, size_t params_size, uint32_t* out_id)
{
  if (!ctx || !out_id) return fail(PT_INVALID_ARG, "pt_material_create: null argument");
  MatDev m;
  ScatDev sc;
  pt_status st = make_material(type, params, params_size, m, sc);
  if (st != PT_OK) return st;
  if (ctx->c.mats.size() >= (1u << 20)) return fail(PT_CAP_EXCEEDED, "pt_material_create: too many materials");
  *out_id = (uint32_t)ctx->c.mats.size();
  ctx->c.mats.push_back(m);
  ctx->c.scat.push_back(sc);
  ctx->c.dirty_materials = true;
  return PT_OK;
}

pt_status pt_material_update(pt_ctx* ctx, uint32_t id, const void* params, size_t params_size)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  if (id >= ctx->c.mats.size()) return fail(PT_INVALID_ARG, "pt_material_update: no such material");
  MatDev m;
  ScatDev sc;
  pt_status st = make_material(ctx->c.mats[id].type, params, params_size, m, sc);
  if (st != PT_OK) return st;
  m.aux = ctx->c.mats[id].aux;    // translucent_index stays with the material
  m.tmap = ctx->c.mats[id].tmap;  // and so does its texture
  ctx->c.mats[id] = m;
  ctx->c.scat[id] = sc;
  ctx->c.dirty_materials = true;
  return PT_OK;
}

pt_status pt_mesh_add(pt_ctx* ctx, const float* positions, uint32_t n_vertices, const int32_t* vindex, uint32_t n_triangles,
                      const float* normals, uint32_t n_normals, const int32_t* nindex, uint32_t material_id,
                      uint32_t* out_first_triangle)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  Context& c = ctx->c;
  if (n_triangles == 0) return fail(PT_INVALID_ARG, "pt_mesh_add: empty mesh");
  if (!positions || !vindex) return fail(PT_INVALID_ARG, "pt_mesh_add: null positions or indices");
  if (material_id >= c.mats.size()) return fail(PT_INVALID_ARG, "pt_mesh_add: unknown material id");
  if ((uint64_t)c.n_tris + n_triangles >= (1ull << 27)) return fail(PT_CAP_EXCEEDED, "pt_mesh_add: scene exceeds 2^27 triangles");
  if (n_normals && (!normals || !nindex)) return fail(PT_INVALID_ARG, "pt_mesh_add: normals without normal indices");
  for (uint64_t k = 0; k < 3ull * n_vertices; ++k)
    if (!std::isfinite(positions[k])) return fail(PT_INVALID_ARG, "pt_mesh_add: non-finite vertex position");
  for (uint64_t k = 0; k < 3ull * n_triangles; ++k) {
    if (vindex[k] < 0 || (uint32_t)vindex[k] >= n_vertices) return fail(PT_INVALID_ARG, "pt_mesh_add: vertex index out of range");
    if (n_normals && (nindex[k] >= (int32_t)n_normals)) return fail(PT_INVALID_ARG, "pt_mesh_add: normal index out of range");
  }
  uint32_t normal_base = (uint32_t)c.normals.size();
  for (uint32_t k = 0; k < n_normals; ++k)
    c.normals.push_back(make_float4(normals[3 * k], normals[3 * k + 1], normals[3 * k + 2], 0.0f));
  if (out_first_triangle) *out_first_triangle = c.n_tris;
  for (uint32_t t = 0; t < n_triangles; ++t) {
    for (int k = 0; k < 3; ++k) {
      const float* p = positions + 3 * (size_t)vindex[3 * t + k];
      c.tri_pos.push_back(p[0]);
      c.tri_pos.push_back(p[1]);
      c.tri_pos.push_back(p[2]);
    }
    int4 info = make_int4(-1, -1, -1, (int)material_id);
    if (n_normals && nindex[3 * t] >= 0 && nindex[3 * t + 1] >= 0 && nindex[3 * t + 2] >= 0) {
      info.x = (int)normal_base + nindex[3 * t];
      info.y = (int)normal_base + nindex[3 * t + 1];
      info.z = (int)normal_base + nindex[3 * t + 2];
    }
    c.tri_info.push_back(info);
  }
  if (c.mats[material_id].type == PT_TRANSLUCENT_SHADER || c.mats[material_id].type == PT_ROUGH_TRANSLUCENT_SHADER) {
    // a translucent object with its own probe set; the material's translucent_index is the last
    // object registered with it (OptixSceneLoader.cpp:509-510)
    if (c.trans_objs.size() >= 1024) return fail(PT_CAP_EXCEEDED, "pt_mesh_add: at most 1024 translucent objects");
    c.trans_objs.push_back(make_uint4(material_id, c.n_tris, n_triangles, (uint32_t)(c.trans_pos.size() / 9)));
    c.trans_pos.insert(c.trans_pos.end(), c.tri_pos.end() - 9 * (size_t)n_triangles, c.tri_pos.end());
    c.mats[material_id].aux = (uint32_t)c.trans_objs.size() - 1;
    c.dirty_materials = true;
  }
  c.n_tris += n_triangles;
  c.built = false;
  return PT_OK;
}

pt_status pt_lights_upload(pt_ctx* ctx, const void* lights, uint32_t n_lights, const void* triangle_lights, uint32_t n_triangle_lights)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  if ((n_lights && !lights) || (n_triangle_lights && !triangle_lights)) return fail(PT_INVALID_ARG, "pt_lights_upload: null buffer");
  Context& c = ctx->c;
  c.lights.assign((const LightRaw*)lights, (const LightRaw*)lights + n_lights);
  c.tri_lights.assign((const TriLightRaw*)triangle_lights, (const TriLightRaw*)triangle_lights + n_triangle_lights);
  std::vector<float4> ana;
  for (uint32_t k = 0; k < n_lights; ++k) {
    const LightRaw& l = c.lights[k];
    if (l.type > ENVMAP_LIGHT) return fail(PT_INVALID_ARG, "pt_lights_upload: unknown light_type");
    if (l.type == TRIANGLES_AREA_LIGHT) {
      float cnt, start;
      memcpy(&cnt, &l.p[0], 4);
      memcpy(&start, &l.p[1], 4);
      if (!(cnt >= 1.0f) || !(start >= 0.0f) || (uint64_t)(start + cnt) > n_triangle_lights)
        return fail(PT_INVALID_ARG, "pt_lights_upload: triangle range of a TrianglesAreaLight is outside triangle_light_buffer");
    }
    if (l.type == DISK_LIGHT || l.type == SPHERICAL_LIGHT) {
      // DiskLightStruct (position, radius, phi, theta) / SphericalLightStruct (position, radius), structs.h:76-93
      for (int i = 0; i < 3; ++i)
        if (!std::isfinite(l.p[i]) || !std::isfinite(l.emitted[i])) return fail(PT_INVALID_ARG, "pt_lights_upload: non-finite disk or sphere light");
      const float radius = l.pad[0];
      if (!(radius > 0.0f) || !std::isfinite(radius)) return fail(PT_INVALID_ARG, "pt_lights_upload: disk and sphere lights need a finite radius > 0");
      float3 normal = f3(0.0f, 1.0f, 0.0f);
      if (l.type == DISK_LIGHT) {
        if (!std::isfinite(l.pad[1]) || !std::isfinite(l.pad[2])) return fail(PT_INVALID_ARG, "pt_lights_upload: non-finite disk light angles");
        // DiskAreaLight::computeNormal (Light.cpp:469-474), evaluated on the host as there
        const float t_rad = l.pad[2] * kPi / 180.0f, p_rad = l.pad[1] * kPi / 180.0f;
        normal = f3(sinf(t_rad) * sinf(p_rad), cosf(t_rad), sinf(t_rad) * cosf(p_rad));
      }
      const int kind = l.type == DISK_LIGHT ? ANA_DISK : ANA_SPHERE;
      float kind_f, idx_f;
      memcpy(&kind_f, &kind, 4);
      memcpy(&idx_f, &k, 4);
      ana.push_back(make_float4(l.p[0], l.p[1], l.p[2], radius));
      ana.push_back(make_float4(normal.x, normal.y, normal.z, kind_f));
      ana.push_back(make_float4(l.emitted[0], l.emitted[1], l.emitted[2], idx_f));
    }
  }
  c.ana.swap(ana);
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  pt_status st = upload(c.d_lights, c.lights, c.stream, "light buffer");
  if (st == PT_OK) st = upload(c.d_tri_lights, c.tri_lights, c.stream, "triangle light buffer");
  if (st == PT_OK) st = upload(c.d_ana, c.ana, c.stream, "analytic emitters");
  return st;
}

pt_status pt_build(pt_ctx* ctx)
{
  CTX_CHECK(ctx);
  Context& c = ctx->c;
  if (c.n_tris == 0) return fail(PT_NOT_READY, "pt_build: no meshes");
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  c.trav_scale = scene_diagonal(c.tri_pos.data(), c.n_tris);
  const auto t0 = std::chrono::steady_clock::now();
  pt_status st = PT_OK;
  bool on_device = false;
  memset(&c.build_info, 0, sizeof(c.build_info));
  if (c.bvh_builder == 1 && c.n_tris >= 2) {
    st = build_bvh_device(c);
    on_device = st == PT_OK;
    if (st != PT_OK && st != PT_CAP_EXCEEDED) return st;  // too deep: the host builder takes over
    st = PT_OK;
  }
  if (!on_device) {
    BvhHost bvh;
    if (!build_bvh(c.tri_pos.data(), c.n_tris, bvh, c.bvh_params)) return fail(PT_CAP_EXCEEDED, "pt_build: scene too large or BVH too deep");
    c.bvh_depth = bvh.depth;
    std::vector<float4> nodes4;
    int depth4 = 0;
    c.has_bvh4 = build_bvh4(bvh, nodes4, depth4, c.bvh_params);
    st = upload(c.d_nodes, bvh.nodes, c.stream, "BVH nodes");
    if (st == PT_OK && c.has_bvh4) st = upload(c.d_nodes4, nodes4, c.stream, "4-wide BVH nodes");
    if (st == PT_OK) st = upload(c.d_v0, bvh.tri_v0, c.stream, "triangles");
    if (st == PT_OK) st = upload(c.d_e1, bvh.tri_e1, c.stream, "triangles");
    if (st == PT_OK) st = upload(c.d_e2, bvh.tri_e2, c.stream, "triangles");
    if (st == PT_OK) PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_build upload");
    c.build_info.builder = 0;
    c.build_info.bvh2_nodes = (uint32_t)(bvh.nodes.size() / 4);
    c.build_info.bvh2_depth = (uint32_t)bvh.depth;
    c.build_info.wide_nodes = c.has_bvh4 ? (uint32_t)(nodes4.size() / kWideStride) : 0u;
    c.build_info.wide_depth = c.has_bvh4 ? (uint32_t)depth4 : 0u;
  }
  c.build_info.n_triangles = c.n_tris;
  c.build_info.build_ms = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (st == PT_OK) st = upload(c.d_info, c.tri_info, c.stream, "triangle info");
  if (st == PT_OK) st = upload(c.d_normals, c.normals, c.stream, "normals");
  if (st == PT_OK) st = upload(c.d_mats, c.mats, c.stream, "materials");
  if (st == PT_OK) st = upload(c.d_scat, c.scat, c.stream, "scattering properties");
  if (st == PT_OK) st = upload(c.d_trans_objs, c.trans_objs, c.stream, "translucent objects");
  if (st == PT_OK) st = upload(c.d_trans_pos, c.trans_pos, c.stream, "translucent triangles");
  if (st != PT_OK) return st;
  if (c.lights.empty()) {
    // light_buffer of size 0 is legal; keep a valid pointer for the kernels
    st = c.d_lights.reserve(sizeof(LightRaw), "light buffer");
    if (st == PT_OK) st = c.d_tri_lights.reserve(sizeof(TriLightRaw), "triangle light buffer");
    if (st != PT_OK) return st;
  }
  PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_build upload");
  c.dirty_materials = false;
  c.geo_stale = true;
  c.built = true;
  return PT_OK;
}

pt_status pt_readback(pt_ctx* ctx, float* host_rgba)
{
  CTX_CHECK(ctx);
  Context& c = ctx->c;
  if (!host_rgba) return fail(PT_INVALID_ARG, "pt_readback: null buffer");
  if (!c.camera_set) return fail(PT_NOT_READY, "pt_readback: camera not set");
  PT_CHECK_CUDA(cudaMemcpyAsync(host_rgba, c.d_accum.p, (size_t)c.cam.width * c.cam.height * sizeof(float4), cudaMemcpyDeviceToHost, c.stream),
                "pt_readback");
  PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_readback");
  return PT_OK;
}

pt_status pt_readback_device(pt_ctx* ctx, float* d_rgba)
{
  CTX_CHECK(ctx);
  Context& c = ctx->c;
  if (!d_rgba) return fail(PT_INVALID_ARG, "pt_readback_device: null buffer");
  if (!c.camera_set) return fail(PT_NOT_READY, "pt_readback_device: camera not set");
  PT_CHECK_CUDA(cudaMemcpyAsync(d_rgba, c.d_accum.p, (size_t)c.cam.width * c.cam.height * sizeof(float4), cudaMemcpyDeviceToDevice, c.stream),
                "pt_readback_device");
  return PT_OK;
}

pt_status pt_sync(pt_ctx* ctx)
{
  CTX_CHECK(ctx);
  PT_CHECK_CUDA(cudaStreamSynchronize(ctx->c.stream), "pt_sync");
  return PT_OK;
}

pt_status pt_texture_create(pt_ctx* ctx, const float* host_data, uint32_t width, uint32_t height, uint32_t channels, uint32_t* out_id)
{
  if (!ctx || !host_data || !out_id) return fail(PT_INVALID_ARG, "pt_texture_create: null argument");
  Context& c = ctx->c;
  if (width < 3 || height < 2 || (channels != 1 && channels != 3)) return fail(PT_INVALID_ARG, "pt_texture_create: need width >= 3, height >= 2, 1 or 3 channels");
  if ((uint64_t)width * height * channels > (1ull << 30)) return fail(PT_CAP_EXCEEDED, "pt_texture_create: texture too large");
  const size_t n = (size_t)width * height * channels;
  for (size_t k = 0; k < n; ++k)
    if (!std::isfinite(host_data[k])) return fail(PT_INVALID_ARG, "pt_texture_create: non-finite texel");
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  c.tex_own.emplace_back(new DevBuf());
  pt_status st = c.tex_own.back()->reserve(n * 4, "texture");
  if (st != PT_OK) return st;
  PT_CHECK_CUDA(cudaMemcpyAsync(c.tex_own.back()->p, host_data, n * 4, cudaMemcpyHostToDevice, c.stream), "texture upload");
  TexDev t;
  memset(&t, 0, sizeof(t));
  t.data = c.tex_own.back()->as<float>();
  t.w = width;
  t.h = height;
  t.ch = channels;
  *out_id = (uint32_t)c.textures.size();
  c.textures.push_back(t);
  c.dirty_textures = true;
  return PT_OK;
}

pt_status pt_texture_bind(pt_ctx* ctx, uint32_t id, const float* d_data)
{
  if (!ctx || !d_data) return fail(PT_INVALID_ARG, "pt_texture_bind: null argument");
  if (id >= ctx->c.textures.size()) return fail(PT_INVALID_ARG, "pt_texture_bind: no such texture");
  ctx->c.textures[id].data = d_data;
  ctx->c.dirty_textures = true;
  return PT_OK;
}

pt_status pt_texture_bind_grad(pt_ctx* ctx, uint32_t id, float* d_grad)
{
  if (!ctx) return fail(PT_INVALID_ARG, "pt_texture_bind_grad: null context");
  if (id >= ctx->c.textures.size()) return fail(PT_INVALID_ARG, "pt_texture_bind_grad: no such texture");
  ctx->c.textures[id].grad = d_grad;
  ctx->c.dirty_textures = true;
  return PT_OK;
}

pt_status pt_material_set_texture(pt_ctx* ctx, uint32_t material_id, uint32_t tex_id, const float center[3])
{
  if (!ctx || !center) return fail(PT_INVALID_ARG, "pt_material_set_texture: null argument");
  Context& c = ctx->c;
  if (material_id >= c.mats.size()) return fail(PT_INVALID_ARG, "pt_material_set_texture: no such material");
  if (tex_id >= c.textures.size()) return fail(PT_INVALID_ARG, "pt_material_set_texture: no such texture");
  MatDev& m = c.mats[material_id];
  const TexDev& t = c.textures[tex_id];
  if (m.type == PT_DIFFUSE_SHADER) {
    if (t.ch != 3) return fail(PT_INVALID_ARG, "pt_material_set_texture: a diffuse albedo texture has 3 channels");
  } else if (m.type == PT_METALLIC_SHADER) {
    if (t.ch != 1) return fail(PT_INVALID_ARG, "pt_material_set_texture: a roughness texture has 1 channel");
    if (m.model == PT_MULTISCATTERING_MODEL) return fail(PT_INVALID_ARG, "pt_material_set_texture: textured roughness supports the Walter and visible-normal models");
  } else {
    return fail(PT_INVALID_ARG, "pt_material_set_texture: only diffuse and metallic materials take a texture");
  }
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(center[k])) return fail(PT_INVALID_ARG, "pt_material_set_texture: non-finite center");
  m.tmap = make_float4(center[0], center[1], center[2], __int_as_float_host((int)tex_id));
  c.dirty_materials = true;
  return PT_OK;
}

pt_status pt_material_bind_sigma_grad(pt_ctx* ctx, uint32_t material_id, float* d_grad6)
{
  if (!ctx) return fail(PT_INVALID_ARG, "pt_material_bind_sigma_grad: null context");
  Context& c = ctx->c;
  if (material_id >= c.mats.size()) return fail(PT_INVALID_ARG, "pt_material_bind_sigma_grad: no such material");
  if (c.mats[material_id].type != PT_TRANSLUCENT_SHADER) return fail(PT_INVALID_ARG, "pt_material_bind_sigma_grad: not a translucent material");
  if (d_grad6 && c.mats[material_id].model != PT_STANDARD_DIPOLE)
    return fail(PT_INVALID_ARG, "pt_material_bind_sigma_grad: gradients are implemented for the standard dipole");
  c.mat_grad.resize(c.mats.size(), nullptr);
  c.mat_grad[material_id] = d_grad6;
  c.dirty_mat_grad = true;
  return PT_OK;
}

pt_status pt_set_probe_count(pt_ctx* ctx, uint32_t samples)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  if (samples < 1 || samples > (1u << 24)) return fail(PT_INVALID_ARG, "pt_set_probe_count: must be in [1, 2^24]");
  ctx->c.probe_samples = samples;
  return PT_OK;
}

pt_status pt_get_scattering_properties(pt_ctx* ctx, uint32_t material_id, void* out260)
{
  if (!ctx || !out260) return fail(PT_INVALID_ARG, "pt_get_scattering_properties: null argument");
  if (material_id >= ctx->c.mats.size()) return fail(PT_INVALID_ARG, "pt_get_scattering_properties: no such material");
  if (ctx->c.mats[material_id].type != PT_TRANSLUCENT_SHADER && ctx->c.mats[material_id].type != PT_ROUGH_TRANSLUCENT_SHADER)
    return fail(PT_INVALID_ARG, "pt_get_scattering_properties: not a translucent material");
  memcpy(out260, &ctx->c.scat[material_id], sizeof(ScatDev));
  return PT_OK;
}

pt_status pt_set_max_paths_in_flight(pt_ctx* ctx, uint64_t max_paths)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  if (max_paths < 1 || max_paths > (1ull << 30)) return fail(PT_INVALID_ARG, "pt_set_max_paths_in_flight: must be in [1, 2^30]");
  ctx->c.max_paths = max_paths;
  return PT_OK;
}

pt_status pt_set_option(pt_ctx* ctx, const char* name, int64_t value)
{
  if (!ctx || !name) return fail(PT_INVALID_ARG, "pt_set_option: null argument");
  std::string k(name);
  if (k == "differentiable") {
    if (value != 0 && value != 1) return fail(PT_INVALID_ARG, "pt_set_option: differentiable must be 0 or 1");
    ctx->c.differentiable = value != 0;
    ctx->c.adj_valid = false;
    return PT_OK;
  }
  if (k == "bvh_trav_cost_milli") {  // SAH node-step cost x 1000 (default 1200), for the next pt_build
    if (value < 100 || value > 20000) return fail(PT_INVALID_ARG, "pt_set_option: bvh_trav_cost_milli must be in [100, 20000]");
    ctx->c.bvh_params.trav_cost = (float)value / 1000.0f;
    return PT_OK;
  }
  if (k == "bvh_max_leaf") {  // largest SAH leaf (default 8), for the next pt_build
    if (value < 1 || value > 15) return fail(PT_INVALID_ARG, "pt_set_option: bvh_max_leaf must be in [1, 15]");
    ctx->c.bvh_params.max_leaf = (int)value;
    return PT_OK;
  }
  if (k == "bvh_collapse") {  // 4-wide collapse of either builder: 0 greedy, 1 SAH-optimal (default); next pt_build
    if (value != 0 && value != 1) return fail(PT_INVALID_ARG, "pt_set_option: bvh_collapse must be 0 or 1");
    ctx->c.bvh_params.collapse = (int)value;
    return PT_OK;
  }
  if (k == "bvh_wide_cost_milli") {  // SAH cost of a wide node visit x 1000 (default 1500), for the next pt_build
    if (value < 100 || value > 20000) return fail(PT_INVALID_ARG, "pt_set_option: bvh_wide_cost_milli must be in [100, 20000]");
    ctx->c.bvh_params.wide_cost = (float)value / 1000.0f;
    return PT_OK;
  }
  if (k == "bvh_treelet_min") {  // device builder: smallest subtree (triangles) that forms a treelet (default 8)
    if (value < 2 || value > 1 << 20) return fail(PT_INVALID_ARG, "pt_set_option: bvh_treelet_min must be in [2, 2^20]");
    ctx->c.bvh_params.treelet_min = (int)value;
    return PT_OK;
  }
  if (k == "bvh_treelets") {  // device builder: rounds of treelet restructuring (default 3), for the next pt_build
    if (value < 0 || value > 4) return fail(PT_INVALID_ARG, "pt_set_option: bvh_treelets must be in [0, 4]");
    ctx->c.bvh_params.treelet_rounds = (int)value;
    return PT_OK;
  }
  if (k == "bvh_builder") {
    if (value != 0 && value != 1) return fail(PT_INVALID_ARG, "pt_set_option: bvh_builder must be 0 (host SAH) or 1 (device LBVH)");
    ctx->c.bvh_builder = (int)value;
    return PT_OK;
  }
  if (k == "bvh4") {
    if (value != 0 && value != 1) return fail(PT_INVALID_ARG, "pt_set_option: bvh4 must be 0 or 1");
    ctx->c.use_bvh4 = value != 0;
    return PT_OK;
  }
  if (k == "extend_mode") {
    if (value != 0 && value != 1) return fail(PT_INVALID_ARG, "pt_set_option: extend_mode must be 0 or 1");
    ctx->c.opt.extend_mode = (int)value;
  } else if (k == "refill") {
    if (value < 1 || value > 32) return fail(PT_INVALID_ARG, "pt_set_option: refill must be in [1, 32]");
    ctx->c.opt.refill = (int)value;
  } else if (k == "bin_items") {
    if (value != 4 && value != 8 && value != 16) return fail(PT_INVALID_ARG, "pt_set_option: bin_items must be 4, 8 or 16");
    ctx->c.opt.bin_items = (int)value;
  } else if (k == "dual") {
    if (value != 0 && value != 1) return fail(PT_INVALID_ARG, "pt_set_option: dual must be 0 or 1");
    ctx->c.opt.dual = (int)value;
  } else if (k == "overlap") {
    if (value != 0 && value != 1) return fail(PT_INVALID_ARG, "pt_set_option: overlap must be 0 or 1");
    ctx->c.opt.overlap = (int)value;
  } else {
    return fail(PT_INVALID_ARG, "pt_set_option: unknown option " + k);
  }
  return PT_OK;
}

pt_status pt_set_profiling(pt_ctx* ctx, int enable)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  ctx->c.profile = enable != 0;
  return PT_OK;
}

pt_status pt_get_build_info(pt_ctx* ctx, pt_build_info* out)
{
  CTX_CHECK(ctx);
  Context& c = ctx->c;
  if (!out) return fail(PT_INVALID_ARG, "pt_get_build_info: null output");
  if (!c.built) return fail(PT_NOT_READY, "pt_get_build_info: call pt_build first");
  *out = c.build_info;
  // SAH cost of the BVH2 from its child-pair nodes: cost(node) = trav_cost + sum over its two children
  // of area(child) / area(node) * cost(child), a leaf costing its triangle count
  std::vector<float4> nodes(4 * (size_t)c.build_info.bvh2_nodes);
  PT_CHECK_CUDA(cudaMemcpyAsync(nodes.data(), c.d_nodes.p, nodes.size() * sizeof(float4), cudaMemcpyDeviceToHost, c.stream), "pt_get_build_info");
  PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_get_build_info");
  const float trav = c.bvh_params.trav_cost;
  auto area = [](float lx, float hx, float ly, float hy, float lz, float hz) {
    const float dx = std::max(0.0f, hx - lx), dy = std::max(0.0f, hy - ly), dz = std::max(0.0f, hz - lz);
    return (double)(dx * dy + dy * dz + dz * dx);
  };
  // post-order over an explicit stack: cost[node] once both children are done
  std::vector<double> cost(c.build_info.bvh2_nodes, -1.0);
  std::vector<int> stack{0};
  while (!stack.empty()) {
    const int p = stack.back();
    const float4* nd = nodes.data() + 4 * (size_t)p;
    int code[2];
    memcpy(&code[0], &nd[3].x, 4);
    memcpy(&code[1], &nd[3].y, 4);
    bool ready = true;
    for (int k = 0; k < 2; ++k)
      if (code[k] >= 0 && cost[code[k]] < 0.0) {
        if ((uint32_t)code[k] >= c.build_info.bvh2_nodes) return fail(PT_CUDA_ERROR, "pt_get_build_info: malformed BVH");
        stack.push_back(code[k]);
        ready = false;
      }
    if (!ready) continue;
    stack.pop_back();
    const double a0 = area(nd[0].x, nd[0].y, nd[0].z, nd[0].w, nd[2].x, nd[2].y);
    const double a1 = area(nd[1].x, nd[1].y, nd[1].z, nd[1].w, nd[2].z, nd[2].w);
    const double A = area(std::min(nd[0].x, nd[1].x), std::max(nd[0].y, nd[1].y), std::min(nd[0].z, nd[1].z), std::max(nd[0].w, nd[1].w),
                          std::min(nd[2].x, nd[2].z), std::max(nd[2].y, nd[2].w));
    double sum = trav;
    for (int k = 0; k < 2; ++k) {
      const double ck = code[k] >= 0 ? cost[code[k]] : (double)((uint32_t)code[k] & 15u);
      const double ak = k == 0 ? a0 : a1;
      if (A > 0.0 && ak < 1e20) sum += ak / A * ck;
    }
    cost[p] = sum;
  }
  out->sah_cost = (float)cost[0];
  return PT_OK;
}

pt_status pt_trace_closest(pt_ctx* ctx, const float* d_orig_tmin, const float* d_dir_tmax, uint32_t n, int32_t* d_prim, float* d_t, float* d_bary)
{
  CTX_CHECK(ctx);
  Context& c = ctx->c;
  if (!c.built) return fail(PT_NOT_READY, "pt_trace_closest: call pt_build first");
  if (n == 0) return PT_OK;
  if (!d_orig_tmin || !d_dir_tmax || !d_prim || !d_t || !d_bary) return fail(PT_INVALID_ARG, "pt_trace_closest: null pointer");
  k_trace_closest<<<grid_for(n, 128, 16), 128, 0, c.stream>>>(c.view(), (const float4*)d_orig_tmin, (const float4*)d_dir_tmax, n, d_prim, d_t, d_bary);
  count_launch();
  PT_CHECK_CUDA(cudaGetLastError(), "pt_trace_closest launch");
  return PT_OK;
}

pt_status pt_trace_any(pt_ctx* ctx, const float* d_orig_tmin, const float* d_dir_tmax, uint32_t n, int32_t* d_hit)
{
  CTX_CHECK(ctx);
  Context& c = ctx->c;
  if (!c.built) return fail(PT_NOT_READY, "pt_trace_any: call pt_build first");
  if (n == 0) return PT_OK;
  if (!d_orig_tmin || !d_dir_tmax || !d_hit) return fail(PT_INVALID_ARG, "pt_trace_any: null pointer");
  k_trace_any<<<grid_for(n, 128, 16), 128, 0, c.stream>>>(c.view(), (const float4*)d_orig_tmin, (const float4*)d_dir_tmax, n, d_hit);
  count_launch();
  PT_CHECK_CUDA(cudaGetLastError(), "pt_trace_any launch");
  return PT_OK;
}

}  // extern "C"
