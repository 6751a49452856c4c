// Test infrastructure (oracle only).  This translation unit compiles the REFERENCE's own
// device-math headers (open_rendering_framework/*.h, included in place from the reference
// tree, never copied) on the host with g++ and exports a plain C interface over them.  It is
// the "reference run here" that pins the oracle restatement under oracle/orc/ and the golden
// fixtures under tests/golden/.  Only tests, the smoke check and the CPU-baseline leg of the
// benchmark load the resulting library (oracle/_ref/libref_oracle.so).
//
// Build: oracle/Makefile target `ref` (needs the reference sources; the built library travels
// with the repository snapshot).
//
// One compile-time workaround, no source edits: structs.h:268 declares `static enum ...`, an
// MSVC-only construct that g++ rejects.  `static` is defined away while structs.h itself is
// parsed (random.h, the only other header it pulls in, is included first so its function-local
// statics are untouched).  All other reference headers compile unmodified against the shim
// under oracle/ref_shim/.
#include <optixu/optixu_math_namespace.h>
#include "random.h"
#define static
#include "structs.h"
#undef static
#include "helpers.h"
#include "sampler.h"
#include "Fresnel.h"
#include "MyComplex.h"
#include "Microfacet.h"
#include "LightSampler.h"
#include "Envmap.h"
#include "dipoles/standard_dipole.h"
#include "dipoles/directional_dipole.h"

#include <cstring>

unsigned long long g_shim_oob_reads = 0;

#define EXPORT extern "C" __attribute__((visibility("default")))

static inline float3 ld3(const float* p) { return make_float3(p[0], p[1], p[2]); }
static inline void st3(float* p, const float3& v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }

EXPORT unsigned long long ref_oob_reads(void) { return g_shim_oob_reads; }
EXPORT int ref_sizeof(const char* name)
{
  if (!strcmp(name, "LightStruct")) return (int)sizeof(LightStruct);
  if (!strcmp(name, "TriangleLight")) return (int)sizeof(TriangleLight);
  if (!strcmp(name, "PositionSample")) return (int)sizeof(PositionSample);
  if (!strcmp(name, "ScatteringMaterialProperties")) return (int)sizeof(ScatteringMaterialProperties);
  if (!strcmp(name, "PerRayData_radiance")) return (int)sizeof(PerRayData_radiance);
  if (!strcmp(name, "MyComplex3")) return (int)sizeof(MyComplex3);
  if (!strcmp(name, "Seed64")) return (int)sizeof(Seed64);
  return -1;
}

// ---------------------------------------------------------------- RNG (random.h, md5.h)
EXPORT unsigned int ref_tea16(unsigned int a, unsigned int b) { return tea<16>(a, b); }
EXPORT void ref_tea16_batch(const unsigned int* a, const unsigned int* b, unsigned int* out, long n)
{
  for (long i = 0; i < n; ++i) out[i] = tea<16>(a[i], b[i]);
}
// n successive rnd_tea draws starting from `seed`; returns the final seed.
EXPORT unsigned int ref_rnd_tea_stream(unsigned int seed, float* out, long n)
{
  for (long i = 0; i < n; ++i) out[i] = rnd_tea(seed);
  return seed;
}
EXPORT unsigned int ref_rnd_lcg_stream(unsigned int seed, float* out, long n)
{
  for (long i = 0; i < n; ++i) out[i] = rnd(seed);
  return seed;
}
// n successive rnd_accurate draws from a 64-bit MD5 seed (x = low word, y = high word).
EXPORT void ref_rnd_md5_stream(unsigned int* sx, unsigned int* sy, float* out, long n)
{
  Seed64 s;
  s.seed = make_uint2(*sx, *sy);
  for (long i = 0; i < n; ++i) out[i] = rnd_accurate(s);
  *sx = s.seed.x;
  *sy = s.seed.y;
}
EXPORT void ref_md5_u2(unsigned int x, unsigned int y, unsigned int scrambler, unsigned int* out4)
{
  uint4 r = rand_md5(make_uint2(x, y), scrambler);
  out4[0] = r.x; out4[1] = r.y; out4[2] = r.z; out4[3] = r.w;
}

// ---------------------------------------------------------------- scalar helpers
EXPORT double ref_erfinv(double x) { return erfinv(x); }
EXPORT float ref_gauss_inv_cdf(float z) { return GaussianHeightInvCDF(z); }
EXPORT float ref_gauss_cdf(float h) { return GaussianHeightCDF(h); }

// ---------------------------------------------------------------- config-1 BSDF query batch
// For each query i: dist = ggx_mask[i] ? GGX : Beckmann; n = (0,0,1);
//   (u1,u2) = two rnd_tea draws from tea<16>(i, 0)           (random.h:117-127)
//   m   = microfacet_sample_visible_normal(wo, n, a, a, u1, u2)  (Microfacet.h:71-82)
//   wi  = reflect(-wo, m)
//   f   = microfacet_eval_BSDF(wo, wi, n, a, eta)              (Microfacet.h:61-69)
//   pdf = microfacet_eval_visible_normal(wo, m, n, a, a) / (4 |wo.m|)  (Microfacet.h:84-96)
//   F   = fresnel_R(wo, m, eta)                                  (Fresnel.h:42-54)
EXPORT void ref_bsdf_queries(long n, long first_index, long n_ggx_below, const float* wo_soa,
                             const float* alpha, float eta, float* wi_soa, float* f, float* pdf,
                             float* F)
{
  const float3 nrm = make_float3(0.0f, 0.0f, 1.0f);
  for (long k = 0; k < n; ++k) {
    long i = first_index + k;
    unsigned int s = tea<16>((unsigned int)i, 0u);
    float u1 = rnd_tea(s);
    float u2 = rnd_tea(s);
    uint dist = (i < n_ggx_below) ? GGX_DISTRIBUTION : BECKMANN_DISTRIBUTION;
    float3 wo = make_float3(wo_soa[k], wo_soa[n + k], wo_soa[2 * n + k]);
    float a = alpha[k];
    float3 m;
    microfacet_sample_visible_normal(wo, nrm, m, a, a, u1, u2, dist);
    float3 wi = reflect(-wo, m);
    f[k] = microfacet_eval_BSDF(wo, wi, nrm, a, eta, dist);
    pdf[k] = microfacet_eval_visible_normal(wo, m, nrm, a, a, dist) / (4.0f * fabsf(dot(wo, m)));
    F[k] = fresnel_R(wo, m, eta);
    wi_soa[k] = wi.x; wi_soa[n + k] = wi.y; wi_soa[2 * n + k] = wi.z;
  }
}

// ---------------------------------------------------------------- microfacet pieces
EXPORT void ref_sample_visible_normal(const float* wi, const float* n, float ax, float ay, float z1,
                                      float z2, unsigned int dist, float* m_out)
{
  float3 m;
  microfacet_sample_visible_normal(ld3(wi), ld3(n), m, ax, ay, z1, z2, dist);
  st3(m_out, m);
}
EXPORT float ref_eval_visible_normal(const float* wi, const float* m, const float* n, float ax,
                                     float ay, unsigned int dist)
{
  return microfacet_eval_visible_normal(ld3(wi), ld3(m), ld3(n), ax, ay, dist);
}
EXPORT void ref_sample_normal(const float* n, float z1, float z2, float alpha, unsigned int dist,
                              float* m_out)
{
  float3 m;
  microfacet_sample_normal(ld3(n), m, z1, z2, alpha, dist);
  st3(m_out, m);
}
EXPORT float ref_masking_G1(const float* v, const float* m, const float* n, float alpha,
                            unsigned int dist)
{
  return masking_G1(ld3(v), ld3(m), ld3(n), alpha, dist);
}
EXPORT float ref_masking_G1_aniso(const float* v, const float* m, const float* n, float ax, float ay,
                                  unsigned int dist)
{
  return masking_G1(ld3(v), ld3(m), ld3(n), ax, ay, dist);
}
EXPORT float ref_eval_bsdf(const float* wi, const float* wo, const float* n, float alpha, float eta,
                           unsigned int dist)
{
  return microfacet_eval_BSDF(ld3(wi), ld3(wo), ld3(n), alpha, eta, dist);
}
EXPORT float ref_fresnel_R_vec(const float* wi, const float* m, float eta)
{
  return fresnel_R(ld3(wi), ld3(m), eta);
}
EXPORT float ref_fresnel_R_cos(float cos_i, float cos_t, float eta) { return fresnel_R(cos_i, cos_t, eta); }

static MyComplex3 ld_c3(const double* c)
{
  MyComplex3 r;
  r.x.real = c[0]; r.x.im = c[1]; r.y.real = c[2]; r.y.im = c[3]; r.z.real = c[4]; r.z.im = c[5];
  return r;
}
// Conductor Fresnel with complex relative IOR `eta` = (re,im) x RGB, as metallic_shader.cu uses it.
EXPORT void ref_fresnel_complex(const float* wi, const float* m, const double* eta6, float* out3)
{
  st3(out3, fresnel_MyComplex_R(ld3(wi), ld3(m), ld_c3(eta6)));
}
// eta = n1 / ior with n1 = 1 (metallic_shader.cu:61).
EXPORT void ref_complex_recip(const double* ior6, double* out6)
{
  MyComplex3 e = 1.0f / ld_c3(ior6);
  out6[0] = e.x.real; out6[1] = e.x.im; out6[2] = e.y.real; out6[3] = e.y.im; out6[4] = e.z.real; out6[5] = e.z.im;
}

// Multiscattering walks (Microfacet.h:95-177).  `seed` is advanced in place.
EXPORT float ref_ms_dielectric_eval(const float* wi, const float* wo, const float* n, float eta, float ax,
                                    float ay, unsigned int* seed, unsigned int order, unsigned int dist)
{
  uint s = *seed;
  float r = microfacet_multiscattering_dielectric_BSDF_eval(ld3(wi), ld3(wo), ld3(n), eta, ax, ay, s, order, dist);
  *seed = s;
  return r;
}
EXPORT void ref_ms_dielectric_sample(const float* wi, const float* n, float eta, float ax, float ay,
                                     unsigned int* seed, unsigned int* order, unsigned int dist, float* wo_out)
{
  uint s = *seed, o = *order;
  float3 wo, weight;
  microfacet_multiscattering_dielectric_BSDF_sample(ld3(wi), wo, ld3(n), eta, ax, ay, s, o, weight, dist);
  *seed = s; *order = o;
  st3(wo_out, wo);
}
EXPORT void ref_ms_conductor_eval(const float* wi, const float* wo, const float* n, const double* eta6,
                                  float ax, float ay, unsigned int* seed, unsigned int order,
                                  unsigned int dist, float* out3)
{
  uint s = *seed;
  float3 r = microfacet_multiscattering_conductor_BSDF_eval(ld3(wi), ld3(wo), ld3(n), ld_c3(eta6), ax, ay, s, order, dist);
  *seed = s;
  st3(out3, r);
}
EXPORT void ref_ms_conductor_sample(const float* wi, const float* n, const double* eta6, float ax, float ay,
                                    unsigned int* seed, unsigned int* order, unsigned int dist, float* wo_out,
                                    float* weight_out)
{
  uint s = *seed, o = *order;
  float3 wo, wm, weight;
  microfacet_multiscattering_conductor_BSDF_sample(ld3(wi), wo, wm, ld3(n), ld_c3(eta6), ax, ay, s, o, weight, dist);
  *seed = s; *order = o;
  st3(wo_out, wo);
  st3(weight_out, weight);
}
EXPORT void ref_ms_diffuse_eval(const float* wi, const float* wo, const float* n, float ax, float ay,
                                unsigned int* seed, unsigned int order, const float* rho, unsigned int dist,
                                float* out3)
{
  uint s = *seed;
  float3 r = microfacet_multiscattering_diffuse_BSDF_eval(ld3(wi), ld3(wo), ld3(n), ax, ay, s, order, ld3(rho), dist);
  *seed = s;
  st3(out3, r);
}
EXPORT void ref_ms_diffuse_sample(const float* wi, const float* n, float ax, float ay, unsigned int* seed,
                                  unsigned int* order, const float* rho, unsigned int dist, float* wo_out,
                                  float* weight_out)
{
  uint s = *seed, o = *order;
  float3 wo, wm, weight;
  microfacet_multiscattering_diffuse_BSDF_sample(ld3(wi), wo, wm, ld3(n), ax, ay, s, o, weight, ld3(rho), dist);
  *seed = s; *order = o;
  st3(wo_out, wo);
  st3(weight_out, weight);
}

// The batch of walk / conductor-Fresnel queries of orc_microfacet_queries_f (same layout and ops), on
// the reference's own functions.
EXPORT void ref_microfacet_queries(unsigned int op, unsigned int dist, const float* n3, float eta, const double* ior6, const float* rho3,
                                   long n, const float* wi, const float* wo, const float* alpha, unsigned int* seed,
                                   unsigned int* order, float* out, float* weight)
{
  for (long k = 0; k < n; ++k) {
    const float a[3] = {wi[k], wi[n + k], wi[2 * n + k]};
    const float b[3] = {wo[k], wo[n + k], wo[2 * n + k]};
    float r[3] = {0.0f, 0.0f, 0.0f}, w[3] = {1.0f, 1.0f, 1.0f};
    switch (op) {
      case 0: r[0] = r[1] = r[2] = ref_ms_dielectric_eval(a, b, n3, eta, alpha[k], alpha[k], seed + k, order[k], dist); break;
      case 1: ref_ms_dielectric_sample(a, n3, eta, alpha[k], alpha[k], seed + k, order + k, dist, r); break;
      case 2: ref_ms_conductor_eval(a, b, n3, ior6, alpha[k], alpha[k], seed + k, order[k], dist, r); break;
      case 3: ref_ms_conductor_sample(a, n3, ior6, alpha[k], alpha[k], seed + k, order + k, dist, r, w); break;
      case 4: ref_ms_diffuse_eval(a, b, n3, alpha[k], alpha[k], seed + k, order[k], rho3, dist, r); break;
      case 5: ref_ms_diffuse_sample(a, n3, alpha[k], alpha[k], seed + k, order + k, rho3, dist, r, w); break;
      case 7: {
        uint s = seed[k];
        const float z1 = rnd_tea(s), z2 = rnd_tea(s);
        seed[k] = s;
        ref_sample_visible_normal(a, n3, alpha[k], alpha[k], z1, z2, dist, r);
        break;
      }
      default: ref_fresnel_complex(a, b, ior6, r); break;
    }
    out[k] = r[0]; out[n + k] = r[1]; out[2 * n + k] = r[2];
    if (weight) { weight[k] = w[0]; weight[n + k] = w[1]; weight[2 * n + k] = w[2]; }
  }
}

// ---------------------------------------------------------------- sampling helpers
EXPORT void ref_sample_cosine_weighted(const float* n, unsigned int* seed, float* out3)
{
  uint s = *seed;
  st3(out3, sample_cosine_weighted(ld3(n), s));
  *seed = s;
}
EXPORT void ref_sample_barycentric(unsigned int* seed, float* out3)
{
  uint s = *seed;
  st3(out3, sample_barycentric(s));
  *seed = s;
}
EXPORT void ref_create_onb(const float* n, float* u, float* v)
{
  float3 U, V;
  create_onb(ld3(n), U, V);
  st3(u, U); st3(v, V);
}

// ---------------------------------------------------------------- lights (LightSampler.h)
EXPORT void ref_set_light_buffers(void* lights, long n_lights, void* tri_lights, long n_tri)
{
  light_buffer.data = (LightStruct*)lights;
  light_buffer.n = (size_t)n_lights;
  triangle_light_buffer.data = (TriangleLight*)tri_lights;
  triangle_light_buffer.n = (size_t)n_tri;
}
// evaluate_direct_illumination for light `light_idx` at `pos` (LightSampler.h:143-166).
EXPORT void ref_direct_illumination(const float* pos, long light_idx, unsigned int* seed, float* dir3,
                                    float* L3, float* dist)
{
  uint s = *seed;
  LightStruct l = light_buffer[(size_t)light_idx];
  float3 dir = make_float3(0.0f), L = make_float3(0.0f);
  float d = 0.0f;
  evaluate_direct_illumination(ld3(pos), &l, dir, L, d, s);
  *seed = s;
  st3(dir3, dir); st3(L3, L);
  *dist = d;
}

// ---------------------------------------------------------------- environment map (Envmap.h)
EXPORT void ref_set_envmap(const float* rgba, int w, int h, float* marginal_pdf_p, float* marginal_cdf_p,
                           float* conditional_pdf_p, float* conditional_cdf_p)
{
  envmap.texels = (const float4*)rgba;
  envmap.w = w;
  envmap.h = h;
  marginal_pdf.data = marginal_pdf_p; marginal_pdf.n = (size_t)h;
  marginal_cdf.data = marginal_cdf_p; marginal_cdf.n = (size_t)h;
  conditional_pdf.data = conditional_pdf_p; conditional_pdf.nx = (size_t)w; conditional_pdf.ny = (size_t)h;
  conditional_cdf.data = conditional_cdf_p; conditional_cdf.nx = (size_t)w; conditional_cdf.ny = (size_t)h;
}
EXPORT void ref_env_lookup(const float* dir, float* out3) { st3(out3, env_lookup(ld3(dir))); }
EXPORT void ref_sample_environment(const float* pos, unsigned int* seed, float* dir3, float* L3)
{
  uint s = *seed;
  float3 dir, L;
  sample_environment(ld3(pos), dir, L, s);
  *seed = s;
  st3(dir3, dir); st3(L3, L);
}
EXPORT unsigned int ref_cdf_bsearch_marginal(float xi) { return cdf_bsearch_marginal(xi); }
EXPORT unsigned int ref_cdf_bsearch_conditional(float xi, unsigned int row) { return cdf_bsearch_conditional(xi, row); }

// ---------------------------------------------------------------- dipoles
static ScatteringMaterialProperties g_props;
EXPORT void ref_set_scattering_properties(const void* props, long size)
{
  if (size == (long)sizeof(ScatteringMaterialProperties)) memcpy(&g_props, props, sizeof(g_props));
}
EXPORT void ref_dipole_bssrdf(float dist, float* out3) { st3(out3, dipole_bssrdf(dist, g_props)); }
EXPORT void ref_dirpole_bssrdf(const float* xi, const float* ni, const float* w12, const float* xo,
                               const float* no, float* out3)
{
  st3(out3, dirpole_bssrdf(ld3(xi), ld3(ni), ld3(w12), ld3(xo), ld3(no), g_props));
}
// A batch of BSSRDF queries on the properties set last: standard dipole (model 0) on dist[n], or the
// directional dipole (model 1) on 15 x n SoA geometry (xi, ni, w12, xo, no); S is 3 x n SoA.
EXPORT void ref_bssrdf_queries(unsigned int model, long n, const float* in, float* S)
{
  for (long k = 0; k < n; ++k) {
    float3 r;
    if (model == 0) {
      r = dipole_bssrdf(in[k], g_props);
    } else {
      float3 v[5];
      for (int j = 0; j < 5; ++j) v[j] = make_float3(in[(3 * j) * n + k], in[(3 * j + 1) * n + k], in[(3 * j + 2) * n + k]);
      r = dirpole_bssrdf(v[0], v[1], v[2], v[3], v[4], g_props);
    }
    S[k] = r.x; S[n + k] = r.y; S[2 * n + k] = r.z;
  }
}
EXPORT float ref_C_phi(float n) { return C_phi(n); }
EXPORT float ref_C_E(float n) { return C_E(n); }
