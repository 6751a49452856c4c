// Test infrastructure (oracle only): C interface over the oracle restatement's math, exported in
// an FP32 instantiation (`orc_*_f`, bit-identical to the compiled reference) and an FP64
// instantiation (`orc_*_d`, the error yardstick).  Loaded only by tests, the smoke check and the
// CPU-baseline leg of the benchmark (oracle/liboracle.so).
#include "orc_math.hpp"
#include "orc_microfacet.hpp"
#include "orc_light.hpp"

#include <cstring>
#include <thread>
#include <vector>

using namespace orc;

#define EXPORT extern "C" __attribute__((visibility("default")))

template <class R> static inline V3<R> ld(const float* p) { return v3((R)p[0], (R)p[1], (R)p[2]); }
template <class R> static inline V3<R> ldd(const double* p) { return v3((R)p[0], (R)p[1], (R)p[2]); }
template <class R, class T> static inline void st(T* p, const V3<R>& v) { p[0] = (T)v.x; p[1] = (T)v.y; p[2] = (T)v.z; }

// --------------------------------------------------------------------------- RNG
EXPORT unsigned int orc_tea16(unsigned int a, unsigned int b) { return tea<16>(a, b); }
EXPORT unsigned int orc_rnd_tea_stream(unsigned int seed, float* out, long n)
{
  for (long i = 0; i < n; ++i) out[i] = rnd_tea(seed);
  return seed;
}
EXPORT unsigned int orc_rnd_lcg_stream(unsigned int seed, float* out, long n)
{
  for (long i = 0; i < n; ++i) out[i] = rnd(seed);
  return seed;
}
EXPORT void orc_rnd_md5_stream(unsigned int* sx, unsigned int* sy, float* out, long n)
{
  Seed64 s = {*sx, *sy};
  for (long i = 0; i < n; ++i) out[i] = rnd_accurate(s);
  *sx = s.x;
  *sy = s.y;
}
EXPORT void orc_md5_u2(unsigned int x, unsigned int y, unsigned int* out4) { md5_u2(x, y, out4); }
EXPORT double orc_erfinv(double x) { return erfinv_d(x); }

// --------------------------------------------------------------------------- config-1 BSDF queries
// Same definition as ref_bsdf_queries in oracle/ref_driver.cpp (query i: GGX when i < n_ggx_below,
// (u1,u2) = two rnd_tea draws from tea<16>(i,0), n = +z).  Multi-threaded over `threads`.
template <class R, class T>
static void bsdf_queries(long n, long first, long n_ggx_below, const float* wo_soa, const float* alpha, float eta, T* wi_soa,
                         T* f, T* pdf, T* F, int threads)
{
  auto work = [&](long b, long e) {
    const V3<R> nrm = v3(R(0), R(0), R(1));
    for (long k = b; k < e; ++k) {
      long i = first + k;
      u32 s = tea<16>((u32)i, 0u);
      R u1 = (R)rnd_tea(s), u2 = (R)rnd_tea(s);
      int dist = (i < n_ggx_below) ? GGX : BECKMANN;
      V3<R> wo = v3((R)wo_soa[k], (R)wo_soa[n + k], (R)wo_soa[2 * n + k]);
      R a = (R)alpha[k], e_r = (R)eta;
      V3<R> m = sample_visible_normal(dist, wo, nrm, a, a, u1, u2);
      V3<R> wi = reflect(-wo, m);
      f[k] = (T)walter_bsdf(dist, wo, wi, nrm, a, e_r);
      pdf[k] = (T)(eval_visible_normal(dist, wo, m, nrm, a, a) / (R(4) * std::fabs(dot(wo, m))));
      F[k] = (T)fresnel_R(wo, m, e_r);
      wi_soa[k] = (T)wi.x; wi_soa[n + k] = (T)wi.y; wi_soa[2 * n + k] = (T)wi.z;
    }
  };
  if (threads <= 1 || n < 4096) { work(0, n); return; }
  std::vector<std::thread> th;
  long chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    long b = t * chunk, e = std::min(n, b + chunk);
    if (b < e) th.emplace_back(work, b, e);
  }
  for (auto& x : th) x.join();
}
EXPORT void orc_bsdf_queries_f(long n, long first, long n_ggx_below, const float* wo, const float* alpha, float eta, float* wi,
                               float* f, float* pdf, float* F, int threads)
{
  bsdf_queries<float, float>(n, first, n_ggx_below, wo, alpha, eta, wi, f, pdf, F, threads);
}
EXPORT void orc_bsdf_queries_d(long n, long first, long n_ggx_below, const float* wo, const float* alpha, float eta, double* wi,
                               double* f, double* pdf, double* F, int threads)
{
  bsdf_queries<double, double>(n, first, n_ggx_below, wo, alpha, eta, wi, f, pdf, F, threads);
}

// Synthetic config-1 inputs: alpha = 0.05 + 0.95 u, cos(theta_o) = 0.01 + 0.99 u, phi = 2 pi u with
// u drawn by rnd_tea from tea<16>(i, 1); wo = (sin cos(phi), sin sin(phi), cos).  Identical to the
// generator in the product library (pt_c1_make_inputs), restated here so tests can check it.
EXPORT void orc_c1_make_inputs(long n, long first, float* wo_soa, float* alpha)
{
  for (long k = 0; k < n; ++k) {
    u32 s = tea<16>((u32)(first + k), 1u);
    float a = 0.05f + 0.95f * rnd_tea(s);
    float ct = 0.01f + 0.99f * rnd_tea(s);
    float phi = 2.0f * 3.14159265358979323846f * rnd_tea(s);
    float st = sqrtf(1.0f - ct * ct);
    alpha[k] = a;
    wo_soa[k] = st * cosf(phi);
    wo_soa[n + k] = st * sinf(phi);
    wo_soa[2 * n + k] = ct;
  }
}

// --------------------------------------------------------------------------- microfacet pieces
EXPORT void orc_sample_visible_normal_f(const float* wi, const float* n, float ax, float ay, float z1, float z2, unsigned dist, float* m)
{
  st(m, sample_visible_normal<float>((int)dist, ld<float>(wi), ld<float>(n), ax, ay, z1, z2));
}
EXPORT void orc_sample_visible_normal_d(const float* wi, const float* n, float ax, float ay, float z1, float z2, unsigned dist, double* m)
{
  st(m, sample_visible_normal<double>((int)dist, ld<double>(wi), ld<double>(n), ax, ay, z1, z2));
}
EXPORT float orc_eval_visible_normal_f(const float* wi, const float* m, const float* n, float ax, float ay, unsigned dist)
{
  return eval_visible_normal<float>((int)dist, ld<float>(wi), ld<float>(m), ld<float>(n), ax, ay);
}
EXPORT void orc_sample_normal_f(const float* n, float z1, float z2, float alpha, unsigned dist, float* m)
{
  st(m, sample_normal<float>((int)dist, ld<float>(n), z1, z2, alpha));
}
EXPORT float orc_masking_G1_f(const float* v, const float* m, const float* n, float alpha, unsigned dist)
{
  return masking_G1<float>((int)dist, ld<float>(v), ld<float>(m), ld<float>(n), alpha);
}
EXPORT float orc_masking_G1_aniso_f(const float* v, const float* m, const float* n, float ax, float ay, unsigned dist)
{
  return masking_G1_aniso<float>((int)dist, ld<float>(v), ld<float>(m), ld<float>(n), ax, ay);
}
EXPORT float orc_eval_bsdf_f(const float* wi, const float* wo, const float* n, float alpha, float eta, unsigned dist)
{
  return walter_bsdf<float>((int)dist, ld<float>(wi), ld<float>(wo), ld<float>(n), alpha, eta);
}
EXPORT double orc_eval_bsdf_d(const float* wi, const float* wo, const float* n, float alpha, float eta, unsigned dist)
{
  return walter_bsdf<double>((int)dist, ld<double>(wi), ld<double>(wo), ld<double>(n), alpha, eta);
}
EXPORT float orc_fresnel_R_vec_f(const float* wi, const float* m, float eta) { return fresnel_R<float>(ld<float>(wi), ld<float>(m), eta); }

static Cx3 ldc(const double* c)
{
  Cx3 r = {{c[0], c[1]}, {c[2], c[3]}, {c[4], c[5]}};
  return r;
}
EXPORT void orc_fresnel_complex_f(const float* wi, const float* m, const double* eta6, float* out3)
{
  st(out3, fresnel_complex<float>(ld<float>(wi), ld<float>(m), ldc(eta6)));
}
EXPORT void orc_fresnel_complex_d(const float* wi, const float* m, const double* eta6, double* out3)
{
  st(out3, fresnel_complex<double>(ld<double>(wi), ld<double>(m), ldc(eta6)));
}
EXPORT void orc_complex_recip_f(const double* ior6, double* out6)
{
  Cx3 e = crecip3<float>(ldc(ior6));
  out6[0] = e.x.re; out6[1] = e.x.im; out6[2] = e.y.re; out6[3] = e.y.im; out6[4] = e.z.re; out6[5] = e.z.im;
}

// Multiscattering walks in the shading frame of normal n (Microfacet.h:95-177).
template <class R> static R ms_diel_eval(const float* wi, const float* wo, const float* n, float eta, float ax, float ay, unsigned* seed,
                                         unsigned order, unsigned dist)
{
  u32 s = *seed;
  V3<R> nn = ld<R>(n);
  int capped = 0;
  R r = ms_dielectric_eval<R>((int)dist, to_local(ld<R>(wi), nn), to_local(ld<R>(wo), nn), (R)eta, (R)ax, (R)ay, s, order, 1 << 24, &capped);
  *seed = s;
  return r;
}
EXPORT float orc_ms_dielectric_eval_f(const float* wi, const float* wo, const float* n, float eta, float ax, float ay, unsigned* seed,
                                      unsigned order, unsigned dist)
{
  return ms_diel_eval<float>(wi, wo, n, eta, ax, ay, seed, order, dist);
}
EXPORT double orc_ms_dielectric_eval_d(const float* wi, const float* wo, const float* n, float eta, float ax, float ay, unsigned* seed,
                                       unsigned order, unsigned dist)
{
  return ms_diel_eval<double>(wi, wo, n, eta, ax, ay, seed, order, dist);
}
EXPORT void orc_ms_dielectric_sample_f(const float* wi, const float* n, float eta, float ax, float ay, unsigned* seed, unsigned* order,
                                       unsigned dist, float* wo_out)
{
  u32 s = *seed, o = *order;
  V3<float> nn = ld<float>(n);
  int capped = 0;
  V3<float> lwo = ms_dielectric_sample<float>((int)dist, to_local(ld<float>(wi), nn), eta, ax, ay, s, o, 1 << 24, &capped);
  *seed = s; *order = o;
  st(wo_out, to_world(lwo, nn));
}
EXPORT void orc_ms_conductor_eval_f(const float* wi, const float* wo, const float* n, const double* eta6, float ax, float ay, unsigned* seed,
                                    unsigned order, unsigned dist, float* out3)
{
  u32 s = *seed;
  V3<float> nn = ld<float>(n);
  Cx3 e = ldc(eta6), ie = crecip3<float>(e);
  int capped = 0;
  st(out3, ms_conductor_eval<float>((int)dist, to_local(ld<float>(wi), nn), to_local(ld<float>(wo), nn), e, ie, ax, ay, s, order, 1 << 24, &capped));
  *seed = s;
}
EXPORT void orc_ms_conductor_sample_f(const float* wi, const float* n, const double* eta6, float ax, float ay, unsigned* seed, unsigned* order,
                                      unsigned dist, float* wo_out, float* weight_out)
{
  u32 s = *seed, o = *order;
  V3<float> nn = ld<float>(n), wm, weight;
  Cx3 e = ldc(eta6), ie = crecip3<float>(e);
  int capped = 0;
  V3<float> lwo = ms_conductor_sample<float>((int)dist, to_local(ld<float>(wi), nn), wm, e, ie, ax, ay, s, o, weight, 1 << 24, &capped);
  *seed = s; *order = o;
  st(wo_out, to_world(lwo, nn));
  st(weight_out, weight);
}
EXPORT void orc_ms_diffuse_eval_f(const float* wi, const float* wo, const float* n, float ax, float ay, unsigned* seed, unsigned order,
                                  const float* rho, unsigned dist, float* out3)
{
  u32 s = *seed;
  V3<float> nn = ld<float>(n);
  int capped = 0;
  st(out3, ms_diffuse_eval<float>((int)dist, to_local(ld<float>(wi), nn), to_local(ld<float>(wo), nn), ax, ay, s, ld<float>(rho), order, 1 << 24, &capped));
  *seed = s;
}
EXPORT void orc_ms_diffuse_sample_f(const float* wi, const float* n, float ax, float ay, unsigned* seed, unsigned* order, const float* rho,
                                    unsigned dist, float* wo_out, float* weight_out)
{
  u32 s = *seed, o = *order;
  V3<float> nn = ld<float>(n), wm, weight;
  V3<float> lwo = ms_diffuse_sample<float>((int)dist, to_local(ld<float>(wi), nn), wm, ax, ay, s, o, weight, ld<float>(rho));
  *seed = s; *order = o;
  st(wo_out, to_world(lwo, nn));
  st(weight_out, weight);
}

// --------------------------------------------------------------------------- sampling helpers, lights
EXPORT void orc_sample_cosine_weighted_f(const float* n, unsigned* seed, float* out3)
{
  u32 s = *seed;
  st(out3, sample_cosine_weighted<float>(ld<float>(n), s));
  *seed = s;
}
EXPORT void orc_sample_barycentric_f(unsigned* seed, float* out3)
{
  u32 s = *seed;
  st(out3, sample_barycentric<float>(s));
  *seed = s;
}
EXPORT void orc_create_onb_f(const float* n, float* u, float* v)
{
  V3<float> U, V;
  create_onb(ld<float>(n), U, V);
  st(u, U); st(v, V);
}
EXPORT void orc_direct_illumination_f(const float* pos, const void* lights, long n_lights, const void* tris, long n_tris, long light_idx,
                                      unsigned* seed, float* dir3, float* L3, float* dist)
{
  LightSet set;
  set.lights = (const LightStructRaw*)lights; set.n_lights = n_lights;
  set.tris = (const TriangleLightRaw*)tris; set.n_tris = n_tris;
  u32 s = *seed;
  V3<float> dir = v3s(0.0f), L = v3s(0.0f);
  float d = 0.0f;
  eval_direct<float>(ld<float>(pos), set.lights[light_idx], set, dir, L, d, s);
  *seed = s;
  st(dir3, dir); st(L3, L);
  *dist = d;
}
EXPORT float orc_C_phi_f(float n) { return C_phi<float>(n); }
EXPORT float orc_C_E_f(float n) { return C_E<float>(n); }

// --------------------------------------------------------------------------- batched walk queries
// A batch of multiscattering-walk or conductor-Fresnel queries in the frame of the normal n3, the
// calls the shaders make (Microfacet.h:95-177 in the world frame; Fresnel.h:78-91).  SoA inputs
// wi[3][n], wo[3][n] (the evaluated direction; the microfacet normal for op 6), alpha[n] (ax = ay),
// seed[n] (advanced in place), order[n] (the eval ops read it; the sample ops add the walk's
// scattering events to it).  Outputs out[3][n]: the value (dielectric eval: the scalar in all three
// channels), the sampled direction (sample ops) or F (op 6); weight[3][n]: the sample ops' weight
// (conductor, diffuse).  ops: 0 dielectric eval, 1 dielectric sample, 2 conductor eval, 3 conductor
// sample, 4 diffuse eval, 5 diffuse sample, 6 conductor Fresnel, 7 visible-normal sample with (z1, z2)
// two rnd_tea draws from the seed.
template <class R>
static void mf_batch(unsigned op, unsigned dist, const float* n3, float eta, const double* ior6, const float* rho3, long n, const float* wi,
                     const float* wo, const float* alpha, unsigned* seed, unsigned* order, R* out, R* weight, int threads)
{
  const V3<R> nn = ld<R>(n3);
  const Cx3 e = ldc(ior6), ie = crecip3<R>(e);
  const V3<R> rho = ld<R>(rho3);
  auto work = [&](long k0, long k1) {
    for (long k = k0; k < k1; ++k) {
      const V3<R> a = v3((R)wi[k], (R)wi[n + k], (R)wi[2 * n + k]);
      const V3<R> b = v3((R)wo[k], (R)wo[n + k], (R)wo[2 * n + k]);
      const R al = (R)alpha[k];
      u32 s = seed[k], o = order[k];
      int capped = 0;
      V3<R> r = v3s(R(0)), w = v3s(R(1)), wm;
      switch (op) {
        case 0: r = v3s(ms_dielectric_eval<R>((int)dist, to_local(a, nn), to_local(b, nn), (R)eta, al, al, s, o, 1 << 24, &capped)); break;
        case 1: r = to_world(ms_dielectric_sample<R>((int)dist, to_local(a, nn), (R)eta, al, al, s, o, 1 << 24, &capped), nn); break;
        case 2: r = ms_conductor_eval<R>((int)dist, to_local(a, nn), to_local(b, nn), e, ie, al, al, s, o, 1 << 24, &capped); break;
        case 3: r = to_world(ms_conductor_sample<R>((int)dist, to_local(a, nn), wm, e, ie, al, al, s, o, w, 1 << 24, &capped), nn); break;
        case 4: r = ms_diffuse_eval<R>((int)dist, to_local(a, nn), to_local(b, nn), al, al, s, rho, o, 1 << 24, &capped); break;
        case 5: r = to_world(ms_diffuse_sample<R>((int)dist, to_local(a, nn), wm, al, al, s, o, w, rho), nn); break;
        case 7: {
          const R z1 = (R)rnd_tea(s), z2 = (R)rnd_tea(s);
          r = sample_visible_normal<R>((int)dist, a, nn, al, al, z1, z2);
          break;
        }
        default: r = fresnel_complex<R>(a, b, e); break;
      }
      seed[k] = s;
      order[k] = o;
      out[k] = r.x; out[n + k] = r.y; out[2 * n + k] = r.z;
      if (weight) { weight[k] = w.x; weight[n + k] = w.y; weight[2 * n + k] = w.z; }
    }
  };
  if (threads <= 1 || n < 1024) { work(0, n); return; }
  std::vector<std::thread> th;
  long chunk = (n + threads - 1) / threads;
  for (int t = 0; t < threads; ++t) {
    long k0 = t * chunk, k1 = std::min(n, k0 + chunk);
    if (k0 < k1) th.emplace_back(work, k0, k1);
  }
  for (auto& x : th) x.join();
}
EXPORT void orc_microfacet_queries_f(unsigned op, unsigned dist, const float* n3, float eta, const double* ior6, const float* rho3, long n,
                                     const float* wi, const float* wo, const float* alpha, unsigned* seed, unsigned* order, float* out,
                                     float* weight, int threads)
{
  mf_batch<float>(op, dist, n3, eta, ior6, rho3, n, wi, wo, alpha, seed, order, out, weight, threads);
}
EXPORT void orc_microfacet_queries_d(unsigned op, unsigned dist, const float* n3, float eta, const double* ior6, const float* rho3, long n,
                                     const float* wi, const float* wo, const float* alpha, unsigned* seed, unsigned* order, double* out,
                                     double* weight, int threads)
{
  mf_batch<double>(op, dist, n3, eta, ior6, rho3, n, wi, wo, alpha, seed, order, out, weight, threads);
}

// The config-1 composition of bsdf_queries with the microfacet normal given instead of sampled:
// wi = reflect(-wo, m), f, pdf and F as there (FP32).  Used to trace a query whose GPU result differs
// from the oracle back to the sampled normal.
EXPORT void orc_bsdf_given_m_f(long n, const int* dist_of, const float* wo_soa, const float* alpha, float eta, const float* m_soa,
                               float* wi_soa, float* f, float* pdf, float* F)
{
  const V3<float> nrm = v3(0.0f, 0.0f, 1.0f);
  for (long k = 0; k < n; ++k) {
    const int dist = dist_of[k];
    V3<float> wo = v3(wo_soa[k], wo_soa[n + k], wo_soa[2 * n + k]);
    V3<float> m = v3(m_soa[k], m_soa[n + k], m_soa[2 * n + k]);
    const float a = alpha[k];
    V3<float> wi = reflect(-wo, m);
    f[k] = walter_bsdf(dist, wo, wi, nrm, a, eta);
    pdf[k] = eval_visible_normal(dist, wo, m, nrm, a, a) / (4.0f * std::fabs(dot(wo, m)));
    F[k] = fresnel_R(wo, m, eta);
    wi_soa[k] = wi.x; wi_soa[n + k] = wi.y; wi_soa[2 * n + k] = wi.z;
  }
}
