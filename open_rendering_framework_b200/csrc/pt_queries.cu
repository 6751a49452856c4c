// Per-query batches of the BSSRDF and of the multiscattering walks: the device functions that the
// shading kernels call (pt_dipole.cuh, pt_math.cuh), one query per thread, so that each can be
// checked against the reference's own functions compiled for the host and against FP64.
//
// pt_bssrdf_queries: the standard dipole reads 4 B and writes 12 B per query, the directional one
// reads 60 B and writes 12 B; both are a handful of expf/sqrtf per query (ALU-light, bandwidth-bound
// at large n).  The FP64 variant derives the coefficients and evaluates the dipole in double.
// pt_microfacet_queries: one random walk per thread (2-4 tea draws and an erf / erfinv per step),
// one kernel instance per (op, distribution) so that a launch holds only the code it runs.
#include <cmath>
#include <cstring>

#include "pt_common.cuh"
#include "pt_context.h"
#include "pt_dipole.cuh"
#include "pt_math.cuh"

namespace pt {

// ------------------------------------------------------------------ FP64 dipoles
// Double 3-vectors for the FP64 evaluation (same formulas and operation order as the FP32 ones).
struct d3 {
  double x, y, z;
};
PT_HD d3 mk(double x, double y, double z) { return d3{x, y, z}; }
PT_HD d3 mks(double s) { return d3{s, s, s}; }
PT_HD d3 operator+(const d3& a, const d3& b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
PT_HD d3 operator-(const d3& a, const d3& b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
PT_HD d3 operator*(const d3& a, const d3& b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
PT_HD d3 operator/(const d3& a, const d3& b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
PT_HD d3 operator*(const d3& a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
PT_HD d3 operator*(double s, const d3& a) { return mk(s * a.x, s * a.y, s * a.z); }
PT_HD d3 operator/(const d3& a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
PT_HD d3 operator/(double s, const d3& a) { return mk(s / a.x, s / a.y, s / a.z); }
PT_HD d3 operator+(const d3& a, double s) { return mk(a.x + s, a.y + s, a.z + s); }
PT_HD d3 operator+(double s, const d3& a) { return mk(s + a.x, s + a.y, s + a.z); }
PT_HD d3 operator-(double s, const d3& a) { return mk(s - a.x, s - a.y, s - a.z); }
PT_HD d3 operator-(const d3& a) { return mk(-a.x, -a.y, -a.z); }
PT_HD double dotd(const d3& a, const d3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PT_HD d3 crossd(const d3& a, const d3& b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
PT_HD d3 normalized(const d3& a) { return a * (1.0 / sqrt(dotd(a, a))); }
PT_HD d3 sqrtd3(const d3& a) { return mk(sqrt(a.x), sqrt(a.y), sqrt(a.z)); }
PT_HD d3 expd3(const d3& a) { return mk(exp(a.x), exp(a.y), exp(a.z)); }
PT_HD d3 maxd3(const d3& a, const d3& b) { return mk(fmax(a.x, b.x), fmax(a.y, b.y), fmax(a.z, b.z)); }

// The fields of ScatteringMaterialProperties (structs.h:116-144) that the dipoles read, in double.
struct ScatD {
  d3 reducedExtinction, D, transport, C_phi, C_E, A, de, three_D, two_A_de, one_over_three_ext;
};

// TranslucentMaterial::computeCoefficients (TranslucentMaterial.cpp:303-330) in double, from the same
// FP32 parameters and with the reference's float constants.
static ScatD compute_coefficients_d(const pt_translucent_params& q)
{
  ScatD p;
  const double sc = q.scale;
  const d3 absorption = mk(q.absorption[0], q.absorption[1], q.absorption[2]) * sc;
  const d3 scattering = mk(q.scattering[0], q.scattering[1], q.scattering[2]) * sc;
  const d3 meancosine = mk(q.meancosine[0], q.meancosine[1], q.meancosine[2]);
  const double n = q.ior;  // ior_rgb = ior / ior_outside with ior_outside = 1
  const d3 reducedScattering = scattering * (1.0 - meancosine);
  const d3 extinction = scattering + absorption;
  p.reducedExtinction = reducedScattering + absorption;
  p.D = 1.0 / (3.0 * p.reducedExtinction);
  p.transport = sqrtd3(absorption / p.D);
  p.C_phi = mks(C_phi_t<double>(n));
  p.C_E = mks(C_E_t<double>(n));
  const d3 reducedAlbedo = reducedScattering / p.reducedExtinction;
  p.de = (double)2.131f * p.D / sqrtd3(reducedAlbedo);
  p.A = (1.0 - p.C_E) / (2.0 * p.C_phi);
  p.three_D = 3.0 * p.D;
  p.two_A_de = 2.0 * p.A * p.de;
  p.one_over_three_ext = 1.0 / (3.0 * extinction);
  return p;
}

// dipole_bssrdf, standard_dipole.h:8-30, in double.
PT_D d3 dipole_bssrdf_d(double dist, const ScatD& P)
{
  d3 real_source = P.three_D * P.three_D;
  d3 extrapolation = 4.0 * P.A * P.D;
  d3 virtual_source = extrapolation * extrapolation;
  d3 corrected_mean_free = P.three_D + extrapolation;
  d3 r_sqr = mks(dist * dist);
  d3 d_r_sqr = r_sqr + real_source;
  d3 d_r = sqrtd3(d_r_sqr);
  d3 d_v_sqr = r_sqr + virtual_source;
  d3 d_v = sqrtd3(d_v_sqr);
  d3 tr_r = P.transport * d_r;
  d3 S_r = P.three_D * (1.0 + tr_r) / (d_r_sqr * d_r) * expd3(-tr_r);
  d3 tr_v = P.transport * d_v;
  d3 S_v = corrected_mean_free * (1.0 + tr_v) / (d_v_sqr * d_v) * expd3(-tr_v);
  return S_r + S_v;
}
// S_infinite_vec, directional_dipole.h:8-34, in double.
PT_D d3 dd_S_infinite_d(const d3& r_sqr, const d3& x_dot_w12, double no_dot_w12, const d3& x_dot_no, const ScatD& P)
{
  d3 r = sqrtd3(r_sqr);
  d3 r_tr = P.transport * r;
  d3 r_tr_p1 = r_tr + 1.0;
  d3 coeff = expd3(-r_tr) / (r * r_sqr);
  d3 first = P.C_phi * (r_sqr * P.reducedExtinction + r_tr_p1 * x_dot_w12) * 3.0;
  d3 second = P.C_E * (P.three_D * r_tr_p1 * no_dot_w12 - (r_tr_p1 + P.three_D * (3.0 * r_tr_p1 + r_tr * r_tr) / r_sqr * x_dot_w12) * x_dot_no);
  return coeff * (first - second);
}
// dirpole_bssrdf, directional_dipole.h:37-72, in double.
PT_D d3 dirpole_bssrdf_d(const d3& xi, const d3& ni, const d3& w12, const d3& xo, const d3& no, const ScatD& P)
{
  d3 x = xo - xi;
  double r_sqr = dotd(x, x);
  double dot_x_w12 = dotd(x, w12);
  d3 cos_beta = -sqrtd3(mks(r_sqr - dot_x_w12 * dot_x_w12) / (r_sqr + P.de * P.de));
  double mu0 = -dotd(no, w12);
  double edge = mu0 > 0.0 ? 1.0 : 0.0;
  d3 D_prime = P.D * mu0 * edge + P.one_over_three_ext * (1.0 - edge);
  d3 dr_sqr = mks(r_sqr) + D_prime * (D_prime - 2.0 * P.de * cos_beta * edge);
  d3 t = normalized(crossd(ni, x));
  d3 nistar = r_sqr < (double)1.0e-12f ? ni : crossd(normalized(x), t);
  d3 wv = w12 - (2.0 * dotd(w12, nistar)) * nistar;
  d3 xr = x - P.two_A_de.x * nistar, xg = x - P.two_A_de.y * nistar, xb = x - P.two_A_de.z * nistar;
  d3 dv_sqr = mk(dotd(xr, xr), dotd(xg, xg), dotd(xb, xb));
  d3 x_dot_wv = mk(dotd(xr, wv), dotd(xg, wv), dotd(xb, wv));
  d3 x_dot_no = mk(dotd(xr, no), dotd(xg, no), dotd(xb, no));
  d3 Sr = dd_S_infinite_d(dr_sqr, mks(dot_x_w12), -mu0, mks(dotd(x, no)), P);
  d3 Sv = dd_S_infinite_d(dv_sqr, x_dot_wv, dotd(no, wv), x_dot_no, P);
  return maxd3(Sr - Sv, mks(0.0));
}

// ------------------------------------------------------------------ BSSRDF kernels
__global__ void __launch_bounds__(256) k_bssrdf_standard(const ScatDev P, const float* __restrict__ dist, uint64_t n, float* __restrict__ S)
{
  const StdDipole t = std_dipole_terms(P);
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    float3 r = dipole_bssrdf(__ldg(dist + k), t);
    S[k] = r.x;
    S[n + k] = r.y;
    S[2 * n + k] = r.z;
  }
}
PT_D float3 ld3soa(const float* __restrict__ in, uint64_t n, uint64_t k, int row)
{
  return f3(__ldg(in + (3 * row) * n + k), __ldg(in + (3 * row + 1) * n + k), __ldg(in + (3 * row + 2) * n + k));
}
__global__ void __launch_bounds__(256) k_bssrdf_directional(const ScatDev P, const float* __restrict__ in, uint64_t n, float* __restrict__ S)
{
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    float3 r = dirpole_bssrdf(ld3soa(in, n, k, 0), ld3soa(in, n, k, 1), ld3soa(in, n, k, 2), ld3soa(in, n, k, 3), ld3soa(in, n, k, 4), P);
    S[k] = r.x;
    S[n + k] = r.y;
    S[2 * n + k] = r.z;
  }
}
__global__ void __launch_bounds__(256) k_bssrdf_standard_d(const ScatD P, const float* __restrict__ dist, uint64_t n, double* __restrict__ S)
{
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    d3 r = dipole_bssrdf_d((double)__ldg(dist + k), P);
    S[k] = r.x;
    S[n + k] = r.y;
    S[2 * n + k] = r.z;
  }
}
PT_D d3 ld3soa_d(const float* __restrict__ in, uint64_t n, uint64_t k, int row)
{
  return mk(__ldg(in + (3 * row) * n + k), __ldg(in + (3 * row + 1) * n + k), __ldg(in + (3 * row + 2) * n + k));
}
__global__ void __launch_bounds__(256) k_bssrdf_directional_d(const ScatD P, const float* __restrict__ in, uint64_t n, double* __restrict__ S)
{
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    d3 r = dirpole_bssrdf_d(ld3soa_d(in, n, k, 0), ld3soa_d(in, n, k, 1), ld3soa_d(in, n, k, 2), ld3soa_d(in, n, k, 3), ld3soa_d(in, n, k, 4),
                            P);
    S[k] = r.x;
    S[n + k] = r.y;
    S[2 * n + k] = r.z;
  }
}

// ------------------------------------------------------------------ walk / conductor-Fresnel kernel
struct MfBatch {
  float3 normal;
  float eta;
  Cx3 ior, inv_ior;
  float3 rho;
};

__device__ unsigned long long g_mf_capped = 0;

template <uint32_t kOp, uint32_t kDist>
__global__ void __launch_bounds__(128) k_microfacet_queries(const MfBatch B, const float* __restrict__ wi_soa, const float* __restrict__ wo_soa,
                                                            const float* __restrict__ alpha, uint32_t* __restrict__ seeds,
                                                            uint32_t* __restrict__ orders, uint64_t n, float* __restrict__ out,
                                                            float* __restrict__ weight)
{
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    const float3 wi = f3(__ldg(wi_soa + k), __ldg(wi_soa + n + k), __ldg(wi_soa + 2 * n + k));
    const float a = __ldg(alpha + k);
    uint32_t seed = seeds[k], order = orders[k];
    int capped = 0;
    float3 r, w = f3s(1.0f);
    if (kOp == PT_MSQ_VISIBLE_NORMAL) {
      const float z1 = rnd_tea(seed);
      const float z2 = rnd_tea(seed);
      r = sample_visible_normal(kDist, wi, B.normal, a, a, z1, z2, &capped);
    } else if (kOp == PT_MSQ_DIELECTRIC_SAMPLE) {
      r = to_world(ms_dielectric_sample(kDist, to_local(wi, B.normal), B.eta, a, a, seed, order, &capped), B.normal);
    } else if (kOp == PT_MSQ_CONDUCTOR_SAMPLE) {
      r = to_world(ms_conductor_sample(kDist, to_local(wi, B.normal), B.ior, B.inv_ior, a, a, seed, order, w, &capped), B.normal);
    } else if (kOp == PT_MSQ_DIFFUSE_SAMPLE) {
      float3 wm;
      r = to_world(ms_diffuse_sample(kDist, to_local(wi, B.normal), a, a, seed, order, w, B.rho, wm, &capped), B.normal);
    } else {
      const float3 wo = f3(__ldg(wo_soa + k), __ldg(wo_soa + n + k), __ldg(wo_soa + 2 * n + k));
      if (kOp == PT_MSQ_DIELECTRIC_EVAL)
        r = f3s(ms_dielectric_eval(kDist, to_local(wi, B.normal), to_local(wo, B.normal), B.eta, a, a, seed, order, &capped));
      else if (kOp == PT_MSQ_CONDUCTOR_EVAL)
        r = ms_conductor_eval(kDist, to_local(wi, B.normal), to_local(wo, B.normal), B.ior, B.inv_ior, a, a, seed, order, &capped);
      else if (kOp == PT_MSQ_DIFFUSE_EVAL)
        r = ms_diffuse_eval(kDist, to_local(wi, B.normal), to_local(wo, B.normal), a, a, seed, B.rho, order, &capped);
      else
        r = fresnel_complex(wi, wo, B.ior);
    }
    seeds[k] = seed;
    orders[k] = order;
    out[k] = r.x;
    out[n + k] = r.y;
    out[2 * n + k] = r.z;
    if (weight) {
      weight[k] = w.x;
      weight[n + k] = w.y;
      weight[2 * n + k] = w.z;
    }
    if (capped) atomicAdd(&g_mf_capped, 1ull);
  }
}

template <uint32_t kOp>
static void launch_mf(uint32_t dist, int grid, cudaStream_t st, const MfBatch& B, const float* wi, const float* wo, const float* alpha,
                      uint32_t* seed, uint32_t* order, uint64_t n, float* out, float* weight)
{
  if (dist == GGX)
    k_microfacet_queries<kOp, GGX><<<grid, 128, 0, st>>>(B, wi, wo, alpha, seed, order, n, out, weight);
  else
    k_microfacet_queries<kOp, BECKMANN><<<grid, 128, 0, st>>>(B, wi, wo, alpha, seed, order, n, out, weight);
}

}  // namespace pt

using namespace pt;

extern "C" {

pt_status pt_bssrdf_queries(const pt_translucent_params* params, uint32_t precision, const float* d_in, uint64_t n, void* d_S, void* stream)
{
  if (!params) return fail(PT_INVALID_ARG, "pt_bssrdf_queries: null parameters");
  if (params->dipole_model > PT_DIRECTIONAL_DIPOLE) return fail(PT_INVALID_ARG, "pt_bssrdf_queries: bad dipole_model");
  if (precision > 1) return fail(PT_INVALID_ARG, "pt_bssrdf_queries: precision must be 0 (FP32) or 1 (FP64)");
  for (int c = 0; c < 3; ++c)
    if (!(params->absorption[c] >= 0.0f && params->scattering[c] > 0.0f && std::isfinite(params->absorption[c]) &&
          std::isfinite(params->scattering[c]) && params->meancosine[c] < 1.0f))
      return fail(PT_INVALID_ARG, "pt_bssrdf_queries: absorption must be >= 0, scattering > 0 and meancosine < 1");
  if (!(params->ior > 0.0f && params->scale > 0.0f)) return fail(PT_INVALID_ARG, "pt_bssrdf_queries: ior and scale must be > 0");
  if (n == 0) return PT_OK;
  if (!d_in || !d_S) return fail(PT_INVALID_ARG, "pt_bssrdf_queries: null pointer");
  const int grid = grid_for(n, 256, 8);
  cudaStream_t st = (cudaStream_t)stream;
  if (precision == 0) {
    const ScatDev P = compute_coefficients(*params);
    if (params->dipole_model == PT_STANDARD_DIPOLE)
      k_bssrdf_standard<<<grid, 256, 0, st>>>(P, d_in, n, (float*)d_S);
    else
      k_bssrdf_directional<<<grid, 256, 0, st>>>(P, d_in, n, (float*)d_S);
  } else {
    const ScatD P = compute_coefficients_d(*params);
    if (params->dipole_model == PT_STANDARD_DIPOLE)
      k_bssrdf_standard_d<<<grid, 256, 0, st>>>(P, d_in, n, (double*)d_S);
    else
      k_bssrdf_directional_d<<<grid, 256, 0, st>>>(P, d_in, n, (double*)d_S);
  }
  count_launch();
  PT_CHECK_CUDA(cudaGetLastError(), "pt_bssrdf_queries launch");
  return PT_OK;
}

pt_status pt_microfacet_queries(const pt_microfacet_batch* batch, const float* d_wi, const float* d_wo, const float* d_alpha, uint32_t* d_seed,
                                uint32_t* d_order, uint64_t n, float* d_out, float* d_weight, void* stream)
{
  if (!batch) return fail(PT_INVALID_ARG, "pt_microfacet_queries: null batch");
  const uint32_t op = batch->op, dist = batch->normal_distribution;
  if (op > PT_MSQ_VISIBLE_NORMAL) return fail(PT_INVALID_ARG, "pt_microfacet_queries: bad op");
  if (dist > PT_GGX_DISTRIBUTION) return fail(PT_INVALID_ARG, "pt_microfacet_queries: bad normal_distribution");
  const float* nv = batch->normal;
  const float nn = nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2];
  if (!(std::isfinite(nn) && fabsf(nn - 1.0f) < 1e-4f)) return fail(PT_INVALID_ARG, "pt_microfacet_queries: normal must be a unit vector");
  if (n == 0) return PT_OK;
  const bool eval = op == PT_MSQ_DIELECTRIC_EVAL || op == PT_MSQ_CONDUCTOR_EVAL || op == PT_MSQ_DIFFUSE_EVAL || op == PT_MSQ_CONDUCTOR_FRESNEL;
  if (!d_wi || !d_alpha || !d_seed || !d_order || !d_out || (eval && !d_wo)) return fail(PT_INVALID_ARG, "pt_microfacet_queries: null pointer");
  MfBatch B;
  B.normal = f3(nv[0], nv[1], nv[2]);
  B.eta = batch->eta;
  B.rho = f3(batch->rho[0], batch->rho[1], batch->rho[2]);
  for (int c = 0; c < 3; ++c) {
    B.ior.c[c] = Cx{batch->ior[2 * c], batch->ior[2 * c + 1]};
    if (op == PT_MSQ_CONDUCTOR_EVAL || op == PT_MSQ_CONDUCTOR_SAMPLE) {
      if (B.ior.c[c].re == 0.0 && B.ior.c[c].im == 0.0) return fail(PT_INVALID_ARG, "pt_microfacet_queries: ior must be non-zero");
      B.inv_ior.c[c] = host_recip(B.ior.c[c]);
    } else {
      B.inv_ior.c[c] = B.ior.c[c];
    }
  }
  const int grid = grid_for(n, 128, 16);
  cudaStream_t st = (cudaStream_t)stream;
  switch (op) {
    case PT_MSQ_DIELECTRIC_EVAL: launch_mf<PT_MSQ_DIELECTRIC_EVAL>(dist, grid, st, B, d_wi, d_wo, d_alpha, d_seed, d_order, n, d_out, d_weight); break;
    case PT_MSQ_DIELECTRIC_SAMPLE: launch_mf<PT_MSQ_DIELECTRIC_SAMPLE>(dist, grid, st, B, d_wi, d_wo, d_alpha, d_seed, d_order, n, d_out, d_weight); break;
    case PT_MSQ_CONDUCTOR_EVAL: launch_mf<PT_MSQ_CONDUCTOR_EVAL>(dist, grid, st, B, d_wi, d_wo, d_alpha, d_seed, d_order, n, d_out, d_weight); break;
    case PT_MSQ_CONDUCTOR_SAMPLE: launch_mf<PT_MSQ_CONDUCTOR_SAMPLE>(dist, grid, st, B, d_wi, d_wo, d_alpha, d_seed, d_order, n, d_out, d_weight); break;
    case PT_MSQ_DIFFUSE_EVAL: launch_mf<PT_MSQ_DIFFUSE_EVAL>(dist, grid, st, B, d_wi, d_wo, d_alpha, d_seed, d_order, n, d_out, d_weight); break;
    case PT_MSQ_DIFFUSE_SAMPLE: launch_mf<PT_MSQ_DIFFUSE_SAMPLE>(dist, grid, st, B, d_wi, d_wo, d_alpha, d_seed, d_order, n, d_out, d_weight); break;
    case PT_MSQ_VISIBLE_NORMAL: launch_mf<PT_MSQ_VISIBLE_NORMAL>(dist, grid, st, B, d_wi, d_wo, d_alpha, d_seed, d_order, n, d_out, d_weight); break;
    default: launch_mf<PT_MSQ_CONDUCTOR_FRESNEL>(dist, grid, st, B, d_wi, d_wo, d_alpha, d_seed, d_order, n, d_out, d_weight); break;
  }
  count_launch();
  PT_CHECK_CUDA(cudaGetLastError(), "pt_microfacet_queries launch");
  return PT_OK;
}

}  // extern "C"
