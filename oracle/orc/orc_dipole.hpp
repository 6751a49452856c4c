// Test infrastructure (oracle only): restatement of the dipole BSSRDFs (dipoles/standard_dipole.h,
// dipoles/directional_dipole.h) and of the scattering coefficients of
// TranslucentMaterial::computeCoefficients (TranslucentMaterial.cpp:303-330), in FP32 with the
// reference's operation order.
#pragma once
#include "orc_math.hpp"

namespace orc {

// ScatteringMaterialProperties, structs.h:116-144 (260 bytes).
struct ScatProps {
  float relative_ior;
  V3<float> ior_real, ior_imag, absorption, scattering, meancosine, extinction, reducedExtinction, deltaEddExtinction, D, transport,
      C_phi, C_phi_inv, C_E, A, albedo, reducedAlbedo, de, three_D, two_A_de, global_coeff, one_over_three_ext;
  float mean_transport;
};
static_assert(sizeof(ScatProps) == 260, "ScatteringMaterialProperties layout");

typedef V3<float> F3v;
static inline F3v sqrt3(const F3v& v) { return v3(std::sqrt(v.x), std::sqrt(v.y), std::sqrt(v.z)); }

// TranslucentMaterial::computeCoefficients with ior_outside = (1,1,1) (TranslucentMaterial.cpp:303-330).
static inline ScatProps compute_coefficients(const float* absorption, const float* scattering, const float* meancosine, float ior, float scale)
{
  ScatProps p;
  memset(&p, 0, sizeof(p));
  const F3v ior_outside = v3(1.0f, 1.0f, 1.0f);
  p.absorption = v3(absorption[0], absorption[1], absorption[2]) * scale;
  p.scattering = v3(scattering[0], scattering[1], scattering[2]) * scale;
  p.meancosine = v3(meancosine[0], meancosine[1], meancosine[2]);
  p.relative_ior = ior;
  p.ior_real = v3s(ior);
  F3v ior_rgb = p.ior_real / ior_outside;
  F3v reducedScattering = p.scattering * (1.0f - p.meancosine);
  p.relative_ior /= (ior_outside.x + ior_outside.y + ior_outside.z) / 3.0f;
  p.ior_real = ior_rgb;
  p.extinction = p.scattering + p.absorption;
  p.reducedExtinction = reducedScattering + p.absorption;
  p.deltaEddExtinction = p.scattering * (1.0f - p.meancosine * p.meancosine) + p.absorption;
  p.D = v3s(1.0f) / (3.0f * p.reducedExtinction);
  p.transport = sqrt3(p.absorption / p.D);
  p.C_phi = v3(C_phi<float>(ior_rgb.x), C_phi<float>(ior_rgb.y), C_phi<float>(ior_rgb.z));
  p.C_phi_inv = v3(C_phi<float>(1.0f / ior_rgb.x), C_phi<float>(1.0f / ior_rgb.y), C_phi<float>(1.0f / ior_rgb.z));
  p.C_E = v3(C_E<float>(ior_rgb.x), C_E<float>(ior_rgb.y), C_E<float>(ior_rgb.z));
  p.albedo = p.scattering / p.extinction;
  p.reducedAlbedo = reducedScattering / p.reducedExtinction;
  p.de = 2.131f * p.D / sqrt3(p.reducedAlbedo);
  p.A = (1.0f - p.C_E) / (2.0f * p.C_phi);
  p.three_D = 3.0f * p.D;
  p.two_A_de = 2.0f * p.A * p.de;
  p.global_coeff = v3s(1.0f) / (4.0f * p.C_phi_inv) * 1.0f / (4.0f * K<float>::PI * K<float>::PI);
  p.one_over_three_ext = v3s((float)1.0) / (3.0f * p.extinction);
  p.mean_transport = (p.transport.x + p.transport.y + p.transport.z) / 3.0f;
  return p;
}

// dipole_bssrdf, standard_dipole.h:8-30.
static inline F3v dipole_bssrdf(float dist, const ScatProps& P)
{
  F3v real_source = P.three_D * P.three_D;
  F3v extrapolation = 4.0f * P.A * P.D;
  F3v virtual_source = extrapolation * extrapolation;
  F3v corrected_mean_free = P.three_D + extrapolation;
  F3v r_sqr = v3s(dist * dist);
  F3v d_r_sqr = r_sqr + real_source;
  F3v d_r = v3(std::sqrt(d_r_sqr.x), std::sqrt(d_r_sqr.y), std::sqrt(d_r_sqr.z));
  F3v d_v_sqr = r_sqr + virtual_source;
  F3v d_v = v3(std::sqrt(d_v_sqr.x), std::sqrt(d_v_sqr.y), std::sqrt(d_v_sqr.z));
  F3v tr_r = P.transport * d_r;
  F3v S_r = P.three_D * (1.0f + tr_r) / (d_r_sqr * d_r);
  S_r = S_r * vexp(-tr_r);
  F3v tr_v = P.transport * d_v;
  F3v S_v = corrected_mean_free * (1.0f + tr_v) / (d_v_sqr * d_v);
  S_v = S_v * vexp(-tr_v);
  return S_r + S_v;
}

// S_infinite / S_infinite_vec, directional_dipole.h:8-34.
static inline F3v S_infinite(const F3v& r_sqr, const F3v& x_dot_w12, const float no_dot_w12, const F3v& x_dot_no, const ScatProps& P)
{
  F3v r = sqrt3(r_sqr);
  F3v r_tr = P.transport * r;
  F3v r_tr_p1 = r_tr + 1.0f;
  F3v T = vexp(-r_tr);
  F3v coeff = T / (r * r_sqr);
  F3v first = P.C_phi * (r_sqr * P.reducedExtinction + r_tr_p1 * x_dot_w12) * 3.0f;
  F3v second = P.C_E * (P.three_D * r_tr_p1 * no_dot_w12 - (r_tr_p1 + P.three_D * (3.0f * r_tr_p1 + r_tr * r_tr) / r_sqr * x_dot_w12) * x_dot_no);
  return coeff * (first - second);
}
// dirpole_bssrdf, directional_dipole.h:37-72.
static inline F3v dirpole_bssrdf(const F3v& xi, const F3v& ni, const F3v& w12, const F3v& xo, const F3v& no, const ScatProps& P)
{
  F3v x = xo - xi;
  float r_sqr = dot(x, x);
  F3v dr_sqr = v3s(r_sqr);
  float dot_x_w12 = dot(x, w12);
  F3v cos_beta = -sqrt3(v3s(r_sqr - dot_x_w12 * dot_x_w12) / (r_sqr + P.de * P.de));
  float mu0 = -dot(no, w12);
  float edge = mu0 > 0.0f ? 1.0f : 0.0f;
  F3v D_prime = P.D * mu0 * edge + P.one_over_three_ext * (1.0f - edge);
  dr_sqr = dr_sqr + D_prime * (D_prime - 2.0f * P.de * cos_beta * edge);
  F3v t = normalize(cross(ni, x));
  F3v nistar = r_sqr < 1.0e-12f ? ni : cross(normalize(x), t);
  F3v wv = w12 - (2.0f * dot(w12, nistar)) * nistar;
  F3v xoxv_r = x - P.two_A_de.x * nistar;
  F3v xoxv_g = x - P.two_A_de.y * nistar;
  F3v xoxv_b = x - P.two_A_de.z * nistar;
  F3v dv_sqr = v3(dot(xoxv_r, xoxv_r), dot(xoxv_g, xoxv_g), dot(xoxv_b, xoxv_b));
  F3v x_dot_wv = v3(dot(xoxv_r, wv), dot(xoxv_g, wv), dot(xoxv_b, wv));
  F3v x_dot_no = v3(dot(xoxv_r, no), dot(xoxv_g, no), dot(xoxv_b, no));
  F3v Sr = S_infinite(dr_sqr, v3s(dot_x_w12), -mu0, v3s(dot(x, no)), P);
  F3v Sv = S_infinite(dv_sqr, x_dot_wv, dot(no, wv), x_dot_no, P);
  return vmax(Sr - Sv, v3s(0.0f));
}

}  // namespace orc
