// Test infrastructure (oracle only): restatement of the dipole BSSRDFs (dipoles/standard_dipole.h,
// dipoles/directional_dipole.h) and of the scattering coefficients of
// TranslucentMaterial::computeCoefficients (TranslucentMaterial.cpp:303-330), templated on the
// scalar type: FP32 in the reference's operation order, FP64 as the error yardstick.
#pragma once
#include "orc_math.hpp"

namespace orc {

// ScatteringMaterialProperties, structs.h:116-144 (260 bytes with R = float), templated on the
// scalar type: the FP32 instantiation is the reference's struct, the FP64 one the error yardstick
// (coefficients derived and dipoles evaluated in double from the same FP32 inputs).
template <class R> struct ScatPropsT {
  R relative_ior;
  V3<R> ior_real, ior_imag, absorption, scattering, meancosine, extinction, reducedExtinction, deltaEddExtinction, D, transport,
      C_phi, C_phi_inv, C_E, A, albedo, reducedAlbedo, de, three_D, two_A_de, global_coeff, one_over_three_ext;
  R mean_transport;
};
typedef ScatPropsT<float> ScatProps;
static_assert(sizeof(ScatProps) == 260, "ScatteringMaterialProperties layout");

typedef V3<float> F3v;
template <class R> static inline V3<R> sqrt3(const V3<R>& v) { return v3(std::sqrt(v.x), std::sqrt(v.y), std::sqrt(v.z)); }

// TranslucentMaterial::computeCoefficients with ior_outside = (1,1,1) (TranslucentMaterial.cpp:303-330).
template <class R>
static inline ScatPropsT<R> compute_coefficients_t(const float* absorption, const float* scattering, const float* meancosine, float ior,
                                                   float scale)
{
  ScatPropsT<R> p;
  memset(&p, 0, sizeof(p));
  const V3<R> ior_outside = v3<R>(1, 1, 1);
  const R sc = (R)scale;
  p.absorption = v3<R>(absorption[0], absorption[1], absorption[2]) * sc;
  p.scattering = v3<R>(scattering[0], scattering[1], scattering[2]) * sc;
  p.meancosine = v3<R>(meancosine[0], meancosine[1], meancosine[2]);
  p.relative_ior = (R)ior;
  p.ior_real = v3s<R>((R)ior);
  V3<R> ior_rgb = p.ior_real / ior_outside;
  V3<R> reducedScattering = p.scattering * (R(1) - p.meancosine);
  p.relative_ior /= (ior_outside.x + ior_outside.y + ior_outside.z) / R(3);
  p.ior_real = ior_rgb;
  p.extinction = p.scattering + p.absorption;
  p.reducedExtinction = reducedScattering + p.absorption;
  p.deltaEddExtinction = p.scattering * (R(1) - p.meancosine * p.meancosine) + p.absorption;
  p.D = v3s<R>(1) / (R(3) * p.reducedExtinction);
  p.transport = sqrt3(p.absorption / p.D);
  p.C_phi = v3(C_phi<R>(ior_rgb.x), C_phi<R>(ior_rgb.y), C_phi<R>(ior_rgb.z));
  p.C_phi_inv = v3(C_phi<R>(R(1) / ior_rgb.x), C_phi<R>(R(1) / ior_rgb.y), C_phi<R>(R(1) / ior_rgb.z));
  p.C_E = v3(C_E<R>(ior_rgb.x), C_E<R>(ior_rgb.y), C_E<R>(ior_rgb.z));
  p.albedo = p.scattering / p.extinction;
  p.reducedAlbedo = reducedScattering / p.reducedExtinction;
  p.de = R(2.131f) * p.D / sqrt3(p.reducedAlbedo);
  p.A = (R(1) - p.C_E) / (R(2) * p.C_phi);
  p.three_D = R(3) * p.D;
  p.two_A_de = R(2) * p.A * p.de;
  p.global_coeff = v3s<R>(1) / (R(4) * p.C_phi_inv) * R(1) / (R(4) * K<R>::PI * K<R>::PI);
  p.one_over_three_ext = v3s<R>(1) / (R(3) * p.extinction);
  p.mean_transport = (p.transport.x + p.transport.y + p.transport.z) / R(3);
  return p;
}
static inline ScatProps compute_coefficients(const float* absorption, const float* scattering, const float* meancosine, float ior, float scale)
{
  return compute_coefficients_t<float>(absorption, scattering, meancosine, ior, scale);
}

// dipole_bssrdf, standard_dipole.h:8-30.
template <class R> static inline V3<R> dipole_bssrdf(R dist, const ScatPropsT<R>& P)
{
  V3<R> real_source = P.three_D * P.three_D;
  V3<R> extrapolation = R(4) * P.A * P.D;
  V3<R> virtual_source = extrapolation * extrapolation;
  V3<R> corrected_mean_free = P.three_D + extrapolation;
  V3<R> r_sqr = v3s<R>(dist * dist);
  V3<R> d_r_sqr = r_sqr + real_source;
  V3<R> d_r = sqrt3(d_r_sqr);
  V3<R> d_v_sqr = r_sqr + virtual_source;
  V3<R> d_v = sqrt3(d_v_sqr);
  V3<R> tr_r = P.transport * d_r;
  V3<R> S_r = P.three_D * (R(1) + tr_r) / (d_r_sqr * d_r);
  S_r = S_r * vexp(-tr_r);
  V3<R> tr_v = P.transport * d_v;
  V3<R> S_v = corrected_mean_free * (R(1) + tr_v) / (d_v_sqr * d_v);
  S_v = S_v * vexp(-tr_v);
  return S_r + S_v;
}

// S_infinite / S_infinite_vec, directional_dipole.h:8-34.
template <class R>
static inline V3<R> S_infinite(const V3<R>& r_sqr, const V3<R>& x_dot_w12, const R no_dot_w12, const V3<R>& x_dot_no, const ScatPropsT<R>& P)
{
  V3<R> r = sqrt3(r_sqr);
  V3<R> r_tr = P.transport * r;
  V3<R> r_tr_p1 = r_tr + R(1);
  V3<R> T = vexp(-r_tr);
  V3<R> coeff = T / (r * r_sqr);
  V3<R> first = P.C_phi * (r_sqr * P.reducedExtinction + r_tr_p1 * x_dot_w12) * R(3);
  V3<R> second = P.C_E * (P.three_D * r_tr_p1 * no_dot_w12 - (r_tr_p1 + P.three_D * (R(3) * r_tr_p1 + r_tr * r_tr) / r_sqr * x_dot_w12) * x_dot_no);
  return coeff * (first - second);
}
// dirpole_bssrdf, directional_dipole.h:37-72.
template <class R>
static inline V3<R> dirpole_bssrdf(const V3<R>& xi, const V3<R>& ni, const V3<R>& w12, const V3<R>& xo, const V3<R>& no, const ScatPropsT<R>& P)
{
  V3<R> x = xo - xi;
  R r_sqr = dot(x, x);
  V3<R> dr_sqr = v3s(r_sqr);
  R dot_x_w12 = dot(x, w12);
  V3<R> cos_beta = -sqrt3(v3s(r_sqr - dot_x_w12 * dot_x_w12) / (r_sqr + P.de * P.de));
  R mu0 = -dot(no, w12);
  R edge = mu0 > R(0) ? R(1) : R(0);
  V3<R> D_prime = P.D * mu0 * edge + P.one_over_three_ext * (R(1) - edge);
  dr_sqr = dr_sqr + D_prime * (D_prime - R(2) * P.de * cos_beta * edge);
  V3<R> t = normalize(cross(ni, x));
  V3<R> nistar = r_sqr < R(1.0e-12f) ? ni : cross(normalize(x), t);
  V3<R> wv = w12 - (R(2) * dot(w12, nistar)) * nistar;
  V3<R> xoxv_r = x - P.two_A_de.x * nistar;
  V3<R> xoxv_g = x - P.two_A_de.y * nistar;
  V3<R> xoxv_b = x - P.two_A_de.z * nistar;
  V3<R> dv_sqr = v3(dot(xoxv_r, xoxv_r), dot(xoxv_g, xoxv_g), dot(xoxv_b, xoxv_b));
  V3<R> x_dot_wv = v3(dot(xoxv_r, wv), dot(xoxv_g, wv), dot(xoxv_b, wv));
  V3<R> x_dot_no = v3(dot(xoxv_r, no), dot(xoxv_g, no), dot(xoxv_b, no));
  V3<R> Sr = S_infinite(dr_sqr, v3s(dot_x_w12), -mu0, v3s(dot(x, no)), P);
  V3<R> Sv = S_infinite(dv_sqr, x_dot_wv, dot(no, wv), x_dot_no, P);
  return vmax(Sr - Sv, v3s<R>(0));
}

}  // namespace orc
