// Dipole BSSRDFs of the reference (dipoles/standard_dipole.h, dipoles/directional_dipole.h) on the
// 260-byte ScatteringMaterialProperties, in the reference's operation order and FP32 precision.
#pragma once
#include "pt_scene.cuh"

namespace pt {

PT_D float3 sqrtf3(const float3& a) { return f3(sqrtf(a.x), sqrtf(a.y), sqrtf(a.z)); }
PT_D float3 fmaxf3(const float3& a, const float3& b) { return f3(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
PT_D float3 operator+(float s, const float3& a) { return f3(s + a.x, s + a.y, s + a.z); }

// The per-material terms of dipole_bssrdf (standard_dipole.h:10-13), hoisted out of the probe loop.
struct StdDipole {
  float3 three_D, transport, real_source, virtual_source, corrected_mean_free;
};
PT_D StdDipole std_dipole_terms(const ScatDev& P)
{
  StdDipole s;
  s.three_D = P.three_D;
  s.transport = P.transport;
  s.real_source = P.three_D * P.three_D;
  float3 extrapolation = 4.0f * P.A * P.D;
  s.virtual_source = extrapolation * extrapolation;
  s.corrected_mean_free = P.three_D + extrapolation;
  return s;
}
// dipole_bssrdf, standard_dipole.h:8-29: real and virtual point sources of the classical dipole.
PT_D float3 dipole_bssrdf(float dist, const StdDipole& s)
{
  float3 r_sqr = f3s(dist * dist);
  float3 d_r_sqr = r_sqr + s.real_source;
  float3 d_r = sqrtf3(d_r_sqr);
  float3 d_v_sqr = r_sqr + s.virtual_source;
  float3 d_v = sqrtf3(d_v_sqr);
  float3 tr_r = s.transport * d_r;
  float3 S_r = s.three_D * (1.0f + tr_r) / (d_r_sqr * d_r);
  S_r = S_r * expf3(-tr_r);
  float3 tr_v = s.transport * d_v;
  float3 S_v = s.corrected_mean_free * (1.0f + tr_v) / (d_v_sqr * d_v);
  S_v = S_v * expf3(-tr_v);
  return S_r + S_v;
}

// S_infinite / S_infinite_vec, directional_dipole.h:8-34 (the scalar form widens its arguments).
PT_D float3 dd_S_infinite(const float3& r_sqr, const float3& x_dot_w12, float no_dot_w12, const float3& x_dot_no, const ScatDev& P)
{
  float3 r = sqrtf3(r_sqr);
  float3 r_tr = P.transport * r;
  float3 r_tr_p1 = r_tr + 1.0f;
  float3 T = expf3(-r_tr);
  float3 coeff = T / (r * r_sqr);
  float3 first = P.C_phi * (r_sqr * P.reducedExtinction + r_tr_p1 * x_dot_w12) * 3.0f;
  float3 second = P.C_E * (P.three_D * r_tr_p1 * no_dot_w12 - (r_tr_p1 + P.three_D * (3.0f * r_tr_p1 + r_tr * r_tr) / r_sqr * x_dot_w12) * x_dot_no);
  return coeff * (first - second);
}
// dirpole_bssrdf, directional_dipole.h:37-72 (Frisvad et al.'s directional dipole).
PT_D float3 dirpole_bssrdf(const float3& xi, const float3& ni, const float3& w12, const float3& xo, const float3& no, const ScatDev& P)
{
  float3 x = xo - xi;
  float r_sqr = dot(x, x);
  float3 dr_sqr = f3s(r_sqr);
  float dot_x_w12 = dot(x, w12);
  float3 cos_beta = -sqrtf3(f3s(r_sqr - dot_x_w12 * dot_x_w12) / (r_sqr + P.de * P.de));
  float mu0 = -dot(no, w12);
  float edge = mu0 > 0.0f ? 1.0f : 0.0f;
  float3 D_prime = P.D * mu0 * edge + P.one_over_three_ext * (1.0f - edge);
  dr_sqr = dr_sqr + D_prime * (D_prime - 2.0f * P.de * cos_beta * edge);
  float3 t = normalize(cross(ni, x));
  float3 nistar = r_sqr < 1.0e-12f ? ni : cross(normalize(x), t);
  float3 wv = w12 - (2.0f * dot(w12, nistar)) * nistar;
  float3 xoxv_r = x - P.two_A_de.x * nistar;
  float3 xoxv_g = x - P.two_A_de.y * nistar;
  float3 xoxv_b = x - P.two_A_de.z * nistar;
  float3 dv_sqr = f3(dot(xoxv_r, xoxv_r), dot(xoxv_g, xoxv_g), dot(xoxv_b, xoxv_b));
  float3 x_dot_wv = f3(dot(xoxv_r, wv), dot(xoxv_g, wv), dot(xoxv_b, wv));
  float3 x_dot_no = f3(dot(xoxv_r, no), dot(xoxv_g, no), dot(xoxv_b, no));
  float3 Sr = dd_S_infinite(dr_sqr, f3s(dot_x_w12), -mu0, f3s(dot(x, no)), P);
  float3 Sv = dd_S_infinite(dv_sqr, x_dot_wv, dot(no, wv), x_dot_no, P);
  return fmaxf3(Sr - Sv, f3s(0.0f));
}

}  // namespace pt
