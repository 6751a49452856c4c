// Test infrastructure (oracle only): restatement of MicrofacetGGX.h, MicrofacetBeckmann.h and
// the Microfacet.h dispatchers, templated on the scalar type R (see orc_math.hpp).  Line
// numbers cite open_rendering_framework/<file>.  The multiscattering random walks take an
// iteration cap `cap` (the reference loops `while(true)`); `*capped` is set when it is reached.
#pragma once
#include "orc_math.hpp"

namespace orc {

enum { BECKMANN = 0, GGX = 1 };  // structs.h:256-261
enum { WALTER = 0, VISIBLE_NORMALS = 1, MULTISCATTERING = 2 };  // structs.h:242-248

struct Slope2 { double x, y; };
template <class R> struct S2 { R x, y; };

// ================================================================ GGX (MicrofacetGGX.h)
template <class R> static inline R ggx_alpha_i(const V3<R>& wi, R ax, R ay)  // :9-17
{
  R inv_sin2 = R(1) / (R(1) - wi.z * wi.z);
  if (wi.z == R(1) || wi.z == R(-1)) inv_sin2 = R(0);
  R cos_phi2 = wi.x * wi.x * inv_sin2;
  R sin_phi2 = wi.y * wi.y * inv_sin2;
  return std::sqrt(cos_phi2 * ax * ax + sin_phi2 * ay * ay);
}
template <class R> static inline R ggx_lambda(const V3<R>& wi, R ax, R ay)  // :20-30
{
  if (wi.z > R(0.99999f)) return R(0);
  if (wi.z < R(-0.99999f)) return R(-1);
  R th = std::acos(wi.z);
  R a = R(1) / std::tan(th) / ggx_alpha_i(wi, ax, ay);
  return R(0.5f) * (R(-1) + std::sqrt(R(1) + R(1) / (a * a)) * (R)(a > 0 ? 1 : -1));
}
template <class R> static inline R ggx_projected_area(const V3<R>& wi, R ax, R ay)  // :33-45
{
  if (wi.z > R(0.9999f)) return R(1);
  if (wi.z < R(-0.9999f)) return R(0);
  R alpha = ggx_alpha_i(wi, ax, ay);
  R th = std::acos(wi.z);
  R st = std::sin(th);
  return R(0.5f) * (wi.z + std::sqrt(wi.z * wi.z + st * st * alpha * alpha));
}
template <class R> static inline R ggx_slope_pdf(R sx, R ax, R sy, R ay)  // :48-53
{
  R tmp = R(1) + sx * sx / (ax * ax) + sy * sy / (ay * ay);
  return R(1) / (K<R>::PI * ax * ay) / (tmp * tmp);
}
template <class R> static inline R ggx_G1_cos(R c, R a2)  // :54-60
{
  R c2 = c * c;
  R t2 = (R(1) - c2) / c2;
  return R(2) / (R(1) + std::sqrt(R(1) + a2 * t2));
}
template <class R> static inline R ggx_G1_aniso(const V3<R>& v, const V3<R>& m, const V3<R>& n, R ax, R ay)  // :63-74
{
  R alpha = ggx_alpha_i(normalize(to_local(v, n)), ax, ay);
  R a2 = alpha * alpha;
  R cv = dot(v, n);
  if (cv * dot(v, m) <= 0) return R(0);
  return ggx_G1_cos(cv, a2);
}
template <class R> static inline R ggx_G1(const V3<R>& v, const V3<R>& m, const V3<R>& n, R ag)  // :77-83
{
  R cv = dot(v, n);
  if (cv * dot(v, m) <= 0) return R(0);
  return ggx_G1_cos(cv, ag * ag);
}
template <class R> static inline R ggx_G_height(const V3<R>& wi, R h, R ax, R ay)  // :93-107
{
  if (wi.z > R(0.9999f)) return R(1);
  if (wi.z <= R(0)) return R(0);
  R c1 = gauss_cdf(h);
  R lam = ggx_lambda(wi, ax, ay);
  return std::pow(c1, lam);
}
template <class R> static inline V3<R> ggx_sample_hemisphere(const V3<R>& n, R z1, R z2, R ag)  // :123-139
{
  R phi = R(2) * K<R>::PI * z2;
  R tan_t = ag * std::sqrt(z1) / std::sqrt(R(1) - z1);
  R th = std::atan(tan_t);
  R ct = std::cos(th), st = std::sin(th);
  V3<R> m = v3(st * std::cos(phi), st * std::sin(phi), ct);
  V3<R> v1, v2;
  create_onb(n, v1, v2);
  return v1 * m.x + v2 * m.y + n * m.z;
}
template <class R> static inline S2<R> ggx_P22(R theta_i, R z1, R z2)  // :142-187
{
  S2<R> s;
  if (theta_i < R(0.0001f)) {
    R r = std::sqrt(z1 / (R(1) - z1));
    R phi = K<R>::PI * R(2) * z2;
    s.x = r * std::cos(phi);
    s.y = r * std::sin(phi);
    return s;
  }
  R sin_i = std::sin(theta_i);
  R cos_i = std::fmax(std::cos(theta_i), (R)1e-7);
  R tan_i = sin_i / cos_i;
  R proj = R(0.5f) * (cos_i + R(1));
  if (proj < R(0.0001f) || proj != proj) { s.x = 0; s.y = 0; return s; }
  R c = R(1) / proj;
  R A = R(2) * z1 / cos_i / c - R(1);
  R B = tan_i;
  R tmp = R(1) / (A * A - R(1));
  R D = std::sqrt(std::fmax(R(0), B * B * tmp * tmp - (A * A - B * B) * tmp));
  R sx1 = B * tmp - D, sx2 = B * tmp + D;
  s.x = (A < R(0) || sx2 > R(1) / tan_i) ? sx1 : sx2;
  R S, zz2;
  if (z2 > R(0.5f)) { S = R(1); zz2 = R(2) * (z2 - R(0.5f)); }
  else { S = R(-1); zz2 = R(2) * (R(0.5f) - z2); }
  R z = (zz2 * (zz2 * (zz2 * R(0.27385f) - R(0.73369f)) + R(0.46341f))) /
        (zz2 * (zz2 * (zz2 * R(0.093073f) + R(0.309420f)) - R(1.0000f)) + R(0.597999f));
  s.y = S * z * std::sqrt(R(1) + s.x * s.x);
  return s;
}
template <class R> static inline V3<R> ggx_sample_vndf(const V3<R>& wi, R ax, R ay, R z1, R z2)  // :190-207
{
  V3<R> w11 = normalize(v3(ax * wi.x, ay * wi.y, wi.z));
  S2<R> s11 = ggx_P22(std::acos(w11.z), z1, z2);
  R phi = std::atan2(w11.y, w11.x);
  R sx = std::cos(phi) * s11.x - std::sin(phi) * s11.y;
  R sy = std::sin(phi) * s11.x + std::cos(phi) * s11.y;
  sx *= ax;
  sy *= ay;
  if (!std::isfinite(sx) || sx != sx) {
    if (wi.z > 0) return v3(R(0), R(0), R(1));
    return normalize(v3(wi.x, wi.y, R(0)));
  }
  return normalize(v3(-sx, -sy, R(1)));
}
template <class R> static inline R ggx_eval_ndf(const V3<R>& wm, R ax, R ay)  // :219-231
{
  if (wm.z <= R(0)) return R(0);
  R sx = -wm.x / wm.z, sy = -wm.y / wm.z;
  return ggx_slope_pdf(sx, ax, sy, ay) / (wm.z * wm.z * wm.z * wm.z);
}
template <class R> static inline R ggx_eval_vndf(const V3<R>& wi, const V3<R>& wm, R ax, R ay)  // :234-251
{
  if (wm.z <= R(0)) return R(0);
  R area = ggx_projected_area(wi, ax, ay);
  if (area == R(0)) return R(0);
  R c = R(1) / area;
  R D = ggx_eval_ndf(wm, ax, ay);
  return c * std::fmax(R(0), dot(wi, wm)) * D;
}
template <class R> static inline R ggx_sample_height(const V3<R>& wr, R hr, R z, R ax, R ay)  // :254-276
{
  if (wr.z > R(0.9999f)) return (R)DEFAULT_MAX;
  if (wr.z < R(-0.9999f)) return gauss_inv_cdf(z * gauss_cdf(hr));
  if (std::fabs(wr.z) < R(0.00001f)) return hr;
  R G1 = ggx_G_height(wr, hr, ax, ay);
  if (z > R(1) - G1) return (R)DEFAULT_MAX;
  return gauss_inv_cdf(gauss_cdf(hr) / std::pow((R(1) - z), R(1) / ggx_lambda(wr, ax, ay)));
}
template <class R> static inline R ggx_distribution(const V3<R>& m, const V3<R>& n, R alpha)  // :643-655
{
  R D = R(0);
  R c = dot(m, n);
  if (c > R(0)) {
    R c2 = c * c, s2 = R(1) - c2, a2 = alpha * alpha;
    R coeff = c2 * (a2 + s2 / c2);
    D = a2 * K<R>::INV_PI / (coeff * coeff);
  }
  return D;
}

// ================================================================ Beckmann (MicrofacetBeckmann.h)
template <class R> static inline R bk_lambda(const V3<R>& wi, R ax, R ay)  // :24-42
{
  if (wi.z > R(0.9999f)) return R(0);
  if (wi.z < R(-0.9999f)) return R(-1);
  R th = std::acos(wi.z);
  R t = std::tan(th);
  if (std::isinf(t)) return R(0);
  R a = R(1) / (t * ggx_alpha_i(wi, ax, ay));
  return R(0.5f) * ((R)std::erf(a) - R(1)) + R(0.25f) * K<R>::TWO_SQRTPI / a * std::exp(-a * a);
}
template <class R> static inline R bk_projected_area(const V3<R>& wi, R ax, R ay)  // :45-58
{
  if (wi.z > R(0.9999f)) return R(1);
  if (wi.z < R(-0.9999f)) return R(0);
  R alpha = ggx_alpha_i(wi, ax, ay);
  R th = std::acos(wi.z);
  R a = R(1) / std::tan(th) / alpha;
  double rhs = 0.25 * (double)K<R>::TWO_SQRTPI * (double)alpha * (double)std::sin(th) * (double)std::exp(-a * a);
  return (R)((double)(R(0.5f) * ((R)std::erf(a) + R(1)) * wi.z) + rhs);
}
template <class R> static inline R bk_slope_pdf(R sx, R ax, R sy, R ay)  // :61-65
{
  return R(1) / (K<R>::PI * ax * ay) * std::exp(-sx * sx / (ax * ax) - sy * sy / (ay * ay));
}
template <class R> static inline R bk_G1_cos(R c, R ab2)  // :68-75
{
  R c2 = c * c;
  R t2 = (R(1) - c2) / c2;
  R a2 = R(1) / (ab2 * t2);
  R a = std::sqrt(a2);
  if (!(a < R(1.6f))) return R(1);
  double den = (double)(R(1) + R(2.276f) * a) + 2.577 * (double)a2;
  return (R)((double)(R(3.535f) * a + R(2.181f) * a2) / den);
}
template <class R> static inline R bk_G1(const V3<R>& v, const V3<R>& m, const V3<R>& n, R width)  // :78-86
{
  R cv = dot(v, n);
  if (dot(v, m) * cv <= 0) return R(0);
  return bk_G1_cos(cv, width * width);
}
template <class R> static inline R bk_G1_aniso(const V3<R>& v, const V3<R>& m, const V3<R>& n, R ax, R ay)  // :89-98
{
  R width = ggx_alpha_i(to_local(v, n), ax, ay);
  R cv = dot(v, n);
  if (dot(v, m) * cv <= 0) return R(0);
  return bk_G1_cos(cv, width * width);
}
template <class R> static inline R bk_G_height(const V3<R>& wi, R h, R ax, R ay)  // :108-127
{
  if (wi.z > R(0.9999f)) return R(1);
  if (wi.z <= R(0)) return R(0);
  R c1 = gauss_cdf(h);
  R lam = bk_lambda(wi, ax, ay);
  return std::pow(c1, lam);
}
template <class R> static inline R bk_G_avg(const V3<R>& wi, R ax, R ay)  // :130-141
{
  if (wi.z > R(0.9999f)) return R(1);
  if (wi.z <= R(0)) return R(0);
  R lam = bk_lambda(wi, ax, ay);
  return R(1) / (R(1) + lam);
}
template <class R> static inline V3<R> bk_sample_hemisphere(const V3<R>& n, R z1, R z2, R width)  // :144-158
{
  R phi = R(2) * K<R>::PI * z2;
  R tan_t = -width * width * std::log(R(1) - z1);
  R th = std::atan(std::sqrt(tan_t));
  R ct = std::cos(th), st = std::sin(th);
  V3<R> m = v3(st * std::cos(phi), st * std::sin(phi), ct);
  V3<R> v1, v2;
  create_onb(n, v1, v2);
  return v1 * m.x + v2 * m.y + n * m.z;
}
// Visible-slope sampling by Newton/bisection on erf (:161-210).  `cap` bounds the loop.
template <class R> static inline S2<R> bk_P22(R theta_i, R z1, R z2, int cap = 1 << 20, int* capped = nullptr)
{
  S2<R> s;
  if (theta_i < R(0.0001f)) {
    R r = std::sqrt(-std::log(z1));
    R phi = K<R>::PI * R(2) * z2;
    s.x = r * std::cos(phi);
    s.y = r * std::sin(phi);
    return s;
  }
  R sin_i = std::sin(theta_i), cos_i = std::cos(theta_i);
  R slope_i = cos_i / sin_i;
  R a = cos_i / sin_i;
  R proj = R(0.5f) * ((R)std::erf(a) + R(1)) * cos_i + R(0.25f) * K<R>::TWO_SQRTPI * sin_i * std::exp(-a * a);
  if (proj < R(0.0001f) || proj != proj) { s.x = 0; s.y = 0; return s; }
  R c = R(1) / proj;
  R emin = R(-0.9999f);
  R emax = std::fmax(emin, (R)std::erf(slope_i));
  R ecur = R(0.5f) * (emin + emax);
  int it = 0;
  while (emax - emin > R(0.00001f)) {
    if (++it > cap) { if (capped) *capped = 1; break; }
    if (!(ecur >= emin && ecur <= emax)) ecur = R(0.5f) * (emin + emax);
    R sv = (R)erfinv_d(ecur);
    R cdf;
    if (sv >= slope_i) cdf = R(1);
    else {
      double inner = 0.25 * (double)K<R>::TWO_SQRTPI * (double)sin_i * (double)std::exp(-sv * sv) +
                     (double)(cos_i * (R(0.5f) + R(0.5f) * (R)std::erf(sv)));
      cdf = (R)((double)c * inner);
    }
    R diff = cdf - z1;
    if (std::fabs(diff) < R(0.00001f)) break;
    if (diff > R(0)) {
      if (emax == ecur) break;
      emax = ecur;
    } else {
      if (emin == ecur) break;
      emin = ecur;
    }
    R deriv = R(0.5f) * c * cos_i - R(0.5f) * c * sin_i * sv;
    ecur -= diff / deriv;
  }
  s.x = (R)erfinv_d(std::fmin(emax, std::fmax(emin, ecur)));
  s.y = (R)erfinv_d(R(2) * z2 - R(1));
  return s;
}
template <class R> static inline V3<R> bk_sample_vndf(const V3<R>& wi, R ax, R ay, R z1, R z2, int cap = 1 << 20, int* capped = nullptr)  // :213-231
{
  V3<R> w11 = normalize(v3(ax * wi.x, ay * wi.y, wi.z));
  S2<R> s11 = bk_P22(std::acos(w11.z), z1, z2, cap, capped);
  R phi = std::atan2(w11.y, w11.x);
  R sx = std::cos(phi) * s11.x - std::sin(phi) * s11.y;
  R sy = std::sin(phi) * s11.x + std::cos(phi) * s11.y;
  sx *= ax;
  sy *= ay;
  if (!std::isfinite(sx) || sx != sx) {
    if (wi.z > 0) return v3(R(0), R(0), R(1));
    return normalize(v3(wi.x, wi.y, R(0)));
  }
  return normalize(v3(-sx, -sy, R(1)));
}
template <class R> static inline R bk_eval_ndf(const V3<R>& wm, R ax, R ay)  // :249-261
{
  if (wm.z <= R(0)) return R(0);
  R sx = -wm.x / wm.z, sy = -wm.y / wm.z;
  return bk_slope_pdf(sx, ax, sy, ay) / (wm.z * wm.z * wm.z * wm.z);
}
template <class R> static inline R bk_eval_vndf(const V3<R>& wi, const V3<R>& wm, R ax, R ay)  // :264-281
{
  if (wm.z <= R(0)) return R(0);
  R area = bk_projected_area(wi, ax, ay);
  if (area == R(0)) return R(0);
  R c = R(1) / area;
  R D = bk_eval_ndf(wm, ax, ay);
  return c * std::fmax(R(0), dot(wi, wm)) * D;
}
template <class R> static inline R bk_sample_height(const V3<R>& wr, R hr, R z, R ax, R ay)  // :284-307
{
  if (wr.z > R(0.999f)) return (R)DEFAULT_MAX;
  if (wr.z < R(-0.999f)) return gauss_inv_cdf(z * gauss_cdf(hr));
  if (std::fabs(wr.z) < R(0.00001f)) return hr;
  R G1 = bk_G_avg(wr, ax, ay);
  if (z > R(1) - G1) return (R)DEFAULT_MAX;
  R gcdf = gauss_cdf(hr);
  R p = std::pow((R(1) - z), R(1) / bk_lambda(wr, ax, ay));
  return gauss_inv_cdf(gcdf / p);
}
template <class R> static inline R bk_distribution(const V3<R>& m, const V3<R>& n, R alpha)  // :739-750
{
  R D = R(0);
  R c = dot(m, n);
  if (c > R(0.0001f)) {
    R c2 = c * c, s2 = R(1) - c2, a2 = alpha * alpha;
    D = std::exp(-s2 / (c2 * a2)) * K<R>::INV_PI / (a2 * c2 * c2);
  }
  return D;
}

// ================================================================ distribution-generic pieces
template <class R> static inline V3<R> sample_vndf(int dist, const V3<R>& wi, R ax, R ay, R z1, R z2, int* capped = nullptr)
{
  return dist == GGX ? ggx_sample_vndf(wi, ax, ay, z1, z2) : bk_sample_vndf(wi, ax, ay, z1, z2, 1 << 20, capped);
}
template <class R> static inline R eval_vndf(int dist, const V3<R>& wi, const V3<R>& wm, R ax, R ay)
{
  return dist == GGX ? ggx_eval_vndf(wi, wm, ax, ay) : bk_eval_vndf(wi, wm, ax, ay);
}
template <class R> static inline R sample_height(int dist, const V3<R>& wr, R hr, R z, R ax, R ay)
{
  return dist == GGX ? ggx_sample_height(wr, hr, z, ax, ay) : bk_sample_height(wr, hr, z, ax, ay);
}
template <class R> static inline R G_height(int dist, const V3<R>& wi, R h, R ax, R ay)
{
  return dist == GGX ? ggx_G_height(wi, h, ax, ay) : bk_G_height(wi, h, ax, ay);
}

// Dielectric phase function sample, GGX :279-304 / Beckmann :310-338 (identical steps).
template <class R> static inline V3<R> sample_dielectric_phase(int dist, const V3<R>& wi, V3<R>& wm, R m_eta, u32& seed,
                                                               bool wi_out, bool& wo_out, R& F, R ax, R ay)
{
  R z1 = (R)rnd_tea(seed), z2 = (R)rnd_tea(seed);
  R eta = wi_out ? m_eta : R(1) / m_eta;
  wm = wi_out ? sample_vndf(dist, wi, ax, ay, z1, z2) : -sample_vndf(dist, -wi, ax, ay, z1, z2);
  R ct = std::fabs(dot(wm, wi));
  R st2 = eta * eta * (R(1) - ct * ct);
  R ctt = std::sqrt(R(1) - st2);
  F = st2 < R(1) ? fresnel_R(ct, ctt, eta) : R(1);
  if ((R)rnd_tea(seed) <= F) return normalize(-wi + R(2) * wm * dot(wi, wm));
  wo_out = !wi_out;
  return normalize(-eta * wi + wm * (eta * ct - ctt));
}
// Dielectric phase function eval, GGX :307-339 / Beckmann :341-372.
template <class R> static inline R eval_dielectric_phase(int dist, const V3<R>& wi, const V3<R>& wo, bool wi_out, bool wo_out,
                                                         R m_eta, R ax, R ay)
{
  R eta = wi_out ? m_eta : R(1) / m_eta;
  if (wi_out == wo_out) {
    V3<R> wh = normalize(wi + wo);
    R D = wi_out ? eval_vndf(dist, wi, wh, ax, ay) : eval_vndf(dist, -wi, -wh, ax, ay);
    R F = wi_out ? fresnel_R(wi, wh, eta) : fresnel_R(-wi, -wh, eta);
    R a = wi_out ? R(0.25f) / dot(wi, wh) : R(0.25f) / dot(-wi, -wh);
    return F * D * a;
  }
  V3<R> wh = -normalize(wi + wo / eta);
  R sg = wi_out ? wh.z / std::fabs(wh.z) : -wh.z / std::fabs(wh.z);
  wh = wh * sg;
  if (dot(wh, wi) < R(0)) return R(0);
  R D = wi_out ? eval_vndf(dist, wi, wh, ax, ay) : eval_vndf(dist, -wi, -wh, ax, ay);
  R F = wi_out ? fresnel_R(wi, wh, eta) : fresnel_R(-wi, -wh, eta);
  R b = R(1) / (eta * eta);
  R c = wi_out ? std::fmax(R(0), -dot(wo, wh)) : std::fmax(R(0), -dot(-wo, -wh));
  R e = wi_out ? dot(wi, wh) + dot(wo, wh) / eta : dot(-wi, -wh) + dot(-wo, -wh) / eta;
  R d = e * e;
  R a = b * c / d;
  return a * D * (R(1) - F);
}
// Diffuse phase sample, GGX :342-375 / Beckmann :375-408.
template <class R> static inline V3<R> sample_diffuse_phase(int dist, const V3<R>& wi, V3<R>& wm, u32& seed, R ax, R ay)
{
  R z1 = (R)rnd_tea(seed), z2 = (R)rnd_tea(seed), z3 = (R)rnd_tea(seed), z4 = (R)rnd_tea(seed);
  wm = sample_vndf(dist, wi, ax, ay, z1, z2);
  V3<R> w1, w2;
  create_onb(wm, w1, w2);
  R r1 = R(2) * z3 - R(1), r2 = R(2) * z4 - R(1);
  R phi, r;
  if (r1 == 0 && r2 == 0) { r = phi = 0; }
  else if (r1 * r1 > r2 * r2) { r = r1; phi = (K<R>::PI / R(4)) * (r2 / r1); }
  else { r = r2; phi = (K<R>::PI / R(2)) - (r1 / r2) * (K<R>::PI / R(4)); }
  R x = r * std::cos(phi), y = r * std::sin(phi);
  R z = std::sqrt(std::fmax(R(0), R(1) - x * x - y * y));
  return x * w1 + y * w2 + z * wm;
}
// Diffuse phase eval, GGX :378-387 (1/pi) / Beckmann :411-420 (1*M_1_PI).
template <class R> static inline R eval_diffuse_phase(int dist, const V3<R>& wi, const V3<R>& wo, V3<R>& wm, R ax, R ay, u32& seed)
{
  R z1 = (R)rnd_tea(seed), z2 = (R)rnd_tea(seed);
  wm = sample_vndf(dist, wi, ax, ay, z1, z2);
  if (dist == GGX) return R(1) / K<R>::PI * std::fmax(R(0), dot(wo, wm));
  return R(1) * K<R>::INV_PI * std::fmax(R(0), dot(wo, wm));
}
// Conductor phase sample / eval, GGX :390-409 / Beckmann :423-442.
template <class R> static inline V3<R> sample_conductor_phase(int dist, const V3<R>& wi, V3<R>& wm, u32& seed, R ax, R ay)
{
  R z1 = (R)rnd_tea(seed), z2 = (R)rnd_tea(seed);
  wm = sample_vndf(dist, wi, ax, ay, z1, z2);
  return -wi + R(2) * wm * dot(wi, wm);
}
template <class R> static inline R eval_conductor_phase(int dist, const V3<R>& wi, const V3<R>& wo, V3<R>& wm, R ax, R ay)
{
  wm = normalize(wi + wo);
  if (wm.z < R(0)) return R(0);
  return R(0.25f) * eval_vndf(dist, wi, wm, ax, ay);
}

// Multiscattering dielectric sample, GGX :412-442 / Beckmann :445-476 (local frame).
template <class R> static inline V3<R> ms_dielectric_sample(int dist, const V3<R>& lwi, R eta, R ax, R ay, u32& seed, u32& order,
                                                            int cap, int* capped)
{
  R hr = R(1) + gauss_inv_cdf(R(0.9999f));
  V3<R> wo = -lwi, wm;
  R F;
  bool out = (-wo.z) > 0;
  for (int it = 0;; ++it) {
    if (it >= cap) { if (capped) *capped = 1; break; }
    R z = (R)rnd_tea(seed);
    hr = out ? sample_height(dist, wo, hr, z, ax, ay) : -sample_height(dist, -wo, -hr, z, ax, ay);
    if (hr == (R)DEFAULT_MAX || hr == -(R)DEFAULT_MAX) break;
    order++;
    bool wi_out = out;
    wo = sample_dielectric_phase(dist, -wo, wm, eta, seed, wi_out, out, F, ax, ay);
    if (hr != hr || wo.z != wo.z) { wo = v3(R(0), R(0), R(1)); break; }
  }
  return wo;
}
// Multiscattering dielectric eval: GGX :445-481 (orders < N, all summed, no finiteness test);
// Beckmann :479-527 (orders <= N, only the matching order summed, finite terms only).
template <class R> static inline R ms_dielectric_eval(int dist, const V3<R>& wi, const V3<R>& wo, R eta, R ax, R ay, u32& seed,
                                                      u32 order, int cap, int* capped)
{
  V3<R> wr = -wi, wm;
  R hr = R(1) + gauss_inv_cdf(R(0.9999f));
  int cur = 0;
  R sum = R(0), F;
  bool wr_out = (-wr.z > 0);
  bool wo_out = wo.z > 0;
  for (int it = 0;; ++it) {
    if (dist == GGX) { if (!(order == 0 || cur < (int)order)) break; }
    else { if (!(order == 0 || (u32)cur <= order)) break; }
    if (it >= cap) { if (capped) *capped = 1; break; }
    R z = (R)rnd_tea(seed);
    hr = wr_out ? sample_height(dist, wr, hr, z, ax, ay) : -sample_height(dist, -wr, -hr, z, ax, ay);
    if (hr == (R)DEFAULT_MAX || hr == -(R)DEFAULT_MAX || std::isinf(hr)) break;
    cur++;
    R phase = eval_dielectric_phase(dist, -wr, wo, wr_out, wo_out, eta, ax, ay);
    R shadow = wo_out ? G_height(dist, wo, hr, ax, ay) : G_height(dist, -wo, -hr, ax, ay);
    R I = phase * shadow;
    if (dist == GGX) sum += I;
    else if (std::isfinite(I) && (order == 0 || (u32)cur == order)) sum += I;
    bool wi_out = wr_out;
    wr = sample_dielectric_phase(dist, -wr, wm, eta, seed, wi_out, wr_out, F, ax, ay);
    if (hr != hr || wr.z != wr.z) { sum = R(0); break; }
  }
  return sum;
}
// Multiscattering diffuse sample, GGX :519-544 / Beckmann :613-640 (capped at 100 orders).
template <class R> static inline V3<R> ms_diffuse_sample(int dist, const V3<R>& wi, V3<R>& wm, R ax, R ay, u32& seed, u32& order,
                                                         V3<R>& weight, const V3<R>& rho)
{
  weight = v3s(R(1));
  R hr = R(1) + gauss_inv_cdf(R(0.9999f));
  V3<R> wo = -wi;
  while (order < 100u) {
    R u = (R)rnd_tea(seed);
    hr = sample_height(dist, wo, hr, u, ax, ay);
    if (hr == (R)DEFAULT_MAX) break;
    order++;
    weight = weight * rho;
    wo = sample_diffuse_phase(dist, -wo, wm, seed, ax, ay);
    if (hr != hr || wo.z != wo.z) { wo = v3(R(0), R(0), R(1)); break; }
  }
  return wo;
}
// Multiscattering diffuse eval, GGX :547-577 / Beckmann :643-674.
template <class R> static inline V3<R> ms_diffuse_eval(int dist, const V3<R>& wi, const V3<R>& wo, R ax, R ay, u32& seed,
                                                       const V3<R>& rho, u32 order, int cap, int* capped)
{
  V3<R> wr = -wi, wm, sum = v3s(R(0));
  R hr = R(1) + gauss_inv_cdf(R(0.9999f));
  int cur = 0;
  for (int it = 0; order == 0 || cur < (int)order; ++it) {
    if (it >= cap) { if (capped) *capped = 1; break; }
    R u = (R)rnd_tea(seed);
    hr = sample_height(dist, wr, hr, u, ax, ay);
    if (hr == (R)DEFAULT_MAX) break;
    cur++;
    R phase = eval_diffuse_phase(dist, -wr, wo, wm, ax, ay, seed);
    R shadow = G_height(dist, wo, hr, ax, ay);
    V3<R> I = rho * phase * shadow;
    if (finite3(I)) sum = sum + I;
    wr = sample_diffuse_phase(dist, -wr, wm, seed, ax, ay);
    if (hr != hr || wr.z != wr.z) { sum = v3s(R(0)); break; }
  }
  return sum;
}
// Multiscattering conductor eval, GGX :580-611 / Beckmann :677-708.
template <class R> static inline V3<R> ms_conductor_eval(int dist, const V3<R>& wi, const V3<R>& wo, const Cx3& eta, const Cx3& inv_eta,
                                                         R ax, R ay, u32& seed, u32 order, int cap, int* capped)
{
  V3<R> wr = -wi, wm, sum = v3s(R(0));
  R hr = R(1) + gauss_inv_cdf(R(0.9999f));
  int cur = 0;
  for (int it = 0; order == 0 || cur < (int)order; ++it) {
    if (it >= cap) { if (capped) *capped = 1; break; }
    R u = (R)rnd_tea(seed);
    hr = sample_height(dist, wr, hr, u, ax, ay);
    if (hr == (R)DEFAULT_MAX) break;
    cur++;
    R phase = eval_conductor_phase(dist, -wr, wo, wm, ax, ay);
    R shadow = G_height(dist, wo, hr, ax, ay);
    V3<R> F = fresnel_complex(-wr, wm, (-wr.z > 0) ? eta : inv_eta);
    V3<R> I = F * phase * shadow;
    if (finite3(I)) sum = sum + I;
    wr = sample_conductor_phase(dist, -wr, wm, seed, ax, ay);
    if (hr != hr || wr.z != wr.z) { sum = v3s(R(0)); break; }
  }
  return sum;
}
// Multiscattering conductor sample, GGX :614-640 / Beckmann :711-736.
template <class R> static inline V3<R> ms_conductor_sample(int dist, const V3<R>& wi, V3<R>& wm, const Cx3& eta, const Cx3& inv_eta,
                                                           R ax, R ay, u32& seed, u32& order, V3<R>& weight, int cap, int* capped)
{
  R hr = R(1) + gauss_inv_cdf(R(0.9999f));
  V3<R> wo = -wi;
  weight = v3s(R(1));
  for (int it = 0;; ++it) {
    if (it >= cap) { if (capped) *capped = 1; break; }
    R u = (R)rnd_tea(seed);
    hr = sample_height(dist, wo, hr, u, ax, ay);
    if (hr == (R)DEFAULT_MAX) break;
    order++;
    V3<R> wt = -wo;
    wo = sample_conductor_phase(dist, -wo, wm, seed, ax, ay);
    weight = weight * fresnel_complex(wt, wm, (wt.z > 0) ? eta : inv_eta);
    if (hr != hr || wo.z != wo.z) { wo = v3(R(0), R(0), R(1)); break; }
  }
  return wo;
}

// Walter BSDF eval, GGX :658-688 / Beckmann :753-786.
template <class R> static inline R walter_bsdf(int dist, const V3<R>& wi, const V3<R>& wo, const V3<R>& n, R alpha, R eta)
{
  bool refl = dot(wo, n) > R(0);
  V3<R> m = refl ? normalize(wo + wi) : -normalize(eta * wi + wo);
  R Rf = fresnel_R(wi, m, eta);
  R idn = std::fabs(dot(wi, n)), odn = std::fabs(dot(wo, n));
  R Gi = dist == GGX ? ggx_G1(wi, m, n, alpha) : bk_G1(wi, m, n, alpha);
  R Go = dist == GGX ? ggx_G1(wo, m, n, alpha) : bk_G1(wo, m, n, alpha);
  R G = Gi * Go;
  R T = R(1) - Rf;
  R D = dist == GGX ? ggx_distribution(m, n, alpha) : bk_distribution(m, n, alpha);
  if (refl) return Rf * G * D / (R(4) * idn * odn);
  R idm = std::fabs(dot(wi, m)), odm = std::fabs(dot(wo, m));
  R coeff = (idm * odm) / (idn * odn);
  R den = (eta * idm + odm);
  return T * G * D * coeff / (den * den);
}

// ================================================================ Microfacet.h dispatchers
template <class R> static inline R masking_G1(int dist, const V3<R>& v, const V3<R>& m, const V3<R>& n, R alpha)  // :20-26
{
  return dist == GGX ? ggx_G1(v, m, n, alpha) : bk_G1(v, m, n, alpha);
}
template <class R> static inline R masking_G1_aniso(int dist, const V3<R>& v, const V3<R>& m, const V3<R>& n, R ax, R ay)  // :28-36
{
  return dist == GGX ? ggx_G1_aniso(v, m, n, ax, ay) : bk_G1_aniso(v, m, n, ax, ay);
}
template <class R> static inline V3<R> sample_normal(int dist, const V3<R>& n, R z1, R z2, R alpha)  // :54-64
{
  return dist == GGX ? ggx_sample_hemisphere(n, z1, z2, alpha) : bk_sample_hemisphere(n, z1, z2, alpha);
}
template <class R> static inline V3<R> sample_visible_normal(int dist, const V3<R>& wi, const V3<R>& n, R ax, R ay, R z1, R z2,
                                                             int* capped = nullptr)  // :76-87
{
  V3<R> lwi = to_local(wi, n);
  V3<R> m = sample_vndf(dist, lwi, ax, ay, z1, z2, capped);
  return to_world(m, n);
}
template <class R> static inline R eval_visible_normal(int dist, const V3<R>& wi, const V3<R>& wm, const V3<R>& n, R ax, R ay)  // :89-101
{
  return eval_vndf(dist, to_local(wi, n), to_local(wm, n), ax, ay);
}

}  // namespace orc
