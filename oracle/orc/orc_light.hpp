// Test infrastructure (oracle only): restatement of the light sampling in LightSampler.h and of
// the environment map lookup / importance sampling in Envmap.h plus the CDF construction of
// CUDA_files/env_cameras.cu, templated on the scalar type R (see orc_math.hpp).
#pragma once
#include "orc_math.hpp"
#include <cstring>
#include <vector>

namespace orc {

// Byte layouts of structs.h:42-103 (40-byte LightStruct, 92-byte TriangleLight).
struct LightStructRaw { u32 light_type; float emitted[3]; float p[3]; float pad[3]; };
struct TriangleLightRaw { float v0[3], v1[3], v2[3], n0[3], n1[3], n2[3]; u32 has_normals; float emission[3]; float area; };
static_assert(sizeof(LightStructRaw) == 40, "LightStruct layout");
static_assert(sizeof(TriangleLightRaw) == 92, "TriangleLight layout");
enum { POINT_LIGHT = 0, DIRECTIONAL_LIGHT = 1, TRIANGLES_AREA_LIGHT = 2, DISK_LIGHT = 3, SPHERICAL_LIGHT = 4, ENVMAP_LIGHT = 5 };

template <class R> static inline V3<R> ldv(const float* p) { return v3((R)p[0], (R)p[1], (R)p[2]); }

struct EnvMap;
struct LightSet {
  const EnvMap* env = nullptr;  // ENVMAP_LIGHT (type 5): the environment map as a light
  const LightStructRaw* lights = nullptr;
  long n_lights = 0;
  const TriangleLightRaw* tris = nullptr;
  long n_tris = 0;
  long oob = 0;  // clamped out-of-range triangle indices (reference indexes unguarded)
};

// evaluate_triangle_area_light, LightSampler.h:40-71.
template <class R> static inline void eval_triangle_area_light(const V3<R>& pos, const LightStructRaw& ls, LightSet& set,
                                                               V3<R>& dir, V3<R>& L, R& dist, u32& seed)
{
  float count_f, start_f;
  memcpy(&count_f, &ls.p[0], 4);   // triangle_count (float)
  memcpy(&start_f, &ls.p[1], 4);   // buffer_start_idx (float)
  u32 triangles = (u32)count_f;
  u32 tid = (u32)((float)(u32)(rnd_tea(seed) * (float)triangles) + start_f);
  if ((long)tid >= set.n_tris) { ++set.oob; tid = (u32)(set.n_tris - 1); }
  const TriangleLightRaw& tl = set.tris[tid];
  V3<R> uvw = sample_barycentric<R>(seed);
  V3<R> v0 = ldv<R>(tl.v0), v1 = ldv<R>(tl.v1), v2 = ldv<R>(tl.v2);
  V3<R> lp = v0 * uvw.x + v1 * uvw.y + v2 * uvw.z;
  V3<R> n = tl.has_normals ? normalize(ldv<R>(tl.n0) * uvw.x + ldv<R>(tl.n1) * uvw.y + ldv<R>(tl.n2) * uvw.z)
                           : normalize(cross(v1 - v0, v2 - v0));
  dir = lp - pos;
  R sq = dot(dir, dir);
  dist = std::sqrt(sq);
  dir = normalize(dir);
  R cp = std::fmax(dot(n, -dir), R(0));
  L = ldv<R>(ls.emitted) * ((R)tl.area * cp / sq * (R)triangles);
}
// evaluate_point_light :20-28, evaluate_directional_light :31-37.
template <class R> static inline void eval_point_light(const V3<R>& pos, const LightStructRaw& ls, V3<R>& dir, V3<R>& L, R& dist)
{
  dir = ldv<R>(ls.p) - pos;
  R r2 = dot(dir, dir);
  dist = std::sqrt(r2);
  dir = dir / dist;
  L = ldv<R>(ls.emitted) / r2;
}
template <class R> static inline void eval_directional_light(const LightStructRaw& ls, V3<R>& dir, V3<R>& L, R& dist)
{
  dir = normalize(-ldv<R>(ls.p));
  dist = (R)DEFAULT_MAX;
  L = ldv<R>(ls.emitted);
}
// evaluate_disk_area_light :73-101 (position p, radius/phi/theta in pad[0..2]).
template <class R> static inline void eval_disk_light(const V3<R>& pos, const LightStructRaw& ls, V3<R>& dir, V3<R>& L, R& dist, u32& seed)
{
  V3<R> lp = ldv<R>(ls.p);
  R radius = (R)ls.pad[0];
  R theta = (R)ls.pad[2] * K<R>::PI / R(180), phi = (R)ls.pad[1] * K<R>::PI / R(180);
  R area = K<R>::PI * radius * radius;
  R pdf = R(1) / area;
  V3<R> nrm = v3(std::sin(theta) * std::sin(phi), std::cos(theta), std::sin(theta) * std::cos(phi));
  V3<R> U, V;
  create_onb(nrm, U, V);
  R u1 = (R)rnd_tea(seed), u2 = (R)rnd_tea(seed);
  R r = std::sqrt(u1) * radius;
  R t = R(2) * K<R>::PI * u2;
  V3<R> dp = v3(r * std::cos(t), r * std::sin(t), R(0));
  dp = dp.x * U + dp.y * V + dp.z * nrm;
  lp = lp + dp;
  dir = lp - pos;
  R sq = dot(dir, dir);
  dist = std::sqrt(sq);
  dir = normalize(dir);
  R cp = std::fmax(dot(nrm, -dir), R(0));
  L = ldv<R>(ls.emitted) * (cp / sq) / pdf;
}
// evaluate_spherical_area_light :103-141 (position p, radius pad[0]).
template <class R> static inline void eval_sphere_light(const V3<R>& pos, const LightStructRaw& ls, V3<R>& dir, V3<R>& L, R& dist, u32& seed)
{
  V3<R> lp = ldv<R>(ls.p);
  R radius = (R)ls.pad[0];
  V3<R> vn = normalize(pos - lp);
  V3<R> U, V;
  create_onb(vn, U, V);
  R area = R(4) * K<R>::PI * radius * radius;
  R pdf = R(1) / area;
  R u1 = (R)rnd_tea(seed), u2 = (R)rnd_tea(seed);
  R z = u1;
  V3<R> sp = radius * v3(std::cos(R(2) * K<R>::PI * u2) * std::sqrt(R(1) - z * z), std::sin(R(2) * K<R>::PI * u2) * std::sqrt(R(1) - z * z), z);
  sp = sp.x * U + sp.y * V + sp.z * vn + lp;
  V3<R> nrm = normalize(sp - lp);
  dir = sp - pos;
  R sq = dot(dir, dir);
  dist = std::sqrt(sq);
  dir = normalize(dir);
  R cp = std::fmax(dot(nrm, -dir), R(0));
  L = ldv<R>(ls.emitted) * (cp / sq) / pdf;
}
}  // namespace orc

namespace orc {

// ------------------------------------------------------------------ environment map (Envmap.h)
// float4 texels (row-major, j = v row), normalized coordinates, bilinear filtering with REPEAT wrap
// (HDRLoader.cpp:232-236,286 sampler state); software FP32 weights, identical to the CUDA lookup.
struct EnvMap {
  const float* rgba = nullptr;
  int w = 0, h = 0;
  std::vector<float> marginal_pdf, marginal_cdf, conditional_pdf, conditional_cdf;
};
static inline int wrap_i(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }
static inline V3<float> env_tex(const EnvMap& E, float u, float v)
{
  float x = u * (float)E.w - 0.5f, y = v * (float)E.h - 0.5f;
  float fx = std::floor(x), fy = std::floor(y);
  float ax = x - fx, ay = y - fy;
  int i0 = wrap_i((int)fx, E.w), j0 = wrap_i((int)fy, E.h), i1 = wrap_i((int)fx + 1, E.w), j1 = wrap_i((int)fy + 1, E.h);
  const float* t00 = E.rgba + 4 * ((size_t)j0 * E.w + i0);
  const float* t10 = E.rgba + 4 * ((size_t)j0 * E.w + i1);
  const float* t01 = E.rgba + 4 * ((size_t)j1 * E.w + i0);
  const float* t11 = E.rgba + 4 * ((size_t)j1 * E.w + i1);
  float w00 = (1.0f - ax) * (1.0f - ay), w10 = ax * (1.0f - ay), w01 = (1.0f - ax) * ay, w11 = ax * ay;
  float c[3];
  for (int k = 0; k < 3; ++k) c[k] = t00[k] * w00 + t10[k] * w10 + t01[k] * w01 + t11[k] * w11;
  return v3(c[0], c[1], c[2]);
}
// env_lookup, Envmap.h:57-64
static inline V3<float> env_lookup(const EnvMap& E, const V3<float>& dir)
{
  float theta = std::acos(dir.y);
  float phi = std::atan2(dir.x, dir.z);
  float u = (phi + K<float>::PI) * 0.5f * K<float>::INV_PI;
  float v = (float)(1.0 - (double)(theta * K<float>::INV_PI));
  return env_tex(E, u, v);
}
// CDF construction of env_cameras.cu:23-75 (luminance x sin(theta), row marginal, conditional
// pdf/cdf, marginal pdf/cdf; the last conditional entry of the last row and the last marginal entry
// are set to 1).  Sums are accumulated sequentially in float in the reference's order.
static inline void env_build_cdf(EnvMap& E)
{
  const int W = E.w, H = E.h;
  std::vector<float> lum((size_t)W * H), mf(H);
  for (int j = 0; j < H; ++j)
    for (int i = 0; i < W; ++i) {
      float u = ((float)i + 0.5f) / (float)W, v = ((float)j + 0.5f) / (float)H;
      float theta = (1.0f - v) * K<float>::PI;
      V3<float> t = env_tex(E, u, v);
      lum[(size_t)j * W + i] = (t.x * 0.2989f + t.y * 0.5866f + t.z * 0.1145f) * std::sin(theta);
    }
  for (int j = 0; j < H; ++j) {
    float s = 0.0f;
    for (int i = 0; i < W; ++i) s += lum[(size_t)j * W + i];
    mf[j] = s / (float)W;
  }
  E.conditional_pdf.assign((size_t)W * H, 0.0f);
  E.conditional_cdf.assign((size_t)W * H, 0.0f);
  for (int j = 0; j < H; ++j) {
    float s = 0.0f;
    for (int i = 0; i < W; ++i) {
      s += lum[(size_t)j * W + i];
      E.conditional_pdf[(size_t)j * W + i] = lum[(size_t)j * W + i] / mf[j];
      E.conditional_cdf[(size_t)j * W + i] = (s / (float)W) / mf[j];
    }
  }
  E.conditional_cdf[(size_t)(H - 1) * W + (W - 1)] = 1.0f;
  E.marginal_pdf.assign(H, 0.0f);
  E.marginal_cdf.assign(H, 0.0f);
  float total = 0.0f;
  for (int j = 0; j < H; ++j) total += mf[j];
  float s = 0.0f;
  for (int j = 0; j < H; ++j) {
    s += mf[j];
    float m = total / (float)H;
    E.marginal_pdf[j] = mf[j] / m;
    E.marginal_cdf[j] = (s / (float)H) / m;
  }
  E.marginal_cdf[H - 1] = 1.0f;
}
// cdf_bsearch_marginal / cdf_bsearch_conditional, Envmap.h:23-55 (the read at middle-1 is skipped
// when middle is 0; for power-of-two sizes the search never reaches it).
static inline unsigned cdf_bsearch(const float* cdf, unsigned size, float xi)
{
  unsigned ts = size;
  unsigned middle = ts = ts >> 1;
  while (ts > 0) {
    unsigned odd = ts & 1;
    ts = ts >> 1;
    unsigned tmp = ts + odd;
    if (xi > cdf[middle]) middle = middle + tmp;
    else if (middle > 0 && xi < cdf[middle - 1]) middle = middle - tmp;
  }
  return middle;
}
// sample_environment, Envmap.h:66-98.
static inline void sample_environment(const EnvMap& E, V3<float>& dir, V3<float>& L, u32& t)
{
  const float M_2PIPI = 2.0f * K<float>::PI * K<float>::PI;
  float xi1 = rnd_tea(t), xi2 = rnd_tea(t);
  unsigned v_idx = cdf_bsearch(E.marginal_cdf.data(), (unsigned)E.h, xi1);
  float dv = v_idx > 0 ? (xi1 - E.marginal_cdf[v_idx - 1]) / (E.marginal_cdf[v_idx] - E.marginal_cdf[v_idx - 1]) : xi1 / E.marginal_cdf[v_idx];
  float pdf_m = E.marginal_pdf[v_idx];
  float v = ((float)v_idx + dv) / (float)E.h;
  const float* crow = E.conditional_cdf.data() + (size_t)v_idx * E.w;
  unsigned u_idx = cdf_bsearch(crow, (unsigned)E.w, xi2);
  float du = u_idx > 0 ? (xi2 - crow[u_idx - 1]) / (crow[u_idx] - crow[u_idx - 1]) : xi2 / crow[u_idx];
  float pdf_c = E.conditional_pdf[(size_t)v_idx * E.w + u_idx];
  float u = ((float)u_idx + du) / (float)E.w;
  float prob = pdf_m * pdf_c;
  float theta = (1.0f - v) * K<float>::PI;
  float phi = (2.0f * u - 1.0f) * K<float>::PI;
  float st, ct, sp, cp;
  ::sincosf(theta, &st, &ct);
  ::sincosf(phi, &sp, &cp);
  dir = v3(st * sp, ct, st * cp);
  V3<float> em = env_tex(E, u, v);
  L = em * st * M_2PIPI / prob;
}

}  // namespace orc

namespace orc {

// evaluate_direct_illumination dispatch, LightSampler.h:143-166.
template <class R> static inline void eval_direct(const V3<R>& pos, const LightStructRaw& ls, LightSet& set, V3<R>& dir, V3<R>& L,
                                                  R& dist, u32& seed)
{
  switch (ls.light_type) {
    case POINT_LIGHT: eval_point_light(pos, ls, dir, L, dist); break;
    case DIRECTIONAL_LIGHT: eval_directional_light(ls, dir, L, dist); break;
    case TRIANGLES_AREA_LIGHT: eval_triangle_area_light(pos, ls, set, dir, L, dist, seed); break;
    case DISK_LIGHT: eval_disk_light(pos, ls, dir, L, dist, seed); break;
    case SPHERICAL_LIGHT: eval_sphere_light(pos, ls, dir, L, dist, seed); break;
    case ENVMAP_LIGHT:
      if (set.env) {
        V3<float> d3, L3;
        sample_environment(*set.env, d3, L3, seed);
        dir = cvt<R>(d3);
        L = cvt<R>(L3);
        dist = (R)DEFAULT_MAX;
      }
      break;
    default: break;
  }
}

}  // namespace orc
