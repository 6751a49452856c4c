// Test infrastructure (oracle only): restatement of the light sampling in LightSampler.h and of
// the environment map lookup / importance sampling in Envmap.h plus the CDF construction of
// CUDA_files/env_cameras.cu, templated on the scalar type R (see orc_math.hpp).
#pragma once
#include "orc_math.hpp"
#include <cstring>

namespace orc {

// Byte layouts of structs.h:42-103 (40-byte LightStruct, 92-byte TriangleLight).
struct LightStructRaw { u32 light_type; float emitted[3]; float p[3]; float pad[3]; };
struct TriangleLightRaw { float v0[3], v1[3], v2[3], n0[3], n1[3], n2[3]; u32 has_normals; float emission[3]; float area; };
static_assert(sizeof(LightStructRaw) == 40, "LightStruct layout");
static_assert(sizeof(TriangleLightRaw) == 92, "TriangleLight layout");
enum { POINT_LIGHT = 0, DIRECTIONAL_LIGHT = 1, TRIANGLES_AREA_LIGHT = 2, DISK_LIGHT = 3, SPHERICAL_LIGHT = 4 };

template <class R> static inline V3<R> ldv(const float* p) { return v3((R)p[0], (R)p[1], (R)p[2]); }

struct LightSet {
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
    default: break;
  }
}

}  // namespace orc
