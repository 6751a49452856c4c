// Device math for the B200 path tracer: vector helpers, the reference's RNG streams, Fresnel
// terms, the double-precision complex conductor Fresnel, and the GGX / Beckmann microfacet
// models (sample, eval, pdf, multiscattering walks).  Every function follows the reference
// function it cites (open_rendering_framework/<file>:<line>); the arithmetic keeps the
// reference's operation order and its float/double promotions, because per-query results must
// agree with the reference's math within 1e-5 relative.  The translation units that include this
// header are compiled with --fmad=false so that no multiply-add is contracted implicitly; fused
// operations appear only where written as __fmaf_rn.
//
// Vector conventions (shared with the oracle): normalize(v) = v * (1/sqrtf(dot(v,v))), dot sums
// x, y, z left to right, reflect(i,n) = i - 2 n dot(n,i), faceforward(n,i,nref) =
// n * copysignf(1, dot(i,nref)).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define PT_HD __host__ __device__ __forceinline__
#define PT_D __device__ __forceinline__

namespace pt {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float kTwoSqrtPi = 1.12837916709551257390f;
constexpr float kSqrt2 = 1.41421356237309504880f;
constexpr float kSqrt1_2 = 0.707106781186547524401f;
constexpr float kDefaultMax = 1.e27f;  // RT_DEFAULT_MAX sentinel of the reference

enum Distribution : uint32_t { BECKMANN = 0, GGX = 1 };                       // structs.h:256-261
enum MicrofacetModel : uint32_t { WALTER = 0, VISIBLE_NORMALS = 1, MULTISCATTERING = 2 };  // structs.h:242-248

// Iteration cap for the reference's unbounded `while(true)` random walks; hitting it ends the
// walk as if the path had left the surface and is counted in the context's cap counter.
constexpr int kWalkCap = 4096;
constexpr int kNewtonCap = 256;

// ------------------------------------------------------------------ float3 helpers
PT_HD float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
PT_HD float3 f3s(float s) { return make_float3(s, s, s); }
PT_HD float3 operator-(const float3& a) { return f3(-a.x, -a.y, -a.z); }
PT_HD float3 operator+(const float3& a, const float3& b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
PT_HD float3 operator-(const float3& a, const float3& b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
PT_HD float3 operator*(const float3& a, const float3& b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
PT_HD float3 operator/(const float3& a, const float3& b) { return f3(a.x / b.x, a.y / b.y, a.z / b.z); }
PT_HD float3 operator*(const float3& a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
PT_HD float3 operator*(float s, const float3& a) { return f3(s * a.x, s * a.y, s * a.z); }
PT_HD float3 operator/(const float3& a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
PT_HD float3 operator+(const float3& a, float s) { return f3(a.x + s, a.y + s, a.z + s); }
PT_HD float3 operator-(float s, const float3& a) { return f3(s - a.x, s - a.y, s - a.z); }
PT_HD float dot(const float3& a, const float3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PT_HD float length(const float3& a) { return sqrtf(dot(a, a)); }
PT_HD float3 normalize(const float3& a) { float inv = 1.0f / sqrtf(dot(a, a)); return a * inv; }
PT_HD float3 cross(const float3& a, const float3& b)
{
  return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
PT_HD float3 reflect(const float3& i, const float3& n) { return i - 2.0f * n * dot(n, i); }
PT_HD float3 faceforward(const float3& n, const float3& i, const float3& nref) { return n * copysignf(1.0f, dot(i, nref)); }
PT_HD bool finite3(const float3& a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
PT_D float3 expf3(const float3& a) { return f3(expf(a.x), expf(a.y), expf(a.z)); }

// ------------------------------------------------------------------ RNG (random.h, md5.h)
// tea<16>, random.h:25-40.
PT_HD uint32_t tea16(uint32_t v0, uint32_t v1)
{
  uint32_t s0 = 0;
#pragma unroll
  for (int n = 0; n < 16; n++) {
    s0 += 0x9e3779b9u;
    v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
    v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
  }
  return v0;
}
// tea_hash / rnd_tea, random.h:117-127 (the draw may round up to exactly 1.0f).
PT_HD float rnd_tea(uint32_t& prev)
{
  prev = tea16(prev, 100u);
  return (float)(prev & 0x7FFFFFFFu) / (float)0x80000000u;
}
// lcg / rnd, random.h:43-61.
PT_HD float rnd_lcg(uint32_t& prev)
{
  prev = 1664525u * prev + 1013904223u;
  return (float)(prev & 0x00FFFFFFu) / (float)0x01000000;
}
// MD5 (RFC 1321) of the 8-byte message (x, y): md5.h:58-200 with length 8 and rand_md5(uint2)
// :218-225 (scrambler 0).  Fully unrolled so that message-word selection and shift amounts are
// compile-time constants.
struct Md5Tables {
  __host__ __device__ static constexpr uint32_t T(int i)
  {
    constexpr uint32_t t[64] = {
        0xd76aa478u, 0xe8c7b756u, 0x242070dbu, 0xc1bdceeeu, 0xf57c0fafu, 0x4787c62au, 0xa8304613u, 0xfd469501u,
        0x698098d8u, 0x8b44f7afu, 0xffff5bb1u, 0x895cd7beu, 0x6b901122u, 0xfd987193u, 0xa679438eu, 0x49b40821u,
        0xf61e2562u, 0xc040b340u, 0x265e5a51u, 0xe9b6c7aau, 0xd62f105du, 0x02441453u, 0xd8a1e681u, 0xe7d3fbc8u,
        0x21e1cde6u, 0xc33707d6u, 0xf4d50d87u, 0x455a14edu, 0xa9e3e905u, 0xfcefa3f8u, 0x676f02d9u, 0x8d2a4c8au,
        0xfffa3942u, 0x8771f681u, 0x6d9d6122u, 0xfde5380cu, 0xa4beea44u, 0x4bdecfa9u, 0xf6bb4b60u, 0xbebfbc70u,
        0x289b7ec6u, 0xeaa127fau, 0xd4ef3085u, 0x04881d05u, 0xd9d4d039u, 0xe6db99e5u, 0x1fa27cf8u, 0xc4ac5665u,
        0xf4292244u, 0x432aff97u, 0xab9423a7u, 0xfc93a039u, 0x655b59c3u, 0x8f0ccc92u, 0xffeff47du, 0x85845dd1u,
        0x6fa87e4fu, 0xfe2ce6e0u, 0xa3014314u, 0x4e0811a1u, 0xf7537e82u, 0xbd3af235u, 0x2ad7d2bbu, 0xeb86d391u};
    return t[i];
  }
};
PT_HD uint32_t rotl32(uint32_t x, int n) { return (x << n) | (x >> (32 - n)); }
PT_HD void md5_u2(uint32_t x, uint32_t y, uint32_t& h0, uint32_t& h1)
{
  const uint32_t M[16] = {x, y, 0x80u, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 64u, 0};
  constexpr int S[16] = {7, 12, 17, 22, 5, 9, 14, 20, 4, 11, 16, 23, 6, 10, 15, 21};
  uint32_t a = 0x67452301u, b = 0xefcdab89u, c = 0x98badcfeu, d = 0x10325476u;
#pragma unroll
  for (int i = 0; i < 64; ++i) {
    uint32_t f;
    int g;
    if (i < 16) { f = (b & c) | (~b & d); g = i; }
    else if (i < 32) { f = (b & d) | (c & ~d); g = (5 * i + 1) & 15; }
    else if (i < 48) { f = b ^ c ^ d; g = (3 * i + 5) & 15; }
    else { f = c ^ (b | ~d); g = (7 * i) & 15; }
    uint32_t t = d;
    d = c;
    c = b;
    b = b + rotl32(a + f + M[g] + Md5Tables::T(i), S[(i >> 4) * 4 + (i & 3)]);
    a = t;
  }
  h0 = a + 0x67452301u;
  h1 = b + 0xefcdab89u;
}
// rnd_accurate, random.h:134-142: the seed becomes the low 64 bits of the digest; the draw is
// (digest & 0x7FFF...) / 2^63 in double, rounded to float.
PT_HD float md5_draw(uint32_t h0, uint32_t h1)
{
  unsigned long long l = (((unsigned long long)h1 << 32) | h0) & 0x7FFFFFFFFFFFFFFFull;
  return (float)((double)l / 9223372036854775808.0);
}
PT_HD float rnd_md5(uint2& s)
{
  uint32_t h0, h1;
  md5_u2(s.x, s.y, h0, h1);
  s.x = h0;
  s.y = h1;
  return md5_draw(h0, h1);
}

// ------------------------------------------------------------------ helpers.h
// create_onb(n, U, V) for a normalized n, helpers.h:92-103.
PT_HD void create_onb(const float3& n, float3& U, float3& V)
{
  U = cross(n, f3(0.0f, 1.0f, 0.0f));
  if (dot(U, U) < 1e-3f) U = cross(n, f3(1.0f, 0.0f, 0.0f));
  U = normalize(U);
  V = cross(n, U);
}
PT_HD float3 to_local(const float3& w, const float3& n)  // helpers.h:284-291
{
  float3 u, v;
  create_onb(n, u, v);
  return normalize(f3(dot(w, u), dot(w, v), dot(w, n)));
}
PT_HD float3 to_world(const float3& w, const float3& n)  // helpers.h:294-299
{
  float3 u, v;
  create_onb(n, u, v);
  return normalize(u * w.x + v * w.y + n * w.z);
}
// Double-precision erfinv of helpers.h:301-377: M. Giles, "Approximating the erfinv function",
// GPU Computing Gems Jade Edition (2011), three polynomial branches in w = -log((1-x)(1+x)).
// One out-of-line copy: the Beckmann sampler calls it three times, and inlined copies (a double log
// and three long polynomials each) crowded the instruction cache of the kernels that use it.
static __host__ __device__ __noinline__ double erfinv_giles(double x)
{
  double w = -log((1.0 - x) * (1.0 + x)), p;
  if (w < 6.25) {
    w = w - 3.125;
    p = -3.6444120640178196996e-21;
    p = -1.685059138182016589e-19 + p * w;
    p = 1.2858480715256400167e-18 + p * w;
    p = 1.115787767802518096e-17 + p * w;
    p = -1.333171662854620906e-16 + p * w;
    p = 2.0972767875968561637e-17 + p * w;
    p = 6.6376381343583238325e-15 + p * w;
    p = -4.0545662729752068639e-14 + p * w;
    p = -8.1519341976054721522e-14 + p * w;
    p = 2.6335093153082322977e-12 + p * w;
    p = -1.2975133253453532498e-11 + p * w;
    p = -5.4154120542946279317e-11 + p * w;
    p = 1.051212273321532285e-09 + p * w;
    p = -4.1126339803469836976e-09 + p * w;
    p = -2.9070369957882005086e-08 + p * w;
    p = 4.2347877827932403518e-07 + p * w;
    p = -1.3654692000834678645e-06 + p * w;
    p = -1.3882523362786468719e-05 + p * w;
    p = 0.0001867342080340571352 + p * w;
    p = -0.00074070253416626697512 + p * w;
    p = -0.0060336708714301490533 + p * w;
    p = 0.24015818242558961693 + p * w;
    p = 1.6536545626831027356 + p * w;
  } else if (w < 16.0) {
    w = sqrt(w) - 3.25;
    p = 2.2137376921775787049e-09;
    p = 9.0756561938885390979e-08 + p * w;
    p = -2.7517406297064545428e-07 + p * w;
    p = 1.8239629214389227755e-08 + p * w;
    p = 1.5027403968909827627e-06 + p * w;
    p = -4.013867526981545969e-06 + p * w;
    p = 2.9234449089955446044e-06 + p * w;
    p = 1.2475304481671778723e-05 + p * w;
    p = -4.7318229009055733981e-05 + p * w;
    p = 6.8284851459573175448e-05 + p * w;
    p = 2.4031110387097893999e-05 + p * w;
    p = -0.0003550375203628474796 + p * w;
    p = 0.00095328937973738049703 + p * w;
    p = -0.0016882755560235047313 + p * w;
    p = 0.0024914420961078508066 + p * w;
    p = -0.0037512085075692412107 + p * w;
    p = 0.005370914553590063617 + p * w;
    p = 1.0052589676941592334 + p * w;
    p = 3.0838856104922207635 + p * w;
  } else {
    w = sqrt(w) - 5.0;
    p = -2.7109920616438573243e-11;
    p = -2.5556418169965252055e-10 + p * w;
    p = 1.5076572693500548083e-09 + p * w;
    p = -3.7894654401267369937e-09 + p * w;
    p = 7.6157012080783393804e-09 + p * w;
    p = -1.4960026627149240478e-08 + p * w;
    p = 2.9147953450901080826e-08 + p * w;
    p = -6.7711997758452339498e-08 + p * w;
    p = 2.2900482228026654717e-07 + p * w;
    p = -9.9298272942317002539e-07 + p * w;
    p = 4.5260625972231537039e-06 + p * w;
    p = -1.9681778105531670567e-05 + p * w;
    p = 7.5995277030017761139e-05 + p * w;
    p = -0.00021503011930044477347 + p * w;
    p = -0.00013871931833623122026 + p * w;
    p = 1.0103004648645343977 + p * w;
    p = 4.8499064014085844221 + p * w;
  }
  return p * x;
}
PT_D float gauss_inv_cdf(float z) { return kSqrt2 * (float)erfinv_giles(2.0f * z - 1.0f); }  // helpers.h:380-383
PT_D float gauss_cdf(float h) { return 0.5f + 0.5f * erff(kSqrt1_2 * h); }                     // helpers.h:386-389

// ------------------------------------------------------------------ sampler.h
PT_HD void rotate_to_normal(const float3& n, float3& v)  // :12-24
{
  if (n.z < -0.999999f) { v = f3(-v.y, -v.x, -v.z); return; }
  float a = 1.0f / (1.0f + n.z);
  float b = -n.x * n.y * a;
  v = f3(1.0f - n.x * n.x * a, b, -n.x) * v.x + f3(b, 1.0f - n.y * n.y * a, -n.y) * v.y + n * v.z;
}
PT_D float3 sample_cosine_weighted(const float3& n, uint32_t& t)  // :51-64
{
  float ct = sqrtf(rnd_tea(t));
  float phi = 2.0f * kPi * rnd_tea(t);
  float st = sqrtf(1.0f - ct * ct);
  float sp, cp;
  sincosf(phi, &sp, &cp);
  float3 v = f3(st * cp, st * sp, ct);
  rotate_to_normal(n, v);
  return v;
}
PT_D float3 sample_barycentric(uint32_t& t)  // :103-116
{
  float sx = sqrtf(rnd_tea(t));
  float xi2 = rnd_tea(t);
  return f3(1.0f - sx, (1.0f - xi2) * sx, xi2 * sx);
}

// ------------------------------------------------------------------ Fresnel.h
PT_HD float fresnel_rs(float c1, float c2, float e) { return (e * c1 - c2) / (e * c1 + c2); }
PT_HD float fresnel_rp(float c1, float c2, float e) { return (c1 - e * c2) / (c1 + e * c2); }
PT_HD float fresnel_R(float c1, float c2, float e)  // :26-32
{
  float rs = fresnel_rs(c1, c2, e), rp = fresnel_rp(c1, c2, e);
  return (rs * rs + rp * rp) * 0.5f;
}
// Reflectance of a smooth interface for the cosine of incidence c and relative index e, 1 under total
// internal reflection: the block `R = 1; sin2 = e*e*(1 - c*c); if (sin2 < 1) R = fresnel_R(c, sqrt(1 - sin2), e)`
// that lambertian_interface_shader.cu:69-76 and rough_diffuse_shader.cu:90-97 repeat for every direction.
PT_HD float fresnel_interface(float c, float e)
{
  float R = 1.0f;
  const float st2 = e * e * (1.0f - c * c);
  if (st2 < 1.0f) R = fresnel_R(c, sqrtf(1.0f - st2), e);
  return R;
}
PT_HD float fresnel_R(const float3& wi, const float3& wm, float e)  // :42-54
{
  float c1 = dot(wi, wm);
  float c22 = 1.0f - e * e * (1.0f - c1 * c1);
  if (c22 <= 0.0f) return 1.0f;
  float c2 = sqrtf(c22);
  float rs = fresnel_rs(c1, c2, e), rp = fresnel_rp(c1, c2, e);
  return (rs * rs + rp * rp) * 0.5f;
}

// ------------------------------------------------------------------ MyComplex.h (double parts)
struct Cx { double re, im; };
struct Cx3 { Cx c[3]; };
PT_D float cabs_f(const Cx& c) { float r = (float)c.re, i = (float)c.im; return sqrtf(r * r + i * i); }  // :18-23
PT_D Cx cmul(const Cx& a, const Cx& b) { return Cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
PT_D Cx cdiv(const Cx& a, const Cx& b)  // :148-153 (den = powf(|b|, 2) in float)
{
  Cx num = cmul(a, Cx{b.re, -b.im});
  double den = (double)powf(cabs_f(b), 2.0f);
  double s = 1.0 / den;
  return Cx{num.re * s, num.im * s};
}
PT_D Cx cdiv_f(float a, const Cx& b)  // :155-160
{
  Cx num{(double)a * b.re, (double)a * -b.im};
  double den = (double)powf(cabs_f(b), 2.0f);
  double s = 1.0 / den;
  return Cx{num.re * s, num.im * s};
}
PT_D float cphase(const Cx& c)  // :169-185
{
  double r = c.re, i = c.im, th;
  if (r == 0 && i > 0) th = (double)(kPi / 2.0f);
  else if (r == 0 && i < 0) th = (double)(-kPi / 2.0f);
  else if (r == 0 && i == 0) th = 0;
  else th = atan(i / r);
  if (r < 0) th += (double)kPi;
  return (float)th;
}
PT_D Cx csq_polar(const Cx& c)  // pow(c, 2), :187-193
{
  double ab = pow((double)cabs_f(c), 2.0);
  double th = (double)(cphase(c) * 2.0f);
  double s, co;
  sincos(th, &s, &co);
  return Cx{ab * co, ab * s};
}
PT_D Cx csqrt_polar(const Cx& c)  // :195-202
{
  double ab = (double)sqrtf(cabs_f(c));
  double th = (double)(cphase(c) / 2.0f);
  double s, co;
  sincos(th, &s, &co);
  return Cx{ab * co, ab * s};
}
// One channel of fresnel_MyComplex_R, Fresnel.h:78-91.  Out of line: its three inlined copies per
// conductor (double atan, sincos and divisions each) crowded the conductor kernel's instruction cache.
static __device__ __noinline__ float fresnel_complex1(float ci, float si, const Cx& e)
{
  Cx st{e.re * (double)si, e.im * (double)si};
  Cx p2 = csq_polar(st);
  Cx ct = csqrt_polar(Cx{(double)1.0f - p2.re, -p2.im});
  Cx ec{e.re * (double)ci, e.im * (double)ci};
  Cx r_ort = cdiv(Cx{ec.re - ct.re, ec.im - ct.im}, Cx{ec.re + ct.re, ec.im + ct.im});
  Cx ect = cmul(e, ct);
  Cx r_par = cdiv(Cx{(double)ci - ect.re, -ect.im}, Cx{(double)ci + ect.re, ect.im});
  float a = cabs_f(r_ort), b = cabs_f(r_par);
  return 0.5f * (powf(a, 2.0f) + powf(b, 2.0f));
}
PT_D float3 fresnel_complex(const float3& wi, const float3& wm, const Cx3& e)
{
  float ci = dot(wi, wm);
  float si = sqrtf(1.0f - ci * ci);
  return f3(fresnel_complex1(ci, si, e.c[0]), fresnel_complex1(ci, si, e.c[1]), fresnel_complex1(ci, si, e.c[2]));
}

// ------------------------------------------------------------------ GGX (MicrofacetGGX.h)
PT_D float alpha_i(const float3& wi, float ax, float ay)  // :9-17 (same in MicrofacetBeckmann.h:13-21)
{
  float inv_sin2 = 1.0f / (1.0f - wi.z * wi.z);
  if (wi.z == 1.0f || wi.z == -1.0f) inv_sin2 = 0.0f;
  float c2 = wi.x * wi.x * inv_sin2;
  float s2 = wi.y * wi.y * inv_sin2;
  return sqrtf(c2 * ax * ax + s2 * ay * ay);
}
PT_D float ggx_lambda(const float3& wi, float ax, float ay)  // :20-30
{
  if (wi.z > 0.99999f) return 0.0f;
  if (wi.z < -0.99999f) return -1.0f;
  float th = acosf(wi.z);
  float a = 1.0f / tanf(th) / alpha_i(wi, ax, ay);
  return 0.5f * (-1.0f + sqrtf(1.0f + 1.0f / (a * a)) * (a > 0 ? 1.0f : -1.0f));
}
PT_D float ggx_projected_area(const float3& wi, float ax, float ay)  // :33-45
{
  if (wi.z > 0.9999f) return 1.0f;
  if (wi.z < -0.9999f) return 0.0f;
  float alpha = alpha_i(wi, ax, ay);
  float th = acosf(wi.z);
  float st = sinf(th);
  return 0.5f * (wi.z + sqrtf(wi.z * wi.z + st * st * alpha * alpha));
}
PT_D float ggx_G1_cos(float c, float a2)  // :54-60
{
  float c2 = c * c;
  float t2 = (1.0f - c2) / c2;
  return 2.0f / (1.0f + sqrtf(1.0f + a2 * t2));
}
PT_D float ggx_G1(const float3& v, const float3& m, const float3& n, float ag)  // :77-83
{
  float cv = dot(v, n);
  if (cv * dot(v, m) <= 0) return 0.0f;
  return ggx_G1_cos(cv, ag * ag);
}
PT_D float ggx_G1_aniso(const float3& v, const float3& m, const float3& n, float ax, float ay)  // :63-74
{
  float alpha = alpha_i(normalize(to_local(v, n)), ax, ay);
  float a2 = alpha * alpha;
  float cv = dot(v, n);
  if (cv * dot(v, m) <= 0) return 0.0f;
  return ggx_G1_cos(cv, a2);
}
PT_D float ggx_G_height(const float3& wi, float h, float ax, float ay)  // :93-107
{
  if (wi.z > 0.9999f) return 1.0f;
  if (wi.z <= 0.0f) return 0.0f;
  return powf(gauss_cdf(h), ggx_lambda(wi, ax, ay));
}
PT_D float3 ggx_sample_hemisphere(const float3& n, float z1, float z2, float ag)  // :123-139
{
  float phi = 2.0f * kPi * z2;
  float th = atanf(ag * sqrtf(z1) / sqrtf(1.0f - z1));
  float ct = cosf(th), st = sinf(th);
  float3 m = f3(st * cosf(phi), st * sinf(phi), ct);
  float3 v1, v2;
  create_onb(n, v1, v2);
  return v1 * m.x + v2 * m.y + n * m.z;
}
PT_D float2 ggx_P22(float theta_i, float z1, float z2)  // :142-187
{
  if (theta_i < 0.0001f) {
    float r = sqrtf(z1 / (1.0f - z1));
    float phi = kPi * 2.0f * z2;
    return make_float2(r * cosf(phi), r * sinf(phi));
  }
  float sin_i = sinf(theta_i);
  float cos_i = fmaxf(cosf(theta_i), (float)1e-7);
  float tan_i = sin_i / cos_i;
  float proj = 0.5f * (cos_i + 1.0f);
  if (proj < 0.0001f || proj != proj) return make_float2(0.0f, 0.0f);
  float c = 1.0f / proj;
  float A = 2.0f * z1 / cos_i / c - 1.0f;
  float B = tan_i;
  float tmp = 1.0f / (A * A - 1.0f);
  float D = sqrtf(fmaxf(0.0f, B * B * tmp * tmp - (A * A - B * B) * tmp));
  float sx1 = B * tmp - D, sx2 = B * tmp + D;
  float sx = (A < 0.0f || sx2 > 1.0f / tan_i) ? sx1 : sx2;
  float S, zz2;
  if (z2 > 0.5f) { S = 1.0f; zz2 = 2.0f * (z2 - 0.5f); }
  else { S = -1.0f; zz2 = 2.0f * (0.5f - z2); }
  float z = (zz2 * (zz2 * (zz2 * 0.27385f - 0.73369f) + 0.46341f)) /
            (zz2 * (zz2 * (zz2 * 0.093073f + 0.309420f) - 1.0000f) + 0.597999f);
  return make_float2(sx, S * z * sqrtf(1.0f + sx * sx));
}
PT_D float ggx_eval_ndf(const float3& wm, float ax, float ay)  // :219-231 with :48-53
{
  if (wm.z <= 0.0f) return 0.0f;
  float sx = -wm.x / wm.z, sy = -wm.y / wm.z;
  float tmp = 1.0f + sx * sx / (ax * ax) + sy * sy / (ay * ay);
  float pdf = 1.0f / (kPi * ax * ay) / (tmp * tmp);
  return pdf / (wm.z * wm.z * wm.z * wm.z);
}
PT_D float ggx_eval_vndf(const float3& wi, const float3& wm, float ax, float ay)  // :234-251
{
  if (wm.z <= 0.0f) return 0.0f;
  float area = ggx_projected_area(wi, ax, ay);
  if (area == 0.0f) return 0.0f;
  float c = 1.0f / area;
  return c * fmaxf(0.0f, dot(wi, wm)) * ggx_eval_ndf(wm, ax, ay);
}
PT_D float ggx_distribution(const float3& m, const float3& n, float alpha)  // :643-655
{
  float D = 0.0f;
  float c = dot(m, n);
  if (c > 0.0f) {
    float c2 = c * c, s2 = 1.0f - c2, a2 = alpha * alpha;
    float coeff = c2 * (a2 + s2 / c2);
    D = a2 * kInvPi / (coeff * coeff);
  }
  return D;
}

// ------------------------------------------------------------------ Beckmann (MicrofacetBeckmann.h)
PT_D float bk_lambda(const float3& wi, float ax, float ay)  // :24-42
{
  if (wi.z > 0.9999f) return 0.0f;
  if (wi.z < -0.9999f) return -1.0f;
  float th = acosf(wi.z);
  float t = tanf(th);
  if (isinf(t)) return 0.0f;
  float a = 1.0f / (t * alpha_i(wi, ax, ay));
  return 0.5f * (erff(a) - 1.0f) + 0.25f * kTwoSqrtPi / a * expf(-a * a);
}
PT_D float bk_projected_area(const float3& wi, float ax, float ay)  // :45-58
{
  if (wi.z > 0.9999f) return 1.0f;
  if (wi.z < -0.9999f) return 0.0f;
  float alpha = alpha_i(wi, ax, ay);
  float th = acosf(wi.z);
  float a = 1.0f / tanf(th) / alpha;
  double rhs = 0.25 * (double)kTwoSqrtPi * (double)alpha * (double)sinf(th) * (double)expf(-a * a);
  return (float)((double)(0.5f * (erff(a) + 1.0f) * wi.z) + rhs);
}
PT_D float bk_G1_cos(float c, float ab2)  // :68-75 (denominator in double, as written there)
{
  float c2 = c * c;
  float t2 = (1.0f - c2) / c2;
  float a2 = 1.0f / (ab2 * t2);
  float a = sqrtf(a2);
  if (!(a < 1.6f)) return 1.0f;
  double den = (double)(1.0f + 2.276f * a) + 2.577 * (double)a2;
  return (float)((double)(3.535f * a + 2.181f * a2) / den);
}
PT_D float bk_G1(const float3& v, const float3& m, const float3& n, float width)  // :78-86
{
  float cv = dot(v, n);
  if (dot(v, m) * cv <= 0) return 0.0f;
  return bk_G1_cos(cv, width * width);
}
PT_D float bk_G1_aniso(const float3& v, const float3& m, const float3& n, float ax, float ay)  // :89-98
{
  float width = alpha_i(to_local(v, n), ax, ay);
  float cv = dot(v, n);
  if (dot(v, m) * cv <= 0) return 0.0f;
  return bk_G1_cos(cv, width * width);
}
PT_D float bk_G_height(const float3& wi, float h, float ax, float ay)  // :108-127
{
  if (wi.z > 0.9999f) return 1.0f;
  if (wi.z <= 0.0f) return 0.0f;
  return powf(gauss_cdf(h), bk_lambda(wi, ax, ay));
}
PT_D float bk_G_avg(const float3& wi, float ax, float ay)  // :130-141
{
  if (wi.z > 0.9999f) return 1.0f;
  if (wi.z <= 0.0f) return 0.0f;
  return 1.0f / (1.0f + bk_lambda(wi, ax, ay));
}
PT_D float3 bk_sample_hemisphere(const float3& n, float z1, float z2, float width)  // :144-158
{
  float phi = 2.0f * kPi * z2;
  float tan_t = -width * width * logf(1.0f - z1);
  float th = atanf(sqrtf(tan_t));
  float ct = cosf(th), st = sinf(th);
  float3 m = f3(st * cosf(phi), st * sinf(phi), ct);
  float3 v1, v2;
  create_onb(n, v1, v2);
  return v1 * m.x + v2 * m.y + n * m.z;
}
// Visible-slope sampling by Newton/bisection on erf, :161-210.  Bounded by kNewtonCap.
PT_D float2 bk_P22(float theta_i, float z1, float z2, int* capped)
{
  if (theta_i < 0.0001f) {
    float r = sqrtf(-logf(z1));
    float phi = kPi * 2.0f * z2;
    return make_float2(r * cosf(phi), r * sinf(phi));
  }
  float sin_i = sinf(theta_i), cos_i = cosf(theta_i);
  float slope_i = cos_i / sin_i;
  float a = cos_i / sin_i;
  float proj = 0.5f * (erff(a) + 1.0f) * cos_i + 0.25f * kTwoSqrtPi * sin_i * expf(-a * a);
  if (proj < 0.0001f || proj != proj) return make_float2(0.0f, 0.0f);
  float c = 1.0f / proj;
  float emin = -0.9999f;
  float emax = fmaxf(emin, erff(slope_i));
  float ecur = 0.5f * (emin + emax);
  int it = 0;
  while (emax - emin > 0.00001f) {
    if (++it > kNewtonCap) { *capped = 1; break; }
    if (!(ecur >= emin && ecur <= emax)) ecur = 0.5f * (emin + emax);
    float sv = (float)erfinv_giles((double)ecur);
    float cdf;
    if (sv >= slope_i) cdf = 1.0f;
    else {
      double inner = 0.25 * (double)kTwoSqrtPi * (double)sin_i * (double)expf(-sv * sv) +
                     (double)(cos_i * (0.5f + 0.5f * erff(sv)));
      cdf = (float)((double)c * inner);
    }
    float diff = cdf - z1;
    if (fabsf(diff) < 0.00001f) break;
    if (diff > 0.0f) {
      if (emax == ecur) break;
      emax = ecur;
    } else {
      if (emin == ecur) break;
      emin = ecur;
    }
    float deriv = 0.5f * c * cos_i - 0.5f * c * sin_i * sv;
    ecur -= diff / deriv;
  }
  return make_float2((float)erfinv_giles((double)fminf(emax, fmaxf(emin, ecur))), (float)erfinv_giles((double)(2.0f * z2 - 1.0f)));
}
PT_D float bk_eval_ndf(const float3& wm, float ax, float ay)  // :249-261 with :61-65
{
  if (wm.z <= 0.0f) return 0.0f;
  float sx = -wm.x / wm.z, sy = -wm.y / wm.z;
  float pdf = 1.0f / (kPi * ax * ay) * expf(-sx * sx / (ax * ax) - sy * sy / (ay * ay));
  return pdf / (wm.z * wm.z * wm.z * wm.z);
}
PT_D float bk_eval_vndf(const float3& wi, const float3& wm, float ax, float ay)  // :264-281
{
  if (wm.z <= 0.0f) return 0.0f;
  float area = bk_projected_area(wi, ax, ay);
  if (area == 0.0f) return 0.0f;
  float c = 1.0f / area;
  return c * fmaxf(0.0f, dot(wi, wm)) * bk_eval_ndf(wm, ax, ay);
}
PT_D float bk_distribution(const float3& m, const float3& n, float alpha)  // :739-750
{
  float D = 0.0f;
  float c = dot(m, n);
  if (c > 0.0001f) {
    float c2 = c * c, s2 = 1.0f - c2, a2 = alpha * alpha;
    D = expf(-s2 / (c2 * a2)) * kInvPi / (a2 * c2 * c2);
  }
  return D;
}

// ------------------------------------------------------------------ distribution dispatch
// GGX :190-207 / Beckmann :213-231 (identical apart from the slope sampler).
PT_D float3 sample_vndf(uint32_t dist, const float3& wi, float ax, float ay, float z1, float z2, int* capped)
{
  float3 w11 = normalize(f3(ax * wi.x, ay * wi.y, wi.z));
  float th = acosf(w11.z);
  float2 s11 = (dist == GGX) ? ggx_P22(th, z1, z2) : bk_P22(th, z1, z2, capped);
  float phi = atan2f(w11.y, w11.x);
  float sp = sinf(phi), cp = cosf(phi);
  float sx = cp * s11.x - sp * s11.y;
  float sy = sp * s11.x + cp * s11.y;
  sx *= ax;
  sy *= ay;
  if (!isfinite(sx) || sx != sx) {
    if (wi.z > 0) return f3(0.0f, 0.0f, 1.0f);
    return normalize(f3(wi.x, wi.y, 0.0f));
  }
  return normalize(f3(-sx, -sy, 1.0f));
}
PT_D float eval_vndf(uint32_t dist, const float3& wi, const float3& wm, float ax, float ay)
{
  return dist == GGX ? ggx_eval_vndf(wi, wm, ax, ay) : bk_eval_vndf(wi, wm, ax, ay);
}
// Microfacet.h:76-87 and :89-101.
PT_D float3 sample_visible_normal(uint32_t dist, const float3& wi, const float3& n, float ax, float ay, float z1, float z2, int* capped)
{
  return to_world(sample_vndf(dist, to_local(wi, n), ax, ay, z1, z2, capped), n);
}
PT_D float eval_visible_normal(uint32_t dist, const float3& wi, const float3& wm, const float3& n, float ax, float ay)
{
  return eval_vndf(dist, to_local(wi, n), to_local(wm, n), ax, ay);
}
// Microfacet.h:20-36, :54-64.
PT_D float masking_G1(uint32_t dist, const float3& v, const float3& m, const float3& n, float alpha)
{
  return dist == GGX ? ggx_G1(v, m, n, alpha) : bk_G1(v, m, n, alpha);
}
PT_D float masking_G1_aniso(uint32_t dist, const float3& v, const float3& m, const float3& n, float ax, float ay)
{
  return dist == GGX ? ggx_G1_aniso(v, m, n, ax, ay) : bk_G1_aniso(v, m, n, ax, ay);
}
PT_D float3 sample_normal(uint32_t dist, const float3& n, float z1, float z2, float alpha)
{
  return dist == GGX ? ggx_sample_hemisphere(n, z1, z2, alpha) : bk_sample_hemisphere(n, z1, z2, alpha);
}
// Walter BSDF eval, GGX :658-688 / Beckmann :753-786.
PT_D float walter_bsdf(uint32_t dist, const float3& wi, const float3& wo, const float3& n, float alpha, float eta)
{
  bool refl = dot(wo, n) > 0.0f;
  float3 m = refl ? normalize(wo + wi) : -normalize(eta * wi + wo);
  float Rf = fresnel_R(wi, m, eta);
  float idn = fabsf(dot(wi, n)), odn = fabsf(dot(wo, n));
  float G = masking_G1(dist, wi, m, n, alpha) * masking_G1(dist, wo, m, n, alpha);
  float T = 1.0f - Rf;
  float D = dist == GGX ? ggx_distribution(m, n, alpha) : bk_distribution(m, n, alpha);
  if (refl) return Rf * G * D / (4.0f * idn * odn);
  float idm = fabsf(dot(wi, m)), odm = fabsf(dot(wo, m));
  float coeff = (idm * odm) / (idn * odn);
  float den = (eta * idm + odm);
  return T * G * D * coeff / (den * den);
}

// ------------------------------------------------------------------ multiscattering walks
PT_D float sample_height(uint32_t dist, const float3& wr, float hr, float z, float ax, float ay)
{
  if (dist == GGX) {  // MicrofacetGGX.h:254-276
    if (wr.z > 0.9999f) return kDefaultMax;
    if (wr.z < -0.9999f) return gauss_inv_cdf(z * gauss_cdf(hr));
    if (fabsf(wr.z) < 0.00001f) return hr;
    float G1 = ggx_G_height(wr, hr, ax, ay);
    if (z > 1.0f - G1) return kDefaultMax;
    return gauss_inv_cdf(gauss_cdf(hr) / powf(1.0f - z, 1.0f / ggx_lambda(wr, ax, ay)));
  }
  // MicrofacetBeckmann.h:284-307
  if (wr.z > 0.999f) return kDefaultMax;
  if (wr.z < -0.999f) return gauss_inv_cdf(z * gauss_cdf(hr));
  if (fabsf(wr.z) < 0.00001f) return hr;
  float G1 = bk_G_avg(wr, ax, ay);
  if (z > 1.0f - G1) return kDefaultMax;
  float gcdf = gauss_cdf(hr);
  float p = powf(1.0f - z, 1.0f / bk_lambda(wr, ax, ay));
  return gauss_inv_cdf(gcdf / p);
}
PT_D float G_height(uint32_t dist, const float3& wi, float h, float ax, float ay)
{
  return dist == GGX ? ggx_G_height(wi, h, ax, ay) : bk_G_height(wi, h, ax, ay);
}
// Dielectric phase sample, GGX :279-304 / Beckmann :310-338.
PT_D float3 sample_dielectric_phase(uint32_t dist, const float3& wi, float3& wm, float m_eta, uint32_t& seed, bool wi_out,
                                    bool& wo_out, float ax, float ay, int* capped)
{
  float z1 = rnd_tea(seed), z2 = rnd_tea(seed);
  float eta = wi_out ? m_eta : 1.0f / m_eta;
  wm = wi_out ? sample_vndf(dist, wi, ax, ay, z1, z2, capped) : -sample_vndf(dist, -wi, ax, ay, z1, z2, capped);
  float ct = fabsf(dot(wm, wi));
  float st2 = eta * eta * (1.0f - ct * ct);
  float ctt = sqrtf(1.0f - st2);
  float F = st2 < 1.0f ? fresnel_R(ct, ctt, eta) : 1.0f;
  if (rnd_tea(seed) <= F) return normalize(-wi + 2.0f * wm * dot(wi, wm));
  wo_out = !wi_out;
  return normalize(-eta * wi + wm * (eta * ct - ctt));
}
// Dielectric phase eval, GGX :307-339 / Beckmann :341-372.
PT_D float eval_dielectric_phase(uint32_t dist, const float3& wi, const float3& wo, bool wi_out, bool wo_out, float m_eta, float ax, float ay)
{
  float eta = wi_out ? m_eta : 1.0f / m_eta;
  if (wi_out == wo_out) {
    float3 wh = normalize(wi + wo);
    float D = wi_out ? eval_vndf(dist, wi, wh, ax, ay) : eval_vndf(dist, -wi, -wh, ax, ay);
    float F = wi_out ? fresnel_R(wi, wh, eta) : fresnel_R(-wi, -wh, eta);
    float a = wi_out ? 0.25f / dot(wi, wh) : 0.25f / dot(-wi, -wh);
    return F * D * a;
  }
  float3 wh = -normalize(wi + wo / eta);
  float sg = wi_out ? wh.z / fabsf(wh.z) : -wh.z / fabsf(wh.z);
  wh = wh * sg;
  if (dot(wh, wi) < 0.0f) return 0.0f;
  float D = wi_out ? eval_vndf(dist, wi, wh, ax, ay) : eval_vndf(dist, -wi, -wh, ax, ay);
  float F = wi_out ? fresnel_R(wi, wh, eta) : fresnel_R(-wi, -wh, eta);
  float b = 1.0f / (eta * eta);
  float c = wi_out ? fmaxf(0.0f, -dot(wo, wh)) : fmaxf(0.0f, -dot(-wo, -wh));
  float e = wi_out ? dot(wi, wh) + dot(wo, wh) / eta : dot(-wi, -wh) + dot(-wo, -wh) / eta;
  float d = e * e;
  float a = b * c / d;
  return a * D * (1.0f - F);
}
// Conductor phase sample / eval, GGX :390-409 / Beckmann :423-442.
PT_D float3 sample_conductor_phase(uint32_t dist, const float3& wi, float3& wm, uint32_t& seed, float ax, float ay, int* capped)
{
  float z1 = rnd_tea(seed), z2 = rnd_tea(seed);
  wm = sample_vndf(dist, wi, ax, ay, z1, z2, capped);
  return -wi + 2.0f * wm * dot(wi, wm);
}
PT_D float eval_conductor_phase(uint32_t dist, const float3& wi, const float3& wo, float3& wm, float ax, float ay)
{
  wm = normalize(wi + wo);
  if (wm.z < 0.0f) return 0.0f;
  return 0.25f * eval_vndf(dist, wi, wm, ax, ay);
}
// Diffuse phase sample / eval, GGX :342-387 / Beckmann :375-420.
PT_D float3 sample_diffuse_phase(uint32_t dist, const float3& wi, float3& wm, uint32_t& seed, float ax, float ay, int* capped)
{
  float z1 = rnd_tea(seed), z2 = rnd_tea(seed), z3 = rnd_tea(seed), z4 = rnd_tea(seed);
  wm = sample_vndf(dist, wi, ax, ay, z1, z2, capped);
  float3 w1, w2;
  create_onb(wm, w1, w2);
  float r1 = 2.0f * z3 - 1.0f, r2 = 2.0f * z4 - 1.0f;
  float phi, r;
  if (r1 == 0 && r2 == 0) { r = phi = 0.0f; }
  else if (r1 * r1 > r2 * r2) { r = r1; phi = (kPi / 4.0f) * (r2 / r1); }
  else { r = r2; phi = (kPi / 2.0f) - (r1 / r2) * (kPi / 4.0f); }
  float x = r * cosf(phi), y = r * sinf(phi);
  float z = sqrtf(fmaxf(0.0f, 1.0f - x * x - y * y));
  return x * w1 + y * w2 + z * wm;
}
PT_D float eval_diffuse_phase(uint32_t dist, const float3& wi, const float3& wo, float3& wm, float ax, float ay, uint32_t& seed, int* capped)
{
  float z1 = rnd_tea(seed), z2 = rnd_tea(seed);
  wm = sample_vndf(dist, wi, ax, ay, z1, z2, capped);
  if (dist == GGX) return 1.0f / kPi * fmaxf(0.0f, dot(wo, wm));
  return 1.0f * kInvPi * fmaxf(0.0f, dot(wo, wm));
}

// Multiscattering dielectric sample in the local frame, GGX :412-442 / Beckmann :445-476.
PT_D float3 ms_dielectric_sample(uint32_t dist, const float3& lwi, float eta, float ax, float ay, uint32_t& seed, uint32_t& order, int* capped)
{
  float hr = 1.0f + gauss_inv_cdf(0.9999f);
  float3 wo = -lwi, wm;
  bool out = (-wo.z) > 0;
  for (int it = 0;; ++it) {
    if (it >= kWalkCap) { *capped = 1; break; }
    float z = rnd_tea(seed);
    hr = out ? sample_height(dist, wo, hr, z, ax, ay) : -sample_height(dist, -wo, -hr, z, ax, ay);
    if (hr == kDefaultMax || hr == -kDefaultMax) break;
    order++;
    bool wi_out = out;
    wo = sample_dielectric_phase(dist, -wo, wm, eta, seed, wi_out, out, ax, ay, capped);
    if (hr != hr || wo.z != wo.z) { wo = f3(0.0f, 0.0f, 1.0f); break; }
  }
  return wo;
}
// Multiscattering dielectric eval in the local frame: GGX :445-481 (orders < N, all summed);
// Beckmann :479-527 (orders <= N, only the matching order and finite terms summed).
PT_D float ms_dielectric_eval(uint32_t dist, const float3& wi, const float3& wo, float eta, float ax, float ay, uint32_t& seed,
                              uint32_t order, int* capped)
{
  float3 wr = -wi, wm;
  float hr = 1.0f + gauss_inv_cdf(0.9999f);
  int cur = 0;
  float sum = 0.0f;
  bool wr_out = (-wr.z > 0);
  bool wo_out = wo.z > 0;
  for (int it = 0;; ++it) {
    if (dist == GGX) { if (!(order == 0 || cur < (int)order)) break; }
    else { if (!(order == 0 || (uint32_t)cur <= order)) break; }
    if (it >= kWalkCap) { *capped = 1; break; }
    float z = rnd_tea(seed);
    hr = wr_out ? sample_height(dist, wr, hr, z, ax, ay) : -sample_height(dist, -wr, -hr, z, ax, ay);
    if (hr == kDefaultMax || hr == -kDefaultMax || isinf(hr)) break;
    cur++;
    float phase = eval_dielectric_phase(dist, -wr, wo, wr_out, wo_out, eta, ax, ay);
    float shadow = wo_out ? G_height(dist, wo, hr, ax, ay) : G_height(dist, -wo, -hr, ax, ay);
    float I = phase * shadow;
    if (dist == GGX) sum += I;
    else if (isfinite(I) && (order == 0 || (uint32_t)cur == order)) sum += I;
    bool wi_out = wr_out;
    wr = sample_dielectric_phase(dist, -wr, wm, eta, seed, wi_out, wr_out, ax, ay, capped);
    if (hr != hr || wr.z != wr.z) { sum = 0.0f; break; }
  }
  return sum;
}
// Multiscattering conductor sample in the local frame, GGX :614-640 / Beckmann :711-736.
PT_D float3 ms_conductor_sample(uint32_t dist, const float3& wi, const Cx3& eta, const Cx3& inv_eta, float ax, float ay, uint32_t& seed,
                                uint32_t& order, float3& weight, int* capped)
{
  float hr = 1.0f + gauss_inv_cdf(0.9999f);
  float3 wo = -wi, wm;
  weight = f3s(1.0f);
  for (int it = 0;; ++it) {
    if (it >= kWalkCap) { *capped = 1; break; }
    float u = rnd_tea(seed);
    hr = sample_height(dist, wo, hr, u, ax, ay);
    if (hr == kDefaultMax) break;
    order++;
    float3 wt = -wo;
    wo = sample_conductor_phase(dist, -wo, wm, seed, ax, ay, capped);
    weight = weight * fresnel_complex(wt, wm, (wt.z > 0) ? eta : inv_eta);
    if (hr != hr || wo.z != wo.z) { wo = f3(0.0f, 0.0f, 1.0f); break; }
  }
  return wo;
}
// Multiscattering conductor eval in the local frame, GGX :580-611 / Beckmann :677-708.
PT_D float3 ms_conductor_eval(uint32_t dist, const float3& wi, const float3& wo, const Cx3& eta, const Cx3& inv_eta, float ax, float ay,
                              uint32_t& seed, uint32_t order, int* capped)
{
  float3 wr = -wi, wm, sum = f3s(0.0f);
  float hr = 1.0f + gauss_inv_cdf(0.9999f);
  int cur = 0;
  for (int it = 0; order == 0 || cur < (int)order; ++it) {
    if (it >= kWalkCap) { *capped = 1; break; }
    float u = rnd_tea(seed);
    hr = sample_height(dist, wr, hr, u, ax, ay);
    if (hr == kDefaultMax) break;
    cur++;
    float phase = eval_conductor_phase(dist, -wr, wo, wm, ax, ay);
    float shadow = G_height(dist, wo, hr, ax, ay);
    float3 I = fresnel_complex(-wr, wm, (-wr.z > 0) ? eta : inv_eta) * phase * shadow;
    if (finite3(I)) sum = sum + I;
    wr = sample_conductor_phase(dist, -wr, wm, seed, ax, ay, capped);
    if (hr != hr || wr.z != wr.z) { sum = f3s(0.0f); break; }
  }
  return sum;
}
// Multiscattering diffuse sample / eval in the local frame, GGX :519-577 / Beckmann :613-674.
// wm receives the microfacet normal of the walk's last scattering event (the reference's w_m output,
// which rough_diffuse_shader.cu:196 reads); it stays +z if the walk never scatters.
PT_D float3 ms_diffuse_sample(uint32_t dist, const float3& wi, float ax, float ay, uint32_t& seed, uint32_t& order, float3& weight,
                              const float3& rho, float3& wm, int* capped)
{
  weight = f3s(1.0f);
  float hr = 1.0f + gauss_inv_cdf(0.9999f);
  float3 wo = -wi;
  wm = f3(0.0f, 0.0f, 1.0f);
  while (order < 100u) {
    float u = rnd_tea(seed);
    hr = sample_height(dist, wo, hr, u, ax, ay);
    if (hr == kDefaultMax) break;
    order++;
    weight = weight * rho;
    wo = sample_diffuse_phase(dist, -wo, wm, seed, ax, ay, capped);
    if (hr != hr || wo.z != wo.z) { wo = f3(0.0f, 0.0f, 1.0f); break; }
  }
  return wo;
}
PT_D float3 ms_diffuse_eval(uint32_t dist, const float3& wi, const float3& wo, float ax, float ay, uint32_t& seed, const float3& rho,
                            uint32_t order, int* capped)
{
  float3 wr = -wi, wm, sum = f3s(0.0f);
  float hr = 1.0f + gauss_inv_cdf(0.9999f);
  int cur = 0;
  for (int it = 0; order == 0 || cur < (int)order; ++it) {
    if (it >= kWalkCap) { *capped = 1; break; }
    float u = rnd_tea(seed);
    hr = sample_height(dist, wr, hr, u, ax, ay);
    if (hr == kDefaultMax) break;
    cur++;
    float phase = eval_diffuse_phase(dist, -wr, wo, wm, ax, ay, seed, capped);
    float shadow = G_height(dist, wo, hr, ax, ay);
    float3 I = rho * phase * shadow;
    if (finite3(I)) sum = sum + I;
    wr = sample_diffuse_phase(dist, -wr, wm, seed, ax, ay, capped);
    if (hr != hr || wr.z != wr.z) { sum = f3s(0.0f); break; }
  }
  return sum;
}

}  // namespace pt
