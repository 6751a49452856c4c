// Test infrastructure (oracle only): CPU restatement of the reference's hot-path device math,
// templated on the scalar type R.  With R = float it reproduces the reference bit-for-bit when
// both are compiled with g++ -ffp-contract=off (checked against oracle/_ref/libref_oracle.so
// by tests/test_oracle_pin.py); with R = double it is the FP64 oracle used to state each
// kernel's maximum error.  Every function cites the reference file:line it restates; paths are
// relative to open_rendering_framework/.  Where the reference mixes precisions (double literals,
// double complex arithmetic, float casts of erf/erfinv) the float instantiation keeps exactly
// those promotions and the double instantiation computes everything in double.
//
// Vector conventions (normalize = v * (1/sqrt(dot)), dot left to right, reflect, faceforward)
// are the ones fixed by oracle/ref_shim/optixu/optixu_math_namespace.h.
#pragma once
#include <cmath>
#include <cstdint>

namespace orc {

typedef unsigned int u32;

template <class R> struct K;
template <> struct K<float> {
  static constexpr float PI = 3.14159265358979323846f;
  static constexpr float INV_PI = 0.318309886183790671538f;
  static constexpr float TWO_SQRTPI = 1.12837916709551257390f;
  static constexpr float SQRT2 = 1.41421356237309504880f;
  static constexpr float SQRT1_2 = 0.707106781186547524401f;
};
template <> struct K<double> {
  static constexpr double PI = 3.14159265358979323846;
  static constexpr double INV_PI = 0.318309886183790671538;
  static constexpr double TWO_SQRTPI = 1.12837916709551257390;
  static constexpr double SQRT2 = 1.41421356237309504880;
  static constexpr double SQRT1_2 = 0.707106781186547524401;
};
static constexpr float DEFAULT_MAX = 1.e27f;  // RT_DEFAULT_MAX

template <class R> struct V3 { R x, y, z; };
template <class R> static inline V3<R> v3(R x, R y, R z) { V3<R> r = {x, y, z}; return r; }
template <class R> static inline V3<R> v3s(R s) { V3<R> r = {s, s, s}; return r; }
template <class R> static inline V3<R> operator-(const V3<R>& a) { return v3(-a.x, -a.y, -a.z); }
template <class R> static inline V3<R> operator+(const V3<R>& a, const V3<R>& b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class R> static inline V3<R> operator-(const V3<R>& a, const V3<R>& b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class R> static inline V3<R> operator*(const V3<R>& a, const V3<R>& b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
template <class R> static inline V3<R> operator/(const V3<R>& a, const V3<R>& b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
template <class R> static inline V3<R> operator*(const V3<R>& a, R s) { return v3(a.x * s, a.y * s, a.z * s); }
template <class R> static inline V3<R> operator*(R s, const V3<R>& a) { return v3(s * a.x, s * a.y, s * a.z); }
template <class R> static inline V3<R> operator/(const V3<R>& a, R s) { return v3(a.x / s, a.y / s, a.z / s); }
template <class R> static inline V3<R> operator/(R s, const V3<R>& a) { return v3(s / a.x, s / a.y, s / a.z); }
template <class R> static inline V3<R> operator+(const V3<R>& a, R s) { return v3(a.x + s, a.y + s, a.z + s); }
template <class R> static inline V3<R> operator+(R s, const V3<R>& a) { return v3(s + a.x, s + a.y, s + a.z); }
template <class R> static inline V3<R> operator-(const V3<R>& a, R s) { return v3(a.x - s, a.y - s, a.z - s); }
template <class R> static inline V3<R> operator-(R s, const V3<R>& a) { return v3(s - a.x, s - a.y, s - a.z); }
template <class R> static inline R dot(const V3<R>& a, const V3<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> static inline R length(const V3<R>& a) { return std::sqrt(dot(a, a)); }
template <class R> static inline V3<R> normalize(const V3<R>& a) { R inv = R(1) / std::sqrt(dot(a, a)); return a * inv; }
template <class R> static inline V3<R> cross(const V3<R>& a, const V3<R>& b)
{
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class R> static inline V3<R> reflect(const V3<R>& i, const V3<R>& n) { return i - R(2) * n * dot(n, i); }
template <class R> static inline V3<R> faceforward(const V3<R>& n, const V3<R>& i, const V3<R>& nref)
{
  return n * std::copysign(R(1), dot(i, nref));
}
template <class R> static inline V3<R> vexp(const V3<R>& a) { return v3(std::exp(a.x), std::exp(a.y), std::exp(a.z)); }
template <class R> static inline V3<R> vsqrt(const V3<R>& a) { return v3(std::sqrt(a.x), std::sqrt(a.y), std::sqrt(a.z)); }
template <class R> static inline V3<R> vmax(const V3<R>& a, const V3<R>& b) { return v3(std::fmax(a.x, b.x), std::fmax(a.y, b.y), std::fmax(a.z, b.z)); }
template <class To, class From> static inline V3<To> cvt(const V3<From>& a) { return v3((To)a.x, (To)a.y, (To)a.z); }
template <class R> static inline bool finite3(const V3<R>& a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }

// ------------------------------------------------------------------ RNG (random.h, md5.h)
// tea<N>, random.h:25-40.
template <unsigned N>
static inline u32 tea(u32 v0, u32 v1)
{
  u32 s0 = 0;
  for (unsigned n = 0; n < N; n++) {
    s0 += 0x9e3779b9u;
    v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
    v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
  }
  return v0;
}
// lcg / rnd, random.h:43-61.
static inline u32 lcg(u32& prev) { prev = 1664525u * prev + 1013904223u; return prev & 0x00FFFFFFu; }
static inline float rnd(u32& prev) { return (float)lcg(prev) / (float)0x01000000; }
// tea_hash / rnd_tea, random.h:117-127.  Returns float for every R (the draw is an FP32 value
// in the reference; the FP64 oracle consumes the same draws).
static inline float rnd_tea(u32& prev) { prev = tea<16>(prev, 100u); return (float)(prev & 0x7FFFFFFFu) / (float)0x80000000u; }

// MD5 of an 8-byte message (md5.h:58-200 for length 8, rand_md5(uint2) :218-225).  RFC 1321
// round constants and shifts; the padded block is (x, y, 0x80, 0..., bitlen=64, 0).
static inline u32 rotl(u32 x, int n) { return (x << n) | (x >> (32 - n)); }
static inline void md5_u2(u32 x, u32 y, u32 out[4])
{
  static const u32 T[64] = {
      0xd76aa478u, 0xe8c7b756u, 0x242070dbu, 0xc1bdceeeu, 0xf57c0fafu, 0x4787c62au, 0xa8304613u, 0xfd469501u,
      0x698098d8u, 0x8b44f7afu, 0xffff5bb1u, 0x895cd7beu, 0x6b901122u, 0xfd987193u, 0xa679438eu, 0x49b40821u,
      0xf61e2562u, 0xc040b340u, 0x265e5a51u, 0xe9b6c7aau, 0xd62f105du, 0x02441453u, 0xd8a1e681u, 0xe7d3fbc8u,
      0x21e1cde6u, 0xc33707d6u, 0xf4d50d87u, 0x455a14edu, 0xa9e3e905u, 0xfcefa3f8u, 0x676f02d9u, 0x8d2a4c8au,
      0xfffa3942u, 0x8771f681u, 0x6d9d6122u, 0xfde5380cu, 0xa4beea44u, 0x4bdecfa9u, 0xf6bb4b60u, 0xbebfbc70u,
      0x289b7ec6u, 0xeaa127fau, 0xd4ef3085u, 0x04881d05u, 0xd9d4d039u, 0xe6db99e5u, 0x1fa27cf8u, 0xc4ac5665u,
      0xf4292244u, 0x432aff97u, 0xab9423a7u, 0xfc93a039u, 0x655b59c3u, 0x8f0ccc92u, 0xffeff47du, 0x85845dd1u,
      0x6fa87e4fu, 0xfe2ce6e0u, 0xa3014314u, 0x4e0811a1u, 0xf7537e82u, 0xbd3af235u, 0x2ad7d2bbu, 0xeb86d391u};
  static const int S[64] = {7, 12, 17, 22, 7, 12, 17, 22, 7, 12, 17, 22, 7, 12, 17, 22,
                            5, 9,  14, 20, 5, 9,  14, 20, 5, 9,  14, 20, 5, 9,  14, 20,
                            4, 11, 16, 23, 4, 11, 16, 23, 4, 11, 16, 23, 4, 11, 16, 23,
                            6, 10, 15, 21, 6, 10, 15, 21, 6, 10, 15, 21, 6, 10, 15, 21};
  u32 M[16] = {x, y, 0x80u, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 64u, 0};
  u32 a = 0x67452301u, b = 0xefcdab89u, c = 0x98badcfeu, d = 0x10325476u;
  for (int i = 0; i < 64; ++i) {
    u32 f;
    int g;
    if (i < 16) { f = (b & c) | (~b & d); g = i; }
    else if (i < 32) { f = (b & d) | (c & ~d); g = (5 * i + 1) & 15; }
    else if (i < 48) { f = b ^ c ^ d; g = (3 * i + 5) & 15; }
    else { f = c ^ (b | ~d); g = (7 * i) & 15; }
    u32 t = d;
    d = c;
    c = b;
    b = b + rotl(a + f + M[g] + T[i], S[i]);
    a = t;
  }
  out[0] = a + 0x67452301u; out[1] = b + 0xefcdab89u; out[2] = c + 0x98badcfeu; out[3] = d + 0x10325476u;
}
struct Seed64 { u32 x, y; };
// rnd_accurate, random.h:134-142: next = md5(seed) low two words; value = (63-bit) / 2^63.
static inline float rnd_accurate(Seed64& s)
{
  u32 h[4];
  md5_u2(s.x, s.y, h);
  s.x = h[0];
  s.y = h[1];
  unsigned long long l = (((unsigned long long)s.y << 32) | s.x) & 0x7FFFFFFFFFFFFFFFull;
  double val = (double)l / (double)0x8000000000000000ull;
  return (float)val;
}

// ------------------------------------------------------------------ helpers.h
// create_onb(n, U, V) for a normalized n, helpers.h:92-103.
template <class R> static inline void create_onb(const V3<R>& n, V3<R>& U, V3<R>& V)
{
  U = cross(n, v3(R(0), R(1), R(0)));
  if (dot(U, U) < R(1e-3f)) U = cross(n, v3(R(1), R(0), R(0)));
  U = normalize(U);
  V = cross(n, U);
}
// helpers.h:284-291
template <class R> static inline V3<R> to_local(const V3<R>& w, const V3<R>& n)
{
  V3<R> u, v;
  create_onb(n, u, v);
  return normalize(v3(dot(w, u), dot(w, v), dot(w, n)));
}
// helpers.h:294-299
template <class R> static inline V3<R> to_world(const V3<R>& w, const V3<R>& n)
{
  V3<R> u, v;
  create_onb(n, u, v);
  return normalize(u * w.x + v * w.y + n * w.z);
}
// Double-precision erfinv of helpers.h:301-377 (M. Giles, "Approximating the erfinv function",
// GPU Computing Gems Jade Edition, 2011: three polynomial branches in w = -log((1-x)(1+x))).
static inline double erfinv_d(double x)
{
  double w = -std::log((1.0 - x) * (1.0 + x)), p;
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
    w = std::sqrt(w) - 3.25;
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
    w = std::sqrt(w) - 5.0;
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
// helpers.h:380-383 and :386-389
template <class R> static inline R gauss_inv_cdf(R z) { return K<R>::SQRT2 * (R)erfinv_d(R(2) * z - R(1)); }
template <class R> static inline R gauss_cdf(R h) { return R(0.5f) + R(0.5f) * (R)std::erf(K<R>::SQRT1_2 * h); }

// ------------------------------------------------------------------ sampler.h
template <class R> static inline void rotate_to_normal(const V3<R>& n, V3<R>& v)  // :12-24
{
  if (n.z < R(-0.999999f)) { v = v3(-v.y, -v.x, -v.z); return; }
  R a = R(1) / (R(1) + n.z);
  R b = -n.x * n.y * a;
  v = v3(R(1) - n.x * n.x * a, b, -n.x) * v.x + v3(b, R(1) - n.y * n.y * a, -n.y) * v.y + n * v.z;
}
static inline void sincos_r(float a, float* s, float* c) { ::sincosf(a, s, c); }
static inline void sincos_r(double a, double* s, double* c) { ::sincos(a, s, c); }
template <class R> static inline V3<R> spherical_direction(R sin_t, R cos_t, R phi)  // :29-34
{
  R sp, cp;
  sincos_r(phi, &sp, &cp);
  return v3(sin_t * cp, sin_t * sp, cos_t);
}
template <class R> static inline V3<R> sample_cosine_weighted(const V3<R>& n, u32& t)  // :51-64
{
  R cos_t = std::sqrt((R)rnd_tea(t));
  R phi = R(2) * K<R>::PI * (R)rnd_tea(t);
  R sin_t = std::sqrt(R(1) - cos_t * cos_t);
  V3<R> v = spherical_direction(sin_t, cos_t, phi);
  rotate_to_normal(n, v);
  return v;
}
template <class R> static inline V3<R> sample_barycentric(u32& t)  // :103-116
{
  R sx = std::sqrt((R)rnd_tea(t));
  R xi2 = (R)rnd_tea(t);
  return v3(R(1) - sx, (R(1) - xi2) * sx, xi2 * sx);
}

// ------------------------------------------------------------------ Fresnel.h
template <class R> static inline R fresnel_rs(R c1, R c2, R e) { return (e * c1 - c2) / (e * c1 + c2); }  // :14-18
template <class R> static inline R fresnel_rp(R c1, R c2, R e) { return (c1 - e * c2) / (c1 + e * c2); }  // :20-24
template <class R> static inline R fresnel_R(R c1, R c2, R e)  // :26-32
{
  R rs = fresnel_rs(c1, c2, e), rp = fresnel_rp(c1, c2, e);
  return (rs * rs + rp * rp) * R(0.5f);
}
template <class R> static inline R fresnel_R(const V3<R>& wi, const V3<R>& wm, R e)  // :42-54
{
  R c1 = dot(wi, wm);
  R c22 = R(1) - e * e * (R(1) - c1 * c1);
  if (c22 <= R(0)) return R(1);
  R c2 = std::sqrt(c22);
  R rs = fresnel_rs(c1, c2, e), rp = fresnel_rp(c1, c2, e);
  return (rs * rs + rp * rp) * R(0.5f);
}
template <class R> static inline R two_C1(R n)  // :93-101
{
  if (n >= R(1))
    return R(-9.23372f) + n * (R(22.2272f) + n * (R(-20.9292f) + n * (R(10.2291f) + n * (R(-2.54396f) + n * R(0.254913f)))));
  return R(0.919317f) + n * (R(-3.4793f) + n * (R(6.75335f) + n * (R(-7.80989f) + n * (R(4.98554f) - n * R(1.36881f)))));
}
template <class R> static inline R three_C2(R n)  // :103-114
{
  R r;
  if (n >= R(1)) {
    r = R(-1641.1f) + n * (R(1213.67f) + n * (R(-568.556f) + n * (R(164.798f) + n * (R(-27.0181f) + n * R(1.91826f)))));
    r += (((R(135.926f) / n) - R(656.175f)) / n + R(1376.53f)) / n;
  } else
    r = R(0.828421f) + n * (R(-2.62051f) + n * (R(3.36231f) + n * (R(-1.95284f) + n * (R(0.236494f) + n * R(0.145787f)))));
  return r;
}
template <class R> static inline R C_phi(R n) { return R(0.25f) * (R(1) - two_C1(n)); }  // :116-119
template <class R> static inline R C_E(R n) { return R(0.5f) * (R(1) - three_C2(n)); }    // :121-124

// ------------------------------------------------------------------ MyComplex.h (double members)
struct Cx { double re, im; };
struct Cx3 { Cx x, y, z; };
template <class R> static inline R cabs(const Cx& c) { R r = (R)c.re, i = (R)c.im; return std::sqrt(r * r + i * i); }  // :18-23
static inline Cx cconj(const Cx& c) { Cx r = {c.re, -c.im}; return r; }
static inline Cx cmul(const Cx& a, const Cx& b) { Cx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }  // :98-104
static inline Cx cmuls(const Cx& a, double s) { Cx r = {a.re * s, a.im * s}; return r; }
template <class R> static inline Cx cdiv(const Cx& a, const Cx& b)  // :148-153
{
  Cx num = cmul(a, cconj(b));
  double den = (double)std::pow(cabs<R>(b), R(2));
  return cmuls(num, 1.0 / den);
}
template <class R> static inline Cx cdiv_s(R a, const Cx& b)  // :155-160 (float numerator)
{
  Cx num = {(double)a * b.re, (double)a * -b.im};
  double den = (double)std::pow(cabs<R>(b), R(2));
  return cmuls(num, 1.0 / den);
}
template <class R> static inline R cphase(const Cx& c)  // :169-185
{
  double r = c.re, i = c.im, th;
  if (r == 0 && i > 0) th = (double)(K<R>::PI / R(2));
  else if (r == 0 && i < 0) th = (double)(-K<R>::PI / R(2));
  else if (r == 0 && i == 0) th = 0;
  else th = std::atan(i / r);
  if (r < 0) th += (double)K<R>::PI;
  return (R)th;
}
template <class R> static inline Cx cpow_int(const Cx& c, int e)  // :187-193
{
  double ab = std::pow((double)cabs<R>(c), (double)e);
  double th = (double)(cphase<R>(c) * (R)e);
  Cx r = {ab * std::cos(th), ab * std::sin(th)};
  return r;
}
template <class R> static inline Cx csqrt(const Cx& c)  // :195-202
{
  double ab = (double)std::sqrt(cabs<R>(c));
  double th = (double)(cphase<R>(c) / R(2));
  Cx r = {ab * std::cos(th), ab * std::sin(th)};
  return r;
}
template <class R> static inline Cx3 crecip3(const Cx3& ior)  // 1.0f / MyComplex3, :352-356 with :155-160
{
  Cx3 r = {cdiv_s<R>(R(1), ior.x), cdiv_s<R>(R(1), ior.y), cdiv_s<R>(R(1), ior.z)};
  return r;
}
// fresnel_MyComplex_R for one channel, Fresnel.h:78-91.
template <class R> static inline R fresnel_complex1(R cos_i, R sin_i, const Cx& e)
{
  Cx st = {e.re * (double)sin_i, e.im * (double)sin_i};                    // MyComplex * float
  Cx p2 = cpow_int<R>(st, 2);
  Cx one_m = {(double)R(1) - p2.re, -p2.im};                                  // float - MyComplex
  Cx ct = csqrt<R>(one_m);
  Cx ec = {e.re * (double)cos_i, e.im * (double)cos_i};
  Cx n1 = {ec.re - ct.re, ec.im - ct.im}, d1 = {ec.re + ct.re, ec.im + ct.im};
  Cx r_ort = cdiv<R>(n1, d1);
  Cx ect = cmul(e, ct);
  Cx n2 = {(double)cos_i - ect.re, -ect.im}, d2 = {(double)cos_i + ect.re, ect.im};
  Cx r_par = cdiv<R>(n2, d2);
  R a = cabs<R>(r_ort), b = cabs<R>(r_par);
  return R(0.5f) * (std::pow(a, R(2)) + std::pow(b, R(2)));
}
template <class R> static inline V3<R> fresnel_complex(const V3<R>& wi, const V3<R>& wm, const Cx3& e)
{
  R ci = dot(wi, wm);
  R si = std::sqrt(R(1) - ci * ci);
  return v3(fresnel_complex1<R>(ci, si, e.x), fresnel_complex1<R>(ci, si, e.y), fresnel_complex1<R>(ci, si, e.z));
}

}  // namespace orc
