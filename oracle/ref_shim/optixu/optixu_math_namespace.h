// Test infrastructure (oracle only): a host-side stand-in for the OptiX 5.1 vector-math header
// that the reference's device math headers include.  It is NOT OptiX code: every definition
// below is written from the mathematics, and it exists so that the reference's own
// Microfacet*/Fresnel/MyComplex/helpers/sampler/random/md5/LightSampler/Envmap/dipole headers
// compile unmodified with g++ on the host.  Nothing in the product links against it.
//
// Conventions fixed here (and mirrored bit-for-bit by the CUDA kernels and by the oracle
// restatement, so all three agree on them):
//   normalize(v) = v * (1.0f / sqrtf(dot(v, v)))
//   dot(a, b)    = a.x*b.x + a.y*b.y + a.z*b.z     (left to right, no fused multiply-add)
//   cross(a, b)  = (a.y*b.z - a.z*b.y, a.z*b.x - a.x*b.z, a.x*b.y - a.y*b.x)
//   reflect(i,n) = i - 2.0f*n*dot(n, i)
//   faceforward(n, i, nref) = n * copysignf(1.0f, dot(i, nref))
//   RT_DEFAULT_MAX = 1.e27f
// Scalar math: the C++ float overloads of sqrt/exp/log/erf/pow/abs... are brought into the
// global namespace, which is what CUDA does for device code, so `erf(float)` means erff and
// `abs(float)` means fabsf exactly as in the reference's GPU build.
#pragma once

#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstddef>
#include <cstdint>

using std::sqrt; using std::exp; using std::log; using std::erf; using std::pow; using std::abs;
using std::sin; using std::cos; using std::tan; using std::atan; using std::atan2; using std::acos;
using std::isfinite; using std::isinf; using std::isnan; using std::floor; using std::ceil;
using std::fabs;

#ifndef __host__
#define __host__
#endif
#ifndef __device__
#define __device__
#endif
#ifndef __inline__
#define __inline__ inline
#endif
#ifndef __forceinline__
#define __forceinline__ inline
#endif
#define RT_HOSTDEVICE
#define RT_PROGRAM
#define RT_DEFAULT_MAX 1.e27f

typedef unsigned int uint;

// Mathematical constants rounded to float (glibc defines some of the same names).
#undef M_Ef
#define M_Ef        2.71828182845904523536f
#undef M_LOG2Ef
#define M_LOG2Ef    1.44269504088896340736f
#undef M_LOG10Ef
#define M_LOG10Ef   0.434294481903251827651f
#undef M_LN2f
#define M_LN2f      0.693147180559945309417f
#undef M_LN10f
#define M_LN10f     2.30258509299404568402f
#undef M_PIf
#define M_PIf       3.14159265358979323846f
#undef M_PI_2f
#define M_PI_2f     1.57079632679489661923f
#undef M_PI_4f
#define M_PI_4f     0.785398163397448309616f
#undef M_1_PIf
#define M_1_PIf     0.318309886183790671538f
#undef M_2_PIf
#define M_2_PIf     0.636619772367581343076f
#undef M_2_SQRTPIf
#define M_2_SQRTPIf 1.12837916709551257390f
#undef M_SQRT2f
#define M_SQRT2f    1.41421356237309504880f
#undef M_SQRT1_2f
#define M_SQRT1_2f  0.707106781186547524401f
#undef M_4PIf
#define M_4PIf      12.5663706143591729538f

struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct float4 { float x, y, z, w; };
struct int2 { int x, y; };
struct int3 { int x, y, z; };
struct int4 { int x, y, z, w; };
struct uint2 { unsigned int x, y; };
struct uint3 { unsigned int x, y, z; };
struct uint4 { unsigned int x, y, z, w; };
struct uchar4 { unsigned char x, y, z, w; };
struct size_t2 { size_t x, y; };

// CUDA-style scalar min/max for float (fminf/fmaxf semantics).
static inline float max(float a, float b) { return fmaxf(a, b); }
static inline float min(float a, float b) { return fminf(a, b); }
static inline int max(int a, int b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline unsigned int max(unsigned int a, unsigned int b) { return a > b ? a : b; }
static inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }

static inline float2 make_float2(float x, float y) { float2 r = {x, y}; return r; }
static inline float2 make_float2(float s) { return make_float2(s, s); }
static inline float2 make_float2(const uint2& u) { return make_float2((float)u.x, (float)u.y); }
static inline float3 make_float3(float x, float y, float z) { float3 r = {x, y, z}; return r; }
static inline float3 make_float3(float s) { return make_float3(s, s, s); }
static inline float3 make_float3(const float4& v) { return make_float3(v.x, v.y, v.z); }
static inline float3 make_float3(const float2& v) { return make_float3(v.x, v.y, 0.0f); }
static inline float4 make_float4(float x, float y, float z, float w) { float4 r = {x, y, z, w}; return r; }
static inline float4 make_float4(float s) { return make_float4(s, s, s, s); }
static inline float4 make_float4(const float3& v, float w) { return make_float4(v.x, v.y, v.z, w); }
static inline int2 make_int2(int x, int y) { int2 r = {x, y}; return r; }
static inline int3 make_int3(int x, int y, int z) { int3 r = {x, y, z}; return r; }
static inline int4 make_int4(int x, int y, int z, int w) { int4 r = {x, y, z, w}; return r; }
static inline uint2 make_uint2(unsigned int x, unsigned int y) { uint2 r = {x, y}; return r; }
static inline uint3 make_uint3(unsigned int x, unsigned int y, unsigned int z) { uint3 r = {x, y, z}; return r; }
static inline uint4 make_uint4(unsigned int x, unsigned int y, unsigned int z, unsigned int w) { uint4 r = {x, y, z, w}; return r; }
static inline uchar4 make_uchar4(unsigned char x, unsigned char y, unsigned char z, unsigned char w) { uchar4 r = {x, y, z, w}; return r; }

// float2
static inline float2 operator-(const float2& a) { return make_float2(-a.x, -a.y); }
static inline float2 operator+(const float2& a, const float2& b) { return make_float2(a.x + b.x, a.y + b.y); }
static inline float2 operator-(const float2& a, const float2& b) { return make_float2(a.x - b.x, a.y - b.y); }
static inline float2 operator*(const float2& a, const float2& b) { return make_float2(a.x * b.x, a.y * b.y); }
static inline float2 operator/(const float2& a, const float2& b) { return make_float2(a.x / b.x, a.y / b.y); }
static inline float2 operator+(const float2& a, float s) { return make_float2(a.x + s, a.y + s); }
static inline float2 operator-(const float2& a, float s) { return make_float2(a.x - s, a.y - s); }
static inline float2 operator*(const float2& a, float s) { return make_float2(a.x * s, a.y * s); }
static inline float2 operator*(float s, const float2& a) { return make_float2(a.x * s, a.y * s); }
static inline float2 operator/(const float2& a, float s) { return make_float2(a.x / s, a.y / s); }

// float3
static inline float3 operator-(const float3& a) { return make_float3(-a.x, -a.y, -a.z); }
static inline float3 operator+(const float3& a, const float3& b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline float3 operator-(const float3& a, const float3& b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline float3 operator*(const float3& a, const float3& b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline float3 operator/(const float3& a, const float3& b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline float3 operator+(const float3& a, float s) { return make_float3(a.x + s, a.y + s, a.z + s); }
static inline float3 operator+(float s, const float3& a) { return make_float3(s + a.x, s + a.y, s + a.z); }
static inline float3 operator-(const float3& a, float s) { return make_float3(a.x - s, a.y - s, a.z - s); }
static inline float3 operator-(float s, const float3& a) { return make_float3(s - a.x, s - a.y, s - a.z); }
static inline float3 operator*(const float3& a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
static inline float3 operator*(float s, const float3& a) { return make_float3(s * a.x, s * a.y, s * a.z); }
static inline float3 operator/(const float3& a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
static inline float3 operator/(float s, const float3& a) { return make_float3(s / a.x, s / a.y, s / a.z); }
static inline void operator+=(float3& a, const float3& b) { a.x += b.x; a.y += b.y; a.z += b.z; }
static inline void operator-=(float3& a, const float3& b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; }
static inline void operator*=(float3& a, const float3& b) { a.x *= b.x; a.y *= b.y; a.z *= b.z; }
static inline void operator/=(float3& a, const float3& b) { a.x /= b.x; a.y /= b.y; a.z /= b.z; }
static inline void operator*=(float3& a, float s) { a.x *= s; a.y *= s; a.z *= s; }
static inline void operator/=(float3& a, float s) { a.x /= s; a.y /= s; a.z /= s; }

// float4
static inline float4 operator+(const float4& a, const float4& b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static inline float4 operator*(const float4& a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
static inline float4 operator/(const float4& a, float s) { return make_float4(a.x / s, a.y / s, a.z / s, a.w / s); }

static inline bool operator==(const uint2& a, const uint2& b) { return a.x == b.x && a.y == b.y; }
static inline uint2 operator-(const uint2& a, unsigned int s) { return make_uint2(a.x - s, a.y - s); }

static inline float dot(const float2& a, const float2& b) { return a.x * b.x + a.y * b.y; }
static inline float dot(const float3& a, const float3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float length(const float3& v) { return sqrtf(dot(v, v)); }
static inline float3 normalize(const float3& v) { float inv_len = 1.0f / sqrtf(dot(v, v)); return v * inv_len; }
static inline float2 normalize(const float2& v) { float inv_len = 1.0f / sqrtf(dot(v, v)); return v * inv_len; }
static inline float3 cross(const float3& a, const float3& b)
{
  return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float3 reflect(const float3& i, const float3& n) { return i - 2.0f * n * dot(n, i); }
static inline float3 faceforward(const float3& n, const float3& i, const float3& nref)
{
  return n * copysignf(1.0f, dot(i, nref));
}
static inline float3 fminf(const float3& a, const float3& b) { return make_float3(::fminf(a.x, b.x), ::fminf(a.y, b.y), ::fminf(a.z, b.z)); }
static inline float3 fmaxf(const float3& a, const float3& b) { return make_float3(::fmaxf(a.x, b.x), ::fmaxf(a.y, b.y), ::fmaxf(a.z, b.z)); }
static inline float3 expf(const float3& v) { return make_float3(::expf(v.x), ::expf(v.y), ::expf(v.z)); }
static inline float clamp(float f, float a, float b) { return fmaxf(a, fminf(f, b)); }
static inline float lerp(float a, float b, float t) { return a + t * (b - a); }

// 3x3 matrix used only as a default argument (identity rotation) in Envmap.h.
struct Matrix3x3Shim {
  float m[9];
  static Matrix3x3Shim identity() { Matrix3x3Shim r = {{1, 0, 0, 0, 1, 0, 0, 0, 1}}; return r; }
};
static inline float3 operator*(const Matrix3x3Shim& M, const float3& v)
{
  return make_float3(M.m[0] * v.x + M.m[1] * v.y + M.m[2] * v.z,
                     M.m[3] * v.x + M.m[4] * v.y + M.m[5] * v.z,
                     M.m[6] * v.x + M.m[7] * v.y + M.m[8] * v.z);
}

// Buffer stand-in: indexes host memory owned by the oracle driver.  Out-of-range reads are
// clamped to the last element and counted, so the reference's unguarded indexing (for example
// a light index computed from a random number equal to 1.0) cannot read outside the array.
extern unsigned long long g_shim_oob_reads;
template <typename T, int Dim = 1>
struct rtBufferShim;
template <typename T>
struct rtBufferShim<T, 1> {
  T* data = nullptr;
  size_t n = 0;
  size_t size() const { return n; }
  T& operator[](size_t i)
  {
    if (i >= n) { ++g_shim_oob_reads; i = n ? n - 1 : 0; }
    return data[i];
  }
};
template <typename T>
struct rtBufferShim<T, 2> {
  T* data = nullptr;
  size_t nx = 0, ny = 0;
  size_t2 size() const { size_t2 s = {nx, ny}; return s; }
  T& operator[](const uint2& ij)
  {
    size_t i = ij.x, j = ij.y;
    if (i >= nx || j >= ny) { ++g_shim_oob_reads; i = i < nx ? i : nx - 1; j = j < ny ? j : ny - 1; }
    return data[j * nx + i];
  }
};
#define rtBuffer rtBufferShim

// Texture stand-in: float4 texels, normalized coordinates, bilinear filtering, REPEAT wrap
// (the sampler state the reference sets in HDRLoader.cpp loadHDRTexture).  Software FP32
// bilinear weights, identical to the CUDA kernels' env-map lookup.
template <typename T, int Dim>
struct rtTextureSamplerShim {
  const float4* texels = nullptr;
  int w = 0, h = 0;
};
#define rtTextureSampler rtTextureSamplerShim
static inline int shim_wrap(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }
template <typename T>
static inline float4 tex2D(const rtTextureSamplerShim<T, 2>& s, float u, float v)
{
  float x = u * (float)s.w - 0.5f;
  float y = v * (float)s.h - 0.5f;
  float fx = floorf(x), fy = floorf(y);
  float ax = x - fx, ay = y - fy;
  int i0 = shim_wrap((int)fx, s.w), j0 = shim_wrap((int)fy, s.h);
  int i1 = shim_wrap((int)fx + 1, s.w), j1 = shim_wrap((int)fy + 1, s.h);
  const float4& t00 = s.texels[j0 * s.w + i0];
  const float4& t10 = s.texels[j0 * s.w + i1];
  const float4& t01 = s.texels[j1 * s.w + i0];
  const float4& t11 = s.texels[j1 * s.w + i1];
  float w00 = (1.0f - ax) * (1.0f - ay), w10 = ax * (1.0f - ay), w01 = (1.0f - ax) * ay, w11 = ax * ay;
  return make_float4(t00.x * w00 + t10.x * w10 + t01.x * w01 + t11.x * w11,
                     t00.y * w00 + t10.y * w10 + t01.y * w01 + t11.y * w11,
                     t00.z * w00 + t10.z * w10 + t01.z * w01 + t11.z * w11,
                     t00.w * w00 + t10.w * w10 + t01.w * w01 + t11.w * w11);
}

static inline void rtPrintf(const char*, ...) {}

namespace optix {
using ::float2; using ::float3; using ::float4; using ::int2; using ::int3; using ::int4;
using ::uint2; using ::uint3; using ::uint4; using ::uchar4; using ::size_t2;
typedef unsigned int uint;
typedef Matrix3x3Shim Matrix3x3;
using ::make_float2; using ::make_float3; using ::make_float4; using ::make_int2; using ::make_int3;
using ::make_int4; using ::make_uint2; using ::make_uint3; using ::make_uint4; using ::make_uchar4;
using ::dot; using ::length; using ::normalize; using ::cross; using ::reflect; using ::faceforward;
using ::fminf; using ::fmaxf; using ::expf; using ::clamp; using ::lerp;
}  // namespace optix
