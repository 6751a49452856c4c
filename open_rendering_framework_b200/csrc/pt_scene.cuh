// Device-side scene layout and the stackless BVH traversal.
//
// HBM layout (all 16-byte aligned, loaded as float4 / int4):
//   nodes    : BVH2 with child-pair nodes, 4 x float4 = 64 B per node
//              n0 = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)   n1 = same for child 1
//              n2 = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)   n3 = (child0, child1, parent, 0) as int
//              child >= 0: internal node index; child < 0: leaf, bits = 0x80000000 | first<<4 | count
//   tri_v0/e1/e2 : Moller-Trumbore triangles in leaf order, 3 x float4 = 48 B per triangle
//              (v0.xyz, original index), (v1-v0, 0), (v2-v0, 0)
//   tri_info : per ORIGINAL triangle, int4 (normal index 0,1,2 or -1, material id)
//   normals  : float4 per shading normal (xyz, 0)
// A radiance or shadow query reads one node (64 B) per visited node, 48 B per tested triangle;
// the BVH of the single-scene configuration (~100k triangles, ~7 MB of nodes and triangles) stays
// resident in the 126 MB L2.
#pragma once
#include <string.h>

#include "pt_math.cuh"

// Loads through the read-only path on the device; plain loads when the traversal is compiled for the
// host (the CPU check of the traversal in tests/ builds it that way).
#ifdef __CUDA_ARCH__
#define PT_LDG(p) __ldg(p)
#else
#define PT_LDG(p) (*(p))
#endif

namespace pt {

PT_HD float as_float(int i)
{
#ifdef __CUDA_ARCH__
  return __int_as_float(i);
#else
  float f;
  memcpy(&f, &i, 4);
  return f;
#endif
}
PT_HD int as_int(float f)
{
#ifdef __CUDA_ARCH__
  return __float_as_int(f);
#else
  int i;
  memcpy(&i, &f, 4);
  return i;
#endif
}

constexpr uint32_t kLeafFlag = 0x80000000u;
constexpr int kMaxDepth = 62;  // depth bound of the build; the traversal trail has 64 bits

enum MatType : uint32_t {
  MAT_DIFFUSE = 0,
  MAT_TRANSPARENT = 2,
  MAT_ROUGH_GLASS = 3,
  MAT_METAL = 4,
  MAT_TRANSLUCENT = 5,
  MAT_ROUGH_TRANSLUCENT = 6,
  MAT_LAMBERTIAN_INTERFACE = 7,
  MAT_ROUGH_DIFFUSE = 9,
  MAT_LIGHT = 100
};
enum DipoleModel : uint32_t { STANDARD_DIPOLE = 0, DIRECTIONAL_DIPOLE = 1 };

// Material record, 16-byte aligned (128 B).
struct __align__(16) MatDev {
  uint32_t type, model, dist, aux;  // translucent: model = dipole_model, aux = translucent_index (rough: dist = normal distribution,
                                    // a = (scale, roughness x, roughness y, microfacet model))
  float4 a;   // diffuse: color.xyz | metal: roughness.xy | glass: ior, roughness | transparent: ior | light: radiance.xyz
              // lambertian interface, rough diffuse: color.xyz, ior
  float4 b;   // glass, transparent: absorption.xyz | lambertian interface: two_C1(ior) | rough diffuse: two_C1(ior), roughness.xy
  Cx3 eta;    // metal: 1 / ior (metallic_shader.cu:61) | rough diffuse: (1 / ior, 0) per channel; computed on the host
  Cx3 inv_eta;// 1 / eta (the walk's inside branch)
  float4 tmap;// texture: cube-map center xyz, texture id in w (int bits, -1 = none)
};

// A float texture (1 or 3 channels), texel (x, y) channel c at data[(y * w + x) * ch + c], and the
// buffer its gradient accumulates into (adjoint renders; may be null).
struct TexDev {
  const float* data;
  float* grad;
  uint32_t w, h, ch, pad;
};

// Nearest texel of a cube map around c, the six faces laid out 3 x 2 in the texture: the largest
// component of p - c picks the face, the other two divided by it give the face coordinates.
// Divisions, comparisons and truncations only, so host and device pick the same texel.
PT_HD uint32_t cube_texel(const float3& p, const float3& c, uint32_t w, uint32_t h)
{
  float3 d = p - c;
  float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  uint32_t face;
  float s, t, m;
  if (ax >= ay && ax >= az) { face = d.x >= 0.0f ? 0u : 1u; m = ax; s = d.z; t = d.y; }
  else if (ay >= az) { face = d.y >= 0.0f ? 2u : 3u; m = ay; s = d.x; t = d.z; }
  else { face = d.z >= 0.0f ? 4u : 5u; m = az; s = d.x; t = d.y; }
  float u = 0.5f, v = 0.5f;
  if (m > 0.0f) {
    u = 0.5f * (s / m + 1.0f);
    v = 0.5f * (t / m + 1.0f);
  }
  const uint32_t fw = w / 3u, fh = h / 2u;
  float fu = u * (float)fw, fv = v * (float)fh;
  uint32_t x = fu > 0.0f ? (uint32_t)fu : 0u, y = fv > 0.0f ? (uint32_t)fv : 0u;
  if (x >= fw) x = fw - 1u;
  if (y >= fh) y = fh - 1u;
  return ((face / 3u) * fh + y) * w + (face % 3u) * fw + x;
}

// ScatteringMaterialProperties, structs.h:116-144 (260 bytes), one per material id (filled for
// translucent materials).
struct ScatDev {
  float relative_ior;
  float3 ior_real, ior_imag, absorption, scattering, meancosine, extinction, reducedExtinction, deltaEddExtinction, D, transport, C_phi,
      C_phi_inv, C_E, A, albedo, reducedAlbedo, de, three_D, two_A_de, global_coeff, one_over_three_ext;
  float mean_transport;
};
static_assert(sizeof(ScatDev) == 260, "ScatteringMaterialProperties layout");

struct LightRaw { uint32_t type; float emitted[3]; float p[3]; float pad[3]; };  // structs.h:42-48 (40 B)
struct TriLightRaw { float v0[3], v1[3], v2[3], n0[3], n1[3], n2[3]; uint32_t has_normals; float emission[3]; float area; };  // :96-103
static_assert(sizeof(LightRaw) == 40, "LightStruct layout");
static_assert(sizeof(TriLightRaw) == 92, "TriangleLight layout");
enum LightType : uint32_t { POINT_LIGHT = 0, DIRECTIONAL_LIGHT = 1, TRIANGLES_AREA_LIGHT = 2, DISK_LIGHT = 3, SPHERICAL_LIGHT = 4,
                            ENVMAP_LIGHT = 5 /* the environment map as a light (sample_environment, Envmap.h:66-98) */ };

// Environment map: float4 texels (row-major, row j = v), bilinear with REPEAT wrap, and the
// marginal / conditional pdf and cdf tables of env_cameras.cu:23-75.
struct EnvDev {
  const float4* tex;
  const float* marginal_pdf;
  const float* marginal_cdf;
  const float* conditional_pdf;
  const float* conditional_cdf;
  int w, h;
  int present;   // EnvMapBackground set: misses return env_lookup(dir)
  int is_light;  // an ENVMAP_LIGHT is in the light buffer: misses after next-event estimation return 0
};

struct CameraDev {
  float3 eye, U, V, W;
  uint32_t width, height;
  uint2 patch_origin, patch_dims;
};
struct IntegratorDev {
  int max_depth;
  float scene_epsilon;
  int rr_start;
  float3 exception_color;
};

struct SceneDev {
  const float4* nodes;
  const float4* nodes4;  // the wide BVH (kWide children per node, kWideStride float4 each) or null
  float trav_scale;      // the diagonal of the triangles' bounding box (sizes the box tests' margin)
  const float4* tri_v0;
  const float4* tri_e1;
  const float4* tri_e2;
  const int4* tri_info;
  const float4* normals;
  const float4* geo;    // per original triangle: cross(v1 - v0, v2 - v0), unnormalised
  const MatDev* mats;
  const ScatDev* scat;  // per material id
  const TexDev* tex;    // textures (diffuse albedo, conductor roughness)
  const LightRaw* lights;
  const TriLightRaw* tri_lights;
  int n_lights, n_tri_lights;
  uint32_t n_tris;
  float3 bg_color;
  EnvDev env;
  CameraDev cam;
  IntegratorDev integ;
  float4* accum;        // the running mean, width * height
  // translucent objects: (material, first triangle, triangle count, offset into trans_pos) and their
  // vertex positions as given (9 floats per triangle)
  const uint4* trans_objs;
  const float* trans_pos;
  uint32_t n_trans, probe_samples;
  // differentiable renders: per camera path of frames [adj_first, adj_first + adj_frames), its radiance
  // (adj_L) and the value of each of its dipole gathers (adj_G, adj_slots per path), written by the
  // forward render and read by the adjoint; the image gradient dLoss/d(running mean) and its factor
  // d(running mean)/d(path radiance); per material, the buffer of 6 floats that the gradient of a
  // translucent material's (sigma_a, sigma_s') per RGB channel accumulates into (or null)
  float4* adj_L;
  float4* adj_G;
  uint32_t adj_first, adj_frames, adj_slots;
  const float4* adj_dimg;
  float adj_dscale;
  float* const* mat_grad;
  // analytic emitters: the disk and sphere geometry that DiskAreaLight and SphericalLight add to the
  // scene (Light.cpp:370-503, 505-610), 3 float4 each (see AnaKind); their hits carry index n_tris + k
  const float4* ana;
  uint32_t n_ana;
};
// The traversal's view of a scene (the four arrays it reads), held in registers by kernels that
// trace rays of several scenes.
struct TravGeom {
  const float4* nodes;
  const float4* tri_v0;
  const float4* tri_e1;
  const float4* tri_e2;
  const float4* nodes4;
  float trav_scale;
};
PT_HD TravGeom trav_geom(const SceneDev& S) { return TravGeom{S.nodes, S.tri_v0, S.tri_e1, S.tri_e2, S.nodes4, S.trav_scale}; }

struct Ray {
  float3 o, d;
  float tmin, tmax;
};
struct Hit {
  float t, u, v;
  int prim;  // original triangle index, -1 = miss
};

// ------------------------------------------------------------------ intersection primitives
// The box tests only prune: the triangle test alone decides hits, so a box must never be culled when
// the triangle test reports a hit inside it.  The triangle test rounds too: a ray aimed at a vertex or an
// edge can be reported to hit a triangle at a point that lies just outside the triangle (a barycentric
// that is slightly negative rounds to 0), i.e. just outside its box, by a distance of the order of the
// float spacing of the coordinates and of the distance travelled.  Seen along the ray, that point can
// lie far before the box's entry distance when the ray runs nearly parallel to the face it crosses
// (the distance is divided by the direction component).  Every box test therefore widens each slab by a
// margin in space of 2^-18 (|o_axis| + S) + 2^-40, S the diagonal of the scene's triangles (trav_scale):
// in distance along the ray that is the margin times |1/d_axis|.  (Observed: a hit 1e-8 outside a face
// crossed with d.x = 3e-4, 3e-5 before the box's entry distance -- beyond a relative slack of 1e-5.)
constexpr float kMarginRel = 3.814697265625e-06f;   // 2^-18
constexpr float kMarginAbs = 9.094947017729282e-13f; // 2^-40
PT_HD float slab_margin(float o, float inv, float scale) { return (kMarginRel * (fabsf(o) + scale) + kMarginAbs) * fabsf(inv); }
struct RayPre {
  float3 inv;
  int sx, sy, sz;  // 1 where the direction component is negative: the near slab plane is the box's hi
  float E;         // the largest per-axis margin along the ray (axes with a finite reciprocal)
};
PT_HD RayPre ray_pre(const float3& o, const float3& d, float scale)
{
  // IEEE reciprocals: a zero component gives +-inf, so a slab distance (plane - o) * inv is +-inf, or
  // NaN when the origin lies exactly on the plane; the slab tests take near / far planes by the
  // direction's sign and combine with fminf / fmaxf, which drop a NaN, so a ray running inside a
  // face plane is kept (a clamped reciprocal would give distance 0 there and cull the box).
  RayPre r;
  r.inv = f3(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
  r.sx = r.inv.x < 0.0f;
  r.sy = r.inv.y < 0.0f;
  r.sz = r.inv.z < 0.0f;
  const float inf = as_float(0x7f800000);
  const float ex = fabsf(r.inv.x) < inf ? slab_margin(o.x, r.inv.x, scale) : 0.0f;
  const float ey = fabsf(r.inv.y) < inf ? slab_margin(o.y, r.inv.y, scale) : 0.0f;
  const float ez = fabsf(r.inv.z) < inf ? slab_margin(o.z, r.inv.z, scale) : 0.0f;
  r.E = fmaxf(fmaxf(ex, ey), ez);
  return r;
}
// Slab test of one child box; returns the (lowered) entry distance, or +inf on a miss.  Each slab
// distance is (plane - origin) * (1/d): two correctly rounded operations, so its relative error is at
// most 2 ulp plus the 1 ulp of the reciprocal, which the relative slack kSlack (>> 3 ulp) covers (the
// robust slab test of T. Ize, "Robust BVH Ray Traversal", JCGT 2013); the margin E widens the interval
// as described above.
constexpr float kSlack = 1.00001f;
PT_HD float slab(float lox, float hix, float loy, float hiy, float loz, float hiz, const float3& o, const RayPre& r, float tmin, float tmax)
{
  const float tnx = ((r.sx ? hix : lox) - o.x) * r.inv.x, tfx = ((r.sx ? lox : hix) - o.x) * r.inv.x;
  const float tny = ((r.sy ? hiy : loy) - o.y) * r.inv.y, tfy = ((r.sy ? loy : hiy) - o.y) * r.inv.y;
  const float tnz = ((r.sz ? hiz : loz) - o.z) * r.inv.z, tfz = ((r.sz ? loz : hiz) - o.z) * r.inv.z;
  const float tn = fmaxf(fmaxf(fmaxf(tnx, tny), tnz) - r.E, tmin);
  const float tf = fminf(fminf(fminf(tfx, tfy), tfz) + r.E, tmax * kSlack);
  return tn <= tf * kSlack ? tn : as_float(0x7f800000);
}
// Moller-Trumbore (T. Moller, B. Trumbore, "Fast, minimum storage ray-triangle intersection",
// JGT 1997) on (v0, e1 = v1-v0, e2 = v2-v0).  u weights v1, v weights v2.  Plain IEEE single
// operations in a fixed order (no contraction), mirrored by the CPU oracle.
PT_HD bool tri_mt(const float3& o, const float3& d, const float3& v0, const float3& e1, const float3& e2, float& t, float& u, float& v)
{
  float3 p = cross(d, e2);
  float det = dot(e1, p);
  if (det == 0.0f) return false;
  float inv = 1.0f / det;
  float3 tv = o - v0;
  u = dot(tv, p) * inv;
  if (!(u >= 0.0f && u <= 1.0f)) return false;
  float3 q = cross(tv, e1);
  v = dot(d, q) * inv;
  if (!(v >= 0.0f && u + v <= 1.0f)) return false;
  t = dot(e2, q) * inv;
  return true;
}

PT_HD float3 ld3(const float4& a) { return f3(a.x, a.y, a.z); }

// Intersect the triangles of leaf `code` and keep the closest hit (ties -> lower original index).
template <class G> PT_HD void leaf_closest(const G& S, uint32_t code, const float3& o, const float3& d, float tmin, Hit& h)
{
  uint32_t first = (code & 0x7fffffffu) >> 4, count = code & 15u;
  for (uint32_t j = first; j < first + count; ++j) {
    float4 a = PT_LDG(S.tri_v0 + j), b = PT_LDG(S.tri_e1 + j), c = PT_LDG(S.tri_e2 + j);
    float t, u, v;
    if (!tri_mt(o, d, ld3(a), ld3(b), ld3(c), t, u, v)) continue;
    int prim = as_int(a.w);
    if (t > tmin && (t < h.t || (t == h.t && h.prim >= 0 && prim < h.prim))) {
      h.t = t;
      h.u = u;
      h.v = v;
      h.prim = prim;
    }
  }
}
template <class G> PT_HD bool leaf_any(const G& S, uint32_t code, const float3& o, const float3& d, float tmin, float tmax)
{
  uint32_t first = (code & 0x7fffffffu) >> 4, count = code & 15u;
  for (uint32_t j = first; j < first + count; ++j) {
    float4 a = PT_LDG(S.tri_v0 + j), b = PT_LDG(S.tri_e1 + j), c = PT_LDG(S.tri_e2 + j);
    float t, u, v;
    if (tri_mt(o, d, ld3(a), ld3(b), ld3(c), t, u, v) && t > tmin && t < tmax) return true;
  }
  return false;
}

// Stackless traversal state.  A 64-bit trail marks, per depth, whether the far child of the node at
// that depth is still pending (`pend`), and a second 64-bit word records which child it is
// (`farc1`); the way back up follows the parent index stored in each node.  No per-ray stack lives
// in local memory.
//
// Optionally a short stack (kShortStack entries, caller-provided, typically shared memory laid out
// [slot][thread]) caches the pending far children: entry = (far child index, entry distance with its
// 6 low mantissa bits replaced by the level).  Backtracking then jumps to the deepest pending far child
// directly instead of walking up through the parents; when the stack has dropped older entries (more
// than kShortStack pending), the parent walk takes over.  The stored entry distance is rounded down
// (conservative), and tn <= t_closest * kSlack at pop time decides exactly as re-testing the box would.
#ifndef PT_SHORT_STACK
#define PT_SHORT_STACK 8
#endif
constexpr int kShortStack = PT_SHORT_STACK;  // a power of two
struct TravState {
  int cur, depth;
  unsigned long long pend, farc1;
  uint2* stk;   // short stack or null
  int stride;   // element stride between the stack's slots
  int top, lo;  // entries [lo, top) are valid (slot = index mod kShortStack)
};
PT_HD void trav_init(TravState& st, uint2* stk = nullptr, int stride = 1)
{
  st.cur = 0;
  st.depth = 0;
  st.pend = 0ull;
  st.farc1 = 0ull;
  st.stk = stk;
  st.stride = stride;
  st.top = st.lo = 0;
}
PT_HD void trav_push(TravState& st, int far, int level, float tn)
{
  if (!st.stk) return;
  uint32_t tb = (uint32_t)as_int(tn);
  st.stk[(st.top & (kShortStack - 1)) * st.stride] = make_uint2((uint32_t)far, (tb & ~63u) | (uint32_t)level);
  ++st.top;
  if (st.top - st.lo > kShortStack) st.lo = st.top - kShortStack;
}
PT_HD int highest_bit(unsigned long long x)
{
#ifdef __CUDA_ARCH__
  return 63 - __clzll((long long)x);
#else
  return 63 - __builtin_clzll(x);
#endif
}

// Backtrack to the deepest pending child.  Closest-hit: the pending far child's box is re-tested
// against the current closest distance when it is resumed.  Returns false when the root is done.
template <class G> PT_HD bool trav_backtrack(const G& S, const float3& o, const RayPre& rp, float tmin, float tlimit, TravState& st, bool retest)
{
  // short stack: the deepest pending level is the top entry's
  while (st.pend && st.top > st.lo) {
    const int L = highest_bit(st.pend);
    const uint2 e = st.stk[((st.top - 1) & (kShortStack - 1)) * st.stride];
    if ((int)(e.y & 63u) != L) break;
    --st.top;
    st.pend &= ~(1ull << L);
    if (!retest || as_float((int)(e.y & ~63u)) <= tlimit * kSlack) {
      st.cur = (int)e.x;
      st.depth = L + 1;
      return true;
    }
  }
  for (;;) {
    if (st.depth == 0) return false;
    int parent = PT_LDG(reinterpret_cast<const int*>(S.nodes + 4 * (size_t)st.cur + 3) + 2);
    --st.depth;
    unsigned long long bit = 1ull << st.depth;
    if (st.pend & bit) {
      st.pend &= ~bit;
      const float4* pn = S.nodes + 4 * (size_t)parent;
      int4 p3 = PT_LDG(reinterpret_cast<const int4*>(pn + 3));
      int far = (st.farc1 & bit) ? p3.y : p3.x;
      bool go = true;
      if (retest) {
        float tf;
        if (st.farc1 & bit) {
          float4 b1 = PT_LDG(pn + 1), b2 = PT_LDG(pn + 2);
          tf = slab(b1.x, b1.y, b1.z, b1.w, b2.z, b2.w, o, rp, tmin, tlimit);
        } else {
          float4 b0 = PT_LDG(pn), b2 = PT_LDG(pn + 2);
          tf = slab(b0.x, b0.y, b0.z, b0.w, b2.x, b2.y, o, rp, tmin, tlimit);
        }
        go = tf <= tlimit * kSlack;
      }
      if (go) {
        st.cur = far;
        ++st.depth;
        return true;
      }
    }
    st.cur = parent;
  }
}

// One closest-hit step: visit node st.cur (test both child boxes, intersect leaf children, descend
// near-first or backtrack).  Returns true when the traversal is finished.
template <class G> PT_HD bool trav_step_closest(const G& S, const float3& o, const float3& d, const RayPre& rp, float tmin, Hit& h, TravState& st)
{
  const float4* nd = S.nodes + 4 * (size_t)st.cur;
  float4 n0 = PT_LDG(nd), n1 = PT_LDG(nd + 1), n2 = PT_LDG(nd + 2);
  int4 n3 = PT_LDG(reinterpret_cast<const int4*>(nd + 3));
  float t0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, rp, tmin, h.t);
  float t1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, rp, tmin, h.t);
  bool h0 = t0 != as_float(0x7f800000), h1 = t1 != as_float(0x7f800000);
  if (h0 && n3.x < 0) { leaf_closest(S, (uint32_t)n3.x, o, d, tmin, h); h0 = false; }
  if (h1 && n3.y < 0) { leaf_closest(S, (uint32_t)n3.y, o, d, tmin, h); h1 = false; }
  h0 = h0 && t0 <= h.t * kSlack;
  h1 = h1 && t1 <= h.t * kSlack;
  if (h0 && h1) {
    bool near1 = t1 < t0;
    unsigned long long bit = 1ull << st.depth;
    st.pend |= bit;
    if (near1) st.farc1 &= ~bit; else st.farc1 |= bit;
    trav_push(st, near1 ? n3.x : n3.y, st.depth, near1 ? t0 : t1);
    st.cur = near1 ? n3.y : n3.x;
    ++st.depth;
    return false;
  }
  if (h0 || h1) {
    st.cur = h0 ? n3.x : n3.y;
    ++st.depth;
    return false;
  }
  return !trav_backtrack(S, o, rp, tmin, h.t, st, true);
}

// One any-hit step (children in fixed order, child 1 pending when both are hit).  Returns 1 when a
// triangle with tmin < t < tmax was found, -1 when the traversal finished without one, 0 otherwise.
template <class G> PT_HD int trav_step_any(const G& S, const float3& o, const float3& d, const RayPre& rp, float tmin, float tmax, TravState& st)
{
  const float4* nd = S.nodes + 4 * (size_t)st.cur;
  float4 n0 = PT_LDG(nd), n1 = PT_LDG(nd + 1), n2 = PT_LDG(nd + 2);
  int4 n3 = PT_LDG(reinterpret_cast<const int4*>(nd + 3));
  float t0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, rp, tmin, tmax);
  float t1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, rp, tmin, tmax);
  bool h0 = t0 != as_float(0x7f800000), h1 = t1 != as_float(0x7f800000);
  if (h0 && n3.x < 0) { if (leaf_any(S, (uint32_t)n3.x, o, d, tmin, tmax)) return 1; h0 = false; }
  if (h1 && n3.y < 0) { if (leaf_any(S, (uint32_t)n3.y, o, d, tmin, tmax)) return 1; h1 = false; }
  if (h0 && h1) {
    unsigned long long bit = 1ull << st.depth;
    st.pend |= bit;
    st.farc1 |= bit;
    trav_push(st, n3.y, st.depth, t1);
    st.cur = n3.x;
    ++st.depth;
    return 0;
  }
  if (h0 || h1) {
    st.cur = h0 ? n3.x : n3.y;
    ++st.depth;
    return 0;
  }
  return trav_backtrack(S, o, rp, tmin, tmax, st, false) ? 0 : -1;
}

// Node-only steps for the persistent kernels' postponed-leaf traversal (T. Aila, S. Laine, "Understanding
// the efficiency of ray traversal on GPUs", HPG 2009, speculative while-while): the hit leaf children
// of the node are recorded in (leafA, leafB) instead of being intersected, and the caller intersects
// them in a warp-wide leaf phase.  The inner children are culled against the closest hit found so far
// (the postponed leaves can only shorten it, so this is conservative).  Returns true when no node is
// left (leaves may still be pending).
template <class G> PT_HD bool trav_node_closest(const G& S, const float3& o, const RayPre& rp, float tmin, const Hit& h, TravState& st,
                                                uint32_t& leafA, uint32_t& leafB)
{
  const float4* nd = S.nodes + 4 * (size_t)st.cur;
  float4 n0 = PT_LDG(nd), n1 = PT_LDG(nd + 1), n2 = PT_LDG(nd + 2);
  int4 n3 = PT_LDG(reinterpret_cast<const int4*>(nd + 3));
  float t0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, rp, tmin, h.t);
  float t1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, rp, tmin, h.t);
  bool h0 = t0 != as_float(0x7f800000), h1 = t1 != as_float(0x7f800000);
  if (h0 && n3.x < 0) { leafA = (uint32_t)n3.x; h0 = false; }
  if (h1 && n3.y < 0) {
    if (leafA) leafB = (uint32_t)n3.y;
    else leafA = (uint32_t)n3.y;
    h1 = false;
  }
  h0 = h0 && t0 <= h.t * kSlack;
  h1 = h1 && t1 <= h.t * kSlack;
  if (h0 && h1) {
    bool near1 = t1 < t0;
    unsigned long long bit = 1ull << st.depth;
    st.pend |= bit;
    if (near1) st.farc1 &= ~bit; else st.farc1 |= bit;
    trav_push(st, near1 ? n3.x : n3.y, st.depth, near1 ? t0 : t1);
    st.cur = near1 ? n3.y : n3.x;
    ++st.depth;
    return false;
  }
  if (h0 || h1) {
    st.cur = h0 ? n3.x : n3.y;
    ++st.depth;
    return false;
  }
  return !trav_backtrack(S, o, rp, tmin, h.t, st, true);
}
template <class G> PT_HD bool trav_node_any(const G& S, const float3& o, const RayPre& rp, float tmin, float tmax, TravState& st, uint32_t& leafA,
                                            uint32_t& leafB)
{
  const float4* nd = S.nodes + 4 * (size_t)st.cur;
  float4 n0 = PT_LDG(nd), n1 = PT_LDG(nd + 1), n2 = PT_LDG(nd + 2);
  int4 n3 = PT_LDG(reinterpret_cast<const int4*>(nd + 3));
  float t0 = slab(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, rp, tmin, tmax);
  float t1 = slab(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, rp, tmin, tmax);
  bool h0 = t0 != as_float(0x7f800000), h1 = t1 != as_float(0x7f800000);
  if (h0 && n3.x < 0) { leafA = (uint32_t)n3.x; h0 = false; }
  if (h1 && n3.y < 0) {
    if (leafA) leafB = (uint32_t)n3.y;
    else leafA = (uint32_t)n3.y;
    h1 = false;
  }
  if (h0 && h1) {
    unsigned long long bit = 1ull << st.depth;
    st.pend |= bit;
    st.farc1 |= bit;
    trav_push(st, n3.y, st.depth, t1);
    st.cur = n3.x;
    ++st.depth;
    return false;
  }
  if (h0 || h1) {
    st.cur = h0 ? n3.x : n3.y;
    ++st.depth;
    return false;
  }
  return !trav_backtrack(S, o, rp, tmin, tmax, st, false);
}

// ------------------------------------------------------------------ wide BVH traversal
// Width kWide = 4 or 8 children per node (PT_BVH_WIDE at compile time).  Node: six plane rows -- lo.x
// of the children, hi.x, lo.y, hi.y, lo.z, hi.z -- of kWide floats each (kWide / 4 float4 per row),
// then kWide int child codes (>= 0: node, < 0: leaf code as in the BVH2; empty slots are leaves of no
// triangles behind a box at 1e30); 4-wide nodes are padded to 128 bytes (8 float4), 8-wide nodes take
// 224 bytes (14 float4).  Traversal keeps the hit children that are not visited next on a stack, nearest
// last, with their entry distance; closest-hit pops skip entries beyond the closest hit found so far
// (entry distance > t * kSlack), as re-testing the box would.  The stack is a ring of kRing4 entries
// (caller memory, typically shared, [slot][thread]) whose oldest entries spill to a per-thread array of
// kSpill4 entries (caller memory, typically a local array) when it overflows.
#ifndef PT_BVH_WIDE
#define PT_BVH_WIDE 4
#endif
constexpr int kWide = PT_BVH_WIDE;
static_assert(kWide == 4 || kWide == 8, "the wide BVH has 4 or 8 children per node");
constexpr int kWideRow = kWide / 4;                  // float4 per plane row
constexpr int kWideStride = kWide == 4 ? 8 : 14;     // float4 per node
constexpr int kMaxDepthWide = kWide == 4 ? 40 : 24;  // levels the stack is sized for
#ifndef PT_RING4
#define PT_RING4 8
#endif
constexpr int kRing4 = PT_RING4;  // a power of two
static_assert((kRing4 & (kRing4 - 1)) == 0, "the ring stack's size is a power of two");
constexpr int kSpill4 = (kWide - 1) * kMaxDepthWide + 8;  // kWide - 1 pending children per level
constexpr int kDone4 = 0x7fffffff;

struct Stack4 {
  uint2* ring;
  uint2* spill;
  int stride;
  int sp, spilled;
};
PT_HD void stack4_init(Stack4& s, uint2* ring, int stride, uint2* spill)
{
  s.ring = ring;
  s.spill = spill;
  s.stride = stride;
  s.sp = 0;
  s.spilled = 0;
}
PT_HD void stack4_push(Stack4& s, int code, float tn)
{
  if (s.sp - s.spilled == kRing4) {
    s.spill[s.spilled] = s.ring[(s.spilled & (kRing4 - 1)) * s.stride];
    ++s.spilled;
  }
  s.ring[(s.sp & (kRing4 - 1)) * s.stride] = make_uint2((uint32_t)code, (uint32_t)as_int(tn));
  ++s.sp;
}
PT_HD uint2 stack4_pop(Stack4& s)
{
  const int i = --s.sp;
  if (i >= s.spilled) return s.ring[(i & (kRing4 - 1)) * s.stride];
  s.spilled = i;
  return s.spill[i];
}
// Next node or leaf to visit (kDone4 when none): pops, skipping entries beyond tlimit * kSlack.
PT_HD int stack4_next(Stack4& s, float tlimit, bool cull)
{
  while (s.sp > 0) {
    const uint2 e = stack4_pop(s);
    if (!cull || as_float((int)e.y) <= tlimit * kSlack) return (int)e.x;
  }
  return kDone4;
}
// Tests the four children of node `node`; returns their count of hits, with (code, t) sorted near to
// far (misses last, at t = +inf).  A five-comparator sorting network on registers.
PT_HD void cswap4(int code[4], float t[4], int a, int b)
{
  const bool sw = t[b] < t[a];
  const float ta = t[a], tb = t[b];
  const int ca = code[a], cb = code[b];
  t[a] = sw ? tb : ta;
  t[b] = sw ? ta : tb;
  code[a] = sw ? cb : ca;
  code[b] = sw ? ca : cb;
}
// Ray constants of the wide BVH's slab test, which takes one fused multiply-add per plane:
// t = fma(plane, inv, -o * inv).  The product o * inv is rounded once per ray, an absolute error of
// at most 2^-24 |o * inv| in every slab distance of that axis (the fma itself rounds once, a relative
// error that the relative slack kSlack covers as in `slab`).  Each axis carries the margin of `slab`,
// (2^-18 (|o| + S) + 2^-40) |inv| -- more than 16 x that rounding bound as well: near distances are
// lowered and far distances raised by it (cn = -o*inv - E, cf = -o*inv + E), so the test keeps every box
// the exact test keeps, and more.  A direction component of magnitude below 2^-64 (a zero one included)
// is taken as +-2^-64 so that every constant is finite: the ray then drifts at most 2^-64 t off its
// line, which the absolute part of the margin (2^-40 in space) covers for t up to 2^24 -- far beyond any
// scene, whose other axes bound t.
constexpr float kInvMax = 18446744073709551616.0f;  // 2^64
struct RayPre4 {
  float3 inv;     // 1 / d, clamped to +-2^64
  float3 cn, cf;  // per axis: -(o * inv) - E, -(o * inv) + E
  int sx, sy, sz; // 1 where the direction component is negative: the near plane is the box's hi
};
PT_HD float clamp_inv(float d)
{
  const float r = 1.0f / d;
  return fabsf(r) <= kInvMax ? r : copysignf(kInvMax, d);
}
PT_HD RayPre4 ray_pre4(const float3& o, const float3& d, float scale)
{
  RayPre4 r;
  r.inv = f3(clamp_inv(d.x), clamp_inv(d.y), clamp_inv(d.z));
  const float ox = o.x * r.inv.x, oy = o.y * r.inv.y, oz = o.z * r.inv.z;
  const float ex = slab_margin(o.x, r.inv.x, scale), ey = slab_margin(o.y, r.inv.y, scale), ez = slab_margin(o.z, r.inv.z, scale);
  r.cn = f3(-ox - ex, -oy - ey, -oz - ez);
  r.cf = f3(-ox + ex, -oy + ey, -oz + ez);
  r.sx = r.inv.x < 0.0f;
  r.sy = r.inv.y < 0.0f;
  r.sz = r.inv.z < 0.0f;
  return r;
}
PT_HD float fma_rn(float a, float b, float c)
{
#ifdef __CUDA_ARCH__
  return __fmaf_rn(a, b, c);
#else
  return fmaf(a, b, c);
#endif
}
PT_HD float max3f(float a, float b, float c)
{
#ifdef __CUDA_ARCH__
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
#else
  return fmaxf(fmaxf(a, b), c);
#endif
}
PT_HD float min3f(float a, float b, float c)
{
#ifdef __CUDA_ARCH__
  float r;
  asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
#else
  return fminf(fminf(a, b), c);
#endif
}
// The wide node's slab test of one child, with the near and far planes of each axis chosen by the
// direction's sign (loaded from the node's lo or hi plane row): one fma per plane and three-input
// min / max; returns the (lowered) entry distance, or +inf on a miss.  The planes are finite (an empty
// slot's are 1e30) and so are the constants, so no distance is NaN.
PT_HD float slab4(float nx, float fx, float ny, float fy, float nz, float fz, const RayPre4& r, float tmin, float tmax)
{
  const float tn = fmaxf(max3f(fma_rn(nx, r.inv.x, r.cn.x), fma_rn(ny, r.inv.y, r.cn.y), fma_rn(nz, r.inv.z, r.cn.z)), tmin);
  const float tf = min3f(fma_rn(fx, r.inv.x, r.cf.x), fma_rn(fy, r.inv.y, r.cf.y), fminf(fma_rn(fz, r.inv.z, r.cf.z), tmax * kSlack));
  return tn <= tf * kSlack ? tn : as_float(0x7f800000);
}
PT_HD int popc32(unsigned m)
{
#ifdef __CUDA_ARCH__
  return __popc(m);
#else
  return __builtin_popcount(m);
#endif
}
// Tests the kWide children of node `node`: their codes and entry distances (+inf for a miss); with
// kSort and kWide == 4 sorted near to far by a five-comparator network (else in slot order),
// returning the count of hits.
template <bool kSort = true, class G>
PT_HD int node4_hits(const G& S, int node, const RayPre4& rp, float tmin, float tmax, int code[kWide], float t[kWide])
{
  const float4* nd = S.nodes4 + kWideStride * (size_t)node;
#pragma unroll
  for (int r = 0; r < kWideRow; ++r) {
    const float4 nx = PT_LDG(nd + (0 + rp.sx) * kWideRow + r), fx = PT_LDG(nd + (1 - rp.sx) * kWideRow + r);
    const float4 ny = PT_LDG(nd + (2 + rp.sy) * kWideRow + r), fy = PT_LDG(nd + (3 - rp.sy) * kWideRow + r);
    const float4 nz = PT_LDG(nd + (4 + rp.sz) * kWideRow + r), fz = PT_LDG(nd + (5 - rp.sz) * kWideRow + r);
    const int4 c = PT_LDG(reinterpret_cast<const int4*>(nd + 6 * kWideRow + r));
    t[4 * r + 0] = slab4(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, rp, tmin, tmax);
    t[4 * r + 1] = slab4(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, rp, tmin, tmax);
    t[4 * r + 2] = slab4(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, rp, tmin, tmax);
    t[4 * r + 3] = slab4(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, rp, tmin, tmax);
    code[4 * r + 0] = c.x;
    code[4 * r + 1] = c.y;
    code[4 * r + 2] = c.z;
    code[4 * r + 3] = c.w;
  }
  const float inf = as_float(0x7f800000);
  int n = 0;
#pragma unroll
  for (int k = 0; k < kWide; ++k) n += t[k] != inf;
  if constexpr (kSort && kWide == 4) {
    cswap4(code, t, 0, 1);
    cswap4(code, t, 2, 3);
    cswap4(code, t, 0, 2);
    cswap4(code, t, 1, 3);
    cswap4(code, t, 1, 2);
  }
  return n;
}
// Pushes the hit children other than the nearest, farthest first (so that they pop nearest first),
// and returns the nearest, or pops the next target when no child was hit.  4-wide: the children come
// sorted; 8-wide: repeated selection of the farthest remaining hit child over registers.
PT_HD int node4_advance(int n, const int code[kWide], const float t[kWide], Stack4& stk, float tlimit, bool cull)
{
  if constexpr (kWide == 4) {
#pragma unroll
    for (int j = 3; j >= 1; --j)
      if (j < n) stack4_push(stk, code[j], t[j]);
    return n ? code[0] : stack4_next(stk, tlimit, cull);
  } else {
    if (!n) return stack4_next(stk, tlimit, cull);
    const float inf = as_float(0x7f800000);
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < kWide; ++k) m |= (t[k] != inf ? 1u : 0u) << k;
    while (popc32(m) > 1) {
      float best = -1.0f;
      int bc = 0;
      unsigned bb = 0;
#pragma unroll
      for (int k = 0; k < kWide; ++k) {
        const bool take = ((m >> k) & 1u) && t[k] > best;
        best = take ? t[k] : best;
        bc = take ? code[k] : bc;
        bb = take ? 1u << k : bb;
      }
      stack4_push(stk, bc, best);
      m &= ~bb;
    }
    int c = 0;
#pragma unroll
    for (int k = 0; k < kWide; ++k) c = (m >> k) & 1u ? code[k] : c;
    return c;
  }
}
// One closest-hit node step: cur must be a node; returns the next target (node, leaf or kDone4).
template <class G> PT_HD int trav4_node_closest(const G& S, int cur, const RayPre4& rp, float tmin, const Hit& h, Stack4& stk)
{
  int code[kWide];
  float t[kWide];
  const int n = node4_hits(S, cur, rp, tmin, h.t, code, t);
  return node4_advance(n, code, t, stk, h.t, true);
}
// Any-hit node step.  Whether some triangle lies in (tmin, tmax) does not depend on the order in which
// the hit children are visited, so they are taken in slot order without sorting: all but the last hit
// child are pushed, the last is visited next.
template <class G> PT_HD int trav4_node_any(const G& S, int cur, const RayPre4& rp, float tmin, float tmax, Stack4& stk)
{
  int code[kWide];
  float t[kWide];
  node4_hits<false>(S, cur, rp, tmin, tmax, code, t);
  const float inf = as_float(0x7f800000);
  int next = kDone4;
  float tnext = 0.0f;
#pragma unroll
  for (int k = 0; k < kWide; ++k) {
    if (t[k] != inf) {
      if (next != kDone4) stack4_push(stk, next, tnext);
      next = code[k];
      tnext = t[k];
    }
  }
  return next != kDone4 ? next : stack4_next(stk, tmax, false);
}

template <class G> PT_HD Hit trace_closest(const G& S, const float3& o, const float3& d, float tmin, float tmax)
{
  Hit h;
  h.t = tmax;
  h.u = h.v = 0.0f;
  h.prim = -1;
  RayPre rp = ray_pre(o, d, S.trav_scale);
  TravState st;
  trav_init(st);
  while (!trav_step_closest(S, o, d, rp, tmin, h, st)) {}
  return h;
}

template <class G> PT_HD bool trace_any(const G& S, const float3& o, const float3& d, float tmin, float tmax)
{
  RayPre rp = ray_pre(o, d, S.trav_scale);
  TravState st;
  trav_init(st);
  int r;
  while ((r = trav_step_any(S, o, d, rp, tmin, tmax, st)) == 0) {}
  return r > 0;
}

// ------------------------------------------------------------------ analytic emitters
// Record k of SceneDev::ana: (position, radius), (disk normal, kind), (radiance, light index); the
// kind is stored as int bits.  Hits are tested after the triangles, emitters in light order, and
// replace the current hit only when strictly closer (a tie stays with the lower index).
enum AnaKind : int { ANA_DISK = 3, ANA_SPHERE = 4 };

// disk_mesh.cu:33-55: the ray's parameter at the disk's plane (rays within scene_epsilon of parallel
// miss) if that point lies inside the radius.
PT_HD bool ana_disk_t(const float4& a, const float4& b, const float3& o, const float3& d, float eps, float& t)
{
  const float3 position = ld3(a), normal = ld3(b);
  const float3 O = o - position;
  const float den = dot(normal, d);
  if (!(fabsf(den) > eps)) return false;
  t = -dot(O, normal) / den;
  const float3 point = o + t * d;
  const float3 v = point - position;
  return dot(v, v) <= a.w * a.w;
}
// sphere_mesh.cu:44-95: the near root (refined by a second solve from the near point when it lies
// beyond 10 radii) if it is inside (tmin, tmax), else the far root if that is.
PT_HD bool ana_sphere_t(const float4& a, const float3& o, const float3& d, float tmin, float tmax, float& t)
{
  const float3 O = o - ld3(a);
  const float radius = a.w;
  float b = dot(O, d);
  float c = dot(O, O) - radius * radius;
  float disc = b * b - c;
  if (!(disc > 0.0f)) return false;
  float sdisc = sqrtf(disc);
  const float root1 = (-b - sdisc);
  const bool do_refine = fabsf(root1) > 10.f * radius;
  float root11 = 0.0f;
  if (do_refine) {
    const float3 O1 = O + root1 * d;
    b = dot(O1, d);
    c = dot(O1, O1) - radius * radius;
    disc = b * b - c;
    if (disc > 0.0f) {
      sdisc = sqrtf(disc);
      root11 = (-b - sdisc);
    }
  }
  const float t1 = root1 + root11;
  if (t1 > tmin && t1 < tmax) {
    t = t1;
    return true;
  }
  const float root2 = (-b + sdisc) + (do_refine ? root1 : 0.0f);
  if (root2 > tmin && root2 < tmax) {
    t = root2;
    return true;
  }
  return false;
}
// Closest analytic hit in (tmin, h.t): updates h.
PT_HD void ana_closest(const SceneDev& S, const float3& o, const float3& d, float tmin, Hit& h)
{
  for (uint32_t k = 0; k < S.n_ana; ++k) {
    const float4 a = PT_LDG(S.ana + 3 * k), b = PT_LDG(S.ana + 3 * k + 1);
    float t;
    const bool hit = as_int(b.w) == ANA_DISK ? (ana_disk_t(a, b, o, d, S.integ.scene_epsilon, t) && t > tmin && t < h.t)
                                             : ana_sphere_t(a, o, d, tmin, h.t, t);
    if (hit) {
      h.t = t;
      h.u = h.v = 0.0f;
      h.prim = (int)(S.n_tris + k);
    }
  }
}
// Any analytic hit in (tmin, tmax): the emitters are opaque to shadow rays (arealight_shader.cu:27-32).
PT_HD bool ana_any(const SceneDev& S, const float3& o, const float3& d, float tmin, float tmax)
{
  for (uint32_t k = 0; k < S.n_ana; ++k) {
    const float4 a = PT_LDG(S.ana + 3 * k), b = PT_LDG(S.ana + 3 * k + 1);
    float t;
    if (as_int(b.w) == ANA_DISK ? (ana_disk_t(a, b, o, d, S.integ.scene_epsilon, t) && t > tmin && t < tmax)
                                : ana_sphere_t(a, o, d, tmin, tmax, t))
      return true;
  }
  return false;
}
// Unit normal of analytic hit k at parameter t of ray (o, d): the disk's normal, or the sphere's
// (O + t D) / radius with O = o - center (sphere_mesh.cu:78,87), normalised as the emitter program does.
PT_HD float3 ana_normal(const SceneDev& S, uint32_t k, const float3& o, const float3& d, float t)
{
  const float4 a = PT_LDG(S.ana + 3 * k), b = PT_LDG(S.ana + 3 * k + 1);
  if (as_int(b.w) == ANA_DISK) return normalize(ld3(b));
  const float3 O = o - ld3(a);
  return normalize((O + t * d) / a.w);
}
// Closest hit / any hit of the whole scene: the BVH's triangles, then the analytic emitters.
PT_HD Hit scene_closest(const SceneDev& S, const float3& o, const float3& d, float tmin, float tmax)
{
  Hit h = trace_closest(trav_geom(S), o, d, tmin, tmax);
  if (S.n_ana) ana_closest(S, o, d, tmin, h);
  return h;
}
PT_HD bool scene_any(const SceneDev& S, const float3& o, const float3& d, float tmin, float tmax)
{
  return trace_any(trav_geom(S), o, d, tmin, tmax) || (S.n_ana && ana_any(S, o, d, tmin, tmax));
}

// ------------------------------------------------------------------ environment map (Envmap.h)
PT_HD int wrap_index(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }
// Software FP32 bilinear filtering with REPEAT wrap and normalised coordinates (the sampler state of
// HDRLoader.cpp:232-236,286); the same weights as the oracle.
PT_HD float3 env_tex(const EnvDev& E, float u, float v)
{
  float x = u * (float)E.w - 0.5f, y = v * (float)E.h - 0.5f;
  float fx = floorf(x), fy = floorf(y);
  float ax = x - fx, ay = y - fy;
  int i0 = wrap_index((int)fx, E.w), j0 = wrap_index((int)fy, E.h), i1 = wrap_index((int)fx + 1, E.w), j1 = wrap_index((int)fy + 1, E.h);
  float4 t00 = PT_LDG(E.tex + (size_t)j0 * E.w + i0), t10 = PT_LDG(E.tex + (size_t)j0 * E.w + i1);
  float4 t01 = PT_LDG(E.tex + (size_t)j1 * E.w + i0), t11 = PT_LDG(E.tex + (size_t)j1 * E.w + i1);
  float w00 = (1.0f - ax) * (1.0f - ay), w10 = ax * (1.0f - ay), w01 = (1.0f - ax) * ay, w11 = ax * ay;
  return f3(t00.x * w00 + t10.x * w10 + t01.x * w01 + t11.x * w11, t00.y * w00 + t10.y * w10 + t01.y * w01 + t11.y * w11,
            t00.z * w00 + t10.z * w10 + t01.z * w01 + t11.z * w11);
}
// env_lookup, Envmap.h:57-64.
PT_D float3 env_lookup(const EnvDev& E, const float3& dir)
{
  float theta = acosf(dir.y);
  float phi = atan2f(dir.x, dir.z);
  float u = (phi + kPi) * 0.5f * kInvPi;
  float v = (float)(1.0 - (double)(theta * kInvPi));
  return env_tex(E, u, v);
}
// cdf_bsearch_marginal / cdf_bsearch_conditional, Envmap.h:23-55 (the read at middle-1 is skipped at
// middle 0, which a power-of-two table size never reaches).
PT_D unsigned cdf_bsearch(const float* cdf, unsigned size, float xi)
{
  unsigned ts = size >> 1;
  unsigned middle = ts;
  while (ts > 0) {
    unsigned odd = ts & 1;
    ts >>= 1;
    unsigned tmp = ts + odd;
    if (xi > PT_LDG(cdf + middle)) middle = middle + tmp;
    else if (middle > 0 && xi < PT_LDG(cdf + middle - 1)) middle = middle - tmp;
  }
  return middle;
}
// sample_environment, Envmap.h:66-98.
PT_D void sample_environment(const EnvDev& E, float3& dir, float3& L, uint32_t& t)
{
  const float M_2PIPI = 2.0f * kPi * kPi;
  float xi1 = rnd_tea(t), xi2 = rnd_tea(t);
  unsigned v_idx = cdf_bsearch(E.marginal_cdf, (unsigned)E.h, xi1);
  float mc = PT_LDG(E.marginal_cdf + v_idx);
  float dv = v_idx > 0 ? (xi1 - PT_LDG(E.marginal_cdf + v_idx - 1)) / (mc - PT_LDG(E.marginal_cdf + v_idx - 1)) : xi1 / mc;
  float pdf_m = PT_LDG(E.marginal_pdf + v_idx);
  float v = ((float)v_idx + dv) / (float)E.h;
  const float* crow = E.conditional_cdf + (size_t)v_idx * E.w;
  unsigned u_idx = cdf_bsearch(crow, (unsigned)E.w, xi2);
  float cc = PT_LDG(crow + u_idx);
  float du = u_idx > 0 ? (xi2 - PT_LDG(crow + u_idx - 1)) / (cc - PT_LDG(crow + u_idx - 1)) : xi2 / cc;
  float pdf_c = PT_LDG(E.conditional_pdf + (size_t)v_idx * E.w + u_idx);
  float u = ((float)u_idx + du) / (float)E.w;
  float prob = pdf_m * pdf_c;
  float theta = (1.0f - v) * kPi;
  float phi = (2.0f * u - 1.0f) * kPi;
  float st, ct, sp, cp;
  sincosf(theta, &st, &ct);
  sincosf(phi, &sp, &cp);
  dir = f3(st * sp, ct, st * cp);
  float3 em = env_tex(E, u, v);
  L = em * st * M_2PIPI / prob;
}

}  // namespace pt
