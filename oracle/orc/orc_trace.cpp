// Test infrastructure (oracle only): CPU restatement of the reference's recursive OptiX path
// tracer -- the path_tracer.cu ray generation and accumulation, the closest-hit programs of
// diffuse_shader.cu, metallic_shader.cu, rough_transparent_shader.cu and arealight_shader.cu, and
// the constantbg.cu miss program -- with the random numbers consumed in exactly the reference's
// order.  OptiX's traversal is replaced by a CPU BVH whose closest hit equals a brute-force loop over
// all triangles with the same Moller-Trumbore test as the CUDA kernels (closest t, ties to the lower
// triangle index); orc_trace_brute exposes that brute-force loop for BVH parity tests.
//
// Used by tests (image and per-path parity on small scenes) and as the CPU baseline of the
// benchmark (multi-threaded over pixels).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "orc_dipole.hpp"
#include "orc_light.hpp"
#include "orc_math.hpp"
#include "orc_microfacet.hpp"

using namespace orc;

#define EXPORT extern "C" __attribute__((visibility("default")))

namespace {

typedef V3<float> F3;

enum { MT_DIFFUSE = 0, MT_TRANSPARENT = 2, MT_GLASS = 3, MT_METAL = 4, MT_TRANSLUCENT = 5, MT_ROUGH_TRANSLUCENT = 6, MT_LAMBERTIAN_INTERFACE = 7,
       MT_ROUGH_DIFFUSE = 9, MT_LIGHT = 100 };
enum { STANDARD_DIPOLE = 0, DIRECTIONAL_DIPOLE = 1 };

struct Mat {
  u32 type, model, dist;
  float a[4], b[4];
  Cx3 eta, inv_eta;
  ScatProps props;       // translucent: scattering_properties
  u32 dipole_model = 0;  // translucent: dipole_model
  int translucent_index = -1;
  int tex = -1;          // texture (diffuse albedo / conductor roughness), -1 = none
  F3 tcenter;            // its cube-map center
  // translucent: the parameters the scattering properties were derived from (FP64 tape evaluation)
  double sig_a[3] = {0, 0, 0}, sig_sr[3] = {0, 0, 0}, mcos[3] = {0, 0, 0}, ior = 1.0, scale = 1.0;
};

struct Tex {
  unsigned w, h, ch;
  std::vector<float> data;
};

// Nearest texel of a cube map around c, faces laid out 3 x 2 (the device's cube_texel): face by the
// largest component of p - c, face coordinates from the other two divided by it.
static unsigned cube_texel(const F3& p, const F3& c, unsigned w, unsigned h)
{
  F3 d = p - c;
  float ax = std::fabs(d.x), ay = std::fabs(d.y), az = std::fabs(d.z);
  unsigned face;
  float s, t, m;
  if (ax >= ay && ax >= az) { face = d.x >= 0.0f ? 0u : 1u; m = ax; s = d.z; t = d.y; }
  else if (ay >= az) { face = d.y >= 0.0f ? 2u : 3u; m = ay; s = d.x; t = d.z; }
  else { face = d.z >= 0.0f ? 4u : 5u; m = az; s = d.x; t = d.y; }
  float u = 0.5f, v = 0.5f;
  if (m > 0.0f) {
    u = 0.5f * (s / m + 1.0f);
    v = 0.5f * (t / m + 1.0f);
  }
  const unsigned fw = w / 3u, fh = h / 2u;
  float fu = u * (float)fw, fv = v * (float)fh;
  unsigned x = fu > 0.0f ? (unsigned)fu : 0u, y = fv > 0.0f ? (unsigned)fv : 0u;
  if (x >= fw) x = fw - 1u;
  if (y >= fh) y = fh - 1u;
  return ((face / 3u) * fh + y) * w + (face % 3u) * fw + x;
}

// PositionSample, structs.h:105-114 (80 bytes).
struct Probe {
  F3 pos, dir, normal, L, transmitted, weight;
  float pad[2];
};
static_assert(sizeof(Probe) == 80, "PositionSample layout");

struct TranslucentObject {
  int material;
  unsigned first_tri, n_tris;
};

struct Tri {
  F3 v0, e1, e2;
};

// Path tape (test infrastructure for the adjoint): what each vertex of a camera path adds to the path
// radiance and what it multiplies the rest of the path by, with every sampled quantity (directions,
// Russian-roulette and acceptance decisions and probabilities) frozen, so that the path's radiance
// can be re-evaluated in FP64 for other parameter values (see orc_tape_*).
enum TapeType { TAPE_EMIT = 0, TAPE_CONST_W = 1, TAPE_NEE = 2, TAPE_DIFF_W = 3, TAPE_METAL_W = 4, TAPE_BEER = 5, TAPE_GATHER = 6 };
struct TapeRec {
  int type = TAPE_EMIT;
  int tex = -1, texel = -1, mat = -1;
  float v[3] = {0.0f, 0.0f, 0.0f};     // emission | constant weight | NEE factor (albedo excluded) | metal weight at alpha0
  float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};  // diffuse: prob0 | metal: cos(m,n), cos(wi,n), cos(wo,n), alpha0 | beer: t, prob0
  int g_begin = 0, g_count = 0;       // gather: accepted probes
};
struct TapeProbe {
  float dist, wl[3], exp0;
};
struct Tape {
  std::vector<TapeRec> recs;
  std::vector<TapeProbe> probes;
  bool valid = true;
};

struct Scene {
  std::vector<Tri> tris;
  std::vector<float> pos9;     // vertex positions as given, 9 per triangle (the probe pass reads these)
  std::vector<int> info;       // 4 per triangle
  std::vector<F3> normals;
  std::vector<Mat> mats;
  LightSet lights;
  F3 eye, U, V, W;
  u32 width, height, po_x, po_y, pd_x, pd_y;
  int max_depth;
  float eps;
  int rr_start;
  F3 bg;
  EnvMap env;
  std::vector<float> env_texels;
  std::vector<TranslucentObject> translucent;
  std::vector<Tex> textures;
  // path tapes of the last recorded render: [frame][pixel] over its pixel range
  bool record = false;
  std::vector<Tape> tapes;
  unsigned tape_first = 0, tape_frames = 0, tape_p0 = 0, tape_p1 = 0;
  unsigned samples = 500;                // context["samples"] (OptixSceneLoader.cpp:11,17)
  std::vector<Probe> probes;             // samples_output_buffer of the current frame
  unsigned probe_frame = 0xffffffffu;
  bool env_present = false, env_is_light = false;
  // BVH
  struct Node { float lo[3], hi[3]; int left, right, first, count; };
  std::vector<Node> nodes;
  std::vector<int> order;
  std::atomic<long> capped{0};
  // the geometry of the disk and sphere lights (Light.cpp:370-503, 505-610), in light order
  struct Ana { int kind; F3 pos; float radius; F3 normal; F3 radiance; };
  std::vector<Ana> ana;
};

// Moller-Trumbore in the same operation order as the CUDA kernel (pt_scene.cuh tri_mt).
static inline bool tri_mt(const F3& o, const F3& d, const Tri& T, float& t, float& u, float& v)
{
  F3 p = cross(d, T.e2);
  float det = dot(T.e1, p);
  if (det == 0.0f) return false;
  float inv = 1.0f / det;
  F3 tv = o - T.v0;
  u = dot(tv, p) * inv;
  if (!(u >= 0.0f && u <= 1.0f)) return false;
  F3 q = cross(tv, T.e1);
  v = dot(d, q) * inv;
  if (!(v >= 0.0f && u + v <= 1.0f)) return false;
  t = dot(T.e2, q) * inv;
  return true;
}

struct HitRec {
  float t, u, v;
  int prim;
};

static void build_bvh(Scene& S)
{
  size_t n = S.tris.size();
  S.order.resize(n);
  for (size_t i = 0; i < n; ++i) S.order[i] = (int)i;
  std::vector<float> lo(3 * n), hi(3 * n), c(3 * n);
  for (size_t i = 0; i < n; ++i) {
    const Tri& T = S.tris[i];
    F3 v1 = T.v0 + T.e1, v2 = T.v0 + T.e2;  // only for bounds; widened below
    float p[3][3] = {{T.v0.x, T.v0.y, T.v0.z}, {v1.x, v1.y, v1.z}, {v2.x, v2.y, v2.z}};
    for (int k = 0; k < 3; ++k) {
      lo[3 * i + k] = std::min(p[0][k], std::min(p[1][k], p[2][k]));
      hi[3 * i + k] = std::max(p[0][k], std::max(p[1][k], p[2][k]));
      c[3 * i + k] = 0.5f * (lo[3 * i + k] + hi[3 * i + k]);
    }
  }
  S.nodes.clear();
  S.nodes.reserve(2 * n + 1);
  struct Item { int node, b, e; };
  std::vector<Item> work;
  S.nodes.push_back(Scene::Node());
  work.push_back({0, 0, (int)n});
  while (!work.empty()) {
    Item it = work.back();
    work.pop_back();
    Scene::Node nd;
    for (int k = 0; k < 3; ++k) { nd.lo[k] = INFINITY; nd.hi[k] = -INFINITY; }
    for (int i = it.b; i < it.e; ++i)
      for (int k = 0; k < 3; ++k) {
        nd.lo[k] = std::min(nd.lo[k], lo[3 * S.order[i] + k]);
        nd.hi[k] = std::max(nd.hi[k], hi[3 * S.order[i] + k]);
      }
    // widen by a relative margin so the box test is conservative for the single-precision hits
    for (int k = 0; k < 3; ++k) {
      float m = 1e-5f * (std::fabs(nd.lo[k]) + std::fabs(nd.hi[k])) + 1e-6f;
      nd.lo[k] -= m;
      nd.hi[k] += m;
    }
    if (it.e - it.b <= 4) {
      nd.left = nd.right = -1;
      nd.first = it.b;
      nd.count = it.e - it.b;
      S.nodes[it.node] = nd;
      continue;
    }
    int axis = 0;
    float ext[3] = {nd.hi[0] - nd.lo[0], nd.hi[1] - nd.lo[1], nd.hi[2] - nd.lo[2]};
    if (ext[1] > ext[axis]) axis = 1;
    if (ext[2] > ext[axis]) axis = 2;
    int mid = (it.b + it.e) / 2;
    std::nth_element(S.order.begin() + it.b, S.order.begin() + mid, S.order.begin() + it.e,
                     [&](int x, int y) { return c[3 * x + axis] < c[3 * y + axis]; });
    nd.left = (int)S.nodes.size();
    nd.right = nd.left + 1;
    nd.first = nd.count = 0;
    S.nodes[it.node] = nd;
    S.nodes.push_back(Scene::Node());
    S.nodes.push_back(Scene::Node());
    work.push_back({nd.left, it.b, mid});
    work.push_back({nd.right, mid, it.e});
  }
}

static inline bool box_hit(const Scene::Node& n, const double* o, const double* inv, double tmin, double tmax)
{
  double t0 = tmin, t1 = tmax;
  for (int k = 0; k < 3; ++k) {
    double a = (n.lo[k] - o[k]) * inv[k], b = (n.hi[k] - o[k]) * inv[k];
    if (a > b) std::swap(a, b);
    t0 = std::max(t0, a);
    t1 = std::min(t1, b);
  }
  return t0 <= t1 * (1.0 + 1e-9) + 1e-12;
}

// disk_mesh.cu:33-55
static bool ana_disk_t(const Scene::Ana& A, const F3& o, const F3& d, float eps, float& t)
{
  F3 O = o - A.pos;
  float den = dot(A.normal, d);
  if (!(std::fabs(den) > eps)) return false;
  t = -dot(O, A.normal) / den;
  F3 point = o + t * d;
  F3 v = point - A.pos;
  float square_dist = dot(v, v);
  return square_dist <= A.radius * A.radius;
}
// sphere_mesh.cu:44-95: the (refined) near root if rtPotentialIntersection accepts it, else the far root
static bool ana_sphere_t(const Scene::Ana& A, const F3& o, const F3& d, float tmin, float tmax, float& t)
{
  F3 O = o - A.pos;
  F3 D = d;
  float radius = A.radius;
  float b = dot(O, D);
  float c = dot(O, O) - radius * radius;
  float disc = b * b - c;
  if (!(disc > 0.0f)) return false;
  float sdisc = std::sqrt(disc);
  float root1 = (-b - sdisc);
  bool do_refine = false;
  float root11 = 0.0f;
  if (std::fabs(root1) > 10.f * radius) do_refine = true;
  if (do_refine) {
    F3 O1 = O + root1 * D;
    b = dot(O1, D);
    c = dot(O1, O1) - radius * radius;
    disc = b * b - c;
    if (disc > 0.0f) {
      sdisc = std::sqrt(disc);
      root11 = (-b - sdisc);
    }
  }
  if (root1 + root11 > tmin && root1 + root11 < tmax) {
    t = root1 + root11;
    return true;
  }
  float root2 = (-b + sdisc) + (do_refine ? root1 : 0);
  if (root2 > tmin && root2 < tmax) {
    t = root2;
    return true;
  }
  return false;
}
// The analytic emitters after the triangles, in light order; a hit replaces the current one only when
// strictly closer.  Their hits carry index n_tris + k.
static void ana_closest(const Scene& S, const F3& o, const F3& d, float tmin, HitRec& h)
{
  for (size_t k = 0; k < S.ana.size(); ++k) {
    const Scene::Ana& A = S.ana[k];
    float t;
    bool hit = A.kind == DISK_LIGHT ? (ana_disk_t(A, o, d, S.eps, t) && t > tmin && t < h.t) : ana_sphere_t(A, o, d, tmin, h.t, t);
    if (hit) h = {t, 0.0f, 0.0f, (int)(S.tris.size() + k)};
  }
}
static bool ana_any(const Scene& S, const F3& o, const F3& d, float tmin, float tmax)
{
  for (const Scene::Ana& A : S.ana) {
    float t;
    if (A.kind == DISK_LIGHT ? (ana_disk_t(A, o, d, S.eps, t) && t > tmin && t < tmax) : ana_sphere_t(A, o, d, tmin, tmax, t)) return true;
  }
  return false;
}

static HitRec closest(const Scene& S, const F3& o, const F3& d, float tmin, float tmax)
{
  HitRec h = {tmax, 0.0f, 0.0f, -1};
  double od[3] = {o.x, o.y, o.z};
  double inv[3] = {1.0 / (d.x != 0 ? d.x : 1e-30), 1.0 / (d.y != 0 ? d.y : 1e-30), 1.0 / (d.z != 0 ? d.z : 1e-30)};
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const Scene::Node& n = S.nodes[stack[--sp]];
    if (!box_hit(n, od, inv, tmin, (double)h.t * (1.0 + 1e-6))) continue;
    if (n.left < 0) {
      for (int i = n.first; i < n.first + n.count; ++i) {
        int prim = S.order[i];
        float t, u, v;
        if (!tri_mt(o, d, S.tris[prim], t, u, v)) continue;
        if (t > tmin && (t < h.t || (t == h.t && h.prim >= 0 && prim < h.prim))) h = {t, u, v, prim};
      }
    } else {
      stack[sp++] = n.left;
      stack[sp++] = n.right;
    }
  }
  if (!S.ana.empty()) ana_closest(S, o, d, tmin, h);
  return h;
}

static bool occluded(const Scene& S, const F3& o, const F3& d, float tmin, float tmax)
{
  double od[3] = {o.x, o.y, o.z};
  double inv[3] = {1.0 / (d.x != 0 ? d.x : 1e-30), 1.0 / (d.y != 0 ? d.y : 1e-30), 1.0 / (d.z != 0 ? d.z : 1e-30)};
  int stack[128];
  int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    const Scene::Node& n = S.nodes[stack[--sp]];
    if (!box_hit(n, od, inv, tmin, (double)tmax * (1.0 + 1e-6))) continue;
    if (n.left < 0) {
      for (int i = n.first; i < n.first + n.count; ++i) {
        float t, u, v;
        if (tri_mt(o, d, S.tris[S.order[i]], t, u, v) && t > tmin && t < tmax) return true;
      }
    } else {
      stack[sp++] = n.left;
      stack[sp++] = n.right;
    }
  }
  return !S.ana.empty() && ana_any(S, o, d, tmin, tmax);
}

// Shading normal: normalize(rtTransformNormal(normalize(n))) with the identity transform.
static F3 shading_normal(const Scene& S, int prim, float u, float v)
{
  const int* in = &S.info[4 * (size_t)prim];
  F3 n;
  if (in[0] >= 0) {
    const F3 &n0 = S.normals[in[0]], &n1 = S.normals[in[1]], &n2 = S.normals[in[2]];
    n = normalize(n1 * u + n2 * v + n0 * (1.0f - u - v));
  } else {
    n = normalize(cross(S.tris[prim].e1, S.tris[prim].e2));
  }
  return normalize(n);
}

struct PRD {
  F3 result;
  int emit_light;
  int depth;
  u32 seed;
  Seed64 seed64;
  bool probe_path = false;  // traced by the probe pass: translucent hits do not gather
  Tape* tape = nullptr;     // camera path being recorded
};

static inline int tape_add(PRD& prd, const TapeRec& r)
{
  if (!prd.tape) return -1;
  prd.tape->recs.push_back(r);
  return (int)prd.tape->recs.size() - 1;
}
static inline void tape_emit(PRD& prd, const F3& e)
{
  if (!prd.tape || (e.x == 0.0f && e.y == 0.0f && e.z == 0.0f)) return;
  TapeRec r;
  r.type = TAPE_EMIT;
  r.v[0] = e.x; r.v[1] = e.y; r.v[2] = e.z;
  prd.tape->recs.push_back(r);
}
static inline void tape_const_w(PRD& prd, int slot, const F3& w)
{
  if (!prd.tape || slot < 0) return;
  TapeRec& r = prd.tape->recs[slot];
  r.type = TAPE_CONST_W;
  r.v[0] = w.x; r.v[1] = w.y; r.v[2] = w.z;
}

static void trace(Scene& S, const F3& o, const F3& d, PRD& prd, LightSet& ls);

// diffuse_shader.cu:42-107
static void shade_diffuse(Scene& S, const Mat& m, const F3& o, const F3& d, const HitRec& h, PRD& prd, LightSet& ls)
{
  if (prd.depth > S.max_depth) return;
  F3 hit_pos = o + h.t * d;
  F3 normal = shading_normal(S, h.prim, h.u, h.v);
  F3 ffnormal = faceforward(normal, -d, normal);
  F3 dc = v3(m.a[0], m.a[1], m.a[2]);
  int texel = -1;
  if (m.tex >= 0) {
    const Tex& T = S.textures[m.tex];
    unsigned tx = cube_texel(hit_pos, m.tcenter, T.w, T.h);
    dc = v3(T.data[3 * tx], T.data[3 * tx + 1], T.data[3 * tx + 2]);
    texel = (int)tx;
  }
  u32& t = prd.seed;
  F3 result = v3s(0.0f);
  float draw = rnd_tea(t);
  if (ls.n_lights > 0) {
    u32 li = (u32)((float)ls.n_lights * draw);
    if ((long)li >= ls.n_lights) { li = (u32)(ls.n_lights - 1); ++ls.oob; }
    float light_pdf = 1.0f / (float)ls.n_lights;
    F3 w_l = v3s(0.0f), radiance = v3s(0.0f);
    float dist = 0.0f;
    eval_direct<float>(hit_pos, ls.lights[li], ls, w_l, radiance, dist, t);
    radiance = radiance / light_pdf;
    float cos_theta = dot(ffnormal, w_l);
    if (cos_theta > 0.0f) {
      float V = occluded(S, hit_pos, w_l, S.eps, dist - S.eps) ? 0.0f : 1.0f;
      F3 Li = V * radiance;
      result = result + Li * K<float>::INV_PI * cos_theta * dc;
      prd.emit_light = 0;
      if (prd.tape && V != 0.0f) {
        if (texel >= 0) {
          TapeRec r;
          r.type = TAPE_NEE;
          r.tex = m.tex;
          r.texel = texel;
          F3 f = Li * K<float>::INV_PI * cos_theta;
          r.v[0] = f.x; r.v[1] = f.y; r.v[2] = f.z;
          tape_add(prd, r);
        } else {
          tape_emit(prd, Li * K<float>::INV_PI * cos_theta * dc);
        }
      }
    }
  }
  float prob = (dc.x + dc.y + dc.z) / 3.0f;
  float xi = rnd_tea(t);
  bool forced = prd.depth < S.rr_start;
  if (forced) prob = 1.0f;
  if (xi < prob || forced) {
    if (prd.tape) {
      TapeRec r;
      if (texel >= 0) {
        r.type = TAPE_DIFF_W;
        r.tex = m.tex;
        r.texel = texel;
        r.c[0] = prob;
      } else {
        r.type = TAPE_CONST_W;
        F3 wgt = dc / prob;
        r.v[0] = wgt.x; r.v[1] = wgt.y; r.v[2] = wgt.z;
      }
      tape_add(prd, r);
    }
    F3 nd = sample_cosine_weighted<float>(ffnormal, t);
    PRD child;
    child.probe_path = prd.probe_path;
    child.tape = prd.tape;
    child.depth = prd.depth + 1;
    child.seed = t;
    child.seed64 = prd.seed64;
    child.result = v3s(0.0f);
    child.emit_light = prd.emit_light;
    trace(S, hit_pos, nd, child, ls);
    result = result + child.result * dc / prob;
    prd.seed = child.seed;
  }
  prd.result = result;
}

// metallic_shader.cu:45-161
static void shade_metal(Scene& S, const Mat& m, const F3& o, const F3& d, const HitRec& h, PRD& prd, LightSet& ls)
{
  if (prd.depth >= S.max_depth) { prd.result = v3s(0.0f); return; }
  F3 result = v3s(0.0f);
  F3 hit_point = o + h.t * d;
  F3 normal = shading_normal(S, h.prim, h.u, h.v);
  F3 ffnormal = faceforward(normal, -d, normal);
  F3 w_i = -d;
  u32& seed = prd.seed;
  float a_x = m.a[0], a_y = m.a[1];
  int rtexel = -1;
  if (m.tex >= 0) {
    const Tex& T = S.textures[m.tex];
    rtexel = (int)cube_texel(hit_point, m.tcenter, T.w, T.h);
    a_x = a_y = T.data[rtexel];
  }
  int capped = 0;
  if (m.model == MULTISCATTERING) {
    u32 order = 0;
    F3 wm, weight;
    F3 lwo = ms_conductor_sample<float>((int)m.dist, to_local(w_i, normal), wm, m.eta, m.inv_eta, a_x, a_y, seed, order, weight, 4096, &capped);
    F3 w_o = to_world(lwo, normal);
    PRD child;
    child.probe_path = prd.probe_path;
    child.tape = prd.tape;
    child.depth = prd.depth + 1;
    child.result = v3s(0.0f);
    child.seed = seed;
    child.seed64 = prd.seed64;
    child.emit_light = 1;
    tape_const_w(prd, tape_add(prd, TapeRec()), weight);
    trace(S, hit_point, w_o, child, ls);
    result = result + child.result * weight;
  } else {
    float z1 = rnd_tea(seed), z2 = rnd_tea(seed);
    F3 mn;
    float G_i_m;
    if (m.model == WALTER) {
      mn = sample_normal<float>((int)m.dist, ffnormal, z1, z2, a_x);
      G_i_m = masking_G1<float>((int)m.dist, w_i, mn, ffnormal, a_x);
    } else {
      mn = sample_visible_normal<float>((int)m.dist, w_i, ffnormal, a_x, a_y, z1, z2, &capped);
      G_i_m = masking_G1_aniso<float>((int)m.dist, w_i, mn, ffnormal, a_x, a_y);
    }
    if (G_i_m <= 0.0f) { prd.result = result; S.capped += capped; return; }
    F3 F = fresnel_complex<float>(w_i, mn, m.eta);
    F3 w_o = -w_i + 2.0f * mn * dot(w_i, mn);
    float abs_i_m = std::fabs(dot(w_i, mn)), abs_i_n = std::fabs(dot(w_i, ffnormal)), abs_n_m = std::fabs(dot(normal, mn));
    PRD child;
    child.probe_path = prd.probe_path;
    child.tape = prd.tape;
    child.depth = prd.depth + 1;
    child.result = v3s(0.0f);
    child.seed = seed;
    child.seed64 = prd.seed64;
    child.emit_light = 1;
    F3 weight = F;
    float G_o_m = (m.model == WALTER) ? masking_G1<float>((int)m.dist, w_o, mn, ffnormal, a_x) : masking_G1_aniso<float>((int)m.dist, w_o, mn, ffnormal, a_x, a_y);
    if (G_o_m <= 0.0f) { prd.result = result; S.capped += capped; return; }
    const int slot = tape_add(prd, TapeRec());
    trace(S, hit_point, w_o, child, ls);
    if (m.model == WALTER) weight = weight * (abs_i_m * G_i_m * G_o_m / (abs_i_n * abs_n_m));
    else weight = weight * G_o_m;
    if (slot >= 0) {
      tape_const_w(prd, slot, weight);
      if (rtexel >= 0 && m.dist == GGX) {
        TapeRec& r = prd.tape->recs[slot];
        r.type = TAPE_METAL_W;
        r.tex = m.tex;
        r.texel = rtexel;
        r.c[0] = dot(mn, ffnormal);
        r.c[1] = dot(w_i, ffnormal);
        r.c[2] = dot(w_o, ffnormal);
        r.c[3] = a_x;
      }
    }
    prd.seed = child.seed;
    result = result + child.result * weight;
  }
  S.capped += capped;
  prd.result = result;
}

// rough_transparent_shader.cu:66-225
static void shade_glass(Scene& S, const Mat& m, const F3& o, const F3& d, const HitRec& h, PRD& prd, LightSet& ls)
{
  if (prd.depth >= S.max_depth) { prd.result = v3s(0.0f); return; }
  F3 result = v3s(0.0f);
  F3 hit_point = o + h.t * d;
  F3 normal = shading_normal(S, h.prim, h.u, h.v);
  F3 ffnormal = faceforward(normal, -d, normal);
  F3 w_i = -d;
  u32& t = prd.seed;
  const float ior = m.a[0], rough = m.a[1];
  F3 beam_T = v3s(1.0f);
  float cos_theta = dot(-d, normal);
  if (cos_theta < 0.0f) {
    beam_T = vexp((-h.t) * v3(m.b[0], m.b[1], m.b[2]));
    float prob = (beam_T.x + beam_T.y + beam_T.z) / 3.0f;
    if (rnd_tea(t) >= prob) return;
    beam_T = beam_T / prob;
  }
  float z1 = rnd_tea(t), z2 = rnd_tea(t);
  int capped = 0;
  if (m.model == MULTISCATTERING) {
    u32 order = 0;
    F3 lwo = ms_dielectric_sample<float>((int)m.dist, to_local(w_i, normal), 1.0f / ior, rough, rough, t, order, 4096, &capped);
    F3 w_o = to_world(lwo, normal);
    PRD child;
    child.probe_path = prd.probe_path;
    child.tape = prd.tape;
    child.depth = prd.depth + 1;
    child.result = v3s(0.0f);
    child.seed = t;
    child.seed64 = prd.seed64;
    child.emit_light = 1;
    tape_const_w(prd, tape_add(prd, TapeRec()), beam_T);
    trace(S, hit_point, w_o, child, ls);
    prd.seed = child.seed;
    result = result + child.result;
  } else {
    F3 mn = (m.model == WALTER) ? sample_normal<float>((int)m.dist, ffnormal, z1, z2, rough)
                                : sample_visible_normal<float>((int)m.dist, w_i, ffnormal, rough, rough, z1, z2, &capped);
    float cos_in = dot(normal, w_i);
    float eta = cos_in < 0.0f ? ior : 1.0f / ior;
    float G_i_m = (m.model == WALTER) ? masking_G1<float>((int)m.dist, w_i, mn, ffnormal, rough) : masking_G1_aniso<float>((int)m.dist, w_i, mn, ffnormal, rough, rough);
    if (G_i_m <= 0.0f) { prd.result = result; S.capped += capped; return; }
    float ct = std::fabs(dot(mn, -d));
    float st2 = eta * eta * (1.0f - ct * ct);
    float ctt = std::sqrt(1.0f - st2);
    float R = st2 < 1.0f ? fresnel_R(ct, ctt, eta) : 1.0f;
    F3 refr = eta * d + mn * (eta * ct - ctt);
    F3 refl = reflect(d, mn);
    float abs_i_m = std::fabs(dot(w_i, mn)), abs_i_n = std::fabs(dot(w_i, ffnormal)), abs_n_m = std::fabs(dot(normal, mn));
    float rr = rnd_tea(t);
    PRD child;
    child.probe_path = prd.probe_path;
    child.tape = prd.tape;
    child.depth = prd.depth + 1;
    child.result = v3s(0.0f);
    child.seed = t;
    child.seed64 = prd.seed64;
    child.emit_light = 1;
    F3 w_o = rr > R ? refr : refl;
    float G_o_m = (m.model == WALTER) ? masking_G1<float>((int)m.dist, w_o, mn, ffnormal, rough) : masking_G1_aniso<float>((int)m.dist, w_o, mn, ffnormal, rough, rough);
    if (G_o_m <= 0.0f) { prd.result = result; S.capped += capped; return; }
    const int slot = tape_add(prd, TapeRec());
    trace(S, hit_point, w_o, child, ls);
    float weight = (m.model == WALTER) ? abs_i_m * G_i_m * G_o_m / (abs_i_n * abs_n_m) : G_o_m;
    tape_const_w(prd, slot, weight * beam_T);
    prd.seed = child.seed;
    result = result + child.result * weight;
  }
  S.capped += capped;
  prd.result = result * beam_T;
}

// A child path of `prd` with the given emission flag (the reference's fresh PerRayData_radiance: depth + 1,
// the parent's tea seed, zero result; its MD5 state follows the parent's).
static inline PRD child_of(const PRD& prd, int emit_light)
{
  PRD child;
  child.probe_path = prd.probe_path;
  child.tape = prd.tape;
  child.depth = prd.depth + 1;
  child.result = v3s(0.0f);
  child.seed = prd.seed;
  child.seed64 = prd.seed64;
  child.emit_light = emit_light;
  return child;
}

// transparent_shader.cu:47-115 (DIFFUSE_PART undefined): smooth glass.  The shader increments the
// payload's own depth and traces the child with that payload, so the child sees depth + 1 and its
// random numbers and emission flag flow back into this vertex.
static void shade_transparent(Scene& S, const Mat& m, const F3& o, const F3& d, const HitRec& h, PRD& prd, LightSet& ls)
{
  prd.result = v3s(0.0f);
  if (prd.depth > S.max_depth) return;
  ++prd.depth;
  F3 hit_pos = o + h.t * d;
  F3 normal = shading_normal(S, h.prim, h.u, h.v);
  u32& t = prd.seed;
  const float ior = m.a[0];
  F3 beam_T = v3s(1.0f);
  float n1_over_n2 = 1.0f / ior;
  float cos_theta = dot(-d, normal);
  if (cos_theta < 0.0f) {
    beam_T = vexp(-h.t * v3(m.b[0], m.b[1], m.b[2]));
    float prob = (beam_T.x + beam_T.y + beam_T.z) / 3.0f;
    if (rnd_tea(t) >= prob) return;
    beam_T = beam_T / prob;
    n1_over_n2 = ior;
    normal = -normal;
    cos_theta = -cos_theta;
  }
  float R = 1.0f;
  float sin_theta_t_sqr = n1_over_n2 * n1_over_n2 * (1.0f - cos_theta * cos_theta);
  float cos_theta_t = 0;
  if (sin_theta_t_sqr < 1.0f) {
    cos_theta_t = std::sqrt(1.0f - sin_theta_t_sqr);
    R = fresnel_R(cos_theta, cos_theta_t, n1_over_n2);
  }
  float reflect_xi = rnd_tea(t);
  F3 dir;
  if (reflect_xi < R) dir = reflect(d, normal);
  else dir = n1_over_n2 * d + normal * (n1_over_n2 * cos_theta - cos_theta_t);
  prd.emit_light = 1;
  tape_const_w(prd, tape_add(prd, TapeRec()), beam_T);
  trace(S, hit_pos, dir, prd, ls);
  prd.result = prd.result * beam_T;
}

// R of the interface for cos_i: the repeated block of lambertian_interface_shader.cu:69-76.
static inline float interface_R(float cos_i, float n1_over_n2)
{
  float R = 1.0f;
  float sin_t_sqr = n1_over_n2 * n1_over_n2 * (1.0f - cos_i * cos_i);
  if (sin_t_sqr < 1.0f) R = fresnel_R(cos_i, std::sqrt(1.0f - sin_t_sqr), n1_over_n2);
  return R;
}

// lambertian_interface_shader.cu:51-173
static void shade_lambertian_interface(Scene& S, const Mat& m, const F3& o, const F3& d, const HitRec& h, PRD& prd, LightSet& ls)
{
  if (prd.depth > S.max_depth) return;
  F3 hit_pos = o + h.t * d;
  F3 normal = shading_normal(S, h.prim, h.u, h.v);
  F3 ffnormal = faceforward(normal, -d, normal);
  F3 result = v3s(0.0f);
  u32& t = prd.seed;
  const F3 dc = v3(m.a[0], m.a[1], m.a[2]);
  const float ior = m.a[3];
  float n1_over_n2 = 1.0f / ior;
  float r_10 = two_C1(ior);
  float cos_theta_i = dot(-d, ffnormal);
  float R_i = interface_R(cos_theta_i, n1_over_n2);
  float T_01_i = 1.0f - R_i;
  u32 light_idx = (u32)((float)ls.n_lights * rnd_tea(t));
  if ((long)light_idx >= ls.n_lights) { light_idx = (u32)(ls.n_lights - 1); ++ls.oob; }
  float light_pdf = 1.0f / (float)ls.n_lights;
  F3 w_l = v3s(0.0f), radiance = v3s(0.0f);
  float dist = 0.0f;
  eval_direct<float>(hit_pos, ls.lights[light_idx], ls, w_l, radiance, dist, t);
  radiance = radiance / light_pdf;
  float cos_theta_l = dot(ffnormal, w_l);
  if (cos_theta_l > 0.0) {
    float V = occluded(S, hit_pos, w_l, S.eps, dist) ? 0.0f : 1.0f;
    F3 Li = V * radiance;
    float T_01_l = 1.0f - interface_R(cos_theta_l, n1_over_n2);
    F3 e = Li * K<float>::INV_PI * cos_theta_l * dc * n1_over_n2 * n1_over_n2 * T_01_l * T_01_i / (1.0f - dc * r_10);
    result = result + e;
    tape_emit(prd, e);
    prd.emit_light = 0;
  }
  float prob = R_i;
  float xi = rnd_tea(t);
  if (xi > prob) {
    F3 diffuse_dir = sample_cosine_weighted<float>(ffnormal, t);
    float cos_theta_r = dot(diffuse_dir, ffnormal);
    float T_01_r = 1.0f - interface_R(cos_theta_r, n1_over_n2);
    PRD child = child_of(prd, prd.emit_light);
    const int slot = tape_add(prd, TapeRec());
    trace(S, hit_pos, diffuse_dir, child, ls);
    F3 wgt = dc * n1_over_n2 * n1_over_n2 * T_01_r / (1.0f - dc * r_10);
    tape_const_w(prd, slot, wgt);
    result = result + child.result * dc * n1_over_n2 * n1_over_n2 * T_01_r / (1.0f - dc * r_10);
    prd.seed = child.seed;
  } else {
    F3 refl_dir = reflect(d, normal);
    PRD child = child_of(prd, 1);
    tape_const_w(prd, tape_add(prd, TapeRec()), v3s(1.0f));
    trace(S, hit_pos, refl_dir, child, ls);
    result = result + child.result;
    prd.seed = child.seed;
  }
  prd.result = result;
}

// rough_diffuse_shader.cu:55-292
static void shade_rough_diffuse(Scene& S, const Mat& m, const F3& o, const F3& d, const HitRec& h, PRD& prd, LightSet& ls)
{
  if (prd.depth > S.max_depth) return;
  F3 hit_pos = o + h.t * d;
  F3 normal = shading_normal(S, h.prim, h.u, h.v);
  F3 ffnormal = faceforward(normal, -d, normal);
  F3 w_i = -d;
  F3 result = v3s(0.0f);
  u32& t = prd.seed;
  const F3 dc = v3(m.a[0], m.a[1], m.a[2]);
  const float ior = m.a[3];
  float n1_over_n2 = 1.0f / ior;
  float r_10 = two_C1(ior);
  const float a_x = m.b[1], a_y = m.b[2];
  const int dist = (int)m.dist;
  int capped = 0;
  float z1 = rnd_tea(t);
  float z2 = rnd_tea(t);
  F3 microfacet_normal = sample_visible_normal<float>(dist, w_i, ffnormal, a_x, a_y, z1, z2, &capped);
  float cos_theta_i = dot(w_i, microfacet_normal);
  float R_i = interface_R(cos_theta_i, n1_over_n2);
  float T_01_i = 1.0f - R_i;
  // direct illumination (:100-178)
  u32 light_idx = (u32)((float)ls.n_lights * rnd_tea(t));
  if ((long)light_idx >= ls.n_lights) { light_idx = (u32)(ls.n_lights - 1); ++ls.oob; }
  float light_pdf = 1.0f / (float)ls.n_lights;
  F3 w_l = v3s(0.0f), radiance = v3s(0.0f);
  float ldist = 0.0f;
  eval_direct<float>(hit_pos, ls.lights[light_idx], ls, w_l, radiance, ldist, t);
  radiance = radiance / light_pdf;
  float cos_theta_l = dot(ffnormal, w_l);
  if (cos_theta_l > 0.0) {
    float V = occluded(S, hit_pos, w_l, S.eps, ldist) ? 0.0f : 1.0f;
    if (V > 0.0f) {
      F3 Li = V * radiance;
      F3 e;
      if (m.model == MULTISCATTERING) {
        F3 lwi = to_local(w_i, ffnormal), lwl = to_local(w_l, ffnormal);
        F3 diffuse_brdf = ms_diffuse_eval<float>(dist, lwi, lwl, a_x, a_y, t, dc, 0u, 4096, &capped);
        e = Li * diffuse_brdf;
        F3 reflected_brdf = ms_conductor_eval<float>(dist, lwi, lwl, m.eta, m.inv_eta, a_x, a_y, t, 0u, 4096, &capped);
        e = e + Li * reflected_brdf;
      } else {
        F3 refl_normal = normalize(w_i + w_l);
        float R_refl = interface_R(dot(refl_normal, w_l), n1_over_n2);
        float T_01_diff = 1.0f - interface_R(dot(microfacet_normal, w_l), n1_over_n2);
        float G_i_m_refl = masking_G1_aniso<float>(dist, w_i, refl_normal, ffnormal, a_x, a_y);
        float G_o_m_refl = masking_G1_aniso<float>(dist, w_l, refl_normal, ffnormal, a_x, a_y);
        float G_o_m_diff = masking_G1_aniso<float>(dist, w_l, microfacet_normal, ffnormal, a_x, a_y);
        float D_refl = eval_visible_normal<float>(dist, w_i, refl_normal, ffnormal, a_x, a_y);
        float weight_refl = G_i_m_refl * G_o_m_refl * D_refl / (4.0f * std::fabs(dot(w_i, ffnormal) * dot(w_l, ffnormal)));
        float weight_diff = G_o_m_diff;
        e = Li * K<float>::INV_PI * cos_theta_l * dc * n1_over_n2 * n1_over_n2 * T_01_i * T_01_diff / (1.0f - dc * r_10) * weight_diff;
        e = e + Li * R_refl * weight_refl;
      }
      result = result + e;
      tape_emit(prd, e);
      prd.emit_light = 0;
    }
  }
  // indirect illumination (:181-289)
  float prob = R_i;
  float xi = rnd_tea(t);
  F3 w_o;
  if (xi > prob) {
    if (m.model == MULTISCATTERING) {
      u32 order = 0;
      F3 w_m = v3(0.0f, 0.0f, 1.0f), weight;
      F3 lwo = ms_diffuse_sample<float>(dist, to_local(w_i, ffnormal), w_m, a_x, a_y, t, order, weight, dc);
      w_o = to_world(lwo, ffnormal);
      w_m = to_world(w_m, ffnormal);
      float T_01_r = 1.0f - interface_R(dot(w_o, w_m), n1_over_n2);
      PRD child = child_of(prd, prd.emit_light);
      const int slot = tape_add(prd, TapeRec());
      trace(S, hit_pos, w_o, child, ls);
      tape_const_w(prd, slot, n1_over_n2 * n1_over_n2 * T_01_r / (1.0f - dc * r_10) * weight);
      result = result + child.result * n1_over_n2 * n1_over_n2 * T_01_r / (1.0f - dc * r_10) * weight;
      prd.seed = child.seed;
    } else {
      F3 diffuse_dir = sample_cosine_weighted<float>(microfacet_normal, t);
      float cos_theta_r = dot(diffuse_dir, microfacet_normal);
      float G_o_m = masking_G1_aniso<float>(dist, diffuse_dir, microfacet_normal, ffnormal, a_x, a_y);
      if (G_o_m < 0.0f) { prd.result = result; S.capped += capped; return; }
      float T_01_r = 1.0f - interface_R(cos_theta_r, n1_over_n2);
      PRD child = child_of(prd, prd.emit_light);
      const int slot = tape_add(prd, TapeRec());
      trace(S, hit_pos, diffuse_dir, child, ls);
      tape_const_w(prd, slot, dc * n1_over_n2 * n1_over_n2 * T_01_r / (1.0f - dc * r_10) * G_o_m);
      result = result + child.result * dc * n1_over_n2 * n1_over_n2 * T_01_r / (1.0f - dc * r_10) * G_o_m;
      prd.seed = child.seed;
    }
  } else {
    if (m.model == MULTISCATTERING) {
      u32 order = 10;
      F3 w_m, weight;
      F3 lwo = ms_conductor_sample<float>(dist, to_local(w_i, normal), w_m, m.eta, m.inv_eta, a_x, a_y, t, order, weight, 4096, &capped);
      w_o = to_world(lwo, normal);
      PRD child = child_of(prd, prd.emit_light);
      tape_const_w(prd, tape_add(prd, TapeRec()), v3s(1.0f));
      trace(S, hit_pos, w_o, child, ls);
      result = result + child.result;
      prd.seed = child.seed;
    } else {
      F3 refl_dir = reflect(d, microfacet_normal);
      float G_o_m = masking_G1_aniso<float>(dist, refl_dir, microfacet_normal, ffnormal, a_x, a_y);
      if (G_o_m < 0.0f) { prd.result = result; S.capped += capped; return; }
      PRD child = child_of(prd, prd.emit_light);
      tape_const_w(prd, tape_add(prd, TapeRec()), v3s(G_o_m));
      trace(S, hit_pos, refl_dir, child, ls);
      result = result + child.result * G_o_m;
      prd.seed = child.seed;
    }
  }
  S.capped += capped;
  prd.result = result;
}

// subsurface_scattering_shader.cu:55-201 (REFLECT, TRANSMIT and RND_64 defined).
static void shade_translucent(Scene& S, const Mat& m, const F3& o, const F3& d, const HitRec& h, PRD& prd, LightSet& ls)
{
  prd.result = v3s(0.0f);
  if (prd.depth > S.max_depth) return;
  F3 no = shading_normal(S, h.prim, h.u, h.v);
  F3 xo = o + h.t * d;
  F3 wo = -d;
  const ScatProps& P = m.props;
  float recip_ior = 1.0f / P.relative_ior;
  F3 beam_T = v3s(1.0f);
  u32& t = prd.seed;
  Seed64& t64 = prd.seed64;
  float reflect_xi = rnd_accurate(t64);
  float cos_theta_o = dot(wo, no);
  bool inside = cos_theta_o < 0.0f;
  if (inside) {
    const F3& ext = (m.dipole_model == DIRECTIONAL_DIPOLE) ? P.deltaEddExtinction : P.extinction;
    beam_T = vexp((-h.t) * ext);
    float prob = (beam_T.x + beam_T.y + beam_T.z) / 3.0f;
    if (rnd_accurate(t64) >= prob) return;
    beam_T = beam_T / prob;
    if (prd.tape) {
      TapeRec r;
      r.type = TAPE_BEER;
      r.mat = (int)(&m - S.mats.data());
      r.c[0] = h.t;
      r.c[1] = prob;
      r.v[0] = beam_T.x; r.v[1] = beam_T.y; r.v[2] = beam_T.z;
      tape_add(prd, r);
    }
    recip_ior = P.relative_ior;
    no = -no;
    cos_theta_o = -cos_theta_o;
  }
  float sin_theta_t_sqr = recip_ior * recip_ior * (1.0f - cos_theta_o * cos_theta_o);
  float cos_theta_t = 1.0f, R = 1.0f;
  if (sin_theta_t_sqr < 1.0f) {
    cos_theta_t = std::sqrt(1.0f - sin_theta_t_sqr);
    R = fresnel_R(cos_theta_o, cos_theta_t, recip_ior);
  }
  if (reflect_xi >= R) {
    F3 wt = recip_ior * (cos_theta_o * no - wo) - no * cos_theta_t;
    PRD child;
    child.depth = prd.depth + 1;
    child.seed64 = t64;
    child.seed = t;
    child.result = v3s(0.0f);
    child.emit_light = 1;
    child.probe_path = prd.probe_path;
    child.tape = prd.tape;
    const int gslot = (!inside && !prd.probe_path) ? tape_add(prd, TapeRec()) : -1;
    trace(S, xo, wt, child, ls);
    prd.result = prd.result + child.result;
    t = child.seed;
    t64 = child.seed64;
    if (!inside && !prd.probe_path) {
      if (gslot >= 0) {
        TapeRec& r = prd.tape->recs[gslot];
        r.type = TAPE_GATHER;
        r.mat = (int)(&m - S.mats.data());
        r.g_begin = (int)prd.tape->probes.size();
      }
      float chosen = std::fmin(P.transport.x, std::fmin(P.transport.y, P.transport.z));
      F3 acc = v3s(0.0f);
      unsigned N = S.samples;
      const Probe* pr = S.probes.data() + (size_t)m.translucent_index * N;
      for (unsigned i = 0; i < N; ++i) {
        const Probe& sm = pr[i];
        if (dot(sm.L, sm.L) > 0.0f) {
          float dist = length(xo - sm.pos);
          float exp_term = std::exp(-dist * chosen);
          float rnd_number = rnd_accurate(t64);
          if (rnd_number < exp_term) {
            if (gslot >= 0) {
              F3 wl = sm.weight * sm.L;
              prd.tape->probes.push_back(TapeProbe{dist, {wl.x, wl.y, wl.z}, exp_term});
              prd.tape->recs[gslot].g_count += 1;
            }
            if (m.dipole_model == DIRECTIONAL_DIPOLE)
              acc = acc + sm.weight * sm.L * dirpole_bssrdf(sm.pos, sm.normal, sm.transmitted, xo, no, P) / exp_term;
            else
              acc = acc + sm.weight * sm.L * dipole_bssrdf(dist, P) / exp_term;
          }
        }
      }
      prd.result = prd.result + acc * P.global_coeff / (float)N;
    }
  }
  if (reflect_xi < R) {
    F3 wr = 2.0f * cos_theta_o * no - wo;
    PRD child;
    child.depth = prd.depth + 1;
    child.seed = t;
    child.seed64 = t64;
    child.result = v3s(0.0f);
    child.emit_light = 1;
    child.probe_path = prd.probe_path;
    child.tape = prd.tape;
    trace(S, xo, wr, child, ls);
    prd.result = prd.result + child.result;
    t = child.seed;
    t64 = child.seed64;
  }
  prd.result = prd.result * beam_T;
}

// The dipole gather of a translucent entry vertex (subsurface_scattering_shader.cu:126-173 and the rough
// variant rough_subsurface_scattering_shader.cu:240-283,384-427, where a draw must also exceed 0.001
// and every term is multiplied by the refraction weight).
static F3 dipole_gather(Scene& S, const Mat& m, const F3& xo, const F3& no, Seed64& t64, bool rough, const F3& weight)
{
  const ScatProps& P = m.props;
  float chosen = std::fmin(P.transport.x, std::fmin(P.transport.y, P.transport.z));
  F3 acc = v3s(0.0f);
  unsigned N = S.samples;
  const Probe* pr = S.probes.data() + (size_t)m.translucent_index * N;
  for (unsigned i = 0; i < N; ++i) {
    const Probe& sm = pr[i];
    if (dot(sm.L, sm.L) > 0.0f) {
      float dist = length(xo - sm.pos);
      float exp_term = std::exp(-dist * chosen);
      float rnd_number = rnd_accurate(t64);
      if (rnd_number < exp_term && (!rough || rnd_number > 0.001f)) {
        F3 term = (m.dipole_model == DIRECTIONAL_DIPOLE) ? sm.weight * sm.L * dirpole_bssrdf(sm.pos, sm.normal, sm.transmitted, xo, no, P) / exp_term
                                                        : sm.weight * sm.L * dipole_bssrdf(dist, P) / exp_term;
        acc = acc + (rough ? term * weight : term);
      }
    }
  }
  return acc * P.global_coeff / (float)N;
}

// rough_subsurface_scattering_shader.cu:56-455 (REFLECT, TRANSMIT, DIRECTLIGHT and RND_64 defined):
// microfacet normal from MD5 draws, a light sample with its reflection-only estimate (the multiscatter
// model: the multiscatter dielectric BSDF), then as the smooth shader with the microfacet normal in
// the Fresnel choice and the refraction / reflection weight on the child (and on the gather).
static void shade_rough_translucent(Scene& S, const Mat& m, const F3& o, const F3& d, const HitRec& h, PRD& prd, LightSet& ls)
{
  prd.result = v3s(0.0f);
  if (prd.depth > S.max_depth) return;
  F3 result = v3s(0.0f);
  F3 normal = shading_normal(S, h.prim, h.u, h.v);
  F3 ffnormal = faceforward(normal, -d, normal);
  F3 hit_pos = o + h.t * d;
  F3 w_i = -d;
  const ScatProps& P = m.props;
  float recip_ior = 1.0f / P.relative_ior;
  F3 beam_T = v3s(1.0f);
  u32& t = prd.seed;
  Seed64& t64 = prd.seed64;
  float reflect_xi = rnd_accurate(t64);
  float z1 = rnd_accurate(t64);
  float z2 = rnd_accurate(t64);
  const float a_x = m.a[0], a_y = m.a[1];
  const int dist = (int)m.dist;
  int capped = 0;
  F3 mn = (m.model == WALTER) ? sample_normal<float>(dist, ffnormal, z1, z2, a_x)
                              : sample_visible_normal<float>(dist, w_i, ffnormal, a_x, a_y, z1, z2, &capped);
  float cos_theta_i = dot(w_i, mn);
  bool inside = dot(w_i, normal) < 0.0f;
  // light sample (:93-152)
  u32 li = (u32)((float)ls.n_lights * rnd_accurate(t64));
  if ((long)li >= ls.n_lights) { li = (u32)(ls.n_lights - 1); ++ls.oob; }
  float light_pdf = 1.0f / (float)ls.n_lights;
  float ldist = 0.0f;
  F3 light_radiance = v3s(0.0f), w_l = v3s(0.0f);
  eval_direct<float>(hit_pos, ls.lights[li], ls, w_l, light_radiance, ldist, t);
  light_radiance = light_radiance / light_pdf;
  float cos_theta_l = dot(ffnormal, w_l);
  if (!inside && cos_theta_l > 0.0f) {
    float V = occluded(S, hit_pos, w_l, S.eps, ldist) ? 0.0f : 1.0f;
    if (V > 0.0f) {
      F3 Li = V * light_radiance;
      F3 e;
      if (m.model == MULTISCATTERING) {
        float brdf = ms_dielectric_eval<float>(dist, to_local(w_i, ffnormal), to_local(w_l, ffnormal), recip_ior, a_x, a_y, t, 0, 4096, &capped);
        e = Li * brdf;
        prd.emit_light = 0;
      } else {
        F3 refl_normal = normalize(w_i + w_l);
        float cos_refl = dot(refl_normal, w_l);
        float R_refl = 1.0f;
        float st2 = recip_ior * recip_ior * (1.0f - cos_refl * cos_refl);
        if (st2 < 1.0f) R_refl = fresnel_R(cos_refl, std::sqrt(1.0f - st2), recip_ior);
        float G_i = masking_G1_aniso<float>(dist, w_i, refl_normal, ffnormal, a_x, a_y);
        float G_o = masking_G1_aniso<float>(dist, w_l, refl_normal, ffnormal, a_x, a_y);
        float D = eval_visible_normal<float>(dist, w_i, refl_normal, ffnormal, a_x, a_y);
        float weight_refl = G_i * G_o * D / (4.0f * std::fabs(dot(w_i, ffnormal) * dot(w_l, ffnormal)));
        e = Li * R_refl * weight_refl;
        prd.emit_light = 1;
      }
      result = result + e;
      tape_emit(prd, e);
    }
  }
  if (m.model == WALTER || m.model == VISIBLE_NORMALS) {
    if (inside) {
      const F3& ext = (m.dipole_model == DIRECTIONAL_DIPOLE) ? P.deltaEddExtinction : P.extinction;
      beam_T = vexp((-h.t) * ext);
      float prob = (beam_T.x + beam_T.y + beam_T.z) / 3.0f;
      if (rnd_accurate(t64) >= prob) { S.capped += capped; return; }
      beam_T = beam_T / prob;
      recip_ior = P.relative_ior;
      normal = -normal;
    }
    float st2 = recip_ior * recip_ior * (1.0f - cos_theta_i * cos_theta_i);
    float cos_t = 1.0f, R = 1.0f;
    if (st2 < 1.0f) {
      cos_t = std::sqrt(1.0f - st2);
      R = fresnel_R(cos_theta_i, cos_t, recip_ior);
    }
    auto child_weight = [&](const F3& w_o) {
      if (m.model == WALTER) {
        float G_i_m = masking_G1<float>(dist, w_i, mn, ffnormal, a_x);
        float abs_i_m = std::fabs(dot(w_i, mn)), abs_i_n = std::fabs(dot(w_i, ffnormal)), abs_n_m = std::fabs(dot(ffnormal, mn));
        float G_o_m = masking_G1<float>(dist, w_o, mn, ffnormal, a_x);
        return v3s(1.0f) * (abs_i_m * G_i_m * G_o_m / (abs_i_n * abs_n_m));
      }
      return v3s(1.0f) * masking_G1_aniso<float>(dist, w_o, mn, ffnormal, a_x, a_y);
    };
    if (reflect_xi >= R) {
      F3 w_t = recip_ior * (cos_theta_i * mn - w_i) - mn * cos_t;
      PRD child;
      child.depth = prd.depth + 1;
      child.seed = t;
      child.seed64 = t64;
      child.result = v3s(0.0f);
      child.emit_light = 1;
      child.probe_path = prd.probe_path;
      child.tape = prd.tape;
      trace(S, hit_pos, w_t, child, ls);
      F3 weight = child_weight(w_t);
      result = result + child.result * weight;
      t = child.seed;
      t64 = child.seed64;
      if (!inside && !prd.probe_path) result = result + dipole_gather(S, m, hit_pos, normal, t64, true, weight);
    }
    if (reflect_xi < R) {
      F3 w_r = 2.0f * cos_theta_i * mn - w_i;
      PRD child;
      child.depth = prd.depth + 1;
      child.seed = t;
      child.seed64 = t64;
      child.result = v3s(0.0f);
      child.emit_light = prd.emit_light;
      child.probe_path = prd.probe_path;
      child.tape = prd.tape;
      trace(S, hit_pos, w_r, child, ls);
      F3 weight = child_weight(w_r);
      result = result + child.result * weight;
      t = child.seed;
      t64 = child.seed64;
    }
  } else {  // MULTISCATTERING_MODEL (:287-452)
    u32 order = 0;
    F3 w_o = to_world(ms_dielectric_sample<float>(dist, to_local(w_i, normal), 1.0f / P.relative_ior, a_x, a_y, t, order, 4096, &capped), normal);
    const F3 weight = v3s(1.0f);
    bool is_refraction = dot(w_o, ffnormal) < 0.0f;
    if (inside) {
      const F3& ext = (m.dipole_model == DIRECTIONAL_DIPOLE) ? P.deltaEddExtinction : P.extinction;
      beam_T = vexp((-h.t) * ext);
      float prob = (beam_T.x + beam_T.y + beam_T.z) / 3.0f;
      if (rnd_accurate(t64) >= prob) { S.capped += capped; return; }
      beam_T = beam_T / prob;
      recip_ior = P.relative_ior;
      normal = -normal;
    }
    PRD child;
    child.depth = prd.depth + 1;
    child.result = v3s(0.0f);
    child.seed = t;
    child.emit_light = 1;
    child.seed64 = t64;
    child.probe_path = prd.probe_path;
    child.tape = prd.tape;
    trace(S, hit_pos, w_o, child, ls);
    result = result + child.result * weight;
    t = child.seed;
    t64 = child.seed64;
    if (is_refraction && !inside && !prd.probe_path) result = result + dipole_gather(S, m, hit_pos, normal, t64, true, weight);
  }
  S.capped += capped;
  prd.result = result * beam_T;
}

// sample_camera.cu:48-268 for a smooth translucent object (GLOBAL and RND_64 defined): one
// PositionSample per launch index of the probe pass of translucent object k.
static Probe make_probe(Scene& S, unsigned k, unsigned i, unsigned frame, LightSet& ls)
{
  const TranslucentObject& T = S.translucent[k];
  const Mat& m = S.mats[T.material];
  unsigned idx = i + k * S.samples;
  Probe sm;
  memset(&sm, 0, sizeof(sm));
  u32 triangles = T.n_tris;
  u32 t = tea<16>(idx, frame);
  u32 s2 = tea<16>(idx, frame);
  Seed64 t64 = {s2, s2};
  u32 tid = (u32)(int)(rnd_accurate(t64) * (float)triangles);
  if (tid >= triangles) { tid = triangles - 1; ++ls.oob; }
  unsigned prim = T.first_tri + tid;
  const float* pv = &S.pos9[9 * (size_t)prim];
  F3 v0 = v3(pv[0], pv[1], pv[2]), v1 = v3(pv[3], pv[4], pv[5]), v2 = v3(pv[6], pv[7], pv[8]);
  F3 perp = cross(v1 - v0, v2 - v0);
  float area = 0.5f * length(perp);
  float xi1 = std::sqrt(rnd_accurate(t64));
  float xi2 = rnd_accurate(t64);
  float u = 1.0f - xi1, v = (1.0f - xi2) * xi1, w = xi1 * xi2;
  sm.pos = u * v0 + v * v1 + w * v2;
  const int* in = &S.info[4 * (size_t)prim];
  F3 n;
  if (in[0] >= 0) {
    n = normalize(u * S.normals[in[0]] + v * S.normals[in[1]] + w * S.normals[in[2]]);
    n = normalize(n);
  } else {
    n = normalize(perp);
  }
  sm.normal = n;
  float recip_ior = 1.0f / m.props.relative_ior;
  const bool rough = m.type == MT_ROUGH_TRANSLUCENT;
  const float a_x = m.a[0], a_y = m.a[1];
  int capped = 0;
  // rough objects: the probe's normal is a microfacet normal sampled with two MD5 draws (:130-151)
  auto microfacet = [&](const F3& wdir) {
    float z1 = rnd_accurate(t64);
    float z2 = rnd_accurate(t64);
    sm.normal = (m.model == WALTER) ? sample_normal<float>((int)m.dist, n, z1, z2, a_x)
                                    : sample_visible_normal<float>((int)m.dist, wdir, n, a_x, a_y, z1, z2, &capped);
  };
  F3 Le, w_i;
  if (rnd(t) < 0.5f) {
    u32 li = (u32)((float)ls.n_lights * rnd_accurate(t64));
    if ((long)li >= ls.n_lights) { li = (u32)(ls.n_lights - 1); ++ls.oob; }
    float light_pdf = 1.0f / (float)ls.n_lights;
    float r = 0.0f;
    Le = v3s(0.0f);
    w_i = v3s(0.0f);
    eval_direct<float>(sm.pos, ls.lights[li], ls, w_i, Le, r, t);
    sm.dir = w_i;
    if (rough) microfacet(w_i);
    float cos_theta_i = std::fmax(dot(w_i, n), 0.0f);
    if (cos_theta_i > 0.0f) {
      float att = occluded(S, sm.pos, w_i, S.eps, r) ? 0.0f : 1.0f;
      Le = Le * (att * cos_theta_i / light_pdf);
    } else {
      Le = v3s(0.0f);
    }
  } else {
    w_i = sample_cosine_weighted<float>(n, t);
    if (rough) microfacet(w_i);
    PRD pn;
    pn.depth = 0;
    pn.seed = t;
    pn.seed64 = t64;
    pn.result = v3s(0.0f);
    pn.emit_light = 1;
    pn.probe_path = true;
    trace(S, sm.pos, w_i, pn, ls);
    t = pn.seed;
    t64 = pn.seed64;
    Le = pn.result * K<float>::PI;
  }
  Le = Le / 0.5f;
  float cos_theta_i = std::fmax(dot(w_i, sm.normal), 0.0f);
  float cos_i2 = cos_theta_i * cos_theta_i;
  float sin_t2 = recip_ior * recip_ior * (1.0f - cos_i2);
  float cos_t = std::sqrt(1.0f - sin_t2);
  sm.transmitted = recip_ior * (cos_theta_i * sm.normal - w_i) - sm.normal * cos_t;
  float T12 = 1.0f - fresnel_R(cos_theta_i, cos_t, recip_ior);
  F3 weight = v3s(1.0f);
  if (rough) {  // :232-266
    const int dist = (int)m.dist;
    if (m.model == WALTER) {
      float G_i_m = masking_G1_aniso<float>(dist, w_i, sm.normal, n, a_x, a_y);
      float abs_i_m = std::fabs(dot(w_i, sm.normal)), abs_i_n = std::fabs(dot(w_i, n)), abs_n_m = std::fabs(dot(n, sm.normal));
      float G_o_m = masking_G1_aniso<float>(dist, sm.transmitted, sm.normal, n, a_x, a_y);
      weight = weight * (abs_i_m * G_i_m / (abs_i_n * abs_n_m) * G_o_m);
      weight = weight * v3s(T12);
    } else if (m.model == VISIBLE_NORMALS) {
      float G_o_m = masking_G1_aniso<float>(dist, sm.transmitted, sm.normal, n, a_x, a_y);
      weight = weight * G_o_m;
      weight = weight * v3s(T12);
    } else {
      weight = weight * v3s(T12);
    }
  } else {
    weight = weight * v3s(T12);
  }
  sm.weight = weight;
  sm.L = Le * ((float)triangles * area);
  return sm;
}

static void trace(Scene& S, const F3& o, const F3& d, PRD& prd, LightSet& ls)
{
  HitRec h = closest(S, o, d, S.eps, DEFAULT_MAX);
  if (h.prim < 0) {  // constantbg.cu:16-19 / envmap_background.cu:20-23
    if (S.env_present) {
      if (S.env_is_light && !prd.emit_light) prd.result = v3s(0.0f);
      else prd.result = env_lookup(S.env, d);
    } else {
      prd.result = S.bg;
    }
    tape_emit(prd, prd.result);
    return;
  }
  if ((size_t)h.prim >= S.tris.size()) {  // a disk or sphere light: arealight_shader.cu:36-50 on its geometry
    const Scene::Ana& A = S.ana[h.prim - S.tris.size()];
    F3 normal = A.kind == DISK_LIGHT ? A.normal : ((o - A.pos) + h.t * d) / A.radius;  // disk_mesh.cu:47, sphere_mesh.cu:78,87
    normal = normalize(normal);
    F3 result = v3s(0.0f);
    if (dot(normal, -d) > 0.0f && prd.emit_light) result = A.radiance;
    prd.result = result;
    tape_emit(prd, result);
    return;
  }
  const Mat& m = S.mats[S.info[4 * (size_t)h.prim + 3]];
  switch (m.type) {
    case MT_LIGHT: {  // arealight_shader.cu:36-50
      F3 normal = shading_normal(S, h.prim, h.u, h.v);
      F3 result = v3s(0.0f);
      if (dot(normal, -d) > 0.0f && prd.emit_light) result = v3(m.a[0], m.a[1], m.a[2]);
      prd.result = result;
      tape_emit(prd, result);
      return;
    }
    case MT_DIFFUSE: shade_diffuse(S, m, o, d, h, prd, ls); return;
    case MT_METAL: shade_metal(S, m, o, d, h, prd, ls); return;
    case MT_GLASS: shade_glass(S, m, o, d, h, prd, ls); return;
    case MT_TRANSPARENT: shade_transparent(S, m, o, d, h, prd, ls); return;
    case MT_LAMBERTIAN_INTERFACE: shade_lambertian_interface(S, m, o, d, h, prd, ls); return;
    case MT_ROUGH_DIFFUSE: shade_rough_diffuse(S, m, o, d, h, prd, ls); return;
    case MT_TRANSLUCENT: shade_translucent(S, m, o, d, h, prd, ls); return;
    case MT_ROUGH_TRANSLUCENT: shade_rough_translucent(S, m, o, d, h, prd, ls); return;
    default: prd.result = v3s(0.0f); return;
  }
}

}  // namespace

// Scene handle for the C interface.
EXPORT void* orc_scene_create(const float* tri_pos, const int* tri_info, unsigned n_tris, const float* normals, unsigned n_normals,
                              const unsigned* mat_type, const unsigned* mat_model, const unsigned* mat_dist, const float* mat_ab,
                              const double* mat_ior, unsigned n_mats, const void* lights, unsigned n_lights, const void* tri_lights,
                              unsigned n_tri_lights, const float* cam12, unsigned width, unsigned height, const unsigned* patch4,
                              int max_depth, float eps, int rr_start, const float* bg3)
{
  Scene* S = new Scene();
  S->pos9.assign(tri_pos, tri_pos + 9 * (size_t)n_tris);
  S->tris.resize(n_tris);
  for (unsigned i = 0; i < n_tris; ++i) {
    const float* p = tri_pos + 9 * (size_t)i;
    F3 v0 = v3(p[0], p[1], p[2]), v1 = v3(p[3], p[4], p[5]), v2 = v3(p[6], p[7], p[8]);
    S->tris[i] = {v0, v1 - v0, v2 - v0};
  }
  S->info.assign(tri_info, tri_info + 4 * (size_t)n_tris);
  for (unsigned k = 0; k < n_normals; ++k) S->normals.push_back(v3(normals[3 * k], normals[3 * k + 1], normals[3 * k + 2]));
  for (unsigned k = 0; k < n_mats; ++k) {
    Mat m = Mat();  // zero-initialised, then the member defaults
    m.type = mat_type[k];
    m.model = mat_model[k];
    m.dist = mat_dist[k];
    memcpy(m.a, mat_ab + 8 * (size_t)k, 16);
    memcpy(m.b, mat_ab + 8 * (size_t)k + 4, 16);
    if (m.type == MT_METAL) {
      const double* io = mat_ior + 6 * (size_t)k;
      Cx3 ior = {{io[0], io[1]}, {io[2], io[3]}, {io[4], io[5]}};
      m.eta = crecip3<float>(ior);       // eta = n1 / ior, metallic_shader.cu:61
      m.inv_eta = crecip3<float>(m.eta);
    }
    if (m.type == MT_ROUGH_DIFFUSE) {  // MyComplex{ n1_over_n2, 0 } per channel, rough_diffuse_shader.cu:132-133
      const double e = (double)(1.0f / m.a[3]);
      m.eta = {{e, 0.0}, {e, 0.0}, {e, 0.0}};
      m.inv_eta = crecip3<float>(m.eta);
    }
    S->mats.push_back(m);
  }
  S->lights.lights = (const LightStructRaw*)lights;
  S->lights.n_lights = n_lights;
  for (unsigned k = 0; k < n_lights; ++k) {
    const LightStructRaw& l = ((const LightStructRaw*)lights)[k];
    if (l.light_type != DISK_LIGHT && l.light_type != SPHERICAL_LIGHT) continue;
    Scene::Ana A;
    A.kind = (int)l.light_type;
    A.pos = v3(l.p[0], l.p[1], l.p[2]);
    A.radius = l.pad[0];  // DiskLightStruct / SphericalLightStruct radius, structs.h:76-93
    A.normal = v3(0.0f, 1.0f, 0.0f);
    if (A.kind == DISK_LIGHT) {  // DiskAreaLight::computeNormal, Light.cpp:469-474 (theta = pad[2], phi = pad[1], degrees)
      float t_rad = l.pad[2] * K<float>::PI / 180.0f;
      float p_rad = l.pad[1] * K<float>::PI / 180.0f;
      A.normal = v3(std::sin(t_rad) * std::sin(p_rad), std::cos(t_rad), std::sin(t_rad) * std::cos(p_rad));
    }
    A.radiance = v3(l.emitted[0], l.emitted[1], l.emitted[2]);
    S->ana.push_back(A);
  }
  S->lights.tris = (const TriangleLightRaw*)tri_lights;
  S->lights.n_tris = n_tri_lights;
  S->eye = v3(cam12[0], cam12[1], cam12[2]);
  S->U = v3(cam12[3], cam12[4], cam12[5]);
  S->V = v3(cam12[6], cam12[7], cam12[8]);
  S->W = v3(cam12[9], cam12[10], cam12[11]);
  S->width = width;
  S->height = height;
  S->po_x = patch4[0]; S->po_y = patch4[1]; S->pd_x = patch4[2]; S->pd_y = patch4[3];
  S->max_depth = max_depth;
  S->eps = eps;
  S->rr_start = rr_start;
  S->bg = v3(bg3[0], bg3[1], bg3[2]);
  build_bvh(*S);
  return S;
}

EXPORT void orc_scene_destroy(void* s) { delete (Scene*)s; }

// EnvMapBackground for the scene: copies the float4 texels and builds the CDF tables.
EXPORT void orc_scene_set_env(void* s, const float* rgba, int w, int h)
{
  Scene& S = *(Scene*)s;
  S.env_texels.assign(rgba, rgba + 4 * (size_t)w * h);
  S.env.rgba = S.env_texels.data();
  S.env.w = w;
  S.env.h = h;
  env_build_cdf(S.env);
  S.env_present = true;
  S.env_is_light = false;
  for (long k = 0; k < S.lights.n_lights; ++k)
    if (S.lights.lights[k].light_type == ENVMAP_LIGHT) S.env_is_light = true;
}
EXPORT void orc_env_tables(void* s, float* mpdf, float* mcdf, float* cpdf, float* ccdf)
{
  const EnvMap& E = ((Scene*)s)->env;
  memcpy(mpdf, E.marginal_pdf.data(), 4 * (size_t)E.h);
  memcpy(mcdf, E.marginal_cdf.data(), 4 * (size_t)E.h);
  memcpy(cpdf, E.conditional_pdf.data(), 4 * (size_t)E.w * E.h);
  memcpy(ccdf, E.conditional_cdf.data(), 4 * (size_t)E.w * E.h);
}
// Batch env queries: lookups of dirs3[n] and importance samples from seeds[n] (seeds advanced).
EXPORT void orc_env_query(void* s, const float* dirs3, long n_dirs, float* looked3, unsigned* seeds, long n_samples, float* sdir3, float* sL3)
{
  const EnvMap& E = ((Scene*)s)->env;
  for (long i = 0; i < n_dirs; ++i) {
    F3 r = env_lookup(E, v3(dirs3[3 * i], dirs3[3 * i + 1], dirs3[3 * i + 2]));
    looked3[3 * i] = r.x; looked3[3 * i + 1] = r.y; looked3[3 * i + 2] = r.z;
  }
  for (long i = 0; i < n_samples; ++i) {
    u32 t = seeds[i];
    F3 d, L;
    sample_environment(E, d, L, t);
    seeds[i] = t;
    sdir3[3 * i] = d.x; sdir3[3 * i + 1] = d.y; sdir3[3 * i + 2] = d.z;
    sL3[3 * i] = L.x; sL3[3 * i + 1] = L.y; sL3[3 * i + 2] = L.z;
  }
}

// Renders frames [first_frame, first_frame + n_frames) for pixels [p_begin, p_end) with `threads`
// host threads, frame by frame: the probe pass of every translucent object (sample_camera.cu) and
// then the integrator pass (path_tracer.cu), as OptixScene::renderScene launches them
// (OptixScene.cpp:146-159).  path_rad (optional): radiance of every path, [frame][pixel][3] over the
// pixel range.  accum (optional): the float4 running mean over the full image (path_tracer.cu:64-68).
// The light arrays passed to orc_scene_create must outlive the scene.
EXPORT long orc_render(void* scene, unsigned first_frame, unsigned n_frames, unsigned p_begin, unsigned p_end, float* path_rad, float* accum,
                       int threads)
{
  Scene& S = *(Scene*)scene;
  const unsigned W = S.width, H = S.height;
  p_end = std::min(p_end, W * H);
  if (p_begin >= p_end) return 0;
  threads = std::max(1, threads);
  std::atomic<long> oob(0);
  auto parallel = [&](unsigned count, unsigned chunk, auto&& body) {
    std::atomic<unsigned> next(0);
    auto worker = [&]() {
      LightSet ls = S.lights;
      ls.env = S.env_present ? &S.env : nullptr;
      ls.oob = 0;
      for (;;) {
        unsigned b = next.fetch_add(chunk);
        if (b >= count) break;
        unsigned e = std::min(count, b + chunk);
        for (unsigned k = b; k < e; ++k) body(k, ls);
      }
      oob += ls.oob;
    };
    std::vector<std::thread> th;
    for (int i = 1; i < threads; ++i) th.emplace_back(worker);
    worker();
    for (auto& x : th) x.join();
  };
  if (S.record) {
    S.tapes.assign((size_t)n_frames * (p_end - p_begin), Tape());
    S.tape_first = first_frame;
    S.tape_frames = n_frames;
    S.tape_p0 = p_begin;
    S.tape_p1 = p_end;
  }
  for (unsigned fl = 0; fl < n_frames; ++fl) {
    const unsigned frame = first_frame + fl;
    if (!S.translucent.empty()) {
      S.probes.assign((size_t)S.samples * S.translucent.size(), Probe());
      unsigned total = S.samples * (unsigned)S.translucent.size();
      parallel(total, 16, [&](unsigned j, LightSet& ls) { S.probes[j] = make_probe(S, j / S.samples, j % S.samples, frame, ls); });
      S.probe_frame = frame;
    }
    parallel(p_end - p_begin, 64, [&](unsigned k, LightSet& ls) {
      unsigned p = p_begin + k;
      unsigned x = p % W, y = p / W;
      bool inside = !(x < S.po_x || x > S.po_x + S.pd_x || y < S.po_y || y > S.po_y + S.pd_y);
      F3 result = v3s(0.0f);
      if (inside) {
        PRD prd;
        prd.emit_light = 1;
        prd.depth = 0;
        prd.seed = tea<16>(W * y + x, frame);
        u32 s2 = tea<16>(W * y + x, frame);
        prd.seed64 = {s2, s2};
        float jx = rnd_tea(prd.seed), jy = rnd_tea(prd.seed);
        float ipx = ((float)x + jx) / (float)W * 2.0f - 1.0f;
        float ipy = ((float)y + jy) / (float)H * 2.0f - 1.0f;
        F3 dir = normalize(ipx * S.U + ipy * S.V + S.W);
        prd.result = v3s(0.0f);
        if (S.record) prd.tape = &S.tapes[(size_t)fl * (p_end - p_begin) + k];
        trace(S, S.eye, dir, prd, ls);
        result = result + prd.result;
        if (prd.tape) prd.tape->valid = std::isfinite(result.x) && std::isfinite(result.y) && std::isfinite(result.z);
      }
      if (path_rad) {
        float* pr = path_rad + 3 * ((size_t)fl * (p_end - p_begin) + k);
        pr[0] = result.x; pr[1] = result.y; pr[2] = result.z;
      }
      if (accum) {
        float* out = accum + 4 * (size_t)p;
        if (!inside) {
          out[0] = out[1] = out[2] = 0.0f;
          out[3] = 1.0f;
        } else if (std::isfinite(result.x) && std::isfinite(result.y) && std::isfinite(result.z)) {
          float cur[4] = {0, 0, 0, 0};
          if (frame != 0)
            for (int q = 0; q < 4; ++q) cur[q] = out[q] * (float)frame;
          float den = (float)(frame + 1);
          out[0] = (result.x + cur[0]) / den;
          out[1] = (result.y + cur[1]) / den;
          out[2] = (result.z + cur[2]) / den;
          out[3] = (1.0f + cur[3]) / den;
        }
      }
    });
  }
  return oob.load();
}

// Translucent material `mat` (scattering_properties as the 260-byte ScatteringMaterialProperties and
// dipole_model) and the translucent objects: meshes [first_tri, first_tri + n_tris) with their probe
// sets in object order (translucent_index).
EXPORT void orc_scene_set_translucent(void* s, unsigned mat, const void* props260, unsigned dipole_model)
{
  Scene& S = *(Scene*)s;
  memcpy(&S.mats[mat].props, props260, sizeof(ScatProps));
  S.mats[mat].dipole_model = dipole_model;
}
EXPORT void orc_scene_add_translucent_object(void* s, unsigned mat, unsigned first_tri, unsigned n_tris)
{
  Scene& S = *(Scene*)s;
  S.mats[mat].translucent_index = (int)S.translucent.size();
  S.translucent.push_back({(int)mat, first_tri, n_tris});
}
EXPORT void orc_scene_set_samples(void* s, unsigned n) { ((Scene*)s)->samples = n; }
// Texture of material `mat`: w x h texels of ch channels, read at the nearest texel of the cube map
// around center3.
EXPORT void orc_scene_set_texture(void* s, unsigned mat, const float* data, unsigned w, unsigned h, unsigned ch, const float* center3)
{
  Scene& S = *(Scene*)s;
  Tex t;
  t.w = w;
  t.h = h;
  t.ch = ch;
  t.data.assign(data, data + (size_t)w * h * ch);
  S.mats[mat].tex = (int)S.textures.size();
  S.mats[mat].tcenter = v3(center3[0], center3[1], center3[2]);
  S.textures.push_back(std::move(t));
}
EXPORT unsigned orc_cube_texel(const float* p3, const float* c3, unsigned w, unsigned h)
{
  return cube_texel(v3(p3[0], p3[1], p3[2]), v3(c3[0], c3[1], c3[2]), w, h);
}
// The probes of the most recent frame rendered (PositionSample records, 80 bytes each).
EXPORT long orc_scene_probes(void* s, void* out)
{
  Scene& S = *(Scene*)s;
  if (out) memcpy(out, S.probes.data(), S.probes.size() * sizeof(Probe));
  return (long)S.probes.size();
}
EXPORT void orc_compute_coefficients(const float* absorption, const float* scattering, const float* meancosine, float ior, float scale,
                                     void* out260)
{
  ScatProps p = compute_coefficients(absorption, scattering, meancosine, ior, scale);
  memcpy(out260, &p, sizeof(p));
}
EXPORT void orc_dipole_bssrdf(const void* props260, float dist, float* out3)
{
  ScatProps P;
  memcpy(&P, props260, sizeof(P));
  F3 r = dipole_bssrdf(dist, P);
  out3[0] = r.x; out3[1] = r.y; out3[2] = r.z;
}
EXPORT void orc_dirpole_bssrdf(const void* props260, const float* xi, const float* ni, const float* w12, const float* xo, const float* no, float* out3)
{
  ScatProps P;
  memcpy(&P, props260, sizeof(P));
  F3 r = dirpole_bssrdf(v3(xi[0], xi[1], xi[2]), v3(ni[0], ni[1], ni[2]), v3(w12[0], w12[1], w12[2]), v3(xo[0], xo[1], xo[2]),
                        v3(no[0], no[1], no[2]), P);
  out3[0] = r.x; out3[1] = r.y; out3[2] = r.z;
}

// Runs fn(k0, k1) over [0, n) in contiguous chunks on `threads` host threads.
template <class Fn> static void parallel_for(long n, int threads, Fn fn)
{
  threads = std::max(1, threads);
  if (threads == 1 || n < 4096) { fn(0, n); return; }
  const long chunk = (n + threads - 1) / threads;
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t) {
    const long k0 = t * chunk, k1 = std::min(n, k0 + chunk);
    if (k0 >= k1) break;
    th.emplace_back(fn, k0, k1);
  }
  for (auto& x : th) x.join();
}

// A batch of BSSRDF queries of one translucent material given by its raw parameters (absorption,
// scattering, meancosine per RGB, ior, scale: pt_translucent_params), coefficients derived and the
// dipole evaluated in R: standard dipole (model 0) on dist[n], directional (model 1) on 15 x n SoA
// geometry (xi, ni, w12, xo, no).  S is 3 x n SoA.
template <class R>
static void bssrdf_batch(const float* sa, const float* ss, const float* g, float ior, float scale, unsigned model, long n, const float* in, R* S,
                         int threads)
{
  const ScatPropsT<R> P = compute_coefficients_t<R>(sa, ss, g, ior, scale);
  parallel_for(n, threads, [&](long k0, long k1) {
    for (long k = k0; k < k1; ++k) {
      V3<R> r;
      if (model == 0) {
        r = dipole_bssrdf<R>((R)in[k], P);
      } else {
        V3<R> v[5];
        for (int j = 0; j < 5; ++j) v[j] = v3<R>(in[(3 * j) * n + k], in[(3 * j + 1) * n + k], in[(3 * j + 2) * n + k]);
        r = dirpole_bssrdf<R>(v[0], v[1], v[2], v[3], v[4], P);
      }
      S[k] = r.x; S[n + k] = r.y; S[2 * n + k] = r.z;
    }
  });
}
EXPORT void orc_bssrdf_queries_f(const float* sa, const float* ss, const float* g, float ior, float scale, unsigned model, long n,
                                 const float* in, float* S, int threads)
{
  bssrdf_batch<float>(sa, ss, g, ior, scale, model, n, in, S, threads);
}
EXPORT void orc_bssrdf_queries_d(const float* sa, const float* ss, const float* g, float ior, float scale, unsigned model, long n,
                                 const float* in, double* S, int threads)
{
  bssrdf_batch<double>(sa, ss, g, ior, scale, model, n, in, S, threads);
}

EXPORT long orc_capped(void* scene) { return ((Scene*)scene)->capped.load(); }

// Closest / any hit for a batch of rays (origin.xyz, tmin, dir.xyz, tmax per 8 floats): BVH
// result and brute-force result over all triangles.
EXPORT void orc_trace_batch(void* scene, const float* rays8, long n, int brute, int* prim, float* t, float* bary, int* any)
{
  Scene& S = *(Scene*)scene;
  for (long i = 0; i < n; ++i) {
    const float* r = rays8 + 8 * i;
    F3 o = v3(r[0], r[1], r[2]), d = v3(r[4], r[5], r[6]);
    HitRec h;
    if (brute) {
      h = {r[7], 0.0f, 0.0f, -1};
      for (size_t k = 0; k < S.tris.size(); ++k) {
        float tt, u, v;
        if (!tri_mt(o, d, S.tris[k], tt, u, v)) continue;
        if (tt > r[3] && (tt < h.t || (tt == h.t && h.prim >= 0 && (int)k < h.prim))) h = {tt, u, v, (int)k};
      }
      ana_closest(S, o, d, r[3], h);
    } else {
      h = closest(S, o, d, r[3], r[7]);
    }
    prim[i] = h.prim;
    t[i] = h.prim >= 0 ? h.t : -1.0f;
    bary[2 * i] = h.u;
    bary[2 * i + 1] = h.v;
    if (any) {
      if (brute) {
        int a = 0;
        for (size_t k = 0; k < S.tris.size() && !a; ++k) {
          float tt, u, v;
          if (tri_mt(o, d, S.tris[k], tt, u, v) && tt > r[3] && tt < r[7]) a = 1;
        }
        if (!a && ana_any(S, o, d, r[3], r[7])) a = 1;
        any[i] = a;
      } else {
        any[i] = occluded(S, o, d, r[3], r[7]) ? 1 : 0;
      }
    }
  }
}

// ---------------------------------------------------------------- FP64 evaluation of path tapes
namespace {

// Boundary polynomials of Fresnel.h:93-124 in FP64 (same coefficients).
static double c1_64(double n)
{
  if (n >= 1.0) return -9.23372 + n * (22.2272 + n * (-20.9292 + n * (10.2291 + n * (-2.54396 + n * 0.254913))));
  return 0.919317 + n * (-3.4793 + n * (6.75335 + n * (-7.80989 + n * (4.98554 - n * 1.36881))));
}
static double c2_64(double n)
{
  double r;
  if (n >= 1.0) {
    r = -1641.1 + n * (1213.67 + n * (-568.556 + n * (164.798 + n * (-27.0181 + n * 1.91826))));
    r += (((135.926 / n) - 656.175) / n + 1376.53) / n;
  } else {
    r = 0.828421 + n * (-2.62051 + n * (3.36231 + n * (-1.95284 + n * (0.236494 + n * 0.145787))));
  }
  return r;
}

struct Eval64 {
  const Scene& S;
  const double* P;
  const long* tex_off;
  const long* mat_off;
  double albedo(int tex, int texel, int c) const
  {
    long o = tex_off[tex];
    return o >= 0 ? P[o + 3 * (long)texel + c] : (double)S.textures[tex].data[3 * (size_t)texel + c];
  }
  double rough(int tex, int texel) const
  {
    long o = tex_off[tex];
    return o >= 0 ? P[o + texel] : (double)S.textures[tex].data[texel];
  }
  // (sigma_a RGB, sigma_s' RGB) of material mat
  void sigma(int mat, double out[6]) const
  {
    long o = mat_off[mat];
    const Mat& m = S.mats[mat];
    for (int c = 0; c < 3; ++c) {
      out[c] = o >= 0 ? P[o + c] : m.sig_a[c];
      out[3 + c] = o >= 0 ? P[o + 3 + c] : m.sig_sr[c];
    }
  }
};

// GGX D and Smith G1 of a cosine, FP64 (ggx_distribution, ggx_G1_cos).
static double ggx_D64(double c, double a)
{
  double c2 = c * c, t2 = (1.0 - c2) / c2, a2 = a * a;
  double q = a2 + t2;
  return a2 / (M_PI * c2 * c2 * q * q);
}
static double ggx_G164(double c, double a)
{
  double c2 = c * c, t2 = (1.0 - c2) / c2;
  return 2.0 / (1.0 + std::sqrt(1.0 + a * a * t2));
}
static double ggx_dlnD64(double c, double a)
{
  double c2 = c * c, t2 = (1.0 - c2) / c2;
  return 2.0 / a - 4.0 * a / (a * a + t2);
}
static double ggx_dlnG164(double c, double a)
{
  double c2 = c * c, t2 = (1.0 - c2) / c2;
  double q = std::sqrt(1.0 + a * a * t2);
  return -(a * t2 / q) / (1.0 + q);
}

// Standard dipole of one channel in FP64 and its derivatives with respect to (sigma_a, sigma_s').
static void dipole64(double dist, double sa_raw, double ssr_raw, double ior, double scale, double& S, double& dSa, double& dSs)
{
  const double sa = sa_raw * scale, x = (ssr_raw + sa_raw) * scale;  // absorption, reduced extinction
  const double D = 1.0 / (3.0 * x), dD = -D / x * scale;
  const double three_D = 3.0 * D, d3D = 3.0 * dD;
  const double tr = std::sqrt(sa / D);
  const double dtr_a = 3.0 * scale * (x + sa) / (2.0 * tr), dtr_s = 3.0 * sa * scale / (2.0 * tr);
  const double cphi = 0.25 * (1.0 - c1_64(ior)), ce = 0.5 * (1.0 - c2_64(ior));
  const double A = (1.0 - ce) / (2.0 * cphi);
  const double ext = 4.0 * A * D, dext = 4.0 * A * dD;
  const double r2 = dist * dist;
  const double dr2 = r2 + three_D * three_D, dr = std::sqrt(dr2), ddr = three_D * d3D / dr;
  const double dv2 = r2 + ext * ext, dv = std::sqrt(dv2), ddv = ext * dext / dv;
  const double cmf = three_D + ext, dcmf = d3D + dext;
  const double trr = tr * dr, trv = tr * dv;
  const double Sr = three_D * (1.0 + trr) / (dr2 * dr) * std::exp(-trr);
  const double Sv = cmf * (1.0 + trv) / (dv2 * dv) * std::exp(-trv);
  const double dtrr_a = dtr_a * dr + tr * ddr, dtrr_s = dtr_s * dr + tr * ddr;
  const double dtrv_a = dtr_a * dv + tr * ddv, dtrv_s = dtr_s * dv + tr * ddv;
  S = Sr + Sv;
  dSa = Sr * (d3D / three_D + dtrr_a / (1.0 + trr) - dtrr_a - 3.0 * ddr / dr) + Sv * (dcmf / cmf + dtrv_a / (1.0 + trv) - dtrv_a - 3.0 * ddv / dv);
  dSs = Sr * (d3D / three_D + dtrr_s / (1.0 + trr) - dtrr_s - 3.0 * ddr / dr) + Sv * (dcmf / cmf + dtrv_s / (1.0 + trv) - dtrv_s - 3.0 * ddv / dv);
}
static double global_coeff64(double ior)
{
  const double cphi_inv = 0.25 * (1.0 - c1_64(1.0 / ior));
  return 1.0 / (4.0 * cphi_inv) * 1.0 / (4.0 * M_PI * M_PI);
}

// One tape: its radiance (L) and, when grad is given, adds dLoss/dL (dl) times dL/dtheta to grad
// (path replay backprop on the stored vertices: T_k dE_k + (dw_k / w_k) R_{k+1}).
static void eval_tape(const Eval64& E, const Tape& tp, double L[3], const double* dl, double* grad)
{
  const size_t n = tp.recs.size();
  std::vector<double> Tk(3 * n), ck(3 * n, 0.0), wk(3 * n, 1.0);
  double T[3] = {1.0, 1.0, 1.0};
  L[0] = L[1] = L[2] = 0.0;
  for (size_t k = 0; k < n; ++k) {
    const TapeRec& r = tp.recs[k];
    for (int c = 0; c < 3; ++c) Tk[3 * k + c] = T[c];
    double e[3] = {0, 0, 0}, w[3] = {1, 1, 1};
    switch (r.type) {
      case TAPE_EMIT:
        for (int c = 0; c < 3; ++c) e[c] = r.v[c];
        break;
      case TAPE_NEE:
        for (int c = 0; c < 3; ++c) e[c] = (double)r.v[c] * E.albedo(r.tex, r.texel, c);
        break;
      case TAPE_CONST_W:
        for (int c = 0; c < 3; ++c) w[c] = r.v[c];
        break;
      case TAPE_DIFF_W:
        for (int c = 0; c < 3; ++c) w[c] = E.albedo(r.tex, r.texel, c) / (double)r.c[0];
        break;
      case TAPE_METAL_W: {
        const double a = E.rough(r.tex, r.texel), a0 = r.c[3];
        const double ratio = ggx_D64(r.c[0], a) * ggx_G164(r.c[1], a) * ggx_G164(r.c[2], a) /
                             (ggx_D64(r.c[0], a0) * ggx_G164(r.c[1], a0) * ggx_G164(r.c[2], a0));
        for (int c = 0; c < 3; ++c) w[c] = (double)r.v[c] * ratio;
        break;
      }
      case TAPE_BEER: {
        double sg[6];
        E.sigma(r.mat, sg);
        const Mat& m = E.S.mats[r.mat];
        for (int c = 0; c < 3; ++c) {
          const double k = m.dipole_model == DIRECTIONAL_DIPOLE ? (1.0 + m.mcos[c]) : 1.0 / (1.0 - m.mcos[c]);
          const double ext = (sg[3 + c] * k + sg[c]) * m.scale;
          w[c] = std::exp(-(double)r.c[0] * ext) / (double)r.c[1];
        }
        break;
      }
      case TAPE_GATHER: {
        double sg[6];
        E.sigma(r.mat, sg);
        const Mat& m = E.S.mats[r.mat];
        const double gc = global_coeff64(m.ior);
        for (int q = 0; q < r.g_count; ++q) {
          const TapeProbe& pr = tp.probes[r.g_begin + q];
          for (int c = 0; c < 3; ++c) {
            double Sv, da, ds;
            dipole64(pr.dist, sg[c], sg[3 + c], m.ior, m.scale, Sv, da, ds);
            e[c] += (double)pr.wl[c] * Sv / (double)pr.exp0;
          }
        }
        for (int c = 0; c < 3; ++c) e[c] = e[c] * gc / (double)E.S.samples;
        break;
      }
      default:
        break;
    }
    for (int c = 0; c < 3; ++c) {
      ck[3 * k + c] = T[c] * e[c];
      L[c] += ck[3 * k + c];
      wk[3 * k + c] = w[c];
      T[c] *= w[c];
    }
  }
  if (!grad) return;
  // R after record k: what the records beyond k add
  std::vector<double> R(3 * (n + 1), 0.0);
  for (size_t k = n; k-- > 0;)
    for (int c = 0; c < 3; ++c) R[3 * k + c] = R[3 * (k + 1) + c] + ck[3 * k + c];
  for (size_t k = 0; k < n; ++k) {
    const TapeRec& r = tp.recs[k];
    const double* Ra = &R[3 * (k + 1)];  // beyond record k
    const double* Tc = &Tk[3 * k];
    switch (r.type) {
      case TAPE_NEE: {
        long o = E.tex_off[r.tex];
        if (o >= 0)
          for (int c = 0; c < 3; ++c) grad[o + 3 * (long)r.texel + c] += dl[c] * Tc[c] * (double)r.v[c];
        break;
      }
      case TAPE_DIFF_W: {
        long o = E.tex_off[r.tex];
        if (o >= 0)
          for (int c = 0; c < 3; ++c) grad[o + 3 * (long)r.texel + c] += dl[c] * Ra[c] / E.albedo(r.tex, r.texel, c);
        break;
      }
      case TAPE_METAL_W: {
        long o = E.tex_off[r.tex];
        if (o >= 0) {
          const double a = E.rough(r.tex, r.texel);
          const double s = ggx_dlnD64(r.c[0], a) + ggx_dlnG164(r.c[1], a) + ggx_dlnG164(r.c[2], a);
          grad[o + r.texel] += s * (dl[0] * Ra[0] + dl[1] * Ra[1] + dl[2] * Ra[2]);
        }
        break;
      }
      case TAPE_BEER: {
        long o = E.mat_off[r.mat];
        if (o >= 0) {
          const Mat& m = E.S.mats[r.mat];
          for (int c = 0; c < 3; ++c) {
            const double k = m.dipole_model == DIRECTIONAL_DIPOLE ? (1.0 + m.mcos[c]) : 1.0 / (1.0 - m.mcos[c]);
            const double ga = dl[c] * Ra[c] * (-(double)r.c[0] * m.scale);
            grad[o + c] += ga;
            grad[o + 3 + c] += ga * k;
          }
        }
        break;
      }
      case TAPE_GATHER: {
        long o = E.mat_off[r.mat];
        if (o >= 0) {
          double sg[6];
          E.sigma(r.mat, sg);
          const Mat& m = E.S.mats[r.mat];
          const double gc = global_coeff64(m.ior);
          for (int q = 0; q < r.g_count; ++q) {
            const TapeProbe& pr = tp.probes[r.g_begin + q];
            for (int c = 0; c < 3; ++c) {
              double Sv, da, ds;
              dipole64(pr.dist, sg[c], sg[3 + c], m.ior, m.scale, Sv, da, ds);
              const double f = dl[c] * Tc[c] * gc / (double)E.S.samples * (double)pr.wl[c] / (double)pr.exp0;
              grad[o + c] += f * da;
              grad[o + 3 + c] += f * ds;
            }
          }
        }
        break;
      }
      default:
        break;
    }
  }
}

}  // namespace

EXPORT void orc_scene_record(void* s, int on) { ((Scene*)s)->record = on != 0; }
// The raw parameters of translucent material mat (FP64 tape evaluation): absorption and reduced
// scattering per RGB in the material's units, mean cosine, ior, scale.
EXPORT void orc_scene_set_translucent_raw(void* s, unsigned mat, const double* sig_a3, const double* sig_sr3, const double* mcos3, double ior,
                                          double scale)
{
  Mat& m = ((Scene*)s)->mats[mat];
  for (int c = 0; c < 3; ++c) {
    m.sig_a[c] = sig_a3[c];
    m.sig_sr[c] = sig_sr3[c];
    m.mcos[c] = mcos3[c];
  }
  m.ior = ior;
  m.scale = scale;
}
// Records of the last recorded render: count of tapes, records and gathered probes.
EXPORT void orc_tape_stats(void* s, long* out3)
{
  Scene& S = *(Scene*)s;
  long r = 0, p = 0;
  for (const Tape& t : S.tapes) {
    r += (long)t.recs.size();
    p += (long)t.probes.size();
  }
  out3[0] = (long)S.tapes.size();
  out3[1] = r;
  out3[2] = p;
}
// FP64 image of the recorded paths for parameters P (tex_off / mat_off: per texture and material the
// offset of its parameters in P, -1 = the scene's own values): per pixel of the recorded range the
// mean of its frames' path radiance, img_rgb[(pixel - p0) * 3 + c].  With dimg (dLoss/dimage, same
// layout) and grad (same layout as P), also adds the FP64 gradient of the loss.
EXPORT void orc_tape_eval(void* s, const double* P, const long* tex_off, const long* mat_off, double* img_rgb, const double* dimg, double* grad,
                          int threads)
{
  Scene& S = *(Scene*)s;
  const unsigned npix = S.tape_p1 - S.tape_p0;
  Eval64 E{S, P, tex_off, mat_off};
  const double inv = 1.0 / (double)(S.tape_first + S.tape_frames);
  std::fill(img_rgb, img_rgb + 3 * (size_t)npix, 0.0);
  // the gradient is accumulated by one thread (small checking renders); the image alone in parallel
  if (grad) threads = 1;
  threads = std::max(1, threads);
  std::atomic<unsigned> next(0);
  auto worker = [&]() {
    for (;;) {
      unsigned b = next.fetch_add(64);
      if (b >= npix) break;
      unsigned e = std::min(npix, b + 64);
      for (unsigned k = b; k < e; ++k) {
        double acc[3] = {0, 0, 0};
        double dl[3] = {0, 0, 0};
        if (dimg)
          for (int c = 0; c < 3; ++c) dl[c] = dimg[3 * (size_t)k + c] * inv;
        for (unsigned fl = 0; fl < S.tape_frames; ++fl) {
          const Tape& tp = S.tapes[(size_t)fl * npix + k];
          if (!tp.valid) continue;
          double L[3];
          eval_tape(E, tp, L, dl, grad);
          for (int c = 0; c < 3; ++c) acc[c] += L[c];
        }
        for (int c = 0; c < 3; ++c) img_rgb[3 * (size_t)k + c] = acc[c] * inv;
      }
    }
  };
  std::vector<std::thread> th;
  for (int i = 1; i < threads; ++i) th.emplace_back(worker);
  worker();
  for (auto& x : th) x.join();
}
