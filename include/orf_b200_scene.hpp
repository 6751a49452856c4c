// C++ scene-object classes of open_rendering_framework (Integrator.h, Camera.h, Background.h,
// Light.h, Material.h, OptixScene.h) written over the C ABI in orf_b200.h instead of OptiX.
//
// The reference's classes push parameters into OptiX variables (`context["max_depth"]->setInt`,
// `mtl["roughness"]->setFloat`, ...) and OptixScene::renderScene launches OptiX
// (OptixScene.cpp:139-168).  Here the same setters store the values and `OptixScene::renderScene`
// calls pt_render_frames; everything else -- Qt JSON, widgets, OBJ/HDR loading -- stays with the
// host application.  Errors surface as exceptions on the C++ side only; the C ABI itself
// never throws.  Header-only; link against libpt_b200.so.  (Errors are orf::Error.)
#pragma once
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "orf_b200.h"

namespace orf {

struct Error : std::runtime_error {
  pt_status status;
  Error(pt_status s, const std::string& where) : std::runtime_error(where + ": " + pt_last_error_message()), status(s) {}
};
inline void check(pt_status s, const char* where)
{
  if (s != PT_OK) throw Error(s, where);
}

using float3 = std::array<float, 3>;

// ---------------------------------------------------------------- Integrator.h
class PathTracer {
 public:
  uint32_t getMaxDepth() const { return max_depth; }
  void setMaxDepth(uint32_t d) { max_depth = d; }
  float getSceneEpsilon() const { return scene_epsilon; }
  void setSceneEpsilon(float e) { scene_epsilon = e; }
  float3 getExceptionColor() const { return exception_color; }
  void setExceptionColor(float3 c) { exception_color = c; }
  // Depth from which the diffuse shader's Russian roulette applies (0 = the reference's behaviour).
  void setRussianRouletteStartDepth(uint32_t d) { rr_start_depth = d; }
  void apply(pt_ctx* ctx) const { check(pt_set_integrator(ctx, max_depth, scene_epsilon, exception_color.data(), rr_start_depth), "pt_set_integrator"); }

 private:
  uint32_t max_depth = 50;         // Integrator.cpp:10
  float scene_epsilon = 1e-4f;     // Integrator.cpp:11
  float3 exception_color{1, 0, 0};  // Integrator.cpp:12
  uint32_t rr_start_depth = 0;
};

// ---------------------------------------------------------------- Camera.h
class PinholeCamera {
 public:
  PinholeCamera(float3 eye, float3 lookat, float3 up, float vfov, uint32_t width, uint32_t height)
      : eye(eye), lookat(lookat), up(up), vfov(vfov), WIDTH(width), HEIGHT(height), patch_origin{0, 0}, patch_dims{width, height}
  {
    calculateCameraVariables();
  }
  void setEye(float3 e) { eye = e; calculateCameraVariables(); }
  void setLookat(float3 l) { lookat = l; calculateCameraVariables(); }
  void setUp(float3 u) { up = u; calculateCameraVariables(); }
  void setFov(float f) { vfov = f; calculateCameraVariables(); }
  void setPatchOrigin(std::array<uint32_t, 2> o) { patch_origin = o; }
  void setPatchDims(std::array<uint32_t, 2> d) { patch_dims = d; }
  void resizeCamera(uint32_t w, uint32_t h)
  {
    WIDTH = w;
    HEIGHT = h;
    patch_dims = {w, h};
    calculateCameraVariables();
  }
  uint32_t getWidth() const { return WIDTH; }
  uint32_t getHeight() const { return HEIGHT; }
  void apply(pt_ctx* ctx) const
  {
    check(pt_set_camera(ctx, eye.data(), U.data(), V.data(), W.data(), WIDTH, HEIGHT, patch_origin.data(), patch_dims.data()), "pt_set_camera");
  }

 private:
  // PinholeCamera::calculateCameraVariables (Camera.cpp:83-103).
  void calculateCameraVariables()
  {
    float3 w = {lookat[0] - eye[0], lookat[1] - eye[1], lookat[2] - eye[2]};
    double wlen = std::sqrt((double)w[0] * w[0] + (double)w[1] * w[1] + (double)w[2] * w[2]);
    double u[3] = {(double)w[1] * up[2] - (double)w[2] * up[1], (double)w[2] * up[0] - (double)w[0] * up[2], (double)w[0] * up[1] - (double)w[1] * up[0]};
    double ul = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
    float uf[3] = {(float)(u[0] / ul), (float)(u[1] / ul), (float)(u[2] / ul)};
    double v[3] = {(double)uf[1] * w[2] - (double)uf[2] * w[1], (double)uf[2] * w[0] - (double)uf[0] * w[2], (double)uf[0] * w[1] - (double)uf[1] * w[0]};
    double vl = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    float vlen = (float)wlen * (float)std::tan(0.5 * vfov * 3.14159265358979323846 / 180.0);
    float ulen = vlen * (float)((double)WIDTH / (double)HEIGHT);
    for (int k = 0; k < 3; ++k) {
      V[k] = (float)(v[k] / vl) * vlen;
      U[k] = uf[k] * ulen;
      W[k] = w[k];
    }
  }
  float3 eye, lookat, up;
  float vfov;
  uint32_t WIDTH, HEIGHT;
  std::array<uint32_t, 2> patch_origin, patch_dims;
  float3 U{}, V{}, W{};
};

// ---------------------------------------------------------------- Background.h
class ConstantBackground {
 public:
  explicit ConstantBackground(float3 c = {1, 1, 1}) : background_color(c) {}  // Background.cpp:10
  void setBackgroundColor(float3 c) { background_color = c; }
  float3 getBackgroundColor() const { return background_color; }
  void apply(pt_ctx* ctx) const { check(pt_set_background_constant(ctx, background_color.data()), "pt_set_background_constant"); }

 private:
  float3 background_color;
};

// ---------------------------------------------------------------- Material.h
class MyMaterial {
 public:
  virtual ~MyMaterial() = default;
  virtual uint32_t getType() const = 0;
  virtual std::vector<unsigned char> params() const = 0;
};
class DiffuseMaterial : public MyMaterial {
 public:
  explicit DiffuseMaterial(float3 c = {0.8f, 0.8f, 0.8f}) : color(c) {}
  void setColor(float3 c) { color = c; }
  uint32_t getType() const override { return PT_DIFFUSE_SHADER; }
  std::vector<unsigned char> params() const override
  {
    pt_diffuse_params p;
    memcpy(p.diffuse_color, color.data(), 12);
    return bytes(p);
  }
  template <class T> static std::vector<unsigned char> bytes(const T& p) { return std::vector<unsigned char>((const unsigned char*)&p, (const unsigned char*)&p + sizeof(T)); }

 private:
  float3 color;
};
class MetallicMaterial : public MyMaterial {
 public:
  // gold (Material.h:328), roughness 0.1, Walter model, Beckmann (MetallicMaterial.cpp:7-26)
  std::array<double, 6> ior{0.170265, 3.01893, 0.511516, 2.44734, 1.47544, 1.87263};
  std::array<float, 2> roughness{0.1f, 0.1f};
  uint32_t microfacet_model = PT_WALTER_MODEL, normal_distribution = PT_BECKMANN_DISTRIBUTION;
  void setIor(std::array<double, 6> i) { ior = i; }
  void setRoughness(std::array<float, 2> r) { roughness = r; }
  void setMicrofacetModel(uint32_t m) { microfacet_model = m; }
  void setNormalDistribution(uint32_t d) { normal_distribution = d; }
  uint32_t getType() const override { return PT_METALLIC_SHADER; }
  std::vector<unsigned char> params() const override
  {
    pt_metallic_params p;
    memcpy(p.ior, ior.data(), sizeof(p.ior));
    memcpy(p.roughness, roughness.data(), sizeof(p.roughness));
    p.microfacet_model = microfacet_model;
    p.normal_distribution = normal_distribution;
    return DiffuseMaterial::bytes(p);
  }
};
class RoughTransparentMaterial : public MyMaterial {
 public:
  // ior 1.3, roughness 0.1, no absorption, Walter, Beckmann (RoughTransparentMaterial.cpp:7-28)
  float ior = 1.3f, roughness = 0.1f;
  float3 glass_absorption{0, 0, 0};
  uint32_t microfacet_model = PT_WALTER_MODEL, normal_distribution = PT_BECKMANN_DISTRIBUTION;
  uint32_t getType() const override { return PT_ROUGH_TRANSPARENT_SHADER; }
  std::vector<unsigned char> params() const override
  {
    pt_rough_transparent_params p;
    p.ior = ior;
    p.roughness = roughness;
    memcpy(p.glass_absorption, glass_absorption.data(), 12);
    p.microfacet_model = microfacet_model;
    p.normal_distribution = normal_distribution;
    return DiffuseMaterial::bytes(p);
  }
};

// ---------------------------------------------------------------- Light.h
// LightStruct / TriangleLight byte layouts (structs.h:42-103).
struct LightStruct { uint32_t light_type; float emitted_radiance[3]; float p[3]; float padding[3]; };
struct TriangleLight { float v0[3], v1[3], v2[3], n0[3], n1[3], n2[3]; uint32_t has_normals; float emission[3]; float area; };
static_assert(sizeof(LightStruct) == 40 && sizeof(TriangleLight) == 92, "reference light layouts");

class TriangleAreaLight {
 public:
  TriangleAreaLight(std::vector<float> positions, std::vector<int32_t> vindex, float3 radiance)
      : positions(std::move(positions)), vindex(std::move(vindex)), radiance(radiance) {}
  std::vector<float> positions;
  std::vector<int32_t> vindex;
  float3 radiance;
};

struct Mesh {
  std::vector<float> positions;
  std::vector<int32_t> vindex;
  std::vector<float> normals;
  std::vector<int32_t> nindex;
  std::shared_ptr<MyMaterial> material;
};

// ---------------------------------------------------------------- OptixScene.h
class OptixScene {
 public:
  explicit OptixScene(int device = 0) { check(pt_context_create(device, &ctx), "pt_context_create"); }
  ~OptixScene() { pt_context_destroy(ctx); }
  OptixScene(const OptixScene&) = delete;
  OptixScene& operator=(const OptixScene&) = delete;

  void setIntegrator(const PathTracer& p) { p.apply(ctx); }
  void setCamera(const PinholeCamera& c)
  {
    c.apply(ctx);
    width = c.getWidth();
    height = c.getHeight();
    frame = 0;
  }
  void setBackground(const ConstantBackground& b) { b.apply(ctx); }
  uint32_t addMaterial(const MyMaterial& m)
  {
    auto p = m.params();
    uint32_t id;
    check(pt_material_create(ctx, m.getType(), p.data(), p.size(), &id), "pt_material_create");
    return id;
  }
  void updateMaterial(uint32_t id, const MyMaterial& m)
  {
    auto p = m.params();
    check(pt_material_update(ctx, id, p.data(), p.size()), "pt_material_update");
  }
  void addMesh(const Mesh& m, uint32_t material_id)
  {
    uint32_t first;
    check(pt_mesh_add(ctx, m.positions.data(), (uint32_t)(m.positions.size() / 3), m.vindex.data(), (uint32_t)(m.vindex.size() / 3),
                      m.normals.empty() ? nullptr : m.normals.data(), (uint32_t)(m.normals.size() / 3), m.nindex.empty() ? nullptr : m.nindex.data(),
                      material_id, &first),
          "pt_mesh_add");
  }
  // Adds the lights' emitter meshes and uploads light_buffer / triangle_light_buffer as
  // OptixSceneLoader::addLight / loadTriangleLightBuffer / updateLights do (OptixSceneLoader.cpp:284-410).
  void setLights(const std::vector<TriangleAreaLight>& lights)
  {
    std::vector<LightStruct> ls;
    std::vector<TriangleLight> tl;
    for (const TriangleAreaLight& L : lights) {
      pt_area_light_params ap;
      memcpy(ap.radiance, L.radiance.data(), 12);
      uint32_t mid;
      check(pt_material_create(ctx, PT_AREA_LIGHT_MATERIAL, &ap, sizeof(ap), &mid), "pt_material_create");
      Mesh m{L.positions, L.vindex, {}, {}, nullptr};
      addMesh(m, mid);
      LightStruct s{};
      s.light_type = 2;  // TRIANGLES_AREA_LIGHT
      memcpy(s.emitted_radiance, L.radiance.data(), 12);
      size_t ntri = L.vindex.size() / 3;
      s.p[0] = (float)ntri;
      s.p[1] = (float)tl.size();
      s.p[2] = (float)(tl.size() + ntri - 1);
      ls.push_back(s);
      for (size_t t = 0; t < ntri; ++t) {
        TriangleLight r{};
        const float* a = &L.positions[3 * L.vindex[3 * t]];
        const float* b = &L.positions[3 * L.vindex[3 * t + 1]];
        const float* c = &L.positions[3 * L.vindex[3 * t + 2]];
        memcpy(r.v0, a, 12);
        memcpy(r.v1, b, 12);
        memcpy(r.v2, c, 12);
        float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        float px = e1[1] * e2[2] - e1[2] * e2[1], py = e1[2] * e2[0] - e1[0] * e2[2], pz = e1[0] * e2[1] - e1[1] * e2[0];
        r.area = (float)(0.5 * std::sqrt(px * px + py * py + pz * pz));  // Light.cpp:296
        memcpy(r.emission, L.radiance.data(), 12);
        tl.push_back(r);
      }
    }
    check(pt_lights_upload(ctx, ls.data(), (uint32_t)ls.size(), tl.data(), (uint32_t)tl.size()), "pt_lights_upload");
  }
  void initContext() { check(pt_build(ctx), "pt_build"); }
  // OptixScene::renderScene (OptixScene.cpp:139-168): frame++ and one integrator pass.
  void renderScene() { check(pt_render_frames(ctx, frame++, 1), "pt_render_frames"); }
  // Several frames in one wavefront launch group (same result as calling renderScene n times).
  void renderFrames(uint32_t n)
  {
    check(pt_render_frames(ctx, frame, n), "pt_render_frames");
    frame += n;
  }
  std::vector<float> getBuffer() const
  {
    std::vector<float> out((size_t)width * height * 4);
    check(pt_readback(ctx, out.data()), "pt_readback");
    return out;
  }
  uint32_t getFrame() const { return frame; }
  pt_ctx* handle() const { return ctx; }

 private:
  pt_ctx* ctx = nullptr;
  uint32_t width = 0, height = 0, frame = 0;
};

}  // namespace orf
