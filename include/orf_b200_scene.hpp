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

// EnvMapBackground (Background.h:44, Background.cpp:57-69): an equirectangular environment map, either
// float4 texels (width x height, row 0 at v = 0) or a Radiance .hdr file read as the reference's
// loadHDRTexture reads it (pt_set_envmap_hdr: host parse, device RGBE expansion, CDF build).
class EnvMapBackground {
 public:
  explicit EnvMapBackground(std::string hdr_path) : path(std::move(hdr_path)) {}
  EnvMapBackground(std::vector<float> rgba, uint32_t width, uint32_t height) : texels(std::move(rgba)), w(width), h(height) {}
  void apply(pt_ctx* ctx) const
  {
    if (!path.empty())
      check(pt_set_envmap_hdr(ctx, path.c_str()), "pt_set_envmap_hdr");
    else
      check(pt_set_envmap(ctx, texels.data(), w, h), "pt_set_envmap");
  }

 private:
  std::string path;
  std::vector<float> texels;
  uint32_t w = 0, h = 0;
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

// TransparentMaterial (Material.h:230, TransparentMaterial.cpp:7-20): smooth dielectric.
class TransparentMaterial : public MyMaterial {
 public:
  float ior = 1.3f;
  float3 glass_absorption{0, 0, 0};
  void setIor(float i) { ior = i; }
  void setAbsorption(float3 a) { glass_absorption = a; }
  uint32_t getType() const override { return PT_TRANSPARENT_SHADER; }
  std::vector<unsigned char> params() const override
  {
    pt_transparent_params p;
    p.ior = ior;
    memcpy(p.glass_absorption, glass_absorption.data(), 12);
    return DiffuseMaterial::bytes(p);
  }
};
// LambertianInterfaceMaterial (Material.h:133, LambertianInterfaceMaterial.cpp:7-20): a Lambertian base
// under a smooth dielectric interface.
class LambertianInterfaceMaterial : public MyMaterial {
 public:
  float3 color{1, 1, 1};
  float ior = 1.3f;
  void setColor(float3 c) { color = c; }
  void setIor(float i) { ior = i; }
  uint32_t getType() const override { return PT_LAMBERTIAN_INTERFACE_SHADER; }
  std::vector<unsigned char> params() const override
  {
    pt_lambertian_interface_params p;
    memcpy(p.diffuse_color, color.data(), 12);
    p.ior = ior;
    return DiffuseMaterial::bytes(p);
  }
};
// RoughDiffuseMaterial (Material.h:167, RoughDiffuseMaterial.cpp:7-28): a Lambertian base under a
// rough dielectric interface.
class RoughDiffuseMaterial : public MyMaterial {
 public:
  float3 color{1, 1, 1};
  float ior = 1.3f;
  std::array<float, 2> roughness{0.1f, 0.1f};
  uint32_t microfacet_model = PT_WALTER_MODEL, normal_distribution = PT_BECKMANN_DISTRIBUTION;
  void setColor(float3 c) { color = c; }
  void setIor(float i) { ior = i; }
  void setRoughness(std::array<float, 2> r) { roughness = r; }
  void setMicrofacetModel(uint32_t m) { microfacet_model = m; }
  void setNormalDistribution(uint32_t d) { normal_distribution = d; }
  uint32_t getType() const override { return PT_ROUGH_DIFFUSE_SHADER; }
  std::vector<unsigned char> params() const override
  {
    pt_rough_diffuse_params p;
    memcpy(p.diffuse_color, color.data(), 12);
    p.ior = ior;
    memcpy(p.roughness, roughness.data(), 8);
    p.microfacet_model = microfacet_model;
    p.normal_distribution = normal_distribution;
    return DiffuseMaterial::bytes(p);
  }
};
// TranslucentMaterial (Material.h:357, TranslucentMaterial.cpp:7-30): dipole BSSRDF under a smooth
// boundary.  Coefficients per RGB in 1/mm, scaled by `scale`; defaults: the "Apple" entry of
// getDefaultMaterial (TranslucentMaterial.cpp:245-250), scale 100, standard dipole.
class TranslucentMaterial : public MyMaterial {
 public:
  float3 scattering{2.29f, 2.39f, 1.97f}, absorption{0.0030f, 0.0034f, 0.0046f}, meancosine{0, 0, 0};
  float ior = 1.3f, scale = 100.0f;
  uint32_t dipole_model = PT_STANDARD_DIPOLE;
  void setScattering(float3 v) { scattering = v; }
  void setAbsorption(float3 v) { absorption = v; }
  void setMeanCosine(float3 v) { meancosine = v; }
  void setIor(float i) { ior = i; }
  void setScale(float v) { scale = v; }
  void setDipoleModel(uint32_t m) { dipole_model = m; }
  uint32_t getType() const override { return PT_TRANSLUCENT_SHADER; }
  std::vector<unsigned char> params() const override { return DiffuseMaterial::bytes(translucent()); }

 protected:
  pt_translucent_params translucent() const
  {
    pt_translucent_params p;
    memcpy(p.scattering, scattering.data(), 12);
    memcpy(p.absorption, absorption.data(), 12);
    memcpy(p.meancosine, meancosine.data(), 12);
    p.ior = ior;
    p.scale = scale;
    p.dipole_model = dipole_model;
    return p;
  }
};
// RoughTranslucentMaterial (Material.h:416, RoughTranslucentMaterial.cpp:360-395): the dipole under a
// rough dielectric boundary.
class RoughTranslucentMaterial : public TranslucentMaterial {
 public:
  std::array<float, 2> roughness{0.1f, 0.1f};
  uint32_t microfacet_model = PT_WALTER_MODEL, normal_distribution = PT_BECKMANN_DISTRIBUTION;
  void setRoughness(std::array<float, 2> r) { roughness = r; }
  void setMicrofacetModel(uint32_t m) { microfacet_model = m; }
  void setNormalDistribution(uint32_t d) { normal_distribution = d; }
  uint32_t getType() const override { return PT_ROUGH_TRANSLUCENT_SHADER; }
  std::vector<unsigned char> params() const override
  {
    const pt_translucent_params t = translucent();
    pt_rough_translucent_params p;
    memcpy(p.scattering, t.scattering, 12);
    memcpy(p.absorption, t.absorption, 12);
    memcpy(p.meancosine, t.meancosine, 12);
    p.ior = t.ior;
    p.scale = t.scale;
    p.dipole_model = t.dipole_model;
    memcpy(p.roughness, roughness.data(), 8);
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

// light_type values of LightStruct (structs.h:27-34).
enum : uint32_t { POINT_LIGHT = 0, DIRECTIONAL_LIGHT = 1, TRIANGLES_AREA_LIGHT = 2, DISK_LIGHT = 3, SPHERICAL_LIGHT = 4, ENVMAP_LIGHT = 5 };

// Light (Light.h:10): each light adds its light_buffer record (and a TrianglesAreaLight its emitter
// mesh and triangle_light_buffer records) as OptixSceneLoader::addLight / updateLights do.
class OptixScene;
class Light {
 public:
  virtual ~Light() = default;
  virtual void append(OptixScene& scene, std::vector<LightStruct>& lights, std::vector<TriangleLight>& tris) const = 0;
};
// PointLight (Light.h:28, Light.cpp:26-60).
class PointLight : public Light {
 public:
  PointLight(float3 position, float3 radiance) : position(position), radiance(radiance) {}
  void setPosition(float3 p) { position = p; }
  void setRadiance(float3 r) { radiance = r; }
  void append(OptixScene&, std::vector<LightStruct>& ls, std::vector<TriangleLight>&) const override
  {
    LightStruct s{};
    s.light_type = POINT_LIGHT;
    memcpy(s.emitted_radiance, radiance.data(), 12);
    memcpy(s.p, position.data(), 12);
    ls.push_back(s);
  }
  float3 position, radiance;
};
// DirectionalLight (Light.h:49, Light.cpp:62-100): the stored direction is normalised in FP32.
class DirectionalLight : public Light {
 public:
  DirectionalLight(float3 direction, float3 radiance) : direction(direction), radiance(radiance) {}
  void setDirection(float3 d) { direction = d; }
  void setRadiance(float3 r) { radiance = r; }
  void append(OptixScene&, std::vector<LightStruct>& ls, std::vector<TriangleLight>&) const override
  {
    LightStruct s{};
    s.light_type = DIRECTIONAL_LIGHT;
    memcpy(s.emitted_radiance, radiance.data(), 12);
    const float len = std::sqrt(direction[0] * direction[0] + direction[1] * direction[1] + direction[2] * direction[2]);
    for (int k = 0; k < 3; ++k) s.p[k] = direction[k] / len;
    ls.push_back(s);
  }
  float3 direction, radiance;
};
// DiskAreaLight (Light.h:133, Light.cpp:370-503): position, radius and the normal's angles theta / phi
// in degrees (DiskLightStruct, structs.h:76-84); its geometry is intersected analytically.
class DiskAreaLight : public Light {
 public:
  DiskAreaLight(float3 position, float3 radiance, float radius = 1.0f, float theta = 0.0f, float phi = 0.0f)
      : position(position), radiance(radiance), radius(radius), theta(theta), phi(phi) {}
  void append(OptixScene&, std::vector<LightStruct>& ls, std::vector<TriangleLight>&) const override
  {
    LightStruct s{};
    s.light_type = DISK_LIGHT;
    memcpy(s.emitted_radiance, radiance.data(), 12);
    memcpy(s.p, position.data(), 12);
    s.padding[0] = radius;
    s.padding[1] = phi;
    s.padding[2] = theta;
    ls.push_back(s);
  }
  float3 position, radiance;
  float radius, theta, phi;
};
// SphericalLight (Light.h:167, Light.cpp:505-610): position and radius (SphericalLightStruct,
// structs.h:86-93); its geometry is intersected analytically.
class SphericalLight : public Light {
 public:
  SphericalLight(float3 position, float3 radiance, float radius = 0.05f) : position(position), radiance(radiance), radius(radius) {}
  void append(OptixScene&, std::vector<LightStruct>& ls, std::vector<TriangleLight>&) const override
  {
    LightStruct s{};
    s.light_type = SPHERICAL_LIGHT;
    memcpy(s.emitted_radiance, radiance.data(), 12);
    memcpy(s.p, position.data(), 12);
    s.padding[0] = radius;
    ls.push_back(s);
  }
  float3 position, radiance;
  float radius;
};
// The environment map as a light (light_type 5): next-event estimation samples it through its
// marginal / conditional CDFs (Envmap.h:66-98).  Needs an EnvMapBackground.
class EnvMapLight : public Light {
 public:
  void append(OptixScene&, std::vector<LightStruct>& ls, std::vector<TriangleLight>&) const override
  {
    LightStruct s{};
    s.light_type = ENVMAP_LIGHT;
    s.emitted_radiance[0] = s.emitted_radiance[1] = s.emitted_radiance[2] = 1.0f;
    ls.push_back(s);
  }
};
// TrianglesAreaLight (Light.h:97, Light.cpp:240-368): an emitting triangle mesh.
class TriangleAreaLight : public Light {
 public:
  TriangleAreaLight(std::vector<float> positions, std::vector<int32_t> vindex, float3 radiance)
      : positions(std::move(positions)), vindex(std::move(vindex)), radiance(radiance) {}
  void append(OptixScene& scene, std::vector<LightStruct>& ls, std::vector<TriangleLight>& tl) const override;
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
  void setBackground(const EnvMapBackground& b) { b.apply(ctx); }
  // context["samples"]: probe points per translucent object and frame (OptixSceneLoader.cpp:11-17).
  void setProbeCount(uint32_t samples) { check(pt_set_probe_count(ctx, samples), "pt_set_probe_count"); }
  // Adds the lights' emitter meshes and uploads light_buffer / triangle_light_buffer as
  // OptixSceneLoader::addLight / loadTriangleLightBuffer / updateLights do (OptixSceneLoader.cpp:284-410).
  void setLights(const std::vector<std::shared_ptr<Light>>& lights)
  {
    std::vector<LightStruct> ls;
    std::vector<TriangleLight> tl;
    for (const auto& L : lights) L->append(*this, ls, tl);
    check(pt_lights_upload(ctx, ls.empty() ? nullptr : ls.data(), (uint32_t)ls.size(), tl.empty() ? nullptr : tl.data(), (uint32_t)tl.size()),
          "pt_lights_upload");
  }
  void setLights(const std::vector<TriangleAreaLight>& lights)
  {
    std::vector<std::shared_ptr<Light>> all;
    for (const TriangleAreaLight& L : lights) all.push_back(std::make_shared<TriangleAreaLight>(L));
    setLights(all);
  }
  // The groups of an OBJ file (glm's reader as ObjLoader flattens it, pt_obj_read) as meshes of one
  // material, sharing the file's vertex and normal arrays.
  void addObj(const std::string& path, uint32_t material_id)
  {
    pt_obj* obj = nullptr;
    check(pt_obj_read(path.c_str(), &obj), "pt_obj_read");
    pt_obj_info info;
    pt_status st = pt_obj_get_info(obj, &info);
    Mesh m;
    if (st == PT_OK) {
      m.positions.resize(3 * (size_t)info.n_vertices);
      m.normals.resize(3 * (size_t)info.n_normals);
      m.vindex.resize(3 * (size_t)info.n_triangles);
      m.nindex.resize(3 * (size_t)info.n_triangles);
      st = pt_obj_get_arrays(obj, m.positions.data(), m.normals.empty() ? nullptr : m.normals.data(), nullptr, m.vindex.data(),
                             m.normals.empty() ? nullptr : m.nindex.data(), nullptr, nullptr);
    }
    pt_obj_free(obj);
    check(st, "pt_obj_get_arrays");
    if (m.normals.empty()) m.nindex.clear();
    addMesh(m, material_id);
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

inline void TriangleAreaLight::append(OptixScene& scene, std::vector<LightStruct>& ls, std::vector<TriangleLight>& tl) const
{
  pt_area_light_params ap;
  memcpy(ap.radiance, radiance.data(), 12);
  uint32_t mid;
  check(pt_material_create(scene.handle(), PT_AREA_LIGHT_MATERIAL, &ap, sizeof(ap), &mid), "pt_material_create");
  Mesh m{positions, vindex, {}, {}, nullptr};
  scene.addMesh(m, mid);
  LightStruct s{};
  s.light_type = TRIANGLES_AREA_LIGHT;
  memcpy(s.emitted_radiance, radiance.data(), 12);
  size_t ntri = vindex.size() / 3;
  s.p[0] = (float)ntri;
  s.p[1] = (float)tl.size();
  s.p[2] = (float)(tl.size() + ntri - 1);
  ls.push_back(s);
  for (size_t t = 0; t < ntri; ++t) {
    TriangleLight r{};
    const float* a = &positions[3 * vindex[3 * t]];
    const float* b = &positions[3 * vindex[3 * t + 1]];
    const float* c = &positions[3 * vindex[3 * t + 2]];
    memcpy(r.v0, a, 12);
    memcpy(r.v1, b, 12);
    memcpy(r.v2, c, 12);
    float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    float px = e1[1] * e2[2] - e1[2] * e2[1], py = e1[2] * e2[0] - e1[0] * e2[2], pz = e1[0] * e2[1] - e1[1] * e2[0];
    r.area = (float)(0.5 * std::sqrt(px * px + py * py + pz * pz));  // Light.cpp:296
    memcpy(r.emission, radiance.data(), 12);
    tl.push_back(r);
  }
}

}  // namespace orf
