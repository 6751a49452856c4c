// Example host program: the reference's scene-object classes (include/orf_b200_scene.hpp) driving
// the B200 path tracer through the C ABI, in the order OptixScene/OptixSceneLoader use them.  Renders
// one of two scenes and writes the float4 accumulation buffer to a raw file (the .raw format of
// OptixScene::saveScene: width*height float4, row-major):
//   render_box <out.raw> [width height frames]
//       a diffuse box lit by a quad light (TrianglesAreaLight);
//   render_box --translucent <out.raw> <mesh.obj> <sky.hdr> width height frames
//       a translucent object read from an OBJ file (TranslucentMaterial, standard dipole, 64 probes per
//       frame) on a rough-diffuse floor, lit by an .hdr environment map (EnvMapBackground + its
//       EnvMapLight), a PointLight, a DirectionalLight, a SphericalLight and a DiskAreaLight.
#include <cstdio>
#include <cstdlib>
#include <string>

#include "../../include/orf_b200_scene.hpp"

static int write_raw(const char* path, const std::vector<float>& img, uint32_t w, uint32_t h, uint32_t frames)
{
  FILE* fh = fopen(path, "wb");
  if (!fh) return 3;
  fwrite(img.data(), sizeof(float), img.size(), fh);
  fclose(fh);
  double sum = 0;
  for (size_t i = 0; i < img.size(); i += 4) sum += img[i];
  printf("rendered %ux%u x %u frames, mean red %.6f\n", w, h, frames, sum / (w * h));
  return 0;
}

static int translucent(int argc, char** argv)
{
  if (argc < 8) {
    fprintf(stderr, "usage: %s --translucent out.raw mesh.obj sky.hdr width height frames\n", argv[0]);
    return 2;
  }
  const char* out = argv[2];
  const uint32_t w = (uint32_t)atoi(argv[5]), h = (uint32_t)atoi(argv[6]), frames = (uint32_t)atoi(argv[7]);
  try {
    orf::OptixScene scene(0);
    orf::PathTracer integrator;
    integrator.setMaxDepth(6);
    scene.setIntegrator(integrator);
    scene.setCamera(orf::PinholeCamera({0.0f, 0.35f, 2.0f}, {0.0f, 0.0f, 0.0f}, {0.0f, 1.0f, 0.0f}, 36.0f, w, h));
    scene.setBackground(orf::EnvMapBackground(std::string(argv[4])));
    scene.setProbeCount(64);
    orf::TranslucentMaterial skin;  // the reference's default coefficients, standard dipole
    orf::RoughDiffuseMaterial floor_mat;
    floor_mat.setColor({0.5f, 0.45f, 0.4f});
    floor_mat.setRoughness({0.3f, 0.3f});
    floor_mat.setNormalDistribution(PT_GGX_DISTRIBUTION);
    const uint32_t m_skin = scene.addMaterial(skin), m_floor = scene.addMaterial(floor_mat);
    scene.addObj(argv[3], m_skin);
    orf::Mesh floor;
    floor.positions = {-3, -0.55f, -3, 3, -0.55f, -3, 3, -0.55f, 3, -3, -0.55f, 3};
    floor.vindex = {0, 2, 1, 0, 3, 2};
    scene.addMesh(floor, m_floor);
    scene.setLights({std::make_shared<orf::EnvMapLight>(),
                     std::make_shared<orf::PointLight>(orf::float3{0.6f, 1.5f, 0.8f}, orf::float3{3.0f, 3.0f, 3.0f}),
                     std::make_shared<orf::DirectionalLight>(orf::float3{0.0f, -1.0f, 0.0f}, orf::float3{0.5f, 0.5f, 0.5f}),
                     std::make_shared<orf::SphericalLight>(orf::float3{-0.8f, 0.6f, 0.3f}, orf::float3{20.0f, 15.0f, 10.0f}, 0.05f),
                     std::make_shared<orf::DiskAreaLight>(orf::float3{0.5f, 1.2f, -0.5f}, orf::float3{5.0f, 5.0f, 5.0f}, 0.2f, 180.0f, 0.0f)});
    scene.initContext();
    scene.renderFrames(frames);
    return write_raw(out, scene.getBuffer(), w, h, frames);
  } catch (const orf::Error& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}

int main(int argc, char** argv)
{
  if (argc > 1 && std::string(argv[1]) == "--translucent") return translucent(argc, argv);
  if (argc < 2) {
    fprintf(stderr, "usage: %s out.raw [width height frames] | --translucent out.raw mesh.obj sky.hdr width height frames\n", argv[0]);
    return 2;
  }
  uint32_t w = argc > 3 ? (uint32_t)atoi(argv[2]) : 64, h = argc > 3 ? (uint32_t)atoi(argv[3]) : 64;
  uint32_t frames = argc > 4 ? (uint32_t)atoi(argv[4]) : 16;
  try {
    orf::OptixScene scene(0);
    orf::PathTracer integrator;
    integrator.setMaxDepth(8);
    scene.setIntegrator(integrator);
    orf::PinholeCamera camera({0.0f, 0.0f, 0.9f}, {0.0f, 0.0f, -1.0f}, {0.0f, 1.0f, 0.0f}, 60.0f, w, h);
    scene.setCamera(camera);
    scene.setBackground(orf::ConstantBackground({0.0f, 0.0f, 0.0f}));
    orf::DiffuseMaterial white({0.7f, 0.7f, 0.7f});
    uint32_t mid = scene.addMaterial(white);
    // closed box [-1,1]^3, 12 triangles (same winding as open_rendering_framework_b200/scenes.py box())
    orf::Mesh box;
    box.positions = {-1, -1, -1, 1, -1, -1, 1, 1, -1, -1, 1, -1, -1, -1, 1, 1, -1, 1, 1, 1, 1, -1, 1, 1};
    int q[6][4] = {{0, 1, 2, 3}, {5, 4, 7, 6}, {4, 0, 3, 7}, {1, 5, 6, 2}, {4, 5, 1, 0}, {3, 2, 6, 7}};
    for (auto& f : q) {
      int t[6] = {f[0], f[1], f[2], f[0], f[2], f[3]};
      box.vindex.insert(box.vindex.end(), t, t + 6);
    }
    scene.addMesh(box, mid);
    float y = 0.99f, s = 0.125f;
    orf::TriangleAreaLight light({-s, y, -s, s, y, -s, s, y, s, -s, y, s}, {0, 1, 2, 0, 2, 3}, {15.0f, 15.0f, 15.0f});
    scene.setLights(std::vector<orf::TriangleAreaLight>{light});
    scene.initContext();
    scene.renderFrames(frames);
    return write_raw(argv[1], scene.getBuffer(), w, h, frames);
  } catch (const orf::Error& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
