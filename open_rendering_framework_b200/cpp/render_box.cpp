// Example host program: the reference's scene-object classes (include/orf_b200_scene.hpp) driving
// the B200 path tracer through the C ABI, in the order OptixScene/OptixSceneLoader use them.  Renders
// a diffuse box lit by a quad light and writes the float4 accumulation buffer to a raw file
// (the .raw format of OptixScene::saveScene: width*height float4, row-major).
//   usage: render_box <out.raw> [width height frames]
#include <cstdio>
#include <cstdlib>

#include "../../include/orf_b200_scene.hpp"

int main(int argc, char** argv)
{
  if (argc < 2) {
    fprintf(stderr, "usage: %s out.raw [width height frames]\n", argv[0]);
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
    scene.setLights({light});
    scene.initContext();
    scene.renderFrames(frames);
    std::vector<float> img = scene.getBuffer();
    FILE* fh = fopen(argv[1], "wb");
    if (!fh) return 3;
    fwrite(img.data(), sizeof(float), img.size(), fh);
    fclose(fh);
    double sum = 0;
    for (size_t i = 0; i < img.size(); i += 4) sum += img[i];
    printf("rendered %ux%u x %u frames, mean red %.6f\n", w, h, frames, sum / (w * h));
  } catch (const orf::Error& e) {
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
