// Test infrastructure (oracle only).  This translation unit compiles two of the REFERENCE's own
// scene-ingestion sources in place (open_rendering_framework/HDRLoader.cpp and glm.cpp, included
// from the reference tree, never copied) on the host with g++ and exports a plain C interface over
// them: the RGBE .hdr texture exactly as loadHDRTexture hands it to OptiX, and an OBJ model read by
// glmReadOBJ flattened group by group the way ObjLoader::loadVertexData (ObjLoader.cpp:193-260)
// builds its index buffers.  It pins the library's .hdr and .obj readers.  Only tests load the
// resulting library (oracle/_ref/libref_io.so).
//
// HDRLoader.h includes <optixu/optixpp_namespace.h>; the stand-in under oracle/ref_shim/optixu/
// provides the handful of object-API names loadHDRTexture calls.
#include "HDRLoader.cpp"
#include "glm.cpp"

#include <clocale>
#include <locale>
#include <cstring>
#include <string>

#define EXPORT extern "C" __attribute__((visibility("default")))

// loadHDRTexture(path): the float4 buffer (row j = the file's scanline ny-1-j) and its size.  The
// reference leaves the fourth channel uninitialised, so only RGB is defined.  Returns 0 when the
// loader failed (the reference then installs a 1x1 texture of the default color).
// The reference's readers parse numbers with the C library and with iostreams, whose results depend on
// the process's C and C++ locales (a locale with a decimal comma reads "1.5" as 1); they are therefore
// run under the classic "C" locale, for the C library and for the streams they open, whatever locale
// the calling process has set.
struct CLocale {
  std::string saved;
  std::locale saved_cpp;
  CLocale() : saved_cpp(std::locale::global(std::locale::classic())) { saved = setlocale(LC_ALL, nullptr); setlocale(LC_ALL, "C"); }
  ~CLocale() { setlocale(LC_ALL, saved.c_str()); std::locale::global(saved_cpp); }
};

EXPORT int ref_hdr_load(const char* path, float* rgba, unsigned long capacity, unsigned* w, unsigned* h)
{
  CLocale c_locale;
  HDRLoader probe(path);
  if (probe.failed()) return 0;
  optix::Context ctx;
  ctx.p = std::make_shared<optix::ShimContext>();
  optix::TextureSampler s = loadHDRTexture(ctx, path, optix::make_float3(0.0f, 0.0f, 0.0f));
  *w = (unsigned)s->buffer->w;
  *h = (unsigned)s->buffer->h;
  const unsigned long n = 4ul * *w * *h;
  if (rgba && capacity >= n) memcpy(rgba, s->buffer->texels.data(), n * sizeof(float));
  return 1;
}

// glmReadOBJ(path) flattened as ObjLoader does: the groups in list order, empty groups skipped, each
// group's triangles in order, indices 0-based (index - 1: a missing normal or texcoord becomes -1).
// counts = (vertices, normals, texcoords, triangles, non-empty groups).  Arrays may be null to query.
EXPORT int ref_obj_load(const char* path, unsigned* counts, float* positions, float* normals, float* texcoords, int* vindex,
                        int* nindex, int* tindex, unsigned* group_of_triangle, char* group_names, unsigned name_stride)
{
  CLocale c_locale;
  GLMmodel* model = glmReadOBJ(path);
  if (!model) return 0;
  unsigned ntri = 0, ng = 0;
  for (GLMgroup* g = model->groups; g; g = g->next) {
    if (g->numtriangles == 0) continue;
    for (unsigned i = 0; i < g->numtriangles; ++i, ++ntri) {
      const GLMtriangle& T = model->triangles[g->triangles[i]];
      for (int k = 0; k < 3; ++k) {
        if (vindex) vindex[3 * ntri + k] = (int)T.vindices[k] - 1;
        if (nindex) nindex[3 * ntri + k] = (int)T.nindices[k] - 1;
        if (tindex) tindex[3 * ntri + k] = (int)T.tindices[k] - 1;
      }
      if (group_of_triangle) group_of_triangle[ntri] = ng;
    }
    if (group_names) {
      strncpy(group_names + (size_t)ng * name_stride, g->name, name_stride - 1);
      group_names[(size_t)ng * name_stride + name_stride - 1] = 0;
    }
    ++ng;
  }
  counts[0] = model->numvertices;
  counts[1] = model->numnormals;
  counts[2] = model->numtexcoords;
  counts[3] = ntri;
  counts[4] = ng;
  // glm stores element k (1-based) at [3k..3k+2]
  if (positions) memcpy(positions, model->vertices + 3, sizeof(float) * 3 * model->numvertices);
  if (normals && model->numnormals) memcpy(normals, model->normals + 3, sizeof(float) * 3 * model->numnormals);
  if (texcoords && model->numtexcoords) memcpy(texcoords, model->texcoords + 2, sizeof(float) * 2 * model->numtexcoords);
  glmDelete(model);
  return 1;
}
