// Test infrastructure (oracle only): a host-side stand-in for the few OptiX 5.1 object-API names that
// the reference's HDRLoader.cpp uses (context, texture sampler and buffer handles with the calls
// loadHDRTexture makes).  It is NOT OptiX code: a buffer is a std::vector<float> that map() exposes,
// and every sampler setting is recorded or ignored.  It exists so that HDRLoader.cpp compiles
// unmodified with g++ and its decoded texels can pin the library's .hdr reader.
#pragma once

#include <memory>
#include <vector>

#include "optixu_math_namespace.h"

enum RTwrapmode { RT_WRAP_REPEAT = 0 };
enum RTtextureindexmode { RT_TEXTURE_INDEX_NORMALIZED_COORDINATES = 0 };
enum RTtexturereadmode { RT_TEXTURE_READ_NORMALIZED_FLOAT = 0 };
enum RTfiltermode { RT_FILTER_NONE = 0, RT_FILTER_LINEAR = 1 };
enum RTbuffertype { RT_BUFFER_INPUT = 1 };
enum RTformat { RT_FORMAT_FLOAT4 = 4 };

namespace optix {

template <class T> struct ShimHandle {
  std::shared_ptr<T> p;
  T* operator->() const { return p.get(); }
};

struct ShimBuffer {
  size_t w = 0, h = 0;
  std::vector<float> texels;  // float4 per element
  void* map() { return texels.data(); }
  void unmap() {}
};
typedef ShimHandle<ShimBuffer> Buffer;

struct ShimTextureSampler {
  Buffer buffer;
  void setWrapMode(unsigned, RTwrapmode) {}
  void setIndexingMode(RTtextureindexmode) {}
  void setReadMode(RTtexturereadmode) {}
  void setMaxAnisotropy(float) {}
  void setMipLevelCount(unsigned) {}
  void setArraySize(unsigned) {}
  void setBuffer(unsigned, unsigned, Buffer b) { buffer = b; }
  void setFilteringModes(RTfiltermode, RTfiltermode, RTfiltermode) {}
};
typedef ShimHandle<ShimTextureSampler> TextureSampler;

struct ShimContext {
  TextureSampler createTextureSampler() { TextureSampler s; s.p = std::make_shared<ShimTextureSampler>(); return s; }
  Buffer createBuffer(RTbuffertype, RTformat, size_t w, size_t h)
  {
    Buffer b;
    b.p = std::make_shared<ShimBuffer>();
    b.p->w = w;
    b.p->h = h;
    b.p->texels.assign(4 * w * h, 0.0f);
    return b;
  }
};
typedef ShimHandle<ShimContext> Context;

}  // namespace optix
