// Scene ingestion behind the C ABI: the Radiance RGBE (.hdr) environment maps that EnvMapBackground
// loads (HDRLoader.cpp:36-190 with loadHDRTexture, HDRLoader.cpp:225-290) and the Wavefront OBJ models
// that ObjLoader reads through glm (glm.cpp:567-1005, ObjLoader.cpp:120-260).
//
// .hdr: the header and the run-length-encoded scanlines are parsed on the host (the RLE is serial per
// scanline); the 4-byte RGBE texels then go to the device as they are (a quarter of the float4 bytes)
// and one kernel expands them to float4 with loadHDRTexture's vertical flip, straight into the
// context's environment texture, ahead of the CDF build.
//
// .obj: one pass over the file kept in memory, with glm's semantics: v / vn / vt records, faces in the
// four index forms (v, v/t, v//n, v/t/n) fan-triangulated, negative vertex indices relative to the
// vertices read so far, and groups named "<g>_MAT_<usemtl>" listed newest first with empty groups
// dropped, triangles group after group as ObjLoader flattens them.
#include <array>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "pt_context.h"

namespace pt {

// ------------------------------------------------------------------ RGBE (.hdr)
struct RgbeImage {
  uint32_t w = 0, h = 0;
  float exposure = 1.0f;
  std::vector<uchar4> texels;  // file order: scanline 0 first
};

static bool read_file(const char* path, std::vector<unsigned char>& bytes, std::string& err)
{
  FILE* f = fopen(path, "rb");
  if (!f) {
    err = std::string("cannot open ") + path + ": " + strerror(errno);
    return false;
  }
  bytes.clear();
  unsigned char buf[1 << 16];
  size_t n;
  while ((n = fread(buf, 1, sizeof buf, f)) > 0) bytes.insert(bytes.end(), buf, buf + n);
  fclose(f);
  return true;
}

// Next line of the header starting at `pos` (without its '\n'); false at the end of the data.
static bool next_line(const std::vector<unsigned char>& b, size_t& pos, std::string& line)
{
  if (pos >= b.size()) return false;
  size_t e = pos;
  while (e < b.size() && b[e] != '\n') ++e;
  line.assign((const char*)b.data() + pos, e - pos);
  pos = e < b.size() ? e + 1 : e;
  return true;
}

// HDRLoader::HDRLoader / ReadScanline (HDRLoader.cpp:36-130): "#?RADIANCE", header lines (comments and
// whitespace-only lines skipped, FORMAT must be 32-bit_rle_rgbe, the last EXPOSURE= wins) up to an
// empty line, the "-Y <h> +X <w>" resolution, then h scanlines, each run-length encoded (new format:
// 2, 2, width high, width low, then four channel planes of runs and literals) or flat RGBE quadruples.
// Unlike the reference, the width test of an RLE scanline reads the two width bytes unsigned (the
// reference sign-extends the low byte and so rejects RLE files whose width has its low byte >= 128),
// and runs that would write past the scanline are an error instead of a buffer overrun.
static bool parse_rgbe(const std::vector<unsigned char>& b, RgbeImage& img, std::string& err)
{
  size_t pos = 0;
  std::string line;
  if (!next_line(b, pos, line) || line != "#?RADIANCE") {
    err = "not a Radiance file (first line is not #?RADIANCE)";
    return false;
  }
  for (;;) {
    if (!next_line(b, pos, line)) {
      err = "premature end of the header";
      return false;
    }
    if (line.empty()) break;
    const size_t i = line.find_first_not_of("\n\r\t ");
    if (i == std::string::npos || line[i] == '#') continue;
    if (line.find("FORMAT") != std::string::npos) {
      if (line != "FORMAT=32-bit_rle_rgbe") {
        err = "only FORMAT=32-bit_rle_rgbe is supported";
        return false;
      }
      continue;
    }
    const size_t ofs = line.find("EXPOSURE=");
    if (ofs != std::string::npos) img.exposure = (float)strtod(line.c_str() + ofs + 9, nullptr);
  }
  do {  // the resolution line follows the empty line (further blank lines are skipped, as stream extraction does)
    if (!next_line(b, pos, line)) {
      err = "missing resolution line";
      return false;
    }
  } while (line.find_first_not_of("\r\t ") == std::string::npos);
  char minor[8] = {0}, major[8] = {0};
  long ny = 0, nx = 0;
  if (sscanf(line.c_str(), "%7s %ld %7s %ld", minor, &ny, major, &nx) != 4 || strcmp(minor, "-Y") != 0 || strcmp(major, "+X") != 0) {
    err = "only the -Y <height> +X <width> orientation is supported";
    return false;
  }
  if (nx <= 0 || ny <= 0 || nx > 65535 || ny > 65535) {
    err = "invalid image dimensions";
    return false;
  }
  if (!(img.exposure > 0.0f) || !std::isfinite(img.exposure)) {
    err = "EXPOSURE must be finite and > 0";
    return false;
  }
  img.w = (uint32_t)nx;
  img.h = (uint32_t)ny;
  img.texels.assign((size_t)nx * ny, make_uchar4(0, 0, 0, 0));
  const size_t n = b.size();
  for (uint32_t y = 0; y < img.h; ++y) {
    uchar4* row = img.texels.data() + (size_t)y * img.w;
    const bool may_rle = img.w >= 8 && img.w <= 0x7fff;
    if (may_rle && pos + 4 > n) {
      err = "premature end of the file in a scanline header";
      return false;
    }
    if (!may_rle || b[pos] != 2 || b[pos + 1] != 2 || (b[pos + 2] & 0x80)) {  // flat RGBE quadruples
      if (pos + 4 * (size_t)img.w > n) {
        err = "premature end of the file in a flat scanline";
        return false;
      }
      memcpy(row, b.data() + pos, 4 * (size_t)img.w);
      pos += 4 * (size_t)img.w;
      continue;
    }
    if ((((uint32_t)b[pos + 2] << 8) | b[pos + 3]) != img.w) {
      err = "RLE scanline width differs from the image width";
      return false;
    }
    pos += 4;
    for (int ch = 0; ch < 4; ++ch) {
      for (uint32_t x = 0; x < img.w;) {
        if (pos >= n) {
          err = "premature end of the file in an RLE scanline";
          return false;
        }
        uint32_t code = b[pos++];
        if (code > 0x80) {  // a run of one byte value
          code &= 0x7f;
          if (pos >= n) {
            err = "premature end of the file in an RLE run";
            return false;
          }
          const unsigned char v = b[pos++];
          if (x + code > img.w) {
            err = "RLE run overruns the scanline";
            return false;
          }
          for (uint32_t k = 0; k < code; ++k) (&row[x++].x)[ch] = v;
        } else {  // `code` literal bytes
          if (x + code > img.w || pos + code > n) {
            err = "RLE literal span overruns the scanline or the file";
            return false;
          }
          for (uint32_t k = 0; k < code; ++k) (&row[x++].x)[ch] = b[pos++];
        }
      }
    }
  }
  return true;
}

// RGBEtoFloats (HDRLoader.cpp:63-75): 0 for a zero exponent, else (c + 0.5) * 2^(e - 136) / exposure.
// The power of two is exact (formed from its bits in double, then narrowed: exact down to 2^-136).
PT_HD float rgbe_scale(unsigned e, float inv_exposure)
{
  const int n = (int)e - 136;
#ifdef __CUDA_ARCH__
  float s = (float)__longlong_as_double((long long)(n + 1023) << 52);
#else
  float s = (float)std::ldexp(1.0, n);
#endif
  s *= inv_exposure;
  return s;
}
PT_HD float4 rgbe_to_float4(uchar4 c, float inv_exposure)
{
  if (c.w == 0) return make_float4(0.0f, 0.0f, 0.0f, 1.0f);
  const float s = rgbe_scale(c.w, inv_exposure);
  return make_float4(((float)c.x + 0.5f) * s, ((float)c.y + 0.5f) * s, ((float)c.z + 0.5f) * s, 1.0f);
}

// texel (i, j) of the texture = file scanline h - 1 - j (loadHDRTexture, HDRLoader.cpp:274-284); the
// reference leaves the fourth channel undefined, here it is 1.
__global__ void k_rgbe_decode(const uchar4* rgbe, float4* out, uint32_t w, uint32_t h, float inv_exposure)
{
  const uint64_t n = (uint64_t)w * h;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t j = (uint32_t)(k / w), i = (uint32_t)(k - (uint64_t)j * w);
    out[k] = rgbe_to_float4(rgbe[(uint64_t)(h - 1 - j) * w + i], inv_exposure);
  }
}

static pt_status load_rgbe(const char* path, RgbeImage& img)
{
  if (!path) return fail(PT_INVALID_ARG, "hdr: null path");
  std::vector<unsigned char> bytes;
  std::string err;
  if (!read_file(path, bytes, err)) return fail(PT_INVALID_ARG, "hdr: " + err);
  if (!parse_rgbe(bytes, img, err)) return fail(PT_INVALID_ARG, std::string("hdr: ") + path + ": " + err);
  // the largest texel value must stay finite: 255.5 * 2^(e_max - 136) / exposure
  unsigned e_max = 0;
  for (const uchar4& c : img.texels) e_max = c.w > e_max ? c.w : e_max;
  if (e_max && !(255.5 * std::ldexp(1.0, (int)e_max - 136) / (double)img.exposure < 3.0e38))
    return fail(PT_INVALID_ARG, "hdr: texel values overflow float (exposure too small)");
  return PT_OK;
}

}  // namespace pt

using namespace pt;

pt_status pt_hdr_read(const char* path, float* rgba, uint64_t capacity_floats, uint32_t* width, uint32_t* height)
{
  if (!width || !height) return fail(PT_INVALID_ARG, "pt_hdr_read: null size pointer");
  RgbeImage img;
  pt_status st = load_rgbe(path, img);
  if (st != PT_OK) return st;
  *width = img.w;
  *height = img.h;
  if (!rgba) return PT_OK;
  const uint64_t n = (uint64_t)img.w * img.h;
  if (capacity_floats < 4 * n) return fail(PT_INVALID_ARG, "pt_hdr_read: buffer smaller than 4 * width * height floats");
  const float inv_exposure = 1.0f / img.exposure;
  for (uint32_t j = 0; j < img.h; ++j)
    for (uint32_t i = 0; i < img.w; ++i) {
      const float4 v = rgbe_to_float4(img.texels[(size_t)(img.h - 1 - j) * img.w + i], inv_exposure);
      float* o = rgba + 4 * ((size_t)j * img.w + i);
      o[0] = v.x;
      o[1] = v.y;
      o[2] = v.z;
      o[3] = v.w;
    }
  return PT_OK;
}

pt_status pt_set_envmap_hdr(pt_ctx* ctx, const char* path)
{
  if (!ctx) return fail(PT_INVALID_ARG, "null context");
  Context& c = ctx->c;
  RgbeImage img;
  pt_status st = load_rgbe(path, img);
  if (st != PT_OK) return st;
  if (img.w < 2 || img.h < 2 || (uint64_t)img.w * img.h > (1ull << 26)) return fail(PT_INVALID_ARG, "pt_set_envmap_hdr: bad size");
  PT_CHECK_CUDA(cudaSetDevice(c.device), "cudaSetDevice");
  const size_t n = (size_t)img.w * img.h;
  DevBuf staging;
  if ((st = staging.reserve(n * sizeof(uchar4), "RGBE staging")) != PT_OK) return st;
  if ((st = env_reserve(c, img.w, img.h)) != PT_OK) return st;
  PT_CHECK_CUDA(cudaMemcpyAsync(staging.p, img.texels.data(), n * sizeof(uchar4), cudaMemcpyHostToDevice, c.stream), "RGBE upload");
  k_rgbe_decode<<<grid_for(n, 256, 8), 256, 0, c.stream>>>(staging.as<uchar4>(), c.d_env_tex.as<float4>(), img.w, img.h, 1.0f / img.exposure);
  count_launch();
  PT_CHECK_CUDA(cudaGetLastError(), "pt_set_envmap_hdr decode");
  st = env_build_tables(c, img.w, img.h);
  if (st != PT_OK) return st;
  PT_CHECK_CUDA(cudaStreamSynchronize(c.stream), "pt_set_envmap_hdr");  // before the staging buffer is freed
  return PT_OK;
}

// ------------------------------------------------------------------ Wavefront OBJ
struct pt_obj {
  std::vector<float> pos, nrm, tex;
  std::vector<int32_t> vidx, nidx, tidx;  // 0-based, -1 = none
  std::vector<uint32_t> group_of;
  struct Group {
    std::string name, mtlname;
    uint32_t first = 0, count = 0;
    float kd[3] = {0.7f, 0.7f, 0.7f};
    int has_kd = 0;
  };
  std::vector<Group> groups;
};

namespace {

struct Tok {
  const char* p;
  const char* e;
};
// Whitespace-separated tokens of one line.
static void split(const char* b, const char* e, std::vector<Tok>& out)
{
  out.clear();
  while (b < e) {
    while (b < e && (*b == ' ' || *b == '\t' || *b == '\r' || *b == '\f' || *b == '\v')) ++b;
    if (b >= e) break;
    const char* s = b;
    while (b < e && !(*b == ' ' || *b == '\t' || *b == '\r' || *b == '\f' || *b == '\v')) ++b;
    out.push_back(Tok{s, b});
  }
}
static bool tok_float(const Tok& t, float& v)
{
  char buf[64];
  const size_t n = (size_t)(t.e - t.p);
  if (n == 0 || n >= sizeof buf) return false;
  memcpy(buf, t.p, n);
  buf[n] = 0;
  char* end = nullptr;
  v = strtof(buf, &end);  // the conversion fscanf("%f") performs
  return end != buf;
}
// A decimal integer with an optional sign at p (advanced past it).
static bool parse_long(const char*& p, const char* e, long& v)
{
  bool neg = false;
  if (p < e && (*p == '-' || *p == '+')) neg = *p++ == '-';
  if (p >= e || *p < '0' || *p > '9') return false;
  long x = 0;
  while (p < e && *p >= '0' && *p <= '9') x = x * 10 + (*p++ - '0');
  v = neg ? -x : x;
  return true;
}
// One face corner in the form `form` (0: v, 1: v/t, 2: v//n, 3: v/t/n); false if it does not parse.
static bool corner(const Tok& t, int form, long& v, long& tt, long& n)
{
  const char* p = t.p;
  if (!parse_long(p, t.e, v)) return false;
  switch (form) {
    case 0: return p == t.e;
    case 1: return p < t.e && *p++ == '/' && parse_long(p, t.e, tt) && p == t.e;
    case 2: return p + 1 < t.e && p[0] == '/' && p[1] == '/' && (p += 2, parse_long(p, t.e, n)) && p == t.e;
    default: return p < t.e && *p++ == '/' && parse_long(p, t.e, tt) && p < t.e && *p++ == '/' && parse_long(p, t.e, n) && p == t.e;
  }
}
// The index form of a face's first corner (glm.cpp:853-856 tests "//", then v/t/n, then v/t).
static int face_form(const Tok& t)
{
  int slashes = 0;
  for (const char* p = t.p; p < t.e; ++p) {
    if (*p == '/') {
      if (p + 1 < t.e && p[1] == '/') return 2;
      ++slashes;
    }
  }
  return slashes >= 2 ? 3 : slashes == 1 ? 1 : 0;
}

struct ObjGroupBuild {
  std::string name, mtlname;
  std::vector<uint32_t> tris;  // indices into the model's triangle list
};

// newmtl / Kd of a material library (glm.cpp:279-510; only the diffuse color is kept).
static void read_mtl(const std::string& path, std::vector<std::pair<std::string, std::vector<float>>>& mats)
{
  std::vector<unsigned char> b;
  std::string err;
  if (!read_file(path.c_str(), b, err)) return;
  size_t pos = 0;
  std::string line;
  std::vector<Tok> tk;
  while (next_line(b, pos, line)) {
    split(line.data(), line.data() + line.size(), tk);
    if (tk.empty()) continue;
    std::string key(tk[0].p, tk[0].e);
    if (key == "newmtl" && tk.size() >= 2) mats.push_back({std::string(tk[tk.size() >= 3 ? 2 : 1].p, tk[tk.size() >= 3 ? 2 : 1].e), {}});
    else if (key == "Kd" && !mats.empty() && tk.size() >= 4) {
      float r, g, bl;
      if (tok_float(tk[1], r) && tok_float(tk[2], g) && tok_float(tk[3], bl)) mats.back().second = {r, g, bl};
    }
  }
}

static pt_status parse_obj(const char* path, pt_obj& m)
{
  std::vector<unsigned char> b;
  std::string err;
  if (!read_file(path, b, err)) return fail(PT_INVALID_ARG, "obj: " + err);
  std::string dir(path);
  const size_t slash = dir.find_last_of("/\\");
  dir = slash == std::string::npos ? std::string() : dir.substr(0, slash + 1);

  struct Tri { long v[3], t[3], n[3]; };
  std::vector<Tri> tris;
  std::vector<ObjGroupBuild> groups;  // in creation order
  std::vector<std::pair<std::string, std::vector<float>>> mats;
  auto group_index = [&](const std::string& name) -> size_t {
    for (size_t k = 0; k < groups.size(); ++k)
      if (groups[k].name == name) return k;
    groups.push_back(ObjGroupBuild{name, std::string(), {}});
    return groups.size() - 1;
  };
  std::string grpname = "No Group", mtlname = "No Material";
  size_t cur = group_index(grpname);
  long nv = 0, nn = 0, nt = 0;
  std::vector<Tok> tk;
  std::vector<std::array<long, 3>> cs;
  const char* const data = (const char*)b.data();
  for (size_t pos = 0; pos < b.size();) {
    const char* lb = data + pos;
    const char* le = (const char*)memchr(lb, '\n', b.size() - pos);
    if (!le) le = data + b.size();
    pos = (size_t)(le - data) + 1;
    split(lb, le, tk);
    if (tk.empty()) continue;
    const std::string key(tk[0].p, tk[0].e);
    if (key[0] == '#') continue;
    if (key == "v" || key == "vn") {
      float x = 0, y = 0, z = 0;
      if (tk.size() < 4 || !tok_float(tk[1], x) || !tok_float(tk[2], y) || !tok_float(tk[3], z))
        return fail(PT_INVALID_ARG, std::string("obj: malformed ") + key + " record in " + path);
      std::vector<float>& dst = key == "v" ? m.pos : m.nrm;
      dst.push_back(x);
      dst.push_back(y);
      dst.push_back(z);
      (key == "v" ? nv : nn)++;
    } else if (key == "vt") {
      float u = 0, v = 0;
      if (tk.size() < 3 || !tok_float(tk[1], u) || !tok_float(tk[2], v)) return fail(PT_INVALID_ARG, std::string("obj: malformed vt record in ") + path);
      m.tex.push_back(u);
      m.tex.push_back(v);
      ++nt;
    } else if (key == "mtllib" && tk.size() >= 2) {
      read_mtl(dir + std::string(tk[tk.size() >= 3 ? 2 : 1].p, tk[tk.size() >= 3 ? 2 : 1].e), mats);
    } else if (key == "usemtl") {  // glm.cpp:821-833: the group "<g>_MAT_<material>"
      if (tk.size() >= 2) mtlname.assign(tk[tk.size() >= 3 ? 2 : 1].p, tk[tk.size() >= 3 ? 2 : 1].e);
      cur = group_index(grpname + "_MAT_" + mtlname);
      groups[cur].mtlname = mtlname;
    } else if (key == "g") {  // glm.cpp:838-848
      grpname = tk.size() >= 2 ? std::string(tk[1].p, tk[1].e) : std::string();
      cur = group_index(grpname + "_MAT_" + mtlname);
      groups[cur].mtlname = mtlname;
    } else if (key == "f") {  // glm.cpp:850-990: fan triangulation, forms fixed by the first corner
      if (tk.size() < 4) return fail(PT_INVALID_ARG, std::string("obj: face with fewer than 3 corners in ") + path);
      const int form = face_form(tk[1]);
      cs.clear();
      for (size_t k = 1; k < tk.size(); ++k) {
        long v = 0, t = 0, n = 0;
        if (!corner(tk[k], form, v, t, n)) break;
        // negative indices count back from the last record read so far (glm.cpp resolves vertices this
        // way and leaves negative normal / texcoord indices unresolved; here all three are resolved)
        if (v < 0) v = nv + 1 + v;
        if (t < 0) t = nt + 1 + t;
        if (n < 0) n = nn + 1 + n;
        cs.push_back({v, form == 1 || form == 3 ? t : 0, form >= 2 ? n : 0});
      }
      if (cs.size() < 3) return fail(PT_INVALID_ARG, std::string("obj: face with fewer than 3 readable corners in ") + path);
      for (size_t k = 2; k < cs.size(); ++k) {
        Tri T;
        const std::array<long, 3>* c3[3] = {&cs[0], &cs[k - 1], &cs[k]};
        for (int q = 0; q < 3; ++q) {
          T.v[q] = (*c3[q])[0];
          T.t[q] = (*c3[q])[1];
          T.n[q] = (*c3[q])[2];
        }
        groups[cur].tris.push_back((uint32_t)tris.size());
        tris.push_back(T);
      }
    }
    // o, s, l, p and unknown records are ignored, as glm does
  }
  // ObjLoader::loadVertexData walks glm's group list (newest first) and skips empty groups
  for (size_t gi = groups.size(); gi-- > 0;) {
    const ObjGroupBuild& g = groups[gi];
    if (g.tris.empty()) continue;
    pt_obj::Group G;
    G.name = g.name;
    G.mtlname = g.mtlname;
    G.first = (uint32_t)m.vidx.size() / 3;
    G.count = (uint32_t)g.tris.size();
    for (const auto& mt : mats)
      if (mt.first == g.mtlname && mt.second.size() == 3) {
        G.kd[0] = mt.second[0];
        G.kd[1] = mt.second[1];
        G.kd[2] = mt.second[2];
        G.has_kd = 1;
      }
    const uint32_t gid = (uint32_t)m.groups.size();
    for (uint32_t ti : g.tris) {
      const Tri& T = tris[ti];
      for (int q = 0; q < 3; ++q) {
        if (T.v[q] < 1 || T.v[q] > nv) return fail(PT_INVALID_ARG, std::string("obj: vertex index out of range in ") + path);
        if (T.n[q] < 0 || T.n[q] > nn || T.t[q] < 0 || T.t[q] > nt)
          return fail(PT_INVALID_ARG, std::string("obj: normal or texcoord index out of range in ") + path);
        m.vidx.push_back((int32_t)(T.v[q] - 1));
        m.nidx.push_back((int32_t)(T.n[q] - 1));
        m.tidx.push_back((int32_t)(T.t[q] - 1));
      }
      m.group_of.push_back(gid);
    }
    m.groups.push_back(G);
  }
  return PT_OK;
}

}  // namespace

pt_status pt_obj_read(const char* path, pt_obj** out)
{
  if (!path || !out) return fail(PT_INVALID_ARG, "pt_obj_read: null argument");
  *out = nullptr;
  pt_obj* m = new (std::nothrow) pt_obj();
  if (!m) return fail(PT_OOM, "pt_obj_read: out of host memory");
  pt_status st;
  try {
    st = parse_obj(path, *m);
  } catch (const std::bad_alloc&) {
    st = fail(PT_OOM, "pt_obj_read: out of host memory");
  }
  if (st != PT_OK) {
    delete m;
    return st;
  }
  *out = m;
  return PT_OK;
}

pt_status pt_obj_get_info(const pt_obj* m, pt_obj_info* info)
{
  if (!m || !info) return fail(PT_INVALID_ARG, "pt_obj_get_info: null argument");
  info->n_vertices = (uint32_t)(m->pos.size() / 3);
  info->n_normals = (uint32_t)(m->nrm.size() / 3);
  info->n_texcoords = (uint32_t)(m->tex.size() / 2);
  info->n_triangles = (uint32_t)(m->vidx.size() / 3);
  info->n_groups = (uint32_t)m->groups.size();
  return PT_OK;
}

pt_status pt_obj_get_arrays(const pt_obj* m, float* positions, float* normals, float* texcoords, int32_t* vindex, int32_t* nindex,
                            int32_t* tindex, uint32_t* group_of_triangle)
{
  if (!m) return fail(PT_INVALID_ARG, "pt_obj_get_arrays: null model");
  if (positions) memcpy(positions, m->pos.data(), m->pos.size() * sizeof(float));
  if (normals) memcpy(normals, m->nrm.data(), m->nrm.size() * sizeof(float));
  if (texcoords) memcpy(texcoords, m->tex.data(), m->tex.size() * sizeof(float));
  if (vindex) memcpy(vindex, m->vidx.data(), m->vidx.size() * sizeof(int32_t));
  if (nindex) memcpy(nindex, m->nidx.data(), m->nidx.size() * sizeof(int32_t));
  if (tindex) memcpy(tindex, m->tidx.data(), m->tidx.size() * sizeof(int32_t));
  if (group_of_triangle) memcpy(group_of_triangle, m->group_of.data(), m->group_of.size() * sizeof(uint32_t));
  return PT_OK;
}

pt_status pt_obj_get_group(const pt_obj* m, uint32_t group, pt_obj_group* out)
{
  if (!m || !out) return fail(PT_INVALID_ARG, "pt_obj_get_group: null argument");
  if (group >= m->groups.size()) return fail(PT_INVALID_ARG, "pt_obj_get_group: no such group");
  const pt_obj::Group& G = m->groups[group];
  memset(out, 0, sizeof(*out));
  strncpy(out->name, G.name.c_str(), sizeof(out->name) - 1);
  strncpy(out->material, G.mtlname.c_str(), sizeof(out->material) - 1);
  out->first_triangle = G.first;
  out->n_triangles = G.count;
  out->has_diffuse = G.has_kd;
  for (int k = 0; k < 3; ++k) out->diffuse[k] = G.kd[k];
  return PT_OK;
}

pt_status pt_obj_free(pt_obj* m)
{
  delete m;
  return PT_OK;
}
