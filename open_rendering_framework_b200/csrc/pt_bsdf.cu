// Config-1 kernel: batched microfacet BSDF queries (sample visible normal, Walter BSDF value,
// sampling pdf, Fresnel term) and the RNG-stream kernels used for bit-exact stream parity.
//
// Layout: structure-of-arrays, 16 B read (wo.xyz + alpha) and 24 B written (wi.xyz, f, pdf, F) per
// query, all coalesced.  The kernel is ALU-bound (16-round TEA, transcendentals, the Beckmann
// Newton loop in double/float), so it runs a grid-stride loop over a grid sized to a multiple of the
// SM count; queries are ordered GGX-then-Beckmann and each distribution's range is its own launch of
// a kernel specialised on it (Beckmann: two launches, sampling then evaluation).
#include <mutex>
#include <vector>

#include "pt_common.cuh"
#include "pt_math.cuh"

namespace pt {

__device__ unsigned long long g_bsdf_capped = 0;

// One launch per distribution: a kernel instance holds only its own distribution's code, so an SM
// never runs GGX and Beckmann warps side by side (a single kernel over the mixed batch thrashed the
// instruction cache: "no instruction" was its top stall).  Queries k in [k_begin, k_end) of the batch.
// kPart 0: the whole query.  kPart 1 / 2: the Beckmann launch in two halves with smaller code each --
// 1 samples the microfacet normal m and the direction wi (m parked in f, pdf, F), 2 evaluates f, pdf
// and F from wo, wi and m.
template <uint32_t kDist, int kPart = 0>
__global__ void __launch_bounds__(256) k_bsdf_queries(const float* __restrict__ wo_soa, const float* __restrict__ alpha, uint64_t n,
                                                      uint64_t k_begin, uint64_t k_end, uint64_t first, float eta,
                                                      float* __restrict__ wi_soa, float* __restrict__ f_out, float* __restrict__ pdf_out,
                                                      float* __restrict__ F_out)
{
  // Programmatic dependent launch: the GGX and sampling grids let the next launch of the stream place
  // its blocks while their own last blocks drain; the evaluation grid reads the sampling grid's
  // outputs, so it first waits for that grid to complete with its writes visible, and the sampling grid
  // waits for the GGX grid before it exits, so that the evaluation grid's completion implies all three
  // (griddepcontrol.wait is a no-op in a grid launched without a programmatic dependency).
  if constexpr (kPart == 2)
    asm volatile("griddepcontrol.wait;" ::: "memory");
  else
    asm volatile("griddepcontrol.launch_dependents;");
  const float3 nrm = f3(0.0f, 0.0f, 1.0f);
  for (uint64_t k = k_begin + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < k_end; k += (uint64_t)gridDim.x * blockDim.x) {
    float3 wo = f3(__ldg(wo_soa + k), __ldg(wo_soa + n + k), __ldg(wo_soa + 2 * n + k));
    float a = __ldg(alpha + k);
    float3 m, wi;
    if constexpr (kPart != 2) {
      uint64_t i = first + k;
      uint32_t s = tea16((uint32_t)i, 0u);
      float u1 = rnd_tea(s);
      float u2 = rnd_tea(s);
      int capped = 0;
      m = sample_visible_normal(kDist, wo, nrm, a, a, u1, u2, &capped);
      wi = reflect(-wo, m);
      wi_soa[k] = wi.x;
      wi_soa[n + k] = wi.y;
      wi_soa[2 * n + k] = wi.z;
      if (capped) atomicAdd(&g_bsdf_capped, 1ull);
    } else {
      m = f3(f_out[k], pdf_out[k], F_out[k]);
      wi = f3(wi_soa[k], wi_soa[n + k], wi_soa[2 * n + k]);
    }
    if constexpr (kPart == 1) {
      f_out[k] = m.x;
      pdf_out[k] = m.y;
      F_out[k] = m.z;
    } else {
      f_out[k] = walter_bsdf(kDist, wo, wi, nrm, a, eta);
      pdf_out[k] = eval_visible_normal(kDist, wo, m, nrm, a, a) / (4.0f * fabsf(dot(wo, m)));
      F_out[k] = fresnel_R(wo, m, eta);
    }
  }
  if constexpr (kPart == 1) asm volatile("griddepcontrol.wait;" ::: "memory");
}

__global__ void k_rng_streams(int kind, uint32_t* seeds, uint64_t n, uint32_t draws, float* out)
{
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n; k += (uint64_t)gridDim.x * blockDim.x) {
    float* o = out + k * draws;
    if (kind == 2) {
      uint2 s = make_uint2(seeds[2 * k], seeds[2 * k + 1]);
      for (uint32_t j = 0; j < draws; ++j) o[j] = rnd_md5(s);
      seeds[2 * k] = s.x;
      seeds[2 * k + 1] = s.y;
    } else {
      uint32_t s = seeds[k];
      if (kind == 0)
        for (uint32_t j = 0; j < draws; ++j) o[j] = rnd_tea(s);
      else
        for (uint32_t j = 0; j < draws; ++j) o[j] = rnd_lcg(s);
      seeds[k] = s;
    }
  }
}

// Queries per chunk of pt_bsdf_queries_host's copy / compute pipeline (20 MiB of device staging each).
constexpr uint64_t kHostChunkQueries = 1ull << 19;

// Staging area of pt_bsdf_queries_host_noalloc: room for kNoAllocMaxQueries queries, laid out as
// wo (3n) | alpha (n) | wi (3n) | f (n) | pdf (n) | F (n).  Every GPU that loads this library holds
// it (2.5 MiB) until the process exits.
constexpr uint64_t kNoAllocMaxQueries = 65536;
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocMaxQueries * 10];

// Device address of g_noalloc_scratch per device, looked up on the first call on that device.  The
// symbol's name in host code only stands for the device array; its device address must come from
// cudaGetSymbolAddress with that device current.
static std::mutex g_noalloc_mu;
static std::vector<float*> g_noalloc_ptr;

static pt_status noalloc_scratch(float** out)
{
  int dev = 0;
  PT_CHECK_CUDA(cudaGetDevice(&dev), "pt_bsdf_queries_host_noalloc cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if ((int)g_noalloc_ptr.size() <= dev) g_noalloc_ptr.resize(dev + 1, nullptr);
  if (!g_noalloc_ptr[dev]) {
    float* p = nullptr;
    PT_CHECK_CUDA(cudaGetSymbolAddress((void**)&p, g_noalloc_scratch), "pt_bsdf_queries_host_noalloc cudaGetSymbolAddress");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return PT_OK;
}

}  // namespace pt

using namespace pt;

extern "C" {

pt_status pt_bsdf_queries(const float* d_wo_soa, const float* d_alpha, uint64_t n, uint64_t first_index, uint64_t n_ggx_below, float eta,
                          float* d_wi_soa, float* d_f, float* d_pdf, float* d_F, void* stream)
{
  if (n == 0) return PT_OK;
  if (!d_wo_soa || !d_alpha || !d_wi_soa || !d_f || !d_pdf || !d_F) return fail(PT_INVALID_ARG, "pt_bsdf_queries: null pointer");
  if (!(eta > 0.0f)) return fail(PT_INVALID_ARG, "pt_bsdf_queries: eta must be > 0");
  // queries with global index first + k < n_ggx_below are GGX, the rest Beckmann
  const uint64_t n_ggx = n_ggx_below <= first_index ? 0 : (n_ggx_below - first_index < n ? n_ggx_below - first_index : n);
  const int block = 256;
  cudaStream_t st = (cudaStream_t)stream;
  if (n_ggx > 0) {
    k_bsdf_queries<GGX><<<grid_for(n_ggx, block, 8), block, 0, st>>>(d_wo_soa, d_alpha, n, 0, n_ggx, first_index, eta, d_wi_soa, d_f, d_pdf,
                                                                     d_F);
    count_launch();
    PT_CHECK_CUDA(cudaGetLastError(), "pt_bsdf_queries launch (GGX)");
  }
  if (n_ggx < n) {
    // the Beckmann queries in two launches (sample, then evaluate): each kernel's code fits the
    // instruction cache better than the whole query's (+6.6 % on the 2^22-query batch).  Each launch
    // that follows one of this function's own is programmatic: the sampling grid reads only the inputs
    // (complete before the GGX grid began, which was launched in stream order) and writes outside the
    // GGX range; the evaluation grid waits in-kernel for the sampling grid.
    cudaLaunchAttribute pdl[1];
    pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    pdl[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid_for(n - n_ggx, block, 8));
    cfg.blockDim = dim3(block);
    cfg.stream = st;
    cfg.attrs = pdl;
    cfg.numAttrs = n_ggx > 0 ? 1 : 0;
    PT_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_bsdf_queries<BECKMANN, 1>, d_wo_soa, d_alpha, n, n_ggx, n, first_index, eta, d_wi_soa, d_f,
                                     d_pdf, d_F),
                  "pt_bsdf_queries launch (Beckmann sampling)");
    cfg.numAttrs = 1;
    PT_CHECK_CUDA(cudaLaunchKernelEx(&cfg, k_bsdf_queries<BECKMANN, 2>, d_wo_soa, d_alpha, n, n_ggx, n, first_index, eta, d_wi_soa, d_f,
                                     d_pdf, d_F),
                  "pt_bsdf_queries launch (Beckmann evaluation)");
    count_launch(2);
  }
  return PT_OK;
}

pt_status pt_bsdf_queries_host(const float* wo_soa, const float* alpha, uint64_t n, uint64_t first_index, uint64_t n_ggx_below, float eta,
                               float* wi_soa, float* f, float* pdf, float* F)
{
  if (n == 0) return PT_OK;
  if (!wo_soa || !alpha || !wi_soa || !f || !pdf || !F) return fail(PT_INVALID_ARG, "pt_bsdf_queries_host: null pointer");
  // The batch goes through in chunks on two streams, so that one chunk's inputs are copied in while
  // another's queries run and a third's results are copied out (the copy engines of the two directions
  // and the SMs work at once).  Chunk c of m queries starts at query k0 and has its own structure-of-
  // arrays block of 10 m floats on the device: wo (3m) | alpha (m) | wi (3m) | f | pdf | F.  A query's
  // result does not depend on the chunking (its seed is its global index first_index + k).
  float* d = nullptr;
  PT_CHECK_CUDA(cudaMalloc(&d, (size_t)n * 10 * sizeof(float)), "pt_bsdf_queries_host cudaMalloc");
  cudaStream_t s[2] = {nullptr, nullptr};
  pt_status st = PT_OK;
  for (int i = 0; i < 2 && st == PT_OK; ++i) {
    cudaError_t e = cudaStreamCreateWithFlags(&s[i], cudaStreamNonBlocking);
    if (e != cudaSuccess) st = cuda_status(e, "pt_bsdf_queries_host stream");
  }
  const uint64_t chunk = kHostChunkQueries;
  for (uint64_t k0 = 0, c = 0; k0 < n && st == PT_OK; k0 += chunk, ++c) {
    const uint64_t m = n - k0 < chunk ? n - k0 : chunk;
    float* b = d + k0 * 10;
    float *d_wo = b, *d_a = b + 3 * m, *d_wi = b + 4 * m, *d_f = b + 7 * m, *d_pdf = b + 8 * m, *d_F = b + 9 * m;
    cudaStream_t cs = s[c & 1];
    const size_t mb = m * sizeof(float);
    cudaError_t e = cudaSuccess;
    for (int j = 0; j < 3 && e == cudaSuccess; ++j) e = cudaMemcpyAsync(d_wo + j * m, wo_soa + j * n + k0, mb, cudaMemcpyHostToDevice, cs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_a, alpha + k0, mb, cudaMemcpyHostToDevice, cs);
    if (e != cudaSuccess) {
      st = cuda_status(e, "pt_bsdf_queries_host H2D");
      break;
    }
    st = pt_bsdf_queries(d_wo, d_a, m, first_index + k0, n_ggx_below, eta, d_wi, d_f, d_pdf, d_F, cs);
    if (st != PT_OK) break;
    for (int j = 0; j < 3 && e == cudaSuccess; ++j) e = cudaMemcpyAsync(wi_soa + j * n + k0, d_wi + j * m, mb, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(f + k0, d_f, mb, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(pdf + k0, d_pdf, mb, cudaMemcpyDeviceToHost, cs);
    if (e == cudaSuccess) e = cudaMemcpyAsync(F + k0, d_F, mb, cudaMemcpyDeviceToHost, cs);
    if (e != cudaSuccess) st = cuda_status(e, "pt_bsdf_queries_host D2H");
  }
  // wait for both streams whatever happened above, so that no copy still runs into the caller's buffers
  for (int i = 0; i < 2; ++i) {
    if (!s[i]) continue;
    const cudaError_t e = cudaStreamSynchronize(s[i]);
    if (e != cudaSuccess && st == PT_OK) st = cuda_status(e, "pt_bsdf_queries_host synchronize");
    cudaStreamDestroy(s[i]);
  }
  cudaFree(d);
  return st;
}

pt_status pt_bsdf_queries_host_noalloc(const float* wo_soa, const float* alpha, uint64_t n, uint64_t first_index, uint64_t n_ggx_below,
                                       float eta, float* wi_soa, float* f, float* pdf, float* F)
{
  if (n == 0) return PT_OK;
  if (n > kNoAllocMaxQueries)
    return fail(PT_INVALID_ARG, "pt_bsdf_queries_host_noalloc: at most 65536 queries per call (the staging area is a fixed 2.5 MiB "
                                "device array); split the batch or use pt_bsdf_queries_host");
  if (!wo_soa || !alpha || !wi_soa || !f || !pdf || !F) return fail(PT_INVALID_ARG, "pt_bsdf_queries_host_noalloc: null pointer");
  float* d = nullptr;
  pt_status st = noalloc_scratch(&d);
  if (st != PT_OK) return st;
  // Every output element k < n is written by the kernel, and the inputs are copied in before it
  // runs, so nothing left over from an earlier call is read and nothing needs clearing.
  float *d_wo = d, *d_a = d + 3 * n, *d_wi = d + 4 * n, *d_f = d + 7 * n, *d_pdf = d + 8 * n, *d_F = d + 9 * n;
  cudaError_t e = cudaMemcpy(d_wo, wo_soa, 3 * n * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_a, alpha, n * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_status(e, "pt_bsdf_queries_host_noalloc H2D");
  st = pt_bsdf_queries(d_wo, d_a, n, first_index, n_ggx_below, eta, d_wi, d_f, d_pdf, d_F, nullptr);
  if (st != PT_OK) return st;
  e = cudaMemcpy(wi_soa, d_wi, 3 * n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(f, d_f, n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(pdf, d_pdf, n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(F, d_F, n * sizeof(float), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(e, "pt_bsdf_queries_host_noalloc D2H");
  return PT_OK;
}

pt_status pt_c1_make_inputs(uint64_t n, uint64_t first_index, float* wo_soa, float* alpha)
{
  if (n && (!wo_soa || !alpha)) return fail(PT_INVALID_ARG, "pt_c1_make_inputs: null pointer");
  for (uint64_t k = 0; k < n; ++k) {
    uint32_t s = tea16((uint32_t)(first_index + k), 1u);
    float a = 0.05f + 0.95f * rnd_tea(s);
    float ct = 0.01f + 0.99f * rnd_tea(s);
    float phi = 2.0f * kPi * rnd_tea(s);
    float st = sqrtf(1.0f - ct * ct);
    alpha[k] = a;
    wo_soa[k] = st * cosf(phi);
    wo_soa[n + k] = st * sinf(phi);
    wo_soa[2 * n + k] = ct;
  }
  return PT_OK;
}

pt_status pt_rng_streams(int kind, uint32_t* d_seeds, uint64_t n, uint32_t draws, float* d_out, void* stream)
{
  if (kind < 0 || kind > 2) return fail(PT_INVALID_ARG, "pt_rng_streams: kind must be 0, 1 or 2");
  if (n == 0) return PT_OK;
  if (!d_seeds || !d_out) return fail(PT_INVALID_ARG, "pt_rng_streams: null pointer");
  int grid = grid_for(n, 256, 8);
  k_rng_streams<<<grid, 256, 0, (cudaStream_t)stream>>>(kind, d_seeds, n, draws, d_out);
  count_launch();
  PT_CHECK_CUDA(cudaGetLastError(), "pt_rng_streams launch");
  return PT_OK;
}

}  // extern "C"
