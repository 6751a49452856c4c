/* C ABI of the B200 wavefront path tracer (library: open_rendering_framework_b200/libpt_b200.so).
 *
 * This is the drop-in boundary for the OptiX launch of andrea-luongo/open_rendering_framework.
 * The reference's host classes (Integrator, Camera, Background, Light, MyMaterial) write OptiX
 * variables and buffers and OptixScene::renderScene launches OptiX
 * (open_rendering_framework/OptixScene.cpp:139-168).  Here the same classes call these functions
 * instead; include/orf_b200_scene.hpp holds C++ versions of those classes written over this ABI.
 *
 * Conventions: plain pointers and sizes, no C++ or torch types.  Every entry returns pt_status and
 * never throws.  A context is not thread-safe (one host thread per context); its work is ordered on
 * one CUDA stream.  Pointers named d_* are device pointers (CUDA global memory of the context's
 * device); all others are host pointers, copied before the call returns (no aliasing is kept).
 */
#ifndef ORF_B200_H
#define ORF_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

typedef enum pt_status {
  PT_OK = 0,
  PT_INVALID_ARG = 1,     /* bad pointer, size, enum or parameter value                          */
  PT_OOM = 2,             /* device allocation failed                                            */
  PT_CUDA_ERROR = 3,      /* a CUDA runtime call failed (pt_last_error_message() has the text)   */
  PT_DEVICE_TIMEOUT = 4,  /* a bounded device-side wait gave up                                  */
  PT_CAP_EXCEEDED = 5,    /* a queue or iteration cap was reached (results are still written)    */
  PT_NOT_READY = 6        /* the call needs state that has not been set (scene, camera, ...)    */
} pt_status;

/* Text of the most recent error on this thread (empty string if none). */
const char* pt_last_error_message(void);
/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
int pt_version(void);
/* Number of CUDA kernels this library has launched in this process (all contexts). */
uint64_t pt_kernel_launch_count(void);

/* ---------------------------------------------------------------- batched BSDF queries
 * Replaces, for a batch of independent queries, the per-hit calls of the reference's
 * Microfacet.h dispatchers: microfacet_sample_visible_normal (Microfacet.h:76-87),
 * microfacet_eval_BSDF (Microfacet.h:66-74), microfacet_eval_visible_normal (Microfacet.h:89-101)
 * and fresnel_R (Fresnel.h:42-54).  For query i (global index first_index + k) with outgoing
 * direction wo (shading frame, normal +z) and isotropic roughness alpha:
 *   distribution = GGX if i < n_ggx_below else Beckmann
 *   (u1,u2) = two rnd_tea draws from seed tea<16>(i, 0)   (random.h:25-40, :117-127)
 *   m   = sampled visible microfacet normal;   wi = reflect(-wo, m)
 *   f   = Walter BSDF(wo, wi, n, alpha, eta)
 *   pdf = D_wo(m) / (4 |wo.m|)
 *   F   = dielectric Fresnel(wo, m, eta)
 * Arrays are structure-of-arrays: d_wo_soa = x[n] | y[n] | z[n], same for d_wi_soa.  `stream` is
 * a cudaStream_t (NULL = default stream).  The call is asynchronous. */
pt_status pt_bsdf_queries(const float* d_wo_soa, const float* d_alpha, uint64_t n, uint64_t first_index,
                          uint64_t n_ggx_below, float eta, float* d_wi_soa, float* d_f, float* d_pdf, float* d_F,
                          void* stream);
/* Same query batch through host buffers: copies inputs to the device, runs the kernel, copies the
 * results back and synchronizes.  Device scratch is allocated per call. */
pt_status pt_bsdf_queries_host(const float* wo_soa, const float* alpha, uint64_t n, uint64_t first_index,
                               uint64_t n_ggx_below, float eta, float* wi_soa, float* f, float* pdf, float* F);
/* The synthetic query inputs used by the benchmark (alpha in [0.05,1], cos(theta_o) in [0.01,1],
 * phi in [0,2pi) drawn with rnd_tea from tea<16>(i,1)), generated on the host. */
pt_status pt_c1_make_inputs(uint64_t n, uint64_t first_index, float* wo_soa, float* alpha);

/* ---------------------------------------------------------------- RNG streams (parity checks)
 * Each of the n streams starts from seeds[k] and produces `draws` consecutive values into
 * out[k*draws + j]; the final seed is written back.  kind 0: rnd_tea (random.h:117-127),
 * kind 1: rnd / lcg (random.h:43-61), kind 2: rnd_accurate on a 64-bit MD5 seed
 * (random.h:134-142; seeds are uint2 pairs, so d_seeds holds 2*n words). */
pt_status pt_rng_streams(int kind, uint32_t* d_seeds, uint64_t n, uint32_t draws, float* d_out, void* stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* ORF_B200_H */
