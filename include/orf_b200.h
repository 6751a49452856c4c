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
 * results back and synchronizes.  Device scratch is allocated per call.  The batch moves in chunks of
 * 2^19 queries on two streams of its own, so that copies in, kernels and copies out of different
 * chunks overlap (pinned host buffers let the copies run asynchronously); results are identical to
 * one pt_bsdf_queries over the whole batch. */
pt_status pt_bsdf_queries_host(const float* wo_soa, const float* alpha, uint64_t n, uint64_t first_index,
                               uint64_t n_ggx_below, float eta, float* wi_soa, float* f, float* pdf, float* F);
/* Same query batch through host buffers, without allocating any device memory.  This entry point
 * has no counterpart in the reference.  It exists for callers that must not call cudaMalloc: a
 * host application whose device memory is already handed out by its own allocator or pool (for
 * example a renderer that reserved the GPU's memory for its scenes at start-up), and a real-time
 * thread such as an editor's UI thread re-evaluating a material, where cudaMalloc/cudaFree would
 * synchronise the device and stall the frame.  Instead of per-call staging buffers it uses one
 * fixed device array of 65536 queries (2.5 MiB, held by every GPU that loads the library until the
 * process exits); larger batches are rejected with PT_INVALID_ARG.  The first call on a device looks
 * up that array's device address, so make the first call on each device before any stream capture.
 * All calls share the one array: calls that overlap on the GPU (from several host threads) race, so
 * serialise them.  The call is synchronous and allocates nothing; inputs and outputs are host
 * pointers as in pt_bsdf_queries_host, and the results are identical to it. */
pt_status pt_bsdf_queries_host_noalloc(const float* wo_soa, const float* alpha, uint64_t n, uint64_t first_index,
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


/* ---------------------------------------------------------------- scene objects and rendering
 * One pt_ctx per scene: it owns every device buffer (geometry, BVH, materials, lights, the float4
 * accumulation buffer, the wavefront queues) and one CUDA stream. */
typedef struct pt_ctx pt_ctx;

/* Material types: the values of MaterialType (structs.h:209-225) for the shaders this path
 * implements, plus the emitter material that TriangleAreaLight attaches (arealight_shader.cu). */
enum {
  PT_DIFFUSE_SHADER = 0,              /* diffuse_shader.cu            */
  PT_TRANSPARENT_SHADER = 2,          /* transparent_shader.cu        */
  PT_ROUGH_TRANSPARENT_SHADER = 3,    /* rough_transparent_shader.cu  */
  PT_METALLIC_SHADER = 4,             /* metallic_shader.cu           */
  PT_TRANSLUCENT_SHADER = 5,          /* subsurface_scattering_shader.cu */
  PT_ROUGH_TRANSLUCENT_SHADER = 6,    /* rough_subsurface_scattering_shader.cu */
  PT_LAMBERTIAN_INTERFACE_SHADER = 7, /* lambertian_interface_shader.cu */
  PT_ROUGH_DIFFUSE_SHADER = 9,        /* rough_diffuse_shader.cu      */
  PT_AREA_LIGHT_MATERIAL = 100        /* arealight_shader.cu          */
};
/* Microfacet model / normal distribution enums: structs.h:242-261. */
enum { PT_WALTER_MODEL = 0, PT_VISIBLE_NORMALS_MODEL = 1, PT_MULTISCATTERING_MODEL = 2 };
enum { PT_BECKMANN_DISTRIBUTION = 0, PT_GGX_DISTRIBUTION = 1 };

/* mtl["diffuse_color"] (DiffuseMaterial.cpp:16). */
typedef struct pt_diffuse_params { float diffuse_color[3]; } pt_diffuse_params;
/* mtl["ior"] as MyComplex3 (re, im) per RGB, mtl["roughness"] float2, mtl["microfacet_model"],
 * mtl["normal_distribution"] (MetallicMaterial.cpp:19-25).  The shader uses eta = 1 / ior. */
typedef struct pt_metallic_params {
  double ior[6];
  float roughness[2];
  uint32_t microfacet_model;
  uint32_t normal_distribution;
} pt_metallic_params;
/* mtl["ior"], mtl["roughness"], mtl["glass_absorption"], mtl["microfacet_model"],
 * mtl["normal_distribution"] (RoughTransparentMaterial.cpp:20-28). */
typedef struct pt_rough_transparent_params {
  float ior;
  float roughness;
  float glass_absorption[3];
  uint32_t microfacet_model;
  uint32_t normal_distribution;
} pt_rough_transparent_params;
/* mtl["ior"], mtl["glass_absorption"] of TransparentMaterial (TransparentMaterial.cpp:7-20; defaults
 * ior 1.3, absorption 0): smooth glass with Fresnel reflection / refraction and Beer absorption
 * inside (transparent_shader.cu:47-115). */
typedef struct pt_transparent_params {
  float ior;
  float glass_absorption[3];
} pt_transparent_params;
/* mtl["diffuse_color"], mtl["ior"] of LambertianInterfaceMaterial (LambertianInterfaceMaterial.cpp:7-20;
 * defaults 1 and 1.3): a Lambertian base under a smooth dielectric interface
 * (lambertian_interface_shader.cu:51-173). */
typedef struct pt_lambertian_interface_params {
  float diffuse_color[3];
  float ior;
} pt_lambertian_interface_params;
/* mtl["diffuse_color"], mtl["ior"], mtl["roughness"], mtl["normal_distribution"], mtl["microfacet_model"]
 * of RoughDiffuseMaterial (RoughDiffuseMaterial.cpp:7-28; defaults 1, 1.3, (0.1, 0.1), Beckmann,
 * Walter): a Lambertian base under a rough dielectric interface (rough_diffuse_shader.cu:55-292). */
typedef struct pt_rough_diffuse_params {
  float diffuse_color[3];
  float ior;
  float roughness[2];
  uint32_t microfacet_model;
  uint32_t normal_distribution;
} pt_rough_diffuse_params;
/* TranslucentMaterial (TranslucentMaterial.cpp:7-30): scattering and absorption coefficients per
 * RGB channel in 1/mm, the mean cosine of the phase function, the relative index of refraction and
 * the scene-unit scale applied to the coefficients (default 100), plus mtl["dipole_model"]
 * (structs.h:311-316, TranslucentMaterial.cpp:15).  The library derives
 * mtl["scattering_properties"] from them as TranslucentMaterial::computeCoefficients does
 * (TranslucentMaterial.cpp:303-330, ior_outside = 1). */
enum { PT_STANDARD_DIPOLE = 0, PT_DIRECTIONAL_DIPOLE = 1 };
typedef struct pt_translucent_params {
  float scattering[3];
  float absorption[3];
  float meancosine[3];
  float ior;
  float scale;
  uint32_t dipole_model;
} pt_translucent_params;
/* RoughTranslucentMaterial (RoughTranslucentMaterial.cpp:360-395): the translucent parameters plus
 * mtl["roughness"], mtl["microfacet_model"] and mtl["normal_distribution"] of its rough dielectric
 * boundary. */
typedef struct pt_rough_translucent_params {
  float scattering[3];
  float absorption[3];
  float meancosine[3];
  float ior;
  float scale;
  uint32_t dipole_model;
  float roughness[2];
  uint32_t microfacet_model;
  uint32_t normal_distribution;
} pt_rough_translucent_params;
/* gi["radiance"] of a TriangleAreaLight's geometry (Light.cpp:242). */
typedef struct pt_area_light_params { float radiance[3]; } pt_area_light_params;

/* ---------------------------------------------------------------- per-query BSSRDF and walk batches
 * The device functions the shading kernels call, evaluated on a batch of independent queries (for
 * parity checks and for tools that tabulate a material); asynchronous on `stream`. */

/* Dipole BSSRDF values of one translucent material: the per-(hit, probe) terms of the dipole gather
 * (subsurface_scattering_shader.cu:126-173): dipole_bssrdf (dipoles/standard_dipole.h:8-30) of a
 * distance, or dirpole_bssrdf (dipoles/directional_dipole.h:37-72) of (xi, ni, w12, xo, no), as
 * params->dipole_model selects, on the ScatteringMaterialProperties that
 * TranslucentMaterial::computeCoefficients (TranslucentMaterial.cpp:303-330) derives from params.
 * d_in: the standard dipole reads n distances; the directional one 15 x n floats as SoA rows
 * (xi.x, xi.y, xi.z, ni.xyz, w12.xyz, xo.xyz, no.xyz).  precision 0: FP32 in the reference's
 * operation order (what the renders compute), d_S = 3 x n floats (SoA r, g, b); precision 1: the
 * coefficients and the dipole evaluated in FP64, d_S = 3 x n doubles. */
pt_status pt_bssrdf_queries(const pt_translucent_params* params, uint32_t precision, const float* d_in, uint64_t n, void* d_S,
                            void* stream);

/* Multiscattering random walks (Microfacet.h:95-177: MicrofacetGGX.h:412-640,
 * MicrofacetBeckmann.h:445-736) and the complex conductor Fresnel (Fresnel.h:78-91), per query, in
 * the frame of `normal` as the shaders call them. */
enum {
  PT_MSQ_DIELECTRIC_EVAL = 0,    /* microfacet_multiscattering_dielectric_BSDF_eval    */
  PT_MSQ_DIELECTRIC_SAMPLE = 1,  /* microfacet_multiscattering_dielectric_BSDF_sample  */
  PT_MSQ_CONDUCTOR_EVAL = 2,     /* microfacet_multiscattering_conductor_BSDF_eval     */
  PT_MSQ_CONDUCTOR_SAMPLE = 3,   /* microfacet_multiscattering_conductor_BSDF_sample   */
  PT_MSQ_DIFFUSE_EVAL = 4,       /* microfacet_multiscattering_diffuse_BSDF_eval       */
  PT_MSQ_DIFFUSE_SAMPLE = 5,     /* microfacet_multiscattering_diffuse_BSDF_sample     */
  PT_MSQ_CONDUCTOR_FRESNEL = 6,  /* fresnel_MyComplex_R(wi, m, eta)                    */
  PT_MSQ_VISIBLE_NORMAL = 7      /* microfacet_sample_visible_normal (Microfacet.h:76-87) with
                                    (z1, z2) two rnd_tea draws from the query's seed            */
};
typedef struct pt_microfacet_batch {
  uint32_t op;                   /* PT_MSQ_*                                                    */
  uint32_t normal_distribution;  /* PT_BECKMANN_DISTRIBUTION / PT_GGX_DISTRIBUTION              */
  float normal[3];               /* shading normal of every query                                */
  float eta;                     /* dielectric walks: the relative index the shader passes        */
  double ior[6];                 /* conductor walks and Fresnel: complex eta (re, im) per RGB     */
  float rho[3];                  /* diffuse walks: the albedo                                     */
} pt_microfacet_batch;
/* Per query k (SoA arrays of n): d_wi (3 x n), d_wo (3 x n: the evaluated direction; the microfacet
 * normal for PT_MSQ_CONDUCTOR_FRESNEL; unread by the sample ops), d_alpha (ax = ay), d_seed (the tea
 * state, advanced in place), d_order (the eval ops read it as the order bound, 0 = all; the sample
 * ops add the walk's scattering events to it).  d_out (3 x n): the value (the dielectric eval's
 * scalar in all three rows), the sampled direction or microfacet normal, or F; d_weight (3 x n,
 * sample ops; may be NULL): the sampled walk's weight (1 for the dielectric walk and the visible
 * normal). */
pt_status pt_microfacet_queries(const pt_microfacet_batch* batch, const float* d_wi, const float* d_wo, const float* d_alpha,
                                uint32_t* d_seed, uint32_t* d_order, uint64_t n, float* d_out, float* d_weight, void* stream);

/* Counters of the most recent pt_render_frames call. */
typedef struct pt_render_stats {
  uint64_t path_samples;    /* camera samples traced (pixels in the patch x frames)           */
  uint64_t segments;        /* radiance rays traced (closest-hit queries)                     */
  uint64_t shadow_rays;     /* shadow rays traced (any-hit queries)                           */
  uint64_t capped_walks;    /* random walks / Newton loops stopped by their iteration cap     */
  uint64_t clamped_indices; /* light / triangle indices clamped from size to size-1           */
  float gpu_ms;             /* device time of the call (CUDA events on the context stream)    */
  float extend_ms;          /* device time spent in the closest-hit (extend) kernel           */
  uint32_t extend_launches; /* number of extend launches                                      */
  uint32_t kernel_launches; /* all kernels launched by the call                               */
  uint64_t dipole_gathers;  /* dipole gathers evaluated (camera paths entering translucent objects) */
  uint64_t dipole_pairs;    /* (gather, probe) pairs visited by those gathers                 */
  uint64_t gather_overflows;/* gathers dropped because a path's gather stack was full (0)     */
  float gather_ms;          /* device time of the dipole gather kernel (when profiling)       */
} pt_render_stats;

/* The acceleration structure of the last pt_build (no counterpart in the reference, whose OptiX
 * builders report nothing). */
typedef struct pt_build_info {
  uint32_t builder;       /* 0: binned SAH on the host (default); 1: LBVH on the device (option "bvh_builder") */
  uint32_t n_triangles;
  uint32_t bvh2_nodes;    /* child-pair nodes written                                                */
  uint32_t bvh2_depth;    /* levels including the leaves                                             */
  uint32_t wide_nodes;    /* 4-wide nodes (0 when the 4-wide tree is too deep for the traversal)      */
  uint32_t wide_depth;
  float build_ms;         /* wall time of the BVH step of pt_build (the device builder's includes its
                             upload of the triangles and its per-level synchronisations)             */
  float device_ms;        /* device builder: time between CUDA events around its work on the stream */
  float sah_cost;         /* SAH cost of the BVH2: node step cost (option bvh_trav_cost_milli) plus
                             the children's costs weighted by their surface areas, one per triangle
                             in a leaf; computed by pt_get_build_info                                 */
} pt_build_info;

/* Create / destroy a context on CUDA device `device`. */
pt_status pt_context_create(int device, pt_ctx** out);
pt_status pt_context_destroy(pt_ctx* ctx);
/* The context's CUDA stream (cudaStream_t). */
void* pt_context_stream(pt_ctx* ctx);

/* PathTracer parameters: context["max_depth"], ["scene_epsilon"], ["exception_color"]
 * (Integrator.cpp:77-93).  rr_start_depth: the diffuse shader's Russian roulette (p = mean albedo,
 * diffuse_shader.cu:85-104) applies from this depth on; 0 is the reference's behaviour. */
pt_status pt_set_integrator(pt_ctx* ctx, uint32_t max_depth, float scene_epsilon, const float exception_color[3],
                            uint32_t rr_start_depth);
/* PinholeCamera variables eye, U, V, W, patch_origin, patch_dims (Camera.cpp:83-103) and the
 * launch size; the accumulation buffer is (re)allocated to width x height and cleared. */
pt_status pt_set_camera(pt_ctx* ctx, const float eye[3], const float U[3], const float V[3], const float W[3], uint32_t width,
                        uint32_t height, const uint32_t patch_origin[2], const uint32_t patch_dims[2]);
/* ConstantBackground: context["background_color"] (Background.cpp:13). */
pt_status pt_set_background_constant(pt_ctx* ctx, const float color[3]);
/* EnvMapBackground (Background.cpp:57-69): float4 texels (width*height, row-major, row 0 = v 0),
 * looked up bilinearly with REPEAT wrap on every miss (envmap_background.cu:20-23).  The marginal and
 * conditional pdf/cdf tables of env_cameras.cu:23-75 are built on the device.  A LightStruct with
 * light_type 5 (an extension: the environment map as a light, sampled by sample_environment,
 * Envmap.h:66-98) makes the diffuse shader's next-event estimation sample it; misses after such an
 * estimate then add nothing, as emitter hits do. */
pt_status pt_set_envmap(pt_ctx* ctx, const float* rgba, uint32_t width, uint32_t height);
/* EnvMapBackground from a Radiance RGBE file (the loadTexture / loadHDRTexture path of
 * Background.cpp:57-69, HDRLoader.cpp:225-290): the header and run-length-encoded scanlines are read
 * on the host, the 4-byte RGBE texels are uploaded and expanded to float4 on the device (row 0 = the
 * file's last scanline, as loadHDRTexture flips it; alpha 1), then the tables are built as by
 * pt_set_envmap.  A file the reader rejects returns PT_INVALID_ARG and leaves the background as it was
 * (the reference prints the error and installs a 1x1 texture of its default color instead). */
pt_status pt_set_envmap_hdr(pt_ctx* ctx, const char* path);
/* The same file decoded on the host into float4 texels in the same orientation (HDRLoader.cpp:36-190
 * with the flip of :274-284).  With rgba NULL only the size is returned; otherwise rgba holds
 * capacity_floats >= 4 * width * height floats.  Needs no device. */
pt_status pt_hdr_read(const char* path, float* rgba, uint64_t capacity_floats, uint32_t* width, uint32_t* height);
/* Copy the environment tables to host memory (any pointer may be NULL). */
pt_status pt_get_envmap_tables(pt_ctx* ctx, float* marginal_pdf, float* marginal_cdf, float* conditional_pdf, float* conditional_cdf);
/* Environment queries (parity checks): env_lookup of n_dirs directions (3 floats each) into d_looked,
 * and n_samples draws of sample_environment from the rnd_tea seeds in d_seeds (advanced in place)
 * into d_sample_dirs / d_sample_L (3 floats each). */
pt_status pt_env_query(pt_ctx* ctx, const float* d_dirs, uint32_t n_dirs, float* d_looked, uint32_t* d_seeds, uint32_t n_samples,
                       float* d_sample_dirs, float* d_sample_L);
/* Create a material of the given type from its parameter struct; returns its id. */
pt_status pt_material_create(pt_ctx* ctx, uint32_t type, const void* params, size_t params_size, uint32_t* out_id);
/* Replace the parameters of an existing material (same type); takes effect at the next render. */
pt_status pt_material_update(pt_ctx* ctx, uint32_t id, const void* params, size_t params_size);
/* Add a triangle mesh in world space: positions (3 floats per vertex), position indices (3 int32 per
 * triangle), optional normals (3 floats each) and normal indices (3 int32 per triangle, -1 = none),
 * one material id for all its triangles (ObjLoader.cpp:278-373 buffers).  Returns the global index
 * of the mesh's first triangle. */
pt_status pt_mesh_add(pt_ctx* ctx, const float* positions, uint32_t n_vertices, const int32_t* vindex, uint32_t n_triangles,
                      const float* normals, uint32_t n_normals, const int32_t* nindex, uint32_t material_id,
                      uint32_t* out_first_triangle);
/* light_buffer (LightStruct[], 40 B each) and triangle_light_buffer (TriangleLight[], 92 B each) in
 * the reference's byte layout (structs.h:42-103, OptixSceneLoader.cpp:284-347). */
pt_status pt_lights_upload(pt_ctx* ctx, const void* lights, uint32_t n_lights, const void* triangle_lights, uint32_t n_triangle_lights);
/* Build the BVH over all meshes (binned SAH, BVH2 with child-pair nodes) and upload the scene. */
pt_status pt_build(pt_ctx* ctx);
/* Render frames first_frame .. first_frame+n_frames-1 (one camera sample per pixel and frame, seeded
 * with tea<16>(pixel, frame) as path_tracer.cu:48-51) and fold each into the running mean exactly as
 * path_tracer.cu:64-68 does, in frame order.  Replaces the integrator_pass launch of
 * OptixScene::renderScene (OptixScene.cpp:159); asynchronous on the context stream. */
pt_status pt_render_frames(pt_ctx* ctx, uint32_t first_frame, uint32_t n_frames);
/* Copy the float4 accumulation buffer (width*height*4 floats, row-major, y up) to host memory. */
pt_status pt_readback(pt_ctx* ctx, float* host_rgba);
/* Copy the float4 accumulation buffer into caller-owned device memory (width*height*4 floats). */
pt_status pt_readback_device(pt_ctx* ctx, float* d_rgba);
/* Wait for the context's work; returns the first device-side error, if any. */
pt_status pt_sync(pt_ctx* ctx);
/* Counters and timings of the last pt_render_frames (synchronizes). */
pt_status pt_get_render_stats(pt_ctx* ctx, pt_render_stats* out);
/* Launch options (the autotuner's search space) and modes:
 *   "differentiable" 1 = renders keep the forward state pt_render_adjoint needs (default 0)
 *   "extend_mode"  0 = one ray per thread with block-aggregated queue appends,
 *                  1 = persistent warps that refill finished lanes with new rays (default)
 *   "refill"       persistent kernels refill a warp when at least this many lanes are idle (1..32, default 20)
 *   "bin_items"    the sort granularity of the material binning: queue positions per thread, 256 threads
 *                  per chunk (4, 8 or 16; default 8)
 *   "overlap"      1 = each bounce's shading kernels run on two streams and its shadow rays are traced
 *                  beside the next bounce's extend and binning (default); 0 = every launch in order on
 *                  the context stream.  Images are identical either way.
 *   "dual"         1 = a pass without translucent materials splits its paths into chunks of half the
 *                  wavefront and runs them two at a time on two wavefronts with streams of their own
 *                  (default); 0 = one wavefront.  Images are identical either way.
 *   "bvh4"         1 = the persistent kernels walk the 4-wide BVH (default), 0 = the BVH2
 *   "bvh_trav_cost_milli"  SAH cost of a node step x 1000 relative to a triangle test (default 1200) and
 *   "bvh_max_leaf"         the largest leaf the SAH may choose (1..15, default 8): applied by the next pt_build
 *   "bvh_collapse" the 4-wide collapse of either builder: 0 = greedy (the internal child of largest area opened
 *                  first), 1 = SAH-optimal over the BVH2 (dynamic program; default); with
 *   "bvh_wide_cost_milli"  SAH cost of a wide node visit x 1000 for collapse 1 (default 1500): next pt_build
 *   "bvh_treelets" device builder: rounds of treelet restructuring of the LBVH (0..4, default 3; the
 *                  reference's OptiX "Trbvh" builder restructures treelets likewise): next pt_build
 *   "bvh_treelet_min"      device builder: only subtrees of at least this many triangles form treelets
 *                          (default 8): next pt_build
 *   "bvh_builder"  0 = binned SAH on the host threads (default), 1 = LBVH on the device (Morton codes,
 *                  radix sort, Karras hierarchy, SAH leaves, device 4-wide collapse; the reference's
 *                  OptiX builders, OptixSceneLoader.cpp:136, also run on the device): next pt_build */
pt_status pt_set_option(pt_ctx* ctx, const char* name, int64_t value);
/* When enabled, CUDA events bracket every extend (closest-hit) and dipole-gather launch and
 * pt_get_render_stats reports their summed device times in extend_ms and gather_ms.  Off by default (the events serialise nothing
 * but cost a few microseconds per bounce). */
pt_status pt_set_profiling(pt_ctx* ctx, int enable);
/* The acceleration structure of the last pt_build, with its SAH cost evaluated on the host (the
 * device-built tree is read back for that). */
pt_status pt_get_build_info(pt_ctx* ctx, pt_build_info* out);
/* Textures (no counterpart in the reference's shaders, which read constant material parameters; they
 * carry the per-texel parameters of differentiable renders).  A texture is width x height texels of 1
 * or 3 float channels, texel (x, y) channel c at [(y*width + x)*channels + c].  pt_texture_create
 * copies host data into library-owned device memory; pt_texture_bind points a texture at caller-owned
 * device memory of the same shape (not copied: it must stay valid while renders read it);
 * pt_texture_bind_grad gives the device buffer (same layout) that pt_render_adjoint accumulates the
 * texture's gradient into (NULL: none). */
pt_status pt_texture_create(pt_ctx* ctx, const float* host_data, uint32_t width, uint32_t height, uint32_t channels, uint32_t* out_id);
pt_status pt_texture_bind(pt_ctx* ctx, uint32_t texture_id, const float* d_data);
pt_status pt_texture_bind_grad(pt_ctx* ctx, uint32_t texture_id, float* d_grad);
/* A diffuse material's diffuse_color (3-channel texture) or a metallic material's isotropic roughness
 * (1-channel texture; Walter or visible-normal model) read at the nearest texel of a cube map around
 * `center`: the largest component of (hit - center) picks one of six faces, laid out 3 x 2 in the
 * texture, and the other two components divided by it give the face coordinates. */
pt_status pt_material_set_texture(pt_ctx* ctx, uint32_t material_id, uint32_t texture_id, const float center[3]);
/* Gradient buffer (6 device floats: d/d sigma_a RGB, d/d sigma_s' RGB, in the units of
 * pt_translucent_params, sigma_s' = scattering * (1 - meancosine)) of a translucent material
 * (standard dipole) for pt_render_adjoint; NULL to unbind. */
pt_status pt_material_bind_sigma_grad(pt_ctx* ctx, uint32_t material_id, float* d_grad6);
/* Adjoint (path replay backprop; no counterpart in the reference): with the option "differentiable"
 * set, pt_render_frames keeps per camera path its radiance and the value of each dipole gather.
 * pt_render_adjoint then replays the same paths (same random numbers, nothing else stored) and adds
 * to the bound gradient buffers the gradient of a loss whose gradient with respect to the
 * accumulation buffer is d_dimage (device, width*height*4 floats, the w channel ignored).  The
 * differentiated estimator keeps the forward render's sampling fixed (directions, Russian roulette
 * and dipole acceptance with their probabilities); albedo textures enter through next-event
 * estimates and bounce weights, GGX roughness textures through the bounce weights, and sigma_a /
 * sigma_s' through the Beer transmittance inside and the dipole gathers.  Probes are part of the
 * sampling.  Frames must be those of the last differentiable forward render. */
pt_status pt_render_adjoint(pt_ctx* ctx, uint32_t first_frame, uint32_t n_frames, const float* d_dimage);
/* Probe points per translucent object and frame: context["samples"] (SAMPLES_FRAME = 500,
 * OptixSceneLoader.cpp:11-17).  Every frame first runs the probe pass of sample_camera.cu over each
 * translucent object (OptixScene.cpp:146-157), then the camera paths. */
pt_status pt_set_probe_count(pt_ctx* ctx, uint32_t samples);
/* The probe records (PositionSample, structs.h:105-114, 80 bytes each: pos, dir, normal, L,
 * transmitted, weight as float3 plus 8 bytes of padding) of the last frame rendered, object-major
 * (samples_output_buffer, translucent object k at [k*samples, (k+1)*samples)).  Writes at most
 * `capacity` records and the total count to *n_out.  The dir field of probes lit by an indirect path
 * is zero (the reference leaves it unset). */
pt_status pt_get_probes(pt_ctx* ctx, void* out, uint64_t capacity, uint64_t* n_out);
/* The 260-byte ScatteringMaterialProperties (structs.h:116-144) derived for a translucent material. */
pt_status pt_get_scattering_properties(pt_ctx* ctx, uint32_t material_id, void* out260);
/* Upper bound on paths kept in flight by one wavefront pass (frames are grouped to fit). */
pt_status pt_set_max_paths_in_flight(pt_ctx* ctx, uint64_t max_paths);

/* Frame the next batch render of this scene starts at (advanced by pt_render_frames and by batch
 * renders; reset to 0 by pt_set_camera). */
pt_status pt_get_next_frame(pt_ctx* ctx, uint32_t* next_frame);
/* Restores a saved frame (OptixScene::loadBuffer, OptixScene.cpp:253-298): the float4 accumulation
 * buffer (width * height, as pt_readback returns it) and the number of frames it holds, which becomes
 * the next frame, so that pt_render_frames(ctx, next_frame, n) continues the running mean exactly. */
pt_status pt_set_accumulation(pt_ctx* ctx, const float* host_rgba, uint32_t next_frame);

/* ---------------------------------------------------------------- batches of scenes
 * No counterpart in the reference (one OptiX launch per scene).  A batch renders several scenes
 * (built contexts on one device) in one wavefront pass: every scene's frames become items of one
 * path-id space, so small scenes fill the GPU together, and the pass's whole launch sequence is
 * captured once into a CUDA graph and replayed on later renders.  Each scene keeps the semantics of
 * pt_render_frames: a batch render of frames [f, f+n) leaves exactly the image that
 * pt_render_frames(ctx, f, n) would.  The batch works on its own stream; read-backs on a scene's
 * context are ordered after it. */
typedef struct pt_batch pt_batch;
typedef struct pt_tune_result {
  int32_t extend_mode;          /* chosen "extend_mode"                                  */
  int32_t refill;               /* chosen "refill" (rays a warp fetches per refill, 1..32) */
  uint64_t max_paths_in_flight; /* chosen paths per wavefront chunk                     */
  float best_mpaths_per_s;      /* calibration throughput of the winner                 */
  uint32_t trials;              /* configurations timed                                 */
  uint32_t bin_items;           /* chosen "bin_items" (the sort granularity)             */
} pt_tune_result;
pt_status pt_batch_create(int device, pt_batch** out);
pt_status pt_batch_destroy(pt_batch* batch);
/* The batch's CUDA stream (cudaStream_t). */
void* pt_batch_stream(pt_batch* batch);
/* Adds a built scene; each batch render traces frames_per_render frames of it. */
pt_status pt_batch_add(pt_batch* batch, pt_ctx* scene, uint32_t frames_per_render);
/* Options of the batch engine: "extend_mode", "refill" (as pt_set_option), "max_paths_in_flight",
 * "use_graph" (1 = capture and replay the launch sequence, the default), "profile" (1 = CUDA events
 * around every extend and gather launch of a pass without the graph, as pt_set_profiling; their summed
 * times in pt_batch_get_stats). */
pt_status pt_batch_set_option(pt_batch* batch, const char* name, int64_t value);
/* Renders the next frames_per_render frames of every scene (starting at each scene's next frame). */
pt_status pt_batch_render(pt_batch* batch);
/* The same frames rendered scene after scene, each by its own single-scene pass (the plain path), on
 * the batch's buffers: the baseline the batched pass is compared with. */
pt_status pt_batch_render_sequential(pt_batch* batch);
/* Counters and device time of the last batch render (synchronizes). */
pt_status pt_batch_get_stats(pt_batch* batch, pt_render_stats* out);
/* Times short renders (min(frames_per_render, frames_per_trial) frames of every scene) over the
 * engine options -- extend kernel, warp refill threshold, paths per wavefront chunk (the queue tile),
 * then the material binning's positions per thread (the sort granularity) for the winner -- and keeps
 * the fastest.  The trials render from frame 0, so every scene's accumulation restarts at frame 0. */
pt_status pt_batch_autotune(pt_batch* batch, uint32_t frames_per_trial, pt_tune_result* out);

/* ---------------------------------------------------------------- OBJ models (scene ingestion)
 * A Wavefront OBJ file read with the semantics of the reference's glm reader as ObjLoader flattens it
 * (glmReadOBJ, glm.cpp:567-1005 and :1603-1690; ObjLoader::loadVertexData, ObjLoader.cpp:193-260):
 * v / vn / vt records; faces in the forms v, v/t, v//n and v/t/n, polygons fan-triangulated
 * (v0, v[k-1], v[k]); groups named "<g name>_MAT_<usemtl name>" ("No Group" / "No Material" before
 * the first g / usemtl), listed newest first with empty groups dropped, and each group's triangles in
 * file order.  Indices are 0-based; a corner without a normal or texcoord has index -1.  Negative
 * (relative) indices count back from the last record of their kind read so far (glm resolves only
 * vertex indices this way).  A mtllib's newmtl / Kd pairs give each group's diffuse color when its
 * material is defined there.  Needs no device; feed the arrays to pt_mesh_add, one call per group or
 * one for all with one material. */
typedef struct pt_obj pt_obj;
typedef struct pt_obj_info {
  uint32_t n_vertices, n_normals, n_texcoords, n_triangles, n_groups;
} pt_obj_info;
typedef struct pt_obj_group {
  char name[128];       /* "<g>_MAT_<material>" */
  char material[128];   /* the usemtl name */
  uint32_t first_triangle, n_triangles;
  float diffuse[3];     /* Kd of the material, 0.7 (glm's default) when the library does not define it */
  int32_t has_diffuse;  /* 1 if the material library defines Kd for it */
} pt_obj_group;
pt_status pt_obj_read(const char* path, pt_obj** out);
pt_status pt_obj_get_info(const pt_obj* obj, pt_obj_info* info);
/* Any pointer may be NULL.  Sizes: positions / normals 3 floats per record, texcoords 2, the three index
 * arrays 3 int32 per triangle, group_of_triangle 1 per triangle. */
pt_status pt_obj_get_arrays(const pt_obj* obj, float* positions, float* normals, float* texcoords, int32_t* vindex, int32_t* nindex,
                            int32_t* tindex, uint32_t* group_of_triangle);
pt_status pt_obj_get_group(const pt_obj* obj, uint32_t group, pt_obj_group* out);
pt_status pt_obj_free(pt_obj* obj);

/* ---------------------------------------------------------------- ray queries (BVH parity)
 * Closest-hit / any-hit queries against the built scene for n rays given as d_orig_tmin
 * (float4: origin.xyz, tmin) and d_dir_tmax (float4: direction.xyz, tmax).  Closest hit writes the
 * original triangle index (-1 for a miss), t and the barycentrics (beta, gamma) of the hit; ties in t
 * go to the lower triangle index.  Any hit writes 1 if some triangle has tmin < t < tmax, else 0.
 * The disk and sphere lights' geometry counts too: its hits carry index n_triangles + k for the k-th
 * such light in light_buffer order (barycentrics 0), after the triangles in tie order. */
pt_status pt_trace_closest(pt_ctx* ctx, const float* d_orig_tmin, const float* d_dir_tmax, uint32_t n, int32_t* d_prim,
                           float* d_t, float* d_bary);
pt_status pt_trace_any(pt_ctx* ctx, const float* d_orig_tmin, const float* d_dir_tmax, uint32_t n, int32_t* d_hit);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* ORF_B200_H */
