/*
 * volprim_b200 — C ABI of the B200-native per-ray hot path of a volumetric path tracer for
 * Gaussian kernel-mixture volumes (analog decomposition tracking + NEE/MIS + env importance
 * sampling), with no OptiX.
 *
 * The reference renderer (kfernandez31/cuda-volprim) exposes this path only as a C++ facade:
 *   app::Renderer(const Config&, std::vector<Primitive>&&, std::optional<Camera>) + render()
 *   (include/thesis/host/app/renderer.h:77-81, src/thesis/host/app/renderer.cpp:34-439),
 * plus one plain C-ABI kernel, launch_normalize_accumulator_kernel
 *   (device/kernels/normalize_accumulator.h:11-13).
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *  - Every function returns vp_status: 0 = OK, negative = error.  The library never exits the
 *    process (the reference's CUDA_CHECK/try_unwrap_or_exit call std::exit, check.h:16-72,
 *    result.h:89-97); vp_last_error_string() returns the message of the calling thread's last
 *    failure.
 *  - Handles are opaque.  Host arrays passed in are copied; the caller keeps ownership.
 *  - A context owns one CUDA stream; calls on one context are serialised by the caller.
 *  - Pointers tagged with a vp_memory argument are host pointers (VP_MEMORY_HOST) or device
 *    pointers on the context's device (VP_MEMORY_DEVICE).
 */
#ifndef VOLPRIM_B200_H
#define VOLPRIM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VP_VERSION_MAJOR 0
#define VP_VERSION_MINOR 1

typedef int32_t vp_status;
enum {
  VP_OK = 0,
  VP_ERROR_INVALID_ARGUMENT = -1, /* bad pointer, size or parameter */
  VP_ERROR_CUDA = -2,             /* a CUDA runtime call failed */
  VP_ERROR_OUT_OF_MEMORY = -3,    /* device allocation failed */
  VP_ERROR_UNSUPPORTED = -4,      /* option the library does not support */
  VP_ERROR_LIMIT = -5,            /* a size exceeds a documented limit */
  VP_ERROR_DEVICE_STATUS = -6,    /* a kernel reported an error word (e.g. stack bound) */
  VP_ERROR_INTERNAL = -7
};

typedef enum vp_memory { VP_MEMORY_HOST = 0, VP_MEMORY_DEVICE = 1 } vp_memory;

/* Next-event estimator at a scatter vertex.  Replaces the compile-time ENABLE_NEE / ENABLE_MIS
 * switches and the runtime --ris flag (device/core/constants.cuh:156-177; launch_params.h:43;
 * device/entry/path_stages.cuh:148-226). */
typedef enum vp_nee_mode {
  VP_NEE_MIS = 0,   /* balance-heuristic MIS of phase-IS and env-IS, 2 shadow rays (default) */
  VP_NEE_PHASE = 1, /* phase importance sampling only, 1 shadow ray */
  VP_NEE_RIS = 2,   /* product RIS over ris_candidates env-IS candidates, 1 shadow ray */
  VP_NEE_NONE = 3   /* pure analog: env gathered on escape only */
} vp_nee_mode;

/* Which GPU engine runs the path loop. */
typedef enum vp_engine {
  VP_ENGINE_WARP = 0,       /* persistent kernel, one path per warp, warp-cooperative BVH32 traversal */
  VP_ENGINE_MEGAKERNEL = 1, /* plain per-pixel megakernel, thread-per-ray binary-tree traversal */
  VP_ENGINE_WAVEFRONT = 2   /* wavefront of persistent stage kernels over compacted path queues,
                               warp-cooperative BVH32 traversal; same results as VP_ENGINE_WARP */
} vp_engine;

/* Precision of the per-(ray, Gaussian) chord set-up (whitening transform, closest approach,
 * 3-sigma chord) and of the optical-depth sums.  Both are FP32 arithmetic; no precision uses
 * FP64 (the only FP64 on the device is the environment table build).  Both meet the 1e-5
 * relative per-pixel transmittance gate against the FP64 closed form on rays from outside the
 * Gaussians (FAST: 6e-6 worst on the 256-Gaussian absorption image, ACCURATE: 3e-6). */
typedef enum vp_precision {
  VP_PRECISION_AUTO = 0,    /* ACCURATE for absorption-only scenes (albedo == 0), else FAST */
  VP_PRECISION_FAST = 1,    /* FP32, hardware exp/log approximations (the reference's fast math) */
  VP_PRECISION_ACCURATE = 2 /* FP32 with error-free transforms: o - c, the closest approach and d2
                               as float pairs (TwoSum / FMA TwoProduct), correctly rounded exp,
                               compensated optical-depth sums */
} vp_precision;

/* Bits of vp_render_params.measure. */
typedef enum vp_measure {
  VP_MEASURE_COUNTERS = 1,  /* device counters (the reference's --measure-caps and more) */
  VP_MEASURE_STAGES = 2     /* per-stage CUDA-event timing of the wavefront launches */
} vp_measure;

typedef struct vp_context vp_context;
typedef struct vp_scene vp_scene;
typedef struct vp_env vp_env;
typedef struct vp_image vp_image;

/* ---------------------------------------------------------------------------------------- */
/* errors / version                                                                         */
/* ---------------------------------------------------------------------------------------- */

/* Message of the calling thread's most recent failed call ("" if none).  Replaces the
 * reference's Error/make_error (include/thesis/host/utils/result.h:86-101). */
const char* vp_last_error_string(void);
vp_status vp_version(int32_t* major, int32_t* minor);

/* ---------------------------------------------------------------------------------------- */
/* context                                                                                  */
/* ---------------------------------------------------------------------------------------- */

/* Binds a CUDA device and creates the context's stream.  Replaces cuda::Context + StreamDAG
 * construction in Renderer::Renderer (src/thesis/host/app/renderer.cpp:34-51). */
vp_status vp_context_create(int32_t device, vp_context** out);
vp_status vp_context_destroy(vp_context* ctx);
/* The context's cudaStream_t (as void*), for callers that order their own work after it. */
vp_status vp_context_stream(vp_context* ctx, void** out_stream);
vp_status vp_context_synchronize(vp_context* ctx);
/* Number of streaming multiprocessors of the context's device. */
vp_status vp_context_sm_count(vp_context* ctx, int32_t* out);

/* ---------------------------------------------------------------------------------------- */
/* scene: Gaussian primitives + acceleration structure                                       */
/* ---------------------------------------------------------------------------------------- */

/* Gaussian primitive buffers in the reference's PLY semantics (src/thesis/host/utils/io/ply.cpp:
 * 21-27,99-118): centre, per-axis scale (linear, or log when scale_is_log != 0, as the PLY
 * stores it), forward rotation quaternion (w, x, y, z; normalised by the library), density =
 * the primitive's total integrated mass M (multiplied by sigma_multiplier), RGB albedo
 * (clamped to [0, 1], non-finite -> 0, as ply.cpp:124-145).  albedo may be NULL (= 0). */
typedef struct vp_gaussians {
  uint32_t count;
  const float* mean;      /* [3 * count] */
  const float* scale;     /* [3 * count] */
  const float* quat_wxyz; /* [4 * count] */
  const float* density;   /* [count] */
  const float* albedo;    /* [3 * count] or NULL */
  int32_t scale_is_log;
  int32_t memory; /* vp_memory of all five arrays */
} vp_gaussians;

typedef struct vp_scene_info {
  uint32_t count;           /* primitives */
  uint32_t wide_nodes;      /* BVH32 nodes */
  uint32_t wide_depth;      /* BVH32 depth (root = 1) */
  uint32_t binary_nodes;    /* internal nodes of the megakernel's binary tree */
  uint32_t leaves;          /* BVH32 leaf ranges */
  int32_t albedo_all_zero;  /* 1 when every albedo is 0 (absorption-only scene) */
  double build_ms;          /* device time of the whole build (precompute, Morton, sort,
                               clustering / hierarchy, collapse, gathers), CUDA events */
  double bounds_min[3];
  double bounds_max[3];
  uint64_t device_bytes;    /* device memory held by the scene */
  int32_t wide_builder;     /* vp_tree_builder the BVH32 was collapsed from */
  int32_t binary_builder;   /* vp_tree_builder of the megakernel's binary tree */
  uint32_t binary_height;   /* height of the PLOC tree (0 when no PLOC tree was built) */
  uint32_t leaf_max;        /* largest BVH32 leaf the build allowed */
  int32_t wide_collapse;    /* vp_collapse the BVH32 was cut with */
  int32_t tau_order;        /* vp_tau_order in use: VP_TAU_ORDER_LANE or VP_TAU_ORDER_NEAREST */
} vp_scene_info;

/* Validates the primitives (positive finite scales, positive finite density, finite centres;
 * ply.cpp:146-172), precomputes the per-primitive whitening record (primitive.h:70-87), builds
 * the BVH over 3-sigma ellipsoid bounds on the device (Morton codes, radix sort, PLOC clustering
 * or Karras hierarchy + refit, collapse to a 32-wide BVH).  Replaces Renderer::initPrimsAndGAS
 * (renderer.cpp:85-173: host Morton sort + OptiX GAS/IAS build).  No primitive-count cap below
 * 2^26 (the reference caps at 65,535, renderer.cpp:54-59).  count 0 makes an empty scene that
 * every ray misses (the reference's IAS over zero instances); the emission model rejects it. */
vp_status vp_scene_create(vp_context* ctx, const vp_gaussians* prims, float sigma_multiplier,
                          vp_scene** out);

/* Binary tree a scene's traversal structures come from. */
typedef enum vp_tree_builder {
  VP_TREE_PLOC = 0, /* agglomerative clustering of the Morton-sorted 3-sigma boxes (Meister & Bittner
                       2018: nearest neighbour by union surface area in a +-32 window) */
  VP_TREE_LBVH = 1  /* Karras radix tree over the 63-bit Morton codes, refitted */
} vp_tree_builder;

/* How the BVH32 is cut from its binary tree. */
typedef enum vp_collapse {
  VP_COLLAPSE_GREEDY = 0, /* open the largest-area child until 32 slots are used; subtrees of at
                             most leaf_max Gaussians become leaves */
  VP_COLLAPSE_SAH = 1     /* SAH-optimal slot assignment by dynamic programming over the binary
                             tree (Ylitie, Karras & Laine, HPG 2017, with 32 slots); scenes above
                             2^24 Gaussians, or whose optimal cut needs more BVH32 nodes than the
                             greedy bound, use the greedy collapse */
} vp_collapse;

/* The order in which a transmittance query visits the hit children of a BVH32 node after the
 * nearest one.  The optical depth is the same sum either way; the order decides how soon a ray
 * reaches MAX_OPTICAL_DEPTH and stops. */
typedef enum vp_tau_order {
  VP_TAU_ORDER_AUTO = 0,    /* NEAREST when fewer than half of the Gaussians are opaque at their
                               core (central optical depth along their thinnest direction below
                               4 x MAX_OPTICAL_DEPTH) and the BVH32 is at least 3 levels deep,
                               else LANE */
  VP_TAU_ORDER_LANE = 1,    /* in child-slot order (no ranking pass): best when single Gaussians
                               stop most rays */
  VP_TAU_ORDER_NEAREST = 2  /* nearest first (a ranking pass per node): best when a ray needs many
                               overlapping Gaussians to become opaque */
} vp_tau_order;

/* Build choices of vp_scene_create_ex; vp_scene_create uses vp_scene_options_default. */
typedef struct vp_scene_options {
  int32_t wide_builder;   /* vp_tree_builder collapsed into the BVH32 of the warp and wavefront
                             engines (default VP_TREE_PLOC) */
  int32_t binary_builder; /* vp_tree_builder of the megakernel's binary tree (default VP_TREE_PLOC;
                             a PLOC tree deeper than the megakernel's 128-entry stack falls back
                             to VP_TREE_LBVH) */
  uint32_t leaf_max;      /* largest BVH32 leaf in Gaussians, 1..32 (default 24) */
  int32_t wide_collapse;  /* vp_collapse: how the binary tree becomes 32-wide nodes (default
                             VP_COLLAPSE_SAH) */
  int32_t tau_order;      /* vp_tau_order of the scene's transmittance queries (default AUTO) */
} vp_scene_options;

vp_status vp_scene_options_default(vp_scene_options* out);
vp_status vp_scene_create_ex(vp_context* ctx, const vp_gaussians* prims, float sigma_multiplier,
                             const vp_scene_options* options, vp_scene** out);
vp_status vp_scene_info_get(vp_scene* scene, vp_scene_info* out);
vp_status vp_scene_destroy(vp_scene* scene);

/* ---------------------------------------------------------------------------------------- */
/* environment map (lat-long, bilinear, wrap-U / clamp-V) + importance sampling              */
/* ---------------------------------------------------------------------------------------- */

/* rgb: width*height*channels floats, row-major, channels = 3 or 4.  Builds the luminance x
 * sin(theta) sampling distribution in FP64 on the device as per-row alias tables plus a
 * marginal alias table over rows.  Replaces host::params::EnvironmentMap (texture upload +
 * FP32 host buildCdf, include/thesis/host/params/environment_map.h:45-151). */
vp_status vp_env_create(vp_context* ctx, const float* rgb, uint32_t width, uint32_t height,
                        uint32_t channels, int32_t memory, vp_env** out);
/* Constant radiance (r, g, b) on a 2x1 map (the "white_constant" environment when r=g=b=1). */
vp_status vp_env_create_constant(vp_context* ctx, float r, float g, float b, vp_env** out);
/* Device time of the last env build in milliseconds. */
vp_status vp_env_build_ms(vp_env* env, double* out_ms);
/* Copies the sampling tables the device built back to host arrays, for checking them against
 * the reference's distribution (EnvironmentMap::buildCdf,
 * include/thesis/host/params/environment_map.h:45-101).  out_width / out_height receive the map
 * size; the arrays may be NULL to query it.  Per texel (width*height, row-major, row = polar
 * angle): the alias probability and alias texel within its row, and the joint weight
 * luminance x sin(theta); per row (height): the marginal alias probability and alias row.
 * out_total: the sum of the joint weights (0 selects the uniform-sphere fallback). */
vp_status vp_env_read_tables(vp_env* env, uint32_t* out_width, uint32_t* out_height,
                             float* cond_prob, uint32_t* cond_alias, float* marg_prob,
                             uint32_t* marg_alias, float* joint, float* out_total);
vp_status vp_env_destroy(vp_env* env);

/* ---------------------------------------------------------------------------------------- */
/* camera + render parameters                                                               */
/* ---------------------------------------------------------------------------------------- */

/* Mirrors host::params::Camera::createPerspective / createOrthographic
 * (include/thesis/host/params/camera.h:32-150). */
typedef struct vp_camera {
  float eye[3];
  float lookat[3];
  float up[3];
  float vfov_deg;      /* perspective vertical field of view */
  float ortho_height;  /* orthographic viewport height */
  int32_t orthographic;
} vp_camera;

/* Mirrors app::Config's render controls (include/thesis/host/app/config.h:14-50) and
 * RenderParams (include/thesis/common/params/launch_params.h:37-59). */
typedef struct vp_render_params {
  uint32_t width;
  uint32_t height;
  uint32_t spp;            /* --spp */
  uint32_t seed;           /* --seed (launch seed of every PCG32 stream) */
  uint32_t max_bounces;    /* --max-depth (default 128) */
  uint32_t rr_depth;       /* --rr-depth (default 12) */
  float rr_max_survival;   /* --rr-max-survival (default 0.99) */
  float hg_g;              /* --phase-g (default 0.85; |g| < 1e-3 is isotropic) */
  float firefly_clamp;     /* --firefly-clamp (0 = off) */
  float pixel_filter_stddev; /* --filter-width (0 = box) */
  int32_t nee_mode;        /* vp_nee_mode */
  uint32_t ris_candidates; /* --ris-candidates (default 6) */
  uint32_t batch_spp;      /* samples per launch (reference BATCH_SIZE = 16) */
  int32_t engine;          /* vp_engine */
  int32_t precision;       /* vp_precision */
  int32_t measure;         /* bit set: VP_MEASURE_COUNTERS counts crossings, bounces, shadow rays
                              and maxima (costs atomics); VP_MEASURE_STAGES times the wavefront
                              stages with CUDA events (no device-side cost) */
  /* Adaptive sampling (ADAPTIVE_THRESHOLD / ADAPTIVE_MIN_SAMPLES, device/core/constants.cuh:
   * 196-211; the test of device/entry/raygen.cuh:52-67).  Before each batch, a pixel that already
   * holds n >= max(adaptive_min_samples, 2) samples takes none in this batch when
   *   max over r, g, b of  sqrt(M2 * rcp(n - 1)) * rcp(max(mean, 1e-6))  <  adaptive_threshold
   * (M2: the pixel's Welford sum of squared deviations; rcp and sqrt rounded to nearest, as the
   * reference's math::rcp / math::sqrt).  0 (the default, the reference's value) turns it off. */
  float adaptive_threshold;
  uint32_t adaptive_min_samples;   /* default 32 */
} vp_render_params;

/* Fills the reference's defaults (config.h:30-47, launch_params.h:38-58). */
vp_status vp_render_params_default(vp_render_params* out);

typedef struct vp_render_stats {
  double ms_kernels;           /* device time of the render launches (CUDA events) */
  uint64_t paths;              /* paths traced: width * height * spp less paths_skipped */
  uint64_t bounces;            /* scatter-or-escape events        (measure != 0) */
  uint64_t scatters;           /* events that scattered           (measure != 0) */
  uint64_t crossings;          /* closed-form (ray, Gaussian) evaluations (measure != 0) */
  uint64_t shadow_rays;        /* transmittance queries           (measure != 0) */
  uint64_t nodes_visited;      /* inner BVH node visits           (measure != 0) */
  uint64_t leaves_visited;     /* BVH32 leaf visits (warp engine) (measure != 0) */
  uint64_t prim_tests;         /* Gaussian 3-sigma boxes tested at BVH32 leaves (measure != 0) */
  uint64_t geo_loads;          /* Gaussian whitening records loaded for a chord or point test
                                  (box hits)                      (measure != 0) */
  uint64_t query_nodes[3];     /* inner-node visits per query kind: [0] free-flight argmin,
                                  [1] transmittance, [2] albedo point query (measure != 0) */
  uint64_t query_leaves[3];    /* BVH32 leaf visits per query kind (measure != 0) */
  uint32_t max_hits_per_ray;   /* largest candidate count of one query (measure != 0) */
  uint32_t max_point_overlap;  /* largest Gaussian overlap at a path vertex (measure != 0) */
  uint32_t device_status;      /* 0 = fine; else an error word raised by a kernel */
  uint32_t launches;           /* kernels launched by the call (always counted) */
  uint64_t query_prim_tests[3];/* Gaussian boxes tested per query kind        (measure counters) */
  uint64_t query_geo_loads[3]; /* Gaussian records loaded per query kind       (measure counters) */
  double ms_stage[3];          /* device time of the wavefront's [0] extend (free-flight argmin),
                                  [1] shadow (transmittance) and [2] all other launches; the
                                  warp and megakernel engines put their one kernel in [2]
                                                                             (measure stages) */
  uint32_t stage_launches[3];  /* launches in each ms_stage bucket            (measure stages) */
  uint32_t reserved;
  uint64_t paths_skipped;      /* paths not traced because their pixel had converged (adaptive
                                  sampling); paths counts only the traced ones (always counted) */
  uint64_t hits_hist[2][16];   /* queries by the number of Gaussian chords they evaluated, in
                                  power-of-two bins: bin 0 = none, bin k = [2^(k-1), 2^k) for
                                  k = 1..14, bin 15 = 2^14 or more; [0] free-flight argmin
                                  queries, [1] transmittance queries.  The distribution behind
                                  max_hits_per_ray (the reference's --measure-caps hit-buffer
                                  demand; warp and wavefront engines)         (measure != 0) */
} vp_render_stats;

/* ---------------------------------------------------------------------------------------- */
/* rendering                                                                                */
/* ---------------------------------------------------------------------------------------- */

/* Progressive Welford image (float4 mean, float4 M2 and uint32 count per pixel).  Replaces
 * host::params::Image (include/thesis/host/params/image.h) and device::params::Image
 * (include/thesis/device/params/image.h:15-38).  M2, the running sum of squared deviations,
 * is kept on every render (the reference allocates it only when adaptive sampling is compiled
 * in), so adaptive sampling can be switched on for any batch. */
vp_status vp_image_create(vp_context* ctx, uint32_t width, uint32_t height, vp_image** out);
vp_status vp_image_clear(vp_image* image);
vp_status vp_image_destroy(vp_image* image);
/* Copies the mean (RGBA float32, alpha = 1) to out (host or device memory). */
vp_status vp_image_read(vp_image* image, float* out_rgba, int32_t memory);
/* Raw device pointers (float4 mean[W*H], uint32 count[W*H]). */
vp_status vp_image_device_buffers(vp_image* image, void** mean, void** count);
/* Copies the Welford state: out_m2_rgba (W*H*4 floats: M2 per channel, alpha 0) and out_count
 * (W*H samples per pixel), both in `memory` (host or device); either may be NULL. */
vp_status vp_image_read_welford(vp_image* image, float* out_m2_rgba, uint32_t* out_count, int32_t memory);

/* Renders samples [spp_offset, spp_offset + spp_count) of a params->spp-sample render into
 * image (Welford update).  With params->adaptive_threshold > 0 every batch first skips the pixels
 * that pass the adaptive test and keeps M2; that needs every batch since the image's last clear
 * to have kept M2, else VP_ERROR_INVALID_ARGUMENT.  Replaces one Renderer::render batch iteration
 * (renderer.cpp:353-376 -> optixLaunch of __raygen__rg, device/entry/raygen.cuh:21-243). */
vp_status vp_render_accumulate(vp_scene* scene, vp_env* env, const vp_camera* camera,
                               const vp_render_params* params, vp_image* image,
                               uint32_t spp_offset, uint32_t spp_count, vp_render_stats* stats);

/* Whole render: all params->spp samples in batches of params->batch_spp, then the mean is
 * written to out_rgba (width*height*4 floats, host or device).  Replaces Renderer::render
 * (renderer.cpp:341-439) minus the EXR write.  stats may be NULL. */
vp_status vp_render(vp_scene* scene, vp_env* env, const vp_camera* camera,
                    const vp_render_params* params, float* out_rgba, int32_t memory,
                    vp_render_stats* stats);

/* Transmittance exp(-tau) along n rays (origin, unit direction) over [0, inf), each summing
 * the 3-sigma-truncated closed-form optical depth of every Gaussian the ray overlaps.
 * Replaces compute_transmittance_to_env (device/core/sampling.cuh:548-583) with its any-hit
 * TRANSMITTANCE fusion (device/entry/anyhit.cuh:53-66).  Arrays: origins[3n], dirs[3n],
 * out_transmittance[n]; precision as vp_precision; engine as vp_engine. */
vp_status vp_transmittance(vp_scene* scene, const float* origins, const float* dirs, uint32_t n,
                           int32_t precision, int32_t engine, float* out_transmittance,
                           int32_t memory);

/* The same transmittance query as vp_transmittance, for callers that cannot allocate device
 * memory (a plug-in whose host application owns the device-memory budget, or a loop where a
 * cudaMalloc / cudaFree would synchronise the device).  It calls no allocator: its scratch -- the
 * staged host rays and results, the work-queue head and the status word -- is one file-scope
 * static __device__ array sized for at most 65536 rays (about 1.8 MB), which every GPU that loads
 * the library holds until the process exits.  n > 65536 returns VP_ERROR_LIMIT.  The first call
 * on a device looks up the array's address on that device and keeps it for the life of the
 * process, so reset no device (cudaDeviceReset) while the library is in use.  Each call
 * synchronises the context's stream before it returns, so no call can be captured into a CUDA
 * graph.  All calls share the array and leave their data in it (the queue head and status word are
 * cleared at the start of each call): calls whose work overlaps on the GPU race and must be
 * serialised by the caller.  No counterpart in the reference. */
vp_status vp_transmittance_static(vp_scene* scene, const float* origins, const float* dirs,
                                  uint32_t n, int32_t precision, float* out_transmittance,
                                  int32_t memory);

/* Camera rays of n (pixel x, pixel y, sample index) triples for a params->spp-sample render:
 * the per-(pixel, sample) PCG32 stream seeded as the reference's raygen
 * (device/entry/raygen.cuh:82-99, device/core/random.cuh:33-72) and the jittered ray of
 * device/params/camera.h:43-57.  origins[3n], dirs[3n]. */
vp_status vp_camera_rays(vp_context* ctx, const vp_camera* camera, const vp_render_params* params,
                         const uint32_t* px, const uint32_t* py, const uint32_t* sample, uint32_t n,
                         float* out_origins, float* out_dirs, int32_t memory);

/* Albedo at n points: the sigma_t * pdf-weighted mean albedo of the Gaussians whose 3-sigma
 * ellipsoid contains each point, and how many contain it.  Replaces evaluate_albedo over the
 * active set (device/core/sampling.cuh:257-283, 422-458) and point_inside_bvh_bound
 * (include/thesis/common/geometry/intersection.h:56-61).  points[3n], out_rgb[3n] (0 where no
 * Gaussian contains the point), out_overlap[n]. */
vp_status vp_albedo_at(vp_scene* scene, const float* points, uint32_t n, int32_t precision,
                       int32_t engine, float* out_rgb, uint32_t* out_overlap, int32_t memory);

/* ---------------------------------------------------------------------------------------- */
/* absorption-plus-emission image and its adjoint (the differentiation form; no counterpart  */
/* in the reference, which has neither emission nor gradients)                               */
/* ---------------------------------------------------------------------------------------- */

/* Image model.  Along a camera ray, Gaussian i contributes the closed-form optical depth tau_i
 * of its 3-sigma chord over [0, inf) (the vp_transmittance sum) and emits RGB e_i per unit
 * optical depth.  With S = sum tau_i, C = sum tau_i e_i and T = exp(-S) the ray's radiance is
 *     L = (1 - T) C / S + T env(d)          (L = env(d) when S = 0),
 * the exact emission-absorption integral when the emission-to-extinction ratio along the ray
 * is its tau-weighted mean C / S (exact for one Gaussian and in the optically thin limit).  It
 * is independent of the order of the Gaussians along the ray.  Limitation: there is no
 * occlusion between Gaussians -- with opaque Gaussians (the differentiation workload's central
 * tau is in the thousands) a pixel shows the tau-weighted mean emission of every Gaussian its
 * ray crosses, so a Gaussian behind an opaque one still colours it; only the background is
 * attenuated, by the exact closed-form transmittance.  A pixel is the mean of
 * params->spp jittered camera rays seeded as vp_render's (box filter); only width, height, spp,
 * seed, pixel_filter_stddev, precision and measure of params are read. */

/* Sets the emission (RGB per unit optical depth, [3 * count] in the order the scene was built
 * from).  A scene's emission is 0 until set. */
vp_status vp_scene_set_emission(vp_scene* scene, const float* rgb, int32_t memory);

/* Renders the absorption-plus-emission image: width*height*4 floats (alpha = 1). */
vp_status vp_render_emission(vp_scene* scene, vp_env* env, const vp_camera* camera,
                             const vp_render_params* params, float* out_rgba, int32_t memory,
                             vp_render_stats* stats);

/* Gradients of a loss with respect to the arrays the scene was built from (caller order). */
typedef struct vp_gaussian_grads {
  float* mean;      /* [3 * count] */
  float* scale;     /* [3 * count]: d/d(log scale) if the scene was built with scale_is_log,
                       else d/d(scale) */
  float* quat_wxyz; /* [4 * count]: w.r.t. the quaternion as given (before normalisation) */
  float* density;   /* [count]: w.r.t. the density as given (before sigma_multiplier) */
  float* emission;  /* [3 * count] or NULL */
  int32_t memory;   /* vp_memory of all five arrays */
} vp_gaussian_grads;

/* Adjoint of vp_render_emission.  dloss_drgba holds dLoss/d(out_rgba) (width*height*4; alpha
 * ignored; pixels whose RGB gradient is 0 are skipped).  ADDS dLoss/d(parameter) into every
 * array of grads, so calls for several cameras accumulate.  Each ray's Gaussians are found again
 * by traversal (twice: once for the ray's sums, once to scatter gradients); nothing is stored
 * between the forward and backward calls. */
vp_status vp_render_emission_backward(vp_scene* scene, vp_env* env, const vp_camera* camera,
                                      const vp_render_params* params, const float* dloss_drgba,
                                      int32_t memory, vp_gaussian_grads* grads,
                                      vp_render_stats* stats);

/* ---------------------------------------------------------------------------------------- */
/* serving: continuous batching of render requests over resident scenes (the serving form;   */
/* no counterpart in the reference, which renders one configured image per process)          */
/* ---------------------------------------------------------------------------------------- */

/* A server owns a pool of path slots and the wavefront stage kernels over them.  Each iteration
 * refills the slots freed by finished paths with new (pixel, sample) paths of the admitted
 * requests that still have unstarted paths (in the order the schedule gives), then extends,
 * shades, traces shadow rays and gathers every path in flight -- paths of different requests,
 * scenes, resolutions and sample counts share the same launches.  The iteration is captured once as a CUDA graph.  Requests wait in a FIFO until the
 * request table has a free entry and their image accumulator fits the memory budget.  A finished
 * path adds its sample to its request's per-pixel sum; a request completes when all its
 * width*height*spp paths have finished, and its mean image is written to its output buffer.
 * Each path's result is the one vp_render computes for the same scene, camera and params
 * (the same PCG32 stream per (pixel, sample)); only the order of the per-pixel FP32 sums differs. */
typedef struct vp_server vp_server;

/* How an iteration's free path slots are shared among the admitted requests that still have
 * unstarted paths. */
typedef enum vp_schedule {
  VP_SCHEDULE_FIFO = 0,  /* admission order: a request's paths all start before the next's; free
                            slots the oldest request cannot use go to the next (default) */
  VP_SCHEDULE_FAIR = 1,  /* equal shares (processor sharing); leftovers in table order */
  VP_SCHEDULE_SRPT = 2   /* fewest unstarted paths first (shortest remaining work), with a share
                            of the free slots (srpt_reserve, default half) kept for the oldest
                            request so large ones progress */
} vp_schedule;

typedef struct vp_server_config {
  uint64_t memory_budget_bytes;  /* device bytes for resident scenes + path slots + request
                                    accumulators (0 = no limit) */
  uint32_t path_slots;           /* paths in flight (0 = 2^18); fewer slots shorten each iteration,
                                    so a request's last paths finish sooner */
  uint32_t max_requests;         /* request table entries (0 = 256; rounded up to a multiple
                                    of 32, at most 1024) */
  uint32_t iterations_per_step;  /* wavefront iterations per vp_server_step (0 = 4; even) */
  int32_t precision;             /* vp_precision of every request: FAST or ACCURATE (AUTO = FAST) */
  int32_t use_graph;             /* 1: replay the iterations as a captured CUDA graph */
  int32_t schedule;              /* vp_schedule: how free path slots are shared among requests */
  float srpt_reserve;            /* VP_SCHEDULE_SRPT: fraction of each iteration's free slots kept
                                    for the oldest request with unstarted paths (0 = 0.5; at most 1) */
  uint32_t lanes;                /* independent path pools (0 = 1, at most 4), each with
                                    path_slots / lanes slots, its own stream and graph; a request
                                    runs in the least-loaded lane, and one lane's kernels fill the
                                    SMs that another lane's leave idle as they drain */
  float srpt_aging;              /* VP_SCHEDULE_SRPT: a request's key is its unstarted paths minus
                                    srpt_aging x the paths its lane has started since the request's
                                    first iteration (at least 0), so a large request that waits
                                    behind small ones rises in rank (0 = plain SRPT) */
} vp_server_config;

typedef struct vp_request {
  uint32_t scene_id;             /* from vp_server_add_scene */
  vp_camera camera;
  vp_render_params params;       /* width, height, spp, seed and the path-tracing controls;
                                    engine, batch_spp and precision are ignored */
  float* out_rgba;               /* width*height*4 floats, written when the request completes */
  int32_t memory;                /* vp_memory of out_rgba */
  int32_t reserved;
} vp_request;

typedef struct vp_server_stats {
  uint64_t submitted, admitted, completed;
  uint64_t paths_completed;
  uint64_t iterations;
  uint32_t active;               /* admitted, not yet delivered */
  uint32_t pending;              /* submitted, not admitted */
  uint64_t bytes_in_use;         /* scenes + slots + active accumulators (the budget's measure) */
  double device_ms;              /* device time of the iterations run so far (CUDA events; with
                                    several lanes, the busiest lane's) */
  uint64_t cancelled;            /* requests ended by vp_server_cancel (never delivered) */
  uint64_t alloc_failures;       /* accumulator allocations that failed (device out of memory,
                                    or injected by vp_server_inject_alloc_failures) */
} vp_server_stats;

vp_status vp_server_create(vp_context* ctx, const vp_server_config* config, vp_server** out);
/* Makes (scene, env) resident under the returned id.  The scene and env must outlive the server.
 * Call before the first vp_server_step (the graph is captured then). */
vp_status vp_server_add_scene(vp_server* server, vp_scene* scene, vp_env* env, uint32_t* scene_id);
/* Queues a request (copied); returns its id (submission order, from 0). */
vp_status vp_server_submit(vp_server* server, const vp_request* request, uint64_t* request_id);
/* Admits what fits and queues iterations_per_step wavefront iterations (a step) on the GPU when
 * any admitted request is unfinished; then waits for the previous step (every queued step when
 * nothing new was queued) and harvests it: requests whose paths have all finished get their
 * mean formed behind the running step, and host outputs are copied on a second stream.  The GPU
 * never waits for the host between steps.  A request is delivered -- its output written, its
 * memory released and its id visible to vp_server_poll -- by the first call after its copies
 * land; a call with nothing left on the GPU waits for them.  *completed = requests delivered by
 * this call. */
vp_status vp_server_step(vp_server* server, uint32_t* completed);
/* Ends a request that has not been delivered.  A queued request leaves the queue.  An admitted
 * request starts no further paths from the next queued step on; its paths already in flight run
 * to their end, and then its table entry, accumulator and share of the memory budget are released
 * by a later vp_server_step.  A cancelled request never appears in vp_server_poll and its output
 * buffer is never written.  VP_ERROR_INVALID_ARGUMENT for an id that was never submitted, is
 * already cancelled, or that a vp_server_step has already found finished (its output is being
 * or has been delivered). */
vp_status vp_server_cancel(vp_server* server, uint64_t request_id);
/* Ids of requests completed since the last call (up to cap; the rest stay queued). */
vp_status vp_server_poll(vp_server* server, uint64_t* ids, uint32_t cap, uint32_t* n);
vp_status vp_server_get_stats(vp_server* server, vp_server_stats* out);
/* Fault injection on the host, for tests: the next n accumulator allocations of admissions fail
 * as a device out-of-memory would, without calling the allocator.  A failed allocation (injected
 * or real) leaves the request at the head of the queue and ends this step's admissions; while
 * other requests are admitted it waits for the memory they release.  When none is admitted,
 * vp_server_step returns VP_ERROR_OUT_OF_MEMORY, with the request still queued and the server
 * usable: a later vp_server_step retries it, or vp_server_cancel removes it. */
vp_status vp_server_inject_alloc_failures(vp_server* server, uint32_t n);
vp_status vp_server_destroy(vp_server* server);

/* ---------------------------------------------------------------------------------------- */
/* asset IO on the host (replaces src/thesis/host/utils/io/ply.cpp, hdr.cpp, exr.cpp)          */
/* ---------------------------------------------------------------------------------------- */

/* Gaussians in library-allocated host arrays (release with vp_host_gaussians_free).  The arrays
 * go straight into vp_gaussians with scale = log_scale and scale_is_log = 1. */
typedef struct vp_host_gaussians {
  uint32_t count;
  float* mean;       /* [3 * count] */
  float* log_scale;  /* [3 * count] */
  float* quat_wxyz;  /* [4 * count], as stored (vp_scene_create normalises) */
  float* density;    /* [count] total mass (sigma_t_0); sigma_multiplier applies at scene build */
  float* albedo;     /* [3 * count] (clamped at scene build) */
} vp_host_gaussians;

/* Reads the "vertex" element of a Gaussian PLY: x y z rot_0..3 (w, x, y, z) scale_0..2 (log)
 * albedo_0..2 sigma_t_0, any numeric property types, ascii or binary of either byte order.
 * albedo_override (3 floats, or NULL) replaces the file's albedo when all three are >= 0.
 * Replaces io::loadPrimitivesFromPLY (ply.cpp:35-175); its validation is vp_scene_create's. */
vp_status vp_ply_load(const char* path, const float* albedo_override, vp_host_gaussians* out);
/* Writes the same 14 properties as binary little-endian floats (albedo NULL -> 0). */
vp_status vp_ply_save(const char* path, const vp_host_gaussians* gaussians);
vp_status vp_host_gaussians_free(vp_host_gaussians* gaussians);

/* Reads a Radiance RGBE picture ("#?RADIANCE"/"#?RGBE", FORMAT=32-bit_rle_rgbe, "-Y H +X W",
 * new run-length or raw scanlines) into a library-allocated RGB float array (row 0 = the first
 * scanline; release with vp_host_free), ready for vp_env_create(..., channels = 3, HOST).
 * Replaces the reference's .hdr loader (hdr.cpp). */
vp_status vp_hdr_load(const char* path, float** out_rgb, uint32_t* width, uint32_t* height);
vp_status vp_host_free(void* p);

/* Writes width*height RGBA floats (alpha dropped) as a single-part scanline OpenEXR file with
 * uncompressed FLOAT channels B, G, R, flipped vertically when flip_vertical != 0.  Replaces
 * saveExrImage (exr.cpp:36-100). */
vp_status vp_exr_save(const char* path, const float* rgba, uint32_t width, uint32_t height,
                      int32_t flip_vertical);

/* Grid-stride copy out[i] = accumulator[i] * normalization_factor over n float4 pixels on the
 * context's stream (or `stream` when non-NULL).  Same contract as the reference's
 * launch_normalize_accumulator_kernel (device/kernels/normalize_accumulator.cu:27-35). */
vp_status vp_normalize_accumulator(vp_context* ctx, float* out_pixels, const float* accumulator,
                                   size_t n_pixels, float normalization_factor, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VOLPRIM_B200_H */
