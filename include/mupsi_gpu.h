/*
 * mupsi_gpu.h -- C ABI of the B200 GPIS path-tracing library (libmupsi_gpu.so).
 *
 * The reference renderer enters its hot path through per-point virtual calls
 * (SparseGPNoiseGenerator::RawNoise, MeanFunction::eval/gradient,
 * Medium::sampleDistance, BVH::intersect/closest) driven by an OpenMP pixel loop
 * (Renderer::startRenderProgressive). A GPU can only be entered at batch
 * granularity, so this ABI sits at two levels:
 *   - the Renderer level: a scene handle plus a progressive render call, which
 *     a GpuRenderer in the reference host calls instead of its pixel loop;
 *   - batched probes of each per-point interface, used by parity tests and by
 *     hosts that want the kernels without the renderer.
 *
 * Conventions (mirroring the reference's bool + std::cerr error style,
 * controller/controller.cpp:44-47):
 *   - every entry returns int: 0 (MUPSI_OK) or a negative mupsi_status;
 *     mupsi_gpu_last_error() gives a message for the calling thread;
 *   - the caller owns every input/output buffer; `mem` says whether the
 *     buffers of that call are host or device pointers (all of one kind);
 *   - `stream` is a cudaStream_t (NULL = the library's internal stream);
 *     calls are synchronous with respect to the host unless named *_async;
 *   - plain C types only: no CUDA, torch or C++ types cross this boundary.
 */
#ifndef MUPSI_GPU_H
#define MUPSI_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: mupsi_tuning gained block_rays; 3: mupsi_render_stats gained bvh_nodes/bvh_tris,
 * mupsi_tuning gained lane_rays; 4: mupsi_tuning gained mu_batch */
#define MUPSI_GPU_ABI_VERSION 4

typedef enum { MUPSI_MEM_HOST = 0, MUPSI_MEM_DEVICE = 1 } mupsi_mem;

typedef enum {
  MUPSI_OK = 0,
  MUPSI_ERR_INVALID = -1,      /* bad argument or descriptor */
  MUPSI_ERR_CUDA = -2,         /* a CUDA runtime call failed */
  MUPSI_ERR_OOM = -3,          /* device allocation failed */
  MUPSI_ERR_CANCELLED = -4,    /* *cancel became non-zero between passes */
  MUPSI_ERR_UNSUPPORTED = -5,  /* feature not available on this build/device */
  MUPSI_ERR_DEVICE_LIMIT = -6, /* a device-side iteration cap fired */
  MUPSI_ERR_IO = -7            /* file could not be read/parsed */
} mupsi_status;

/* GP correlation modes (gp/gpnoise.h:9-15) */
typedef enum { MUPSI_GP_SINGLE_REALIZATION = 0, MUPSI_GP_RENEWAL_PLUS = 1 } mupsi_gp_mode;
/* BSDFs (bsdf/bsdf.h:38-105) */
typedef enum { MUPSI_BSDF_LAMBERTIAN = 0, MUPSI_BSDF_NULL = 1, MUPSI_BSDF_SPECULAR = 2 } mupsi_bsdf;
/* mean functions (gp/meanfunction.h:10-57) */
typedef enum { MUPSI_MEAN_SPHERE = 0, MUPSI_MEAN_MESH = 1 } mupsi_mean_type;

/* What a scene medium is: a GPMedium (medium/gpmedium.h, the descriptor's
 * default), an SDFMedium (medium/sdfmedium.h) or an ExternalGPMedium
 * (medium/externalgpmedium.h); see mupsi_gpu_scene_set_sdf_medium and
 * mupsi_gpu_scene_set_external_gp_medium. */
typedef enum { MUPSI_MEDIUM_GP = 0, MUPSI_MEDIUM_SDF = 1, MUPSI_MEDIUM_EXTERNAL_GP = 2 } mupsi_medium_kind;
/* primitives (geometry/primitive.h:17-67) */
typedef enum { MUPSI_PRIM_SPHERE = 0, MUPSI_PRIM_MESH = 1 } mupsi_prim_type;

/* SparseSEKernel(sigma, kernelRadius, lengthScale) + impulse density
 * (gp/kernel.h:39-78, gp/gpnoise.h:23-49). JSON keys: kernel.sigma,
 * kernel.length_scale (-> kernel_radius, the grid cell size), kernel.aniso
 * (-> the lengthScale vector; h() uses L2 = |aniso|^2), kernel.points_per_cell. */
typedef struct {
  float sigma;
  float kernel_radius;
  float aniso[3];
  int32_t points_per_cell;
} mupsi_kernel;

/* GPConditioningState (medium/medium.h:12-17), 32 bytes. */
typedef struct {
  float C[3];
  float u_tilde;
  float g_tilde[3];
  uint32_t active;
} mupsi_cond;

/* Ray (geometry/ray.h:10-28): origin, unit direction, nearT, farT; 32 bytes. */
typedef struct {
  float o[3];
  float d[3];
  float near_t;
  float far_t;
} mupsi_ray;

/* MediumSample subset returned by a march (medium/medium.h:21-29), 32 bytes. */
typedef struct {
  uint32_t exited; /* 1: no surface found along the ray */
  float t;
  float p[3];
  float normal[3];
} mupsi_medium_sample;

/* Triangle mesh (primitives/mesh.h:15-78). Object-space arrays plus the
 * Translation(position)*Scaling(scale) transform the JSON schema allows. */
typedef struct {
  int64_t num_vertices;
  const float* vertices; /* [num_vertices*3] */
  int64_t num_faces;
  const int32_t* faces; /* [num_faces*3], 0-based */
  const float* vertex_normals; /* nullable [num_vertices*3] */
  float position[3];
  float scale;
} mupsi_mesh_desc;

/* Mean function + kernel of one GPMedium (medium/gpmedium.h:19-51). */
typedef struct {
  int32_t mean_type;     /* mupsi_mean_type */
  float mean_center[3];  /* sphere mean */
  float mean_radius;
  int32_t mean_mesh;     /* index into scene meshes (mesh mean) */
  mupsi_kernel kernel;
} mupsi_medium_desc;

/* One scene primitive (sphere or mesh) in scene order. */
typedef struct {
  int32_t type;          /* mupsi_prim_type */
  float center[3];       /* sphere: Translation(center)*Scaling(radius) */
  float radius;
  int32_t mesh;          /* mesh: index into scene meshes */
  int32_t bsdf;          /* mupsi_bsdf */
  float albedo[3];       /* Lambertian albedo (reference default 0.8) */
  int32_t has_emission;
  float emission[3];
  int32_t int_medium;    /* index into media, -1 = none */
  int32_t ext_medium;
} mupsi_primitive_desc;

/* Everything Controller::load builds (controller/controller.cpp:40-264) plus
 * the RenderContext snapshot (rendering/render_context.h:16-27). */
typedef struct {
  int32_t width, height, spp;
  int32_t max_bounce;
  int32_t max_medium_bounce; /* parsed but unused by the reference trace loop */
  int32_t gp_mode;           /* mupsi_gp_mode */
  float cam_pos[3], cam_dir[3], cam_up[3];
  float cam_fov;             /* as in scene.json; tan(fov/2) is taken with fov in radians (camera.cpp:10-11) */
  float eps;                 /* PathTracerSettings::eps (1e-4) */
  float nearteps;            /* PathTracerSettings::nearteps (1.5e-3) */
  int32_t has_sky;           /* skydrome present */
  float sky[3];              /* constant skydrome radiance (Skydrome() = 1.0) */
  int32_t num_media;
  const mupsi_medium_desc* media;
  int32_t num_meshes;
  const mupsi_mesh_desc* meshes;
  int32_t num_primitives;
  const mupsi_primitive_desc* primitives;
} mupsi_scene_desc;

typedef struct mupsi_scene mupsi_scene;
typedef struct mupsi_mesh mupsi_mesh;

/* ---------------------------------------------------------------- errors -- */

/* Message of the last failing call on this thread ("" if none). */
const char* mupsi_gpu_last_error(void);
/* ABI version compiled into the library (MUPSI_GPU_ABI_VERSION). */
int32_t mupsi_gpu_abi_version(void);

/* Released scenes leave their device buffers to the library for reuse (the
 * path state of up to 4 scenes per device, and per-scene buffers up to 256 MB
 * per device), so a host that creates a scene per frame pays no cudaMalloc /
 * cudaFree. This hands all of them back to the driver; call it when no scene
 * is rendering. */
int mupsi_gpu_release_pools(void);
/* Number of kernel launches this library has issued on this process. */
int64_t mupsi_gpu_launch_count(void);

/* ------------------------------------------------------- GP noise batch -- */

/* psi and grad psi at n points: SparseGPNoiseGenerator::RawNoise(p, seed)
 * (gp/gpnoise.h:44, gp/gpnoise.cpp:51-87). out[n*4] = (psi, dpsi/dx, dpsi/dy, dpsi/dz).
 * cond (nullable, n entries): adds the Renewal+ terms of GPMedium::evalWithGradient
 * (medium/gpmedium.cpp:26-41) for entries with active != 0, without the mean. */
int mupsi_gpu_psi(const mupsi_kernel* kernel, int64_t n, const float* p, const uint32_t* seed,
                  const mupsi_cond* cond, float* out, mupsi_mem mem, void* stream);
/* psi value only (no gradient), same sum as mupsi_gpu_psi's first output. */
int mupsi_gpu_psi_value(const mupsi_kernel* kernel, int64_t n, const float* p, const uint32_t* seed,
                        const mupsi_cond* cond, float* out, mupsi_mem mem, void* stream);

/* ------------------------------------------- integer known-answer probes -- */

/* The device's own hash, PCG32 and grid-cell routines, one query per thread,
 * so the integer parts of the path can be compared bit for bit with the
 * reference on the GPU.
 * make_seed (math/random.h:13-25): out[i] = make_seed(args[i*nargs .. +nargs)),
 * nargs 4 (per cell / per pixel) or 5 (per bounce). */
int mupsi_gpu_probe_make_seed(int64_t n, int32_t nargs, const uint32_t* args, uint32_t* out, mupsi_mem mem,
                              void* stream);
/* Random(seed) (math/random.h:73-119; zero seed -> 1, two warm-up draws), then
 * `draws` outputs per seed: out_u32[n*draws] = nextUInt(), out_f32[n*draws] =
 * next1D() of a second generator with the same seed; out_cs_i[n] =
 * ConstantSampler(seed).nextI() (math/sampler.h:47-54, seed taken as u32). */
int mupsi_gpu_probe_random(int64_t n, const uint64_t* seeds, int32_t draws, uint32_t* out_u32, float* out_f32,
                           uint32_t* out_cs_i, mupsi_mem mem, void* stream);
/* The impulses SparseGPNoiseGenerator::InternalNoise visits at p
 * (gp/gpnoise.cpp:51-87): out_cells[n*27*3] the neighbour cells (truncated
 * p / kernel_radius + (dx, dy, dz), dx slowest), out_cell_seeds[n*27]
 * make_seed(cell, seed), out_s[n*27*ppc*3] the impulse positions and
 * out_w[n*27*ppc] their weights (+-1), in the order of the sum. */
int mupsi_gpu_probe_impulses(const mupsi_kernel* kernel, int64_t n, const float* p, const uint32_t* seed,
                             int32_t* out_cells, uint32_t* out_cell_seeds, float* out_s, float* out_w, mupsi_mem mem,
                             void* stream);

/* ----------------------------------------------------- meshes and BVHs -- */

/* Host BVH build (bvh/bvh.cpp:115-193): same split rule, leaf size, partition
 * order and post-order node emission as BVH::build, so node arrays and triangle
 * ids match. nodes_out[2*num_faces*8] words per node: min xyz, max xyz (float
 * bits), left, right|0x80000000 for leaves. Returns the node count in
 * *num_nodes and the root (last node) in *root. */
int mupsi_bvh_build_host(int64_t num_vertices, const float* vertices, int64_t num_faces, const int32_t* faces,
                         uint32_t* nodes_out, uint32_t* tri_indices_out, int64_t* num_nodes, uint32_t* root);

/* Device copy of a mesh and its BVH (Mesh::prepareForRender, mesh.cpp:299-319). */
int mupsi_gpu_mesh_create(const mupsi_mesh_desc* desc, mupsi_mesh** out);
void mupsi_gpu_mesh_destroy(mupsi_mesh* mesh);

/* BVH::intersect (bvh.cpp:197-250) in object space for n rays. out_tri[n]
 * (0xFFFFFFFF on miss), out_tuv[n*3] = (t, u, v). */
int mupsi_gpu_bvh_intersect(const mupsi_mesh* mesh, int64_t n, const mupsi_ray* rays, uint32_t* out_tri,
                            float* out_tuv, mupsi_mem mem, void* stream);
/* BVH::occluded (bvh.cpp:254-300), including its traversal start at node 0. */
int mupsi_gpu_bvh_occluded(const mupsi_mesh* mesh, int64_t n, const mupsi_ray* rays, uint8_t* out,
                           mupsi_mem mem, void* stream);
/* Where BVH::occluded starts: REFERENCE (the default) at node 0 as the
 * reference does (bvh/bvh.cpp:259; node 0 is the post-order array's first leaf,
 * so most occluders are missed), ROOT at the root (a full traversal, the same
 * answer as an intersect within [near_t, far_t]). For a mesh handle, or for all
 * meshes of a scene (its shadow rays). */
enum { MUPSI_OCCLUSION_REFERENCE = 0, MUPSI_OCCLUSION_ROOT = 1 };
int mupsi_gpu_mesh_set_occlusion(mupsi_mesh* mesh, int32_t mode);
int mupsi_gpu_scene_set_occlusion(mupsi_scene* scene, int32_t mode);
/* BVH::closest (bvh.cpp:302-353): out_tri[n], out_dq[n*4] = (dist, q xyz). */
int mupsi_gpu_bvh_closest(const mupsi_mesh* mesh, int64_t n, const float* p, uint32_t* out_tri, float* out_dq,
                          mupsi_mem mem, void* stream);
/* Mesh::inside (mesh.cpp:341-362) and Mesh::distToPoint (mesh.cpp:325-339)
 * in world space: out_inside[n], out_tri[n], out_dq[n*4] = (dist, q xyz). */
int mupsi_gpu_mesh_queries(const mupsi_mesh* mesh, int64_t n, const float* p, uint8_t* out_inside,
                           uint32_t* out_tri, float* out_dq, mupsi_mem mem, void* stream);

/* ------------------------------------------------------------ scenes -- */

/* Flatten a scene description to device buffers (builds mesh BVHs on the host).
 * The library copies everything; the descriptor may be freed afterwards. */
int mupsi_gpu_scene_create(const mupsi_scene_desc* desc, mupsi_scene** out);
void mupsi_gpu_scene_destroy(mupsi_scene* scene);

/* MeanFunction::eval + gradient of medium `medium` (gp/meanfunction.cpp:13-39;
 * an external GP medium's GridMeanFunction, meanfunction.cpp:58-86):
 * out[n*4] = (mu, grad xyz). */
int mupsi_gpu_mean(const mupsi_scene* scene, int32_t medium, int64_t n, const float* p, float* out,
                   mupsi_mem mem, void* stream);
/* GPMedium::evalWithGradient(p, seed, state) (gpmedium.cpp:19-41): out[n*4].
 * A field medium gives its own evalWithGradient (sdfmedium.cpp:10-14,
 * externalgpmedium.cpp:33-58; cond unused). */
int mupsi_gpu_medium_eval(const mupsi_scene* scene, int32_t medium, int64_t n, const float* p,
                          const uint32_t* seed, const mupsi_cond* cond, float* out, mupsi_mem mem, void* stream);
/* GPMedium::sampleDistance (gpmedium.cpp:46-103) for n rays; seed[i] is the value
 * the march draws from its ConstantSampler (medium_sampler.nextI()). Field
 * media march as SDFMedium / ExternalGPMedium::sampleDistance. */
int mupsi_gpu_sample_distance(const mupsi_scene* scene, int32_t medium, int64_t n, const mupsi_ray* rays,
                              const uint32_t* seed, const mupsi_cond* cond, mupsi_medium_sample* out,
                              mupsi_mem mem, void* stream);
/* Medium::transmittance for n rays (gpmedium.cpp:105-129, sdfmedium.cpp:65-96,
 * externalgpmedium.cpp:111-130): out[n] = 0 where the field changes sign along
 * the ray, else 1. seed[i] as for sampleDistance. */
int mupsi_gpu_transmittance(const mupsi_scene* scene, int32_t medium, int64_t n, const mupsi_ray* rays,
                            const uint32_t* seed, const mupsi_cond* cond, float* out, mupsi_mem mem, void* stream);
/* GPMedium::sampleCondition (gpmedium.cpp:133-161) for n medium samples; seed[i]
 * is the next bounce's ConstantSampler draw. MUPSI_ERR_INVALID for a field
 * medium (only a GPMedium conditions, trace.cpp:144-147). */
int mupsi_gpu_sample_condition(const mupsi_scene* scene, int32_t medium, int64_t n,
                               const mupsi_medium_sample* samples, const uint32_t* seed, mupsi_cond* out,
                               mupsi_mem mem, void* stream);

/* PathTracer::trace (rendering/trace.cpp:118-213) for n explicit (x, y, k)
 * samples, hash seed 42 as Renderer uses (renderer.cpp:37). out_rgb[n*3]. */
int mupsi_gpu_trace_samples(mupsi_scene* scene, int64_t n, const int32_t* x, const int32_t* y, const int32_t* k,
                            float* out_rgb, mupsi_mem mem, void* stream);

/* Progressive render (Renderer::startRenderProgressive, renderer.cpp:22-49):
 * passes k in [spp_begin, spp_end) are traced and accumulated into the scene's
 * running per-pixel sum (Framebuffer::accumulate, framebuffer.cpp:28-35), in
 * pass order. After the call rgb_out[h*w*3] holds sum / passes-so-far (row y =
 * camera y, as Controller::copyDisplayRawTo). A call continues the running sum
 * when spp_begin equals the previous call's spp_end; otherwise (and always for
 * spp_begin == 0) it starts a new image.
 * cancel (nullable) is polled between waves of passes; on_spp (nullable) is
 * called with the number of completed passes after each wave.
 * moments_out (nullable, h*w*6 doubles) receives per pixel the FP64 sum and
 * sum of squares (r,g,b,r2,g2,b2) of this call's samples. */
typedef struct {
  int32_t spp_begin;
  int32_t spp_end;
  const volatile int32_t* cancel;
  void (*on_spp)(int32_t passes_done, void* user);
  void* user;
  float* rgb_out;
  mupsi_mem out_mem;
  double* moments_out;
  void* stream;
} mupsi_render_args;
int mupsi_gpu_render(mupsi_scene* scene, const mupsi_render_args* args);

/* Allocation-free variant of mupsi_gpu_trace_samples, for callers that cannot
 * allocate device memory while they render: a render thread that must not
 * block on the device-wide synchronisation cudaMalloc/cudaFree can imply, or a
 * host whose allocator owns the GPU's memory budget. It has no counterpart in
 * the reference. The path state lives in one static device array of the library
 * (about 3 MB, held by every GPU that loads the library until exit), so:
 *   - n is at most 16384 samples per call (larger n returns MUPSI_ERR_INVALID);
 *   - x, y, k and out_rgb must be device memory of the current device
 *     (MUPSI_ERR_INVALID otherwise); nothing is staged or allocated;
 *   - the first call on a device looks up the array's device address; make that
 *     first call before any stream capture on that device;
 *   - all calls share the array: calls that overlap on the GPU (other streams or
 *     host threads) race on it and must be serialised by the caller;
 *   - stream NULL means the default stream (no internal stream is created); the
 *     call returns once the trace on that stream has finished;
 *   - a surrogate attached with mupsi_gpu_scene_set_surrogate is not used: the
 *     mesh mean is always evaluated exactly, so for a scene with a surrogate the
 *     radiance can differ from mupsi_gpu_trace_samples' (equal for every other
 *     scene);
 *   - shadow rays through a medium are marched inline rather than deferred to
 *     shadow passes (same results).
 * The scene itself is created with mupsi_gpu_scene_create beforehand. */
int mupsi_gpu_trace_samples_noalloc(mupsi_scene* scene, int64_t n, const int32_t* x, const int32_t* y,
                                    const int32_t* k, float* out_rgb, void* stream);

/* ------------------------------------------------------ instrumentation -- */

/* Work and device time of the wavefront kernels, for roofline reporting. The
 * reference prints only a progress percentage (renderer.h:33-37); this is the
 * GPU path's counterpart. Counting and timing are off until enabled. */
typedef struct {
  uint64_t march_steps;   /* march steps visited (mean function evaluated) */
  uint64_t psi_evals;     /* psi value evaluations inside marches */
  uint64_t impulse_evals; /* sum over those of 27 * points_per_cell */
  uint64_t marches;       /* rays marched */
  double march_ms;        /* device time of the march kernels (CUDA events on the launch stream) */
  double shade_ms;        /* device time of the shading kernels */
  int64_t march_launches;
  int64_t shade_launches;
  /* first wave after profiling was enabled, per bounce iteration (up to 16):
   * rays in the medium queue, live paths, march kernel time */
  uint32_t iter_medium[16];
  uint32_t iter_live[16];
  float iter_march_ms[16];
  uint64_t mean_evals;    /* exact mesh-mean evaluations inside marches */
  uint64_t parity_casts;  /* of which needed the Mesh::inside parity cast */
  uint64_t surr_requests; /* surrogate predictions the marches asked for */
  uint64_t surr_accepted; /* of which outside the band (used as the lazy mean's bound) */
  /* BVH work of the marches' mesh-mean queries and the shading's mesh
   * intersections, counted only with profiling mode 2: nodes loaded (32 bytes
   * each) and triangles tested (48 bytes each: the leaf-ordered record of the
   * three vertices and the triangle id) */
  uint64_t bvh_nodes;
  uint64_t bvh_tris;
} mupsi_render_stats;
/* enable != 0 starts counting work and timing kernels on later renders;
 * enable == 2 also counts BVH work (the traversals then run counted copies,
 * slower: time kernels with enable == 1). */
int mupsi_gpu_scene_profile(mupsi_scene* scene, int32_t enable);
/* Copy the accumulated statistics; reset != 0 clears them afterwards. */
int mupsi_gpu_scene_stats(mupsi_scene* scene, mupsi_render_stats* out, int32_t reset);

/* ------------------------------------------------------- surrogate mean --
 * A learned stand-in for a mesh mean's signed distance (no reference
 * counterpart; the march uses it only to skip steps far from the surface):
 *   x = p - center;  u_f = B_f . x, f < 48;  gamma = (sin u, cos u)  (96)
 *   h1 = relu(W1 gamma + b1);  h_l = relu(W_l h_{l-1} + b_l), l = 2..4  (64 wide)
 *   mu_hat(p) = y_scale * (w5 . h4 + b5)
 * B holds angular frequencies (radians per scene unit). gamma, the weights and
 * h1..h4 are BF16 (round to nearest even); products accumulate in FP32 on the
 * tcgen05 tensor cores, the output layer on CUDA cores. The parameters are
 * one FP32 vector of MUPSI_MLP_PARAMS values: W1[64][96], b1[64], W2[64][64],
 * b2[64], W3, b3, W4, b4, w5[64], b5. Training minimises
 * L = mean over points of (mu_hat - mu)^2 / y_scale^2 with Adam on FP32 master
 * weights (BF16 copies feed the tensor cores). */
#define MUPSI_MLP_PARAMS 18753
#define MUPSI_MLP_FREQS 48
typedef struct mupsi_mlp mupsi_mlp;
typedef struct {
  float center[3];
  float y_scale;
  float fourier[MUPSI_MLP_FREQS * 3]; /* B: row f = (B_f.x, B_f.y, B_f.z) */
  const float* params;                /* host, MUPSI_MLP_PARAMS initial values */
} mupsi_mlp_desc;
int mupsi_gpu_mlp_create(const mupsi_mlp_desc* desc, mupsi_mlp** out);
int mupsi_gpu_mlp_destroy(mupsi_mlp* mlp);
/* Current FP32 parameters (host out[MUPSI_MLP_PARAMS]). */
int mupsi_gpu_mlp_get_params(mupsi_mlp* mlp, float* out);
/* mu_hat at n points p[n*3]; out[n]. */
int mupsi_gpu_mlp_infer(mupsi_mlp* mlp, int64_t n, const float* p, float* out, mupsi_mem mem, void* stream);
/* dL/dparams over the n points (host grad_out[MUPSI_MLP_PARAMS], FP32) and L (host). */
int mupsi_gpu_mlp_grad(mupsi_mlp* mlp, int64_t n, const float* p, const float* target, float* grad_out,
                       float* loss_out, mupsi_mem mem, void* stream);
typedef struct {
  int32_t steps;       /* Adam steps */
  int32_t batch;       /* points per step, drawn with replacement (seeded) from the n */
  float lr, lr_final;  /* learning rate, cosine-decayed from lr to lr_final */
  float beta1, beta2, eps;
  uint64_t seed;
} mupsi_mlp_train_args;
/* Train on n points p[n*3] with exact targets[n]; loss_out (nullable, host,
 * `steps` entries) receives each step's minibatch loss. */
int mupsi_gpu_mlp_train(mupsi_mlp* mlp, int64_t n, const float* p, const float* target,
                        const mupsi_mlp_train_args* args, float* loss_out, mupsi_mem mem, void* stream);
/* Let scene's renders use mlp for medium `medium`'s mesh mean. Where a march
 * would re-evaluate its lazy exact mean far from the last exact value, it
 * suspends and asks the network instead (all suspended marches of a bounce
 * are answered by one tensor-core inference launch, then resume). A
 * prediction m with |m| > band is taken as
 *   |m| / scale - margin <= |mu| <= |m| * scale + margin,  sign(mu) = sign(m)
 * (scale: the Lipschitz safety factor; margin from the held-out error); inside
 * the band, at every conditioning point and for every hit the exact BVH mean
 * is used. At most max_requests (1..32) predictions per march. One surrogate
 * per scene; mlp = NULL detaches. Single-scene renders and traces use it
 * (batches and the allocation-free trace do not). The scene refers to mlp:
 * detach or destroy the scene before destroying mlp. */
int mupsi_gpu_scene_set_surrogate(mupsi_scene* scene, int32_t medium, mupsi_mlp* mlp, float band, float scale,
                                  float margin, int32_t max_requests);

/* Skydrome with a BitmapTexture (controller.cpp:191-195, skydrome.cpp:8-17,
 * texture.cpp:52-69): rays that leave the scene take the nearest texel of the
 * equirectangular image at their direction. rgb: width x height texels of 3
 * floats, row 0 at the top, host memory (copied); it replaces the constant sky
 * of the descriptor. width = height = 0 removes it. */
int mupsi_gpu_scene_set_sky_texture(mupsi_scene* scene, int32_t width, int32_t height, const float* rgb);

/* The scene's image size (Camera width / height). */
int mupsi_gpu_scene_get_size(const mupsi_scene* scene, int32_t* width, int32_t* height);

/* GPSettings::gpMode for the scene's next renders (Controller::setGpMode,
 * controller.cpp:385-391). */
int mupsi_gpu_scene_set_gp_mode(mupsi_scene* scene, int32_t mode);

/* PathTracerSettings::skip_medium (rendering/trace.h:22, trace.cpp:142): with
 * skip != 0 paths pass through every medium without marching it (surfaces
 * only), as Controller::startProgressive(targetSpp, skipMedium = true). */
int mupsi_gpu_scene_set_skip_medium(mupsi_scene* scene, int32_t skip);

/* Replace the SparseSEKernel of GP medium `medium` (Controller::applyGpMedium,
 * controller.cpp:395-425, rebuilds the GPMedium with the UI's sigma, length
 * scale and points per cell). */
int mupsi_gpu_scene_set_kernel(mupsi_scene* scene, int32_t medium, const mupsi_kernel* kernel);

/* Turn medium `medium` into an SDFMedium (controller.cpp:154-182,
 * sdfmedium.cpp:16-98): its descriptor's mean function (sphere or mesh) is the
 * field itself, sphere traced from the ray's nearT (steps max(|f|, 1e-3), at
 * most 512, farT capped at 2000) to the first sign change, refined by 16
 * bisections; transmittance is 0 past a sign change. The kernel, the Renewal+
 * conditioning and any surrogate play no part. */
int mupsi_gpu_scene_set_sdf_medium(mupsi_scene* scene, int32_t medium);

/* Turn medium `medium` into an ExternalGPMedium (controller.cpp:184-189,
 * externalgpmedium.cpp:9-130): f(p) = mean(p) + noise_scale * sqrt(var(p)) *
 * hash(p, seed), mean and var GridMeanFunctions (meanfunction.cpp:41-86) of
 * resolution^3 float samples, x-major (index (i * res + j) * res + k), over
 * [bounds_min, bounds_max]; variance_grid NULL: no noise. Sphere traced with
 * steps max(|f|, 0.005), at most 1024, refined by 16 bisections. Grids are
 * host memory, copied; resolution in [2, 1024]. */
int mupsi_gpu_scene_set_external_gp_medium(mupsi_scene* scene, int32_t medium, int32_t resolution,
                                           const float bounds_min[3], const float bounds_max[3],
                                           const float* mean_grid, const float* variance_grid, float noise_scale);

/* Lambertian BSDF with a BitmapTexture albedo on mesh primitive `primitive`
 * (controller.cpp:240-243, bsdf.cpp:14-37): the albedo at a hit is the nearest
 * texel (texture.cpp:52-69) at the hit's texture coordinate, which is the
 * mesh's OBJ texcoords interpolated with the hit's barycentrics
 * (mesh.cpp:175-181, 232), or the barycentrics themselves when num_texcoords
 * is 0 (an OBJ without vt lines). texcoords: [num_texcoords*2] (u, v);
 * face_texcoords: [num_faces*3] 0-based indices into texcoords, one triple per
 * face of the primitive's mesh; rgb: width x height texels of 3 floats, row 0
 * at the top. Host memory, copied. width = height = 0 removes the texture (the
 * descriptor's constant albedo applies again). MUPSI_ERR_INVALID for a sphere
 * or a non-Lambertian primitive and for indices out of range. */
int mupsi_gpu_scene_set_albedo_texture(mupsi_scene* scene, int32_t primitive, int64_t num_texcoords,
                                       const float* texcoords, const int32_t* face_texcoords, int32_t width,
                                       int32_t height, const float* rgb);

/* How a march evaluates a mesh mean (no reference counterpart: the reference
 * evaluates mu at every step, GPMedium::evalWithGradient per step,
 * medium/gpmedium.cpp:46-103). LAZY (the default) keeps the last exact value
 * and its Lipschitz bounds and queries the BVH only where they cannot settle a
 * step; EVERY_STEP queries the BVH (parity cast + closest point) at every
 * visited step, the plain exact form. Both give the same march results. */
enum { MUPSI_MEAN_EVAL_LAZY = 0, MUPSI_MEAN_EVAL_EVERY_STEP = 1 };
int mupsi_gpu_scene_set_mean_eval(mupsi_scene* scene, int32_t medium, int32_t mode);

/* ------------------------------------------------------------------ tuning
 * Launch shapes of the wave kernels, process-wide. No reference counterpart
 * (the reference's OpenMP loop has no launch shapes); the values come from the
 * project's autotuner (mupsi_b200/autotune.py writes mupsi_b200/tuning.json,
 * which the Python layer applies on import). */
typedef struct mupsi_tuning {
  int32_t march_block; /* threads per block of the persistent march: 32, 64, 96 or 128 */
  int32_t min_group;   /* smallest lane group sharing one ray's psi sums: 4, 8, 16 or 32 */
  int32_t shade_block; /* threads per block of the shading kernel: a multiple of 32 in [32, 128] */
  int32_t wave_paths;  /* paths in flight per wave (the queue tile); 0 = 8 Mi */
  int32_t block_rays;  /* sphere-mean marches: one ray per block, its next 2 x warps psi steps at
                          once, while the queue holds at most block_rays rays per persistent
                          block (late bounces); 0 = never. 0..256 */
  int32_t lane_rays;   /* marches of longer queues: > 0 = one ray per lane, each ray visiting at
                          most this many steps between the warp's psi rounds (psi sums pooled
                          two points at a time); 0 = lane groups of min_group. 0..64 */
  int32_t lane_max_tris; /* mesh means: one ray per lane only while every mesh mean of the scene
                            has at most this many triangles (larger meshes keep lane groups,
                            which share each closest-point query); >= 0 */
  int32_t mu_batch;    /* mesh means marched one ray per lane: a march that needs the exact mean
                          (a BVH query) waits until this many of its warp's marches do, or all of
                          them, and those queries run together; 0 = each at once. 0..32 */
} mupsi_tuning;
int mupsi_gpu_set_tuning(const mupsi_tuning* t);
int mupsi_gpu_get_tuning(mupsi_tuning* out);

/* ------------------------------------------------------------------ batch
 * Several scene instances rendered together (no reference counterpart: the
 * reference renders one scene per Renderer::startRenderProgressive). Every
 * wave is one persistent launch sequence over a shared path queue whose paths
 * carry their instance id, so instances of different sizes, pass counts and
 * bounce limits fill the GPU together. Each instance's image equals what
 * mupsi_gpu_render(scene, spp_begin = 0, spp_end = spp[i]) returns.
 * The batch refers to the scenes (it does not own them); destroy the batch
 * before its scenes. */
typedef struct mupsi_batch mupsi_batch;
int mupsi_gpu_batch_create(int32_t num_scenes, mupsi_scene* const* scenes, mupsi_batch** out);
int mupsi_gpu_batch_destroy(mupsi_batch* batch);

typedef struct mupsi_batch_args {
  const int32_t* spp;           /* [num_scenes] passes per instance (>= 0), host memory */
  float* const* rgb_out;        /* [num_scenes] averaged image per instance (h*w*3) or NULL entries */
  mupsi_mem out_mem;            /* where every rgb_out buffer lives */
  const volatile int32_t* cancel; /* nullable, polled between waves */
  float* done_ms;               /* nullable [num_scenes]: completion time of each instance (the
                                   end of the wave holding its last passes) in ms from the
                                   start of the first wave, by CUDA events; 0 for spp 0 */
  int32_t use_graphs;           /* != 0: each wave replays a captured CUDA graph */
  int32_t schedule;             /* MUPSI_SCHEDULE_*: order in which instances enter waves */
  void* stream;                 /* cudaStream_t or NULL */
} mupsi_batch_args;
enum {
  MUPSI_SCHEDULE_SHORTEST_FIRST = 0, /* instances by ascending paths (least mean completion time) */
  MUPSI_SCHEDULE_IN_ORDER = 1,       /* instances in the order given */
  MUPSI_SCHEDULE_INTERLEAVED = 2     /* every wave takes a share of every instance's passes: all
                                        instances progress together and complete in the last wave */
};
int mupsi_gpu_batch_render(mupsi_batch* batch, const mupsi_batch_args* args);

/* Waves and kernel launches of the last batch_render. */
typedef struct mupsi_batch_info {
  int32_t waves;
  int32_t graph_launches;    /* waves replayed from a graph */
  int32_t graphs_captured;   /* graph captures (instantiations or updates) */
  int32_t max_iters;         /* largest bounce-iteration count of a wave */
  int64_t paths;             /* path samples traced */
} mupsi_batch_info;
int mupsi_gpu_batch_info(const mupsi_batch* batch, mupsi_batch_info* out);

/* ---- headless progressive display (controller/controller.cpp:266-375) ----
 * Controller's render control over one scene: a host thread renders frames
 * of passes (mupsi_gpu_render, on the display's own stream) and after each
 * frame swaps a pinned back buffer holding the averaged image with the front
 * buffer under a mutex (framebufferFront_ / framebufferBack_, displayMtx_);
 * the copy functions read the front buffer, so they always see a complete
 * frame. While a display renders, the scene must not be used by other calls. */
typedef struct mupsi_display mupsi_display;
/* Front and back buffers (black) for the scene's image size. */
int mupsi_gpu_display_create(mupsi_scene* scene, mupsi_display** out);
/* Stops a running render and frees the buffers. */
void mupsi_gpu_display_destroy(mupsi_display* d);
/* Controller::startProgressive: stop any running render, then render passes
 * [0, target_spp) in frames of passes_per_frame passes (1: a frame after every
 * pass, as the reference; 0: frames of about 2^20 paths), publishing each. */
int mupsi_gpu_display_start_progressive(mupsi_display* d, int32_t target_spp, int32_t passes_per_frame);
/* Controller::start: all spp passes, published once at the end. */
int mupsi_gpu_display_start(mupsi_display* d, int32_t spp);
/* Controller::cancel (the render thread stops between waves; an unfinished
 * frame is not published) and Controller::stop (cancel + join). stop returns
 * the render thread's status (its message in mupsi_gpu_last_error). */
void mupsi_gpu_display_cancel(mupsi_display* d);
int mupsi_gpu_display_stop(mupsi_display* d);
/* 1 while the render thread runs. */
int32_t mupsi_gpu_display_running(const mupsi_display* d);
/* isSppPassDone / ackSppPass / getCurrentSpp: a frame was published since the
 * last ack; the passes in the front buffer. */
int32_t mupsi_gpu_display_spp_pass_done(const mupsi_display* d);
void mupsi_gpu_display_ack_spp_pass(mupsi_display* d);
int32_t mupsi_gpu_display_current_spp(const mupsi_display* d);
/* copyDisplayRawTo / copyDisplayTo: the front buffer, dst[(y * w + x) * 3 + c]
 * (row y = camera y), raw or Reinhard tonemapped v / (1 + v)
 * (framebuffer.cpp:37-45). width / height must be the scene's. */
int mupsi_gpu_display_copy_raw(mupsi_display* d, float* dst, int32_t width, int32_t height);
int mupsi_gpu_display_copy_tonemapped(mupsi_display* d, float* dst, int32_t width, int32_t height);

/* ---- OBJ files (primitives/mesh.cpp:20-136, Mesh::fetchFrom) ----
 * Host-side reader with the reference's parsing rules and number extraction:
 * v, vn, vt, triangular f in the v, v/vt, v//vn, v/vt/vn forms, 1-based or
 * negative indices (a missing vt index is texcoord 0), other faces skipped.
 * Arrays are malloc'd; release with mupsi_obj_free. face_texcoords is NULL
 * when the file has no vt lines. MUPSI_ERR_INVALID for an unreadable file,
 * no geometry, or an index out of range. */
typedef struct {
  int64_t num_vertices, num_faces, num_normals, num_texcoords;
  float* vertices;         /* [num_vertices*3] */
  int32_t* faces;          /* [num_faces*3], 0-based */
  float* normals;          /* [num_normals*3] (the reference indexes them by vertex id) */
  float* texcoords;        /* [num_texcoords*2] */
  int32_t* face_texcoords; /* [num_faces*3] */
} mupsi_obj;
int mupsi_obj_load(const char* path, mupsi_obj* out);
void mupsi_obj_free(mupsi_obj* obj);

#ifdef __cplusplus
}
#endif

#endif /* MUPSI_GPU_H */
