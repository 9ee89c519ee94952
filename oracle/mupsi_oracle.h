/*
 * mupsi_oracle.h -- CPU restatement of the reference renderer's GPIS hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker the parity tests,
 * smoke() and bench.py's CPU-baseline leg use; the product never links it.
 * Each function restates, in plain C, the reference function cited beside it.
 * Parity of this restatement is pinned against the reference's own sources
 * (compiled into oracle/_ref) and against the committed fixtures under
 * tests/golden/.
 *
 * Buffers follow include/mupsi_gpu.h (the same structs), always host memory.
 */
#ifndef MUPSI_ORACLE_H
#define MUPSI_ORACLE_H

#include <stdint.h>

#include "../include/mupsi_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* math/random.h:13-25 */
uint32_t mo_make_seed4(uint32_t a, uint32_t b, uint32_t c, uint32_t d);
uint32_t mo_make_seed5(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t e);
/* math/random.h:73-102: n draws of Random(seed) as u32 and as next1D() */
void mo_random_stream(uint64_t seed, int n, uint32_t* out_u32, float* out_f);
/* math/sampler.h:43-61 */
void mo_constant_sampler(uint32_t seed, float* x, float* y, uint32_t* i);

/* gp/gpnoise.cpp:51-87 + gpnoise.h:31,44; cond as in gpmedium.cpp:26-41 (no mean) */
void mo_psi(const mupsi_kernel* k, int64_t n, const float* p, const uint32_t* seed, const mupsi_cond* cond,
            float* out);
/* Same impulses (positions from FP32 as the reference computes them), sums in FP64.
 * out[n*4] doubles; also out_abs[n*4] (nullable) = the sums of the absolute values
 * of the terms of each output times sigma/sqrt(Var): the scale against which a
 * sum's rounding error is measured. */
void mo_psi_f64(const mupsi_kernel* k, int64_t n, const float* p, const uint32_t* seed, double* out,
                double* out_abs);
/* Impulse listing for one (p, seed): positions s[27*ppc*3], weights w[27*ppc],
 * cell indices cells[27*3], cell seeds cell_seed[27] (bit-exact quantities). */
void mo_psi_impulses(const mupsi_kernel* k, const float* p, uint32_t seed, float* s, float* w, int32_t* cells,
                     uint32_t* cell_seed);

/* bvh/bvh.cpp:115-193 */
int64_t mo_bvh_build(int64_t nv, const float* verts, int64_t nf, const int32_t* faces, uint32_t* nodes_out,
                     uint32_t* tri_out, uint32_t* root);

/* Scenes: the same descriptor the GPU library takes. */
typedef struct mo_scene mo_scene;
mo_scene* mo_scene_create(const mupsi_scene_desc* desc);
void mo_scene_free(mo_scene* s);
/* Skydrome with a BitmapTexture (skydrome.cpp:8-17, texture.cpp:52-69): w x h
 * RGB floats, row 0 at the top; it replaces the constant sky. w = 0 removes it. */
void mo_scene_set_sky_texture(mo_scene* s, int w, int h, const float* rgb);
/* LambertianBsdf(BitmapTexture) albedo on mesh primitive `prim`: texcoords
 * tc [ntc*2] indexed per face by ftc [F*3] (ntc 0: the barycentrics), RGB
 * texels w x h, row 0 at the top; w = 0 removes it. 0 ok, -1 bad arguments. */
int mo_scene_set_albedo_texture(mo_scene* s, int prim, int64_t ntc, const float* tc, const int32_t* ftc, int w,
                                int h, const float* rgb);
/* bvh.cpp:197-250 / :254-300 / :302-353 on scene mesh `mesh` (object space) */
void mo_bvh_intersect(const mo_scene* s, int mesh, int64_t n, const mupsi_ray* rays, uint32_t* out_tri,
                      float* out_tuv);
void mo_bvh_occluded(const mo_scene* s, int mesh, int64_t n, const mupsi_ray* rays, uint8_t* out);
void mo_bvh_closest(const mo_scene* s, int mesh, int64_t n, const float* p, uint32_t* out_tri, float* out_dq);
/* mesh.cpp:325-362 (world space) */
void mo_mesh_queries(const mo_scene* s, int mesh, int64_t n, const float* p, uint8_t* out_inside, uint32_t* out_tri,
                     float* out_dq);
/* meanfunction.cpp:13-39 */
void mo_mean(const mo_scene* s, int medium, int64_t n, const float* p, float* out);
/* gpmedium.cpp:19-41 */
void mo_medium_eval(const mo_scene* s, int medium, int64_t n, const float* p, const uint32_t* seed,
                    const mupsi_cond* cond, float* out);
/* gpmedium.cpp:46-103 */
/* SDFMedium / ExternalGPMedium on medium `medium` (0 ok, -1 bad arguments);
 * grids res^3 floats, x-major; var may be NULL. */
int mo_scene_set_sdf_medium(mo_scene* s, int medium);
/* PathTracerSettings::skip_medium */
void mo_scene_set_skip_medium(mo_scene* s, int skip);
int mo_scene_set_external_gp_medium(mo_scene* s, int medium, int res, const float* bmin, const float* bmax,
                                    const float* mean, const float* var, float noise_scale);
/* Medium::transmittance of n rays: out[n] in {0, 1} */
void mo_transmittance(const mo_scene* s, int medium, int64_t n, const mupsi_ray* rays, const uint32_t* seed,
                      const mupsi_cond* cond, float* out);
void mo_sample_distance(const mo_scene* s, int medium, int64_t n, const mupsi_ray* rays, const uint32_t* seed,
                        const mupsi_cond* cond, mupsi_medium_sample* out);
/* gpmedium.cpp:133-161 */
void mo_sample_condition(const mo_scene* s, int medium, int64_t n, const mupsi_medium_sample* samples,
                         const uint32_t* seed, mupsi_cond* out);
/* trace.cpp:118-213 with seed 42 (renderer.cpp:37); OpenMP over samples */
void mo_trace(const mo_scene* s, int64_t n, const int32_t* x, const int32_t* y, const int32_t* k, float* out_rgb);
/* Count the march steps and psi evaluations PathTracer::trace spends on samples
 * (for roofline bookkeeping): out[0] = steps, out[1] = psi evaluations. */
void mo_trace_work(const mo_scene* s, int64_t n, const int32_t* x, const int32_t* y, const int32_t* k,
                   int64_t* out);

/* Surrogate-mean MLP (mupsi_mlp_desc in include/mupsi_gpu.h; no reference
 * counterpart), FP64 with BF16 rounding where the GPU stores BF16 operands. */
void mo_mlp_forward(const float* params, const float* fourier, const float* center, float y_scale, int64_t n,
                    const float* p, float* out);
void mo_mlp_grad(const float* params, const float* fourier, const float* center, float y_scale, int64_t n,
                 const float* p, const float* target, double* grad, double* loss);

#ifdef __cplusplus
}
#endif
#endif
