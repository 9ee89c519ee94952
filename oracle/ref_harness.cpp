// Test-infrastructure harness around the reference renderer's own, unmodified
// sources (compiled from the reference tree against oracle/shim). It exposes the
// reference's per-point interfaces as batched C entry points so that the parity
// tests and the CPU-baseline timing call the reference itself. Nothing in the
// product links this file.
//
// Private members of the reference classes are reached by defining `private`
// as `public` before their headers are included; the reference code itself is
// not changed.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <iostream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>
#include <fstream>
#include <nlohmann/json.hpp>
#ifdef _OPENMP
#include <omp.h>
#endif

#define private public
#define protected public
#include "bsdf/bsdf.h"
#include "bvh/bvh.h"
#include "controller/controller.h"
#include "geometry/intersection.h"
#include "geometry/primitive.h"
#include "geometry/ray.h"
#include "geometry/scene.h"
#include "gp/gpnoise.h"
#include "gp/kernel.h"
#include "gp/meanfunction.h"
#include "math/random.h"
#include "math/sampler.h"
#include "medium/externalgpmedium.h"
#include "medium/gpmedium.h"
#include "medium/medium.h"
#include "medium/sdfmedium.h"
#include "primitives/mesh.h"
#include "primitives/skydrome.h"
#include "primitives/sphere.h"
#include "rendering/camera.h"
#include "rendering/render_context.h"
#include "rendering/renderer.h"
#include "rendering/trace.h"
#include "texture/texture.h"
#undef private
#undef protected

using namespace mupsi;

// Members declared before any access keyword (class-default private) are reached
// with the explicit-instantiation access idiom, which the language exempts from
// access checking.
template <typename Tag, typename Tag::type M>
struct MemberAccess {
  friend typename Tag::type member_of(Tag) { return M; }
};
struct ControllerScene {
  typedef std::shared_ptr<Scene> Controller::*type;
  friend type member_of(ControllerScene);
};
struct ControllerSpp {
  typedef int Controller::*type;
  friend type member_of(ControllerSpp);
};
struct ScenePrimitives {
  typedef std::vector<std::shared_ptr<Primitive>> Scene::*type;
  friend type member_of(ScenePrimitives);
};
template struct MemberAccess<ControllerScene, &Controller::scene_>;
template struct MemberAccess<ControllerSpp, &Controller::spp_>;
template struct MemberAccess<ScenePrimitives, &Scene::primitives_>;
struct ExternalEval {
  typedef Vector4f (ExternalGPMedium::*type)(const Vector3f&, uint32_t) const;
  friend type member_of(ExternalEval);
};
template struct MemberAccess<ExternalEval, &ExternalGPMedium::evalWithGradient>;

namespace {
std::shared_ptr<Scene>& scene_of(Controller& c) { return c.*member_of(ControllerScene()); }

// A sampler whose nextI() returns a fixed value: lets a batch entry hand the
// march/conditioning seed to GPMedium directly (gpmedium.cpp:63,143 read it
// through medium_sampler.nextI()).
class FixedSeedSampler : public Sampler {
  uint32_t s_;

 public:
  explicit FixedSeedSampler(uint32_t s) : s_(s) {}
  float next1D() override { return 0.0f; }
  void next2D(float& x, float& y) override { x = y = 0.0f; }
  uint32_t nextI() override { return s_; }
  uint32_t getSeed() const override { return s_; }
};

struct RefMedium {
  std::shared_ptr<MeanFunction> mean;
  std::shared_ptr<Mesh> mesh;
  std::shared_ptr<SparseSEKernel> kernel;
  std::shared_ptr<SparseGPNoiseGenerator> noise;
  std::shared_ptr<GPMedium> medium;
};

// An SDFMedium or ExternalGPMedium with what it owns.
struct RefField {
  std::shared_ptr<Mesh> mesh;
  std::shared_ptr<MeanFunction> mean;
  std::shared_ptr<SDFMedium> sdf;
  std::shared_ptr<ExternalGPMedium> ext;
  Medium* medium() const { return sdf ? static_cast<Medium*>(sdf.get()) : static_cast<Medium*>(ext.get()); }
};

struct RefScene {
  Controller ctrl;
  std::shared_ptr<RenderContext> ctx;
};

GPConditioningState make_state(const float* cond) {
  GPConditioningState s;
  if (cond) {
    s.active = cond[7] != 0.0f;
    s.C = Vector3f(cond[0], cond[1], cond[2]);
    s.u_tilde = cond[3];
    s.g_tilde = Vector3f(cond[4], cond[5], cond[6]);
  }
  return s;
}

}  // namespace

extern "C" {

// ---- math/random.h ------------------------------------------------------------
uint32_t ref_make_seed4(uint32_t a, uint32_t b, uint32_t c, uint32_t d) { return make_seed(a, b, c, d); }
uint32_t ref_make_seed5(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t e) {
  return make_seed(a, b, c, d, e);
}
// n draws of Random(seed) (constructor warm-up included) as u32 and as next1D().
void ref_random_stream(uint64_t seed, int n, uint32_t* out_u32, float* out_f) {
  Random r(seed);
  Random r2(seed);
  for (int i = 0; i < n; ++i) {
    out_u32[i] = r.nextI();
    out_f[i] = r2.next1D();
  }
}
// ConstantSampler(seed) -> (x, y, i) (sampler.h:43-61)
void ref_constant_sampler(uint32_t seed, float* x, float* y, uint32_t* i) {
  ConstantSampler cs(seed);
  *x = cs.next1D();
  float a, b;
  cs.next2D(a, b);
  *y = b;
  *i = cs.nextI();
}

// ---- gp/ ------------------------------------------------------------------------
// RawNoise for n points: p[n*3], seed[n] -> out[n*4] = (psi, dpsi/dx, dpsi/dy, dpsi/dz).
void ref_psi(float sigma, float kernel_radius, const float* aniso, int ppc, long n, const float* p,
             const uint32_t* seed, float* out) {
  auto k = std::make_shared<SparseSEKernel>(sigma, kernel_radius, Vector3f(aniso[0], aniso[1], aniso[2]));
  SparseGPNoiseGenerator g(k, ppc);
#pragma omp parallel for schedule(dynamic, 256)
  for (long i = 0; i < n; ++i) {
    Vector4f r = g.RawNoise(Vector3f(p[3 * i], p[3 * i + 1], p[3 * i + 2]), seed[i]);
    for (int c = 0; c < 4; ++c) out[4 * i + c] = r[c];
  }
}

// SparseSEKernel pieces (kernel.h:52-68) for a batch: out[n*8] =
// (h, h_grad xyz, h_hessian_vec(v) xyz, oneOverSecondDerivative)
void ref_kernel_terms(float sigma, float kernel_radius, const float* aniso, long n, const float* s,
                      const float* p, const float* v, float* out) {
  SparseSEKernel k(sigma, kernel_radius, Vector3f(aniso[0], aniso[1], aniso[2]));
  for (long i = 0; i < n; ++i) {
    Vector3f S(s[3 * i], s[3 * i + 1], s[3 * i + 2]);
    Vector3f P(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
    Vector3f V(v[3 * i], v[3 * i + 1], v[3 * i + 2]);
    out[8 * i + 0] = k.h(S, P);
    Vector3f g = k.h_grad(S, P);
    Vector3f hv = k.h_hessian_vec(S, P, V);
    for (int c = 0; c < 3; ++c) {
      out[8 * i + 1 + c] = g[c];
      out[8 * i + 4 + c] = hv[c];
    }
    out[8 * i + 7] = k.oneOverSecondDerivative();
  }
}

// ---- medium/ ---------------------------------------------------------------------
// mean_type 0 = sphere(center, radius); 1 = mesh (OBJ path, identity transform unless
// mesh_pos/mesh_scale given).
void* ref_medium_create(int mean_type, const float* center, float radius, const char* obj_path,
                        const float* mesh_pos, float mesh_scale, float sigma, float kernel_radius,
                        const float* aniso, int ppc) {
  auto* m = new RefMedium();
  if (mean_type == 0) {
    m->mean = std::make_shared<SphereMeanFunction>(Vector3f(center[0], center[1], center[2]), radius);
  } else {
    m->mesh = std::make_shared<Mesh>();
    if (!m->mesh->fetchFrom(obj_path)) {
      delete m;
      return nullptr;
    }
    if (mesh_pos) {
      m->mesh->setTransform(
          Affine3f(Translation3f(Vector3f(mesh_pos[0], mesh_pos[1], mesh_pos[2])) * Scaling(mesh_scale)).matrix());
    }
    m->mean = std::make_shared<MeshMeanFunction>(m->mesh);
  }
  m->kernel = std::make_shared<SparseSEKernel>(sigma, kernel_radius, Vector3f(aniso[0], aniso[1], aniso[2]));
  m->noise = std::make_shared<SparseGPNoiseGenerator>(m->kernel, ppc);
  m->medium = std::make_shared<GPMedium>(m->mean, m->noise);
  return m;
}
void ref_medium_free(void* h) { delete static_cast<RefMedium*>(h); }

// MeanFunction::eval + gradient: out[n*4] = (mu, grad xyz)
void ref_mean_eval(void* h, long n, const float* p, float* out) {
  auto* m = static_cast<RefMedium*>(h);
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < n; ++i) {
    Vector3f P(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
    out[4 * i] = m->mean->eval(P);
    Vector3f g = m->mean->gradient(P);
    for (int c = 0; c < 3; ++c) out[4 * i + 1 + c] = g[c];
  }
}

// GPMedium::evalWithGradient(p, seed, state) (gpmedium.cpp:19-41).
// cond: nullptr or n*8 floats (C xyz, u_tilde, g_tilde xyz, active).
void ref_medium_eval(void* h, long n, const float* p, const uint32_t* seed, const float* cond, float* out) {
  auto* m = static_cast<RefMedium*>(h);
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < n; ++i) {
    GPConditioningState st = make_state(cond ? cond + 8 * i : nullptr);
    Vector4f r = m->medium->evalWithGradient(Vector3f(p[3 * i], p[3 * i + 1], p[3 * i + 2]), seed[i], st);
    for (int c = 0; c < 4; ++c) out[4 * i + c] = r[c];
  }
}

// GPMedium::sampleDistance for n rays (gpmedium.cpp:46-103).
// ray[n*8] = (o xyz, d xyz, nearT, farT); seed = march seed (medium_sampler.nextI()).
// out[n*8] = (exited, t, p xyz, normal xyz)
void ref_sample_distance(void* h, long n, const float* ray, const uint32_t* seed, const float* cond, float* out) {
  auto* m = static_cast<RefMedium*>(h);
#pragma omp parallel for schedule(dynamic, 1)
  for (long i = 0; i < n; ++i) {
    const float* r = ray + 8 * i;
    Ray R(Vector3f(r[0], r[1], r[2]), Vector3f(r[3], r[4], r[5]));
    R.setNearT(r[6]);
    R.setFarT(r[7]);
    GPConditioningState st = make_state(cond ? cond + 8 * i : nullptr);
    MediumSample s;
    s.conditioning = &st;
    s.t = 0.0f;
    s.p = Vector3f::Zero();
    s.normal = Vector3f::Zero();
    FixedSeedSampler ms(seed[i]);
    m->medium->sampleDistance(R, s, ms);
    float* o = out + 8 * i;
    o[0] = s.exited ? 1.0f : 0.0f;
    o[1] = s.t;
    for (int c = 0; c < 3; ++c) {
      o[2 + c] = s.p[c];
      o[5 + c] = s.normal[c];
    }
  }
}

// GPMedium::sampleCondition (gpmedium.cpp:133-161) in renewal_plus mode for n hits.
// hit[n*7] = (exited, p xyz, normal xyz); out[n*8] = (C xyz, u_tilde, g_tilde xyz, active)
void ref_sample_condition(void* h, long n, const float* hit, const uint32_t* seed, int renewal_plus, float* out) {
  auto* m = static_cast<RefMedium*>(h);
  GPSettings gs;
  gs.gpMode = renewal_plus ? GPSettings::GPCorrelationMode::RenewalPlus : GPSettings::GPCorrelationMode::SingleRealization;
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < n; ++i) {
    const float* q = hit + 7 * i;
    GPConditioningState st;
    MediumSample s;
    s.conditioning = &st;
    s.exited = q[0] != 0.0f;
    s.p = Vector3f(q[1], q[2], q[3]);
    s.normal = Vector3f(q[4], q[5], q[6]);
    FixedSeedSampler ms(seed[i]);
    m->medium->sampleCondition(s, ms, gs);
    float* o = out + 8 * i;
    for (int c = 0; c < 3; ++c) {
      o[c] = st.C[c];
      o[4 + c] = st.g_tilde[c];
    }
    o[3] = st.u_tilde;
    o[7] = st.active ? 1.0f : 0.0f;
  }
}

// ---- field media: SDFMedium, ExternalGPMedium, GridMeanFunction ----------------------
// kind 1: SDFMedium over a sphere (mean_type 0) or OBJ mesh (mean_type 1) mean;
// kind 2: ExternalGPMedium over GridMeanFunction files (var_path nullable).
void* ref_field_create(int kind, int mean_type, const float* center, float radius, const char* obj_path,
                       const float* mesh_pos, float mesh_scale, int res, const float* bmin, const float* bmax,
                       const char* mean_path, const char* var_path, float noise_scale) {
  auto* f = new RefField();
  if (kind == 1) {
    if (mean_type == 0) {
      f->mean = std::make_shared<SphereMeanFunction>(Vector3f(center[0], center[1], center[2]), radius);
    } else {
      f->mesh = std::make_shared<Mesh>();
      if (!f->mesh->fetchFrom(obj_path)) {
        delete f;
        return nullptr;
      }
      if (mesh_pos)
        f->mesh->setTransform(
            Affine3f(Translation3f(Vector3f(mesh_pos[0], mesh_pos[1], mesh_pos[2])) * Scaling(mesh_scale)).matrix());
      f->mean = std::make_shared<MeshMeanFunction>(f->mesh);
    }
    f->sdf = std::make_shared<SDFMedium>(f->mean);
  } else {
    Vector3f lo(bmin[0], bmin[1], bmin[2]), hi(bmax[0], bmax[1], bmax[2]);
    auto mg = std::make_shared<GridMeanFunction>(mean_path, res, lo, hi);
    std::shared_ptr<GridMeanFunction> vg;
    if (var_path) vg = std::make_shared<GridMeanFunction>(var_path, res, lo, hi);
    f->ext = std::make_shared<ExternalGPMedium>(mg, vg, noise_scale);
  }
  return f;
}
void ref_field_free(void* h) { delete static_cast<RefField*>(h); }

// evalWithGradient(p[, seed]) (sdfmedium.cpp:10-14, externalgpmedium.cpp:33-58): out[n*4]
void ref_field_eval(void* h, long n, const float* p, const uint32_t* seed, float* out) {
  auto* f = static_cast<RefField*>(h);
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < n; ++i) {
    Vector3f P(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
    Vector4f r = f->sdf ? f->sdf->evalWithGradient(P) : ((*f->ext).*member_of(ExternalEval()))(P, seed[i]);
    for (int c = 0; c < 4; ++c) out[4 * i + c] = r[c];
  }
}

// sampleDistance for n rays (ray[n*8] as ref_sample_distance; seed = medium_sampler.nextI()):
// out[n*8] = (exited, t, p xyz, normal xyz)
void ref_field_sample_distance(void* h, long n, const float* ray, const uint32_t* seed, float* out) {
  auto* f = static_cast<RefField*>(h);
#pragma omp parallel for schedule(dynamic, 1)
  for (long i = 0; i < n; ++i) {
    const float* r = ray + 8 * i;
    Ray R(Vector3f(r[0], r[1], r[2]), Vector3f(r[3], r[4], r[5]));
    R.setNearT(r[6]);
    R.setFarT(r[7]);
    GPConditioningState st;
    MediumSample s;
    s.conditioning = &st;
    s.t = 0.0f;
    s.p = Vector3f::Zero();
    s.normal = Vector3f::Zero();
    FixedSeedSampler ms(seed[i]);
    f->medium()->sampleDistance(R, s, ms);
    float* o = out + 8 * i;
    o[0] = s.exited ? 1.0f : 0.0f;
    o[1] = s.t;
    for (int c = 0; c < 3; ++c) {
      o[2 + c] = s.p[c];
      o[5 + c] = s.normal[c];
    }
  }
}

// transmittance for n rays: out[n] (the x component)
void ref_field_transmittance(void* h, long n, const float* ray, const uint32_t* seed, float* out) {
  auto* f = static_cast<RefField*>(h);
#pragma omp parallel for schedule(dynamic, 1)
  for (long i = 0; i < n; ++i) {
    const float* r = ray + 8 * i;
    Ray R(Vector3f(r[0], r[1], r[2]), Vector3f(r[3], r[4], r[5]));
    R.setNearT(r[6]);
    R.setFarT(r[7]);
    GPConditioningState st;
    MediumSample s;
    s.conditioning = &st;
    FixedSeedSampler ms(seed[i]);
    out[i] = f->medium()->transmittance(R, s, ms).x();
  }
}

// GridMeanFunction(path, res, bmin, bmax)::eval + gradient: out[n*4]
void ref_grid_eval(const char* path, int res, const float* bmin, const float* bmax, long n, const float* p,
                   float* out) {
  GridMeanFunction g(path, res, Vector3f(bmin[0], bmin[1], bmin[2]), Vector3f(bmax[0], bmax[1], bmax[2]));
  for (long i = 0; i < n; ++i) {
    Vector3f P(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
    out[4 * i] = g.eval(P);
    Vector3f gr = g.gradient(P);
    for (int c = 0; c < 3; ++c) out[4 * i + 1 + c] = gr[c];
  }
}

// ---- Mesh::fetchFrom ---------------------------------------------------------------
// Loads an OBJ with the reference's reader; sizes[4] = (vertices, faces, normals,
// texcoords); nullptr if fetchFrom fails.
void* ref_obj_load(const char* path, long* sizes) {
  auto* m = new Mesh();
  if (!m->fetchFrom(path)) {
    delete m;
    return nullptr;
  }
  sizes[0] = (long)m->vertices_.size();
  sizes[1] = (long)m->faces_.size();
  sizes[2] = (long)m->normals_.size();
  sizes[3] = (long)m->texcoords_.size();
  return m;
}
void ref_obj_arrays(void* h, float* v, int32_t* f, float* n, float* t, int32_t* ft) {
  auto* m = static_cast<Mesh*>(h);
  for (size_t i = 0; i < m->vertices_.size(); ++i)
    for (int c = 0; c < 3; ++c) v[3 * i + c] = m->vertices_[i][c];
  for (size_t i = 0; i < m->faces_.size(); ++i)
    for (int c = 0; c < 3; ++c) {
      f[3 * i + c] = m->faces_[i][c];
      ft[3 * i + c] = m->faceTexIndices_[i][c];
    }
  for (size_t i = 0; i < m->normals_.size(); ++i)
    for (int c = 0; c < 3; ++c) n[3 * i + c] = m->normals_[i][c];
  for (size_t i = 0; i < m->texcoords_.size(); ++i)
    for (int c = 0; c < 2; ++c) t[2 * i + c] = m->texcoords_[i][c];
}
void ref_obj_free(void* h) { delete static_cast<Mesh*>(h); }

// ---- bvh/ ---------------------------------------------------------------------------
struct RefBvh {
  std::vector<Vector3f> v;
  std::vector<Vector3i> f;
  BVH bvh;
};

void* ref_bvh_build(long nv, const float* verts, long nf, const int32_t* faces) {
  auto* b = new RefBvh();
  b->v.resize(nv);
  b->f.resize(nf);
  for (long i = 0; i < nv; ++i) b->v[i] = Vector3f(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
  for (long i = 0; i < nf; ++i) b->f[i] = Vector3i(faces[3 * i], faces[3 * i + 1], faces[3 * i + 2]);
  b->bvh.build(b->v.data(), b->f.data(), (uint32_t)nf);
  return b;
}
void ref_bvh_free(void* h) { delete static_cast<RefBvh*>(h); }
long ref_bvh_node_count(void* h) { return (long)static_cast<RefBvh*>(h)->bvh.nodes_.size(); }
uint32_t ref_bvh_root(void* h) { return static_cast<RefBvh*>(h)->bvh.rootIndex_; }
// nodes_out[count*8] = (min xyz, max xyz, left bits, right bits) as raw 32-bit words
void ref_bvh_nodes(void* h, uint32_t* nodes_out, uint32_t* tri_indices_out) {
  auto* b = static_cast<RefBvh*>(h);
  for (size_t i = 0; i < b->bvh.nodes_.size(); ++i) {
    const auto& nd = b->bvh.nodes_[i];
    float mm[6] = {nd.bounds.min().x(), nd.bounds.min().y(), nd.bounds.min().z(),
                   nd.bounds.max().x(), nd.bounds.max().y(), nd.bounds.max().z()};
    std::memcpy(nodes_out + 8 * i, mm, sizeof(mm));
    nodes_out[8 * i + 6] = nd.left;
    nodes_out[8 * i + 7] = nd.right;
  }
  for (size_t i = 0; i < b->bvh.triIndices_.size(); ++i) tri_indices_out[i] = b->bvh.triIndices_[i];
}
// BVH::intersect (bvh.cpp:197-250): ray[n*8]; out_tri[n] (0xFFFFFFFF on miss), out[n*3] = (t, u, v)
void ref_bvh_intersect(void* h, long n, const float* ray, uint32_t* out_tri, float* out) {
  auto* b = static_cast<RefBvh*>(h);
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < n; ++i) {
    const float* r = ray + 8 * i;
    Ray R(Vector3f(r[0], r[1], r[2]), Vector3f(r[3], r[4], r[5]));
    R.setNearT(r[6]);
    R.setFarT(r[7]);
    IntersectionTemporary data;
    bool hit = b->bvh.intersect(R, data);
    auto* mi = data.as<MeshIntersection>();
    out_tri[i] = hit ? mi->triIndex : 0xFFFFFFFFu;
    out[3 * i] = hit ? R.farT() : -1.0f;
    out[3 * i + 1] = hit ? mi->u : 0.0f;
    out[3 * i + 2] = hit ? mi->v : 0.0f;
  }
}
// BVH::occluded (bvh.cpp:254-300), including its traversal start at node 0.
void ref_bvh_occluded(void* h, long n, const float* ray, uint8_t* out) {
  auto* b = static_cast<RefBvh*>(h);
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < n; ++i) {
    const float* r = ray + 8 * i;
    Ray R(Vector3f(r[0], r[1], r[2]), Vector3f(r[3], r[4], r[5]));
    R.setNearT(r[6]);
    R.setFarT(r[7]);
    out[i] = b->bvh.occluded(R) ? 1 : 0;
  }
}
// BVH::closest (bvh.cpp:302-353): out_tri[n], out[n*4] = (dist, q xyz)
void ref_bvh_closest(void* h, long n, const float* p, uint32_t* out_tri, float* out) {
  auto* b = static_cast<RefBvh*>(h);
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < n; ++i) {
    uint32_t tri = 0xFFFFFFFFu;
    Vector3f q = Vector3f::Zero();
    float d = b->bvh.closest(Vector3f(p[3 * i], p[3 * i + 1], p[3 * i + 2]), tri, q);
    out_tri[i] = tri;
    out[4 * i] = d;
    for (int c = 0; c < 3; ++c) out[4 * i + 1 + c] = q[c];
  }
}

// Mesh::inside / Mesh::distToPoint through a Mesh loaded from OBJ
// (mesh.cpp:325-362). out_inside[n], out_tri[n], out[n*4] = (dist, q xyz)
void ref_mesh_queries(void* medium, long n, const float* p, uint8_t* out_inside, uint32_t* out_tri, float* out) {
  auto* m = static_cast<RefMedium*>(medium);
#pragma omp parallel for schedule(dynamic, 64)
  for (long i = 0; i < n; ++i) {
    Vector3f P(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
    out_inside[i] = m->mesh->inside(P) ? 1 : 0;
    uint32_t tri = 0xFFFFFFFFu;
    Vector3f q = Vector3f::Zero();
    out[4 * i] = m->mesh->distToPoint(P, tri, q);
    out_tri[i] = tri;
    for (int c = 0; c < 3; ++c) out[4 * i + 1 + c] = q[c];
  }
}

// ---- scenes and the trace loop -------------------------------------------------------
// Load scene.json through Controller::load (controller.cpp:40-264). sky < 0: no sky;
// otherwise a constant skydrome of that radiance (Skydrome() has 1.0, skydrome.cpp:7).
void* ref_scene_load(const char* json_path, float sky) {
  auto* s = new RefScene();
  if (!s->ctrl.load(json_path)) {
    delete s;
    return nullptr;
  }
  if (sky >= 0.0f) {
    if (sky == 1.0f)
      scene_of(s->ctrl)->setSkydrome(std::make_shared<Skydrome>());
    else
      scene_of(s->ctrl)->setSkydrome(std::make_shared<Skydrome>(std::make_shared<ConstantTexture>(Vector3f(sky, sky, sky))));
  }
  return s;
}
// Add a Lambertian mesh with a constant albedo (a scene.json cannot express one).
int ref_scene_add_mesh(void* h, const char* obj_path, float albedo) {
  auto* s = static_cast<RefScene*>(h);
  auto bsdf = std::make_shared<LambertianBsdf>(std::make_shared<ConstantTexture>(Vector3f(albedo, albedo, albedo)));
  auto m = std::make_shared<Mesh>(bsdf);
  if (!m->fetchFrom(obj_path)) return -1;
  scene_of(s->ctrl)->addPrimitive(m);
  return 0;
}
// PathTracerSettings::skip_medium of the render contexts snapshotted from now on
// (Controller::startProgressive sets the global the same way, controller.cpp:302).
void ref_set_skip_medium(int skip) { g_pathTracerSettings.skip_medium = skip != 0; }
// Snapshot the render context and prepare primitives (renderer.cpp:10-16).
void ref_scene_prepare(void* h) {
  auto* s = static_cast<RefScene*>(h);
  s->ctx = std::make_shared<RenderContext>(scene_of(s->ctrl)->cam(), g_pathTracerSettings, g_gpSettings, scene_of(s->ctrl));
  for (auto& prim : (*s->ctx->scene).*member_of(ScenePrimitives())) prim->prepareForRender();
}
void ref_scene_free(void* h) { delete static_cast<RefScene*>(h); }
int ref_scene_spp(void* h) { return static_cast<RefScene*>(h)->ctrl.*member_of(ControllerSpp()); }
void ref_scene_size(void* h, int* w, int* hh) {
  auto* s = static_cast<RefScene*>(h);
  *w = s->ctx->camera.width();
  *hh = s->ctx->camera.height();
}

// PathTracer::trace for n (x, y, k) samples, each exactly as renderer.cpp:36-37 does
// (new PathTracer, seed 42). out[n*3]. OpenMP over samples.
void ref_trace(void* h, long n, const int32_t* x, const int32_t* y, const int32_t* k, float* out) {
  auto* s = static_cast<RefScene*>(h);
  const RenderContext& ctx = *s->ctx;
#pragma omp parallel for schedule(dynamic, 16)
  for (long i = 0; i < n; ++i) {
    PathTracer tracer;
    Vector3f e = tracer.trace(Vector2i(x[i], y[i]), ctx, 42, k[i]);
    out[3 * i] = e.x();
    out[3 * i + 1] = e.y();
    out[3 * i + 2] = e.z();
  }
}

// Full progressive render through Renderer::startRenderProgressive
// (renderer.cpp:22-49). rgb_out[h*w*3] = the averaged framebuffer (row y = camera y).
int ref_render(void* h, int spp, float* rgb_out) {
  auto* s = static_cast<RefScene*>(h);
  Renderer r;
  r.prepareRender(*s->ctx);
  bool ok = r.startRenderProgressive(*s->ctx, spp);
  auto fb = r.getFramebuffer();
  int w = fb->width(), hh = fb->height();
  for (int yy = 0; yy < hh; ++yy)
    for (int xx = 0; xx < w; ++xx) {
      const auto& c = (*fb)(xx, yy).rgb;
      float* o = rgb_out + 3 * ((long)yy * w + xx);
      o[0] = c.x();
      o[1] = c.y();
      o[2] = c.z();
    }
  return ok ? 0 : -1;
}

int ref_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
