// GpuRenderer (gpu_renderer.h): the reference scene flattened into the C ABI
// of libmupsi_gpu.so, and the progressive render through it.
#include "gpu_renderer.h"

#include <cmath>
#include <iostream>
#include <map>

#include "geometry/primitive.h"
#include "geometry/scene.h"
#include "gp/gpnoise.h"
#include "gp/kernel.h"
#include "gp/meanfunction.h"
#include "medium/externalgpmedium.h"
#include "medium/gpmedium.h"
#include "medium/sdfmedium.h"
#include "primitives/mesh.h"
#include "primitives/skydrome.h"
#include "primitives/sphere.h"
#include "rendering/camera.h"
#include "texture/texture.h"

namespace mupsi {
namespace gpu_access {
// The private members GpuRenderer reads. In the reference tree these are plain
// member reads (the classes declare GpuRenderer a friend). Built beside an
// unmodified reference, the same reads go through pointers to the members,
// formed in explicit template instantiations (where the language allows
// naming private members).
template <typename Tag, typename Tag::type M>
struct Reader {
  friend typename Tag::type member(Tag) { return M; }
};
#define MUPSI_MEMBER(TAG, CLASS, TYPE, NAME) \
  struct TAG {                               \
    using type = TYPE CLASS::*;              \
    friend type member(TAG);                 \
  };                                         \
  template struct Reader<TAG, &CLASS::NAME>;

MUPSI_MEMBER(ScenePrimitives, Scene, std::vector<std::shared_ptr<Primitive>>, primitives_)
MUPSI_MEMBER(CameraUp, Camera, Vector3f, up_)
MUPSI_MEMBER(GpMean, GPMedium, std::shared_ptr<MeanFunction>, mean_)
MUPSI_MEMBER(GpNoise, GPMedium, std::shared_ptr<SparseGPNoiseGenerator>, noiseGenerator_)
MUPSI_MEMBER(SdfMean, SDFMedium, std::shared_ptr<MeanFunction>, mean_)
MUPSI_MEMBER(ExtMean, ExternalGPMedium, std::shared_ptr<GridMeanFunction>, mean_)
MUPSI_MEMBER(ExtVar, ExternalGPMedium, std::shared_ptr<GridMeanFunction>, variance_)
MUPSI_MEMBER(ExtScale, ExternalGPMedium, float, noiseScale_)
MUPSI_MEMBER(NoiseDensity, SparseGPNoiseGenerator, int, impulseDensity_)
MUPSI_MEMBER(SphereCenter, SphereMeanFunction, Vector3f, center_)
MUPSI_MEMBER(SphereRadius, SphereMeanFunction, float, radius_)
MUPSI_MEMBER(MeshOfMean, MeshMeanFunction, std::shared_ptr<Mesh>, mesh_)
MUPSI_MEMBER(GridData, GridMeanFunction, std::vector<float>, data_)
MUPSI_MEMBER(GridRes, GridMeanFunction, int, res_)
MUPSI_MEMBER(GridMin, GridMeanFunction, Vector3f, bounds_min_)
MUPSI_MEMBER(GridMax, GridMeanFunction, Vector3f, bounds_max_)
MUPSI_MEMBER(MeshVertices, Mesh, std::vector<Vector3f>, vertices_)
MUPSI_MEMBER(MeshNormals, Mesh, std::vector<Vector3f>, normals_)
MUPSI_MEMBER(MeshTexcoords, Mesh, std::vector<Vector2f>, texcoords_)
MUPSI_MEMBER(MeshFaces, Mesh, std::vector<Vector3i>, faces_)
MUPSI_MEMBER(MeshFaceTex, Mesh, std::vector<Vector3i>, faceTexIndices_)
MUPSI_MEMBER(LambertAlbedo, LambertianBsdf, std::shared_ptr<Texture>, albedo_)
MUPSI_MEMBER(BitmapW, BitmapTexture, int, w_)
MUPSI_MEMBER(BitmapH, BitmapTexture, int, h_)
MUPSI_MEMBER(BitmapData, BitmapTexture, std::vector<Vector3f>, data_)
#undef MUPSI_MEMBER
}  // namespace gpu_access

namespace {
using namespace gpu_access;

void put3(float* d, const Vector3f& v) {
  d[0] = v[0];
  d[1] = v[1];
  d[2] = v[2];
}

// What the library needs of a texture: a constant colour (ConstantTexture, read
// through its lookup), or the texels of a BitmapTexture (row 0 at the top).
struct TexInfo {
  bool bitmap = false;
  Vector3f color;
  int w = 0, h = 0;
  std::vector<float> rgb;
};
TexInfo texture_info(const Texture* t) {
  TexInfo ti;
  if (const auto* b = dynamic_cast<const BitmapTexture*>(t)) {
    ti.bitmap = true;
    ti.w = b->*member(BitmapW{});
    ti.h = b->*member(BitmapH{});
    const auto& px = b->*member(BitmapData{});
    ti.rgb.resize(px.size() * 3);
    for (size_t i = 0; i < px.size(); ++i) put3(&ti.rgb[3 * i], px[i]);
  } else if (t) {
    ti.color = (*t)[Vector2f(0.0f, 0.0f)];
  }
  return ti;
}

// A Primitive transform the descriptor can express: Translation(c) * Scaling(s).
bool translation_scaling(const Matrix4f& m, float* c, float* s) {
  const float k = m(0, 0);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      if (m(i, j) != (i == j ? k : 0.0f)) return false;
  if (m(3, 0) != 0.0f || m(3, 1) != 0.0f || m(3, 2) != 0.0f || m(3, 3) != 1.0f) return false;
  for (int i = 0; i < 3; ++i) c[i] = m(i, 3);
  *s = k;
  return true;
}

// Host copies of the arrays the descriptors point at (valid until create).
struct MeshArrays {
  const Mesh* mesh = nullptr;
  std::vector<float> v, n;
  std::vector<int32_t> f;
};

}  // namespace

GpuRenderer::~GpuRenderer() {
  if (scene_) mupsi_gpu_scene_destroy(scene_);
}

bool GpuRenderer::fail(const std::string& msg) {
  error_ = msg;
  std::cerr << "GpuRenderer: " << msg << std::endl;
  return false;
}

bool GpuRenderer::prepareRender(const RenderContext& ctx) {
  if (scene_) {
    mupsi_gpu_scene_destroy(scene_);
    scene_ = nullptr;
  }
  const Camera& cam = ctx.camera;
  const Scene& sc = *ctx.scene;
  mupsi_scene_desc d{};
  d.width = cam.width();
  d.height = cam.height();
  d.spp = ctx.pts.spp;
  d.max_bounce = ctx.pts.max_bounce;
  d.max_medium_bounce = ctx.pts.max_medium_bounce;
  d.gp_mode = ctx.gp.gpMode == GPSettings::GPCorrelationMode::RenewalPlus ? MUPSI_GP_RENEWAL_PLUS
                                                                         : MUPSI_GP_SINGLE_REALIZATION;
  // Camera keeps its direction and up normalised; the library normalises them
  // again, which returns them unchanged unless the stored vector's squared
  // norm rounds below 1 (then the frame moves by an ulp)
  put3(d.cam_pos, cam.pos());
  put3(d.cam_dir, cam.dir());
  put3(d.cam_up, cam.*member(CameraUp{}));
  d.cam_fov = cam.fov();
  d.eps = ctx.pts.eps;
  d.nearteps = ctx.pts.nearteps;
  TexInfo sky;
  if (auto sd = sc.getSkydrome()) {
    sky = texture_info(sd->getEmission());
    d.has_sky = 1;
    if (!sky.bitmap) put3(d.sky, sky.color);
  }

  std::vector<mupsi_primitive_desc> prims;
  std::vector<mupsi_medium_desc> media;
  std::vector<mupsi_mesh_desc> meshes;
  std::vector<MeshArrays> arrays;
  std::vector<const Medium*> medium_of;
  std::map<const Medium*, int> medium_index;
  std::map<const Mesh*, int> mesh_index;
  struct Later {  // settings applied after the scene exists
    int medium = -1, kind = MUPSI_MEDIUM_GP;
    const ExternalGPMedium* ext = nullptr;
  };
  std::vector<Later> later;
  struct TexLater {
    int prim;
    const Mesh* mesh;
    TexInfo tex;
  };
  std::vector<TexLater> textures;

  auto add_mesh = [&](const Mesh* m, const Matrix4f& T) -> int {
    auto it = mesh_index.find(m);
    if (it != mesh_index.end()) return it->second;
    mupsi_mesh_desc md{};
    float c[3], s;
    if (!translation_scaling(T, c, &s)) return -1;
    MeshArrays a;
    a.mesh = m;
    const auto& V = m->*member(MeshVertices{});
    const auto& N = m->*member(MeshNormals{});
    const auto& F = m->*member(MeshFaces{});
    a.v.resize(V.size() * 3);
    for (size_t i = 0; i < V.size(); ++i) put3(&a.v[3 * i], V[i]);
    // Mesh::interpolateNormal indexes normals_ by vertex id; fewer normals than
    // vertices leave the shading on face normals
    if (N.size() >= V.size() && !V.empty()) {
      a.n.resize(V.size() * 3);
      for (size_t i = 0; i < V.size(); ++i) put3(&a.n[3 * i], N[i]);
    }
    a.f.resize(F.size() * 3);
    for (size_t i = 0; i < F.size(); ++i)
      for (int k = 0; k < 3; ++k) a.f[3 * i + k] = F[i][k];
    arrays.push_back(std::move(a));
    md.num_vertices = (int64_t)V.size();
    md.num_faces = (int64_t)F.size();
    md.position[0] = c[0];
    md.position[1] = c[1];
    md.position[2] = c[2];
    md.scale = s;
    meshes.push_back(md);
    const int idx = (int)meshes.size() - 1;
    mesh_index[m] = idx;
    return idx;
  };

  // a medium: its descriptor (mean + kernel) and, for SDF / external GP media,
  // the setter applied after create
  std::string why;
  auto add_medium = [&](const std::shared_ptr<Medium>& mp) -> int {
    if (!mp) return -1;
    const Medium* m = mp.get();
    auto it = medium_index.find(m);
    if (it != medium_index.end()) return it->second;
    mupsi_medium_desc md{};
    md.mean_type = MUPSI_MEAN_SPHERE;
    md.mean_radius = 1.0f;
    md.kernel.sigma = 1.0f;
    md.kernel.kernel_radius = 1.0f;
    md.kernel.aniso[0] = md.kernel.aniso[1] = md.kernel.aniso[2] = 1.0f;
    md.kernel.points_per_cell = 3;
    Later lt;
    const MeanFunction* mean = nullptr;
    if (const auto* g = dynamic_cast<const GPMedium*>(m)) {
      mean = (g->*member(GpMean{})).get();
      const auto& gen = g->*member(GpNoise{});
      const auto* k = dynamic_cast<const SparseSEKernel*>(gen->getKernel().get());
      if (!k) {
        why = "GPMedium without a SparseSEKernel";
        return -2;
      }
      md.kernel.sigma = k->getSigma();
      md.kernel.kernel_radius = k->getKernelRadius();
      put3(md.kernel.aniso, k->getLengthScale());
      md.kernel.points_per_cell = (*gen).*member(NoiseDensity{});
    } else if (const auto* s = dynamic_cast<const SDFMedium*>(m)) {
      mean = (s->*member(SdfMean{})).get();
      lt.kind = MUPSI_MEDIUM_SDF;
    } else if (const auto* e = dynamic_cast<const ExternalGPMedium*>(m)) {
      lt.kind = MUPSI_MEDIUM_EXTERNAL_GP;
      lt.ext = e;
    } else {
      why = "unknown medium type";
      return -2;
    }
    if (const auto* sm = dynamic_cast<const SphereMeanFunction*>(mean)) {
      md.mean_type = MUPSI_MEAN_SPHERE;
      put3(md.mean_center, sm->*member(SphereCenter{}));
      md.mean_radius = sm->*member(SphereRadius{});
    } else if (const auto* mm = dynamic_cast<const MeshMeanFunction*>(mean)) {
      const auto& mesh = mm->*member(MeshOfMean{});
      md.mean_type = MUPSI_MEAN_MESH;
      md.mean_mesh = add_mesh(mesh.get(), mesh->getTransform());
      if (md.mean_mesh < 0) {
        why = "mesh mean transform is not a translation and uniform scaling";
        return -2;
      }
    } else if (mean) {
      why = "unsupported mean function";
      return -2;
    }
    media.push_back(md);
    const int idx = (int)media.size() - 1;
    medium_index[m] = idx;
    if (lt.kind != MUPSI_MEDIUM_GP) {
      lt.medium = idx;
      later.push_back(lt);
    }
    return idx;
  };

  const auto& P = sc.*member(ScenePrimitives{});
  for (size_t i = 0; i < P.size(); ++i) {
    const Primitive* pr = P[i].get();
    mupsi_primitive_desc pd{};
    if (dynamic_cast<const Sphere*>(pr)) {
      pd.type = MUPSI_PRIM_SPHERE;
      if (!translation_scaling(pr->getTransform(), pd.center, &pd.radius))
        return fail("sphere transform is not a translation and uniform scaling");
    } else if (const auto* m = dynamic_cast<const Mesh*>(pr)) {
      pd.type = MUPSI_PRIM_MESH;
      pd.mesh = add_mesh(m, m->getTransform());
      if (pd.mesh < 0) return fail("mesh transform is not a translation and uniform scaling");
    } else {
      return fail("unsupported primitive type");
    }
    const Bsdf* b = pr->getBsdf(0);
    if (const auto* lb = dynamic_cast<const LambertianBsdf*>(b)) {
      pd.bsdf = MUPSI_BSDF_LAMBERTIAN;
      TexInfo ti = texture_info((lb->*member(LambertAlbedo{})).get());
      if (ti.bitmap) {
        if (pd.type != MUPSI_PRIM_MESH) return fail("bitmap albedo on a sphere");
        textures.push_back({(int)i, dynamic_cast<const Mesh*>(pr), std::move(ti)});
        pd.albedo[0] = pd.albedo[1] = pd.albedo[2] = 0.8f;
      } else {
        put3(pd.albedo, ti.color);
      }
    } else if (dynamic_cast<const NullBsdf*>(b)) {
      pd.bsdf = MUPSI_BSDF_NULL;
    } else if (dynamic_cast<const SpecularBsdf*>(b)) {
      pd.bsdf = MUPSI_BSDF_SPECULAR;
    } else {
      return fail("unsupported BSDF");
    }
    // Scene::chooseLight takes every primitive with an emission texture
    if (const Texture* em = pr->getEmission()) {
      TexInfo ti = texture_info(em);
      if (ti.bitmap) return fail("bitmap emission");
      pd.has_emission = 1;
      put3(pd.emission, ti.color);
    }
    pd.int_medium = add_medium(pr->getIntMedium());
    pd.ext_medium = add_medium(pr->getExtMedium());
    if (pd.int_medium == -2 || pd.ext_medium == -2) return fail(why);
    prims.push_back(pd);
  }
  for (size_t i = 0; i < meshes.size(); ++i) {
    meshes[i].vertices = arrays[i].v.data();
    meshes[i].faces = arrays[i].f.data();
    meshes[i].vertex_normals = arrays[i].n.empty() ? nullptr : arrays[i].n.data();
  }
  d.num_media = (int32_t)media.size();
  d.media = media.data();
  d.num_meshes = (int32_t)meshes.size();
  d.meshes = meshes.data();
  d.num_primitives = (int32_t)prims.size();
  d.primitives = prims.data();
  if (mupsi_gpu_scene_create(&d, &scene_) != MUPSI_OK) return fail(mupsi_gpu_last_error());

  int rc = MUPSI_OK;
  if (sky.bitmap) rc = mupsi_gpu_scene_set_sky_texture(scene_, sky.w, sky.h, sky.rgb.data());
  for (const auto& lt : later) {
    if (rc != MUPSI_OK) break;
    if (lt.kind == MUPSI_MEDIUM_SDF) {
      rc = mupsi_gpu_scene_set_sdf_medium(scene_, lt.medium);
    } else {
      const GridMeanFunction& gm = *(lt.ext->*member(ExtMean{}));
      const auto& var = lt.ext->*member(ExtVar{});
      float lo[3], hi[3];
      put3(lo, gm.*member(GridMin{}));
      put3(hi, gm.*member(GridMax{}));
      rc = mupsi_gpu_scene_set_external_gp_medium(scene_, lt.medium, gm.*member(GridRes{}), lo, hi,
                                                  (gm.*member(GridData{})).data(),
                                                  var ? ((*var).*member(GridData{})).data() : nullptr,
                                                  lt.ext->*member(ExtScale{}));
    }
  }
  for (const auto& t : textures) {
    if (rc != MUPSI_OK) break;
    const auto& uv = t.mesh->*member(MeshTexcoords{});
    const auto& ft = t.mesh->*member(MeshFaceTex{});
    std::vector<float> tc(uv.size() * 2);
    for (size_t i = 0; i < uv.size(); ++i) {
      tc[2 * i] = uv[i][0];
      tc[2 * i + 1] = uv[i][1];
    }
    std::vector<int32_t> fi(ft.size() * 3);
    for (size_t i = 0; i < ft.size(); ++i)
      for (int k = 0; k < 3; ++k) fi[3 * i + k] = ft[i][k];
    const bool has_uv = !uv.empty() && !ft.empty();
    rc = mupsi_gpu_scene_set_albedo_texture(scene_, t.prim, has_uv ? (int64_t)uv.size() : 0,
                                            has_uv ? tc.data() : nullptr, has_uv ? fi.data() : nullptr, t.tex.w,
                                            t.tex.h, t.tex.rgb.data());
  }
  if (rc == MUPSI_OK && ctx.pts.skip_medium) rc = mupsi_gpu_scene_set_skip_medium(scene_, 1);
  if (rc != MUPSI_OK) return fail(mupsi_gpu_last_error());

  width_ = d.width;
  height_ = d.height;
  rgb_.assign((size_t)width_ * height_ * 3, 0.0f);
  framebuffer_ = std::make_shared<Framebuffer>(width_, height_);
  error_.clear();
  return true;
}

bool GpuRenderer::startRenderProgressive(const RenderContext& ctx, int targetSpp,
                                         std::function<void(int currentSpp)> onSpp) {
  (void)ctx;  // the scene was flattened from it in prepareRender
  if (!scene_) return fail("prepareRender has not succeeded");
  // the library polls a plain word between waves; the host's atomic flag is
  // mirrored into it before the render and after every wave
  volatile int32_t cancel_word = (cancel_ && cancel_->load()) ? 1 : 0;
  struct Hook {
    std::function<void(int)>* on;
    std::atomic<bool>* cancel;
    volatile int32_t* word;
  } hook{&onSpp, cancel_, &cancel_word};
  mupsi_render_args a{};
  a.spp_begin = 0;
  a.spp_end = targetSpp;
  a.cancel = &cancel_word;
  a.on_spp = [](int32_t passes, void* user) {
    auto* h = static_cast<Hook*>(user);
    if (*h->on) (*h->on)(passes);
    if (h->cancel && h->cancel->load()) *h->word = 1;
  };
  a.user = &hook;
  a.rgb_out = rgb_.data();
  a.out_mem = MUPSI_MEM_HOST;
  const int rc = mupsi_gpu_render(scene_, &a);
  if (rc == MUPSI_ERR_CANCELLED) return false;
  if (rc != MUPSI_OK) return fail(mupsi_gpu_last_error());
  // pixels = running sum / passes, as Framebuffer::accumulate leaves them
  for (int y = 0; y < height_; ++y)
    for (int x = 0; x < width_; ++x) {
      const float* v = &rgb_[((size_t)y * width_ + x) * 3];
      (*framebuffer_)(x, y).rgb = Vec3f(v[0], v[1], v[2]);
    }
  while (framebuffer_->sampleCount() < targetSpp) framebuffer_->incrementSampleCount();
  return true;
}

}  // namespace mupsi
