// lgpu_flatten.hpp — flattens the reference host's nl::cg::scene into the
// plain structs of include/lambda_gpu.h.
//
// This is the host half of the drop-in for Renderer::render
// (src/renderer.cpp:14).  Mesh geometry and BVH arrays are passed as
// pointers into the scene's own vectors (trimeshdata V/N/F/GN and
// bvh::nodes/bbs/prim_idxs, cg.hpp:766-820, 596-631); only the small
// per-object, per-material and per-light records and the spectra table are
// copied into the flat_scene that owns them.  Compile against the
// reference's headers (cg.hpp) — the host application already has them.
#pragma once

#include <cstring>
#include <vector>

#include "cg.hpp"
#include "lambda_gpu.h"

namespace lgpu_host {

static_assert(sizeof(nl::ℝ3) == 12, "ℝ3 must be three packed floats");
static_assert(sizeof(nl::cg::triangle) == 9 * sizeof(uint32_t),
              "triangle is {V[3], N[3], u[3]}");
static_assert(sizeof(nl::cg::aabb_avx2) == 48 * sizeof(float),
              "aabb_avx2 is inf[3][8], sup[3][8]");
static_assert(sizeof(nl::ℝ4x4) == 16 * sizeof(float), "ℝ4x4 is 16 floats");

struct flat_scene {
  std::vector<lgpu_object> objects;
  std::vector<lgpu_material> materials;
  std::vector<lgpu_light> lights;
  std::vector<lgpu_mesh> meshes;
  std::vector<float> spectra;
  lgpu_scene scene{};
};

inline void copy_transform(nl::cg::transform const& T, lgpu_transform& out) {
  std::memcpy(out.M, T.M.elem, sizeof(out.M));
  std::memcpy(out.M_inv, T.M_inv.elem, sizeof(out.M_inv));
}

inline void copy3(nl::ℝ3 const& v, float* out) {
  out[0] = v[0];
  out[1] = v[1];
  out[2] = v[2];
}

// Appends one coefficientλ<Nλ> to the spectra table, returns its index.
inline int32_t add_spectrum(flat_scene& fs,
                            nl::cg::coefficientλ<nl::cg::Nλ> const& s) {
  int32_t const idx = int32_t(fs.spectra.size() / nl::cg::Nλ);
  for (uint32_t i = 0; i < nl::cg::Nλ; i++) fs.spectra.push_back(s.v[i]);
  return idx;
}

inline void flatten(nl::cg::scene const& sc, flat_scene& fs) {
  using namespace nl::cg;
  using nl::Overload;
  fs = flat_scene{};

  // camera (cg.hpp:1151-1165)
  lgpu_camera& cam = fs.scene.cam;
  copy3(sc.cam.base.x, cam.base_x);
  copy3(sc.cam.base.y, cam.base_y);
  copy3(sc.cam.base.z, cam.base_z);
  copy3(sc.cam.pos, cam.pos);
  cam.fov = sc.cam.fov;
  cam.dof = sc.cam.dof;
  cam.D = sc.cam.D;
  cam.delta = sc.cam.Δ;
  cam.h = sc.cam.h;
  cam.w = sc.cam.w;
  cam.width = sc.cam.width;
  cam.height = sc.cam.height;

  // spectral discretisation (cg.hpp:40-41, 241-247, 329-331)
  coefficientλ<Nλ> const probe(0.f);
  fs.scene.spec.n_bins = Nλ;
  fs.scene.spec.hero_k = HERO_SAMPLES;
  fs.scene.spec.lambda_inf = probe.inf;
  fs.scene.spec.lambda_sup = probe.sup;
  fs.scene.spec.cmf_x = CMF_X.v.elem;
  fs.scene.spec.cmf_y = CMF_Y.v.elem;
  fs.scene.spec.cmf_z = CMF_Z.v.elem;

  // materials (cg.hpp:921-1085)
  for (Material const& m : sc.materials) {
    lgpu_material lm{};
    for (int k = 0; k < 5; k++) lm.spectrum[k] = -1;
    lm.type = int32_t(m.index());
    std::visit(
        Overload{[&](lambertian const& x) {
                   lm.spectrum[0] = add_spectrum(fs, x.albedo);
                 },
                 [&](blinn const& x) {
                   lm.spectrum[0] = add_spectrum(fs, x.Kd);
                   lm.spectrum[1] = add_spectrum(fs, x.Ks);
                   lm.spectrum[2] = add_spectrum(fs, x.Kt);
                   lm.spectrum[3] = add_spectrum(fs, x.Le);
                   lm.spectrum[4] = add_spectrum(fs, x.ior);
                   lm.alpha = x.α;
                   lm.p_d = x.p_d;
                   lm.p_spec = x.p_spec;
                   lm.w_r = x.w_r;
                   lm.w_t = x.w_t;
                 },
                 [&](thinfilm const& x) {
                   lm.spectrum[0] = add_spectrum(fs, x.film_ior);
                   lm.spectrum[1] = add_spectrum(fs, x.base_ior);
                   lm.alpha = x.α;
                   lm.d = x.d;
                 },
                 [&](microfacet const& x) {
                   lm.spectrum[0] = add_spectrum(fs, x.albedo);
                   lm.spectrum[1] = add_spectrum(fs, x.ior);
                 },
                 [&](emitter const& x) {
                   lm.spectrum[0] = add_spectrum(fs, x.radiance);
                 },
                 [&](diremitter const& x) {
                   lm.spectrum[0] = add_spectrum(fs, x.radiance);
                   lm.specular = x.specular;
                 }},
        m);
    fs.materials.push_back(lm);
  }

  // objects (cg.hpp:835-857)
  for (Object const& o : sc.objects) {
    lgpu_object lo{};
    lo.type = int32_t(o.index());
    std::visit(Overload{[&](sphere const& x) {
                          lo.mat = x.mat;
                          copy_transform(x.T, lo.T);
                        },
                        [&](plane const& x) {
                          lo.mat = x.mat;
                          copy_transform(x.T, lo.T);
                        },
                        [&](trimesh const& x) {
                          lo.mat = x.mat;
                          lo.mesh = x.mesh;
                          copy_transform(x.T, lo.T);
                        }},
               o);
    fs.objects.push_back(lo);
  }

  // lights (cg.hpp:875-905)
  for (Light const& l : sc.lights) {
    lgpu_light ll{};
    ll.type = int32_t(l.index());
    std::visit(Overload{[&](ambientlight const& x) {
                          ll.spectrum = add_spectrum(fs, x.radiance);
                        },
                        [&](pointlight const& x) {
                          ll.spectrum = add_spectrum(fs, x.radiant_intensity);
                          copy3(x.pos, ll.pos);
                        },
                        [&](dirlight const& x) {
                          ll.spectrum = add_spectrum(fs, x.radiant_intensity);
                          copy3(x.dir, ll.dir);
                        },
                        [&](spherelight const& x) {
                          ll.spectrum = add_spectrum(fs, x.radiance);
                          ll.size = x.size;
                          ll.obj = x._sphere.obj;
                          copy_transform(x._sphere.T, ll.T);
                        },
                        [&](quaddirlight const& x) {
                          ll.spectrum = add_spectrum(fs, x.radiance);
                          ll.inv_area = x.inv_area;
                          ll.spec = x.spec;
                          ll.obj = x._plane.obj;
                          copy_transform(x._plane.T, ll.T);
                        }},
               l);
    fs.lights.push_back(ll);
  }

  // meshes: zero-copy views of trimeshdata and its bvh (cg.hpp:766-820)
  for (Mesh const& mv : sc.meshes) {
    trimeshdata const& m = std::get<trimeshdata>(mv);
    lgpu_mesh lm{};
    lm.n_positions = uint32_t(m.V.size());
    lm.n_normals = uint32_t(m.N.size());
    lm.n_faces = uint32_t(m.F.size());
    lm.f_stride = 9;
    lm.V = m.V.empty() ? nullptr : m.V.data()->elem;
    lm.N = m.N.empty() ? nullptr : m.N.data()->elem;
    lm.F = m.F.empty() ? nullptr : m.F.data()->V;
    lm.GN = m.GN.empty() ? nullptr : m.GN.data()->elem;
    copy3(m.bounds.inf, lm.bounds);
    copy3(m.bounds.sup, lm.bounds + 3);
    lm.n_nodes = uint32_t(m._bvh.nodes.size());
    lm.n_bbs = uint32_t(m._bvh.bbs.size());
    lm.n_prim_idxs = uint32_t(m._bvh.prim_idxs.size());
    lm.nodes = reinterpret_cast<uint32_t const*>(m._bvh.nodes.data());
    lm.bbs = reinterpret_cast<float const*>(m._bvh.bbs.data());
    lm.prim_idxs = m._bvh.prim_idxs.data();
    fs.meshes.push_back(lm);
  }

  fs.scene.n_objects = uint32_t(fs.objects.size());
  fs.scene.n_materials = uint32_t(fs.materials.size());
  fs.scene.n_lights = uint32_t(fs.lights.size());
  fs.scene.n_meshes = uint32_t(fs.meshes.size());
  fs.scene.n_spectra = uint32_t(fs.spectra.size() / Nλ);
  fs.scene.objects = fs.objects.data();
  fs.scene.materials = fs.materials.data();
  fs.scene.lights = fs.lights.data();
  fs.scene.meshes = fs.meshes.data();
  fs.scene.spectra = fs.spectra.data();
}

}  // namespace lgpu_host
