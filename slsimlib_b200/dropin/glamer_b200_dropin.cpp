// Link-level drop-in for GLAMER's ray shooting: the ray-shooting members of
// class Lens, compiled against the application's own GLAMER headers
// (include/lens.h) and linked in place of FullRange/internal_rayshooter_multi.cpp.
// Every caller of Lens::rayshooterInternal -- GridMap, Grid and its
// refinement (TreeCode_link/grid_maintenance.cpp), ImageFinding::find_crit
// (TreeCode_link/find_crit.cpp), the image finders -- then shoots its rays on
// the GPU through the C ABI of libglamer_b200.so without a source change.
//
// Each Lens gets a mirror on the device (a glb_lens holding the same main
// halos in the same order, so the same planes): built on the lens's first
// ray-shooting call, rebuilt when its halos or plane redshifts change, and
// kept until glamer_b200_dropin::release(lens) or the end of the process.
// Supported main halos: LensHaloParticles<ParticleType<float>>, spherical
// LensHaloNFW and LensHaloRealNSIE; anything else (other profiles, field
// planes) throws std::runtime_error -- there is no CPU path.
//
// Build: g++ -std=c++17 -I<GLAMER>/include -I<this repo>/include -c
//        glamer_b200_dropin.cpp, link with -lglamer_b200 and without
//        internal_rayshooter_multi.o (its other members -- info_rayshooter,
//        mass_on_planes, compute_rays_parallel, find_image_min,
//        find_images_min_parallel -- evaluate planes on the CPU and are not
//        defined here).
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "lens.h"
#include "particle_halo.h"
#include "glamer_b200.h"
#include "glamer_b200_dropin.hpp"

namespace {

using PartT = ParticleType<float>;
static_assert(sizeof(PartT) == sizeof(glb_particle), "ParticleType<float> must be the 24-byte record");

// Protected members of the reference's classes, read through pointers to
// members named in derived classes (the access rule of [class.protected]
// applies to naming the member, not to using the pointer).
template <class P>
struct ParticlesView : LensHaloParticles<P> {
  static P *LensHaloParticles<P>::*pp_member() { return &ParticlesView::pp; }
  static size_t LensHaloParticles<P>::*n_member() { return &ParticlesView::Npoints; }
  static double LensHaloParticles<P>::*inv_area_member() { return &ParticlesView::inv_area; }
  static TreeQuadParticles<P> *LensHaloParticles<P>::*tree_member() { return &ParticlesView::qtree; }
};
template <class P>
struct TreeView : TreeQuadParticles<P> {
  static PosType TreeQuadParticles<P>::*screen2_member() { return &TreeView::inv_screening_scale2; }
};
struct HaloView : LensHalo {
  static float LensHalo::*fratio_member() { return &HaloView::fratio; }
  static float LensHalo::*pa_member() { return &HaloView::pa; }
};

void check(int rc) {
  if (rc != 0) throw std::runtime_error(std::string("glamer_b200 drop-in: ") + glb_last_error());
}

// A float c with Rsize / c == rscale in float arithmetic, as the NFW
// constructor forms rscale (MultiPlane/lens_halos.cpp:411).
float concentration_for(float Rsize, float rscale) {
  float c = Rsize / rscale;
  for (int k = 0; k < 64 && Rsize / c != rscale; ++k) c = std::nextafter(c, (Rsize / c > rscale) ? 1e38f : 0.0f);
  if (Rsize / c != rscale) throw std::runtime_error("glamer_b200 drop-in: NFW scale radius not reproducible");
  return c;
}

struct Mirror {
  glb_lens *g = nullptr;
  std::vector<const LensHalo *> halos;  // the main halos mirrored, in order
  std::vector<PosType> plane_z;         // the reference's plane redshifts at mirroring
  ~Mirror() {
    if (g) glb_lens_destroy(g);
  }
};

std::mutex g_mu;
std::map<const Lens *, std::unique_ptr<Mirror>> g_mirrors;
int g_precision = GLB_PREC_FP64;

glb_halo *mirror_halo(LensHalo *h, const COSMOLOGY &) {
  glb_halo *out = nullptr;
  PosType theta[2];
  h->getTheta(theta);
  if (auto *p = dynamic_cast<LensHaloParticles<PartT> *>(h)) {
    const PartT *pp = p->*ParticlesView<PartT>::pp_member();
    const size_t n = p->*ParticlesView<PartT>::n_member();
    const double inv_area = p->*ParticlesView<PartT>::inv_area_member();
    TreeQuadParticles<PartT> *t = p->*ParticlesView<PartT>::tree_member();
    const double screen2 = t ? (double)(t->*TreeView<PartT>::screen2_member()) : 0.0;
    // glb_halo_particles screens by the square of its max_range argument, as
    // LensHaloParticles::set_up passes max_range to the tree (particle_halo.h:416)
    check(glb_halo_particles(reinterpret_cast<const glb_particle *>(pp), n, (double)p->getZlens(), inv_area,
                             std::sqrt(screen2), &out));
  } else if (auto *f = dynamic_cast<LensHaloNFW *>(h)) {
    if (f->*HaloView::fratio_member() != 1.0f)
      throw std::runtime_error("glamer_b200 drop-in: elliptical NFW halos are not supported");
    check(glb_halo_nfw(f->get_mass(), f->getRsize(), f->getZlens(), concentration_for(f->getRsize(), f->get_rscale()),
                       1.0f, 0.0f, &out));
  } else if (auto *s = dynamic_cast<LensHaloRealNSIE *>(h)) {
    check(glb_halo_nsie_state(s->get_mass(), s->getRsize(), s->get_Rmax(), s->getZlens(), s->get_sigma(),
                              s->get_rcore(), s->get_fratio(), s->get_pa(), &out));
  } else {
    throw std::runtime_error("glamer_b200 drop-in: unsupported main halo type (particles, NFW and NSIE only)");
  }
  if (int rc = glb_halo_set_theta(out, theta[0], theta[1])) {
    glb_halo_destroy(out);
    check(rc);
  }
  return out;
}

}  // namespace

namespace glamer_b200_dropin {

void set_precision(int precision) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_precision = precision;
}

void release(const Lens *lens) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_mirrors.erase(lens);
}

}  // namespace glamer_b200_dropin

// The device mirror of this lens, (re)built when its main halos or plane
// redshifts differ from the mirrored ones; its source plane follows the
// lens's (ResetSourcePlane / RevertSourcePlane).
static glb_lens *mirror_of(Lens *L, const std::vector<PosType> &plane_z, bool toggle, PosType zs_implant,
                           size_t nfield, const COSMOLOGY &cosmo) {
  if (nfield) throw std::runtime_error("glamer_b200 drop-in: field halos are not supported");
  std::lock_guard<std::mutex> lk(g_mu);
  std::unique_ptr<Mirror> &m = g_mirrors[L];
  std::vector<const LensHalo *> halos(L->getNMainHalos());
  for (size_t i = 0; i < halos.size(); ++i) halos[i] = L->getMainHalo(i);
  if (!m || m->halos != halos || m->plane_z != plane_z) {
    auto n = std::make_unique<Mirror>();
    check(glb_lens_create(plane_z.back(), cosmo.getOmega_matter(), cosmo.getOmega_lambda(), cosmo.gethubble(),
                          &n->g));
    for (size_t i = 0; i < halos.size(); ++i)
      check(glb_lens_insert_halo(n->g, mirror_halo(L->getMainHalo(i), cosmo), 1));
    std::vector<double> z(plane_z.size());
    check(glb_lens_planes(n->g, z.data(), nullptr, nullptr));
    for (size_t j = 0; j + 1 < plane_z.size(); ++j)
      if (z[j] != plane_z[j]) throw std::runtime_error("glamer_b200 drop-in: mirrored planes differ from the lens's");
    n->halos = halos;
    n->plane_z = plane_z;
    m = std::move(n);
  }
  int j = 0;
  check(glb_lens_reset_source(m->g, toggle ? zs_implant : plane_z.back(), 0, &j));
  return m->g;
}

// Lens::rayshooterInternal(Npoints, Point*) (FullRange/internal_rayshooter_multi.cpp:53-118):
// source positions into i_points[].image->x, the Jacobian into A of both
// points, dt = 0; points with in_image == MAYBE untouched.
void Lens::rayshooterInternal(unsigned long Npoints, Point *i_points, bool) {
  if (flag_switch_lensing_off || flag_switch_deflection_off)
    throw std::runtime_error("glamer_b200 drop-in: lensing/deflection switches are not supported");
  if (plane_redshifts.size() == 1) {  // no lens plane
    for (unsigned long i = 0; i < Npoints; ++i) {
      i_points[i].image->x[0] = i_points[i].x[0];
      i_points[i].image->x[1] = i_points[i].x[1];
      i_points[i].dt = i_points[i].image->dt = 0;
      i_points[i].A.setToI();
      i_points[i].image->A.setToI();
    }
    return;
  }
  if (Npoints == 0) return;
  glb_lens *g = mirror_of(this, plane_redshifts, toggle_source_plane, zs_implant, field_halos.size(), cosmo);
  std::vector<double> x(2 * Npoints), y(2 * Npoints), A(4 * Npoints);
  std::vector<unsigned char> skip(Npoints), status(Npoints);
  for (unsigned long i = 0; i < Npoints; ++i) {
    x[2 * i] = i_points[i].x[0];
    x[2 * i + 1] = i_points[i].x[1];
    skip[i] = i_points[i].in_image == MAYBE;
  }
  check(glb_lens_rayshoot_status(g, Npoints, x.data(), nullptr, skip.data(), y.data(), A.data(), status.data(),
                                 g_precision));
  for (unsigned long i = 0; i < Npoints; ++i) {
    if (status[i] == GLB_RAY_SKIPPED) continue;
    Point &p = i_points[i];
    p.image->x[0] = y[2 * i];
    p.image->x[1] = y[2 * i + 1];
    for (int c = 0; c < 4; ++c) p.A.a[c] = A[4 * i + c];
    p.image->A = p.A;
    p.dt = p.image->dt = 0;
  }
}

// Lens::rayshooterInternal(Npoints, LinkedPoint*, source_zs) (internal_rayshooter_multi.cpp:120-182).
void Lens::rayshooterInternal(unsigned long Npoints, LinkedPoint *i_points, std::vector<double> &source_zs, bool) {
  if (source_zs.size() != Npoints) throw std::invalid_argument("missing redshifts");
  if (flag_switch_lensing_off || flag_switch_deflection_off)
    throw std::runtime_error("glamer_b200 drop-in: lensing/deflection switches are not supported");
  if (plane_redshifts.size() == 1) {
    for (unsigned long i = 0; i < Npoints; ++i) {
      i_points[i].image->x[0] = i_points[i].x[0];
      i_points[i].image->x[1] = i_points[i].x[1];
      i_points[i].dt = i_points[i].image->dt = 0;
      i_points[i].A.setToI();
      i_points[i].image->A.setToI();
    }
    return;
  }
  if (Npoints == 0) return;
  glb_lens *g = mirror_of(this, plane_redshifts, toggle_source_plane, zs_implant, field_halos.size(), cosmo);
  std::vector<double> x(2 * Npoints), y(2 * Npoints), A(4 * Npoints);
  std::vector<unsigned char> skip(Npoints), status(Npoints);
  for (unsigned long i = 0; i < Npoints; ++i) {
    x[2 * i] = i_points[i].x[0];
    x[2 * i + 1] = i_points[i].x[1];
    skip[i] = i_points[i].in_image == MAYBE;
  }
  check(glb_lens_rayshoot_status(g, Npoints, x.data(), source_zs.data(), skip.data(), y.data(), A.data(),
                                 status.data(), g_precision));
  for (unsigned long i = 0; i < Npoints; ++i) {
    if (status[i] == GLB_RAY_SKIPPED) continue;
    LinkedPoint &p = i_points[i];
    p.image->x[0] = y[2 * i];
    p.image->x[1] = y[2 * i + 1];
    for (int c = 0; c < 4; ++c) p.A.a[c] = A[4 * i + c];
    p.image->A = p.A;
    p.dt = p.image->dt = 0;
  }
}

// Lens::rayshooterInternal(Npoints, RAY*) (internal_rayshooter_multi.cpp:184-235):
// one source redshift per ray (RAY::z; a RAY's default z = -1 lies in front
// of every plane, so such a ray is not deflected, as in the reference).
void Lens::rayshooterInternal(unsigned long Npoints, RAY *rays) {
  if (flag_switch_lensing_off || flag_switch_deflection_off)
    throw std::runtime_error("glamer_b200 drop-in: lensing/deflection switches are not supported");
  if (plane_redshifts.size() == 1) {
    for (unsigned long i = 0; i < Npoints; ++i) {
      rays[i].y[0] = rays[i].x[0];
      rays[i].y[1] = rays[i].x[1];
      rays[i].dt = 0;
      rays[i].A.setToI();
    }
    return;
  }
  if (Npoints == 0) return;
  glb_lens *g = mirror_of(this, plane_redshifts, toggle_source_plane, zs_implant, field_halos.size(), cosmo);
  std::vector<double> x(2 * Npoints), zs(Npoints), y(2 * Npoints), A(4 * Npoints);
  for (unsigned long i = 0; i < Npoints; ++i) {
    x[2 * i] = rays[i].x[0];
    x[2 * i + 1] = rays[i].x[1];
    zs[i] = rays[i].z;
  }
  check(glb_lens_rayshoot(g, Npoints, x.data(), zs.data(), y.data(), A.data(), g_precision));
  for (unsigned long i = 0; i < Npoints; ++i) {
    rays[i].y[0] = y[2 * i];
    rays[i].y[1] = y[2 * i + 1];
    for (int c = 0; c < 4; ++c) rays[i].A.a[c] = A[4 * i + c];
    rays[i].dt = 0;
  }
}

// Lens::rayshooterInternal(RAY&) (internal_rayshooter_multi.cpp:237-251).
void Lens::rayshooterInternal(RAY &ray) { rayshooterInternal(1, &ray); }

// Lens::rayshooter(RAY&) (internal_rayshooter_multi.cpp:42-51): the ray's
// position through the Point overload, the result copied back as the
// reference does (RAY from a LinkedPoint).
void Lens::rayshooter(RAY &ray) {
  LinkedPoint point;
  point.x[0] = ray.x[0];
  point.x[1] = ray.x[1];
  rayshooterInternal(1, &point);
  ray = point;
}
