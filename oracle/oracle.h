/*
 * ORACLE -- test infrastructure only.
 *
 * A plain-C CPU restatement of GLAMER/SLsimLib's ray-shooting path, used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the
 * checker for the CUDA library.  Nothing in the product links or calls this.
 * Each routine cites the reference file:line it restates (paths relative to
 * the SLsimLib source root).  Parity of this restatement is pinned against the
 * reference itself, compiled in place into oracle/_ref (see oracle/Makefile).
 *
 * Units follow the reference: positions on a plane in physical Mpc, masses in
 * Msun, alpha in Msun/Mpc, kappa/gamma in Msun/Mpc^2, ray angles in radians.
 */
#ifndef GLAMER_ORACLE_H
#define GLAMER_ORACLE_H
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ParticleType<float> (include/particle_types.h:46-58): 24-byte record. */
typedef struct {
  float x[3];
  float Mass;
  float Size;
  int type;
} orc_particle;

/* ---------------- flat LambdaCDM distances (CosmoLib stand-in) ---------- */
void orc_set_cosmology(double omega_m, double omega_l, double h);
double orc_coordist(double z);                  /* comoving, Mpc */
double orc_coordist2(double z1, double z2);     /* coorDist(z2)-coorDist(z1) */
double orc_angdist(double z);                   /* coorDist(z)/(1+z) */
double orc_invcoordist(double d);               /* inverse of orc_coordist */

/* ---------------- TreeQuadParticles (include/quadTree.h) --------------- */
typedef struct orc_tree orc_tree;

/* TreeQuadParticles ctor, include/quadTree.h:247-285.  Returns NULL and sets
 * *err (1 = particles in same place, quadTree.h:327-329) on failure. */
orc_tree *orc_tree_build(const orc_particle *p, size_t n, float mass_fixed,
                         float size_fixed, double inv_area, int bucket,
                         double theta, int periodic, double inv_screening,
                         double max_range, int *err);
void orc_tree_free(orc_tree *t);
/* TreeQuadParticles::force2D_recur, include/quadTree.h:932-987. */
void orc_tree_force2D_recur(orc_tree *t, const double *ray, double *alpha,
                            double *kappa, double *gamma, double *phi);
/* Direct (no tree) FP64 sum with the same point-mass + B-spline kernel and
 * inv_area sheet: the absolute-accuracy oracle. */
void orc_direct_sum(const orc_particle *p, size_t n, double inv_area,
                    const double *ray, double *alpha, double *kappa,
                    double *gamma, double *phi);
/* Number of branches (including empty children). */
size_t orc_tree_nbranches(const orc_tree *t);
/* Preorder export of every branch: per branch 16 doubles
 * {level, p1x, p1y, p2x, p2y, nparticles, nbig, mass, comx, comy, quad0,
 *  quad1, quad2, r2crit, is_leaf, boxsize2}. */
void orc_tree_export(const orc_tree *t, double *out);
/* Per-branch sorted membership check: for branch k (preorder) writes the
 * sum over its particles of (index+1) and of (index+1)^2 (exact in double
 * for the sizes tested), to compare memberships without storing them. */
void orc_tree_membership(const orc_tree *t, double *out);

/* ---------------- halos (include/lens_halos.h, MultiPlane/lens_halos.cpp) */
typedef struct orc_halo orc_halo;
/* LensHaloNFW(float mass, float Rsize, z, float conc, float fratio, float pa)
 * MultiPlane/lens_halos.cpp:389-431; fratio must be 1 (spherical). */
orc_halo *orc_halo_nfw(float mass, float Rsize, double z, float conc,
                       float fratio, float pa);
/* LensHaloRealNSIE(float mass, z, float sigma, float rcore, float fratio,
 * float pa), MultiPlane/lens_halos.cpp:1043-1078. */
orc_halo *orc_halo_nsie(float mass, double z, float sigma, float rcore,
                        float fratio, float pa);
/* LensHaloParticles vector ctor (include/particle_halo.h:58-75,342-417):
 * bucket 20, theta 0.1, no rotation, no recentering. */
orc_halo *orc_halo_particles(const orc_particle *p, size_t n, double z,
                             double inv_area, double max_range);
void orc_halo_set_theta(orc_halo *h, double tx, double ty);
void orc_halo_free(orc_halo *h);
float orc_halo_mass(const orc_halo *h);
float orc_halo_rsize(const orc_halo *h);
float orc_halo_rmax(const orc_halo *h);
/* LensHalo::force_halo / LensHaloRealNSIE::force_halo /
 * LensHaloParticles::force_halo for n positions xcm (2n, physical Mpc).
 * Outputs alpha 2n, kappa n, gamma 3n, phi n (accumulated from zero). */
void orc_halo_force(orc_halo *h, size_t n, const double *xcm, double *alpha,
                    double *kappa, double *gamma, double *phi);

/* LensPlaneTree(z, halos, n, sigma_background, inv_screening_scale)
 * (MultiPlane/planes.cpp:13-18) over NFW / NSIE haloes: a TreeQuadHalos
 * (include/quadTreeHalos.h) as a halo of its own whose force is
 * TreeQuadHalos::force2D (overwrites its outputs).  Takes ownership of the
 * haloes and moves them to redshift z.  Returns NULL with *err = 1 when the
 * haloes' positions span no area ("particles in same place."; the caller
 * keeps its haloes then). */
orc_halo *orc_halo_field_plane(orc_halo **halos, int n, double z,
                               double sigma_back, double inv_screening,
                               int *err);

/* Source::SurfaceBrightness at n source-plane positions y (2n, radians).
 * p = {x, y, ...}: kind 0 SourceUniform {radius}; 1 SourceGaussian {r_size};
 * 2 SourceSersic {flux, Reff (arcsec), PA, index, q, sb_limit}. */
void orc_source_sb(int kind, const double *p, size_t n, const double *y,
                   double *out);

/* ---------------- Lens (MultiPlane/lens.cpp, include/lens.h) ---------- */
typedef struct orc_lens orc_lens;
orc_lens *orc_lens_create(double zsource);
void orc_lens_free(orc_lens *l);
/* Lens::insertMainHalo / moveinMainHalo with addplanes (lens.h:149-185):
 * the lens takes ownership of h. */
void orc_lens_add_halo(orc_lens *l, orc_halo *h, int addplanes);
/* A field plane (orc_halo_field_plane) among the lens planes, as
 * Lens::createFieldPlanes adds a LensPlaneTree; the lens takes ownership. */
void orc_lens_add_field_plane(orc_lens *l, orc_halo *plane);
int orc_lens_nplanes(const orc_lens *l);
/* plane_redshifts, Dl, dDl (each nplanes+1 long, source pseudo-plane last) */
void orc_lens_planes(const orc_lens *l, double *z, double *Dl, double *dDl);
/* Lens::ResetSourcePlane (lens.cpp:2609-2657); returns j. */
int orc_lens_reset_source(orc_lens *l, double z, int nearest);
/* Lens::rayshooterInternal(N, Point*) (FullRange/internal_rayshooter_multi.cpp
 * :53-118 + include/lens.h:913-1103) over SoA buffers: x 2n in, y 2n and
 * A 4n out.  zs == NULL: the lens source plane; otherwise per-ray source
 * redshifts (the LinkedPoint / RAY overloads). threads <= 0: all cores. */
void orc_lens_rayshoot(orc_lens *l, size_t n, const double *x, const double *zs,
                       double *y, double *A, int threads);
/* One plane's LensPlaneSingular::force (MultiPlane/planes.cpp:114-161). */
void orc_lens_plane_force(orc_lens *l, int j, size_t n, const double *xx,
                          double *alpha, double *kappa, double *gamma,
                          double *phi);

/* GridMap::AdaptiveRefreshSurfaceBrightnesses (gridmap.cpp:189-258): sb
 * (N1d^2) the refined per-pixel surface brightness; returns the total flux.
 * Refinement levels are capped at 6 (n = 729). */
double orc_gridmap_adaptive_sb(orc_lens *l, size_t N1d, const double *center,
                               double range, int kind, const double *p,
                               double *sb);
/* One pixel's refinement (sub-grid around its source position ysrc). */
double orc_refine_pixel(orc_lens *l, const double *ysrc, double resolution,
                        double sb0, int kind, const double *p);

/* ---------------- GridMap (TreeCode_link/gridmap.cpp:93-120) ----------- */
/* xygridpoints + PositionFromIndex (gridmap.cpp:293-321, utilities.cpp:149-158) */
void orc_grid_positions(size_t N1d, const double *center, double range,
                        double *x);

/* ---------- adaptive kNN smoothing (include/particle_halo.h:683-730) --- */
/* Sets p[i].Size to TreeSimple::NNDistance(x_i, nsmooth+1) over a 3-d
 * median-split tree with bucket 2*nsmooth.  Returns 0, or -1 when nsmooth < 1
 * or n <= nsmooth+1. */
int orc_calculate_smoothing(orc_particle *p, size_t n, int nsmooth);

#ifdef __cplusplus
}
#endif
#endif
