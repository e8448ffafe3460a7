/*
 * glamer_b200.h -- C ABI of the B200 ray-shooting library (libglamer_b200.so).
 *
 * Drop-in boundary for GLAMER/SLsimLib's ray-shooting path.  Every entry
 * point is plain C: opaque handles, host pointers and sizes, an int status
 * (0 = success, negative = error; glb_last_error() gives the message).  The
 * comment on each function names the reference interface it replaces
 * (file:line relative to the SLsimLib source root).
 *
 * Units follow the reference: ray angles in radians; positions on a plane in
 * physical Mpc; masses in Msun; alpha in Msun/Mpc, kappa and gamma in
 * Msun/Mpc^2 (multiply by 4 pi G to get the dimensionless plane values).
 * Particle records are ParticleType<float> (include/particle_types.h:46-58).
 */
#ifndef GLAMER_B200_H
#define GLAMER_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ParticleType<float>: float x[3]; float Mass; float Size; int type (24 bytes) */
typedef struct {
  float x[3];
  float Mass;
  float Size;
  int type;
} glb_particle;

typedef struct glb_tree glb_tree;
typedef struct glb_halo glb_halo;
typedef struct glb_lens glb_lens;

enum {
  GLB_OK = 0,
  GLB_ERR_ARG = -1,          /* std::invalid_argument in the reference */
  GLB_ERR_CUDA = -2,         /* CUDA runtime failure (message has the call) */
  GLB_ERR_OOM = -3,
  GLB_ERR_SAME_PLACE = -4,   /* "particles in same place." (quadTree.h:327-329) */
  GLB_ERR_DEPTH = -5,        /* more than 32 tree levels needed */
  GLB_ERR_UNSUPPORTED = -6,  /* a reference feature outside this library's scope */
  GLB_ERR_NO_DEVICE = -7
};

/* Precision of the tree walk. */
enum {
  GLB_PREC_FP64 = 0,  /* plain FP64 walk, the reference's arithmetic */
  GLB_PREC_SPLIT = 1  /* FP32 walk with compensated sums, FP64 offsets and recursion */
};

/* Message of the last failure on this thread ("" if none). */
const char *glb_last_error(void);
/* Library version string. */
const char *glb_version(void);
/* Options: GLB_OPT_KEEP_TREE_EXPORT (1) keeps per-branch build data so that
 * glb_tree_export can be called (test and debugging use). */
enum { GLB_OPT_KEEP_TREE_EXPORT = 1 };
int glb_set_option(int option, long long value);

/* ---------------------------------------------------------------- trees */

/* TreeQuadParticles<ParticleType<float>>::TreeQuadParticles
 * (include/quadTree.h:49-60, 247-285): builds the quadtree on the GPU from n
 * host particle records.  mass_fixed / size_fixed <= 0 mean per-particle
 * masses / sizes, as in the reference. */
int glb_tree_create(const glb_particle *particles, size_t n, float mass_fixed, float size_fixed,
                    double inv_area, int bucket, double theta_force, int periodic_buffer,
                    double inv_screening_scale, double maximum_range, glb_tree **out);
int glb_tree_destroy(glb_tree *t);

/* TreeQuadParticles::force2D_recur (include/quadTree.h:932-987) for n rays
 * (2n doubles, physical Mpc, host memory).  Outputs (host): alpha 2n,
 * kappa n, gamma 3n, phi n; gamma[2] is always 0 as in the reference. */
int glb_tree_force2D_recur(glb_tree *t, size_t n, const double *rays, double *alpha, double *kappa,
                           double *gamma, double *phi);

/* Per-branch build data in depth-first order, 16 doubles per branch
 * (level, p1x, p1y, p2x, p2y, nparticles, Nbig_particles, mass, com_x, com_y,
 *  quad[0..2], r2crit_angle, is_leaf, boxsize^2).  Call with out == NULL to
 * get *nbranches.  Needs GLB_OPT_KEEP_TREE_EXPORT at build time. */
int glb_tree_export(glb_tree *t, size_t *nbranches, double *out);
/* Device build time of the tree in milliseconds. */
int glb_tree_build_ms(glb_tree *t, double *ms);

/* ---------------------------------------------------------------- halos */

/* LensHaloParticles(std::vector<ParticleType<float>>&, float redshift, cosmo,
 * Point_2d(0,0), recenter=false, inv_area, MinPSize=0, max_range)
 * (include/particle_halo.h:58-75, 342-417).  As in the reference, max_range
 * reaches the tree as its inv_screening_scale (particle_halo.h:416). */
int glb_halo_particles(const glb_particle *particles, size_t n, double z, double inv_area,
                       double max_range, glb_halo **out);
/* LensHaloNFW(float mass, float Rsize, z, float concentration, float fratio,
 * float pa, cosmo) (MultiPlane/lens_halos.cpp:389-431).  fratio must be 1. */
int glb_halo_nfw(float mass, float Rsize, double z, float concentration, float fratio, float pa,
                 glb_halo **out);
/* LensHaloRealNSIE(float mass, z, float sigma, float rcore, float fratio,
 * float pa, cosmo) (MultiPlane/lens_halos.cpp:1043-1078). */
int glb_halo_nsie(float mass, double z, float sigma, float rcore, float fratio, float pa,
                  glb_halo **out);
/* LensHalo::setTheta (include/lens_halos.h:105): angular position, radians. */
int glb_halo_set_theta(glb_halo *h, double tx, double ty);
/* LensHalo::force_halo (include/lens_halos.h:182-190) at n positions xcm
 * relative to the halo centre (physical Mpc).  Outputs as for
 * glb_tree_force2D_recur; analytic halos start from zero. */
int glb_halo_force(glb_halo *h, size_t n, const double *xcm, double *alpha, double *kappa,
                   double *gamma, double *phi);
/* mass, Rsize, Rmax (float members of LensHalo) */
int glb_halo_params(glb_halo *h, float *mass, float *rsize, float *rmax);
int glb_halo_destroy(glb_halo *h);

/* ----------------------------------------------------------------- lens */

/* Lens(long *seed, z_source, const COSMOLOGY&) (MultiPlane/lens.cpp:59-77)
 * with a flat LambdaCDM cosmology (omega_m + omega_l must be 1). */
int glb_lens_create(double zsource, double omega_m, double omega_l, double hubble, glb_lens **out);
int glb_lens_destroy(glb_lens *l);
/* Lens::moveinMainHalo / insertMainHalo (include/lens.h:149-185): the lens
 * takes ownership of h.  addplanes selects addMainHaloToPlane (1) or
 * addMainHaloToNearestPlane (0). */
int glb_lens_insert_halo(glb_lens *l, glb_halo *h, int addplanes);
/* Lens::getNplanes and the plane_redshifts / Dl / dDl arrays (nplanes + 1
 * entries each, source pseudo-plane last; any pointer may be NULL). */
int glb_lens_nplanes(glb_lens *l, int *nplanes);
int glb_lens_planes(glb_lens *l, double *z, double *Dl, double *dDl);
/* Lens::ResetSourcePlane (MultiPlane/lens.cpp:2609-2657). */
int glb_lens_reset_source(glb_lens *l, double z, int nearest, int *plane_index);

/* Lens::rayshooterInternal (FullRange/internal_rayshooter_multi.cpp:53-235):
 * x (2n, radians) -> y (2n, source-plane angle) and A (4n, Jacobian
 * a[0..3] = A11, A12, A21, A22; kappa = 1-(a0+a3)/2 etc., include/point.h).
 * zs == NULL: the lens's source plane (the Point* overload); otherwise one
 * source redshift per ray (the LinkedPoint + source_zs and RAY* overloads).
 * Host buffers; the call returns when the results are in y and A. */
int glb_lens_rayshoot(glb_lens *l, size_t n, const double *x, const double *zs, double *y,
                      double *A, int precision);
/* The same on device buffers, enqueued on `stream` (a cudaStream_t, NULL for
 * the lens's own stream); returns once enqueued. */
int glb_lens_rayshoot_device(glb_lens *l, size_t n, const double *x_dev, const double *zs_dev,
                             double *y_dev, double *A_dev, int precision, void *stream);

/* GridMap(LensHndl, N1d, center, range) (TreeCode_link/gridmap.cpp:93-120):
 * the N1d x N1d grid (x fastest, spacing range/(N1d-1)) is generated on the
 * GPU and shot; y (2 N1d^2) and A (4 N1d^2) are written to host memory. */
int glb_gridmap(glb_lens *l, size_t n1d, const double *center, double range, double *y, double *A,
                int precision);

/* No counterpart in the reference.  glb_lens_rayshoot_device for callers that
 * cannot allocate device memory while they shoot rays: cudaMalloc / cudaFree
 * synchronise the whole device and can fail under a memory cap, which grid
 * refinement loops shooting a few thousand rays at a time, applications that
 * reserve all their memory up front, or processes sharing a GPU under a quota
 * cannot accept.  This entry point allocates nothing: its scratch is one
 * fixed device array of about 13.5 MB inside the library, held by every GPU
 * that loads the library until the process exits.  Limits: n <= 65536 rays
 * per call, at most 64 lens planes and 256 halos (larger calls return
 * GLB_ERR_ARG).  The first call on a device does a one-time set-up (looks up
 * the array's device address and copies the NFW tables) and should come
 * before any stream capture.  All calls share the one array, so calls that
 * overlap on the GPU (different streams or threads) race; serialise them.
 * Buffers are device pointers; the call returns once the work is enqueued on
 * `stream` (NULL: the lens's own stream). */
int glb_lens_rayshoot_noalloc(glb_lens *l, size_t n, const double *x_dev, const double *zs_dev,
                              double *y_dev, double *A_dev, int precision, void *stream);

/* Measurement aid with no counterpart in the reference: shoots n rays (host
 * buffers) in FP64 and returns the interaction counts summed over rays and
 * planes: counts[0..4] = nodes tested, far-field cells, leaf point masses,
 * big-particle distance checks, B-spline corrections (the event counts of the
 * algorithmic-flop roofline); counts[5..6] = node-loop and leaf-particle-loop
 * iterations summed over lanes (32 per warp iteration), whose ratio to
 * counts[0] and counts[2] is the lane efficiency of the warp-cooperative walk. */
int glb_lens_count_interactions(glb_lens *l, size_t n, const double *x, const double *zs,
                                unsigned long long *counts);

/* Timing of the last rayshoot on this lens: device milliseconds of the
 * per-plane kernels and of the whole call (CUDA events). */
int glb_lens_last_timing(glb_lens *l, double *kernel_ms, double *total_ms);

#ifdef __cplusplus
}
#endif
#endif
