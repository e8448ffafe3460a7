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
  GLB_ERR_NO_DEVICE = -7,
  GLB_ERR_TIMEOUT = -8       /* glb_server_wait ran out of time */
};

/* Per-ray status of glb_lens_rayshoot_status / glb_lens_rayshoot_device_status. */
enum {
  GLB_RAY_OK = 0,        /* y and A written, all finite */
  GLB_RAY_SKIPPED = 1,   /* skip flag set (the reference's in_image == MAYBE points,
                            include/lens.h:959): y and A left as they were */
  GLB_RAY_NONFINITE = 2  /* y or A written but not finite (the reference asserts,
                            include/lens.h:1012-1037) */
};

/* Precision of the tree walk. */
enum {
  GLB_PREC_FP64 = 0,  /* plain FP64 walk, the reference's arithmetic */
  GLB_PREC_SPLIT = 1, /* FP32 walk with compensated sums, FP64 offsets and recursion; in
                         ray shooting, rays are walked in blocks of 128 spatially sorted
                         rays that share the classification of the tree's cells, so a
                         ray's result can change at the rounding level (~1e-9; the order
                         of its terms) with the other rays of its block, never its set of
                         interactions; tree-force calls and the FP64 form are per-ray
                         exact */
  GLB_PREC_FP32 = 2   /* plain FP32 tree walk (tree-force calls only; the precision sweep) */
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

/* force2D_recur for n rays already on the device (2n doubles, physical Mpc),
 * in any precision form; out_dev gets 5 doubles per ray {alpha0, alpha1,
 * kappa, gamma0, gamma1} (no potential).  Enqueued on `stream` (NULL: the
 * tree's own stream).  Rays are walked 32 to a warp in the given order (64,
 * two per thread, in the split form from 2^20 rays on with opening angles
 * under 0.2), so spatially sorted rays walk fastest. */
int glb_tree_force_device(glb_tree *t, size_t n, const double *rays_dev, double *out_dev, int precision,
                          void *stream);

/* No counterpart in the reference: FP64 direct summation over all n particles
 * (device records) at nrays device rays -- the point mass plus the B-spline
 * correction within two sizes and the inv_area sheet, as at a tree leaf --
 * for reports of a tree form's absolute error.  out_dev: 5 doubles per ray as
 * glb_tree_force_device. */
int glb_direct_sum_device(const glb_particle *particles_dev, size_t n, double inv_area, const double *rays_dev,
                          size_t nrays, double *out_dev, void *stream);

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
/* An NSIE with the member values a constructed LensHaloRealNSIE holds
 * (include/lens_halos.h:1023-1070; constructor MultiPlane/lens_halos.cpp:1043-1078):
 * mass (after the cored halo's mass reset by integration, lens_halos.cpp:1073-1075),
 * Rsize, Rmax, sigma, rcore, fratio and the stored angle pa_internal
 * (= pi/2 - the constructor's pa, lens_halos.cpp:1058).  For mirroring an
 * existing reference halo exactly (the link-level drop-in). */
int glb_halo_nsie_state(float mass, float Rsize, float Rmax, double z, float sigma, float rcore, float fratio,
                        float pa_internal, glb_halo **out);
/* LensHalo::setTheta (include/lens_halos.h:105): angular position, radians. */
int glb_halo_set_theta(glb_halo *h, double tx, double ty);
/* LensHalo::force_halo (include/lens_halos.h:182-190) at n positions xcm
 * relative to the halo centre (physical Mpc).  Outputs as for
 * glb_tree_force2D_recur; analytic halos start from zero. */
int glb_halo_force(glb_halo *h, size_t n, const double *xcm, double *alpha, double *kappa,
                   double *gamma, double *phi);
/* LensHalo::force_halo(alpha, kappa, gamma, phi, xcm, subtract_point, screening)
 * (MultiPlane/lens_halos.cpp:1528-1640): with subtract_point != 0 an NFW or
 * NSIE halo adds, inside Rmax, the point mass scaled by `screening`
 * (force_point) -- and NFW's force_halo_sym adds the unscaled point mass once
 * more (alpha_h + 1, gamma_h + 2, -log(r^2)/2 in phi), as the reference does
 * -- and contributes nothing beyond Rmax.  Particle haloes and field planes
 * take no such argument (LensHaloParticles::force_halo ignores it). */
int glb_halo_force_ex(glb_halo *h, size_t n, const double *xcm, double *alpha, double *kappa, double *gamma,
                      double *phi, int subtract_point, double screening);
/* LensPlaneTree(z, halos, n, sigma_background, inv_screening_scale)
 * (MultiPlane/planes.cpp:13-18): a plane of field haloes whose force is
 * TreeQuadHalos::force2D (include/quadTreeHalos.h:556-815) -- every halo of a
 * visited branch evaluated in full, distant cells as monopole + quadrupole,
 * the sigma_background sheet -- with the reference's tree (bucket 5, opening
 * angle 0.5; with screening: opening angle 0.1, periodic buffer).  The members
 * must be NFW or NSIE haloes (GLB_ERR_UNSUPPORTED otherwise); the plane takes
 * ownership of them (on failure the caller keeps them) and moves them to
 * redshift z (LensHalo::setZlensDist, as Lens::createFieldPlanes does,
 * MultiPlane/lens.cpp:418-426).  glb_halo_force on the result gives
 * LensPlaneTree::force at plane positions (outputs overwritten, alpha as the
 * tree gives it).  Positions spanning no area: GLB_ERR_SAME_PLACE. */
int glb_halo_field_plane(glb_halo *const *halos, int n, double z, double sigma_background,
                         double inv_screening_scale, glb_halo **out);
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
/* A field plane (glb_halo_field_plane) among the lens planes, as
 * Lens::createFieldPlanes adds each LensPlaneTree (MultiPlane/lens.cpp:443-452)
 * and Lens::combinePlanes sorts field and main planes together by distance
 * (lens.cpp:2397-2515).  The lens takes ownership of the plane; its tree is
 * rebuilt for the lens's cosmology. */
int glb_lens_insert_field_plane(glb_lens *l, glb_halo *plane);
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
 * the calling thread's stream on this lens); returns once enqueued.
 * Threads: any number of host threads may shoot rays through one lens at the
 * same time (the reference reads the lens read-only during
 * rayshooterInternal); each calling thread gets its own stream and work
 * buffers on the lens, created on its first call and freed with the lens.
 * Successive device-buffer calls of one thread are ordered on the GPU even
 * when they name different streams (they share that thread's buffers).
 * A call of 2^21 rays or more runs its second half of the sorted rays on a
 * second stream of the thread's workspace, forked from and joined back to
 * `stream` through events, so work enqueued on `stream` after the call still
 * sees its results.
 * Adding halos or resetting the source plane while another thread shoots rays
 * through the same lens is not supported (as in the reference). */
int glb_lens_rayshoot_device(glb_lens *l, size_t n, const double *x_dev, const double *zs_dev,
                             double *y_dev, double *A_dev, int precision, void *stream);
/* glb_lens_rayshoot with per-ray flags (Lens::rayshooterInternal(Npoints,
 * Point*), FullRange/internal_rayshooter_multi.cpp:53-118, whose points with
 * in_image == MAYBE are skipped, include/lens.h:959): skip (n bytes, NULL for
 * none) != 0 leaves that ray's y and A untouched; status (n bytes, out) gets
 * GLB_RAY_OK / GLB_RAY_SKIPPED / GLB_RAY_NONFINITE per ray.  The tree walk is
 * stackless (preorder node array with skip links), so there is no stack
 * overflow state. */
int glb_lens_rayshoot_status(glb_lens *l, size_t n, const double *x, const double *zs,
                             const unsigned char *skip, double *y, double *A, unsigned char *status,
                             int precision);
/* The same on device buffers (skip_dev may be NULL), enqueued on `stream`. */
int glb_lens_rayshoot_device_status(glb_lens *l, size_t n, const double *x_dev, const double *zs_dev,
                                    const unsigned char *skip_dev, double *y_dev, double *A_dev,
                                    unsigned char *status_dev, int precision, void *stream);

/* GridMap(LensHndl, N1d, center, range) (TreeCode_link/gridmap.cpp:93-120):
 * the N1d x N1d grid (x fastest, spacing range/(N1d-1)) is generated on the
 * GPU and shot; y (2 N1d^2) and A (4 N1d^2) are written to host memory. */
int glb_gridmap(glb_lens *l, size_t n1d, const double *center, double range, double *y, double *A,
                int precision);

/* GridMap(lens, N1d, center, range).writePixelMap(lensvar)
 * (include/gridmap.h:529-598): the grid shot on the GPU and reduced there to
 * one map value per grid point (N1d^2 doubles, GridMap order, x fastest), so
 * no per-ray y / A arrays reach the host.  lensvar is the reference's
 * LensingVariable (include/standard.h:89-102): 0 DELAYT (0 on this path),
 * 1 ALPHA, 2 ALPHA1, 3 ALPHA2, 4 KAPPA, 5 GAMMA, 6 GAMMA1, 7 GAMMA2, 8 GAMMA3,
 * 9 INVMAG; 10 PHI and 11 SurfBrightness return GLB_ERR_UNSUPPORTED (the
 * reference throws std::runtime_error for PHI; surface brightness needs the
 * sources, which are outside this library). */
int glb_gridmap_pixelmap(glb_lens *l, size_t n1d, const double *center, double range, int lensvar, double *map,
                         int precision);

/* GridMap(lens, N1d, center, range).writePixelMapUniform<double>(map_center,
 * nx, ny, lensvar) (include/gridmap.h:98-102,506-690): a PixelMap of nx x ny
 * pixels of side range / (nx - 1) centred on map_center (cleared to 0); each
 * grid point writes its LensingVariable value into the pixel that
 * PixelMap::find_index gives for its image position
 * (ImageProcessing/pixelmap.cpp: ix = (long)((x - lower corner) / resolution),
 * points outside dropped).  Where several grid points fall in one pixel the
 * reference keeps the last written (from its threads' chunks; one thread: the
 * largest grid index); here the largest grid index.  map: nx * ny doubles,
 * index ix + nx * iy.  lensvar as glb_gridmap_pixelmap; nx >= 2. */
int glb_gridmap_pixelmap_uniform(glb_lens *l, size_t n1d, const double *center, double range,
                                 const double *map_center, size_t nx, size_t ny, int lensvar, double *map,
                                 int precision);

/* GridMap(lens, N1d, center, range).RefreshSurfaceBrightnesses(&source)
 * (TreeCode_link/gridmap.cpp:174-187): the grid shot on the GPU and the
 * source's surface brightness evaluated there at every ray's source-plane
 * position; sb gets N1d^2 values (GridMap order) and *total (optional) the
 * reference's flux sum, sum of sb x resolution^2 in point order
 * (resolution = range / (N1d - 1), N1d >= 2).  source_kind and
 * source_params = {x, y (source position, radians), ...}:
 *   0 SourceUniform(position, z, radius) (AnalyticNSIE/source.cpp:207-209):
 *     {x, y, radius (radians)};
 *   1 SourceGaussian(position, r_size, z, SBlimit, zero_point)
 *     (source.cpp:211-213): {x, y, r_size (radians)};
 *   2 SourceSersic(mag, Reff, PA, index, q, z, band) (Source/sersic.cpp:116-135):
 *     {x, y, total flux (SourceColored::mag_to_flux of the magnitude),
 *      Reff (arcsec), PA (radians), index, q, sb_limit}.
 * Other kinds: GLB_ERR_UNSUPPORTED. */
int glb_gridmap_surface_brightness(glb_lens *l, size_t n1d, const double *center, double range, int source_kind,
                                   const double *source_params, double *sb, double *total, int precision);

/* GridMap::AdaptiveRefreshSurfaceBrightnesses(lens, source)
 * (TreeCode_link/gridmap.cpp:189-258), the reference's grid-refinement client
 * that shoots one ray per rayshooterInternal call: pixels whose surface
 * brightness differs from a neighbour's by more than 1e-4 of the total are
 * resampled on n x n sub-grids (n = 3, 9, 27, ...) until the mean changes by
 * less than 1e-3.  Here every pixel that refines is resampled level by level
 * in batched GPU calls; the pass over the pixels that decides, in the
 * reference's order, which refine and updates the running total stays on the
 * host.  As in the reference the sub-grids are laid around each pixel's
 * source-plane position and pixels of the first row and column never refine.
 * At most 6 levels (n = 729) per pixel.  sb: N1d^2 refined values; *total:
 * the returned flux.  Sources as glb_gridmap_surface_brightness. */
int glb_gridmap_adaptive_surface_brightness(glb_lens *l, size_t n1d, const double *center, double range,
                                            int source_kind, const double *source_params, double *sb,
                                            double *total, int precision);

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
 * before any stream capture.  All calls share the one array, which keeps the
 * last call's contents; so that no two calls use it at once, every call on a
 * device waits on the GPU for the previous call on that device (one event per
 * device, recorded after each call's last launch; the enqueue is serialised on
 * the host), whatever stream or lens it names.  Calls on one device therefore
 * run one after another on the GPU in the order the host made them.
 * Buffers are device pointers; the call returns once the work is enqueued on
 * `stream` (NULL: the lens's own stream, one per lens). */
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

/* --------------------------------------------------- batched lenses */

/* No counterpart in the reference (which shoots one GridMap at a time under a
 * global mutex, TreeCode_link/gridmap.cpp:15,116-119): the GridMaps of many
 * lenses (nlens lenses, grid sides n1d[i], centres centers[2i..2i+1], ranges
 * ranges[i]) shot by one persistent kernel launch.  Each warp takes 32-ray
 * grid tiles (8 x 4 by default) from a shared counter and carries them through
 * all planes of their lens.  The lenses stay owned by the caller and must
 * outlive the batch. */
typedef struct glb_batch glb_batch;
int glb_batch_create_grids(glb_lens *const *lenses, int nlens, const size_t *n1d, const double *centers,
                           const double *ranges, int precision, glb_batch **out);
/* Runs the batch; use_graph != 0 records the launch into a CUDA graph on the
 * first call and replays it afterwards.  Returns when the results are ready. */
int glb_batch_run(glb_batch *b, int use_graph);
/* Autotuner: times block sizes 64, 128 and 256 (persistent grid each) at the
 * current tile, then warp tiles of 8 x 4, 16 x 2 and 32 x 1 rays at the best
 * block size, and keeps the fastest pair (the walk is stackless: no stack
 * depth to tune). */
int glb_batch_autotune(glb_batch *b, int *best_block, double *best_ms);
int glb_batch_set_block(glb_batch *b, int block);
/* The warp tile's width in rays (8, 16 or 32; height 32 / width). */
int glb_batch_tile(glb_batch *b, int *tile_width);
int glb_batch_set_tile(glb_batch *b, int tile_width);
int glb_batch_info(glb_batch *b, size_t *total_rays, double *last_ms, int *block);
/* y (2 n1d^2) and A (4 n1d^2) of lens i, GridMap order, host memory. */
int glb_batch_result(glb_batch *b, int i, double *y, double *A);
int glb_batch_destroy(glb_batch *b);

/* --------------------------------------------------- served requests */

/* No counterpart in the reference (its small-batch callers -- grid refinement
 * in image and critical-curve finding -- call rayshooterInternal one at a
 * time under a global mutex).  A resident request loop over `nmodels` lenses
 * kept on the device: requests (model, rays, source redshift) are queued by
 * glb_server_submit and admitted in arrival order into batches of at most
 * max_rays_per_batch rays; a batch launches as soon as one of `nslots` slots
 * is free, so requests that arrive while others run are batched and overlap
 * on the GPU.  Admission is by device memory: at every dispatch the server
 * reads the HBM free at that moment (plus memory its own stream-ordered pool
 * holds unused), keeps 5 % of the device free, and admits the requests whose
 * batch memory (about 250 bytes per ray) fits; a batch takes its memory from
 * the pool when it launches and gives it back when its results are copied
 * out, so a request that does not fit waits until batches in flight finish
 * (GLB_ERR_OOM from glb_server_wait if none is in flight).  The pool keeps
 * what it has reserved until the server is destroyed.  Requests of fewer than
 * 2^20 rays run in 32-ray chunks of the batched kernel; larger ones through
 * the per-plane kernels of glb_lens_rayshoot on the batch's stream, so their
 * results are those of glb_lens_rayshoot for the same rays and source
 * redshift.  A request's results do not depend on what it is batched with.
 * The lenses must outlive the server. */
typedef struct glb_server glb_server;
int glb_server_create(glb_lens *const *models, int nmodels, size_t max_rays_per_batch, int precision, int nslots,
                      glb_server **out);
/* Queues n rays x (2n, radians, host) for lens `model` with source redshift
 * zs (zs < 0: the lens's own source plane).  x, y (2n) and A (4n) must stay
 * valid until glb_server_wait returns for the ticket. */
int glb_server_submit(glb_server *s, int model, size_t n, const double *x, double zs, double *y, double *A,
                      long long *ticket);
/* Waits for a ticket (timeout_s <= 0: no limit); times (optional, 3 doubles)
 * gets the submit, start and completion times in seconds of a steady clock. */
int glb_server_wait(glb_server *s, long long ticket, double timeout_s, double *times);
int glb_server_poll(glb_server *s, long long ticket, int *done);
/* stats[0..5]: rays done, requests done, batches, busy seconds (first launch
 * to last completion), rays per batch budget, requests pending. */
int glb_server_stats(glb_server *s, double *stats);
/* Admission record: dispatches that waited for batches in flight to give
 * device memory back, and the least admissible HBM (GB) seen at a dispatch. */
int glb_server_admission(glb_server *s, double *memory_waits, double *min_free_gb);
/* Stops the loop; batches already on the GPU finish, queued requests are
 * dropped. */
int glb_server_destroy(glb_server *s);

/* Timing of the last rayshoot on this lens: device milliseconds of the
 * per-plane kernels and of the whole call (CUDA events). */
int glb_lens_last_timing(glb_lens *l, double *kernel_ms, double *total_ms);

/* ---------------------------------------------- adaptive kNN smoothing */
/* Replaces LensHaloParticles<ParticleType<float>>::calculate_smoothing(Nsmooth,
 * pp, Npoints) (include/particle_halo.h:159-162, def :683-730): sets every
 * particle's Size to the distance to its (nsmooth+1)-th nearest particle, the
 * particle itself counted -- the value TreeSimple::NNDistance(x, Nsmooth+1)
 * returns (include/simpleTree.h:483-618): squared distances summed in double
 * from float coordinate differences, square root rounded to float.  For
 * N = 2*nsmooth+1 the reference's walk counts some particles twice for the
 * queries in its top node's first child; those values are reproduced too.
 * Errors: nsmooth < 1 or n <= nsmooth+1 (the reference exits) GLB_ERR_ARG;
 * nsmooth above about 800 GLB_ERR_UNSUPPORTED.  Synchronous; particles are
 * host records, only their Size is written. */
int glb_particles_smoothing(glb_particle *particles, size_t n, int nsmooth);
/* The same on device buffers: n records at particles_dev, n floats written to
 * size_dev, on `stream` (NULL: the legacy default stream).  Returns when the
 * sizes are written.  ms_out (nullable, 2 floats): device milliseconds of the
 * Morton sort and bucket boxes, and of the neighbour search. */
int glb_particles_smoothing_device(const glb_particle *particles_dev, size_t n, int nsmooth, float *size_dev,
                                   void *stream, float *ms_out);

#ifdef __cplusplus
}
#endif
#endif
