/*
 * ORACLE -- test infrastructure only (see oracle.h).  Plain C99 restatement
 * of the reference's ray-shooting path; used only as the checker of the CUDA
 * library.  Reference citations are relative to the SLsimLib source root.
 */
#define _GNU_SOURCE
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define ORC_PI M_PI                 /* include/standard.h:39 (PI = M_PI) */
#define ORC_GRAV 4.7788e-20         /* include/standard.h:43, G/c^2 in Mpc/Msun */
#define ORC_LIGHTSPEED 2.99792458e5 /* km/s */
#define ORC_MIN_PLANE_DIST 1e-6     /* MultiPlane/lens.cpp:15 */

/* ======================= cosmology stand-in ============================ */
static double g_om = 0.3, g_ol = 0.7, g_h = 0.7;

void orc_set_cosmology(double om, double ol, double h) {
  g_om = om;
  g_ol = ol;
  g_h = h;
}

static double inv_E(double z) {
  double a = 1.0 + z;
  return 1.0 / sqrt(g_om * a * a * a + g_ol + (1.0 - g_om - g_ol) * a * a);
}

static double simpson_rec(double a, double b, double fa, double fm, double fb,
                          double whole, double tol, int depth) {
  double m = 0.5 * (a + b), lm = 0.5 * (a + m), rm = 0.5 * (m + b);
  double flm = inv_E(lm), frm = inv_E(rm);
  double left = (m - a) / 6.0 * (fa + 4.0 * flm + fm);
  double right = (b - m) / 6.0 * (fm + 4.0 * frm + fb);
  double delta = left + right - whole;
  if (depth <= 0 || fabs(delta) <= 15.0 * tol) return left + right + delta / 15.0;
  return simpson_rec(a, m, fa, flm, fm, left, 0.5 * tol, depth - 1) +
         simpson_rec(m, b, fm, frm, fb, right, 0.5 * tol, depth - 1);
}

/* Comoving distance (Mpc) for flat LambdaCDM: (c/H0) int_0^z dz/E(z),
 * adaptive Simpson to ~1e-15 absolute in the dimensionless integral. */
double orc_coordist(double z) {
  if (z == 0.0) return 0.0;
  double fa = inv_E(0.0), fb = inv_E(z), fm = inv_E(0.5 * z);
  double whole = z / 6.0 * (fa + 4.0 * fm + fb);
  double integral = simpson_rec(0.0, z, fa, fm, fb, whole, 1e-15, 50);
  return ORC_LIGHTSPEED / (100.0 * g_h) * integral;
}
double orc_coordist2(double z1, double z2) { return orc_coordist(z2) - orc_coordist(z1); }
double orc_angdist(double z) { return orc_coordist(z) / (1.0 + z); }
double orc_invcoordist(double d) {
  double lo = 0.0, hi = 1.0;
  while (orc_coordist(hi) < d) hi *= 2.0;
  for (int i = 0; i < 200 && hi - lo > 1e-15 * hi; ++i) {
    double mid = 0.5 * (lo + hi);
    if (orc_coordist(mid) < d) lo = mid; else hi = mid;
  }
  return 0.5 * (lo + hi);
}

/* ======================= TreeQuadParticles ============================= */
typedef struct orc_branch {
  size_t *particles;
  size_t nparticles;
  size_t *big;
  size_t nbig;
  double center[2];
  double mass;
  int level;
  double p1[2], p2[2];
  struct orc_branch *child[4];
  struct orc_branch *brother;
  double quad[3];
  double rmax;
  double r2crit;
} orc_branch;

struct orc_tree {
  const orc_particle *xxp;
  size_t n;
  int multimass, multiradius;
  double size_fixed; /* the member, which the constructor never assigns */
  double inv_area;
  int bucket;
  double theta;
  int periodic;
  double inv_screen2;
  double max_range;
  size_t *index;
  double *work;
  orc_branch *top;
  orc_branch *current; /* last branch of the moments walk; see walk_recur */
  double original_xl, original_yl;
  size_t nbranches;
  double phiintconst;
};

static orc_branch *new_branch(void) {
  orc_branch *b = (orc_branch *)calloc(1, sizeof(orc_branch));
  return b;
}

/* Utilities::quickPartition, include/Tree.h:409-424: values <= pivot first. */
static void quick_partition(double pivot, size_t *cut, size_t *particles, double *arr, size_t N) {
  size_t i, k = 0;
  for (i = 0; i < N; ++i) {
    if (arr[i] <= pivot) {
      double t = arr[k]; arr[k] = arr[i]; arr[i] = t;
      size_t s = particles[k]; particles[k] = particles[i]; particles[i] = s;
      ++k;
    }
  }
  *cut = k;
}

static float psize(const orc_tree *t, size_t i) { return t->xxp[i * t->multiradius].Size; }
static float pmass(const orc_tree *t, size_t i) { return t->xxp[i * t->multimass].Mass; }

/* TreeQuadParticles::_BuildQTreeNB, include/quadTree.h:358-565. */
static void build_rec(orc_tree *t, orc_branch *cb, int at_top) {
  size_t i, j, cut = 0, cut2 = 0;
  size_t *particles = cb->particles;
  cb->center[0] = (cb->p1[0] + cb->p2[0]) / 2;
  cb->center[1] = (cb->p1[1] + cb->p2[1]) / 2;
  cb->quad[0] = cb->quad[1] = cb->quad[2] = 0;
  cb->mass = 0.0;

  double theta_range = 2 * t->theta;
  if (t->max_range > 0) {
    double boxsize = 1.732 * (cb->p2[0] - cb->p1[0]);
    double d = sqrt(cb->center[0] * cb->center[0] + cb->center[1] * cb->center[1]) - t->max_range;
    theta_range = boxsize / (d > boxsize ? d : boxsize);
  }

  /* leaf case, quadTree.h:379-401 */
  if (cb->nparticles <= (size_t)t->bucket || t->theta > theta_range) {
    double w = cb->p2[0] - cb->p1[0];
    cb->nbig = 0;
    for (i = 0; i < cb->nparticles; ++i)
      if ((double)psize(t, particles[i]) < w) ++cb->nbig;
    if (cb->nbig) {
      cb->big = (size_t *)malloc(cb->nbig * sizeof(size_t));
      for (i = 0, j = 0; i < cb->nparticles; ++i)
        if ((double)psize(t, particles[i]) < w) cb->big[j++] = particles[i];
    }
    return;
  }

  double *x = t->work;
  cb->nbig = 0;
  if (t->multiradius) { /* quadTree.h:410-431 */
    for (i = 0; i < cb->nparticles; ++i) x[i] = t->xxp[particles[i]].Size;
    double maxsize = (cb->p2[0] - cb->p1[0]) / 2;
    quick_partition(maxsize, &cut, particles, x, cb->nparticles);
    if (cut < cb->nparticles) {
      if (at_top) {
        cb->nbig = cut2 = cb->nparticles - cut;
      } else {
        quick_partition(2 * maxsize, &cut2, &particles[cut], &x[cut], cb->nparticles - cut);
        cb->nbig = cut2;
      }
      if (cb->nbig) {
        cb->big = (size_t *)malloc(cb->nbig * sizeof(size_t));
        for (i = cut; i < cut + cut2; ++i) cb->big[i - cut] = particles[i];
      }
    }
  } else {
    /* quadTree.h:433-443 with the never-assigned size_fixed member (0.0):
     * the condition 0 > w/2 never holds, so no big particles here. */
    double s = t->size_fixed, w = cb->p2[0] - cb->p1[0];
    if (s > w / 2 && s < w) {
      cb->nbig = cb->nparticles;
      cb->big = (size_t *)malloc(cb->nbig * sizeof(size_t));
      for (i = 0; i < cb->nparticles; ++i) cb->big[i] = particles[i];
    }
  }

  size_t np = cb->nparticles; /* all particles go on to the children */
  if (np == 0) return;

  orc_branch *c[4];
  for (int k = 0; k < 4; ++k) {
    c[k] = new_branch();
    c[k]->level = cb->level + 1;
    cb->child[k] = c[k];
  }
  t->nbranches += 4;
  c[0]->brother = c[1];
  c[1]->brother = c[2];
  c[2]->brother = c[3];
  c[3]->brother = cb->brother;
  /* child boxes, quadTree.h:466-484 */
  c[0]->p1[0] = cb->center[0]; c[0]->p1[1] = cb->center[1];
  c[0]->p2[0] = cb->p2[0];     c[0]->p2[1] = cb->p2[1];
  c[1]->p1[0] = cb->p1[0];     c[1]->p1[1] = cb->center[1];
  c[1]->p2[0] = cb->center[0]; c[1]->p2[1] = cb->p2[1];
  c[2]->p1[0] = cb->center[0]; c[2]->p1[1] = cb->p1[1];
  c[2]->p2[0] = cb->p2[0];     c[2]->p2[1] = cb->center[1];
  c[3]->p1[0] = cb->p1[0];     c[3]->p1[1] = cb->p1[1];
  c[3]->p2[0] = cb->center[0]; c[3]->p2[1] = cb->center[1];

  double xcut = cb->center[0], ycut = cb->center[1];
  size_t cutx, cuty;
  for (i = 0; i < np; ++i) x[i] = t->xxp[particles[i]].x[1];
  quick_partition(ycut, &cuty, particles, x, np);
  if (cuty > 0) {
    for (i = 0; i < cuty; ++i) x[i] = t->xxp[particles[i]].x[0];
    quick_partition(xcut, &cutx, particles, x, cuty);
    c[3]->nparticles = cutx;
    c[3]->particles = cutx ? particles : NULL;
    c[2]->nparticles = cuty - cutx;
    c[2]->particles = (cuty - cutx) ? &particles[cutx] : NULL;
  }
  if (cuty < np) {
    for (i = cuty; i < np; ++i) x[i - cuty] = t->xxp[particles[i]].x[0];
    quick_partition(xcut, &cutx, &particles[cuty], x, np - cuty);
    c[1]->nparticles = cutx;
    c[1]->particles = cutx ? &particles[cuty] : NULL;
    c[0]->nparticles = np - cuty - cutx;
    c[0]->particles = (np - cuty - cutx) ? &particles[cuty + cutx] : NULL;
  }
  for (int k = 0; k < 4; ++k) build_rec(t, c[k], 0);
}

static int is_leaf(const orc_branch *b) {
  return !b->child[0] && !b->child[1] && !b->child[2] && !b->child[3];
}

/* TreeQuadParticles::CalcMoments, include/quadTree.h:569-628 (per branch). */
static void moments_one(orc_tree *t, orc_branch *cb) {
  size_t i;
  double rcom, xcm[2], xcut, tmp, absmass;
  cb->rmax = sqrt(pow(cb->p2[0] - cb->p1[0], 2) + pow(cb->p2[1] - cb->p1[1], 2));
  for (i = 0, cb->mass = 0, absmass = 0; i < cb->nparticles; ++i) {
    cb->mass += pmass(t, cb->particles[i]);
    absmass += fabs(pmass(t, cb->particles[i]));
  }
  cb->center[0] = cb->center[1] = 0;
  for (i = 0; i < cb->nparticles; ++i) {
    tmp = fabs(pmass(t, cb->particles[i]));
    cb->center[0] += tmp * t->xxp[cb->particles[i]].x[0] / absmass;
    cb->center[1] += tmp * t->xxp[cb->particles[i]].x[1] / absmass;
  }
  cb->quad[0] = cb->quad[1] = cb->quad[2] = 0;
  for (i = 0; i < cb->nparticles; ++i) {
    xcm[0] = t->xxp[cb->particles[i]].x[0] - cb->center[0];
    xcm[1] = t->xxp[cb->particles[i]].x[1] - cb->center[1];
    xcut = pow(xcm[0], 2) + pow(xcm[1], 2);
    tmp = pmass(t, cb->particles[i]);
    cb->quad[0] += (xcut - 2 * xcm[0] * xcm[0]) * tmp;
    cb->quad[1] += (xcut - 2 * xcm[1] * xcm[1]) * tmp;
    cb->quad[2] += -2 * xcm[0] * xcm[1] * tmp;
  }
  for (i = 0, rcom = 0.0; i < 2; ++i) {
    double a = pow(cb->center[i] - cb->p1[i], 2), b = pow(cb->center[i] - cb->p2[i], 2);
    rcom += (a > b) ? a : b;
  }
  rcom = sqrt(rcom);
  if (t->theta > 0.0) {
    cb->r2crit = 1.15470 * rcom / (t->theta);
    cb->r2crit *= cb->r2crit;
  } else
    cb->r2crit = 1.0e100;
}

/* Preorder walk (QTreeNB::WalkStep, include/qTreeNB.h:479-490). */
static orc_branch *walk_step(orc_branch *b) {
  if (b->child[0]) return b->child[0];
  return b->brother;
}

static void free_rec(orc_branch *b) {
  if (!b) return;
  for (int k = 0; k < 4; ++k) free_rec(b->child[k]);
  free(b->big);
  free(b);
}

orc_tree *orc_tree_build(const orc_particle *p, size_t n, float mass_fixed, float size_fixed,
                         double inv_area, int bucket, double theta, int periodic,
                         double inv_screening, double max_range, int *err) {
  if (err) *err = 0;
  orc_tree *t = (orc_tree *)calloc(1, sizeof(orc_tree));
  t->xxp = p;
  t->n = n;
  t->multimass = mass_fixed <= 0 ? 1 : 0; /* quadTree.h:272-273 */
  t->multiradius = size_fixed <= 0 ? 1 : 0;
  t->size_fixed = 0.0;
  t->inv_area = inv_area;
  t->bucket = bucket;
  t->theta = theta;
  t->periodic = periodic;
  t->inv_screen2 = inv_screening * inv_screening;
  t->max_range = max_range;
  t->phiintconst = (120 * log(2.) - 631.) / 840 + 19. / 70; /* quadTree.h:282 */
  t->index = (size_t *)malloc((n ? n : 1) * sizeof(size_t));
  for (size_t i = 0; i < n; ++i) t->index[i] = i;
  if (n == 0) return t;

  /* BuildQTreeNB, quadTree.h:297-350 */
  double p1[2], p2[2];
  for (int j = 0; j < 2; ++j) p1[j] = p2[j] = p[0].x[j];
  for (size_t i = 0; i < n; ++i)
    for (int j = 0; j < 2; ++j) {
      if (p[i].x[j] < p1[j]) p1[j] = p[i].x[j];
      if (p[i].x[j] > p2[j]) p2[j] = p[i].x[j];
    }
  if (n == 1) {
    p1[0] = -0.25; p1[1] = -0.25; p2[0] = 0.25; p2[1] = 0.25;
  }
  double lengths[2] = {p2[0] - p1[0], p2[1] - p1[1]};
  t->original_xl = lengths[0];
  t->original_yl = lengths[1];
  if (lengths[0] == 0 || lengths[1] == 0) {
    if (err) *err = 1;
    free(t->index);
    free(t);
    return NULL;
  }
  int j = lengths[0] > lengths[1] ? 1 : 0;
  p2[j] = p1[j] + lengths[!j];

  t->top = new_branch();
  t->nbranches = 1;
  t->top->p1[0] = p1[0]; t->top->p1[1] = p1[1];
  t->top->p2[0] = p2[0]; t->top->p2[1] = p2[1];
  t->top->nparticles = n;
  t->top->particles = t->index;
  t->top->level = 0;
  t->work = (double *)malloc(n * sizeof(double));
  build_rec(t, t->top, 1);
  free(t->work);
  t->work = NULL;

  orc_branch *b = t->top, *last = t->top;
  while (b) {
    moments_one(t, b);
    last = b;
    b = walk_step(b);
  }
  t->current = last;
  return t;
}

void orc_tree_free(orc_tree *t) {
  if (!t) return;
  free_rec(t->top);
  free(t->index);
  free(t);
}

size_t orc_tree_nbranches(const orc_tree *t) { return t->nbranches; }

void orc_tree_export(const orc_tree *t, double *out) {
  const orc_branch *b = t->top;
  size_t k = 0;
  while (b) {
    double *o = out + 16 * k;
    o[0] = b->level; o[1] = b->p1[0]; o[2] = b->p1[1]; o[3] = b->p2[0]; o[4] = b->p2[1];
    o[5] = (double)b->nparticles; o[6] = (double)b->nbig; o[7] = b->mass;
    o[8] = b->center[0]; o[9] = b->center[1];
    o[10] = b->quad[0]; o[11] = b->quad[1]; o[12] = b->quad[2];
    o[13] = b->r2crit; o[14] = is_leaf(b);
    o[15] = (b->p2[0] - b->p1[0]) * (b->p2[0] - b->p1[0]);
    ++k;
    b = walk_step((orc_branch *)b);
  }
}

void orc_tree_membership(const orc_tree *t, double *out) {
  const orc_branch *b = t->top;
  size_t k = 0;
  while (b) {
    double s1 = 0, s2 = 0;
    for (size_t i = 0; i < b->nparticles; ++i) {
      double v = (double)(b->particles[i] + 1);
      s1 += v;
      s2 += v * v;
    }
    out[2 * k] = s1;
    out[2 * k + 1] = s2;
    ++k;
    b = walk_step((orc_branch *)b);
  }
}

/* TreeQuadParticles::b_spline_profile, include/quadTree.h:147-190 */
static void b_spline_profile(const orc_tree *t, const double *xcm, double r, double Mass,
                             double size, double *alpha, double *kappa, double *gamma,
                             double *phi) {
  double q = r / size, M, sigma;
  if (q > 2) {
    sigma = 0;
    M = 1;
  } else {
    double q2 = q * q, q3 = q2 * q, q4 = q2 * q2, q5 = q4 * q;
    sigma = (8 - 12 * q + 6 * q2 - q3) / 4;
    if (q > 1) {
      sigma *= 10 / size / size / 7 / ORC_PI;
      M = (-1 + 20 * q2 * (1 - q + 3 * q2 / 8 - q3 / 20)) / 7;
      *phi += Mass * (-1232. + 1200 * q2 - 800. * q3 + 225. * q4 - 24 * q5 + 120 * log(2. / q)) / 840 / ORC_PI;
    } else {
      sigma = 10 * (sigma - 1 + 3 * q - 3 * q2 + q3) / size / size / 7 / ORC_PI;
      M = 10 * q2 * (1 - 3 * q / 4 + 3 * q3 / 10) / 7;
      *phi += Mass * (t->phiintconst + 10 * (q2 / 2 - 3 * q4 / 4 + 3 * q5 / 50) / 7) / ORC_PI;
    }
  }
  double alpha_r = (M - 1) / ORC_PI / r;
  double gt = alpha_r / r - sigma;
  alpha[0] -= Mass * alpha_r * xcm[0] / r;
  alpha[1] -= Mass * alpha_r * xcm[1] / r;
  gamma[0] -= gt * Mass * (xcm[0] * xcm[0] - xcm[1] * xcm[1]) / r / r;
  gamma[1] -= gt * Mass * 2 * xcm[0] * xcm[1] / r / r;
  *kappa += Mass * sigma;
  *phi -= Mass * log(r) / ORC_PI;
}

/* TreeQuadParticles::walkTree_recur, include/quadTree.h:990-1128.  The
 * far-field potential reads the mass and quadrupole of tree->current, which
 * after construction is the last branch of the moments walk (quadTree.h:1103-
 * 1104); that quirk is kept. */
static void walk_recur(const orc_tree *t, const orc_branch *b, const double *ray, double *alpha,
                       double *kappa, double *gamma, double *phi) {
  double xcm[2], rcm2cell, rcm2, tmp, boxsize2, prefac;
  size_t i;
  if (b->nparticles == 0) return;
  xcm[0] = b->center[0] - ray[0];
  xcm[1] = b->center[1] - ray[1];
  rcm2cell = xcm[0] * xcm[0] + xcm[1] * xcm[1];
  boxsize2 = (b->p2[0] - b->p1[0]) * (b->p2[0] - b->p1[0]);
  if (rcm2cell < b->r2crit || rcm2cell < 5.83 * boxsize2) {
    if (is_leaf(b)) {
      for (i = 0; i < b->nparticles; ++i) {
        xcm[0] = t->xxp[b->particles[i]].x[0] - ray[0];
        xcm[1] = t->xxp[b->particles[i]].x[1] - ray[1];
        rcm2 = xcm[0] * xcm[0] + xcm[1] * xcm[1];
        double screening = exp(-rcm2 * t->inv_screen2);
        if (rcm2 < 1e-20) rcm2 = 1e-20;
        double mass = pmass(t, b->particles[i]);
        prefac = mass * screening / rcm2 / ORC_PI;
        alpha[0] += (t->inv_area * mass - prefac) * xcm[0];
        alpha[1] += (t->inv_area * mass - prefac) * xcm[1];
        tmp = -2.0 * prefac / rcm2;
        gamma[0] += 0.5 * (xcm[0] * xcm[0] - xcm[1] * xcm[1]) * tmp;
        gamma[1] += xcm[0] * xcm[1] * tmp;
        *kappa -= mass * t->inv_area;
        *phi += prefac * rcm2 * 0.5 * log(rcm2) - mass * t->inv_area * rcm2 / 2;
      }
    }
    if (rcm2cell < 5.83 * boxsize2) {
      for (i = 0; i < b->nbig; ++i) {
        size_t idx = b->big[i];
        xcm[0] = t->xxp[idx].x[0] - ray[0];
        xcm[1] = t->xxp[idx].x[1] - ray[1];
        rcm2 = xcm[0] * xcm[0] + xcm[1] * xcm[1];
        if (rcm2 < 1e-20) rcm2 = 1e-20;
        double size = psize(t, idx);
        if (rcm2 < 4 * size * size)
          b_spline_profile(t, xcm, sqrt(rcm2), pmass(t, idx), size, alpha, kappa, gamma, phi);
      }
    }
    for (int k = 0; k < 4; ++k)
      if (b->child[k]) walk_recur(t, b->child[k], ray, alpha, kappa, gamma, phi);
  } else {
    double screening = exp(-rcm2cell * t->inv_screen2);
    double tt = b->mass * t->inv_area - b->mass / rcm2cell / ORC_PI * screening;
    alpha[0] += tt * xcm[0];
    alpha[1] += tt * xcm[1];
    tt = -2.0 * b->mass / ORC_PI / rcm2cell / rcm2cell * screening;
    gamma[0] += 0.5 * (xcm[0] * xcm[0] - xcm[1] * xcm[1]) * tt;
    gamma[1] += xcm[0] * xcm[1] * tt;
    const orc_branch *c = t->current;
    *phi += 0.5 * c->mass * log(rcm2cell) / ORC_PI * screening;
    *phi -= 0.5 * (c->quad[0] * xcm[0] * xcm[0] + c->quad[1] * xcm[1] * xcm[1] +
                   2 * c->quad[2] * xcm[0] * xcm[1]) /
            (ORC_PI * rcm2cell * rcm2cell) * screening;
    alpha[0] -= (b->quad[0] * xcm[0] + b->quad[2] * xcm[1]) / (rcm2cell * rcm2cell) / ORC_PI * screening;
    alpha[1] -= (b->quad[1] * xcm[1] + b->quad[2] * xcm[0]) / (rcm2cell * rcm2cell) / ORC_PI * screening;
    tt = 4 * (b->quad[0] * xcm[0] * xcm[0] + b->quad[1] * xcm[1] * xcm[1] + 2 * b->quad[2] * xcm[0] * xcm[1]) /
         (rcm2cell * rcm2cell * rcm2cell) / ORC_PI * screening;
    alpha[0] += tt * xcm[0];
    alpha[1] += tt * xcm[1];
    *kappa -= t->inv_area * b->mass;
    *phi -= 0.5 * b->mass * rcm2cell * t->inv_area;
  }
}

/* TreeQuadParticles::force2D_recur, include/quadTree.h:932-987 */
void orc_tree_force2D_recur(orc_tree *t, const double *ray, double *alpha, double *kappa,
                            double *gamma, double *phi) {
  alpha[0] = alpha[1] = gamma[0] = gamma[1] = gamma[2] = 0.0;
  *kappa = *phi = 0.0;
  if (t->n == 0) return;
  if (t->periodic) {
    double tr[2];
    for (int i = -1; i < 2; ++i)
      for (int j = -1; j < 2; ++j) {
        tr[0] = ray[0] + i * t->original_xl;
        tr[1] = ray[1] + j * t->original_yl;
        walk_recur(t, t->top, tr, alpha, kappa, gamma, phi);
      }
  } else {
    walk_recur(t, t->top, ray, alpha, kappa, gamma, phi);
  }
}

void orc_direct_sum(const orc_particle *p, size_t n, double inv_area, const double *ray,
                    double *alpha, double *kappa, double *gamma, double *phi) {
  orc_tree dummy;
  memset(&dummy, 0, sizeof(dummy));
  dummy.phiintconst = (120 * log(2.) - 631.) / 840 + 19. / 70;
  alpha[0] = alpha[1] = gamma[0] = gamma[1] = gamma[2] = 0.0;
  *kappa = *phi = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double xcm[2] = {p[i].x[0] - ray[0], p[i].x[1] - ray[1]};
    double rcm2 = xcm[0] * xcm[0] + xcm[1] * xcm[1];
    if (rcm2 < 1e-20) rcm2 = 1e-20;
    double mass = p[i].Mass, prefac = mass / rcm2 / ORC_PI;
    alpha[0] += (inv_area * mass - prefac) * xcm[0];
    alpha[1] += (inv_area * mass - prefac) * xcm[1];
    double tmp = -2.0 * prefac / rcm2;
    gamma[0] += 0.5 * (xcm[0] * xcm[0] - xcm[1] * xcm[1]) * tmp;
    gamma[1] += xcm[0] * xcm[1] * tmp;
    *kappa -= mass * inv_area;
    *phi += prefac * rcm2 * 0.5 * log(rcm2) - mass * inv_area * rcm2 / 2;
    double size = p[i].Size;
    if (rcm2 < 4 * size * size) b_spline_profile(&dummy, xcm, sqrt(rcm2), mass, size, alpha, kappa, gamma, phi);
  }
}

/* =========================== halos ===================================== */
enum { ORC_PARTICLES = 0, ORC_NFW = 1, ORC_NSIE = 2, ORC_FIELD = 3 };

typedef struct orc_halotree orc_halotree;

struct orc_halo {
  int kind;
  double posHalo[2]; /* radians */
  double zlens;
  double Dist;       /* angular-size distance used by getX */
  float mass, Rsize, Rmax, rscale; /* LensHalo members are float (lens_halos.h:276-356) */
  double xmax, gmax;
  float sigma, fratio, pa, rcore, units;
  orc_tree *tree;
  orc_particle *owned;
  orc_halotree *htree; /* ORC_FIELD: LensPlaneTree's TreeQuadHalos */
};

/* ---- NFW profile functions, AnalyticNSIE/nfw_lens.cpp:82-132 ---- */
static double nfw_g(double x) {
  double ans;
  if (x < 1e-5) x = 1e-5;
  ans = log(x / 2);
  if (x == 1.0) { ans += 1.0; return ans; }
  if (x > 1.0) { ans += 2 * atan(sqrt((x - 1) / (x + 1))) / sqrt(x * x - 1); return ans; }
  ans += 2 * atanh(sqrt((1 - x) / (x + 1))) / sqrt(1 - x * x);
  return ans;
}
static double nfw_f(double x) {
  if (x == 0) x = 1e-5;
  if (x == 1.0) return 1.0 / 3.0;
  if (x > 1.0) return (1 - 2 * atan(sqrt((x - 1) / (x + 1))) / sqrt(x * x - 1)) / (x * x - 1);
  return (1 - 2 * atanh(sqrt((1 - x) / (x + 1))) / sqrt(1 - x * x)) / (x * x - 1);
}
static double nfw_g2(double x) {
  double ans, y;
  if (x == 0) x = 1e-5;
  if (x == 1) return 10 / 3. + 4 * log(0.5);
  y = x * x - 1;
  ans = 4 * log(x / 2) / x / x - 2 / y;
  if (x < 1.0) return ans + 4 * (2 / x / x + 1 / y) * atanh(sqrt((1 - x) / (x + 1))) / sqrt(-y);
  return ans + 4 * (2 / x / x + 1 / y) * atan(sqrt((x - 1) / (x + 1))) / sqrt(y);
}
static double nfw_h(double x) {
  if (x == 0) x = 1e-5;
  if (x <= 1.0) return 2. * ((log(x / 2.) * log(x / 2.)) - atanh(sqrt(1. - x * x)) * atanh(sqrt(1. - x * x)));
  return 2. * ((log(x / 2.) * log(x / 2.)) + atan(sqrt(x * x - 1.)) * atan(sqrt(x * x - 1.)));
}

/* LensHaloNFW static tables, MultiPlane/lens_halos.cpp:352-353,482-508 */
#define NFW_NTABLE 10000
#define NFW_MAXRM 100.0
static double *nfw_xt, *nfw_ft, *nfw_gt, *nfw_g2t, *nfw_ht;
static pthread_once_t nfw_once = PTHREAD_ONCE_INIT;
static void nfw_make_tables(void) {
  double dx = NFW_MAXRM / (double)NFW_NTABLE;
  nfw_xt = (double *)malloc(NFW_NTABLE * sizeof(double));
  nfw_ft = (double *)malloc(NFW_NTABLE * sizeof(double));
  nfw_gt = (double *)malloc(NFW_NTABLE * sizeof(double));
  nfw_g2t = (double *)malloc(NFW_NTABLE * sizeof(double));
  nfw_ht = (double *)malloc(NFW_NTABLE * sizeof(double));
  for (int i = 0; i < NFW_NTABLE; i++) {
    double x = i * dx;
    nfw_xt[i] = x;
    nfw_ft[i] = nfw_f(x);
    nfw_gt[i] = nfw_g(x);
    nfw_g2t[i] = nfw_g2(x);
    nfw_ht[i] = nfw_h(x);
  }
}
/* LensHaloNFW::InterpolateFromTable, lens_halos.cpp:566-580 (bin 0 analytic) */
static double nfw_interp(const double *table, double y) {
  int j = (int)(y / NFW_MAXRM * NFW_NTABLE);
  if (j == 0) {
    if (table == nfw_ft) return nfw_f(y);
    if (table == nfw_gt) return nfw_g(y);
    if (table == nfw_g2t) return nfw_g2(y);
    if (table == nfw_ht) return nfw_h(y);
  }
  return (table[j + 1] - table[j]) / (nfw_xt[j + 1] - nfw_xt[j]) * (y - nfw_xt[j]) + table[j];
}

orc_halo *orc_halo_nfw(float mass, float Rsize, double z, float conc, float fratio, float pa) {
  pthread_once(&nfw_once, nfw_make_tables);
  orc_halo *h = (orc_halo *)calloc(1, sizeof(orc_halo));
  h->kind = ORC_NFW;
  h->zlens = z;
  h->Dist = orc_angdist(z); /* LensHalo(z,cosmo), lens_halos.cpp:25-34 */
  h->Rsize = Rsize;
  h->mass = mass;
  h->fratio = fratio;
  h->pa = (float)(ORC_PI / 2 - pa);
  h->rscale = h->Rsize / conc;            /* float / float */
  h->xmax = (double)(h->Rsize / h->rscale); /* float / float */
  h->gmax = nfw_interp(nfw_gt, h->xmax);
  h->Rmax = h->Rsize;                     /* fratio == 1, lens_halos.cpp:425-428 */
  return h;
}

/* ---- NSIE, AnalyticNSIE/nsie.cpp:14-145,199-204 ---- */
static void rotation(double *xout, const double *xin, double theta) {
  double tmp = xin[0];
  xout[0] = tmp * cos(theta) - xin[1] * sin(theta);
  xout[1] = xin[1] * cos(theta) + tmp * sin(theta);
}
static void alphaNSIE(double *alpha, const double *xt, double f, double bc, double theta) {
  double r = sqrt(xt[0] * xt[0] + xt[1] * xt[1]);
  if (r < 1.0e-20 || r > 1.0e20) { alpha[0] = alpha[1] = 0.0; return; }
  if (f == 1.0) {
    if (bc == 0.0) {
      alpha[0] = -1.0 * xt[0] / r;
      alpha[1] = -1.0 * xt[1] / r;
    } else {
      alpha[0] = -1.0 * (sqrt(r * r + bc * bc) - bc) * xt[0] / r / r;
      alpha[1] = -1.0 * (sqrt(r * r + bc * bc) - bc) * xt[1] / r / r;
    }
    return;
  }
  double x[2], fp, b2;
  int s;
  rotation(x, xt, theta);
  if (x[0] > 0) { s = -1; x[0] *= -1; } else s = 1;
  fp = sqrt(1 - f * f);
  b2 = x[0] * x[0] + f * f * x[1] * x[1];
  double complex c_x = x[0] + x[1] * I;
  double complex tmp = f * f * c_x * c_x - fp * fp * bc * bc;
  double complex xi = fp / csqrt(tmp);
  double complex c_alpha = sqrt(f) * (casinh(xi * sqrt(b2 + bc * bc)) - casinh(xi * bc)) / fp;
  alpha[0] = s * creal(c_alpha);
  alpha[1] = -cimag(c_alpha);
  rotation(alpha, alpha, -theta);
}
static double kappaNSIE(const double *xt, double f, double bc, double theta) {
  double x[2], b2;
  rotation(x, xt, theta);
  b2 = x[0] * x[0] + f * f * x[1] * x[1];
  if ((b2 < 1.0e-20) && (bc < 1.0e-20)) return 1.0e10;
  if (b2 > 1.0e20) return 0.0;
  return 0.5 * sqrt(f / (b2 + bc * bc));
}
static void gammaNSIE(double *gam, const double *xt, double f, double bc, double theta) {
  double r = sqrt(xt[0] * xt[0] + xt[1] * xt[1]);
  if (r < 1.0e-20 || r > 1.0e20) { gam[0] = gam[1] = 0.0; return; }
  double x[2], fp, P, b2;
  rotation(x, xt, theta);
  fp = sqrt(1 - f * f);
  b2 = x[0] * x[0] + f * f * x[1] * x[1];
  P = sqrt(f) * (kappaNSIE(x, f, bc, 0.0) * (x[0] * x[0] + f * f * f * f * x[1] * x[1]) / sqrt(f) -
                 0.5 * (1 + f * f) * sqrt(b2 + bc * bc) + f * bc) /
      (pow(f * r, 4) - 2 * f * f * fp * fp * bc * bc * (x[0] * x[0] - x[1] * x[1]) + pow(fp * bc, 4));
  gam[0] = (f * f * (x[0] * x[0] - x[1] * x[1]) - fp * fp * bc * bc) * P;
  gam[1] = 2 * f * f * x[0] * x[1] * P;
  rotation(gam, gam, -2 * theta);
}

static void nsie_force_inner(const orc_halo *h, const double *xcm, double *alpha, double *kappa,
                             double *gamma);

/* LensHalo::MassBy1DIntegation, lens_halos.cpp:2469-2473: R/2 times the
 * integral over angle of the inward radial deflection on the circle R.  The
 * integrand is smooth and periodic, so a 4096-point trapezoid rule is used. */
static double nsie_mass_1d(orc_halo *h, double R) {
  const int NQ = 4096;
  double sum = 0.0;
  for (int i = 0; i < NQ; ++i) {
    double th = 2 * ORC_PI * i / NQ;
    double x[2] = {R * cos(th), R * sin(th)}, a[2] = {0, 0}, k = 0, g[3] = {0, 0, 0};
    nsie_force_inner(h, x, a, &k, g);
    sum += -a[0] * cos(th) - a[1] * sin(th);
  }
  return R * (sum * 2 * ORC_PI / NQ) / 2;
}

orc_halo *orc_halo_nsie(float mass, double z, float sigma, float rcore, float fratio, float pa) {
  orc_halo *h = (orc_halo *)calloc(1, sizeof(orc_halo));
  h->kind = ORC_NSIE;
  h->rscale = 1.0f;
  h->mass = mass;
  h->zlens = z;
  h->Dist = orc_angdist(z);
  h->sigma = sigma;
  h->rcore = rcore;
  h->fratio = fratio;
  h->pa = (float)(ORC_PI / 2 - pa);
  /* rmax_calc, lens_halos.cpp:1154-1171 (circular or cored branch only) */
  {
    float sf = sqrtf(h->fratio); /* sqrt of a float member is the float overload */
    double a = (double)h->mass * ORC_GRAV * ORC_LIGHTSPEED * ORC_LIGHTSPEED * (double)sf / ORC_PI /
                   (double)h->sigma / (double)h->sigma + (double)h->rcore;
    h->Rsize = (float)sqrt(pow(a, 2) - (double)(h->rcore * h->rcore));
  }
  h->Rmax = 1.2f * h->Rsize; /* Rmax_to_Rsize_ratio (float) * getRsize() */
  h->units = (float)(pow((double)h->sigma / ORC_LIGHTSPEED, 2) / ORC_GRAV);
  if (h->rcore > 0.0) h->mass = (float)nsie_mass_1d(h, (double)h->Rsize);
  return h;
}

orc_halo *orc_halo_particles(const orc_particle *p, size_t n, double z, double inv_area, double max_range) {
  orc_halo *h = (orc_halo *)calloc(1, sizeof(orc_halo));
  h->kind = ORC_PARTICLES;
  h->zlens = (double)(float)z; /* the vector constructor takes a float redshift */
  h->Dist = orc_angdist(h->zlens);
  h->owned = (orc_particle *)malloc((n ? n : 1) * sizeof(orc_particle));
  memcpy(h->owned, p, n * sizeof(orc_particle));
  double m = 0;
  for (size_t i = 0; i < n; ++i) m += h->owned[i].Mass; /* set_up, particle_halo.h:366-378 */
  h->mass = (float)m;
  h->Rsize = h->Rmax = (float)1.0e100;
  int err = 0;
  /* particle_halo.h:416 passes max_range as the ninth constructor argument,
   * which is inv_screening_scale (quadTree.h:49-60): the tree is screened by
   * exp(-r^2 max_range^2) and built without a maximum range. */
  h->tree = orc_tree_build(h->owned, n, -1, -1, inv_area, 20, 0.1, 0, max_range, -1, &err);
  return h;
}

void orc_halo_set_theta(orc_halo *h, double tx, double ty) {
  h->posHalo[0] = tx;
  h->posHalo[1] = ty;
}
static void halotree_free(orc_halotree *t);

void orc_halo_free(orc_halo *h) {
  if (!h) return;
  orc_tree_free(h->tree);
  free(h->owned);
  halotree_free(h->htree);
  free(h);
}
float orc_halo_mass(const orc_halo *h) { return h->mass; }
float orc_halo_rsize(const orc_halo *h) { return h->Rsize; }
float orc_halo_rmax(const orc_halo *h) { return h->Rmax; }

/* LensHalo::force_point, lens_halos.cpp:1555-1598 (subtract_point = false) */
static int force_point(const orc_halo *h, const double *xcm, double rcm2, double *alpha,
                       double *gamma, double *phi) {
  if (rcm2 < (double)(h->Rmax * h->Rmax)) return 0;
  double prefac = h->mass / rcm2 / ORC_PI;
  alpha[0] += -1.0 * prefac * xcm[0];
  alpha[1] += -1.0 * prefac * xcm[1];
  double tmp = -2.0 * prefac / rcm2;
  gamma[0] += 0.5 * (xcm[0] * xcm[0] - xcm[1] * xcm[1]) * tmp;
  gamma[1] += xcm[0] * xcm[1] * tmp;
  *phi += 0.5 * h->mass * log(rcm2) / ORC_PI;
  return 1;
}

/* LensHalo::force_halo_sym, lens_halos.cpp:1608-1672, with LensHaloNFW's
 * alpha_h/kappa_h/gamma_h/phi_h (include/lens_halos.h:842-856) */
static void nfw_force(const orc_halo *h, const double *xcm, double *alpha, double *kappa,
                      double *gamma, double *phi) {
  double rcm2 = xcm[0] * xcm[0] + xcm[1] * xcm[1];
  if (force_point(h, xcm, rcm2, alpha, gamma, phi)) return;
  if (rcm2 < 1e-20) rcm2 = 1e-20;
  if (rcm2 < (double)(h->Rmax * h->Rmax)) {
    double prefac = h->mass / rcm2 / ORC_PI;
    double x = sqrt(rcm2) / h->rscale;
    double tmp = (-1.0 * nfw_interp(nfw_gt, x) / h->gmax) * prefac;
    alpha[0] += tmp * xcm[0];
    alpha[1] += tmp * xcm[1];
    *kappa += 0.5 * x * x * nfw_interp(nfw_ft, x) / h->gmax * prefac;
    tmp = (-0.5 * x * x * nfw_interp(nfw_g2t, x) / h->gmax) * prefac / rcm2;
    gamma[0] += 0.5 * (xcm[0] * xcm[0] - xcm[1] * xcm[1]) * tmp;
    gamma[1] += xcm[0] * xcm[1] * tmp;
    /* phi_h: log of the float Rsize is the float overload */
    double phih = 0.25 * (nfw_interp(nfw_ht, x) - nfw_interp(nfw_ht, (double)(h->Rsize / h->rscale))) / h->gmax +
                  (double)logf(h->Rsize);
    *phi += phih * h->mass / ORC_PI;
  } else {
    double prefac = h->mass / rcm2 / ORC_PI;
    alpha[0] += -1.0 * prefac * xcm[0];
    alpha[1] += -1.0 * prefac * xcm[1];
    double tmp = -2.0 * prefac / rcm2;
    gamma[0] += 0.5 * (xcm[0] * xcm[0] - xcm[1] * xcm[1]) * tmp;
    gamma[1] += xcm[0] * xcm[1] * tmp;
    *phi += 0.5 * log(rcm2) * h->mass / ORC_PI;
  }
}

/* LensHaloRealNSIE::force_halo inside Rmax, lens_halos.cpp:1955-2014 */
static void nsie_force_inner(const orc_halo *h, const double *xcm, double *alpha, double *kappa,
                             double *gamma) {
  double rcm2 = xcm[0] * xcm[0] + xcm[1] * xcm[1];
  if (rcm2 < 1e-20) rcm2 = 1e-20;
  if (!(rcm2 < (double)(h->Rmax * h->Rmax))) return;
  if (rcm2 > (double)(h->Rsize * h->Rsize)) {
    double alpha_iso[2], alpha_ellip[2];
    double r = sqrt(rcm2);
    double f1 = ((double)h->Rmax - r) / (double)(h->Rmax - h->Rsize);
    double f2 = (r - (double)h->Rsize) / (double)(h->Rmax - h->Rsize);
    alpha_ellip[0] = alpha_ellip[1] = 0;
    alphaNSIE(alpha_ellip, xcm, h->fratio, h->rcore, h->pa);
    alpha_ellip[0] *= h->units;
    alpha_ellip[1] *= h->units;
    double tmp = (double)h->mass / rcm2 / ORC_PI;
    alpha_iso[0] = -1.0 * tmp * xcm[0];
    alpha_iso[1] = -1.0 * tmp * xcm[1];
    alpha[0] += alpha_iso[0] * f2 + alpha_ellip[0] * f1;
    alpha[1] += alpha_iso[1] * f2 + alpha_ellip[1] * f1;
    tmp = -2.0 * (double)h->mass / rcm2 / ORC_PI / rcm2;
    gamma[0] += 0.5 * (xcm[0] * xcm[0] - xcm[1] * xcm[1]) * tmp;
    gamma[1] += xcm[0] * xcm[1] * tmp;
  } else {
    double xt[2] = {xcm[0], xcm[1]}, tmp[2] = {0, 0}, g[2] = {0, 0};
    alphaNSIE(tmp, xt, h->fratio, h->rcore, h->pa);
    alpha[0] += h->units * tmp[0];
    alpha[1] += h->units * tmp[1];
    *kappa += h->units * kappaNSIE(xt, h->fratio, h->rcore, h->pa);
    gammaNSIE(g, xt, h->fratio, h->rcore, h->pa);
    gamma[0] += h->units * g[0];
    gamma[1] += h->units * g[1];
  }
}

static void nsie_force(const orc_halo *h, const double *xcm, double *alpha, double *kappa,
                       double *gamma, double *phi) {
  double rcm2 = xcm[0] * xcm[0] + xcm[1] * xcm[1];
  if (force_point(h, xcm, rcm2, alpha, gamma, phi)) return;
  nsie_force_inner(h, xcm, alpha, kappa, gamma);
}

static void halotree_force2D(const orc_halotree *t, const double *ray, double *alpha, double *kappa,
                             double *gamma, double *phi);

/* One halo at one position; the particle halo overwrites and negates alpha
 * (include/particle_halo.h:426-434); a field plane's halo tree overwrites
 * (LensPlaneTree::force, MultiPlane/planes.cpp:65-68). */
static void halo_force_one(orc_halo *h, const double *xcm, double *alpha, double *kappa,
                           double *gamma, double *phi) {
  switch (h->kind) {
    case ORC_FIELD: halotree_force2D(h->htree, xcm, alpha, kappa, gamma, phi); break;
    case ORC_PARTICLES:
      orc_tree_force2D_recur(h->tree, xcm, alpha, kappa, gamma, phi);
      alpha[0] *= -1;
      alpha[1] *= -1;
      break;
    case ORC_NFW: nfw_force(h, xcm, alpha, kappa, gamma, phi); break;
    case ORC_NSIE: nsie_force(h, xcm, alpha, kappa, gamma, phi); break;
  }
}

void orc_halo_force(orc_halo *h, size_t n, const double *xcm, double *alpha, double *kappa,
                    double *gamma, double *phi) {
  for (size_t i = 0; i < n; ++i) {
    double a[2] = {0, 0}, k = 0, g[3] = {0, 0, 0}, p = 0;
    halo_force_one(h, xcm + 2 * i, a, &k, g, &p);
    alpha[2 * i] = a[0];
    alpha[2 * i + 1] = a[1];
    kappa[i] = k;
    gamma[3 * i] = g[0];
    gamma[3 * i + 1] = g[1];
    gamma[3 * i + 2] = g[2];
    phi[i] = p;
  }
}

/* ===================== source surface brightness ======================== */
/* SourceUniform::SurfaceBrightness (AnalyticNSIE/source.cpp:207-209),
 * SourceGaussian::SurfaceBrightness (source.cpp:211-213) and
 * SourceSersic::SurfaceBrightness (Source/sersic.cpp:116-135, constants from
 * ReSet / setReff / setSersicIndex / setAxesRatio, include/sersic_source.h). */
void orc_source_sb(int kind, const double *p, size_t n, const double *y, double *out) {
  for (size_t i = 0; i < n; ++i) {
    const double d0 = y[2 * i] - p[0], d1 = y[2 * i + 1] - p[1];
    if (kind == 0) {
      out[i] = (double)((pow(d0, 2) + pow(d1, 2)) < p[2] * p[2]);
    } else if (kind == 1) {
      out[i] = exp(-(pow(d0, 2) + pow(d1, 2)) / (p[2] * p[2]));
    } else {
      const double flux = p[2], Reff = p[3] * 4.848136811e-6, PA = p[4], index = p[5], sb_limit = p[7];
      double q = p[6];
      if (q > 1) q = 1 / q;
      const double bn = 1.9992 * index - 0.3271;
      const double I_n = 1. / index * pow(bn, 2 * index) / tgamma(2 * index);
      const double I_q = 1. / q, I_r = 1. / 2. / ORC_PI / Reff / Reff;
      const double cosPA = cos(PA), sinPA = sin(PA);
      const double x0 = d0 * cosPA + d1 * sinPA, x1 = d0 * sinPA - d1 * cosPA;
      double r = sqrt(x0 * x0 + x1 * x1 / q / q);
      if (r < 4.848136811e-9) r = 4.848136811e-9;
      double sb = flux * I_n * I_q * I_r * exp(-bn * pow(r / Reff, 1. / index));
      out[i] = sb < sb_limit ? 0. : sb;
    }
  }
}

/* =================== TreeQuadHalos / LensPlaneTree ===================== */
/* A quadtree over analytic haloes (include/quadTreeHalos.h:35-130) as built by
 * LensPlaneTree (MultiPlane/planes.cpp:13-18). */
typedef struct orc_hbranch {
  size_t *particles;
  size_t nparticles;
  size_t *big;
  size_t nbig;
  double center[2];
  double mass;
  double p1[2], p2[2];
  struct orc_hbranch *child[4];
  struct orc_hbranch *brother;
  double quad[3];
  double rmax;
  double r2crit;
} orc_hbranch;

struct orc_halotree {
  int n;
  orc_halo **halos;  /* owned */
  double *xp;        /* 2n: LensHalo::getX at construction */
  size_t *index;
  double *work;
  double inv_area;
  int bucket;
  double theta;
  int periodic;
  double inv_screen2;
  double max_range;
  double original_xl, original_yl;
  orc_hbranch *top;
};

static void hbranch_free(orc_hbranch *b) {
  if (!b) return;
  for (int c = 0; c < 4; ++c) hbranch_free(b->child[c]);
  free(b->big);
  free(b);
}

static void halotree_free(orc_halotree *t) {
  if (!t) return;
  hbranch_free(t->top);
  for (int i = 0; i < t->n; ++i) orc_halo_free(t->halos[i]);
  free(t->halos);
  free(t->xp);
  free(t->index);
  free(t->work);
  free(t);
}

/* TreeQuadHalos::_BuildQTreeNB, include/quadTreeHalos.h:239-450.  Big
 * haloes (Rmax beyond half the box) are listed at the branch and still passed
 * on to its children; a leaf lists all of its haloes as big. */
static void hbuild_rec(orc_halotree *t, orc_hbranch *cb, int at_top) {
  size_t i, cut = 0, cut2 = 0, cutx = 0, cuty = 0;
  size_t *particles = cb->particles;
  const size_t np = cb->nparticles;
  cb->center[0] = (cb->p1[0] + cb->p2[0]) / 2;
  cb->center[1] = (cb->p1[1] + cb->p2[1]) / 2;
  cb->quad[0] = cb->quad[1] = cb->quad[2] = 0;
  cb->mass = 0.0;
  double theta_range = 2 * t->theta;
  if (t->max_range > 0) {
    double boxsize = 1.732 * (cb->p2[0] - cb->p1[0]);
    double d = sqrt(cb->center[0] * cb->center[0] + cb->center[1] * cb->center[1]) - t->max_range;
    theta_range = boxsize / (d > boxsize ? d : boxsize);
  }
  if (np <= (size_t)t->bucket || t->theta > theta_range) {
    cb->nbig = np;
    cb->big = (size_t *)malloc((np ? np : 1) * sizeof(size_t));
    for (i = 0; i < np; ++i) cb->big[i] = particles[i];
    return;
  }
  double *x = t->work;
  cb->nbig = 0;
  for (i = 0; i < np; ++i) x[i] = (double)t->halos[particles[i]]->Rmax;
  double half_box = (cb->p2[0] - cb->p1[0]) / 2;
  quick_partition(half_box, &cut, particles, x, np);
  if (cut < np) {
    if (at_top) {
      cb->nbig = cut2 = np - cut;
    } else {
      quick_partition(2 * half_box, &cut2, &particles[cut], &x[cut], np - cut);
      cb->nbig = cut2;
    }
    cb->big = (size_t *)malloc((cut2 ? cut2 : 1) * sizeof(size_t));
    for (i = cut; i < cut + cut2; ++i) cb->big[i - cut] = particles[i];
  }
  orc_hbranch *c[4];
  for (int k = 0; k < 4; ++k) c[k] = (orc_hbranch *)calloc(1, sizeof(orc_hbranch));
  for (int k = 0; k < 3; ++k) c[k]->brother = c[k + 1];
  c[3]->brother = cb->brother;
  for (int k = 0; k < 4; ++k) cb->child[k] = c[k];
  c[0]->p1[0] = cb->center[0]; c[0]->p1[1] = cb->center[1]; c[0]->p2[0] = cb->p2[0]; c[0]->p2[1] = cb->p2[1];
  c[1]->p1[0] = cb->p1[0]; c[1]->p1[1] = cb->center[1]; c[1]->p2[0] = cb->center[0]; c[1]->p2[1] = cb->p2[1];
  c[2]->p1[0] = cb->center[0]; c[2]->p1[1] = cb->p1[1]; c[2]->p2[0] = cb->p2[0]; c[2]->p2[1] = cb->center[1];
  c[3]->p1[0] = cb->p1[0]; c[3]->p1[1] = cb->p1[1]; c[3]->p2[0] = cb->center[0]; c[3]->p2[1] = cb->center[1];
  const double xcut = cb->center[0], ycut = cb->center[1];
  for (i = 0; i < np; ++i) x[i] = t->xp[2 * particles[i] + 1];
  quick_partition(ycut, &cuty, particles, x, np);
  if (cuty > 0) {
    for (i = 0; i < cuty; ++i) x[i] = t->xp[2 * particles[i]];
    quick_partition(xcut, &cutx, particles, x, cuty);
    c[3]->nparticles = cutx;
    c[3]->particles = cutx > 0 ? particles : NULL;
    c[2]->nparticles = cuty - cutx;
    c[2]->particles = cuty - cutx > 0 ? &particles[cutx] : NULL;
  }
  if (cuty < np) {
    for (i = cuty; i < np; ++i) x[i - cuty] = t->xp[2 * particles[i]];
    quick_partition(xcut, &cutx, &particles[cuty], x, np - cuty);
    c[1]->nparticles = cutx;
    c[1]->particles = cutx > 0 ? &particles[cuty] : NULL;
    c[0]->nparticles = np - cuty - cutx;
    c[0]->particles = np - cuty - cutx > 0 ? &particles[cuty + cutx] : NULL;
  }
  for (int k = 0; k < 4; ++k) hbuild_rec(t, c[k], 0);
}

/* TreeQuadHalos::CalcMoments, include/quadTreeHalos.h:453-513 (one branch). */
static void hmoments_one(orc_halotree *t, orc_hbranch *cb) {
  size_t i;
  cb->rmax = sqrt(pow(cb->p2[0] - cb->p1[0], 2) + pow(cb->p2[1] - cb->p1[1], 2));
  for (i = 0, cb->mass = 0; i < cb->nparticles; ++i) cb->mass += t->halos[cb->particles[i]]->mass;
  cb->center[0] = cb->center[1] = 0;
  for (i = 0; i < cb->nparticles; ++i) {
    double tmp = t->halos[cb->particles[i]]->mass;
    cb->center[0] += tmp * t->xp[2 * cb->particles[i]] / cb->mass;
    cb->center[1] += tmp * t->xp[2 * cb->particles[i] + 1] / cb->mass;
  }
  cb->quad[0] = cb->quad[1] = cb->quad[2] = 0;
  for (i = 0; i < cb->nparticles; ++i) {
    double xcm0 = t->xp[2 * cb->particles[i]] - cb->center[0];
    double xcm1 = t->xp[2 * cb->particles[i] + 1] - cb->center[1];
    double xcut = pow(xcm0, 2) + pow(xcm1, 2);
    double tmp = t->halos[cb->particles[i]]->mass;
    cb->quad[0] += (xcut - 2 * xcm0 * xcm0) * tmp;
    cb->quad[1] += (xcut - 2 * xcm1 * xcm1) * tmp;
    cb->quad[2] += -2 * xcm0 * xcm1 * tmp;
  }
  double rcom = 0.0;
  for (i = 0; i < 2; ++i) {
    double a = pow(cb->center[i] - cb->p1[i], 2), b = pow(cb->center[i] - cb->p2[i], 2);
    rcom += (a > b) ? a : b;
  }
  rcom = sqrt(rcom);
  if (t->theta > 0.0) {
    cb->r2crit = 1.15470 * rcom / (t->theta);
    cb->r2crit *= cb->r2crit;
  } else {
    cb->r2crit = 1.0e100;
  }
}

static void hmoments_rec(orc_halotree *t, orc_hbranch *b) {
  hmoments_one(t, b);
  if (b->child[0])
    for (int k = 0; k < 4; ++k) hmoments_rec(t, b->child[k]);
}

/* LensPlaneTree(z, halos, n, sigma_background, inv_screening_scale),
 * MultiPlane/planes.cpp:13-18: TreeQuadHalos(halos, n, sigma_background) with
 * its defaults (bucket 5, theta 0.5, no periodic buffer, no screening), or
 * with screening: bucket 5, theta 0.1, periodic buffer
 * (include/quadTreeHalos.h:129-159, 173-236).  The haloes are moved to
 * redshift z first (LensHalo::setZlensDist, as Lens::createFieldPlanes does,
 * MultiPlane/lens.cpp:418-426).  Takes ownership of the haloes. */
orc_halo *orc_halo_field_plane(orc_halo **halos, int n, double z, double sigma_back, double inv_screening,
                               int *err) {
  *err = 0;
  orc_halotree *t = (orc_halotree *)calloc(1, sizeof(orc_halotree));
  t->n = n;
  t->halos = (orc_halo **)malloc((n ? n : 1) * sizeof(orc_halo *));
  for (int i = 0; i < n; ++i) t->halos[i] = halos[i];
  t->inv_area = sigma_back;
  if (inv_screening != 0) {
    t->bucket = 5; t->theta = 0.1; t->periodic = 1;
  } else {
    t->bucket = 5; t->theta = 0.5; t->periodic = 0;
  }
  t->inv_screen2 = inv_screening * inv_screening;
  t->max_range = -1;
  t->xp = (double *)malloc((2 * n + 2) * sizeof(double));
  t->index = (size_t *)malloc((n ? n : 1) * sizeof(size_t));
  t->work = (double *)malloc((n ? n : 1) * sizeof(double));
  for (int i = 0; i < n; ++i) {
    orc_halo *h = halos[i];
    h->zlens = z;
    h->Dist = orc_angdist(z);
    t->xp[2 * i] = h->posHalo[0] * h->Dist; /* LensHalo::getX, include/lens_halos.h:95-99 */
    t->xp[2 * i + 1] = h->posHalo[1] * h->Dist;
    t->index[i] = i;
  }
  orc_halo *out = (orc_halo *)calloc(1, sizeof(orc_halo));
  out->kind = ORC_FIELD;
  out->zlens = z;
  out->Dist = orc_angdist(z);
  out->htree = t;
  if (n > 0) {
    /* TreeQuadHalos::BuildQTreeNB, include/quadTreeHalos.h:173-236 */
    double p1[2] = {t->xp[0], t->xp[1]}, p2[2] = {t->xp[0], t->xp[1]};
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < 2; ++j) {
        if (t->xp[2 * i + j] < p1[j]) p1[j] = t->xp[2 * i + j];
        if (t->xp[2 * i + j] > p2[j]) p2[j] = t->xp[2 * i + j];
      }
    if (n == 1) {
      p1[0] = -0.25; p1[1] = -0.25; p2[0] = 0.25; p2[1] = 0.25;
    }
    double lengths[2] = {p2[0] - p1[0], p2[1] - p1[1]};
    t->original_xl = lengths[0];
    t->original_yl = lengths[1];
    if (lengths[0] == 0 || lengths[1] == 0) {
      *err = 1; /* "particles in same place." */
      t->n = 0; /* the caller keeps its haloes */
      orc_halo_free(out);
      return NULL;
    }
    int j = lengths[0] > lengths[1] ? 1 : 0;
    p2[j] = p1[j] + lengths[!j];
    t->top = (orc_hbranch *)calloc(1, sizeof(orc_hbranch));
    t->top->p1[0] = p1[0]; t->top->p1[1] = p1[1];
    t->top->p2[0] = p2[0]; t->top->p2[1] = p2[1];
    t->top->nparticles = n;
    t->top->particles = t->index;
    hbuild_rec(t, t->top, 1);
    hmoments_rec(t, t->top);
  }
  return out;
}

/* TreeQuadHalos::walkTree_iter, include/quadTreeHalos.h:648-815. */
static void hwalk(const orc_halotree *t, const double *ray, double *alpha, double *kappa, double *gamma,
                  double *phi) {
  const orc_hbranch *b = t->top;
  while (b) {
    int descend = 1;
    for (size_t i = 0; i < b->nbig; ++i) {
      size_t k = b->big[i];
      double xcm[2] = {t->xp[2 * k] - ray[0], t->xp[2 * k + 1] - ray[1]};
      double rcm2 = xcm[0] * xcm[0] + xcm[1] * xcm[1];
      (void)exp(-rcm2 * t->inv_screen2); /* screening: unused by force_halo without subtract_point */
      halo_force_one(t->halos[k], xcm, alpha, kappa, gamma, phi);
      double mass = t->halos[k]->mass;
      double prefac = mass * t->inv_area;
      alpha[0] += prefac * xcm[0];
      alpha[1] += prefac * xcm[1];
      *phi += -t->inv_area * rcm2 * mass * 0.5;
      *kappa -= mass * t->inv_area;
    }
    if (b->child[0]) {
      double xc[2] = {b->center[0] - ray[0], b->center[1] - ray[1]};
      double rcm2cell = xc[0] * xc[0] + xc[1] * xc[1];
      if (rcm2cell > b->r2crit) {
        descend = 0;
        double screening = exp(-rcm2cell * t->inv_screen2);
        double tmp = b->mass * (t->inv_area - screening / rcm2cell / ORC_PI);
        alpha[0] += tmp * xc[0];
        alpha[1] += tmp * xc[1];
        tmp = -2.0 * b->mass / ORC_PI / rcm2cell / rcm2cell * screening;
        gamma[0] += 0.5 * (xc[0] * xc[0] - xc[1] * xc[1]) * tmp;
        gamma[1] += xc[0] * xc[1] * tmp;
        *phi += 0.5 * b->mass * log(rcm2cell) / ORC_PI * screening;
        *phi -= 0.5 * (b->quad[0] * xc[0] * xc[0] + b->quad[1] * xc[1] * xc[1] + 2 * b->quad[2] * xc[0] * xc[1]) /
                (ORC_PI * rcm2cell * rcm2cell) * screening;
        alpha[0] -= (b->quad[0] * xc[0] + b->quad[2] * xc[1]) / (rcm2cell * rcm2cell) / ORC_PI * screening;
        alpha[1] -= (b->quad[1] * xc[1] + b->quad[2] * xc[0]) / (rcm2cell * rcm2cell) / ORC_PI * screening;
        tmp = 4 * (b->quad[0] * xc[0] * xc[0] + b->quad[1] * xc[1] * xc[1] + 2 * b->quad[2] * xc[0] * xc[1]) /
              (rcm2cell * rcm2cell * rcm2cell) / ORC_PI * screening;
        alpha[0] += tmp * xc[0];
        alpha[1] += tmp * xc[1];
        *kappa -= b->mass * t->inv_area;
        *phi -= b->mass * t->inv_area * rcm2cell;
      }
    }
    /* QBiterator::TreeWalkStep, include/qTreeNB.h:541-552 */
    b = (descend && b->child[0]) ? b->child[0] : b->brother;
  }
}

/* TreeQuadHalos::force2D, include/quadTreeHalos.h:556-592. */
static void halotree_force2D(const orc_halotree *t, const double *ray, double *alpha, double *kappa,
                             double *gamma, double *phi) {
  alpha[0] = alpha[1] = gamma[0] = gamma[1] = gamma[2] = 0.0;
  *kappa = *phi = 0.0;
  if (t->n == 0) return;
  if (t->periodic) {
    for (int i = -1; i < 2; ++i)
      for (int j = -1; j < 2; ++j) {
        double r[2] = {ray[0] + i * t->original_xl, ray[1] + j * t->original_yl};
        hwalk(t, r, alpha, kappa, gamma, phi);
      }
  } else {
    hwalk(t, ray, alpha, kappa, gamma, phi);
  }
}

/* ============================ Lens ===================================== */
typedef struct {
  double z;
  int nh, cap;
  orc_halo **halos;
} orc_plane;

struct orc_lens {
  double zsource;
  int nmain;          /* main planes, kept sorted by main_Dl */
  orc_plane *main;
  double *main_Dl;
  int nfield;         /* field planes (LensPlaneTree), in insertion order */
  orc_plane *field;
  double *field_Dl;
  int nhalos;
  orc_halo **owned;   /* every halo the lens holds */
  /* combined planes (combinePlanes) */
  int np;             /* lensing planes */
  orc_plane **planes;
  double *plane_z, *Dl, *dDl; /* np+1 entries */
  double charge;
  int toggle_source_plane;
  double zs_implant;
};

/* Lens::combinePlanes, MultiPlane/lens.cpp:2397-2515: field and main planes
 * sorted together by Dl (Utilities::sort_indexes), distances closer than
 * MIN_PLANE_DIST pushed apart, the source pseudo-plane appended. */
static void combine_planes(orc_lens *l) {
  int n = l->nmain + l->nfield;
  free(l->planes); free(l->plane_z); free(l->Dl); free(l->dDl);
  l->np = n;
  l->planes = (orc_plane **)malloc((n + 1) * sizeof(orc_plane *));
  l->plane_z = (double *)malloc((n + 1) * sizeof(double));
  l->Dl = (double *)malloc((n + 1) * sizeof(double));
  l->dDl = (double *)malloc((n + 1) * sizeof(double));
  int *index = (int *)malloc((n + 1) * sizeof(int));
  double *all = (double *)malloc((n + 1) * sizeof(double));
  for (int i = 0; i < l->nfield; ++i) all[i] = l->field_Dl[i];
  for (int i = 0; i < l->nmain; ++i) all[l->nfield + i] = l->main_Dl[i];
  for (int i = 0; i < n; ++i) index[i] = i;
  for (int i = 1; i < n; ++i) { /* stable insertion sort of the indexes by Dl */
    int k = index[i], j = i - 1;
    while (j >= 0 && all[index[j]] > all[k]) { index[j + 1] = index[j]; --j; }
    index[j + 1] = k;
  }
  for (int i = 0; i < n; ++i) l->Dl[i] = all[index[i]];
  for (int i = 1; i < n; ++i)
    if ((l->Dl[i] - l->Dl[i - 1]) < ORC_MIN_PLANE_DIST) l->Dl[i] = l->Dl[i - 1] + ORC_MIN_PLANE_DIST;
  for (int i = 0; i < n; ++i) {
    int k = index[i];
    l->planes[i] = k < l->nfield ? &l->field[k] : &l->main[k - l->nfield];
    l->plane_z[i] = l->planes[i]->z;
  }
  free(index);
  free(all);
  if (n > 0 && l->zsource <= l->plane_z[n - 1]) l->zsource = l->plane_z[n - 1] + 0.1;
  l->plane_z[n] = l->zsource;
  l->Dl[n] = orc_coordist2(0, l->zsource);
  l->dDl[0] = l->Dl[0];
  for (int i = 1; i <= n; ++i) l->dDl[i] = l->Dl[i] - l->Dl[i - 1];
}

orc_lens *orc_lens_create(double zsource) {
  orc_lens *l = (orc_lens *)calloc(1, sizeof(orc_lens));
  l->zsource = zsource;
  l->charge = 4 * ORC_PI * ORC_GRAV; /* lens.cpp:93 */
  combine_planes(l);
  return l;
}

void orc_lens_free(orc_lens *l) {
  if (!l) return;
  for (int i = 0; i < l->nhalos; ++i) orc_halo_free(l->owned[i]);
  for (int i = 0; i < l->nmain; ++i) free(l->main[i].halos);
  for (int i = 0; i < l->nfield; ++i) free(l->field[i].halos);
  free(l->owned); free(l->main); free(l->main_Dl); free(l->field); free(l->field_Dl);
  free(l->planes); free(l->plane_z); free(l->Dl); free(l->dDl);
  free(l);
}

static void plane_push(orc_plane *p, orc_halo *h) {
  if (p->nh == p->cap) {
    p->cap = p->cap ? 2 * p->cap : 4;
    p->halos = (orc_halo **)realloc(p->halos, p->cap * sizeof(orc_halo *));
  }
  p->halos[p->nh++] = h;
}

static void insert_plane(orc_lens *l, int i, double z, double Dl, orc_halo *h) {
  l->main = (orc_plane *)realloc(l->main, (l->nmain + 1) * sizeof(orc_plane));
  l->main_Dl = (double *)realloc(l->main_Dl, (l->nmain + 1) * sizeof(double));
  memmove(&l->main[i + 1], &l->main[i], (l->nmain - i) * sizeof(orc_plane));
  memmove(&l->main_Dl[i + 1], &l->main_Dl[i], (l->nmain - i) * sizeof(double));
  memset(&l->main[i], 0, sizeof(orc_plane));
  l->main[i].z = z;
  l->main_Dl[i] = Dl;
  plane_push(&l->main[i], h);
  l->nmain++;
}

/* Lens::addMainHaloToPlane, lens.cpp:772-815 and addMainHaloToNearestPlane,
 * lens.cpp:821-838; halo->setZlensDist(plane z) gives Dist = angDist. */
void orc_lens_add_halo(orc_lens *l, orc_halo *h, int addplanes) {
  l->owned = (orc_halo **)realloc(l->owned, (l->nhalos + 1) * sizeof(orc_halo *));
  l->owned[l->nhalos++] = h;
  double hz = h->zlens, hD = orc_coordist2(0, hz);
  if (addplanes) {
    int i = 0;
    while (i < l->nmain && !(hD < l->main_Dl[i])) ++i; /* upper_bound */
    if (i > 0 && (hD - l->main_Dl[i - 1]) < ORC_MIN_PLANE_DIST) {
      plane_push(&l->main[i - 1], h);
      h->zlens = l->main[i - 1].z;
      h->Dist = orc_angdist(h->zlens);
    } else if (i == l->nmain) {
      insert_plane(l, i, hz, hD, h);
    } else if ((l->main_Dl[i] - hD) < ORC_MIN_PLANE_DIST) {
      plane_push(&l->main[i], h);
      h->zlens = l->main[i].z;
      h->Dist = orc_angdist(h->zlens);
    } else {
      insert_plane(l, i, hz, hD, h);
      h->Dist = orc_angdist(hz);
    }
  } else {
    if (l->nmain == 0) insert_plane(l, 0, hz, hD, h);
    else {
      int best = 0;
      for (int i = 1; i < l->nmain; ++i)
        if (fabs(l->main_Dl[i] - hD) < fabs(l->main_Dl[best] - hD)) best = i;
      plane_push(&l->main[best], h);
      h->zlens = l->main[best].z;
      h->Dist = orc_angdist(h->zlens);
    }
  }
  combine_planes(l);
}

/* A LensPlaneTree as one of the lens's field planes (Lens::createFieldPlanes,
 * MultiPlane/lens.cpp:443-452; field_Dl = coorDist(z)); the lens takes
 * ownership of the plane. */
void orc_lens_add_field_plane(orc_lens *l, orc_halo *plane) {
  l->owned = (orc_halo **)realloc(l->owned, (l->nhalos + 1) * sizeof(orc_halo *));
  l->owned[l->nhalos++] = plane;
  l->field = (orc_plane *)realloc(l->field, (l->nfield + 1) * sizeof(orc_plane));
  l->field_Dl = (double *)realloc(l->field_Dl, (l->nfield + 1) * sizeof(double));
  memset(&l->field[l->nfield], 0, sizeof(orc_plane));
  l->field[l->nfield].z = plane->zlens;
  l->field_Dl[l->nfield] = orc_coordist2(0, plane->zlens);
  plane_push(&l->field[l->nfield], plane);
  l->nfield++;
  combine_planes(l);
}

int orc_lens_nplanes(const orc_lens *l) { return l->np; }
void orc_lens_planes(const orc_lens *l, double *z, double *Dl, double *dDl) {
  for (int i = 0; i <= l->np; ++i) {
    z[i] = l->plane_z[i];
    Dl[i] = l->Dl[i];
    dDl[i] = l->dDl[i];
  }
}

/* Lens::ResetSourcePlane, lens.cpp:2609-2657 */
int orc_lens_reset_source(orc_lens *l, double z, int nearest) {
  l->toggle_source_plane = 1;
  if (z <= 0.0) return 0;
  double Ds = orc_coordist2(0, z);
  long j;
  if (l->np + 1 > 1) {
    /* locateD(Dl-1, nplanes, Ds, &j): xx[1..n] = Dl[0..n-1] */
    unsigned long n = (unsigned long)l->np, ju = n + 1, jl = 0, jm;
    const double *xx = l->Dl - 1;
    while (ju - jl > 1) { jm = (ju + jl) >> 1; if (Ds >= xx[jm]) jl = jm; else ju = jm; }
    if (Ds == xx[1]) j = 1; else if (Ds == xx[n]) j = (long)n - 1; else j = (long)jl;
  } else
    j = 0;
  if (j > 0) {
    if (l->Dl[j - 1] == Ds) --j;
    else if (nearest) {
      double z1 = orc_invcoordist(l->Dl[j] - 0.5 * l->dDl[j]);
      if (z < z1) --j;
    }
  }
  if (nearest && (j < l->np)) l->zs_implant = l->plane_z[j];
  else l->zs_implant = z;
  return (int)j;
}

/* Lens::FindSourcePlane, lens.cpp:2659-2680 */
static void find_source_plane(const orc_lens *l, double zs, long *jmax, double *Dls, double *Ds) {
  *Ds = orc_coordist(zs);
  if (zs <= l->plane_z[0]) { *jmax = 0; *Dls = *Ds; return; }
  *jmax = l->np; /* plane_redshifts.size() - 1 */
  if (*jmax <= 0) { *Dls = *Ds; return; }
  while (l->plane_z[*jmax - 1] > zs) --(*jmax);
  *Dls = orc_coordist2(l->plane_z[*jmax - 1], zs);
}

/* LensPlaneSingular::force, MultiPlane/planes.cpp:114-161 */
static void plane_force(orc_plane *p, const double *xx, double *alpha, double *kappa,
                        double *gamma, double *phi) {
  alpha[0] = alpha[1] = 0.0;
  *kappa = 0.0;
  gamma[0] = gamma[1] = gamma[2] = 0.0;
  *phi = 0.0;
  for (int i = 0; i < p->nh; ++i) {
    orc_halo *h = p->halos[i];
    double at[2] = {0, 0}, kt = 0, gt[3] = {0, 0, 0}, pt = 0, xt[2];
    xt[0] = xx[0] - h->posHalo[0] * h->Dist; /* LensHalo::getX, lens_halos.h:95-99 */
    xt[1] = xx[1] - h->posHalo[1] * h->Dist;
    halo_force_one(h, xt, at, &kt, gt, &pt);
    if (h->kind == ORC_FIELD) { /* LensPlaneTree::force: the tree's alpha as it is */
      alpha[0] += at[0];
      alpha[1] += at[1];
    } else {
      alpha[0] -= at[0];
      alpha[1] -= at[1];
    }
    *kappa += kt;
    gamma[0] += gt[0];
    gamma[1] += gt[1];
    gamma[2] += gt[2];
    *phi += pt;
  }
}

void orc_lens_plane_force(orc_lens *l, int j, size_t n, const double *xx, double *alpha,
                          double *kappa, double *gamma, double *phi) {
  for (size_t i = 0; i < n; ++i) {
    double a[2], k, g[3], p;
    plane_force(l->planes[j], xx + 2 * i, a, &k, g, &p);
    alpha[2 * i] = a[0]; alpha[2 * i + 1] = a[1];
    kappa[i] = k;
    gamma[3 * i] = g[0]; gamma[3 * i + 1] = g[1]; gamma[3 * i + 2] = g[2];
    phi[i] = p;
  }
}

/* Lens::compute_points_parallel, include/lens.h:913-1103, one ray. */
static void shoot_one(orc_lens *l, const double *x, long jmax, double Dls_Ds, double D_Ds,
                      double *y, double *A) {
  double theta[2] = {x[0], x[1]};
  double spa[2] = {theta[0], theta[1]};
  double sag[4] = {1, 0, 0, 1}, a[4] = {1, 0, 0, 1};
  double alpha[2], kappa, gamma[3], phi, G[4], aa, bb, xx[2];
  for (long j = 0; j < jmax; ++j) {
    double Dphysical = l->Dl[j] / (1 + l->plane_z[j]);
    xx[0] = theta[0] * Dphysical;
    xx[1] = theta[1] * Dphysical;
    plane_force(l->planes[j], xx, alpha, &kappa, gamma, &phi);
    G[0] = kappa + gamma[0]; G[1] = gamma[1];
    G[2] = gamma[1];         G[3] = kappa - gamma[0];
    double fac = l->charge * l->Dl[j] / (1 + l->plane_z[j]);
    for (int k = 0; k < 4; ++k) G[k] *= fac;
    spa[0] -= l->charge * alpha[0];
    spa[1] -= l->charge * alpha[1];
    if (j < jmax - 1) {
      aa = l->dDl[j + 1] / l->Dl[j + 1];
      bb = l->Dl[j] / l->Dl[j + 1];
    } else {
      aa = Dls_Ds;
      bb = D_Ds;
    }
    theta[0] = bb * theta[0] + aa * spa[0];
    theta[1] = bb * theta[1] + aa * spa[1];
    /* SumPrevAG -= G * A  (Matrix2x2 product, include/point.h:249-258) */
    double GA[4] = {G[0] * a[0] + G[1] * a[2], G[0] * a[1] + G[1] * a[3],
                    G[2] * a[0] + G[3] * a[2], G[2] * a[1] + G[3] * a[3]};
    for (int k = 0; k < 4; ++k) sag[k] -= GA[k];
    for (int k = 0; k < 4; ++k) a[k] = a[k] * bb + sag[k] * aa;
  }
  y[0] = theta[0];
  y[1] = theta[1];
  for (int k = 0; k < 4; ++k) A[k] = a[k];
}

typedef struct {
  orc_lens *l;
  size_t start, end;
  const double *x, *zs;
  double *y, *A;
  long jmax;
  double Dls_Ds, D_Ds;
} shoot_job;

static void *shoot_worker(void *arg) {
  shoot_job *jb = (shoot_job *)arg;
  for (size_t i = jb->start; i < jb->end; ++i) {
    long jmax = jb->jmax;
    double Dls_Ds = jb->Dls_Ds, D_Ds = jb->D_Ds;
    if (jb->zs) {
      double Dls, Ds;
      find_source_plane(jb->l, jb->zs[i], &jmax, &Dls, &Ds);
      Dls_Ds = Dls / Ds;
      if (jmax > 0) D_Ds = jb->l->Dl[jmax - 1] / Ds;
    }
    shoot_one(jb->l, jb->x + 2 * i, jmax, Dls_Ds, D_Ds, jb->y + 2 * i, jb->A + 4 * i);
  }
  return NULL;
}

void orc_lens_rayshoot(orc_lens *l, size_t n, const double *x, const double *zs, double *y,
                       double *A, int threads) {
  if (l->np == 0) { /* no lens plane, internal_rayshooter_multi.cpp:62-76 */
    for (size_t i = 0; i < n; ++i) {
      y[2 * i] = x[2 * i]; y[2 * i + 1] = x[2 * i + 1];
      A[4 * i] = 1; A[4 * i + 1] = 0; A[4 * i + 2] = 0; A[4 * i + 3] = 1;
    }
    return;
  }
  if (n == 0) return;
  long jmax = l->np;
  double Dls_Ds = 0, D_Ds = 0;
  if (!zs) {
    double source_z = l->toggle_source_plane ? l->zs_implant : l->plane_z[l->np];
    if (source_z == l->plane_z[l->np]) {
      Dls_Ds = l->dDl[l->np] / l->Dl[l->np];
      D_Ds = l->Dl[l->np - 1] / l->Dl[l->np];
    } else {
      double Dls, Ds;
      find_source_plane(l, source_z, &jmax, &Dls, &Ds);
      Dls_Ds = Dls / Ds;
      if (jmax > 0) D_Ds = l->Dl[jmax - 1] / Ds;
    }
  }
  if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if ((size_t)threads > n) threads = (int)n;
  pthread_t *th = (pthread_t *)malloc(threads * sizeof(pthread_t));
  shoot_job *jobs = (shoot_job *)malloc(threads * sizeof(shoot_job));
  size_t chunk = n / threads;
  for (int t = 0; t < threads; ++t) {
    shoot_job *jb = &jobs[t];
    jb->l = l; jb->x = x; jb->zs = zs; jb->y = y; jb->A = A;
    jb->jmax = jmax; jb->Dls_Ds = Dls_Ds; jb->D_Ds = D_Ds;
    jb->start = t * chunk;
    jb->end = (t == threads - 1) ? n : (t + 1) * chunk;
    pthread_create(&th[t], NULL, shoot_worker, jb);
  }
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  free(th);
  free(jobs);
}

/* GridMap::to_refine (TreeCode_link/gridmap.cpp:248-258).  The neighbour
 * range is MAX<size_t>(i-1, 0) .. MIN<size_t>(i+2, N): for i = 0 (or j = 0)
 * i - 1 wraps to the largest size_t, so pixels of the first row and column
 * never refine. */
static int to_refine(const double *sb, long i, long j, long N, double total, double f) {
  double flux = sb[i + j * N];
  size_t i0 = (size_t)(i - 1), j0 = (size_t)(j - 1); /* MAX<size_t>(., 0) is the identity */
  size_t i1 = (size_t)(i + 2) < (size_t)N ? (size_t)(i + 2) : (size_t)N;
  size_t j1 = (size_t)(j + 2) < (size_t)N ? (size_t)(j + 2) : (size_t)N;
  for (size_t ii = i0; ii < i1; ++ii)
    for (size_t jj = j0; jj < j1; ++jj)
      if (fabs(flux - sb[ii + jj * N]) / total > f) return 1;
  return 0;
}

/* The refinement of one pixel (gridmap.cpp:205-234): rays on an n x n
 * sub-grid of the pixel, n = 3, 9, 27, ..., until the mean surface brightness
 * changes by less than 1e-3; at most ORC_MAX_REFINE levels.  The sub-grid is
 * laid around the pixel's SOURCE position (`*(i_points[k].image)`), as the
 * reference does. */
#define ORC_MAX_REFINE 6
double orc_refine_pixel(orc_lens *l, const double *ysrc, double resolution, double sb0, int kind, const double *p) {
  double ll[2] = {ysrc[0] - resolution / 2, ysrc[1] - resolution / 2};
  double new_flux = sb0, old_flux = 0;
  int n = 1;
  for (int level = 0; level < ORC_MAX_REFINE && fabs(old_flux - new_flux) > 1.0e-3 * new_flux; ++level) {
    old_flux = new_flux;
    n *= 3;
    double res = resolution / n;
    size_t m = (size_t)n * n;
    double *x = (double *)malloc(2 * m * sizeof(double)), *y = (double *)malloc(2 * m * sizeof(double));
    double *A = (double *)malloc(4 * m * sizeof(double)), *sb = (double *)malloc(m * sizeof(double));
    for (int u = 0; u < n; ++u)
      for (int v = 0; v < n; ++v) {
        x[2 * ((size_t)u * n + v)] = ll[0] + (0.5 + u) * res;
        x[2 * ((size_t)u * n + v) + 1] = ll[1] + (0.5 + v) * res;
      }
    orc_lens_rayshoot(l, m, x, NULL, y, A, 0);
    orc_source_sb(kind, p, m, y, sb);
    new_flux = 0;
    for (size_t k = 0; k < m; ++k) new_flux += sb[k];
    new_flux /= n * n;
    free(x); free(y); free(A); free(sb);
  }
  return new_flux;
}

/* GridMap::AdaptiveRefreshSurfaceBrightnesses (gridmap.cpp:189-246) for a grid
 * of N1d x N1d rays: sb gets the final per-pixel surface brightness (GridMap
 * order); returns the total flux (sum x resolution^2). */
double orc_gridmap_adaptive_sb(orc_lens *l, size_t N1d, const double *center, double range, int kind,
                               const double *p, double *sb) {
  const double f = 1.0e-4;
  size_t n = N1d * N1d;
  double resolution = range / (N1d - 1);
  double *x = (double *)malloc(2 * n * sizeof(double)), *y = (double *)malloc(2 * n * sizeof(double));
  double *A = (double *)malloc(4 * n * sizeof(double));
  orc_grid_positions(N1d, center, range, x);
  orc_lens_rayshoot(l, n, x, NULL, y, A, 0);
  orc_source_sb(kind, p, n, y, sb);
  double total = 0, res2 = pow(resolution, 2);
  for (size_t i = 0; i < n; ++i) total += sb[i] * res2; /* RefreshSurfaceBrightnesses */
  double total_flux = total / resolution / resolution;
  if (total_flux == 0) { free(x); free(y); free(A); return 0; }
  for (long j = 0; j < (long)N1d; ++j) {
    size_t k = j * N1d;
    for (long i = 0; i < (long)N1d; ++i, ++k) {
      if (to_refine(sb, i, j, (long)N1d, total_flux, f)) {
        double new_flux = orc_refine_pixel(l, &y[2 * k], resolution, sb[k], kind, p);
        total_flux -= sb[k];
        sb[k] = new_flux;
        total_flux += new_flux;
      }
    }
  }
  free(x); free(y); free(A);
  return total_flux * resolution * resolution;
}

void orc_grid_positions(size_t N1d, const double *center, double range, double *x) {
  for (size_t i = 0; i < N1d * N1d; ++i) {
    if (N1d == 1) {
      x[2 * i] = center[0];
      x[2 * i + 1] = center[1];
      continue;
    }
    x[2 * i] = center[0] + range * (1.0 * (i % N1d) / (N1d - 1) - 0.5);
    x[2 * i + 1] = center[1] + range * (1.0 * (i / N1d) / (N1d - 1) - 0.5);
  }
}

/* ================ adaptive kNN smoothing (calculate_smoothing) ========== */
/* LensHaloParticles::calculate_smoothing (include/particle_halo.h:683-730)
 * builds TreeSimple(pp, N, 2*Nsmooth, 3, median=true) and sets every
 * particle's Size to NNDistance(x_i, Nsmooth+1).
 *
 * The tree (include/simpleTree.h:842-974, 1318-1364): a node holding more than
 * `bucket` particles sorts them on coordinate level%3; child 1 takes the first
 * n/2 and child 2 the rest; both inherit the parent's box except that child
 * 1's upper and child 2's lower bound on that axis become the coordinate of
 * the first particle of child 2.  brother links: child1 -> child2 ->
 * parent's brother.
 *
 * NNDistance (simpleTree.h:483-618): descend by value to a leaf (_findleaf,
 * :625-640: child 1 when its upper bound > x[d]); climb while the node holds
 * fewer than Nneighbors particles (that node is `pass`); fill a max-heap with
 * the Nneighbors smallest squared distances of pass's particles; then walk
 * the whole tree in preorder from the top, skipping pass's subtree and any
 * node whose box misses the interval x[dim] +- bestr on the axis its parent
 * cut (dim = (level-1)%3), and push every leaf particle with r2 < bestr^2
 * (bestr = sqrt(heap top) after every push/pop).  The result is the exact
 * Nneighbors-th smallest distance, except when pass is the top node: then
 * the walk visits leaves whose particles are already in the heap and counts
 * them twice (happens only for N = 2*Nsmooth+1).  Squared distances are
 * summed in double from float coordinate differences; the result is float.
 * The reference sorts with std::sort; this restatement sorts stably, which
 * matters only for particles with equal coordinates. */
typedef struct {
  size_t start, n;
  double p1[3], p2[3];
  int level, child1, child2, parent, brother;
} knn_node;

typedef struct {
  knn_node *v;
  int nn, cap;
  unsigned *perm;
  const orc_particle *p;
  unsigned *tmp;
  int bucket;
} knn_tree;

static void knn_stable_sort(knn_tree *t, size_t start, size_t n, int d) {
  /* bottom-up merge sort of perm[start, start+n) by p[.].x[d] */
  unsigned *a = t->perm + start, *b = t->tmp;
  for (size_t w = 1; w < n; w *= 2) {
    for (size_t lo = 0; lo < n; lo += 2 * w) {
      size_t mid = lo + w < n ? lo + w : n, hi = lo + 2 * w < n ? lo + 2 * w : n;
      size_t i = lo, j = mid, k = lo;
      while (i < mid && j < hi)
        b[k++] = (t->p[a[j]].x[d] < t->p[a[i]].x[d]) ? a[j++] : a[i++];
      while (i < mid) b[k++] = a[i++];
      while (j < hi) b[k++] = a[j++];
    }
    memcpy(a, b, n * sizeof(unsigned));
  }
}

static int knn_new(knn_tree *t, size_t start, size_t n, int level, int parent,
                   const double *p1, const double *p2) {
  if (t->nn == t->cap) {
    t->cap = t->cap ? 2 * t->cap : 1024;
    t->v = (knn_node *)realloc(t->v, (size_t)t->cap * sizeof(knn_node));
  }
  int id = t->nn++;
  knn_node *nd = &t->v[id];
  nd->start = start;
  nd->n = n;
  nd->level = level;
  nd->parent = parent;
  nd->child1 = nd->child2 = nd->brother = -1;
  memcpy(nd->p1, p1, sizeof nd->p1);
  memcpy(nd->p2, p2, sizeof nd->p2);
  return id;
}

/* _BuildTreeNB (simpleTree.h:882-974) */
static void knn_build(knn_tree *t, int id) {
  size_t start = t->v[id].start, n = t->v[id].n;
  if (n <= (size_t)t->bucket) return;
  int level = t->v[id].level, d = level % 3;
  knn_stable_sort(t, start, n, d);
  size_t cut = n / 2;
  double xc = t->p[t->perm[start + cut]].x[d];
  double a1[3], a2[3], b1[3], b2[3];
  memcpy(a1, t->v[id].p1, sizeof a1);
  memcpy(a2, t->v[id].p2, sizeof a2);
  memcpy(b1, t->v[id].p1, sizeof b1);
  memcpy(b2, t->v[id].p2, sizeof b2);
  a2[d] = xc;
  b1[d] = xc;
  int c1 = knn_new(t, start, cut, level + 1, id, a1, a2);
  int c2 = knn_new(t, start + cut, n - cut, level + 1, id, b1, b2);
  t->v[id].child1 = c1;
  t->v[id].child2 = c2;
  t->v[c1].brother = c2;
  t->v[c2].brother = t->v[id].brother;
  knn_build(t, c1);
  knn_build(t, c2);
}

/* std::priority_queue<double> (a max-heap): the walk only ever reads the top */
typedef struct {
  double *h;
  size_t n;
} knn_heap;

static void heap_push(knn_heap *q, double v) {
  size_t i = q->n++;
  while (i > 0) {
    size_t up = (i - 1) / 2;
    if (q->h[up] >= v) break;
    q->h[i] = q->h[up];
    i = up;
  }
  q->h[i] = v;
}

static void heap_pop(knn_heap *q) {
  double v = q->h[--q->n];
  size_t i = 0;
  for (;;) {
    size_t c = 2 * i + 1;
    if (c >= q->n) break;
    if (c + 1 < q->n && q->h[c + 1] > q->h[c]) ++c;
    if (q->h[c] <= v) break;
    q->h[i] = q->h[c];
    i = c;
  }
  if (q->n) q->h[i] = v;
}

static double knn_r2(const float *a, const float *ray) {
  double s = 0.0;
  for (int k = 0; k < 3; ++k) {
    float dx = a[k] - ray[k];
    s += (double)dx * (double)dx;
  }
  return s;
}

/* TreeSimple::iterator::walk (simpleTree.h:131-146); top's brother is -1 */
static int knn_walk(const knn_tree *t, int *cur, int decend) {
  const knn_node *c = &t->v[*cur];
  if (decend && c->child1 >= 0) { *cur = c->child1; return 1; }
  if (decend && c->child2 >= 0) { *cur = c->child2; return 1; }
  if (c->brother == -1) return 0;
  *cur = c->brother;
  return 1;
}

static float knn_nndistance(const knn_tree *t, const float *ray, size_t K, knn_heap *q) {
  int id = 0;
  while (t->v[id].child1 >= 0 || t->v[id].child2 >= 0) {
    int d = t->v[id].level % 3;
    id = (t->v[t->v[id].child1].p2[d] > (double)ray[d]) ? t->v[id].child1 : t->v[id].child2;
  }
  while (t->v[id].n < K) id = t->v[id].parent;
  const int pass = id;
  const knn_node *pn = &t->v[pass];
  q->n = 0;
  size_t i = 0;
  for (; i < K; ++i) heap_push(q, knn_r2(t->p[t->perm[pn->start + i]].x, ray));
  for (; i < pn->n; ++i) {
    double r2 = knn_r2(t->p[t->perm[pn->start + i]].x, ray);
    if (r2 < q->h[0]) {
      heap_push(q, r2);
      heap_pop(q);
    }
  }
  double bestr = sqrt(q->h[0]);
  int cur = 0, decend = 1;
  knn_walk(t, &cur, 1);
  do {
    if (cur == pass) {
      decend = 0;
    } else {
      const knn_node *cb = &t->v[cur];
      int dim = (cb->level - 1) % 3;
      if ((ray[dim] + bestr) > cb->p1[dim] && (ray[dim] - bestr) < cb->p2[dim]) {
        decend = 1;
        if (cb->child1 < 0 && cb->child2 < 0) {
          for (size_t j = 0; j < cb->n; ++j) {
            double r2 = knn_r2(t->p[t->perm[cb->start + j]].x, ray);
            if (r2 < bestr * bestr) {
              heap_push(q, r2);
              heap_pop(q);
              bestr = sqrt(q->h[0]);
            }
          }
        }
      } else {
        decend = 0;
      }
    }
  } while (knn_walk(t, &cur, decend));
  return (float)bestr;
}

int orc_calculate_smoothing(orc_particle *p, size_t n, int nsmooth) {
  if (nsmooth < 1) return -1;
  if (n <= (size_t)nsmooth + 1) return -1; /* simpleTree.h:488-492 */
  knn_tree t;
  memset(&t, 0, sizeof t);
  t.p = p;
  t.bucket = 2 * nsmooth;
  t.perm = (unsigned *)malloc(n * sizeof(unsigned));
  t.tmp = (unsigned *)malloc(n * sizeof(unsigned));
  for (size_t i = 0; i < n; ++i) t.perm[i] = (unsigned)i;
  double p1[3], p2[3];
  for (int k = 0; k < 3; ++k) p1[k] = p2[k] = p[0].x[k];
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      if (p[i].x[k] < p1[k]) p1[k] = p[i].x[k];
      if (p[i].x[k] > p2[k]) p2[k] = p[i].x[k];
    }
  knn_new(&t, 0, n, 0, -1, p1, p2);
  knn_build(&t, 0);
  const size_t K = (size_t)nsmooth + 1;
  knn_heap q;
  q.h = (double *)malloc((K + 1) * sizeof(double));
  float *out = (float *)malloc(n * sizeof(float));
  for (size_t i = 0; i < n; ++i) out[i] = knn_nndistance(&t, p[i].x, K, &q);
  for (size_t i = 0; i < n; ++i) p[i].Size = out[i];
  free(out);
  free(q.h);
  free(t.v);
  free(t.perm);
  free(t.tmp);
  return 0;
}
