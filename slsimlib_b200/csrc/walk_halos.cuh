// Warp-cooperative walk of a field plane's halo tree:
// TreeQuadHalos::force2D / walkTree_iter (include/quadTreeHalos.h:556-815).
//
// The 32 lanes of a warp walk the preorder branch array together, each with
// its own decisions (a lane that uses a cell whole records `resume = skip`).
// At every branch a lane visits, the branch's big haloes are evaluated in
// full (analytic profile + the sigma_background sheet); at an internal branch
// the cell is then used whole (monopole + quadrupole, screened, with the
// sheet) when the lane is beyond the cell's critical radius, and the walk
// descends where any lane is not.  Every lane therefore adds exactly the
// reference's terms in the reference's order.  The arithmetic is FP64 in
// every precision form: field planes hold few haloes next to a particle
// plane's millions of particles.
#pragma once
#include "halos.cuh"
#include "walk.cuh"

namespace glb {

struct Force6 {
  double a0, a1, k, g0, g1, phi;
};

// LensHalo::force_halo of one member halo at xcm (accumulated from zero); the
// screening factor the reference passes reaches only the point-mass
// subtraction, which the tree never requests (lens_halos.cpp:1555-1598).
template <bool PHI>
__device__ __noinline__ Force6 field_member_force(const FieldHaloDev *H, const NFWTables *tab, double x0,
                                                   double x1) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (H->kind == HALO_NFW)
    nfw_force<PHI>(H->nfw, *tab, x0, x1, acc);
  else
    nsie_force<PHI>(H->nsie, x0, x1, acc);
  return Force6{acc[0], acc[1], acc[2], acc[3], acc[4], acc[5]};
}

template <bool PHI>
__device__ __forceinline__ void walk_halos(const HaloTreeDev &T, const NFWTables &tab, double rx, double ry,
                                           bool valid, double *acc) {
  int resume = valid ? 0 : 0x7fffffff;
  int node = 0;
  const int nn = T.nnodes;
  while (node < nn) {
    const HNode *nd = T.nodes + node;
    const int skip = max(nd->skip, node + 1);  // forward progress even on a malformed array
    const bool act = node >= resume;
    // big haloes of the branch (all haloes of a leaf), include/quadTreeHalos.h:663-689
    const int b0 = nd->bstart, b1 = b0 + nd->bcount;
    for (int b = b0; b < b1; ++b) {
      if (!act) continue;
      const FieldHaloDev *H = T.halos + __ldg(T.bigs + b);
      const double x0 = H->px - rx, x1 = H->py - ry;
      const double rcm2 = x0 * x0 + x1 * x1;
      const Force6 f = field_member_force<PHI>(H, &tab, x0, x1);
      acc[0] += f.a0;
      acc[1] += f.a1;
      acc[2] += f.k;
      acc[3] += f.g0;
      acc[4] += f.g1;
      if (PHI) acc[5] += f.phi;
      const double prefac = H->mass * T.inv_area;
      acc[0] += prefac * x0;
      acc[1] += prefac * x1;
      if (PHI) acc[5] += -T.inv_area * rcm2 * H->mass * 0.5;
      acc[2] -= H->mass * T.inv_area;
    }
    bool open = false;
    if (!nd->leaf) {
      // the whole cell, include/quadTreeHalos.h:691-741
      const double xc0 = nd->cx - rx, xc1 = nd->cy - ry;
      const double r2 = xc0 * xc0 + xc1 * xc1;
      const bool far = act && r2 > nd->r2crit;
      open = act && !far;
      if (far) {
        const double mass = nd->mass, q0 = nd->q0, q1 = nd->q1, q2 = nd->q2;
        const double scr = exp(-r2 * T.screen2);
        double tmp = mass * (T.inv_area - scr / r2 / kPi);
        acc[0] += tmp * xc0;
        acc[1] += tmp * xc1;
        tmp = -2.0 * mass / kPi / r2 / r2 * scr;
        acc[3] += 0.5 * (xc0 * xc0 - xc1 * xc1) * tmp;
        acc[4] += xc0 * xc1 * tmp;
        if (PHI) {
          acc[5] += 0.5 * mass * log(r2) / kPi * scr;
          acc[5] -= 0.5 * (q0 * xc0 * xc0 + q1 * xc1 * xc1 + 2 * q2 * xc0 * xc1) / (kPi * r2 * r2) * scr;
        }
        acc[0] -= (q0 * xc0 + q2 * xc1) / (r2 * r2) / kPi * scr;
        acc[1] -= (q1 * xc1 + q2 * xc0) / (r2 * r2) / kPi * scr;
        tmp = 4 * (q0 * xc0 * xc0 + q1 * xc1 * xc1 + 2 * q2 * xc0 * xc1) / (r2 * r2 * r2) / kPi * scr;
        acc[0] += tmp * xc0;
        acc[1] += tmp * xc1;
        acc[2] -= mass * T.inv_area;
        if (PHI) acc[5] -= mass * T.inv_area * r2;
        resume = skip;
      }
    }
    node = __any_sync(kFull, open) ? node + 1 : skip;
  }
}

// TreeQuadHalos::force2D (include/quadTreeHalos.h:556-592): outputs start from
// zero; with a periodic buffer the walk is repeated for eight shifted copies.
template <bool PHI>
__device__ __forceinline__ void field_plane_acc(const HaloTreeDev &T, const NFWTables &tab, double rx, double ry,
                                                bool valid, double *acc) {
  if (T.nnodes == 0) return;
  if (T.periodic) {
    for (int i = -1; i < 2; ++i)
      for (int j = -1; j < 2; ++j) walk_halos<PHI>(T, tab, rx + i * T.period_x, ry + j * T.period_y, valid, acc);
  } else {
    walk_halos<PHI>(T, tab, rx, ry, valid, acc);
  }
}

// The same, out of line and returning by value: the plane kernels call it
// so that the halo-tree walk adds nothing to the register budget (or the
// local-memory traffic) of the particle-tree walk beside it.
template <bool PHI>
__device__ __noinline__ Force6 field_plane_force(const HaloTreeDev *T, const NFWTables *tab, double rx, double ry,
                                                 bool valid) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  field_plane_acc<PHI>(*T, *tab, rx, ry, valid, acc);
  return Force6{acc[0], acc[1], acc[2], acc[3], acc[4], acc[5]};
}

}  // namespace glb
