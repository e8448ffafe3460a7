// Warp-cooperative quadtree walk (TreeQuadParticles::walkTree_recur,
// include/quadTree.h:990-1128).
//
// The 32 lanes of a warp hold 32 (spatially sorted) rays and advance through
// the preorder node array together, so every node, particle and big-particle
// record is fetched once per warp and broadcast.  Each lane still takes its
// own opening decision: a lane that accepts a cell as a far-field term records
// `resume = node.skip` and sits out the cell's subtree; the warp descends
// into a cell whenever any active lane opens it (warp vote) and jumps over it
// when none does.  The set of interactions per ray is therefore exactly the
// reference's.
#pragma once
#include "glb_internal.h"

namespace glb {

constexpr unsigned kFull = 0xffffffffu;

// Interaction counts of one ray's walk, for the algorithmic-flop roofline:
// V nodes tested, F far-field cells, P leaf point masses, B big-particle
// distance checks, S B-spline corrections applied.
// Wn / Wp count the warp's node-loop and leaf-particle-loop iterations (the
// union over its 32 rays), for the lane-efficiency of the warp-cooperative walk.
struct WalkCount {
  unsigned long long V = 0, F = 0, P = 0, B = 0, S = 0, Wn = 0, Wp = 0;
};

// b_spline_profile, include/quadTree.h:147-190 (point mass subtracted).
template <bool PHI>
__device__ __forceinline__ void bspline_f64(double x0, double x1, double r, double Mass, double size,
                                   double phiintconst, double *acc) {
  double q = r / size, M, sigma;
  if (q > 2) {
    sigma = 0;
    M = 1;
  } else {
    double q2 = q * q, q3 = q2 * q, q4 = q2 * q2, q5 = q4 * q;
    sigma = (8 - 12 * q + 6 * q2 - q3) / 4;
    if (q > 1) {
      sigma *= 10 / size / size / 7 / kPi;
      M = (-1 + 20 * q2 * (1 - q + 3 * q2 / 8 - q3 / 20)) / 7;
      if (PHI)
        acc[5] += Mass * (-1232. + 1200 * q2 - 800. * q3 + 225. * q4 - 24 * q5 + 120 * log(2. / q)) / 840 / kPi;
    } else {
      sigma = 10 * (sigma - 1 + 3 * q - 3 * q2 + q3) / size / size / 7 / kPi;
      M = 10 * q2 * (1 - 3 * q / 4 + 3 * q3 / 10) / 7;
      if (PHI) acc[5] += Mass * (phiintconst + 10 * (q2 / 2 - 3 * q4 / 4 + 3 * q5 / 50) / 7) / kPi;
    }
  }
  double alpha_r = (M - 1) / kPi / r;
  double gt = alpha_r / r - sigma;
  acc[0] -= Mass * alpha_r * x0 / r;
  acc[1] -= Mass * alpha_r * x1 / r;
  acc[3] -= gt * Mass * (x0 * x0 - x1 * x1) / r / r;
  acc[4] -= gt * Mass * 2 * x0 * x1 / r / r;
  acc[2] += Mass * sigma;
  if (PHI) acc[5] -= Mass * log(r) / kPi;
}

// One warp-synchronous walk for the ray (rx, ry).  `valid` lanes take part in
// the votes but add nothing.  acc = {alpha0, alpha1, kappa, gamma0, gamma1,
// phi} accumulates in the reference's units (alpha pointing away from mass).
template <bool PHI, bool COUNT = false>
__device__ __forceinline__ void walk_f64(const TreeDev &T, double rx, double ry, bool valid, double *acc,
                                         WalkCount *wc = nullptr) {
  const double inv_pi = 1.0 / kPi;
  const bool screen = T.screen2 != 0.0;
  int resume = valid ? 0 : 0x7fffffff;
  int node = 0;
  const int nn = T.nnodes;
  while (node < nn) {
    const GNode *nd = T.nodes + node;
    const double cx = nd->cx, cy = nd->cy, open2 = nd->open2;
    const int skip = max(nd->skip, node + 1);  // forward progress even on a malformed array
    const bool act = node >= resume;
    const double dx = cx - rx, dy = cy - ry;
    const double r2 = dx * dx + dy * dy;
    const bool open = act && (r2 < open2);
    if (COUNT) wc->Wn++;
    if (COUNT && act) wc->V++;
    if (act && !open) {
      if (COUNT) wc->F++;
      // far field: monopole + quadrupole (quadTree.h:1090-1123)
      const double mass = nd->mass, q0 = nd->q0, q1 = nd->q1, q2 = nd->q2;
      const double scr = screen ? exp(-r2 * T.screen2) : 1.0;
      double tmp = mass * T.inv_area - mass / r2 * inv_pi * scr;
      acc[0] += tmp * dx;
      acc[1] += tmp * dy;
      const double ir4 = 1.0 / (r2 * r2);
      tmp = -2.0 * mass * inv_pi * ir4 * scr;
      acc[3] += 0.5 * (dx * dx - dy * dy) * tmp;
      acc[4] += dx * dy * tmp;
      if (PHI) {
        acc[5] += 0.5 * T.phi_mass * log(r2) * inv_pi * scr;
        acc[5] -= 0.5 * (T.phi_q0 * dx * dx + T.phi_q1 * dy * dy + 2 * T.phi_q2 * dx * dy) * inv_pi * ir4 * scr;
      }
      acc[0] -= (q0 * dx + q2 * dy) * ir4 * inv_pi * scr;
      acc[1] -= (q1 * dy + q2 * dx) * ir4 * inv_pi * scr;
      tmp = 4 * (q0 * dx * dx + q1 * dy * dy + 2 * q2 * dx * dy) * (ir4 / r2) * inv_pi * scr;
      acc[0] += tmp * dx;
      acc[1] += tmp * dy;
      acc[2] -= T.inv_area * mass;
      if (PHI) acc[5] -= 0.5 * mass * r2 * T.inv_area;
      resume = skip;
    }
    if (!__any_sync(kFull, open)) {
      node = skip;
      continue;
    }
    const bool nearc = open && (r2 < nd->near2);
    if (nd->leaf) {
      const int p0 = nd->pstart, p1 = p0 + nd->pcount;
      const double width = nd->width;
      for (int p = p0; p < p1; ++p) {
        const float4 P = __ldg(T.parts + p);
        if (COUNT) wc->Wp++;
        if (open) {
          // leaf particle as a point mass (quadTree.h:1017-1046)
          const double x0 = (double)P.x - rx, x1 = (double)P.y - ry;
          double rcm2 = x0 * x0 + x1 * x1;
          const double scr = screen ? exp(-rcm2 * T.screen2) : 1.0;
          if (rcm2 < 1e-20) rcm2 = 1e-20;
          const double m = (double)P.z;
          const double ir2 = 1.0 / rcm2;
          const double prefac = m * scr * ir2 * inv_pi;
          acc[0] += (T.inv_area * m - prefac) * x0;
          acc[1] += (T.inv_area * m - prefac) * x1;
          const double tmp = -2.0 * prefac * ir2;
          acc[3] += 0.5 * (x0 * x0 - x1 * x1) * tmp;
          acc[4] += x0 * x1 * tmp;
          acc[2] -= m * T.inv_area;
          if (PHI) acc[5] += prefac * rcm2 * 0.5 * log(rcm2) - m * T.inv_area * rcm2 / 2;
          if (COUNT) wc->P++;
          // the leaf's big particles are those smaller than the leaf (quadTree.h:384-395)
          const double size = (double)P.w;
          if (COUNT && nearc && size < width) wc->B++;
          if (nearc && size < width && rcm2 < 4 * size * size) {
            if (COUNT) wc->S++;
            bspline_f64<PHI>(x0, x1, sqrt(rcm2), m, size, T.phiintconst, acc);
          }
        }
      }
      node = skip;
    } else {
      if (__any_sync(kFull, nearc)) {
        const int b0 = nd->bstart, b1 = b0 + nd->bcount;
        for (int b = b0; b < b1; ++b) {
          const float4 P = __ldg(T.bigs + b);
          if (nearc) {
            const double x0 = (double)P.x - rx, x1 = (double)P.y - ry;
            double rcm2 = x0 * x0 + x1 * x1;
            if (rcm2 < 1e-20) rcm2 = 1e-20;
            const double size = (double)P.w;
            if (COUNT) wc->B++;
            if (rcm2 < 4 * size * size) {
              if (COUNT) wc->S++;
              bspline_f64<PHI>(x0, x1, sqrt(rcm2), (double)P.z, size, T.phiintconst, acc);
            }
          }
        }
      }
      node = node + 1;
    }
  }
}

}  // namespace glb
