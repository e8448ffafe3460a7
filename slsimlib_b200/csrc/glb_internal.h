// Device-side data layout of the ray-shooting path.
//
// Tree nodes are stored in depth-first (preorder) order with empty children
// removed, so a walk is a forward scan: opening a node moves to node + 1,
// accepting or leaving it jumps to `skip` (first node after its subtree).
// Leaf particles sit contiguously in key order; "big" particles of internal
// nodes (those whose softening exceeds half the node width,
// include/quadTree.h:403-431) are copied into a separate contiguous list.
#pragma once
#include <stddef.h>
#include <stdint.h>

#include "cosmology.h"

namespace glb {

constexpr double kPi = 3.14159265358979323846;  // include/standard.h:39 (M_PI)
constexpr double kGrav = 4.7788e-20;              // include/standard.h:43
constexpr double kLightspeed = 2.99792458e5;      // km/s
constexpr int kMaxDepth = 32;                     // 2-bit Morton digits in a 64-bit key
// Relative band around an opening threshold inside which the split-precision
// walk repeats its FP32 test in FP64 (~8x the FP32 error of the test).
constexpr float kAmbiguous = 4e-6f;

// One tree node (preorder, non-empty).  96 bytes.
struct __align__(16) GNode {
  double cx, cy;   // centre of |m|-weighted mass (quadTree.h:591-598)
  double open2;    // max(r2crit_angle, 5.83 boxsize^2): open when rcm2cell < open2
  double near2;    // 5.83 boxsize^2: big particles are tested when rcm2cell < near2
  double mass;     // signed mass
  double q0, q1, q2;  // quadrupole about the centre of mass (quadTree.h:602-612)
  double width;    // x-extent of the box (leaf big-particle test, quadTree.h:386)
  int skip;        // preorder index of the first node after this subtree
  int leaf;        // 1 for a leaf
  int pstart, pcount;  // leaf: range in the sorted particle array
  int bstart, bcount;  // internal: range in the big-particle array
};

// FP32 node of the split-precision walk (64 bytes).  The centre of mass is a
// double-float pair (hi + lo, both FP32), so that a ray offset computed as
// (cxh - rxh) + (cxl - rxl) carries FP32 relative precision however far the
// node sits from the origin.  open_band is the half-width of the band around
// open2 inside which the opening test is repeated in FP64.  Mass and
// quadrupole are stored divided by pi; the width is rounded up to FP32, so
// that for an FP32 softening length size < width_ru holds exactly when
// size < width does.  Rows 0, 1 and 3 are read by every opening test (issued
// together, so that their latencies overlap), row 2 by far-field terms and
// leaves.
struct __align__(16) GNodeS {
  float cxh, cyh, cxl, cyl;
  float open2, near2, mpi, open_band;
  float q1pi, q2pi, width_ru, q0pi;
  int skip, leaf, start, count;  // leaf: particle range; internal: big-particle range
};

struct TreeDev {
  const GNode *nodes;
  const GNodeS *snodes;
  const float4 *parts;  // sorted particles {x, y, mass, size}
  const float4 *bigs;   // big-particle list of internal nodes
  const float4 *prel;   // sorted particles {x - leaf cx, y - leaf cy, -mass/pi, near radius^2} (FP32)
  int nnodes;
  int nparticles;
  double inv_area;
  double screen2;       // inv_screening_scale^2
  int periodic;
  double period_x, period_y;  // original (unsquared) bbox lengths
  // mass and quadrupole of the last branch of the reference's moments walk,
  // read by its far-field potential (quadTree.h:1103-1104)
  double phi_mass, phi_q0, phi_q1, phi_q2;
  double phiintconst;
  // masses of one sign: the split walk adds the inv_area sheet's deflection in
  // closed form from the root's mass and centre instead of term by term
  int sheet_closed;
  double root_mass, root_cx, root_cy;
};

enum HaloKind { HALO_PARTICLES = 0, HALO_NFW = 1, HALO_NSIE = 2, HALO_FIELD = 3 };

struct NFWDev {
  double mass, rscale, gmax, Rmax2;  // Rmax2: float(Rmax*Rmax) as the reference compares
  double phi_const;                  // 0.25*h(Rsize/rscale)/gmax - log(Rsize) terms
  double h_xmax;
  double log_rsize;
};

struct NSIEDev {
  double mass, Rsize, Rmax, Rsize2, Rmax2, units;
  double f, bc, sqrt_f, fp;
  double c1, s1;    // cos/sin(pa)      (rotation into the halo frame)
  double c2, s2;    // cos/sin(-pa)     (deflection back)
  double c3, s3;    // cos/sin(-2 pa)   (shear back)
  double c0, s0;    // cos/sin(0)
  double dRmaxRsize;  // float(Rmax - Rsize)
};

// One branch of a field plane's halo tree (TreeQuadHalos, include/quadTreeHalos.h),
// preorder with empty children kept (they carry no haloes and no far field).
struct HNode {
  double cx, cy;      // mass-weighted centre of the branch's haloes (CalcMoments)
  double r2crit;      // (1.15470 rcom / theta)^2: the cell is used whole beyond it
  double mass;
  double q0, q1, q2;  // quadrupole about the centre
  int skip;           // first branch after this subtree
  int leaf;
  int bstart, bcount; // big haloes of the branch (a leaf: all of its haloes)
};

// A member halo of a field plane: its position on the plane and profile.
struct FieldHaloDev {
  int kind;          // HALO_NFW or HALO_NSIE
  double px, py;     // LensHalo::getX at the plane's redshift
  double mass;       // LensHalo::get_mass (a float member)
  NFWDev nfw;
  NSIEDev nsie;
};

// LensPlaneTree's TreeQuadHalos on the device.
struct HaloTreeDev {
  const HNode *nodes;
  const int *bigs;             // member indices, in the reference's list order
  const FieldHaloDev *halos;
  int nnodes;
  int nhalos;
  double inv_area;             // the plane's sigma_background
  double screen2;              // inv_screening_scale^2
  int periodic;
  double period_x, period_y;   // original (unsquared) bbox lengths
};

struct HaloDev {
  int kind;
  double px, py;  // posHalo * Dist (physical Mpc), LensHalo::getX
  TreeDev tree;
  NFWDev nfw;
  NSIEDev nsie;
  HaloTreeDev htree;
};

// One lens plane of the combined list, with the scalars of the recursion
// (include/lens.h:1003-1066) precomputed on the host in the reference's
// operation order.
struct PlaneDev {
  double Dphys;  // Dl[j] / (1 + z_j)
  double Gfac;   // charge * Dl[j] / (1 + z_j)
  double aa, bb; // dDl[j+1]/Dl[j+1], Dl[j]/Dl[j+1] (j < last)
  int halo0, nhalo;
};

struct NFWTables {
  const double *x, *f, *g, *g2, *h;
};

}  // namespace glb
