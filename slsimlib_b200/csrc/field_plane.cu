// Host-side build of a field plane's halo tree: TreeQuadHalos::BuildQTreeNB,
// _BuildQTreeNB and CalcMoments (include/quadTreeHalos.h:173-515), which the
// reference runs once per LensPlaneTree (MultiPlane/planes.cpp:13-18).  Field
// planes hold 10^2-10^5 haloes, so the build stays on the host and only the
// walk runs on the GPU.  The branch order, the partitions (values <= the
// pivot first, include/Tree.h:409-424), the big-halo lists and the moments'
// operation order are the reference's, so the device walk visits the same
// branches and sums the same terms.
#include <cmath>
#include <memory>
#include <utility>

#include "glb_host.h"

namespace glb {
namespace {

struct HB {  // one branch while building
  size_t *particles = nullptr;
  size_t n = 0;
  std::vector<int> big;
  double p1[2] = {0, 0}, p2[2] = {0, 0}, center[2] = {0, 0};
  double mass = 0, quad[3] = {0, 0, 0}, r2crit = 0;
  std::unique_ptr<HB> child[4];
};

void partition(double pivot, size_t *cut, size_t *particles, double *arr, size_t N) {
  size_t k = 0;
  for (size_t i = 0; i < N; ++i)
    if (arr[i] <= pivot) {
      std::swap(arr[k], arr[i]);
      std::swap(particles[k], particles[i]);
      ++k;
    }
  *cut = k;
}

struct Builder {
  const std::vector<double> &xp;
  const std::vector<float> &rmax, &mass;
  int bucket;
  double theta, max_range;
  std::vector<double> work;

  void build(HB *cb, bool at_top) {
    size_t *particles = cb->particles;
    const size_t np = cb->n;
    cb->center[0] = (cb->p1[0] + cb->p2[0]) / 2;
    cb->center[1] = (cb->p1[1] + cb->p2[1]) / 2;
    double theta_range = 2 * theta;
    if (max_range > 0) {
      double boxsize = 1.732 * (cb->p2[0] - cb->p1[0]);
      double d = std::sqrt(cb->center[0] * cb->center[0] + cb->center[1] * cb->center[1]) - max_range;
      theta_range = boxsize / (d > boxsize ? d : boxsize);
    }
    if (np <= (size_t)bucket || theta > theta_range) {  // leaf: every halo is big
      for (size_t i = 0; i < np; ++i) cb->big.push_back((int)particles[i]);
      return;
    }
    double *x = work.data();
    size_t cut = 0, cut2 = 0;
    for (size_t i = 0; i < np; ++i) x[i] = (double)rmax[particles[i]];
    const double half_box = (cb->p2[0] - cb->p1[0]) / 2;
    partition(half_box, &cut, particles, x, np);
    if (cut < np) {
      if (at_top) {
        cut2 = np - cut;
      } else {
        partition(2 * half_box, &cut2, &particles[cut], &x[cut], np - cut);
      }
      for (size_t i = cut; i < cut + cut2; ++i) cb->big.push_back((int)particles[i]);
    }
    for (int k = 0; k < 4; ++k) cb->child[k].reset(new HB);
    HB *c0 = cb->child[0].get(), *c1 = cb->child[1].get(), *c2 = cb->child[2].get(), *c3 = cb->child[3].get();
    c0->p1[0] = cb->center[0]; c0->p1[1] = cb->center[1]; c0->p2[0] = cb->p2[0]; c0->p2[1] = cb->p2[1];
    c1->p1[0] = cb->p1[0]; c1->p1[1] = cb->center[1]; c1->p2[0] = cb->center[0]; c1->p2[1] = cb->p2[1];
    c2->p1[0] = cb->center[0]; c2->p1[1] = cb->p1[1]; c2->p2[0] = cb->p2[0]; c2->p2[1] = cb->center[1];
    c3->p1[0] = cb->p1[0]; c3->p1[1] = cb->p1[1]; c3->p2[0] = cb->center[0]; c3->p2[1] = cb->center[1];
    const double xcut = cb->center[0], ycut = cb->center[1];
    size_t cutx = 0, cuty = 0;
    for (size_t i = 0; i < np; ++i) x[i] = xp[2 * particles[i] + 1];
    partition(ycut, &cuty, particles, x, np);
    if (cuty > 0) {
      for (size_t i = 0; i < cuty; ++i) x[i] = xp[2 * particles[i]];
      partition(xcut, &cutx, particles, x, cuty);
      c3->n = cutx;
      c3->particles = particles;
      c2->n = cuty - cutx;
      c2->particles = particles + cutx;
    }
    if (cuty < np) {
      for (size_t i = cuty; i < np; ++i) x[i - cuty] = xp[2 * particles[i]];
      partition(xcut, &cutx, &particles[cuty], x, np - cuty);
      c1->n = cutx;
      c1->particles = particles + cuty;
      c0->n = np - cuty - cutx;
      c0->particles = particles + cuty + cutx;
    }
    for (int k = 0; k < 4; ++k) build(cb->child[k].get(), false);
  }

  void moments(HB *cb) {
    size_t i;
    for (i = 0, cb->mass = 0; i < cb->n; ++i) cb->mass += mass[cb->particles[i]];
    cb->center[0] = cb->center[1] = 0;
    for (i = 0; i < cb->n; ++i) {
      double tmp = mass[cb->particles[i]];
      cb->center[0] += tmp * xp[2 * cb->particles[i]] / cb->mass;
      cb->center[1] += tmp * xp[2 * cb->particles[i] + 1] / cb->mass;
    }
    cb->quad[0] = cb->quad[1] = cb->quad[2] = 0;
    for (i = 0; i < cb->n; ++i) {
      double xcm0 = xp[2 * cb->particles[i]] - cb->center[0];
      double xcm1 = xp[2 * cb->particles[i] + 1] - cb->center[1];
      double xcut = std::pow(xcm0, 2) + std::pow(xcm1, 2);
      double tmp = mass[cb->particles[i]];
      cb->quad[0] += (xcut - 2 * xcm0 * xcm0) * tmp;
      cb->quad[1] += (xcut - 2 * xcm1 * xcm1) * tmp;
      cb->quad[2] += -2 * xcm0 * xcm1 * tmp;
    }
    double rcom = 0.0;
    for (i = 0; i < 2; ++i) {
      double a = std::pow(cb->center[i] - cb->p1[i], 2), b = std::pow(cb->center[i] - cb->p2[i], 2);
      rcom += (a > b) ? a : b;
    }
    rcom = std::sqrt(rcom);
    if (theta > 0.0) {
      cb->r2crit = 1.15470 * rcom / theta;
      cb->r2crit *= cb->r2crit;
    } else {
      cb->r2crit = 1.0e100;
    }
    if (cb->child[0])
      for (int k = 0; k < 4; ++k) moments(cb->child[k].get());
  }

  // preorder flattening; returns the index one past the subtree
  int flatten(const HB *cb, HaloTreeHost &out) {
    const int me = (int)out.nodes.size();
    out.nodes.emplace_back();
    HNode nd;
    nd.cx = cb->center[0];
    nd.cy = cb->center[1];
    nd.r2crit = cb->r2crit;
    nd.mass = cb->mass;
    nd.q0 = cb->quad[0];
    nd.q1 = cb->quad[1];
    nd.q2 = cb->quad[2];
    nd.leaf = cb->child[0] ? 0 : 1;
    nd.bstart = (int)out.bigs.size();
    nd.bcount = (int)cb->big.size();
    out.bigs.insert(out.bigs.end(), cb->big.begin(), cb->big.end());
    int end = me + 1;
    if (cb->child[0])
      for (int k = 0; k < 4; ++k) end = flatten(cb->child[k].get(), out);
    nd.skip = end;
    out.nodes[me] = nd;
    return end;
  }
};

}  // namespace

bool build_halo_tree(const std::vector<double> &xp, const std::vector<float> &rmax, const std::vector<float> &mass,
                     int bucket, double theta, double max_range, HaloTreeHost &out, std::string &err) {
  const size_t n = rmax.size();
  out = HaloTreeHost();
  if (n == 0) return true;
  double p1[2] = {xp[0], xp[1]}, p2[2] = {xp[0], xp[1]};
  for (size_t i = 0; i < n; ++i)
    for (int j = 0; j < 2; ++j) {
      if (xp[2 * i + j] < p1[j]) p1[j] = xp[2 * i + j];
      if (xp[2 * i + j] > p2[j]) p2[j] = xp[2 * i + j];
    }
  if (n == 1) {
    p1[0] = -0.25;
    p1[1] = -0.25;
    p2[0] = 0.25;
    p2[1] = 0.25;
  }
  const double lengths[2] = {p2[0] - p1[0], p2[1] - p1[1]};
  out.period_x = lengths[0];
  out.period_y = lengths[1];
  if (lengths[0] == 0 || lengths[1] == 0) {
    err = "particles in same place.";
    return false;
  }
  const int j = lengths[0] > lengths[1] ? 1 : 0;
  p2[j] = p1[j] + lengths[!j];
  std::vector<size_t> index(n);
  for (size_t i = 0; i < n; ++i) index[i] = i;
  Builder b{xp, rmax, mass, bucket, theta, max_range, std::vector<double>(n)};
  HB top;
  top.p1[0] = p1[0];
  top.p1[1] = p1[1];
  top.p2[0] = p2[0];
  top.p2[1] = p2[1];
  top.n = n;
  top.particles = index.data();
  b.build(&top, true);
  b.moments(&top);
  b.flatten(&top, out);
  return true;
}

}  // namespace glb
