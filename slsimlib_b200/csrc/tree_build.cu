// On-device construction of the particle quadtree (TreeQuadParticles ctor,
// BuildQTreeNB / _BuildQTreeNB / CalcMoments, include/quadTree.h:247-628).
//
// The reference splits each box at its midpoint, recursively, sending a
// particle with x <= xcut (y <= ycut) to the low side (quickPartition,
// include/Tree.h:409-424) until a box holds <= bucket particles.  Membership
// is purely geometric, so each particle's path is fixed by its coordinates:
//   1. k_keys replays the reference's double-precision midpoint halving for 32
//      levels and writes the quadrant sequence as a 64-bit key whose 2-bit
//      digits follow the reference's child order (0: x>,y>  1: x<=,y>
//      2: x>,y<=  3: x<=,y<=), so key order is the reference's depth-first
//      order;
//   2. a stable radix sort groups the particles of every box contiguously;
//   3. boxes are expanded level by level (all four children of an internal
//      box exist, as in the reference), each child's particle range found by
//      binary search on its digit;
//   4. moments are reduced bottom-up, preorder indices assigned top-down, and
//      the walk's node array, particle array and big-particle lists emitted.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "glb_host.h"

namespace glb {

int g_keep_tree_export = 0;

namespace {

constexpr unsigned kFullMask = 0xffffffffu;

struct Slot {
  double p1x, p1y, p2x, p2y;
  double mass, absm, comx, comy;
  double Fx, Fy, Sxx, Syy, Sxy;
  double r2crit;
  int start, count, child, level;
  int sub, pre, subf, pref;
  int nbig, bstart, pad0, pad1;
};

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return Status::err(-2, std::string("CUDA: ") + cudaGetErrorString(e_) + " at " \
                                 + #call);                                           \
  } while (0)

__device__ inline unsigned f2ord(float f) {
  unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float ord2f(unsigned u) {
  unsigned b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  float f;
  memcpy(&f, &b, 4);
  return f;
}

__global__ void k_bbox(const glb_particle_rec *p, size_t n, unsigned *mm) {
  unsigned mnx = 0xffffffffu, mny = 0xffffffffu, mxx = 0, mxy = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned ux = f2ord(p[i].x[0]), uy = f2ord(p[i].x[1]);
    mnx = min(mnx, ux);
    mny = min(mny, uy);
    mxx = max(mxx, ux);
    mxy = max(mxy, uy);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mnx = min(mnx, __shfl_xor_sync(0xffffffffu, mnx, o));
    mny = min(mny, __shfl_xor_sync(0xffffffffu, mny, o));
    mxx = max(mxx, __shfl_xor_sync(0xffffffffu, mxx, o));
    mxy = max(mxy, __shfl_xor_sync(0xffffffffu, mxy, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(mm + 0, mnx);
    atomicMin(mm + 1, mny);
    atomicMax(mm + 2, mxx);
    atomicMax(mm + 3, mxy);
  }
}

// 1. Morton-like key replaying the reference's midpoint halving in double.
__global__ void k_keys(const glb_particle_rec *p, size_t n, double p1x, double p1y, double p2x, double p2y,
                       unsigned long long *keys, unsigned *idx) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = (double)p[i].x[0], y = (double)p[i].x[1];
  double x1 = p1x, x2 = p2x, y1 = p1y, y2 = p2y;
  unsigned long long key = 0;
  for (int L = 0; L < kMaxDepth; ++L) {
    double cx = (x1 + x2) / 2, cy = (y1 + y2) / 2;
    bool hx = x > cx, hy = y > cy;
    unsigned d = (hx ? 0u : 1u) + (hy ? 0u : 2u);
    key = (key << 2) | d;
    if (hx) x1 = cx; else x2 = cx;
    if (hy) y1 = cy; else y2 = cy;
  }
  keys[i] = key;
  idx[i] = (unsigned)i;
}

__device__ inline unsigned digit_at(unsigned long long key, int L) {
  return (unsigned)(key >> (62 - 2 * L)) & 3u;
}

// 3a. mark internal boxes of one level and hand out child slots.
__global__ void k_mark(Slot *s, int lo, int hi, int bucket, double theta, double max_range, int next_base,
                       int *counter, int *depth_err) {
  int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hi) return;
  Slot &b = s[i];
  b.child = -1;
  if (b.count <= bucket) return;
  // leaf case of the reference (quadTree.h:370-381)
  double cx = (b.p1x + b.p2x) / 2, cy = (b.p1y + b.p2y) / 2;
  double theta_range = 2 * theta;
  if (max_range > 0) {
    double boxsize = 1.732 * (b.p2x - b.p1x);
    double d = sqrt(cx * cx + cy * cy) - max_range;
    theta_range = boxsize / (d > boxsize ? d : boxsize);
  }
  if (theta > theta_range) return;
  if (b.level >= kMaxDepth) {
    atomicAdd(depth_err, 1);
    return;
  }
  int r = atomicAdd(counter, 1);
  b.child = next_base + 4 * r;
}

// 3b. create the four children of every internal box of one level.
__global__ void k_split(Slot *s, int lo, int hi, const unsigned long long *keys) {
  int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hi) return;
  const Slot b = s[i];
  if (b.child < 0) return;
  double cx = (b.p1x + b.p2x) / 2, cy = (b.p1y + b.p2y) / 2;
  int L = b.level;
  // lower bounds of digits 1, 2, 3 inside [start, start+count)
  int bound[5];
  bound[0] = b.start;
  bound[4] = b.start + b.count;
  for (int d = 1; d <= 3; ++d) {
    int lo2 = b.start, hi2 = b.start + b.count;
    while (lo2 < hi2) {
      int mid = (lo2 + hi2) >> 1;
      if (digit_at(keys[mid], L) < (unsigned)d) lo2 = mid + 1; else hi2 = mid;
    }
    bound[d] = lo2;
  }
  for (int k = 0; k < 4; ++k) {
    Slot c;
    memset(&c, 0, sizeof(c));
    // child boxes, quadTree.h:466-484
    c.p1x = (k == 0 || k == 2) ? cx : b.p1x;
    c.p2x = (k == 0 || k == 2) ? b.p2x : cx;
    c.p1y = (k <= 1) ? cy : b.p1y;
    c.p2y = (k <= 1) ? b.p2y : cy;
    c.start = bound[k];
    c.count = bound[k + 1] - bound[k];
    c.child = -1;
    c.level = L + 1;
    c.pre = c.pref = -1;
    s[b.child + k] = c;
  }
}

__device__ inline double pmass(const glb_particle_rec *p, unsigned i, int multimass) {
  return (double)p[multimass ? i : 0].Mass;
}
__device__ inline double psize(const glb_particle_rec *p, unsigned i, int multiradius) {
  return (double)p[multiradius ? i : 0].Size;
}

__device__ inline void finish_moments(Slot &b, double theta) {
  // largest distance from the centre of mass to a corner (quadTree.h:615-618)
  double rcom = 0;
  double a = (b.comx - b.p1x) * (b.comx - b.p1x), c = (b.comx - b.p2x) * (b.comx - b.p2x);
  rcom += a > c ? a : c;
  a = (b.comy - b.p1y) * (b.comy - b.p1y);
  c = (b.comy - b.p2y) * (b.comy - b.p2y);
  rcom += a > c ? a : c;
  rcom = sqrt(rcom);
  if (theta > 0.0) {
    double r = 1.15470 * rcom / theta;
    b.r2crit = r * r;
  } else {
    b.r2crit = 1.0e100;
  }
}

// 4a. leaf moments straight from the particles (one warp per box).
__global__ void k_leaf_moments(Slot *s, int lo, int hi, const glb_particle_rec *p, const unsigned *sidx,
                               int multimass, int multiradius, double theta, float4 *prel) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  int i = lo + warp;
  if (i >= hi) return;
  Slot &b = s[i];
  if (b.child >= 0) return;
  double w = b.p2x - b.p1x;
  double M = 0, A = 0, sx = 0, sy = 0;
  int nbig = 0;
  for (int k = b.start + lane; k < b.start + b.count; k += 32) {
    unsigned id = sidx[k];
    double m = pmass(p, id, multimass);
    M += m;
    A += fabs(m);
    sx += fabs(m) * (double)p[id].x[0];
    sy += fabs(m) * (double)p[id].x[1];
    if (psize(p, id, multiradius) < w) ++nbig;
  }
  for (int o = 16; o > 0; o >>= 1) {
    M += __shfl_xor_sync(kFullMask, M, o);
    A += __shfl_xor_sync(kFullMask, A, o);
    sx += __shfl_xor_sync(kFullMask, sx, o);
    sy += __shfl_xor_sync(kFullMask, sy, o);
    nbig += __shfl_xor_sync(kFullMask, nbig, o);
  }
  double cx = b.count > 0 ? sx / A : 0.0, cy = b.count > 0 ? sy / A : 0.0;
  double Fx = 0, Fy = 0, Sxx = 0, Syy = 0, Sxy = 0;
  for (int k = b.start + lane; k < b.start + b.count; k += 32) {
    unsigned id = sidx[k];
    double m = pmass(p, id, multimass);
    double dx = (double)p[id].x[0] - cx, dy = (double)p[id].x[1] - cy;
    Fx += m * dx;
    Fy += m * dy;
    Sxx += m * dx * dx;
    Syy += m * dy * dy;
    Sxy += m * dx * dy;
  }
  for (int o = 16; o > 0; o >>= 1) {
    Fx += __shfl_xor_sync(kFullMask, Fx, o);
    Fy += __shfl_xor_sync(kFullMask, Fy, o);
    Sxx += __shfl_xor_sync(kFullMask, Sxx, o);
    Syy += __shfl_xor_sync(kFullMask, Syy, o);
    Sxy += __shfl_xor_sync(kFullMask, Sxy, o);
  }
  // records of the split-precision walk: offset from the leaf's centre of
  // mass, -mass/pi and the squared near-field radius (two softening lengths,
  // widened by 2.5e-5 against FP32 rounding; at least 1e-12 so that
  // coincident particles are sent to FP64)
  for (int k = b.start + lane; k < b.start + b.count; k += 32) {
    unsigned id = sidx[k];
    const double sz = (double)p[multiradius ? id : 0].Size;
    prel[k] = make_float4((float)((double)p[id].x[0] - cx), (float)((double)p[id].x[1] - cy),
                          (float)(-(double)p[multimass ? id : 0].Mass / kPi), (float)fmax(4.0001 * sz * sz, 1e-12));
  }
  if (lane == 0) {
    b.mass = M;
    b.absm = A;
    b.comx = cx;
    b.comy = cy;
    b.Fx = Fx;
    b.Fy = Fy;
    b.Sxx = Sxx;
    b.Syy = Syy;
    b.Sxy = Sxy;
    b.nbig = nbig;
    finish_moments(b, theta);
  }
}

// 4b. internal moments from the four children (parallel-axis shifts).
__global__ void k_internal_moments(Slot *s, int lo, int hi, double theta) {
  int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hi) return;
  Slot &b = s[i];
  if (b.child < 0) return;
  double M = 0, A = 0, sx = 0, sy = 0;
  for (int k = 0; k < 4; ++k) {
    const Slot &c = s[b.child + k];
    if (c.count == 0) continue;
    M += c.mass;
    A += c.absm;
    sx += c.absm * c.comx;
    sy += c.absm * c.comy;
  }
  double cx = sx / A, cy = sy / A;
  double Fx = 0, Fy = 0, Sxx = 0, Syy = 0, Sxy = 0;
  for (int k = 0; k < 4; ++k) {
    const Slot &c = s[b.child + k];
    if (c.count == 0) continue;
    double dx = c.comx - cx, dy = c.comy - cy;
    Sxx += c.Sxx + 2 * dx * c.Fx + dx * dx * c.mass;
    Syy += c.Syy + 2 * dy * c.Fy + dy * dy * c.mass;
    Sxy += c.Sxy + dx * c.Fy + dy * c.Fx + dx * dy * c.mass;
    Fx += c.Fx + dx * c.mass;
    Fy += c.Fy + dy * c.mass;
  }
  b.mass = M;
  b.absm = A;
  b.comx = cx;
  b.comy = cy;
  b.Fx = Fx;
  b.Fy = Fy;
  b.Sxx = Sxx;
  b.Syy = Syy;
  b.Sxy = Sxy;
  finish_moments(b, theta);
}

// 5a. subtree sizes (non-empty boxes, and all boxes), bottom-up.
__global__ void k_subtree(Slot *s, int lo, int hi) {
  int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hi) return;
  Slot &b = s[i];
  int sub = b.count > 0 ? 1 : 0, subf = 1;
  if (b.child >= 0)
    for (int k = 0; k < 4; ++k) {
      sub += s[b.child + k].sub;
      subf += s[b.child + k].subf;
    }
  b.sub = sub;
  b.subf = subf;
}

// 5b. preorder indices, top-down.
__global__ void k_preorder(Slot *s, int lo, int hi) {
  int i = lo + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= hi) return;
  const Slot &b = s[i];
  if (b.child < 0) return;
  int run = b.pre + 1, runf = b.pref + 1;
  for (int k = 0; k < 4; ++k) {
    Slot &c = s[b.child + k];
    c.pref = runf;
    runf += c.subf;
    if (c.count > 0) {
      c.pre = run;
      run += c.sub;
    } else {
      c.pre = -1;
    }
  }
}

// 6. which internal box lists each particle as "big" (quadTree.h:403-431):
// the top box takes Size > w/2, any other internal box w/2 < Size <= w.
__global__ void k_big_assign(const Slot *s, const unsigned long long *keys, const unsigned *sidx,
                             const glb_particle_rec *p, int n, unsigned *flag_key, unsigned *flag_val,
                             int *flags) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double size = (double)p[sidx[k]].Size;
  unsigned long long key = keys[k];
  int cur = 0, L = 0, list = -1;
  while (s[cur].child >= 0 && L < kMaxDepth) {
    double w = s[cur].p2x - s[cur].p1x;
    double half = w / 2;
    if (L == 0) {
      if (size > half) { list = cur; break; }
    } else if (size > half && size <= 2 * half) {
      list = cur;
      break;
    }
    cur = s[cur].child + (int)digit_at(key, L);
    ++L;
  }
  flags[k] = list >= 0 ? 1 : 0;
  flag_key[k] = list >= 0 ? (unsigned)s[list].pre : 0xffffffffu;
  flag_val[k] = (unsigned)k;
}

__global__ void k_big_ranges(const unsigned *bkey, int nb, Slot *s, const int *pre2slot) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  if (b == 0 || bkey[b] != bkey[b - 1]) {
    int e = b;
    while (e < nb && bkey[e] == bkey[b]) ++e;
    Slot &x = s[pre2slot[bkey[b]]];
    x.bstart = b;
    x.nbig = e - b;
  }
}

__global__ void k_pre2slot(const Slot *s, int nslots, int *pre2slot) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots) return;
  if (s[i].pre >= 0) pre2slot[s[i].pre] = i;
}

__global__ void k_emit_nodes(const Slot *s, int nslots, double theta, GNode *nodes, GNodeS *snodes) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots) return;
  const Slot &b = s[i];
  if (b.count == 0) return;
  GNode g;
  double w = b.p2x - b.p1x;
  double box2 = w * w;
  g.cx = b.comx;
  g.cy = b.comy;
  g.near2 = 5.83 * box2;
  g.open2 = b.r2crit > g.near2 ? b.r2crit : g.near2;
  g.mass = b.mass;
  // quad[0] = sum m (r^2 - 2x^2), quad[1] = sum m (r^2 - 2y^2), quad[2] = -2 sum m x y
  g.q0 = b.Syy - b.Sxx;
  g.q1 = b.Sxx - b.Syy;
  g.q2 = -2 * b.Sxy;
  g.width = w;
  g.skip = b.pre + b.sub;
  g.leaf = b.child < 0 ? 1 : 0;
  g.pstart = b.start;
  g.pcount = b.count;
  g.bstart = b.child < 0 ? 0 : b.bstart;
  g.bcount = b.child < 0 ? 0 : b.nbig;
  nodes[b.pre] = g;
  GNodeS f;
  f.cxh = (float)g.cx;
  f.cyh = (float)g.cy;
  f.cxl = (float)(g.cx - (double)f.cxh);
  f.cyl = (float)(g.cy - (double)f.cyh);
  f.open2 = (float)g.open2;
  f.near2 = (float)g.near2;
  f.mpi = (float)(g.mass / kPi);
  f.q0pi = (float)(g.q0 / kPi);
  f.q1pi = (float)(g.q1 / kPi);
  f.q2pi = (float)(g.q2 / kPi);
  f.width_ru = __double2float_ru(g.width);
  f.open_band = kAmbiguous * f.open2;
  f.skip = g.skip;
  f.leaf = g.leaf;
  f.start = g.leaf ? g.pstart : g.bstart;
  f.count = g.leaf ? g.pcount : g.bcount;
  snodes[b.pre] = f;
}

__global__ void k_gather_parts(const glb_particle_rec *p, const unsigned *sidx, int n, int multimass,
                               int multiradius, float4 *parts) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const glb_particle_rec &q = p[sidx[k]];
  parts[k] = make_float4(q.x[0], q.x[1], p[multimass ? sidx[k] : 0].Mass, p[multiradius ? sidx[k] : 0].Size);
}

__global__ void k_gather_bigs(const float4 *parts, const unsigned *bval, int nb, float4 *bigs) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  bigs[b] = parts[bval[b]];
}

// out[0..3]: mass and quadrupole of the last branch of the moments walk (the
// far-field potential's); out[4..7]: the root's mass, |mass| sum and centre.
// Every walk moves forward through the preorder array: a node's skip must lie
// in (i, nnodes].  The split walk relies on it without a per-node guard, so
// the build checks it once; *bad counts the nodes that break it.
__global__ void k_check_skips(const GNodeS *sn, int nnodes, int *bad) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nnodes) return;
  const int k = sn[i].skip;
  if (k <= i || k > nnodes) atomicAdd(bad, 1);
}

__global__ void k_phi_node(const Slot *s, double *out) {
  out[4] = s[0].count > 0 ? s[0].mass : 0.0;
  out[5] = s[0].count > 0 ? s[0].absm : 0.0;
  out[6] = s[0].count > 0 ? s[0].comx : 0.0;
  out[7] = s[0].count > 0 ? s[0].comy : 0.0;
  int cur = 0;
  for (int L = 0; L < kMaxDepth && s[cur].child >= 0; ++L) cur = s[cur].child + 3;
  const Slot &b = s[cur];
  if (b.count == 0) {
    out[0] = out[1] = out[2] = out[3] = 0.0;
  } else {
    out[0] = b.mass;
    out[1] = b.Syy - b.Sxx;
    out[2] = b.Sxx - b.Syy;
    out[3] = -2 * b.Sxy;
  }
}

__global__ void k_export(const Slot *s, int nslots, double *out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nslots) return;
  const Slot &b = s[i];
  double *o = out + 16 * (size_t)b.pref;
  double w = b.p2x - b.p1x;
  o[0] = b.level;
  o[1] = b.p1x;
  o[2] = b.p1y;
  o[3] = b.p2x;
  o[4] = b.p2y;
  o[5] = b.count;
  o[6] = b.nbig;
  o[7] = b.mass;
  o[8] = b.comx;
  o[9] = b.comy;
  o[10] = b.Syy - b.Sxx;
  o[11] = b.Sxx - b.Syy;
  o[12] = -2 * b.Sxy;
  o[13] = b.r2crit;
  o[14] = b.child < 0 ? 1.0 : 0.0;
  o[15] = w * w;
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

Status build_tree(const glb_particle_rec *hp, size_t n, const TreeParams &prm, bool want_export,
                  cudaStream_t st, std::unique_ptr<Tree> &out) {
  auto T = std::make_unique<Tree>();
  T->nparticles = n;
  T->theta = prm.theta;
  const int multimass = prm.mass_fixed <= 0 ? 1 : 0;  // quadTree.h:272-273
  const int multiradius = prm.size_fixed <= 0 ? 1 : 0;
  T->dev.inv_area = prm.inv_area;
  T->dev.screen2 = prm.inv_screening * prm.inv_screening;
  T->dev.periodic = prm.periodic;
  T->dev.phiintconst = (120 * log(2.) - 631.) / 840 + 19. / 70;  // quadTree.h:282
  if (n == 0) {
    T->dev.nnodes = 0;
    out = std::move(T);
    return Status::ok();
  }
  if (n > 0x7fffffffull) return Status::err(-1, "too many particles for one tree (max 2^31-1)");

  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, st));

  DBuf<glb_particle_rec> dp;
  CK(dp.alloc(n));
  CK(cudaMemcpyAsync(dp.p, hp, n * sizeof(glb_particle_rec), cudaMemcpyHostToDevice, st));

  // ---- root box (BuildQTreeNB, quadTree.h:297-337)
  DBuf<unsigned> mm;
  CK(mm.alloc(4));
  unsigned init[4] = {0xffffffffu, 0xffffffffu, 0u, 0u};
  CK(cudaMemcpyAsync(mm.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_bbox<<<std::min(nblk(n, 256), 1184), 256, 0, st>>>(dp.p, n, mm.p);
  unsigned hm[4];
  CK(cudaMemcpyAsync(hm, mm.p, sizeof(hm), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  double p1[2] = {ord2f(hm[0]), ord2f(hm[1])}, p2[2] = {ord2f(hm[2]), ord2f(hm[3])};
  if (n == 1) {
    p1[0] = -0.25; p1[1] = -0.25; p2[0] = 0.25; p2[1] = 0.25;
  }
  double lengths[2] = {p2[0] - p1[0], p2[1] - p1[1]};
  T->dev.period_x = lengths[0];
  T->dev.period_y = lengths[1];
  if (lengths[0] == 0 || lengths[1] == 0) return Status::err(-4, "particles in same place.");
  int jj = lengths[0] > lengths[1] ? 1 : 0;
  p2[jj] = p1[jj] + lengths[!jj];

  // ---- keys + stable sort
  DBuf<unsigned long long> keys, keys2;
  DBuf<unsigned> idx, sidx;
  CK(keys.alloc(n));
  CK(keys2.alloc(n));
  CK(idx.alloc(n));
  CK(sidx.alloc(n));
  k_keys<<<nblk(n, 256), 256, 0, st>>>(dp.p, n, p1[0], p1[1], p2[0], p2[1], keys.p, idx.p);
  size_t tmp_bytes = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys.p, keys2.p, idx.p, sidx.p, (int)n, 0, 64, st));
  DBuf<char> tmp;
  CK(tmp.alloc(tmp_bytes));
  CK(cub::DeviceRadixSort::SortPairs(tmp.p, tmp_bytes, keys.p, keys2.p, idx.p, sidx.p, (int)n, 0, 64, st));
  keys.release();
  idx.release();

  // ---- level-by-level expansion
  std::vector<int> off = {0, 1};
  size_t cap = 1024;
  DBuf<Slot> slots;
  CK(slots.alloc(cap));
  Slot root;
  memset(&root, 0, sizeof(root));
  root.p1x = p1[0]; root.p1y = p1[1]; root.p2x = p2[0]; root.p2y = p2[1];
  root.start = 0;
  root.count = (int)n;
  root.child = -1;
  root.level = 0;
  root.pre = 0;
  root.pref = 0;
  CK(cudaMemcpyAsync(slots.p, &root, sizeof(Slot), cudaMemcpyHostToDevice, st));
  DBuf<int> counters;
  CK(counters.alloc(2));
  for (int L = 0;; ++L) {
    int lo = off[L], hi = off[L + 1];
    CK(cudaMemsetAsync(counters.p, 0, 2 * sizeof(int), st));
    k_mark<<<nblk(hi - lo, 256), 256, 0, st>>>(slots.p, lo, hi, prm.bucket, prm.theta, prm.max_range, hi,
                                                counters.p, counters.p + 1);
    int hc[2];
    CK(cudaMemcpyAsync(hc, counters.p, sizeof(hc), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (hc[1] > 0) return Status::err(-5, "tree deeper than 32 levels (coincident particles?)");
    if (hc[0] == 0) break;
    size_t need = (size_t)hi + 4 * (size_t)hc[0];
    if (need > 0x7fffffffull) return Status::err(-1, "tree too large");
    if (need > cap) {
      size_t ncap = std::max(need, cap * 2);
      DBuf<Slot> ns;
      CK(ns.alloc(ncap));
      CK(cudaMemcpyAsync(ns.p, slots.p, (size_t)hi * sizeof(Slot), cudaMemcpyDeviceToDevice, st));
      std::swap(ns.p, slots.p);
      std::swap(ns.n, slots.n);
      cap = ncap;
    }
    k_split<<<nblk(hi - lo, 256), 256, 0, st>>>(slots.p, lo, hi, keys2.p);
    off.push_back((int)need);
  }
  const int nlev = (int)off.size() - 1;
  const int nslots = off[nlev];

  // ---- moments, bottom-up
  CK(T->prel.alloc(n));
  for (int L = nlev - 1; L >= 0; --L) {
    int lo = off[L], hi = off[L + 1];
    k_leaf_moments<<<nblk((long long)(hi - lo) * 32, 256), 256, 0, st>>>(slots.p, lo, hi, dp.p, sidx.p, multimass,
                                                                          multiradius, prm.theta, T->prel.p);
    k_internal_moments<<<nblk(hi - lo, 256), 256, 0, st>>>(slots.p, lo, hi, prm.theta);
    k_subtree<<<nblk(hi - lo, 256), 256, 0, st>>>(slots.p, lo, hi);
  }
  for (int L = 0; L < nlev; ++L) {
    int lo = off[L], hi = off[L + 1];
    k_preorder<<<nblk(hi - lo, 256), 256, 0, st>>>(slots.p, lo, hi);
  }
  Slot rootb;
  CK(cudaMemcpyAsync(&rootb, slots.p, sizeof(Slot), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  const int nnodes = rootb.sub;
  T->nnodes = nnodes;
  T->nbranches = (size_t)rootb.subf;

  // ---- sorted particle records
  CK(T->parts.alloc(n));
  k_gather_parts<<<nblk(n, 256), 256, 0, st>>>(dp.p, sidx.p, (int)n, multimass, multiradius, T->parts.p);

  // ---- big-particle lists of internal boxes
  DBuf<int> pre2slot;
  CK(pre2slot.alloc(nnodes));
  k_pre2slot<<<nblk(nslots, 256), 256, 0, st>>>(slots.p, nslots, pre2slot.p);
  int nbig = 0;
  if (multiradius) {
    DBuf<unsigned> fkey, fval, ckey, cval, skey, sval;
    DBuf<int> flags, nsel;
    CK(fkey.alloc(n));
    CK(fval.alloc(n));
    CK(flags.alloc(n));
    CK(ckey.alloc(n));
    CK(cval.alloc(n));
    CK(nsel.alloc(1));
    k_big_assign<<<nblk(n, 256), 256, 0, st>>>(slots.p, keys2.p, sidx.p, dp.p, (int)n, fkey.p, fval.p, flags.p);
    size_t tb = 0;
    CK(cub::DeviceSelect::Flagged(nullptr, tb, fkey.p, flags.p, ckey.p, nsel.p, (int)n, st));
    if (tb > tmp.n) CK(tmp.alloc(tb));
    tb = tmp.n;
    CK(cub::DeviceSelect::Flagged(tmp.p, tb, fkey.p, flags.p, ckey.p, nsel.p, (int)n, st));
    tb = tmp.n;
    CK(cub::DeviceSelect::Flagged(tmp.p, tb, fval.p, flags.p, cval.p, nsel.p, (int)n, st));
    CK(cudaMemcpyAsync(&nbig, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (nbig > 0) {
      CK(skey.alloc(nbig));
      CK(sval.alloc(nbig));
      size_t tb2 = 0;
      CK(cub::DeviceRadixSort::SortPairs(nullptr, tb2, ckey.p, skey.p, cval.p, sval.p, nbig, 0, 32, st));
      if (tb2 > tmp.n) CK(tmp.alloc(tb2));
      tb2 = tmp.n;
      CK(cub::DeviceRadixSort::SortPairs(tmp.p, tb2, ckey.p, skey.p, cval.p, sval.p, nbig, 0, 32, st));
      k_big_ranges<<<nblk(nbig, 256), 256, 0, st>>>(skey.p, nbig, slots.p, pre2slot.p);
      CK(T->bigs.alloc(nbig));
      k_gather_bigs<<<nblk(nbig, 256), 256, 0, st>>>(T->parts.p, sval.p, nbig, T->bigs.p);
    }
  }

  // ---- node array
  CK(T->nodes.alloc(nnodes));
  CK(T->snodes.alloc(nnodes));
  k_emit_nodes<<<nblk(nslots, 256), 256, 0, st>>>(slots.p, nslots, prm.theta, T->nodes.p, T->snodes.p);
  DBuf<int> dbad;
  CK(dbad.alloc(1));
  CK(cudaMemsetAsync(dbad.p, 0, sizeof(int), st));
  if (nnodes > 0) k_check_skips<<<nblk(nnodes, 256), 256, 0, st>>>(T->snodes.p, nnodes, dbad.p);
  int hbad = 0;
  CK(cudaMemcpyAsync(&hbad, dbad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  DBuf<double> phin;
  CK(phin.alloc(8));
  k_phi_node<<<1, 1, 0, st>>>(slots.p, phin.p);
  double hphi[8];
  CK(cudaMemcpyAsync(hphi, phin.p, sizeof(hphi), cudaMemcpyDeviceToHost, st));
  if (want_export) {
    DBuf<double> ex;
    CK(ex.alloc((size_t)16 * T->nbranches));
    k_export<<<nblk(nslots, 256), 256, 0, st>>>(slots.p, nslots, ex.p);
    T->export_rows.resize((size_t)16 * T->nbranches);
    CK(cudaMemcpyAsync(T->export_rows.data(), ex.p, T->export_rows.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       st));
  }
  CK(cudaEventRecord(e1, st));
  CK(cudaStreamSynchronize(st));
  CK(cudaGetLastError());
  if (hbad != 0) return Status::err(-2, "tree build produced a node array that does not move forward");
  cudaEventElapsedTime(&T->build_ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);

  T->dev.phi_mass = hphi[0];
  T->dev.phi_q0 = hphi[1];
  T->dev.phi_q1 = hphi[2];
  T->dev.phi_q2 = hphi[3];
  // With masses of one sign every cell's |m|-weighted centre is its
  // m-weighted one, so the inv_area sheet summed over any walk's far-field
  // cells and leaf particles is the root's term: inv_area M (centre - ray).
  // Σ|m| and |Σm| are then the same sums of the same values, bit for bit.
  T->dev.sheet_closed = hphi[5] == fabs(hphi[4]) ? 1 : 0;
  T->dev.root_mass = hphi[4];
  T->dev.root_cx = hphi[6];
  T->dev.root_cy = hphi[7];
  T->dev.nodes = T->nodes.p;
  T->dev.snodes = T->snodes.p;
  T->dev.parts = T->parts.p;
  T->dev.bigs = T->bigs.p;
  T->dev.prel = T->prel.p;
  T->dev.nnodes = nnodes;
  T->dev.nparticles = (int)n;
  out = std::move(T);
  return Status::ok();
}

}  // namespace glb
