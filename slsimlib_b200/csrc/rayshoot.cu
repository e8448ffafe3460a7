// Multi-plane ray shooting on the GPU and the C ABI (include/glamer_b200.h).
//
// Lens::rayshooterInternal (FullRange/internal_rayshooter_multi.cpp:53-235)
// hands chunks of rays to std::threads that each run
// Lens::compute_points_parallel (include/lens.h:913-1103): for every ray,
// every plane: LensPlaneSingular::force (MultiPlane/planes.cpp:114-161) over
// the plane's halos, then the position / Jacobian recursion.  Here every
// plane is one kernel launch over all rays (rays sorted along a Morton curve
// so that a warp holds neighbouring rays and walks the tree together); the
// per-ray recursion state (theta, SumPrevAlphas, A, SumPrevAG: 12 doubles)
// stays in HBM between planes.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <string>
#include <vector>

#include "../../include/glamer_b200.h"
#include "glb_host.h"
#include "halos.cuh"
#include "walk.cuh"
#include "walk_split.cuh"
#include "walk_group.cuh"
#include "walk_halos.cuh"

using namespace glb;

// ===================================================================== errors
static thread_local std::string t_err;
static int fail(int code, const std::string &m) {
  t_err = m;
  return code;
}
static int fail(const Status &s) { return fail(s.code, s.msg); }

#define CKR(call)                                                                              \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess)                                                                     \
      return fail(e_ == cudaErrorMemoryAllocation ? GLB_ERR_OOM : GLB_ERR_CUDA,                \
                  std::string("CUDA: ") + cudaGetErrorString(e_) + " at " #call);              \
  } while (0)

static int need_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
    return fail(GLB_ERR_NO_DEVICE, "no CUDA device: the B200 ray-shooting library has no CPU path");
  return 0;
}

// ================================================================ NFW tables
namespace {
struct HostNFWTables {
  std::vector<double> x, f, g, g2, h;
};
std::once_flag g_nfw_host_once;
HostNFWTables g_nfw_host;

// LensHaloNFW::make_tables, MultiPlane/lens_halos.cpp:482-508.
void make_host_tables() {
  HostNFWTables &T = g_nfw_host;
  T.x.resize(kNfwTable);
  T.f.resize(kNfwTable);
  T.g.resize(kNfwTable);
  T.g2.resize(kNfwTable);
  T.h.resize(kNfwTable);
  double dx = kNfwMaxRm / (double)kNfwTable;
  for (int i = 0; i < kNfwTable; i++) {
    double x = i * dx;
    T.x[i] = x;
    T.f[i] = nfw_f(x);
    T.g[i] = nfw_g(x);
    T.g2[i] = nfw_g2(x);
    T.h[i] = nfw_h(x);
  }
}

// InterpolateFromTable (lens_halos.cpp:566-580) on the host, for set-up values.
double nfw_interp_host(int which, double y) {
  const HostNFWTables &T = g_nfw_host;
  int j = (int)(y / kNfwMaxRm * kNfwTable);
  if (j == 0) {
    switch (which) {
      case 0: return nfw_f(y);
      case 1: return nfw_g(y);
      case 2: return nfw_g2(y);
      default: return nfw_h(y);
    }
  }
  const std::vector<double> &t = which == 0 ? T.f : which == 1 ? T.g : which == 2 ? T.g2 : T.h;
  return (t[j + 1] - t[j]) / (T.x[j + 1] - T.x[j]) * (y - T.x[j]) + t[j];
}

// Device copies, one set per device.
struct DevNFWTables {
  double *x = nullptr, *f = nullptr, *g = nullptr, *g2 = nullptr, *h = nullptr;
};
std::mutex g_dev_nfw_mu;
DevNFWTables g_dev_nfw[64];

int device_nfw_tables(NFWTables &out) {
  std::call_once(g_nfw_host_once, make_host_tables);
  int dev = 0;
  CKR(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(GLB_ERR_ARG, "device index beyond the 64 devices the library supports");
  std::lock_guard<std::mutex> lk(g_dev_nfw_mu);
  DevNFWTables &D = g_dev_nfw[dev];
  if (!D.x) {
    double **dst[5] = {&D.x, &D.f, &D.g, &D.g2, &D.h};
    const std::vector<double> *src[5] = {&g_nfw_host.x, &g_nfw_host.f, &g_nfw_host.g, &g_nfw_host.g2,
                                         &g_nfw_host.h};
    for (int i = 0; i < 5; ++i) {
      CKR(cudaMalloc((void **)dst[i], kNfwTable * sizeof(double)));
      CKR(cudaMemcpy(*dst[i], src[i]->data(), kNfwTable * sizeof(double), cudaMemcpyHostToDevice));
    }
  }
  out.x = D.x;
  out.f = D.f;
  out.g = D.g;
  out.g2 = D.g2;
  out.h = D.h;
  return 0;
}
}  // namespace

// ===================================================================== halos
struct glb_halo {
  int kind = HALO_PARTICLES;
  double theta[2] = {0, 0};  // posHalo (radians)
  double zlens = 0;
  double Dist = 0;  // angular-size distance used by LensHalo::getX
  // LensHalo float members (include/lens_halos.h:279-356)
  float mass = 0, Rsize = 0, Rmax = 0, rscale = 1;
  NFWDev nfw{};
  NSIEDev nsie{};
  std::unique_ptr<Tree> tree;
  std::unique_ptr<struct FieldTree> field;  // HALO_FIELD: a LensPlaneTree
  int device = 0;
  cudaStream_t stream = nullptr;
};

// LensPlaneTree (MultiPlane/planes.cpp:13-18): the member haloes (owned) and
// their TreeQuadHalos on the device.
struct FieldTree {
  std::vector<std::unique_ptr<glb_halo>> members;
  double sigma_back = 0, inv_screening = 0;
  int bucket = 5, periodic = 0;
  double theta = 0.5;
  DBuf<HNode> nodes;
  DBuf<int> bigs;
  DBuf<FieldHaloDev> halos;
  HaloTreeDev dev{};
};

// ====================================================================== lens
struct PlaneHost {
  double z, Dl;
  std::vector<glb_halo *> halos;
};

// The per-call workspace of one calling thread on one lens: its stream,
// timing events and device buffers.  Threads that shoot rays through the same
// lens each get their own, so their calls run concurrently on the GPU while
// the lens's device descriptors (planes, halos, trees) are only read.
struct LensWS {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t done = nullptr;  // end of this workspace's last pass (orders reuse across streams)
  // the streams and join events of a large call's slabs (slab 0 runs on the call's stream)
  cudaStream_t sub[3] = {nullptr, nullptr, nullptr};
  cudaEvent_t join[3] = {nullptr, nullptr, nullptr};
  DBuf<double> st;          // 12 n recursion state
  DBuf<double> io;          // host-call staging: x 2n, zs n, y 2n, A 4n
  DBuf<int> jmax_ray;
  DBuf<double> src_ray;     // Dls/Ds, D/Ds per ray
  DBuf<unsigned> keys, keys2, perm0, perm;
  DBuf<char> sort_tmp;
  DBuf<unsigned long long> bbox;
  DBuf<unsigned char> status;  // per-ray status staging
  size_t ws_n = 0;
  float last_kernel_ms = 0, last_total_ms = 0;
  bool timed = false;
  ~LensWS() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
    if (done) cudaEventDestroy(done);
    for (int i = 0; i < 3; ++i) {
      if (sub[i]) cudaStreamSynchronize(sub[i]);
      if (join[i]) cudaEventDestroy(join[i]);
      if (sub[i]) cudaStreamDestroy(sub[i]);
    }
    if (stream) cudaStreamDestroy(stream);
  }
};

struct glb_lens {
  Cosmo cosmo{0.3, 0.7, 0.7};
  double zsource = 0;
  double charge = 0;
  std::vector<std::unique_ptr<glb_halo>> owned;
  std::vector<PlaneHost> main;  // sorted by Dl
  std::vector<PlaneHost> field;  // LensPlaneTree planes, in insertion order
  std::vector<PlaneHost *> planes;  // main and field planes in order of distance (combinePlanes)
  std::vector<char> plane_field;    // per plane: holds a field plane (HALO_FIELD)
  std::vector<double> plane_z, Dl, dDl;  // combined, source pseudo-plane last
  bool toggle_source_plane = false;
  double zs_implant = 0;
  int device = 0;
  cudaStream_t stream = nullptr;  // uploads of the descriptors
  // device copies of the plane / halo descriptors (uploaded once under mu,
  // then only read)
  bool dirty = true;
  DBuf<PlaneDev> d_planes;
  DBuf<HaloDev> d_halos;
  DBuf<double> d_planez, d_Dl;
  // per-thread workspaces (created on a thread's first call, freed with the lens)
  std::mutex mu;
  std::map<std::thread::id, std::unique_ptr<LensWS>> ws;
};

// ================================================================== kernels
namespace {

__device__ inline unsigned long long d2ord(double d) {
  unsigned long long b = (unsigned long long)__double_as_longlong(d);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ inline double ord2d(unsigned long long u) {
  unsigned long long b = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
  return __longlong_as_double((long long)b);
}

__global__ void k_ray_bbox(const double *x, size_t n, unsigned long long *bb) {
  unsigned long long mnx = ~0ull, mny = ~0ull, mxx = 0, mxy = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    // a non-finite ray would stretch the box over everything (its own key is
    // clamped to the box in k_ray_morton)
    if (!isfinite(x[2 * i]) || !isfinite(x[2 * i + 1])) continue;
    unsigned long long ux = d2ord(x[2 * i]), uy = d2ord(x[2 * i + 1]);
    mnx = min(mnx, ux);
    mny = min(mny, uy);
    mxx = max(mxx, ux);
    mxy = max(mxy, uy);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mnx = min(mnx, __shfl_xor_sync(kFull, mnx, o));
    mny = min(mny, __shfl_xor_sync(kFull, mny, o));
    mxx = max(mxx, __shfl_xor_sync(kFull, mxx, o));
    mxy = max(mxy, __shfl_xor_sync(kFull, mxy, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(bb + 0, mnx);
    atomicMin(bb + 1, mny);
    atomicMax(bb + 2, mxx);
    atomicMax(bb + 3, mxy);
  }
}

__device__ inline unsigned spread16(unsigned v) {
  v &= 0xffffu;
  v = (v | (v << 8)) & 0x00ff00ffu;
  v = (v | (v << 4)) & 0x0f0f0f0fu;
  v = (v | (v << 2)) & 0x33333333u;
  v = (v | (v << 1)) & 0x55555555u;
  return v;
}

__global__ void k_ray_morton(const double *x, size_t n, const unsigned long long *bb, unsigned *keys,
                             unsigned *idx) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x0 = ord2d(bb[0]), y0 = ord2d(bb[1]), x1 = ord2d(bb[2]), y1 = ord2d(bb[3]);
  double sx = x1 > x0 ? 65535.0 / (x1 - x0) : 0.0, sy = y1 > y0 ? 65535.0 / (y1 - y0) : 0.0;
  double fx = (x[2 * i] - x0) * sx, fy = (x[2 * i + 1] - y0) * sy;
  unsigned qx = (unsigned)fmin(fmax(fx, 0.0), 65535.0), qy = (unsigned)fmin(fmax(fy, 0.0), 65535.0);
  keys[i] = spread16(qx) | (spread16(qy) << 1);
  idx[i] = (unsigned)i;
}

__global__ void k_identity(unsigned *p, size_t n) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i < n) p[i] = (unsigned)i;
}

struct SrcArgs {
  Cosmo cosmo;
  const double *planez;  // np + 1
  const double *Dl;      // np + 1
  int np;
};

// Lens::FindSourcePlane (MultiPlane/lens.cpp:2659-2680) for one ray.
__device__ inline void find_source_plane(const SrcArgs &s, double zs, int &jmax, double &dls_ds, double &d_ds) {
  double Ds = coordist(s.cosmo, zs), Dls;
  if (zs <= s.planez[0]) {
    jmax = 0;
    Dls = Ds;
  } else {
    jmax = s.np;
    if (jmax <= 0) {
      Dls = Ds;
    } else {
      while (s.planez[jmax - 1] > zs) --jmax;
      Dls = coordist2(s.cosmo, s.planez[jmax - 1], zs);
    }
  }
  dls_ds = Dls / Ds;
  d_ds = jmax > 0 ? s.Dl[jmax - 1] / Ds : 0.0;
}

// State layout: st[c * n + k], c = 0..11:
//   theta0 theta1 | SumPrevAlphas0 1 | A0..A3 | SumPrevAG0..3
__global__ void k_init_state(const double *x, const double *zs, const unsigned *perm, size_t n, double *st,
                             int *jmax_ray, double *src_ray, SrcArgs s) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  unsigned i = perm[k];
  double t0 = x[2 * i], t1 = x[2 * i + 1];
  st[0 * n + k] = t0;
  st[1 * n + k] = t1;
  st[2 * n + k] = t0;
  st[3 * n + k] = t1;
  st[4 * n + k] = 1;
  st[5 * n + k] = 0;
  st[6 * n + k] = 0;
  st[7 * n + k] = 1;
  st[8 * n + k] = 1;
  st[9 * n + k] = 0;
  st[10 * n + k] = 0;
  st[11 * n + k] = 1;
  if (zs) {
    int jm;
    double a, b;
    find_source_plane(s, zs[i], jm, a, b);
    jmax_ray[k] = jm;
    src_ray[2 * k] = a;
    src_ray[2 * k + 1] = b;
  }
}

// Per-ray status (include/glamer_b200.h): a skipped ray (the caller's flag,
// the reference's in_image == MAYBE points, lens.h:959) keeps its y and A
// untouched; a ray whose y or A is not finite is flagged where the reference
// asserts (lens.h:1012-1037).
__device__ __forceinline__ unsigned char ray_status(const double *y, const double *A) {
  bool f = isfinite(y[0]) && isfinite(y[1]);
  for (int c = 0; c < 4; ++c) f = f && isfinite(A[c]);
  return f ? GLB_RAY_OK : GLB_RAY_NONFINITE;
}

__global__ void k_finish(const double *st, const unsigned *perm, size_t n, double *y, double *A,
                         unsigned char *status = nullptr, const unsigned char *skip = nullptr) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  unsigned i = perm[k];
  if (skip && skip[i]) {
    if (status) status[i] = GLB_RAY_SKIPPED;
    return;
  }
  const double yy[2] = {st[0 * n + k], st[1 * n + k]};
  const double AA[4] = {st[4 * n + k], st[5 * n + k], st[6 * n + k], st[7 * n + k]};
  y[2 * i] = yy[0];
  y[2 * i + 1] = yy[1];
  A[4 * i] = AA[0];
  A[4 * i + 1] = AA[1];
  A[4 * i + 2] = AA[2];
  A[4 * i + 3] = AA[3];
  if (status) status[i] = ray_status(yy, AA);
}

__global__ void k_identity_rays(const double *x, size_t n, double *y, double *A, unsigned char *status = nullptr,
                                const unsigned char *skip = nullptr) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (skip && skip[i]) {
    if (status) status[i] = GLB_RAY_SKIPPED;
    return;
  }
  y[2 * i] = x[2 * i];
  y[2 * i + 1] = x[2 * i + 1];
  A[4 * i] = 1;
  A[4 * i + 1] = 0;
  A[4 * i + 2] = 0;
  A[4 * i + 3] = 1;
  const double AA[4] = {1, 0, 0, 1};
  if (status) status[i] = ray_status(x + 2 * i, AA);
}

// xygridpoints + PositionFromIndex (TreeCode_link/gridmap.cpp:293-321,
// TreeCode_link/utilities.cpp:149-158), x fastest.
__global__ void k_grid(size_t N1d, double c0, double c1, double range, double *x) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= N1d * N1d) return;
  if (N1d == 1) {
    x[0] = c0;
    x[1] = c1;
    return;
  }
  x[2 * i] = c0 + range * (1.0 * (double)(i % N1d) / (double)(N1d - 1) - 0.5);
  x[2 * i + 1] = c1 + range * (1.0 * (double)(i / N1d) / (double)(N1d - 1) - 0.5);
}

template <int PREC, bool PHI, bool COUNT = false, bool SKIPNEAR = false, bool MERGE = true>
__device__ __forceinline__ void particle_halo_acc(const TreeDev &T, double rx, double ry, bool valid, double *acc,
                                                  WalkCount *wc = nullptr) {
  if (T.periodic) {
    // force2D_recur with a periodic buffer: nine shifted copies (quadTree.h:944-974)
    for (int i = -1; i < 2; ++i)
      for (int j = -1; j < 2; ++j) {
        if (PREC == GLB_PREC_FP64)
          walk_f64<PHI, COUNT>(T, rx + i * T.period_x, ry + j * T.period_y, valid, acc, wc);
        else if (PREC == GLB_PREC_FP32)
          walk_split<true>(T, rx + i * T.period_x, ry + j * T.period_y, valid, acc);
        else
          walk_split<false, SKIPNEAR, MERGE>(T, rx + i * T.period_x, ry + j * T.period_y, valid, acc);
      }
  } else {
    if (PREC == GLB_PREC_FP64)
      walk_f64<PHI, COUNT>(T, rx, ry, valid, acc, wc);
    else if (PREC == GLB_PREC_FP32)
      walk_split<true>(T, rx, ry, valid, acc);
    else
      walk_split<false, SKIPNEAR, MERGE>(T, rx, ry, valid, acc);
  }
}

// Analytic halo of a plane at one position; kept out of line so that the rare
// NFW / NSIE arithmetic does not add to the register budget of the tree walk.
// The result comes back by value: a caller's accumulator array passed by
// pointer to an out-of-line function would be moved to local memory, and the
// tree walk's flushes into it with it.
struct Force5 {
  double a0, a1, k, g0, g1;
};
__device__ __noinline__ Force5 analytic_halo(const HaloDev *H, const NFWTables *tab, double x0, double x1) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (H->kind == HALO_NFW)
    nfw_force<false>(H->nfw, *tab, x0, x1, acc);
  else
    nsie_force<false>(H->nsie, x0, x1, acc);
  return Force5{acc[0], acc[1], acc[2], acc[3], acc[4]};
}

struct StepArgs {
  const PlaneDev *planes;
  const HaloDev *halos;
  NFWTables tab;
  double *st;
  size_t n;
  int j;
  int jmax;             // uniform source plane
  double dls_ds, d_ds;  // uniform source plane
  const int *jmax_ray;  // per-ray source planes (or null)
  const double *src_ray;
  double charge;
  unsigned long long *counts;  // V F P B S Wn Wp totals (counting launches only)
  // The plane's particle tree and its offset (posHalo * Dist) when the plane
  // holds exactly one particle halo (k_plane_step_split_g): read from
  // kernel parameter space, so the walk's pointers and scalars are uniform
  // operands rather than per-thread registers.
  TreeDev tree;
  double tree_px, tree_py;
};

// The recursion of include/lens.h:1003-1066 for ray slot k once the plane's
// summed halo forces are known (al: the plane's deflection with the sign of
// LensPlaneSingular::force, planes.cpp:151-152; kap, g0, g1 summed).
__device__ __forceinline__ void recursion_step(const StepArgs &a, size_t k, double al0, double al1, double kap,
                                               double g0, double g1) {
  const size_t n = a.n;
  double *st = a.st;
  int jmax = a.jmax;
  double dls = a.dls_ds, dds = a.d_ds;
  if (a.jmax_ray) {
    jmax = a.jmax_ray[k];
    dls = a.src_ray[2 * k];
    dds = a.src_ray[2 * k + 1];
  }
  const PlaneDev &P = a.planes[a.j];
  double G0 = kap + g0, G1 = g1, G2 = g1, G3 = kap - g0;
  G0 *= P.Gfac;
  G1 *= P.Gfac;
  G2 *= P.Gfac;
  G3 *= P.Gfac;
  double th0 = st[0 * n + k], th1 = st[1 * n + k];
  double sa0 = st[2 * n + k] - a.charge * al0;
  double sa1 = st[3 * n + k] - a.charge * al1;
  double aa, bb;
  if (a.j < jmax - 1) {
    aa = P.aa;
    bb = P.bb;
  } else {
    aa = dls;
    bb = dds;
  }
  th0 = bb * th0 + aa * sa0;
  th1 = bb * th1 + aa * sa1;
  const double A0 = st[4 * n + k], A1 = st[5 * n + k], A2 = st[6 * n + k], A3 = st[7 * n + k];
  double s0 = st[8 * n + k], s1 = st[9 * n + k], s2 = st[10 * n + k], s3 = st[11 * n + k];
  // SumPrevAG -= G * A (Matrix2x2 product, include/point.h:249-258)
  s0 -= G0 * A0 + G1 * A2;
  s1 -= G0 * A1 + G1 * A3;
  s2 -= G2 * A0 + G3 * A2;
  s3 -= G2 * A1 + G3 * A3;
  st[0 * n + k] = th0;
  st[1 * n + k] = th1;
  st[2 * n + k] = sa0;
  st[3 * n + k] = sa1;
  st[4 * n + k] = A0 * bb + s0 * aa;
  st[5 * n + k] = A1 * bb + s1 * aa;
  st[6 * n + k] = A2 * bb + s2 * aa;
  st[7 * n + k] = A3 * bb + s3 * aa;
  st[8 * n + k] = s0;
  st[9 * n + k] = s1;
  st[10 * n + k] = s2;
  st[11 * n + k] = s3;
}

// One lens plane for every ray: LensPlaneSingular::force + the recursion of
// include/lens.h:1003-1066.
template <int PREC, bool COUNT = false, bool FIELD = false>
__device__ __forceinline__ void plane_step(const StepArgs &a) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const bool inrange = k < a.n;
  const size_t n = a.n;
  int jmax = a.jmax;
  double dls = a.dls_ds, dds = a.d_ds;
  if (a.jmax_ray && inrange) {
    jmax = a.jmax_ray[k];
    dls = a.src_ray[2 * k];
    dds = a.src_ray[2 * k + 1];
  }
  const bool valid = inrange && a.j < jmax;
  if (!__any_sync(kFull, valid)) return;
  double *st = a.st;
  double th0 = 0, th1 = 0;
  if (valid) {
    th0 = st[0 * n + k];
    th1 = st[1 * n + k];
  }
  const PlaneDev P = a.planes[a.j];
  const double xx0 = th0 * P.Dphys, xx1 = th1 * P.Dphys;
  double al0 = 0, al1 = 0, kap = 0, g0 = 0, g1 = 0;
  for (int h = 0; h < P.nhalo; ++h) {
    const HaloDev *H = a.halos + P.halo0 + h;
    const int kind = H->kind;
    const double xc0 = xx0 - H->px, xc1 = xx1 - H->py;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    if (kind == HALO_PARTICLES) {
      if (COUNT) {
        WalkCount wc;
        particle_halo_acc<PREC, false, true>(H->tree, xc0, xc1, valid, acc, &wc);
        unsigned long long v[7] = {wc.V, wc.F, wc.P, wc.B, wc.S, wc.Wn, wc.Wp};
        for (int c = 0; c < 7; ++c) {
          for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_xor_sync(kFull, v[c], o);
          if ((threadIdx.x & 31) == 0) atomicAdd(a.counts + c, v[c]);
        }
      } else {
        particle_halo_acc<PREC, false>(H->tree, xc0, xc1, valid, acc);
      }
      // LensHaloParticles::force_halo negates alpha (particle_halo.h:432-433)
      acc[0] = -acc[0];
      acc[1] = -acc[1];
    } else if (FIELD && kind == HALO_FIELD) {
      // LensPlaneTree::force is the tree's output as it is (planes.cpp:65-68)
      const Force6 f = field_plane_force<false>(&H->htree, &a.tab, xc0, xc1, valid);
      acc[0] = -f.a0;
      acc[1] = -f.a1;
      acc[2] = f.k;
      acc[3] = f.g0;
      acc[4] = f.g1;
    } else if (valid) {
      const Force5 f = analytic_halo(H, &a.tab, xc0, xc1);
      acc[0] = f.a0;
      acc[1] = f.a1;
      acc[2] = f.k;
      acc[3] = f.g0;
      acc[4] = f.g1;
    }
    al0 -= acc[0];
    al1 -= acc[1];
    kap += acc[2];
    g0 += acc[3];
    g1 += acc[4];
  }
  if (!valid) return;
  double G0 = kap + g0, G1 = g1, G2 = g1, G3 = kap - g0;
  G0 *= P.Gfac;
  G1 *= P.Gfac;
  G2 *= P.Gfac;
  G3 *= P.Gfac;
  double sa0 = st[2 * n + k] - a.charge * al0;
  double sa1 = st[3 * n + k] - a.charge * al1;
  double aa, bb;
  if (a.j < jmax - 1) {
    aa = P.aa;
    bb = P.bb;
  } else {
    aa = dls;
    bb = dds;
  }
  th0 = bb * th0 + aa * sa0;
  th1 = bb * th1 + aa * sa1;
  const double A0 = st[4 * n + k], A1 = st[5 * n + k], A2 = st[6 * n + k], A3 = st[7 * n + k];
  double s0 = st[8 * n + k], s1 = st[9 * n + k], s2 = st[10 * n + k], s3 = st[11 * n + k];
  // SumPrevAG -= G * A (Matrix2x2 product, include/point.h:249-258)
  s0 -= G0 * A0 + G1 * A2;
  s1 -= G0 * A1 + G1 * A3;
  s2 -= G2 * A0 + G3 * A2;
  s3 -= G2 * A1 + G3 * A3;
  st[0 * n + k] = th0;
  st[1 * n + k] = th1;
  st[2 * n + k] = sa0;
  st[3 * n + k] = sa1;
  st[4 * n + k] = A0 * bb + s0 * aa;
  st[5 * n + k] = A1 * bb + s1 * aa;
  st[6 * n + k] = A2 * bb + s2 * aa;
  st[7 * n + k] = A3 * bb + s3 * aa;
  st[8 * n + k] = s0;
  st[9 * n + k] = s1;
  st[10 * n + k] = s2;
  st[11 * n + k] = s3;
}

// The FP64 form keeps the compiler's own register choice; the split form is
// latency-bound (dependent node loads and short arithmetic chains), and
// capping it at 64 registers (8 blocks of 128 per SM, half the warp slots)
// buys the occupancy that hides them, spills included.
// Planes holding a field plane (HALO_FIELD) use the FIELD instances, so that
// the halo-tree walk adds no code to the kernels of particle planes.
template <int PREC, bool COUNT = false, bool FIELD = false>
__global__ void __launch_bounds__(128) k_plane_step(StepArgs a) {
  plane_step<PREC, COUNT, FIELD>(a);
}
// Split-form plane step with the block-level group walk (walk_group.cuh) for
// a plane holding exactly one particle halo (its tree in a.tree, a kernel
// parameter) and any number of analytic halos: one ray per thread, 128
// neighbouring rays per block sharing the classification of the tree's
// cells.  Each ray's FP64 totals sit in shared memory (sacc, five doubles per
// thread at a stride of five: a half-warp's 64-bit accesses on distinct
// banks), and the recursion reloads theta, the plane constants and the
// source-plane scalars after the walk.  The particle halo's terms are added
// first, then the analytic halos' in insertion order.  Measured per 2048^2
// light-cone step against the per-ray walks: 638 ms against 718 (two rays
// per thread) and 771 (one); 512^2 single plane 5.56 against 5.88 ms.
__global__ void __launch_bounds__(128, 6) k_plane_step_split_g(const __grid_constant__ StepArgs a) {
  __shared__ double sacc[5 * 128];
  __shared__ double sxy[2 * 128];
  __shared__ GroupLists G;
  __shared__ double wbox[4][4];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const size_t k = blockIdx.x * (size_t)blockDim.x + t;
  const bool inrange = k < a.n;
  const int jmax = (a.jmax_ray && inrange) ? a.jmax_ray[k] : a.jmax;
  const bool valid = inrange && a.j < jmax;
  double *acc = sacc + 5 * t;
  for (int c = 0; c < 5; ++c) acc[c] = 0.0;
  double rx = 0, ry = 0;
  if (valid) {
    const double D = a.planes[a.j].Dphys;
    rx = a.st[k] * D - a.tree_px;
    ry = a.st[a.n + k] * D - a.tree_py;
  }
  sxy[2 * t] = rx;
  sxy[2 * t + 1] = ry;
  double b0 = valid ? rx : 1e300, b1 = valid ? rx : -1e300, b2 = valid ? ry : 1e300, b3 = valid ? ry : -1e300;
  for (int o = 16; o > 0; o >>= 1) {
    b0 = fmin(b0, __shfl_xor_sync(kFull, b0, o));
    b1 = fmax(b1, __shfl_xor_sync(kFull, b1, o));
    b2 = fmin(b2, __shfl_xor_sync(kFull, b2, o));
    b3 = fmax(b3, __shfl_xor_sync(kFull, b3, o));
  }
  if (lane == 0) {
    wbox[warp][0] = b0;
    wbox[warp][1] = b1;
    wbox[warp][2] = b2;
    wbox[warp][3] = b3;
  }
  __syncthreads();
  if (t == 0) {
    double x0 = wbox[0][0], x1 = wbox[0][1], y0 = wbox[0][2], y1 = wbox[0][3];
    for (int w = 1; w < 4; ++w) {
      x0 = fmin(x0, wbox[w][0]);
      x1 = fmax(x1, wbox[w][1]);
      y0 = fmin(y0, wbox[w][2]);
      y1 = fmax(y1, wbox[w][3]);
    }
    G.box[0] = x0;
    G.box[1] = x1;
    G.box[2] = y0;
    G.box[3] = y1;
    G.any = x0 <= x1 ? 1 : 0;
    G.q[0] = 0;
    G.qhead = 0;
    G.qtail = 1;
    G.nfar = G.nleaf = G.nbig = G.nmixed = 0;
    G.done = 0;
  }
  __syncthreads();
  if (!G.any) return;
  walk_group(a.tree, sxy + 2 * t, valid, acc, G);
  if (!valid) return;
  double al0 = acc[0], al1 = acc[1], kap = acc[2], g0 = acc[3], g1 = acc[4];
  const PlaneDev &P = a.planes[a.j];
  for (int h = 0; h < P.nhalo; ++h) {
    const HaloDev *H = a.halos + P.halo0 + h;
    if (H->kind == HALO_PARTICLES) continue;
    const double D = P.Dphys;
    const Force5 f = analytic_halo(H, &a.tab, a.st[k] * D - H->px, a.st[a.n + k] * D - H->py);
    al0 -= f.a0;
    al1 -= f.a1;
    kap += f.k;
    g0 += f.g0;
    g1 += f.g1;
  }
  recursion_step(a, k, al0, al1, kap, g0, g1);
}

// Split-form plane step of planes with several particle halos or a field
// plane, one ray per thread.
template <bool FIELD = false>
__global__ void __launch_bounds__(128, 8) k_plane_step_split(const __grid_constant__ StepArgs a) {
  plane_step<GLB_PREC_SPLIT, false, FIELD>(a);
}

// force2D_recur / force_halo at arbitrary positions (walk-level API, with phi).
// subtract: LensHalo::force_halo's subtract_point = true with `screening`
// (analytic haloes; particle trees and field planes take no such argument).
__global__ void __launch_bounds__(128) k_halo_force(HaloDev H, NFWTables tab, size_t n, const double *x,
                                                    double *out, int subtract = 0, double screening = 1.0) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const bool valid = k < n;
  if (!__any_sync(kFull, valid)) return;
  double x0 = 0, x1 = 0;
  if (valid) {
    x0 = x[2 * k];
    x1 = x[2 * k + 1];
  }
  double acc[6] = {0, 0, 0, 0, 0, 0};
  if (H.kind == HALO_PARTICLES) {
    particle_halo_acc<GLB_PREC_FP64, true>(H.tree, x0, x1, valid, acc);
  } else if (H.kind == HALO_FIELD) {
    field_plane_acc<true>(H.htree, tab, x0, x1, valid, acc);
  } else if (valid && subtract) {
    if (H.kind == HALO_NFW) {
      if (subtract_point_terms<true>(H.nfw.mass, H.nfw.Rmax2, x0, x1, screening, acc))
        nfw_force<true, true>(H.nfw, tab, x0, x1, acc);
    } else if (subtract_point_terms<true>(H.nsie.mass, H.nsie.Rmax2, x0, x1, screening, acc)) {
      nsie_force<true>(H.nsie, x0, x1, acc);  // lens_halos.cpp:1938-2014 uses the flag only in force_point
    }
  } else if (valid) {
    if (H.kind == HALO_NFW)
      nfw_force<true>(H.nfw, tab, x0, x1, acc);
    else
      nsie_force<true>(H.nsie, x0, x1, acc);
  }
  if (!valid) return;
  for (int c = 0; c < 6; ++c) out[6 * k + c] = acc[c];
}

// force2D_recur on device rays in the three precision forms (no potential):
// out = 5 doubles per ray {alpha0, alpha1, kappa, gamma0, gamma1}.
template <int PREC>
__device__ __forceinline__ void tree_force(const TreeDev &T, size_t n, const double *x, double *out) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const bool valid = k < n;
  if (!__any_sync(kFull, valid)) return;
  double x0 = 0, x1 = 0;
  if (valid) {
    x0 = x[2 * k];
    x1 = x[2 * k + 1];
  }
  double acc[6] = {0, 0, 0, 0, 0, 0};
  particle_halo_acc<PREC, false, false, false, false>(T, x0, x1, valid, acc);  // a flush per opened leaf
  if (!valid) return;
  for (int c = 0; c < 5; ++c) out[5 * k + c] = acc[c];
}

__global__ void __launch_bounds__(128) k_tree_force(const __grid_constant__ TreeDev T, size_t n, const double *x,
                                                    double *out) {
  tree_force<GLB_PREC_FP64>(T, n, x, out);
}
// the FP32-arithmetic forms, capped at 80 registers (6 blocks of 128 per SM) for occupancy
template <int PREC>
__global__ void __launch_bounds__(128, 6) k_tree_force_lo(const __grid_constant__ TreeDev T, size_t n,
                                                          const double *x, double *out) {
  tree_force<PREC>(T, n, x, out);
}

// The split form with two rays per thread (rays 2g and 2g + 1; a warp walks
// 64 rays, sharing node rows, votes and leaf particles between each pair),
// the rays' positions and FP64 totals in shared memory.  Rays come in the
// caller's order; each ray forms its own double-float offsets and sums each
// opened leaf on its own (walk_split2): every result is bit-identical to
// k_tree_force_lo's.
__global__ void __launch_bounds__(128, 6) k_tree_force_split2(const __grid_constant__ TreeDev T, size_t n,
                                                              const double *x, double *out) {
  __shared__ double sacc[10 * 128];
  __shared__ double sxy[4 * 128];
  const size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t k0 = 2 * g, k1 = 2 * g + 1;
  const bool v0 = k0 < n, v1 = k1 < n;
  if (!__any_sync(kFull, v0)) return;
  double *acc0 = sacc + 5 * threadIdx.x, *acc1 = sacc + 5 * (blockDim.x + threadIdx.x);
  double *rxy = sxy + 4 * threadIdx.x;
  for (int c = 0; c < 5; ++c) acc0[c] = acc1[c] = 0.0;
  rxy[0] = v0 ? x[2 * k0] : 0.0;
  rxy[1] = v0 ? x[2 * k0 + 1] : 0.0;
  rxy[2] = v1 ? x[2 * k1] : 0.0;
  rxy[3] = v1 ? x[2 * k1 + 1] : 0.0;
  walk_split2(T, rxy, v0, v1, acc0, acc1);
  if (v0)
    for (int c = 0; c < 5; ++c) out[5 * k0 + c] = acc0[c];
  if (v1)
    for (int c = 0; c < 5; ++c) out[5 * k1 + c] = acc1[c];
}

// FP64 direct summation over every particle (no tree): the point mass and the
// B-spline correction within two sizes, with the inv_area sheet -- the same
// kernel as the tree's leaves (quadTree.h:1017-1077), for absolute-accuracy
// reports.  Particles are staged through shared memory, one ray per thread.
__global__ void __launch_bounds__(256) k_direct_sum(const glb_particle_rec *p, size_t n, double inv_area,
                                                    const double *x, size_t nr, double *out) {
  __shared__ float4 tile[256];
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const bool valid = k < nr;
  double rx = 0, ry = 0;
  if (valid) {
    rx = x[2 * k];
    ry = x[2 * k + 1];
  }
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (size_t base = 0; base < n; base += 256) {
    const size_t i = base + threadIdx.x;
    if (i < n) tile[threadIdx.x] = make_float4(p[i].x[0], p[i].x[1], p[i].Mass, p[i].Size);
    __syncthreads();
    const int cnt = (int)min((size_t)256, n - base);
    if (valid)
      for (int j = 0; j < cnt; ++j) {
        const float4 P = tile[j];
        const double x0 = (double)P.x - rx, x1 = (double)P.y - ry;
        double rcm2 = x0 * x0 + x1 * x1;
        if (rcm2 < 1e-20) rcm2 = 1e-20;
        const double m = (double)P.z, ir2 = 1.0 / rcm2, prefac = m * ir2 * (1.0 / kPi);
        acc[0] += (inv_area * m - prefac) * x0;
        acc[1] += (inv_area * m - prefac) * x1;
        const double tmp = -2.0 * prefac * ir2;
        acc[3] += 0.5 * (x0 * x0 - x1 * x1) * tmp;
        acc[4] += x0 * x1 * tmp;
        acc[2] -= m * inv_area;
        const double size = (double)P.w;
        if (rcm2 < 4 * size * size) bspline_f64<false>(x0, x1, sqrt(rcm2), m, size, 0.0, acc);
      }
    __syncthreads();
  }
  if (valid)
    for (int c = 0; c < 5; ++c) out[5 * k + c] = acc[c];
}

// GridMap::writePixelMap (include/gridmap.h:529-598): one map pixel per grid
// point, the quantity selected by LensingVariable (include/standard.h:89-102):
// 0 DELAYT (0 on this path), 1 ALPHA = |x - y|, 2 ALPHA1, 3 ALPHA2,
// 4 KAPPA = 1 - (a0 + a3)/2, 5 GAMMA = |(gamma1, gamma2)|, 6 GAMMA1 = (a0 - a3)/2,
// 7 GAMMA2 = (a1 + a2)/2, 8 GAMMA3 = (a2 - a1)/2, 9 INVMAG = a0 a3 - a1 a2
// (include/point.h:377-381, 446-448).
__device__ inline double lensing_value(const double *x, const double *y, const double *A, size_t i, int var) {
  const double a0 = A[4 * i], a1 = A[4 * i + 1], a2 = A[4 * i + 2], a3 = A[4 * i + 3];
  const double d0 = x[2 * i] - y[2 * i], d1 = x[2 * i + 1] - y[2 * i + 1];
  double v = 0;
  switch (var) {
    case 1: v = sqrt(d0 * d0 + d1 * d1); break;
    case 2: v = d0; break;
    case 3: v = d1; break;
    case 4: v = 1 - (a0 + a3) / 2; break;
    case 5: {
      const double g1 = (a0 - a3) / 2, g2 = (a1 + a2) / 2;
      v = sqrt(g1 * g1 + g2 * g2);
      break;
    }
    case 6: v = (a0 - a3) / 2; break;
    case 7: v = (a1 + a2) / 2; break;
    case 8: v = (a2 - a1) / 2; break;
    case 9: v = a0 * a3 - a1 * a2; break;
    default: v = 0; break;  // DELAYT: dt = 0
  }
  return v;
}

__global__ void k_pixelmap(const double *x, const double *y, const double *A, size_t n, int var, double *map) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  map[i] = lensing_value(x, y, A, i, var);
}

// GridMap::writePixelMapUniform (include/gridmap.h:506-690): every grid point
// writes its value into the pixel PixelMap::find_index gives for its image
// position (ImageProcessing/pixelmap.cpp: the map's lower corner
// p1 = center - N res / 2, ix = (long)((x - p1) / res), -1 outside).  Where
// several grid points share a pixel the reference keeps the last one written;
// here that is the largest grid index (the order of one thread).
struct UniformMap {
  double p10, p11, res;
  long long nx, ny;
};
__device__ inline long long uniform_pixel(const UniformMap &M, double x0, double x1) {
  const long long ix = (long long)((x0 - M.p10) / M.res), iy = (long long)((x1 - M.p11) / M.res);
  if (ix < 0 || ix >= M.nx || iy < 0 || iy >= M.ny) return -1;
  return ix + M.nx * iy;
}
__global__ void k_uniform_owner(const double *x, size_t n, UniformMap M, long long *owner) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long p = uniform_pixel(M, x[2 * i], x[2 * i + 1]);
  if (p >= 0) atomicMax(owner + p, (long long)i);
}
__global__ void k_uniform_write(const double *x, const double *y, const double *A, size_t n, int var, UniformMap M,
                                const long long *owner, double *map) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long p = uniform_pixel(M, x[2 * i], x[2 * i + 1]);
  if (p >= 0 && owner[p] == (long long)i) map[p] = lensing_value(x, y, A, i, var);
}

// Source::SurfaceBrightness at the source-plane positions y:
// kind 0 SourceUniform (AnalyticNSIE/source.cpp:207-209): 1 inside radius q[0];
// kind 1 SourceGaussian (source.cpp:211-213): exp(-|y - x|^2 / q[0]) (q[0] = r^2);
// kind 2 SourceSersic (Source/sersic.cpp:116-135) with the host-derived
// constants q = {cosPA, sinPA, 1/q^2, flux I_n I_q I_r, bn, 1/Reff, 1/index, sb_limit}.
struct SourceDev {
  int kind;
  double x, y;
  double q[8];
};
__global__ void k_surface_brightness(const double *y, size_t n, SourceDev S, double *sb) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double d0 = y[2 * i] - S.x, d1 = y[2 * i + 1] - S.y;
  double v;
  if (S.kind == 0) {
    v = (d0 * d0 + d1 * d1) < S.q[0] * S.q[0] ? 1.0 : 0.0;
  } else if (S.kind == 1) {
    v = exp(-(d0 * d0 + d1 * d1) / S.q[0]);
  } else {
    const double x0 = d0 * S.q[0] + d1 * S.q[1], x1 = d0 * S.q[1] - d1 * S.q[0];
    double r = sqrt(x0 * x0 + x1 * x1 * S.q[2]);
    if (r < 4.848136811e-9) r = 4.848136811e-9;
    v = S.q[3] * exp(-S.q[4] * pow(r * S.q[5], S.q[6]));
    if (v < S.q[7]) v = 0.0;
  }
  sb[i] = v;
}

inline int nblk(size_t n, int t) { return (int)((n + t - 1) / t); }

}  // namespace

// ================================================================ host side
namespace {

HaloDev make_halo_dev(const glb_halo &h) {
  HaloDev d;
  memset(&d, 0, sizeof(d));
  d.kind = h.kind;
  d.px = h.theta[0] * h.Dist;  // LensHalo::getX (include/lens_halos.h:95-99)
  d.py = h.theta[1] * h.Dist;
  if (h.tree) d.tree = h.tree->dev;
  if (h.field) d.htree = h.field->dev;
  d.nfw = h.nfw;
  d.nsie = h.nsie;
  return d;
}

int set_dev(int device) {
  CKR(cudaSetDevice(device));
  return 0;
}

// Lens::combinePlanes (MultiPlane/lens.cpp:2397-2515): field and main planes
// sorted together by Dl (field planes first among equal distances), planes
// closer than MIN_PLANE_DIST pushed apart, the source pseudo-plane appended.
void combine_planes(glb_lens *l) {
  std::vector<std::pair<double, PlaneHost *>> all;
  for (PlaneHost &p : l->field) all.emplace_back(p.Dl, &p);
  for (PlaneHost &p : l->main) all.emplace_back(p.Dl, &p);
  std::stable_sort(all.begin(), all.end(),
                   [](const std::pair<double, PlaneHost *> &a, const std::pair<double, PlaneHost *> &b) {
                     return a.first < b.first;
                   });
  size_t n = all.size();
  l->planes.resize(n);
  l->plane_z.assign(n + 1, 0);
  l->Dl.assign(n + 1, 0);
  l->dDl.assign(n + 1, 0);
  for (size_t i = 0; i < n; ++i) {
    l->planes[i] = all[i].second;
    l->Dl[i] = all[i].first;
  }
  for (size_t i = 1; i < n; ++i)
    if ((l->Dl[i] - l->Dl[i - 1]) < 1e-6) l->Dl[i] = l->Dl[i - 1] + 1e-6;  // MIN_PLANE_DIST
  for (size_t i = 0; i < n; ++i) l->plane_z[i] = l->planes[i]->z;
  l->plane_field.assign(n, 0);
  for (size_t i = 0; i < n; ++i)
    for (const glb_halo *h : l->planes[i]->halos) l->plane_field[i] |= h->kind == HALO_FIELD;
  if (n > 0 && l->zsource <= l->plane_z[n - 1]) l->zsource = l->plane_z[n - 1] + 0.1;
  l->plane_z[n] = l->zsource;
  l->Dl[n] = coordist2(l->cosmo, 0, l->zsource);
  l->dDl[0] = l->Dl[0];
  for (size_t i = 1; i <= n; ++i) l->dDl[i] = l->Dl[i] - l->Dl[i - 1];
  l->dirty = true;
}

int upload_lens(glb_lens *l) {
  std::lock_guard<std::mutex> lk(l->mu);
  if (!l->dirty) return 0;
  size_t np = l->planes.size();
  std::vector<PlaneDev> P(np);
  std::vector<HaloDev> H;
  for (size_t j = 0; j < np; ++j) {
    PlaneDev &p = P[j];
    p.Dphys = l->Dl[j] / (1 + l->plane_z[j]);
    p.Gfac = l->charge * l->Dl[j] / (1 + l->plane_z[j]);
    p.aa = l->dDl[j + 1] / l->Dl[j + 1];
    p.bb = l->Dl[j] / l->Dl[j + 1];
    p.halo0 = (int)H.size();
    p.nhalo = (int)l->planes[j]->halos.size();
    for (glb_halo *h : l->planes[j]->halos) H.push_back(make_halo_dev(*h));
  }
  CKR(l->d_planes.alloc(std::max<size_t>(np, 1)));
  CKR(l->d_halos.alloc(std::max<size_t>(H.size(), 1)));
  CKR(l->d_planez.alloc(np + 1));
  CKR(l->d_Dl.alloc(np + 1));
  if (np) CKR(cudaMemcpyAsync(l->d_planes.p, P.data(), np * sizeof(PlaneDev), cudaMemcpyHostToDevice, l->stream));
  if (!H.empty())
    CKR(cudaMemcpyAsync(l->d_halos.p, H.data(), H.size() * sizeof(HaloDev), cudaMemcpyHostToDevice, l->stream));
  CKR(cudaMemcpyAsync(l->d_planez.p, l->plane_z.data(), (np + 1) * sizeof(double), cudaMemcpyHostToDevice,
                      l->stream));
  CKR(cudaMemcpyAsync(l->d_Dl.p, l->Dl.data(), (np + 1) * sizeof(double), cudaMemcpyHostToDevice, l->stream));
  CKR(cudaStreamSynchronize(l->stream));
  l->dirty = false;
  return 0;
}

// The calling thread's workspace on lens l (created on its first call).
int thread_ws(glb_lens *l, LensWS **out) {
  std::lock_guard<std::mutex> lk(l->mu);
  std::unique_ptr<LensWS> &w = l->ws[std::this_thread::get_id()];
  if (!w) {
    auto n = std::make_unique<LensWS>();
    n->device = l->device;
    CKR(cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking));
    for (int i = 0; i < 4; ++i) CKR(cudaEventCreate(&n->ev[i]));
    CKR(cudaEventCreateWithFlags(&n->done, cudaEventDisableTiming));
    w = std::move(n);
  }
  *out = w.get();
  return 0;
}

int ensure_ws(LensWS *w, size_t n, bool per_ray) {
  if (n > 0xffffffffull) return fail(GLB_ERR_ARG, "too many rays in one call (max 2^32-1)");
  if (w->ws_n < n || (per_ray && w->jmax_ray.n < n)) {
    size_t m = std::max(n, w->ws_n);
    CKR(w->st.alloc(12 * m));
    CKR(w->keys.alloc(m));
    CKR(w->keys2.alloc(m));
    CKR(w->perm0.alloc(m));
    CKR(w->perm.alloc(m));
    CKR(w->jmax_ray.alloc(m));
    CKR(w->src_ray.alloc(2 * m));
    size_t tb = 0;
    CKR(cub::DeviceRadixSort::SortPairs(nullptr, tb, w->keys.p, w->keys2.p, w->perm0.p, w->perm.p, (int)m, 0, 32,
                                        w->stream));
    CKR(w->sort_tmp.alloc(tb));
    CKR(w->bbox.alloc(4));
    w->ws_n = m;
  }
  return 0;
}

// One launch per plane, in order.  Split-form planes that hold exactly one
// particle halo and no field plane run the group walk (k_plane_step_split_g,
// the tree in the kernel parameters); planes with a field plane use the FIELD
// instances.
constexpr size_t kTwoRayMin = (size_t)1 << 20;  // two-ray tree-force kernel from this many rays on
int launch_plane_steps(const glb_lens *l, StepArgs &a, int jmax_launch, int precision, cudaStream_t s,
                       const unsigned long long *d_counts) {
  const size_t n = a.n;
  for (int j = 0; j < jmax_launch; ++j) {
    a.j = j;
    const bool fld = l->plane_field[j] != 0;
    int npart = 0;
    const glb_halo *ph = nullptr;
    for (const glb_halo *h : l->planes[j]->halos)
      if (h->kind == HALO_PARTICLES) {
        ++npart;
        ph = h;
      }
    const bool ptree = npart == 1 && ph->tree && !fld && !ph->tree->dev.periodic;  // the group walk has no periodic images
    memset(&a.tree, 0, sizeof(a.tree));
    a.tree_px = a.tree_py = 0;
    if (ptree) {
      a.tree = ph->tree->dev;
      a.tree_px = ph->theta[0] * ph->Dist;  // LensHalo::getX, as make_halo_dev
      a.tree_py = ph->theta[1] * ph->Dist;
    }
    if (d_counts && fld)
      k_plane_step<GLB_PREC_FP64, true, true><<<nblk(n, 128), 128, 0, s>>>(a);
    else if (d_counts)
      k_plane_step<GLB_PREC_FP64, true><<<nblk(n, 128), 128, 0, s>>>(a);
    else if (precision == GLB_PREC_SPLIT && fld)
      k_plane_step_split<true><<<nblk(n, 128), 128, 0, s>>>(a);
    else if (precision == GLB_PREC_SPLIT && ptree)
      k_plane_step_split_g<<<nblk(n, 128), 128, 0, s>>>(a);
    else if (precision == GLB_PREC_SPLIT)
      k_plane_step_split<<<nblk(n, 128), 128, 0, s>>>(a);
    else if (fld)
      k_plane_step<GLB_PREC_FP64, false, true><<<nblk(n, 128), 128, 0, s>>>(a);
    else
      k_plane_step<GLB_PREC_FP64><<<nblk(n, 128), 128, 0, s>>>(a);
  }
  CKR(cudaGetLastError());
  return 0;
}

// Calls of at least 2 kSlabMin rays run as kMaxSlabs slabs of consecutive
// sorted rays (multiples of 64 rays, so rays pair as in an uncut call), each
// slab's state set-up, plane steps and results on its own stream.  A slab's
// launches depend only on its own earlier ones, so while one slab's launch
// drains its last blocks the other slab's blocks fill the idle SMs, and the
// per-plane launch tails overlap instead of adding up.  Measured on the
// 2048^2 light cone (split form) with the two-ray walk: 740 ms per step in one
// piece, 728 ms in two slabs, 729 ms in four; with the group walk 647 ms in
// one piece, 644 ms in two; results bit-identical.
constexpr int kMaxSlabs = 2;
constexpr size_t kSlabMin = (size_t)1 << 20;

int ensure_slab_streams(LensWS *w, int nslabs) {
  for (int i = 0; i + 1 < nslabs; ++i) {
    if (!w->sub[i]) CKR(cudaStreamCreateWithFlags(&w->sub[i], cudaStreamNonBlocking));
    if (!w->join[i]) CKR(cudaEventCreateWithFlags(&w->join[i], cudaEventDisableTiming));
  }
  return 0;
}

// The whole ray-shooting pass on device buffers, enqueued on stream s.
// The workspace w is the calling thread's; a pass first waits for the end of
// its previous pass (which may have run on another stream), since both use
// w's buffers.
int rayshoot_device(glb_lens *l, LensWS *w, size_t n, const double *x, const double *zs, double *y, double *A,
                    int precision, cudaStream_t s, unsigned long long *d_counts = nullptr,
                    unsigned char *status = nullptr, const unsigned char *skip = nullptr) {
  if (n == 0) return 0;
  size_t np = l->planes.size();
  if (np == 0) {  // no lens plane (internal_rayshooter_multi.cpp:62-76)
    k_identity_rays<<<nblk(n, 256), 256, 0, s>>>(x, n, y, A, status, skip);
    CKR(cudaGetLastError());
    return 0;
  }
  if (int rc = upload_lens(l)) return rc;
  if (int rc = ensure_ws(w, n, zs != nullptr)) return rc;
  CKR(cudaStreamWaitEvent(s, w->done, 0));
  CKR(cudaEventRecord(w->ev[0], s));
  // spatial ordering of the rays along a Morton curve
  if (n >= 64) {
    unsigned long long init[4] = {~0ull, ~0ull, 0ull, 0ull};
    CKR(cudaMemcpyAsync(w->bbox.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
    k_ray_bbox<<<std::min(nblk(n, 256), 1184), 256, 0, s>>>(x, n, w->bbox.p);
    k_ray_morton<<<nblk(n, 256), 256, 0, s>>>(x, n, w->bbox.p, w->keys.p, w->perm0.p);
    size_t tb = w->sort_tmp.n;
    CKR(cub::DeviceRadixSort::SortPairs(w->sort_tmp.p, tb, w->keys.p, w->keys2.p, w->perm0.p, w->perm.p, (int)n, 0,
                                        32, s));
  } else {
    k_identity<<<nblk(n, 256), 256, 0, s>>>(w->perm.p, n);
  }
  SrcArgs sa{l->cosmo, l->d_planez.p, l->d_Dl.p, (int)np};

  StepArgs a;
  a.planes = l->d_planes.p;
  a.halos = l->d_halos.p;
  if (int rc = device_nfw_tables(a.tab)) return rc;
  a.st = w->st.p;
  a.n = n;
  a.charge = l->charge;
  a.counts = d_counts;
  a.jmax_ray = zs ? w->jmax_ray.p : nullptr;
  a.src_ray = zs ? w->src_ray.p : nullptr;
  int jmax_launch = (int)np;
  a.jmax = (int)np;
  a.dls_ds = 0;
  a.d_ds = 0;
  if (!zs) {
    // Point* overload: compute_points_parallel's !multiZs branch (lens.h:944-955)
    double source_z = l->toggle_source_plane ? l->zs_implant : l->plane_z.back();
    if (source_z == l->plane_z.back()) {
      a.dls_ds = l->dDl.back() / l->Dl.back();
      a.d_ds = l->Dl[np - 1] / l->Dl.back();
    } else {
      double Ds = coordist(l->cosmo, source_z), Dls;
      int jm;
      if (source_z <= l->plane_z[0]) {
        jm = 0;
        Dls = Ds;
      } else {
        jm = (int)np;
        while (l->plane_z[jm - 1] > source_z) --jm;
        Dls = coordist2(l->cosmo, l->plane_z[jm - 1], source_z);
      }
      a.jmax = jm;
      a.dls_ds = Dls / Ds;
      if (jm > 0) a.d_ds = l->Dl[jm - 1] / Ds;
      jmax_launch = jm;
    }
  }
  const int nslabs = d_counts ? 1 : (int)std::max<size_t>(1, std::min<size_t>(kMaxSlabs, n / kSlabMin));
  if (int rc = ensure_slab_streams(w, nslabs)) return rc;
  const size_t m = ((n + nslabs - 1) / nslabs + 63) / 64 * 64;
  CKR(cudaEventRecord(w->ev[1], s));  // also the slabs' start
  for (int i = 0; i < nslabs && (size_t)i * m < n; ++i) {
    const size_t o = i * m, mi = std::min(m, n - o);
    cudaStream_t si = i == 0 ? s : w->sub[i - 1];
    if (i > 0) CKR(cudaStreamWaitEvent(si, w->ev[1], 0));
    k_init_state<<<nblk(mi, 256), 256, 0, si>>>(x, zs, w->perm.p + o, mi, w->st.p + 12 * o, w->jmax_ray.p + o,
                                               w->src_ray.p + 2 * o, sa);
    StepArgs ai = a;
    ai.st = w->st.p + 12 * o;
    ai.n = mi;
    ai.jmax_ray = zs ? w->jmax_ray.p + o : nullptr;
    ai.src_ray = zs ? w->src_ray.p + 2 * o : nullptr;
    if (int rc = launch_plane_steps(l, ai, jmax_launch, precision, si, d_counts)) return rc;
    k_finish<<<nblk(mi, 256), 256, 0, si>>>(ai.st, w->perm.p + o, mi, y, A, status, skip);
    if (i > 0) {
      CKR(cudaEventRecord(w->join[i - 1], si));
      CKR(cudaStreamWaitEvent(s, w->join[i - 1], 0));
    }
  }
  CKR(cudaEventRecord(w->ev[2], s));
  CKR(cudaEventRecord(w->ev[3], s));
  CKR(cudaEventRecord(w->done, s));
  w->timed = true;
  CKR(cudaGetLastError());
  return 0;
}

}  // namespace

// ===================================================================== C ABI
extern "C" {

const char *glb_last_error(void) { return t_err.c_str(); }
const char *glb_version(void) { return "glamer_b200 0.1 (sm_100a)"; }

int glb_set_option(int option, long long value) {
  if (option == GLB_OPT_KEEP_TREE_EXPORT) {
    g_keep_tree_export = value ? 1 : 0;
    return 0;
  }
  return fail(GLB_ERR_ARG, "unknown option");
}

// ------------------------------------------------------------------ trees
struct glb_tree {
  std::unique_ptr<Tree> tree;
  int device = 0;
  cudaStream_t stream = nullptr;
};

int glb_tree_create(const glb_particle *particles, size_t n, float mass_fixed, float size_fixed, double inv_area,
                    int bucket, double theta_force, int periodic_buffer, double inv_screening_scale,
                    double maximum_range, glb_tree **out) {
  if (!out || (n > 0 && !particles)) return fail(GLB_ERR_ARG, "null argument");
  if (bucket < 1) return fail(GLB_ERR_ARG, "bucket must be >= 1");
  if (int rc = need_device()) return rc;
  auto t = std::make_unique<glb_tree>();
  CKR(cudaGetDevice(&t->device));
  CKR(cudaStreamCreateWithFlags(&t->stream, cudaStreamNonBlocking));
  TreeParams prm;
  prm.mass_fixed = mass_fixed;
  prm.size_fixed = size_fixed;
  prm.inv_area = inv_area;
  prm.bucket = bucket;
  prm.theta = theta_force;
  prm.periodic = periodic_buffer;
  prm.inv_screening = inv_screening_scale;
  prm.max_range = maximum_range;
  Status s = build_tree(reinterpret_cast<const glb_particle_rec *>(particles), n, prm, g_keep_tree_export != 0,
                        t->stream, t->tree);
  if (!s.good()) {
    cudaStreamDestroy(t->stream);
    return fail(s);
  }
  *out = t.release();
  return 0;
}

int glb_tree_destroy(glb_tree *t) {
  if (!t) return 0;
  cudaSetDevice(t->device);
  t->tree.reset();
  if (t->stream) cudaStreamDestroy(t->stream);
  delete t;
  return 0;
}

static int force_generic(const HaloDev &H, int device, cudaStream_t s, size_t n, const double *xcm, double *alpha,
                         double *kappa, double *gamma, double *phi, int subtract = 0, double screening = 1.0) {
  if (n == 0) return 0;
  if (!xcm) return fail(GLB_ERR_ARG, "null positions");
  if (int rc = set_dev(device)) return rc;
  NFWTables tab{};
  if (H.kind == HALO_NFW || H.kind == HALO_FIELD)
    if (int rc = device_nfw_tables(tab)) return rc;
  DBuf<double> dx, dout;
  CKR(dx.alloc(2 * n));
  CKR(dout.alloc(6 * n));
  CKR(cudaMemcpyAsync(dx.p, xcm, 2 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  k_halo_force<<<nblk(n, 128), 128, 0, s>>>(H, tab, n, dx.p, dout.p, subtract, screening);
  CKR(cudaGetLastError());
  std::vector<double> o(6 * n);
  CKR(cudaMemcpyAsync(o.data(), dout.p, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CKR(cudaStreamSynchronize(s));
  for (size_t i = 0; i < n; ++i) {
    if (alpha) {
      alpha[2 * i] = o[6 * i];
      alpha[2 * i + 1] = o[6 * i + 1];
    }
    if (kappa) kappa[i] = o[6 * i + 2];
    if (gamma) {
      gamma[3 * i] = o[6 * i + 3];
      gamma[3 * i + 1] = o[6 * i + 4];
      gamma[3 * i + 2] = 0.0;
    }
    if (phi) phi[i] = o[6 * i + 5];
  }
  return 0;
}

int glb_tree_force2D_recur(glb_tree *t, size_t n, const double *rays, double *alpha, double *kappa, double *gamma,
                           double *phi) {
  if (!t) return fail(GLB_ERR_ARG, "null tree");
  HaloDev H;
  memset(&H, 0, sizeof(H));
  H.kind = HALO_PARTICLES;
  H.tree = t->tree->dev;
  if (t->tree->nparticles == 0) {
    for (size_t i = 0; i < n; ++i) {
      if (alpha) alpha[2 * i] = alpha[2 * i + 1] = 0;
      if (kappa) kappa[i] = 0;
      if (gamma) gamma[3 * i] = gamma[3 * i + 1] = gamma[3 * i + 2] = 0;
      if (phi) phi[i] = 0;
    }
    return 0;
  }
  return force_generic(H, t->device, t->stream, n, rays, alpha, kappa, gamma, phi);
}

int glb_tree_force_device(glb_tree *t, size_t n, const double *rays_dev, double *out_dev, int precision,
                          void *stream) {
  if (!t || (n > 0 && (!rays_dev || !out_dev))) return fail(GLB_ERR_ARG, "null argument");
  if (precision < GLB_PREC_FP64 || precision > GLB_PREC_FP32) return fail(GLB_ERR_ARG, "unknown precision");
  if (int rc = set_dev(t->device)) return rc;
  if (n == 0) return 0;
  cudaStream_t s = stream ? (cudaStream_t)stream : t->stream;
  if (t->tree->nparticles == 0) {
    CKR(cudaMemsetAsync(out_dev, 0, 5 * n * sizeof(double), s));
    return 0;
  }
  (void)cudaGetLastError();
  if (precision == GLB_PREC_FP64)
    k_tree_force<<<nblk(n, 128), 128, 0, s>>>(t->tree->dev, n, rays_dev, out_dev);
  else if (precision == GLB_PREC_SPLIT && !t->tree->dev.periodic && n >= kTwoRayMin && t->tree->theta < 0.2)
    k_tree_force_split2<<<nblk((n + 1) / 2, 128), 128, 0, s>>>(t->tree->dev, n, rays_dev, out_dev);
  else if (precision == GLB_PREC_SPLIT)
    k_tree_force_lo<GLB_PREC_SPLIT><<<nblk(n, 128), 128, 0, s>>>(t->tree->dev, n, rays_dev, out_dev);
  else
    k_tree_force_lo<GLB_PREC_FP32><<<nblk(n, 128), 128, 0, s>>>(t->tree->dev, n, rays_dev, out_dev);
  CKR(cudaGetLastError());
  return 0;
}

int glb_direct_sum_device(const glb_particle *particles_dev, size_t n, double inv_area, const double *rays_dev,
                          size_t nrays, double *out_dev, void *stream) {
  if ((n > 0 && !particles_dev) || (nrays > 0 && (!rays_dev || !out_dev))) return fail(GLB_ERR_ARG, "null argument");
  if (int rc = need_device()) return rc;
  if (nrays == 0) return 0;
  (void)cudaGetLastError();
  k_direct_sum<<<nblk(nrays, 256), 256, 0, (cudaStream_t)stream>>>(
      reinterpret_cast<const glb_particle_rec *>(particles_dev), n, inv_area, rays_dev, nrays, out_dev);
  CKR(cudaGetLastError());
  return 0;
}

int glb_tree_export(glb_tree *t, size_t *nbranches, double *out) {
  if (!t || !nbranches) return fail(GLB_ERR_ARG, "null argument");
  *nbranches = t->tree->nbranches;
  if (!out) return 0;
  if (t->tree->export_rows.size() != 16 * t->tree->nbranches)
    return fail(GLB_ERR_ARG, "tree built without GLB_OPT_KEEP_TREE_EXPORT");
  memcpy(out, t->tree->export_rows.data(), t->tree->export_rows.size() * sizeof(double));
  return 0;
}

int glb_tree_build_ms(glb_tree *t, double *ms) {
  if (!t || !ms) return fail(GLB_ERR_ARG, "null argument");
  *ms = t->tree->build_ms;
  return 0;
}

// ------------------------------------------------------------------ halos
static int new_halo(std::unique_ptr<glb_halo> &h) {
  if (int rc = need_device()) return rc;
  h = std::make_unique<glb_halo>();
  CKR(cudaGetDevice(&h->device));
  CKR(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  return 0;
}

int glb_halo_particles(const glb_particle *particles, size_t n, double z, double inv_area, double max_range,
                       glb_halo **out) {
  if (!out || (n > 0 && !particles)) return fail(GLB_ERR_ARG, "null argument");
  std::unique_ptr<glb_halo> h;
  if (int rc = new_halo(h)) return rc;
  h->kind = HALO_PARTICLES;
  h->zlens = (double)(float)z;  // the vector constructor takes a float redshift
  // the cosmology is bound when the halo enters a lens (Dist is reset there)
  double m = 0;
  for (size_t i = 0; i < n; ++i) m += particles[i].Mass;  // set_up, particle_halo.h:366-378
  h->mass = (float)m;
  h->Rsize = h->Rmax = (float)1.0e100;
  TreeParams prm;
  prm.inv_area = inv_area;
  prm.bucket = 20;        // particle_halo.h:416
  prm.theta = 0.1;
  prm.periodic = 0;
  prm.inv_screening = max_range;  // the ninth argument there is inv_screening_scale
  prm.max_range = -1;
  Status s = build_tree(reinterpret_cast<const glb_particle_rec *>(particles), n, prm, g_keep_tree_export != 0,
                        h->stream, h->tree);
  if (!s.good()) return fail(s);
  *out = h.release();
  return 0;
}

int glb_halo_nfw(float mass, float Rsize, double z, float concentration, float fratio, float pa, glb_halo **out) {
  if (!out) return fail(GLB_ERR_ARG, "null argument");
  if (fratio != 1.0f)
    return fail(GLB_ERR_UNSUPPORTED, "elliptical NFW (fratio != 1) is outside this library's scope");
  if (!(concentration > 0) || !(Rsize > 0)) return fail(GLB_ERR_ARG, "Rsize and concentration must be positive");
  std::unique_ptr<glb_halo> h;
  if (int rc = new_halo(h)) return rc;
  std::call_once(g_nfw_host_once, make_host_tables);
  h->kind = HALO_NFW;
  h->zlens = z;
  h->Rsize = Rsize;
  h->mass = mass;
  h->rscale = h->Rsize / concentration;  // float / float (lens_halos.cpp:411)
  double xmax = (double)(h->Rsize / h->rscale);
  if (xmax >= kNfwMaxRm * (kNfwTable - 1) / kNfwTable)
    return fail(GLB_ERR_ARG, "concentration beyond the reference's NFW table");
  double gmax = nfw_interp_host(1, xmax);
  h->Rmax = h->Rsize;  // fratio == 1 (lens_halos.cpp:425-428)
  NFWDev &d = h->nfw;
  d.mass = h->mass;
  d.rscale = h->rscale;
  d.gmax = gmax;
  d.Rmax2 = (double)(h->Rmax * h->Rmax);
  d.h_xmax = nfw_interp_host(3, (double)(h->Rsize / h->rscale));
  d.log_rsize = (double)logf(h->Rsize);  // log of a float member: the float overload
  (void)pa;
  *out = h.release();
  return 0;
}

// LensHalo::MassBy1DIntegation (lens_halos.cpp:2469-2473): R/2 times the
// angular integral of the inward radial deflection on the circle R; the
// integrand is smooth and periodic, so a 4096-point trapezoid rule is used.
static double nsie_mass_1d(const NSIEDev &d, double R) {
  const int NQ = 4096;
  double sum = 0;
  for (int i = 0; i < NQ; ++i) {
    double th = 2 * kPi * i / NQ;
    double out[6] = {0, 0, 0, 0, 0, 0};
    nsie_force<false>(d, R * cos(th), R * sin(th), out);
    sum += -out[0] * cos(th) - out[1] * sin(th);
  }
  return R * (sum * 2 * kPi / NQ) / 2;
}

int glb_halo_nsie(float mass, double z, float sigma, float rcore, float fratio, float pa, glb_halo **out) {
  if (!out) return fail(GLB_ERR_ARG, "null argument");
  if (fratio > 1.0f || fratio < 0.01f) return fail(GLB_ERR_ARG, "invalid fratio");  // lens_halos.cpp:1072
  if (!(sigma > 0)) return fail(GLB_ERR_ARG, "sigma must be positive");
  std::unique_ptr<glb_halo> h;
  if (int rc = new_halo(h)) return rc;
  h->kind = HALO_NSIE;
  h->rscale = 1.0f;
  h->mass = mass;
  h->zlens = z;
  float pa_m = (float)(kPi / 2 - pa);  // lens_halos.cpp:1058
  // rmax_calc (lens_halos.cpp:1154-1171)
  double rs;
  if (fratio == 1.0f || rcore > 0.0f) {
    float sf = sqrtf(fratio);
    double a = (double)h->mass * kGrav * kLightspeed * kLightspeed * (double)sf / kPi / (double)sigma /
                   (double)sigma + (double)rcore;
    rs = sqrt(pow(a, 2) - (double)(rcore * rcore));
  } else {
    // elliptic-integral normalisation: (2/pi) int_0^{pi/2} dt / sqrt(1 + (q^2-1) sin^2 t)
    // = 1 / AGM(1, q), interpolated linearly on the reference's 200-point q table
    auto F = [](double q) {
      double a = 1.0, b = q;
      for (int i = 0; i < 40; ++i) {
        double an = 0.5 * (a + b), bn = sqrt(a * b);
        a = an;
        b = bn;
      }
      return 1.0 / a;
    };
    const int N = 200;
    std::vector<double> qt(N), Ft(N);
    qt[0] = 0.01;
    Ft[0] = F(0.01);
    for (int i = 1; i < N - 1; ++i) {
      qt[i] = i * 1.0 / (N - 1);
      Ft[i] = F(qt[i]);
    }
    qt[N - 1] = 1.0;
    Ft[N - 1] = 1.0;
    double q = fratio;
    int i = 0;
    while (i < N - 2 && qt[i + 1] <= q) ++i;
    double ell = (Ft[i] + (Ft[i + 1] - Ft[i]) * (q - qt[i]) / (qt[i + 1] - qt[i])) * sqrt((double)fratio);
    rs = (double)h->mass * kGrav * kLightspeed * kLightspeed / kPi / (double)sigma / (double)sigma / ell;
  }
  h->Rsize = (float)rs;
  h->Rmax = 1.2f * h->Rsize;
  float units = (float)(pow((double)sigma / kLightspeed, 2) / kGrav);
  NSIEDev &d = h->nsie;
  d.f = (double)fratio;
  d.bc = (double)rcore;
  d.sqrt_f = sqrt(d.f);
  d.fp = sqrt(1 - d.f * d.f);
  double p = (double)pa_m;
  d.c1 = cos(p);
  d.s1 = sin(p);
  d.c2 = cos(-p);
  d.s2 = sin(-p);
  d.c3 = cos(-2 * p);
  d.s3 = sin(-2 * p);
  d.c0 = 1.0;
  d.s0 = 0.0;
  d.units = (double)units;
  d.Rsize = (double)h->Rsize;
  d.Rmax = (double)h->Rmax;
  d.Rsize2 = (double)(h->Rsize * h->Rsize);
  d.Rmax2 = (double)(h->Rmax * h->Rmax);
  d.dRmaxRsize = (double)(h->Rmax - h->Rsize);
  d.mass = (double)h->mass;
  // A cored halo's mass is reset by 1D integration (lens_halos.cpp:1073-1075)
  // with `units` already assigned.
  if (rcore > 0.0f) {
    h->mass = (float)nsie_mass_1d(d, (double)h->Rsize);
    d.mass = (double)h->mass;
  }
  *out = h.release();
  return 0;
}

int glb_halo_nsie_state(float mass, float Rsize, float Rmax, double z, float sigma, float rcore, float fratio,
                        float pa_internal, glb_halo **out) {
  if (!out) return fail(GLB_ERR_ARG, "null argument");
  if (!(Rsize > 0) || !(Rmax >= Rsize)) return fail(GLB_ERR_ARG, "need 0 < Rsize <= Rmax");
  // the constructor's arithmetic for everything but the size, the mass and the
  // angle, which are then set to the values the mirrored halo holds
  glb_halo *h = nullptr;
  if (int rc = glb_halo_nsie(mass, z, sigma, 0.0f, fratio, 0.0f, &h)) return rc;
  h->mass = mass;
  h->Rsize = Rsize;
  h->Rmax = Rmax;
  NSIEDev &d = h->nsie;
  d.bc = (double)rcore;
  const double p = (double)pa_internal;
  d.c1 = cos(p);
  d.s1 = sin(p);
  d.c2 = cos(-p);
  d.s2 = sin(-p);
  d.c3 = cos(-2 * p);
  d.s3 = sin(-2 * p);
  d.Rsize = (double)Rsize;
  d.Rmax = (double)Rmax;
  d.Rsize2 = (double)(Rsize * Rsize);
  d.Rmax2 = (double)(Rmax * Rmax);
  d.dRmaxRsize = (double)(Rmax - Rsize);
  d.mass = (double)mass;
  *out = h;
  return 0;
}

int glb_halo_set_theta(glb_halo *h, double tx, double ty) {
  if (!h) return fail(GLB_ERR_ARG, "null halo");
  if (h->kind == HALO_FIELD) return fail(GLB_ERR_ARG, "a field plane has no position of its own");
  h->theta[0] = tx;
  h->theta[1] = ty;
  return 0;
}

int glb_halo_force(glb_halo *h, size_t n, const double *xcm, double *alpha, double *kappa, double *gamma,
                   double *phi) {
  return glb_halo_force_ex(h, n, xcm, alpha, kappa, gamma, phi, 0, 1.0);
}

int glb_halo_force_ex(glb_halo *h, size_t n, const double *xcm, double *alpha, double *kappa, double *gamma,
                      double *phi, int subtract_point, double screening) {
  if (!h) return fail(GLB_ERR_ARG, "null halo");
  HaloDev H = make_halo_dev(*h);
  if (h->kind == HALO_PARTICLES && h->tree->nparticles == 0) {
    for (size_t i = 0; i < n; ++i) {
      if (alpha) alpha[2 * i] = alpha[2 * i + 1] = 0;
      if (kappa) kappa[i] = 0;
      if (gamma) gamma[3 * i] = gamma[3 * i + 1] = gamma[3 * i + 2] = 0;
      if (phi) phi[i] = 0;
    }
    return 0;
  }
  int rc = force_generic(H, h->device, h->stream, n, xcm, alpha, kappa, gamma, phi, subtract_point, screening);
  if (rc) return rc;
  if (h->kind == HALO_PARTICLES && alpha)  // LensHaloParticles::force_halo negates alpha
    for (size_t i = 0; i < 2 * n; ++i) alpha[i] = -alpha[i];
  return 0;
}

int glb_halo_params(glb_halo *h, float *mass, float *rsize, float *rmax) {
  if (!h) return fail(GLB_ERR_ARG, "null halo");
  if (mass) *mass = h->mass;
  if (rsize) *rsize = h->Rsize;
  if (rmax) *rmax = h->Rmax;
  return 0;
}

int glb_halo_destroy(glb_halo *h) {
  if (!h) return 0;
  cudaSetDevice(h->device);
  h->tree.reset();
  h->field.reset();
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return 0;
}

// ------------------------------------------------------------------- lens
int glb_lens_create(double zsource, double omega_m, double omega_l, double hubble, glb_lens **out) {
  if (!out) return fail(GLB_ERR_ARG, "null argument");
  if (omega_m + omega_l != 1.0)
    return fail(GLB_ERR_ARG, "Lens can only handle flat universes at present");  // lens.cpp:63-67
  if (int rc = need_device()) return rc;
  auto l = std::make_unique<glb_lens>();
  l->cosmo = Cosmo{omega_m, omega_l, hubble};
  l->zsource = zsource;
  l->charge = 4 * kPi * kGrav;  // lens.cpp:93
  CKR(cudaGetDevice(&l->device));
  CKR(cudaStreamCreateWithFlags(&l->stream, cudaStreamNonBlocking));
  combine_planes(l.get());
  *out = l.release();
  return 0;
}

int glb_lens_destroy(glb_lens *l) {
  if (!l) return 0;
  cudaSetDevice(l->device);
  l->ws.clear();  // each workspace synchronises its stream before it is freed
  if (l->stream) cudaStreamSynchronize(l->stream);
  for (auto &h : l->owned) {
    h->tree.reset();
    if (h->stream) cudaStreamDestroy(h->stream);
  }
  cudaStream_t s = l->stream;
  delete l;
  if (s) cudaStreamDestroy(s);
  return 0;
}

// TreeQuadHalos of a field plane for cosmology c: the member haloes are moved
// to the plane's redshift (LensHalo::setZlensDist, lens.cpp:418-426), their
// positions taken (LensHalo::getX) and the tree built on the host and
// uploaded.
static int build_field_tree(glb_halo *h, const Cosmo &c) {
  FieldTree &F = *h->field;
  const size_t n = F.members.size();
  const double Dist = angdist(c, h->zlens);
  h->Dist = Dist;
  std::vector<double> xp(2 * n);
  std::vector<float> rmax(n), mass(n);
  std::vector<FieldHaloDev> fh(n);
  for (size_t i = 0; i < n; ++i) {
    glb_halo *m = F.members[i].get();
    m->zlens = h->zlens;
    m->Dist = Dist;
    xp[2 * i] = m->theta[0] * Dist;
    xp[2 * i + 1] = m->theta[1] * Dist;
    rmax[i] = m->Rmax;
    mass[i] = m->mass;
    FieldHaloDev &d = fh[i];
    memset(&d, 0, sizeof(d));
    d.kind = m->kind;
    d.px = xp[2 * i];
    d.py = xp[2 * i + 1];
    d.mass = (double)m->mass;
    d.nfw = m->nfw;
    d.nsie = m->nsie;
  }
  HaloTreeHost T;
  std::string err;
  if (!build_halo_tree(xp, rmax, mass, F.bucket, F.theta, -1, T, err)) return fail(GLB_ERR_SAME_PLACE, err);
  if (int rc = set_dev(h->device)) return rc;
  CKR(F.nodes.alloc(std::max<size_t>(T.nodes.size(), 1)));
  CKR(F.bigs.alloc(std::max<size_t>(T.bigs.size(), 1)));
  CKR(F.halos.alloc(std::max<size_t>(n, 1)));
  if (!T.nodes.empty())
    CKR(cudaMemcpyAsync(F.nodes.p, T.nodes.data(), T.nodes.size() * sizeof(HNode), cudaMemcpyHostToDevice,
                        h->stream));
  if (!T.bigs.empty())
    CKR(cudaMemcpyAsync(F.bigs.p, T.bigs.data(), T.bigs.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream));
  if (n) CKR(cudaMemcpyAsync(F.halos.p, fh.data(), n * sizeof(FieldHaloDev), cudaMemcpyHostToDevice, h->stream));
  CKR(cudaStreamSynchronize(h->stream));
  HaloTreeDev &D = F.dev;
  D.nodes = F.nodes.p;
  D.bigs = F.bigs.p;
  D.halos = F.halos.p;
  D.nnodes = (int)T.nodes.size();
  D.nhalos = (int)n;
  D.inv_area = F.sigma_back;
  D.screen2 = F.inv_screening * F.inv_screening;
  D.periodic = F.periodic;
  D.period_x = T.period_x;
  D.period_y = T.period_y;
  return 0;
}

int glb_halo_field_plane(glb_halo *const *halos, int n, double z, double sigma_background,
                         double inv_screening_scale, glb_halo **out) {
  if (!out || n < 0 || (n > 0 && !halos)) return fail(GLB_ERR_ARG, "null argument");
  for (int i = 0; i < n; ++i) {
    if (!halos[i]) return fail(GLB_ERR_ARG, "null halo");
    if (halos[i]->kind != HALO_NFW && halos[i]->kind != HALO_NSIE)
      return fail(GLB_ERR_UNSUPPORTED, "field planes hold NFW and NSIE haloes only");
    for (int j = 0; j < i; ++j)
      if (halos[j] == halos[i]) return fail(GLB_ERR_ARG, "a halo appears twice");
  }
  std::unique_ptr<glb_halo> h;
  if (int rc = new_halo(h)) return rc;
  h->kind = HALO_FIELD;
  h->zlens = z;
  h->field = std::make_unique<FieldTree>();
  FieldTree &F = *h->field;
  F.sigma_back = sigma_background;
  F.inv_screening = inv_screening_scale;
  if (inv_screening_scale != 0) {  // planes.cpp:17
    F.bucket = 5;
    F.theta = 0.1;
    F.periodic = 1;
  } else {  // TreeQuadHalos defaults, include/quadTreeHalos.h:37-45
    F.bucket = 5;
    F.theta = 0.5;
    F.periodic = 0;
  }
  for (int i = 0; i < n; ++i) F.members.emplace_back(halos[i]);
  // built for the default cosmology here and again for a lens's when inserted
  if (int rc = build_field_tree(h.get(), Cosmo{0.3, 0.7, 0.7})) {
    for (auto &m : F.members) m.release();  // on failure the caller keeps its haloes
    return rc;
  }
  *out = h.release();
  return 0;
}

int glb_lens_insert_field_plane(glb_lens *l, glb_halo *plane) {
  if (!l || !plane) return fail(GLB_ERR_ARG, "null argument");
  if (plane->kind != HALO_FIELD) return fail(GLB_ERR_ARG, "not a field plane (glb_halo_field_plane)");
  if (int rc = build_field_tree(plane, l->cosmo)) return rc;
  l->owned.emplace_back(plane);
  l->field.push_back(PlaneHost{plane->zlens, coordist2(l->cosmo, 0, plane->zlens), {plane}});
  combine_planes(l);
  return 0;
}

// Lens::addMainHaloToPlane (lens.cpp:772-815) / addMainHaloToNearestPlane
// (lens.cpp:821-838), then combinePlanes.
int glb_lens_insert_halo(glb_lens *l, glb_halo *h, int addplanes) {
  if (!l || !h) return fail(GLB_ERR_ARG, "null argument");
  const Cosmo &c = l->cosmo;
  l->owned.emplace_back(h);
  h->Dist = angdist(c, h->zlens);  // LensHalo(z, cosmo): Dist = angDist(z)
  double hz = h->zlens, hD = coordist2(c, 0, hz);
  auto &M = l->main;
  auto setz = [&](glb_halo *x, double z) {
    x->zlens = z;
    x->Dist = angdist(c, z);
  };
  if (addplanes) {
    size_t i = 0;
    while (i < M.size() && !(hD < M[i].Dl)) ++i;  // upper_bound
    if (i > 0 && (hD - M[i - 1].Dl) < 1e-6) {
      M[i - 1].halos.push_back(h);
      setz(h, M[i - 1].z);
    } else if (i == M.size()) {
      M.push_back(PlaneHost{hz, hD, {h}});
    } else if ((M[i].Dl - hD) < 1e-6) {
      M[i].halos.push_back(h);
      setz(h, M[i].z);
    } else {
      M.insert(M.begin() + i, PlaneHost{hz, hD, {h}});
      setz(h, hz);
    }
  } else {
    if (M.empty()) {
      M.push_back(PlaneHost{hz, hD, {h}});
    } else {
      size_t best = 0;
      for (size_t i = 1; i < M.size(); ++i)
        if (std::fabs(M[i].Dl - hD) < std::fabs(M[best].Dl - hD)) best = i;
      M[best].halos.push_back(h);
      setz(h, M[best].z);
    }
  }
  combine_planes(l);
  return 0;
}

int glb_lens_nplanes(glb_lens *l, int *nplanes) {
  if (!l || !nplanes) return fail(GLB_ERR_ARG, "null argument");
  *nplanes = (int)l->planes.size();
  return 0;
}

int glb_lens_planes(glb_lens *l, double *z, double *Dl, double *dDl) {
  if (!l) return fail(GLB_ERR_ARG, "null lens");
  for (size_t i = 0; i < l->plane_z.size(); ++i) {
    if (z) z[i] = l->plane_z[i];
    if (Dl) Dl[i] = l->Dl[i];
    if (dDl) dDl[i] = l->dDl[i];
  }
  return 0;
}

int glb_lens_reset_source(glb_lens *l, double z, int nearest, int *plane_index) {
  if (!l) return fail(GLB_ERR_ARG, "null lens");
  l->toggle_source_plane = true;
  long j = 0;
  if (z <= 0.0) {
    if (plane_index) *plane_index = 0;
    return 0;
  }
  double Ds = coordist2(l->cosmo, 0, z);
  size_t np = l->planes.size();
  if (l->Dl.size() > 1) {
    // NR locate on Dl[0..np-1] (1-based bisection)
    unsigned long n = (unsigned long)np, ju = n + 1, jl = 0, jm;
    const double *xx = l->Dl.data() - 1;
    while (ju - jl > 1) {
      jm = (ju + jl) >> 1;
      if (Ds >= xx[jm]) jl = jm; else ju = jm;
    }
    if (Ds == xx[1]) j = 1;
    else if (Ds == xx[n]) j = (long)n - 1;
    else j = (long)jl;
  }
  if (j > 0) {
    if (l->Dl[j - 1] == Ds) --j;
    else if (nearest) {
      double z1 = invcoordist(l->cosmo, l->Dl[j] - 0.5 * l->dDl[j]);
      if (z < z1) --j;
    }
  }
  if (nearest && (j < (long)np)) l->zs_implant = l->plane_z[j];
  else l->zs_implant = z;
  if (plane_index) *plane_index = (int)j;
  return 0;
}

int glb_lens_rayshoot_device(glb_lens *l, size_t n, const double *x_dev, const double *zs_dev, double *y_dev,
                             double *A_dev, int precision, void *stream) {
  return glb_lens_rayshoot_device_status(l, n, x_dev, zs_dev, nullptr, y_dev, A_dev, nullptr, precision, stream);
}

int glb_lens_rayshoot_device_status(glb_lens *l, size_t n, const double *x_dev, const double *zs_dev,
                                    const unsigned char *skip_dev, double *y_dev, double *A_dev,
                                    unsigned char *status_dev, int precision, void *stream) {
  if (!l) return fail(GLB_ERR_ARG, "null lens");
  if (n > 0 && (!x_dev || !y_dev || !A_dev)) return fail(GLB_ERR_ARG, "null buffer");
  if (precision != GLB_PREC_FP64 && precision != GLB_PREC_SPLIT) return fail(GLB_ERR_ARG, "unknown precision");
  if (int rc = set_dev(l->device)) return rc;
  LensWS *w;
  if (int rc = thread_ws(l, &w)) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : w->stream;
  return rayshoot_device(l, w, n, x_dev, zs_dev, y_dev, A_dev, precision, s, nullptr, status_dev, skip_dev);
}

// Host buffers in and out through the calling thread's staging buffer and
// stream.  x_on_device: x is already a device array (GridMap positions).
static int rayshoot_host(glb_lens *l, LensWS *w, size_t n, const double *x, const double *zs, double *y,
                         double *A, int precision, bool x_on_device, const unsigned char *skip = nullptr,
                         unsigned char *status = nullptr) {
  if (n == 0) return 0;
  // staging (doubles): x 2n | zs n | y 2n | A 4n | skip + status (2n bytes, rounded up)
  const size_t flag_words = (skip || status) ? (2 * n + 7) / 8 : 0;
  size_t need = (x_on_device ? 0 : 2 * n) + (zs ? n : 0) + 6 * n + flag_words;
  if (w->io.n < need) CKR(w->io.alloc(need));
  cudaStream_t s = w->stream;
  double *dx = x_on_device ? const_cast<double *>(x) : w->io.p;
  double *dzs = zs ? w->io.p + (x_on_device ? 0 : 2 * n) : nullptr;
  double *dy = w->io.p + (x_on_device ? 0 : 2 * n) + (zs ? n : 0);
  double *dA = dy + 2 * n;
  unsigned char *dflags = reinterpret_cast<unsigned char *>(dA + 4 * n);
  unsigned char *dskip = skip ? dflags : nullptr;
  unsigned char *dstatus = status ? dflags + n : nullptr;
  if (!x_on_device) CKR(cudaMemcpyAsync(dx, x, 2 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (zs) CKR(cudaMemcpyAsync(dzs, zs, n * sizeof(double), cudaMemcpyHostToDevice, s));
  if (skip) {
    // skipped rays keep the caller's y and A: start from them
    CKR(cudaMemcpyAsync(dskip, skip, n, cudaMemcpyHostToDevice, s));
    CKR(cudaMemcpyAsync(dy, y, 2 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    CKR(cudaMemcpyAsync(dA, A, 4 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  }
  if (int rc = rayshoot_device(l, w, n, dx, dzs, dy, dA, precision, s, nullptr, dstatus, dskip)) return rc;
  CKR(cudaMemcpyAsync(y, dy, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CKR(cudaMemcpyAsync(A, dA, 4 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  if (status) CKR(cudaMemcpyAsync(status, dstatus, n, cudaMemcpyDeviceToHost, s));
  CKR(cudaStreamSynchronize(s));
  if (l->planes.size() > 0) {
    cudaEventElapsedTime(&w->last_kernel_ms, w->ev[1], w->ev[2]);
    cudaEventElapsedTime(&w->last_total_ms, w->ev[0], w->ev[3]);
  }
  return 0;
}

int glb_lens_rayshoot(glb_lens *l, size_t n, const double *x, const double *zs, double *y, double *A,
                      int precision) {
  return glb_lens_rayshoot_status(l, n, x, zs, nullptr, y, A, nullptr, precision);
}

int glb_lens_rayshoot_status(glb_lens *l, size_t n, const double *x, const double *zs, const unsigned char *skip,
                             double *y, double *A, unsigned char *status, int precision) {
  if (!l) return fail(GLB_ERR_ARG, "null lens");
  if (n > 0 && (!x || !y || !A)) return fail(GLB_ERR_ARG, "null buffer");
  if (precision != GLB_PREC_FP64 && precision != GLB_PREC_SPLIT) return fail(GLB_ERR_ARG, "unknown precision");
  if (int rc = set_dev(l->device)) return rc;
  LensWS *w;
  if (int rc = thread_ws(l, &w)) return rc;
  return rayshoot_host(l, w, n, x, zs, y, A, precision, false, skip, status);
}

int glb_gridmap(glb_lens *l, size_t n1d, const double *center, double range, double *y, double *A, int precision) {
  if (!l || !center || !y || !A) return fail(GLB_ERR_ARG, "null argument");
  if (n1d < 1) return fail(GLB_ERR_ARG, "GridMap size is < 1!");  // gridmap.cpp:102
  if (range <= 0) return fail(GLB_ERR_ARG, "GridMap range is <= 0!");
  if (precision != GLB_PREC_FP64 && precision != GLB_PREC_SPLIT) return fail(GLB_ERR_ARG, "unknown precision");
  if (int rc = set_dev(l->device)) return rc;
  LensWS *w;
  if (int rc = thread_ws(l, &w)) return rc;
  size_t n = n1d * n1d;
  DBuf<double> dx;
  CKR(dx.alloc(2 * n));
  k_grid<<<nblk(n, 256), 256, 0, w->stream>>>(n1d, center[0], center[1], range, dx.p);
  CKR(cudaGetLastError());
  int rc = rayshoot_host(l, w, n, dx.p, nullptr, y, A, precision, true);
  CKR(cudaStreamSynchronize(w->stream));
  return rc;
}

int glb_gridmap_pixelmap(glb_lens *l, size_t n1d, const double *center, double range, int lensvar, double *map,
                         int precision) {
  if (!l || !center || !map) return fail(GLB_ERR_ARG, "null argument");
  if (n1d < 1) return fail(GLB_ERR_ARG, "GridMap size is < 1!");  // gridmap.cpp:102
  if (range <= 0) return fail(GLB_ERR_ARG, "GridMap range is <= 0!");
  if (precision != GLB_PREC_FP64 && precision != GLB_PREC_SPLIT) return fail(GLB_ERR_ARG, "unknown precision");
  if (lensvar == 10 || lensvar == 11)  // PHI, SurfBrightness (gridmap.h:588-594)
    return fail(GLB_ERR_UNSUPPORTED, "GridMap::writePixelMap() does not work for the input LensingVariable");
  if (lensvar < 0 || lensvar > 11) return fail(GLB_ERR_ARG, "unknown LensingVariable");
  if (int rc = set_dev(l->device)) return rc;
  LensWS *w;
  if (int rc = thread_ws(l, &w)) return rc;
  const size_t n = n1d * n1d;
  DBuf<double> dx, dy, dA, dm;
  CKR(dx.alloc(2 * n));
  CKR(dy.alloc(2 * n));
  CKR(dA.alloc(4 * n));
  CKR(dm.alloc(n));
  k_grid<<<nblk(n, 256), 256, 0, w->stream>>>(n1d, center[0], center[1], range, dx.p);
  CKR(cudaGetLastError());
  if (int rc = rayshoot_device(l, w, n, dx.p, nullptr, dy.p, dA.p, precision, w->stream)) return rc;
  k_pixelmap<<<nblk(n, 256), 256, 0, w->stream>>>(dx.p, dy.p, dA.p, n, lensvar, dm.p);
  CKR(cudaGetLastError());
  CKR(cudaMemcpyAsync(map, dm.p, n * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CKR(cudaStreamSynchronize(w->stream));
  return 0;
}

// The device descriptor of a Source (kind, position, derived constants).
static int make_source_dev(int source_kind, const double *source_params, SourceDev &S) {
  memset(&S, 0, sizeof(S));
  S.kind = source_kind;
  S.x = source_params[0];
  S.y = source_params[1];
  const double *p = source_params + 2;
  if (source_kind == 0) {
    S.q[0] = p[0];  // radius (radians)
  } else if (source_kind == 1) {
    S.q[0] = p[0] * p[0];  // source_gauss_r2 = r_size^2
  } else if (source_kind == 2) {
    // SourceSersic::ReSet / setReff / setSersicIndex / setAxesRatio
    // (Source/sersic.cpp:87-113, include/sersic_source.h:62-92)
    const double flux = p[0], reff = p[1] * 4.848136811e-6, pa = p[2], index = p[3];
    double q = p[4];
    if (q > 1) q = 1 / q;
    if (!(reff > 0) || !(index > 0) || !(q > 0)) return fail(GLB_ERR_ARG, "Sersic Reff, index and q must be positive");
    const double bn = 1.9992 * index - 0.3271;
    const double I_n = 1. / index * pow(bn, 2 * index) / tgamma(2 * index);
    const double I_q = 1. / q, I_r = 1. / 2. / kPi / reff / reff;
    S.q[0] = cos(pa);
    S.q[1] = sin(pa);
    S.q[2] = 1. / q / q;
    S.q[3] = flux * I_n * I_q * I_r;
    S.q[4] = bn;
    S.q[5] = 1. / reff;
    S.q[6] = 1. / index;
    S.q[7] = p[5];  // sb_limit
  } else {
    return fail(GLB_ERR_UNSUPPORTED, "source kind outside this library (0 uniform, 1 Gaussian, 2 Sersic)");
  }
  return 0;
}

int glb_gridmap_pixelmap_uniform(glb_lens *l, size_t n1d, const double *center, double range,
                                 const double *map_center, size_t nx, size_t ny, int lensvar, double *map,
                                 int precision) {
  if (!l || !center || !map_center || !map) return fail(GLB_ERR_ARG, "null argument");
  if (n1d < 1) return fail(GLB_ERR_ARG, "GridMap size is < 1!");  // gridmap.cpp:102
  if (range <= 0) return fail(GLB_ERR_ARG, "GridMap range is <= 0!");
  if (nx < 2 || ny < 1) return fail(GLB_ERR_ARG, "the uniform map needs nx >= 2 (resolution range / (nx - 1)) and ny >= 1");
  if (precision != GLB_PREC_FP64 && precision != GLB_PREC_SPLIT) return fail(GLB_ERR_ARG, "unknown precision");
  if (lensvar == 10 || lensvar == 11)  // PHI throws (gridmap.h:640-690); a new grid has no surface brightness
    return fail(GLB_ERR_UNSUPPORTED, "GridMap::writePixelMapUniform() does not work for the input LensingVariable");
  if (lensvar < 0 || lensvar > 11) return fail(GLB_ERR_ARG, "unknown LensingVariable");
  if (int rc = set_dev(l->device)) return rc;
  LensWS *w;
  if (int rc = thread_ws(l, &w)) return rc;
  const size_t n = n1d * n1d, nm = nx * ny;
  UniformMap M;
  M.res = range / (double)(nx - 1);  // x_range / (Nx - 1), gridmap.h:514
  M.p10 = map_center[0] - ((double)nx * M.res) / 2.;
  M.p11 = map_center[1] - ((double)ny * M.res) / 2.;
  M.nx = (long long)nx;
  M.ny = (long long)ny;
  DBuf<double> dx, dy, dA, dm;
  DBuf<long long> own;
  CKR(dx.alloc(2 * n));
  CKR(dy.alloc(2 * n));
  CKR(dA.alloc(4 * n));
  CKR(dm.alloc(nm));
  CKR(own.alloc(nm));
  k_grid<<<nblk(n, 256), 256, 0, w->stream>>>(n1d, center[0], center[1], range, dx.p);
  CKR(cudaGetLastError());
  if (int rc = rayshoot_device(l, w, n, dx.p, nullptr, dy.p, dA.p, precision, w->stream)) return rc;
  CKR(cudaMemsetAsync(dm.p, 0, nm * sizeof(double), w->stream));  // PixelMap::Clean
  CKR(cudaMemsetAsync(own.p, 0xff, nm * sizeof(long long), w->stream));  // -1: no grid point
  k_uniform_owner<<<nblk(n, 256), 256, 0, w->stream>>>(dx.p, n, M, own.p);
  k_uniform_write<<<nblk(n, 256), 256, 0, w->stream>>>(dx.p, dy.p, dA.p, n, lensvar, M, own.p, dm.p);
  CKR(cudaGetLastError());
  CKR(cudaMemcpyAsync(map, dm.p, nm * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CKR(cudaStreamSynchronize(w->stream));
  return 0;
}

int glb_gridmap_surface_brightness(glb_lens *l, size_t n1d, const double *center, double range, int source_kind,
                                   const double *source_params, double *sb, double *total, int precision) {
  if (!l || !center || !source_params || !sb) return fail(GLB_ERR_ARG, "null argument");
  if (n1d < 2) return fail(GLB_ERR_ARG, "GridMap size must be > 1 for a resolution");
  if (range <= 0) return fail(GLB_ERR_ARG, "GridMap range is <= 0!");
  if (precision != GLB_PREC_FP64 && precision != GLB_PREC_SPLIT) return fail(GLB_ERR_ARG, "unknown precision");
  SourceDev S;
  if (int rc = make_source_dev(source_kind, source_params, S)) return rc;
  if (int rc = set_dev(l->device)) return rc;
  LensWS *w;
  if (int rc = thread_ws(l, &w)) return rc;
  const size_t n = n1d * n1d;
  DBuf<double> dx, dy, dA, dsb;
  CKR(dx.alloc(2 * n));
  CKR(dy.alloc(2 * n));
  CKR(dA.alloc(4 * n));
  CKR(dsb.alloc(n));
  k_grid<<<nblk(n, 256), 256, 0, w->stream>>>(n1d, center[0], center[1], range, dx.p);
  CKR(cudaGetLastError());
  if (int rc = rayshoot_device(l, w, n, dx.p, nullptr, dy.p, dA.p, precision, w->stream)) return rc;
  k_surface_brightness<<<nblk(n, 256), 256, 0, w->stream>>>(dy.p, n, S, dsb.p);
  CKR(cudaGetLastError());
  CKR(cudaMemcpyAsync(sb, dsb.p, n * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
  CKR(cudaStreamSynchronize(w->stream));
  if (total) {  // GridMap::RefreshSurfaceBrightnesses: sum in point order times resolution^2
    const double res = range / (double)(n1d - 1), res2 = pow(res, 2);
    double t = 0;
    for (size_t i = 0; i < n; ++i) t += sb[i] * res2;
    *total = t;
  }
  return 0;
}

// GridMap::to_refine (TreeCode_link/gridmap.cpp:248-258).  The neighbour range
// MAX<size_t>(i-1, 0) .. MIN<size_t>(i+2, N) wraps to nothing for i = 0 (and
// j = 0): pixels of the first row and column never refine.
static bool to_refine(const std::vector<double> &sb, long i, long j, long N, double total, double f) {
  const double flux = sb[i + j * N];
  const size_t i0 = (size_t)(i - 1), j0 = (size_t)(j - 1);
  const size_t i1 = std::min<size_t>((size_t)(i + 2), (size_t)N), j1 = std::min<size_t>((size_t)(j + 2), (size_t)N);
  for (size_t ii = i0; ii < i1; ++ii)
    for (size_t jj = j0; jj < j1; ++jj)
      if (std::fabs(flux - sb[ii + jj * N]) / total > f) return true;
  return false;
}

constexpr int kMaxRefine = 6;                 // n = 3 ... 729 sub-rays per side
constexpr size_t kRefineChunk = 4u << 20;     // sub-rays per launch

// The refinement loop of gridmap.cpp:205-234 for many pixels at once, level by
// level: every pixel still changing shoots its n x n sub-grid (laid around its
// source position, as the reference does) in one batched call; the sub-rays'
// surface brightness is summed per pixel on the host in the reference's (u, v)
// order.  out[k] = refined flux of pixel P[k].
static int refine_pixels(glb_lens *l, LensWS *w, const std::vector<size_t> &P, const std::vector<double> &ysrc,
                         const std::vector<double> &sb0, double resolution, const SourceDev &S, int precision,
                         std::vector<double> &out) {
  const size_t np = P.size();
  std::vector<double> nf(np), of(np, 0.0);
  for (size_t k = 0; k < np; ++k) nf[k] = sb0[P[k]];
  int n = 1;
  for (int level = 0; level < kMaxRefine; ++level) {
    std::vector<size_t> act;
    for (size_t k = 0; k < np; ++k)
      if (std::fabs(of[k] - nf[k]) > 1.0e-3 * nf[k]) act.push_back(k);
    if (act.empty()) break;
    n *= 3;
    const double res = resolution / n;
    const size_t m = (size_t)n * n;
    const size_t per = std::max<size_t>(1, kRefineChunk / m);  // pixels per launch
    DBuf<double> dx, dy, dA, dsb;
    const size_t cap = std::min(per, act.size()) * m;
    CKR(dx.alloc(2 * cap));
    CKR(dy.alloc(2 * cap));
    CKR(dA.alloc(4 * cap));
    CKR(dsb.alloc(cap));
    std::vector<double> hx(2 * cap), hsb(cap);
    for (size_t a0 = 0; a0 < act.size(); a0 += per) {
      const size_t a1 = std::min(act.size(), a0 + per), cnt = (a1 - a0) * m;
      for (size_t a = a0; a < a1; ++a) {
        const size_t k = act[a];
        const double ll0 = ysrc[2 * P[k]] - resolution / 2, ll1 = ysrc[2 * P[k] + 1] - resolution / 2;
        double *x = hx.data() + 2 * (a - a0) * m;
        for (int u = 0; u < n; ++u)
          for (int v = 0; v < n; ++v) {
            x[2 * ((size_t)u * n + v)] = ll0 + (0.5 + u) * res;
            x[2 * ((size_t)u * n + v) + 1] = ll1 + (0.5 + v) * res;
          }
      }
      CKR(cudaMemcpyAsync(dx.p, hx.data(), 2 * cnt * sizeof(double), cudaMemcpyHostToDevice, w->stream));
      if (int rc = rayshoot_device(l, w, cnt, dx.p, nullptr, dy.p, dA.p, precision, w->stream)) return rc;
      k_surface_brightness<<<nblk(cnt, 256), 256, 0, w->stream>>>(dy.p, cnt, S, dsb.p);
      CKR(cudaGetLastError());
      CKR(cudaMemcpyAsync(hsb.data(), dsb.p, cnt * sizeof(double), cudaMemcpyDeviceToHost, w->stream));
      CKR(cudaStreamSynchronize(w->stream));
      for (size_t a = a0; a < a1; ++a) {
        const size_t k = act[a];
        of[k] = nf[k];
        double sum = 0;
        const double *v = hsb.data() + (a - a0) * m;
        for (size_t q = 0; q < m; ++q) sum += v[q];
        nf[k] = sum / (n * n);
      }
    }
  }
  out = nf;
  return 0;
}

int glb_gridmap_adaptive_surface_brightness(glb_lens *l, size_t n1d, const double *center, double range,
                                            int source_kind, const double *source_params, double *sb_out,
                                            double *total, int precision) {
  if (!l || !center || !source_params || !sb_out || !total) return fail(GLB_ERR_ARG, "null argument");
  const size_t n = n1d * n1d;
  std::vector<double> sb(n);
  double total0 = 0;
  // the grid, its source positions and RefreshSurfaceBrightnesses
  if (int rc = glb_gridmap_surface_brightness(l, n1d, center, range, source_kind, source_params, sb.data(), &total0,
                                              precision))
    return rc;
  std::vector<double> ysrc(2 * n), A(4 * n);
  if (int rc = glb_gridmap(l, n1d, center, range, ysrc.data(), A.data(), precision)) return rc;
  SourceDev S;
  if (int rc = make_source_dev(source_kind, source_params, S)) return rc;
  LensWS *w;
  if (int rc = thread_ws(l, &w)) return rc;
  const double resolution = range / (double)(n1d - 1);
  double total_flux = total0 / resolution / resolution;  // gridmap.cpp:195
  if (total_flux == 0) {
    memcpy(sb_out, sb.data(), n * sizeof(double));
    *total = 0;
    return 0;
  }
  const double f = 1.0e-4;
  const long N = (long)n1d;
  // pixels that refine on the unrefined map (refined all at once on the GPU)
  std::vector<size_t> cand;
  for (long j = 0; j < N; ++j)
    for (long i = 0; i < N; ++i)
      if (to_refine(sb, i, j, N, total_flux, f)) cand.push_back((size_t)(i + j * N));
  std::vector<double> refined;
  if (int rc = refine_pixels(l, w, cand, ysrc, sb, resolution, S, precision, refined)) return rc;
  std::vector<double> cache(n, 0.0);
  std::vector<char> have(n, 0);
  for (size_t k = 0; k < cand.size(); ++k) {
    cache[cand[k]] = refined[k];
    have[cand[k]] = 1;
  }
  // the reference's sequential pass: later pixels see earlier refinements
  // and the running total (gridmap.cpp:199-239)
  for (long j = 0; j < N; ++j) {
    size_t k = (size_t)j * n1d;
    for (long i = 0; i < N; ++i, ++k) {
      if (!to_refine(sb, i, j, N, total_flux, f)) continue;
      double nfl;
      if (have[k]) {
        nfl = cache[k];
      } else {
        std::vector<double> one;
        if (int rc = refine_pixels(l, w, std::vector<size_t>{k}, ysrc, sb, resolution, S, precision, one)) return rc;
        nfl = one[0];
      }
      total_flux -= sb[k];
      sb[k] = nfl;
      total_flux += nfl;
    }
  }
  memcpy(sb_out, sb.data(), n * sizeof(double));
  *total = total_flux * resolution * resolution;
  return 0;
}

int glb_lens_count_interactions(glb_lens *l, size_t n, const double *x, const double *zs,
                                unsigned long long *counts) {
  if (!l || !counts || (n > 0 && !x)) return fail(GLB_ERR_ARG, "null argument");
  if (int rc = set_dev(l->device)) return rc;
  LensWS *w;
  if (int rc = thread_ws(l, &w)) return rc;
  DBuf<double> dx, dzs, dy, dA;
  DBuf<unsigned long long> dc;
  CKR(dx.alloc(2 * n));
  CKR(dy.alloc(2 * n));
  CKR(dA.alloc(4 * n));
  CKR(dc.alloc(7));
  CKR(cudaMemsetAsync(dc.p, 0, 7 * sizeof(unsigned long long), w->stream));
  CKR(cudaMemcpyAsync(dx.p, x, 2 * n * sizeof(double), cudaMemcpyHostToDevice, w->stream));
  if (zs) {
    CKR(dzs.alloc(n));
    CKR(cudaMemcpyAsync(dzs.p, zs, n * sizeof(double), cudaMemcpyHostToDevice, w->stream));
  }
  if (int rc = rayshoot_device(l, w, n, dx.p, zs ? dzs.p : nullptr, dy.p, dA.p, GLB_PREC_FP64, w->stream, dc.p))
    return rc;
  CKR(cudaMemcpyAsync(counts, dc.p, 7 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, w->stream));
  CKR(cudaStreamSynchronize(w->stream));
  return 0;
}

int glb_lens_last_timing(glb_lens *l, double *kernel_ms, double *total_ms) {
  if (!l) return fail(GLB_ERR_ARG, "null lens");
  if (int rc = set_dev(l->device)) return rc;
  LensWS *w;
  if (int rc = thread_ws(l, &w)) return rc;
  if (l->planes.size() > 0 && w->timed && cudaEventQuery(w->ev[0]) != cudaErrorNotReady) {
    CKR(cudaEventSynchronize(w->ev[3]));
    cudaEventElapsedTime(&w->last_kernel_ms, w->ev[1], w->ev[2]);
    cudaEventElapsedTime(&w->last_total_ms, w->ev[0], w->ev[3]);
  }
  if (kernel_ms) *kernel_ms = w->last_kernel_ms;
  if (total_ms) *total_ms = w->last_total_ms;
  return 0;
}

}  // extern "C"

// ======================================================= allocation-free entry
// glb_lens_rayshoot_noalloc: the same multi-plane pass as
// glb_lens_rayshoot_device for callers that must not allocate device memory
// while they shoot rays -- a cudaMalloc / cudaFree pair synchronises the whole
// device and may fail under a memory cap, which latency-bound callers (grid
// refinement rounds that shoot a few thousand rays at a time, an application
// that reserved its memory up front, or a process sharing the GPU under a
// hard quota) cannot accept.  All scratch memory lives in one file-scope
// device array of fixed size, held by every GPU that loads the library until
// the process exits.
namespace {

constexpr size_t kNoAllocMaxRays = 65536;  // rays per call
constexpr int kNoAllocMaxPlanes = 64;
constexpr int kNoAllocMaxHalos = 256;
constexpr size_t kNoAllocSortBytes = 4u << 20;  // radix-sort temporary storage

constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffState = 0;
constexpr size_t kOffJmax = kOffState + align256(12 * kNoAllocMaxRays * sizeof(double));
constexpr size_t kOffSrc = kOffJmax + align256(kNoAllocMaxRays * sizeof(int));
constexpr size_t kOffKeys = kOffSrc + align256(2 * kNoAllocMaxRays * sizeof(double));
constexpr size_t kOffKeys2 = kOffKeys + align256(kNoAllocMaxRays * sizeof(unsigned));
constexpr size_t kOffPerm0 = kOffKeys2 + align256(kNoAllocMaxRays * sizeof(unsigned));
constexpr size_t kOffPerm = kOffPerm0 + align256(kNoAllocMaxRays * sizeof(unsigned));
constexpr size_t kOffBbox = kOffPerm + align256(kNoAllocMaxRays * sizeof(unsigned));
constexpr size_t kOffPlanes = kOffBbox + align256(4 * sizeof(unsigned long long));
constexpr size_t kOffHalos = kOffPlanes + align256(kNoAllocMaxPlanes * sizeof(PlaneDev));
constexpr size_t kOffPlaneZ = kOffHalos + align256(kNoAllocMaxHalos * sizeof(HaloDev));
constexpr size_t kOffDl = kOffPlaneZ + align256((kNoAllocMaxPlanes + 1) * sizeof(double));
constexpr size_t kOffNfw = kOffDl + align256((kNoAllocMaxPlanes + 1) * sizeof(double));
constexpr size_t kOffSort = kOffNfw + align256(5 * kNfwTable * sizeof(double));
constexpr size_t kNoAllocBytes = kOffSort + kNoAllocSortBytes;  // about 13.5 MB

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_ptr[64] = {};
// Calls on one device are put in order on the GPU: each call's stream waits
// for the previous call's last launch (an event, not an allocation), and the
// enqueue itself is serialised on the host, so two calls never use the
// shared scratch at the same time whatever streams or lenses they name.
cudaEvent_t g_noalloc_ev[64] = {};
std::mutex g_noalloc_call_mu;

// Once per device, with that device current: the device address of the
// scratch array (its host-side name is only a stand-in) and the NFW tables.
int noalloc_setup(int dev, unsigned char **out) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (dev < 0 || dev >= 64) return fail(GLB_ERR_ARG, "device index out of range for the no-alloc scratch");
  if (!g_noalloc_ptr[dev]) {
    unsigned char *p = nullptr;
    CKR(cudaGetSymbolAddress((void **)&p, g_noalloc_scratch));
    std::call_once(g_nfw_host_once, make_host_tables);
    const std::vector<double> *src[5] = {&g_nfw_host.x, &g_nfw_host.f, &g_nfw_host.g, &g_nfw_host.g2,
                                         &g_nfw_host.h};
    for (int i = 0; i < 5; ++i)
      CKR(cudaMemcpy(p + kOffNfw + (size_t)i * kNfwTable * sizeof(double), src[i]->data(),
                     kNfwTable * sizeof(double), cudaMemcpyHostToDevice));
    size_t tb = 0;
    CKR(cub::DeviceRadixSort::SortPairs(nullptr, tb, (unsigned *)nullptr, (unsigned *)nullptr,
                                        (unsigned *)nullptr, (unsigned *)nullptr, (int)kNoAllocMaxRays, 0, 32));
    if (tb > kNoAllocSortBytes) return fail(GLB_ERR_ARG, "no-alloc scratch: radix-sort temporary storage too small");
    CKR(cudaEventCreateWithFlags(&g_noalloc_ev[dev], cudaEventDisableTiming));
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}

}  // namespace

// ------------------------------------------------------ kNN smoothing
extern "C" int glb_particles_smoothing_device(const glb_particle *particles_dev, size_t n, int nsmooth,
                                              float *size_dev, void *stream, float *ms_out) {
  if (n > 0 && (!particles_dev || !size_dev)) return fail(GLB_ERR_ARG, "null buffer");
  if (int rc = need_device()) return rc;
  Status s = smooth_particles_device(reinterpret_cast<const glb_particle_rec *>(particles_dev), n, nsmooth,
                                     size_dev, (cudaStream_t)stream, ms_out);
  return s.good() ? 0 : fail(s);
}

extern "C" int glb_particles_smoothing(glb_particle *particles, size_t n, int nsmooth) {
  if (n > 0 && !particles) return fail(GLB_ERR_ARG, "null particles");
  if (int rc = need_device()) return rc;
  cudaStream_t st;
  CKR(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{st};
  DBuf<glb_particle_rec> d_p;
  DBuf<float> d_size;
  CKR(d_p.alloc(n));
  CKR(d_size.alloc(n));
  if (n) CKR(cudaMemcpyAsync(d_p.p, particles, n * sizeof(glb_particle_rec), cudaMemcpyHostToDevice, st));
  Status s = smooth_particles_device(d_p.p, n, nsmooth, d_size.p, st, nullptr);
  if (!s.good()) return fail(s);
  std::vector<float> sz(n);
  CKR(cudaMemcpyAsync(sz.data(), d_size.p, n * sizeof(float), cudaMemcpyDeviceToHost, st));
  CKR(cudaStreamSynchronize(st));
  for (size_t i = 0; i < n; ++i) particles[i].Size = sz[i];
  return 0;
}

extern "C" int glb_lens_rayshoot_noalloc(glb_lens *l, size_t n, const double *x_dev, const double *zs_dev,
                                         double *y_dev, double *A_dev, int precision, void *stream) {
  if (!l) return fail(GLB_ERR_ARG, "null lens");
  if (n > kNoAllocMaxRays)
    return fail(GLB_ERR_ARG, "glb_lens_rayshoot_noalloc: at most 65536 rays per call");
  if (n > 0 && (!x_dev || !y_dev || !A_dev)) return fail(GLB_ERR_ARG, "null buffer");
  if (precision != GLB_PREC_FP64 && precision != GLB_PREC_SPLIT) return fail(GLB_ERR_ARG, "unknown precision");
  size_t np = l->planes.size(), nh = 0;
  for (const PlaneHost *p : l->planes) nh += p->halos.size();
  if (np > (size_t)kNoAllocMaxPlanes || nh > (size_t)kNoAllocMaxHalos)
    return fail(GLB_ERR_ARG, "glb_lens_rayshoot_noalloc: at most 64 planes and 256 halos");
  if (int rc = set_dev(l->device)) return rc;
  unsigned char *S = nullptr;
  if (int rc = noalloc_setup(l->device, &S)) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : l->stream;
  if (n == 0) return 0;
  if (np == 0) {
    k_identity_rays<<<nblk(n, 256), 256, 0, s>>>(x_dev, n, y_dev, A_dev);
    CKR(cudaGetLastError());
    return 0;
  }
  // from here on the scratch is in use: after the previous call on this device
  std::lock_guard<std::mutex> order(g_noalloc_call_mu);
  CKR(cudaStreamWaitEvent(s, g_noalloc_ev[l->device], 0));
  // plane and halo descriptors of this lens (host stack arrays, no heap),
  // copied into the scratch; pageable copies are staged before they return
  PlaneDev P[kNoAllocMaxPlanes];
  HaloDev H[kNoAllocMaxHalos];
  int nhd = 0;
  for (size_t j = 0; j < np; ++j) {
    PlaneDev &p = P[j];
    p.Dphys = l->Dl[j] / (1 + l->plane_z[j]);
    p.Gfac = l->charge * l->Dl[j] / (1 + l->plane_z[j]);
    p.aa = l->dDl[j + 1] / l->Dl[j + 1];
    p.bb = l->Dl[j] / l->Dl[j + 1];
    p.halo0 = nhd;
    p.nhalo = (int)l->planes[j]->halos.size();
    for (glb_halo *h : l->planes[j]->halos) H[nhd++] = make_halo_dev(*h);
  }
  PlaneDev *d_planes = (PlaneDev *)(S + kOffPlanes);
  HaloDev *d_halos = (HaloDev *)(S + kOffHalos);
  double *d_planez = (double *)(S + kOffPlaneZ), *d_Dl = (double *)(S + kOffDl);
  CKR(cudaMemcpyAsync(d_planes, P, np * sizeof(PlaneDev), cudaMemcpyHostToDevice, s));
  if (nhd) CKR(cudaMemcpyAsync(d_halos, H, nhd * sizeof(HaloDev), cudaMemcpyHostToDevice, s));
  CKR(cudaMemcpyAsync(d_planez, l->plane_z.data(), (np + 1) * sizeof(double), cudaMemcpyHostToDevice, s));
  CKR(cudaMemcpyAsync(d_Dl, l->Dl.data(), (np + 1) * sizeof(double), cudaMemcpyHostToDevice, s));

  double *st = (double *)(S + kOffState);
  int *jmax_ray = (int *)(S + kOffJmax);
  double *src_ray = (double *)(S + kOffSrc);
  unsigned *keys = (unsigned *)(S + kOffKeys), *keys2 = (unsigned *)(S + kOffKeys2);
  unsigned *perm0 = (unsigned *)(S + kOffPerm0), *perm = (unsigned *)(S + kOffPerm);
  unsigned long long *bbox = (unsigned long long *)(S + kOffBbox);
  if (n >= 64) {
    // the bounding box starts from sentinels on every call
    static const unsigned long long init[4] = {~0ull, ~0ull, 0ull, 0ull};
    CKR(cudaMemcpyAsync(bbox, init, sizeof(init), cudaMemcpyHostToDevice, s));
    k_ray_bbox<<<std::min(nblk(n, 256), 1184), 256, 0, s>>>(x_dev, n, bbox);
    k_ray_morton<<<nblk(n, 256), 256, 0, s>>>(x_dev, n, bbox, keys, perm0);
    size_t tb = kNoAllocSortBytes;
    CKR(cub::DeviceRadixSort::SortPairs(S + kOffSort, tb, keys, keys2, perm0, perm, (int)n, 0, 32, s));
  } else {
    k_identity<<<nblk(n, 256), 256, 0, s>>>(perm, n);
  }
  SrcArgs sa{l->cosmo, d_planez, d_Dl, (int)np};
  k_init_state<<<nblk(n, 256), 256, 0, s>>>(x_dev, zs_dev, perm, n, st, jmax_ray, src_ray, sa);

  StepArgs a;
  a.planes = d_planes;
  a.halos = d_halos;
  const double *T = (const double *)(S + kOffNfw);
  a.tab = NFWTables{T, T + kNfwTable, T + 2 * kNfwTable, T + 3 * kNfwTable, T + 4 * kNfwTable};
  a.st = st;
  a.n = n;
  a.charge = l->charge;
  a.counts = nullptr;
  a.jmax_ray = zs_dev ? jmax_ray : nullptr;
  a.src_ray = zs_dev ? src_ray : nullptr;
  int jmax_launch = (int)np;
  a.jmax = (int)np;
  a.dls_ds = 0;
  a.d_ds = 0;
  if (!zs_dev) {
    double source_z = l->toggle_source_plane ? l->zs_implant : l->plane_z.back();
    if (source_z == l->plane_z.back()) {
      a.dls_ds = l->dDl.back() / l->Dl.back();
      a.d_ds = l->Dl[np - 1] / l->Dl.back();
    } else {
      double Ds = coordist(l->cosmo, source_z), Dls;
      int jm;
      if (source_z <= l->plane_z[0]) {
        jm = 0;
        Dls = Ds;
      } else {
        jm = (int)np;
        while (l->plane_z[jm - 1] > source_z) --jm;
        Dls = coordist2(l->cosmo, l->plane_z[jm - 1], source_z);
      }
      a.jmax = jm;
      a.dls_ds = Dls / Ds;
      if (jm > 0) a.d_ds = l->Dl[jm - 1] / Ds;
      jmax_launch = jm;
    }
  }
  if (int rc = launch_plane_steps(l, a, jmax_launch, precision, s, nullptr)) return rc;
  k_finish<<<nblk(n, 256), 256, 0, s>>>(st, perm, n, y_dev, A_dev);
  CKR(cudaGetLastError());
  CKR(cudaEventRecord(g_noalloc_ev[l->device], s));
  return 0;
}

#include "batch.cuh"
