// Batched and served ray shooting.  Included once at the end of rayshoot.cu
// (same translation unit: it uses that file's kernels, lens objects and
// helpers).
//
// Both patterns run one persistent kernel, k_batch, over a table of chunks.
// A chunk is up to 32 rays of one lens, handled by one warp from the first to
// the last plane with the recursion state in registers:
//   * grid tiles (8 x 4 rays of a GridMap, generated in the kernel from
//     PositionFromIndex) for many lens realisations of uneven size in one
//     launch, replayed from a CUDA graph (glb_batch_*);
//   * ray lists (a served request's rays, sorted along a Morton curve inside
//     the request) for the resident request loop (glb_server_*).
// Warps take chunks from a global atomic counter until the table is done, so
// uneven lenses and requests balance across the SMs.  A chunk never mixes
// lenses or requests, so every ray's arithmetic, and even its warp's joint
// traversal, is the same whatever else is in the batch.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

namespace {

struct LensDev {
  const PlaneDev *planes;
  const HaloDev *halos;
  const double *planez, *Dl;
  int np;
  int jmax_default;
  double dls_default, dds_default;  // the lens's own source plane (Point* overload)
  double charge;
  Cosmo cosmo;
};

struct Chunk {
  int lens;
  int kind;   // 0: grid tile of 32 rays (2^lanes wide), 1: ray list
  int n1d;    // grid side
  int lanes;  // list: rays in this chunk (<= 32); grid tile: log2 of its width (3, 4 or 5)
  int a, b;   // grid: tile origin (ix0, iy0); list: first sorted ray
  long long out;  // grid: output offset of the lens's grid
  double c0, c1, range;
  double zs;  // source redshift; < 0 for the lens's own source plane
};

// Shared memory of k_batch, per thread: the recursion state (theta,
// SumPrevAlphas, A, SumPrevAG: 12 doubles) and the plane's summed forces (5)
// at [c * blockDim + t], and one particle halo's walk totals (5 contiguous
// doubles at 5 t, a stride that puts a half-warp's 64-bit accesses on
// distinct banks).  Keeping them out of registers leaves the tree walk the
// registers it needs.
constexpr int kBatchSmemDoubles = 22;
inline size_t batch_smem_bytes(int block) { return (size_t)kBatchSmemDoubles * block * sizeof(double); }

// LensPlaneSingular::force for one plane (planes.cpp:114-161): the plane's
// halos summed into f[c * stride] = {alpha0, alpha1, kappa, gamma0, gamma1};
// h[0..4] receives one particle halo's walk totals.
template <int PREC>
__device__ __forceinline__ void plane_force(const PlaneDev &P, const HaloDev *halos, const NFWTables *tab,
                                            double xx0, double xx1, bool valid, double *f, double *h,
                                            int stride) {
  for (int c = 0; c < 5; ++c) f[c * stride] = 0.0;
  for (int k = 0; k < P.nhalo; ++k) {
    const HaloDev *H = halos + P.halo0 + k;
    const double xc0 = xx0 - H->px, xc1 = xx1 - H->py;
    double a[5];
    if (H->kind == HALO_PARTICLES) {
      for (int c = 0; c < 5; ++c) h[c] = 0.0;
      particle_halo_acc<PREC, false, false, true>(H->tree, xc0, xc1, valid, h);
      // force_halo negates the walk's alpha (particle_halo.h:432-433)
      a[0] = -h[0];
      a[1] = -h[1];
      a[2] = h[2];
      a[3] = h[3];
      a[4] = h[4];
    } else if (H->kind == HALO_FIELD) {
      const Force6 g = field_plane_force<false>(&H->htree, tab, xc0, xc1, valid);
      a[0] = -g.a0;
      a[1] = -g.a1;
      a[2] = g.k;
      a[3] = g.g0;
      a[4] = g.g1;
    } else if (valid) {
      const Force5 g = analytic_halo(H, tab, xc0, xc1);
      a[0] = g.a0;
      a[1] = g.a1;
      a[2] = g.k;
      a[3] = g.g0;
      a[4] = g.g1;
    } else {
      continue;
    }
    f[0] -= a[0];
    f[stride] -= a[1];
    f[2 * stride] += a[2];
    f[3 * stride] += a[3];
    f[4 * stride] += a[4];
  }
}
template <int PREC>
// capped at 80 registers (3 blocks of 256 per SM) for occupancy (64 registers measured slower here);
// dynamic shared memory: batch_smem_bytes(blockDim.x)
__global__ void __launch_bounds__(256, 3) k_batch(const Chunk *chunks, int nchunks, const LensDev *lenses,
                                               NFWTables tab, const double *xs, const unsigned *outidx,
                                               double *y, double *A, int *counter) {
  extern __shared__ double bsm[];
  const int lane = threadIdx.x & 31;
  const int B = blockDim.x;
  double *st = bsm + threadIdx.x;          // st[c * B], c = 0..11
  double *f = bsm + 12 * B + threadIdx.x;  // f[c * B], c = 0..4
  double *h = bsm + 17 * B + 5 * threadIdx.x;  // h[0..4]
  for (;;) {
    int c = 0;
    if (lane == 0) c = atomicAdd(counter, 1);
    c = __shfl_sync(kFull, c, 0);
    if (c >= nchunks) break;
    const Chunk ch = chunks[c];
    const LensDev &L = lenses[ch.lens];
    bool valid;
    double t0 = 0, t1 = 0;
    long long oi = 0;
    if (ch.kind == 0) {
      const int ix = ch.a + (lane & ((1 << ch.lanes) - 1)), iy = ch.b + (lane >> ch.lanes);
      valid = ix < ch.n1d && iy < ch.n1d;
      if (valid) {
        const long long idx = (long long)ix + (long long)iy * ch.n1d;
        oi = ch.out + idx;
        if (ch.n1d == 1) {
          t0 = ch.c0;
          t1 = ch.c1;
        } else {  // PositionFromIndex (TreeCode_link/utilities.cpp:149-158)
          t0 = ch.c0 + ch.range * (1.0 * (double)ix / (double)(ch.n1d - 1) - 0.5);
          t1 = ch.c1 + ch.range * (1.0 * (double)iy / (double)(ch.n1d - 1) - 0.5);
        }
      }
    } else {
      valid = lane < ch.lanes;
      if (valid) {
        const int k = ch.a + lane;
        t0 = xs[2 * (size_t)k];
        t1 = xs[2 * (size_t)k + 1];
        oi = outidx[k];
      }
    }
    int jmax = L.jmax_default;
    double dls = L.dls_default, dds = L.dds_default;
    if (ch.zs >= 0 && valid) {
      SrcArgs sa{L.cosmo, L.planez, L.Dl, L.np};
      find_source_plane(sa, ch.zs, jmax, dls, dds);
    }
    int jw = valid ? jmax : 0;
    for (int o = 16; o > 0; o >>= 1) jw = max(jw, __shfl_xor_sync(kFull, jw, o));
    st[0] = t0;
    st[B] = t1;
    st[2 * B] = t0;
    st[3 * B] = t1;
    st[4 * B] = 1;
    st[5 * B] = 0;
    st[6 * B] = 0;
    st[7 * B] = 1;
    st[8 * B] = 1;
    st[9 * B] = 0;
    st[10 * B] = 0;
    st[11 * B] = 1;
    for (int j = 0; j < jw; ++j) {
      const bool v = valid && j < jmax;
      {
        const PlaneDev &P = L.planes[j];
        plane_force<PREC>(P, L.halos, &tab, st[0] * P.Dphys, st[B] * P.Dphys, v, f, h, B);
      }
      if (v) {
        // include/lens.h:1027-1066, the state reloaded from shared memory
        const PlaneDev &P = L.planes[j];
        const double G0 = (f[2 * B] + f[3 * B]) * P.Gfac, G1 = f[4 * B] * P.Gfac, G2 = G1,
                     G3 = (f[2 * B] - f[3 * B]) * P.Gfac;
        const double sa0 = st[2 * B] - L.charge * f[0], sa1 = st[3 * B] - L.charge * f[B];
        double aa = P.aa, bb = P.bb;
        if (j >= jmax - 1) {
          aa = dls;
          bb = dds;
        }
        st[0] = bb * st[0] + aa * sa0;
        st[B] = bb * st[B] + aa * sa1;
        st[2 * B] = sa0;
        st[3 * B] = sa1;
        const double A0 = st[4 * B], A1 = st[5 * B], A2 = st[6 * B], A3 = st[7 * B];
        const double s0 = st[8 * B] - (G0 * A0 + G1 * A2), s1 = st[9 * B] - (G0 * A1 + G1 * A3);
        const double s2 = st[10 * B] - (G2 * A0 + G3 * A2), s3 = st[11 * B] - (G2 * A1 + G3 * A3);
        st[8 * B] = s0;
        st[9 * B] = s1;
        st[10 * B] = s2;
        st[11 * B] = s3;
        st[4 * B] = A0 * bb + s0 * aa;
        st[5 * B] = A1 * bb + s1 * aa;
        st[6 * B] = A2 * bb + s2 * aa;
        st[7 * B] = A3 * bb + s3 * aa;
      }
    }
    if (valid) {
      y[2 * oi] = st[0];
      y[2 * oi + 1] = st[B];
      A[4 * oi] = st[4 * B];
      A[4 * oi + 1] = st[5 * B];
      A[4 * oi + 2] = st[6 * B];
      A[4 * oi + 3] = st[7 * B];
    }
  }
}

// Descriptor of a lens for k_batch; the lens's device tables must be current.
int make_lens_dev(glb_lens *l, LensDev &d) {
  if (int rc = upload_lens(l)) return rc;
  size_t np = l->planes.size();
  d.planes = l->d_planes.p;
  d.halos = l->d_halos.p;
  d.planez = l->d_planez.p;
  d.Dl = l->d_Dl.p;
  d.np = (int)np;
  d.charge = l->charge;
  d.cosmo = l->cosmo;
  d.jmax_default = (int)np;
  d.dls_default = 0;
  d.dds_default = 0;
  if (np > 0) {
    double source_z = l->toggle_source_plane ? l->zs_implant : l->plane_z.back();
    if (source_z == l->plane_z.back()) {
      d.dls_default = l->dDl.back() / l->Dl.back();
      d.dds_default = l->Dl[np - 1] / l->Dl.back();
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
      d.jmax_default = jm;
      d.dls_default = Dls / Ds;
      if (jm > 0) d.dds_default = l->Dl[jm - 1] / Ds;
    }
  }
  return 0;
}

int persistent_grid(int block, int precision, int *grid) {
  int dev = 0, sms = 0, per_sm = 0;
  CKR(cudaGetDevice(&dev));
  CKR(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (precision == GLB_PREC_SPLIT)
    CKR(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<GLB_PREC_SPLIT>, block,
                                                      batch_smem_bytes(block)));
  else
    CKR(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch<GLB_PREC_FP64>, block,
                                                      batch_smem_bytes(block)));
  *grid = sms * std::max(per_sm, 1);
  return 0;
}

}  // namespace

// ================================================================ batch plan
struct glb_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  int precision = GLB_PREC_FP64;
  int block = 128, grid = 0;
  std::vector<glb_lens *> lenses;
  std::vector<size_t> n1d, offset;
  std::vector<double> centers, ranges;
  int tile_log2w = 3;  // grid tiles of 8 x 4 rays (autotuned: 8 x 4, 16 x 2, 32 x 1)
  size_t total = 0;
  DBuf<LensDev> d_lenses;
  DBuf<Chunk> d_chunks;
  int nchunks = 0;
  DBuf<double> y, A;
  DBuf<int> counter;
  NFWTables tab{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  float last_ms = 0;
};

namespace {
// The chunk list of the batch's grids: tiles of 2^log2w x 32 / 2^log2w rays,
// the largest grids first (uneven lenses finish together).
int batch_chunks(glb_batch *b, int log2w) {
  std::vector<Chunk> C;
  const int tw = 1 << log2w, th = 32 / tw;
  for (size_t i = 0; i < b->lenses.size(); ++i) {
    const int N = (int)b->n1d[i];
    for (int iy = 0; iy < N; iy += th)
      for (int ix = 0; ix < N; ix += tw) {
        Chunk c;
        memset(&c, 0, sizeof(c));
        c.lens = (int)i;
        c.kind = 0;
        c.n1d = N;
        c.lanes = log2w;
        c.a = ix;
        c.b = iy;
        c.out = (long long)b->offset[i];
        c.c0 = b->centers[2 * i];
        c.c1 = b->centers[2 * i + 1];
        c.range = b->ranges[i];
        c.zs = -1;
        C.push_back(c);
      }
  }
  if (C.size() > 0x7fffffffull) return fail(GLB_ERR_ARG, "too many chunks");
  std::stable_sort(C.begin(), C.end(), [&](const Chunk &x, const Chunk &y) { return x.n1d > y.n1d; });
  if (b->d_chunks.n < C.size()) CKR(b->d_chunks.alloc(C.size()));
  CKR(cudaMemcpy(b->d_chunks.p, C.data(), C.size() * sizeof(Chunk), cudaMemcpyHostToDevice));
  b->nchunks = (int)C.size();
  b->tile_log2w = log2w;
  return 0;
}

void drop_graph(glb_batch *b) {
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
  }
}

int batch_enqueue(glb_batch *b) {
  (void)cudaGetLastError();  // launch errors below are this launch's own
  CKR(cudaMemsetAsync(b->counter.p, 0, sizeof(int), b->stream));
  if (b->precision == GLB_PREC_SPLIT)
    k_batch<GLB_PREC_SPLIT><<<b->grid, b->block, batch_smem_bytes(b->block), b->stream>>>(b->d_chunks.p, b->nchunks, b->d_lenses.p, b->tab,
                                                                 nullptr, nullptr, b->y.p, b->A.p, b->counter.p);
  else
    k_batch<GLB_PREC_FP64><<<b->grid, b->block, batch_smem_bytes(b->block), b->stream>>>(b->d_chunks.p, b->nchunks, b->d_lenses.p, b->tab,
                                                                nullptr, nullptr, b->y.p, b->A.p, b->counter.p);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(GLB_ERR_CUDA, std::string("CUDA: ") + cudaGetErrorString(e) + " launching k_batch with block " +
                                  std::to_string(b->block) + " grid " + std::to_string(b->grid));
  return 0;
}
}  // namespace

extern "C" {

int glb_batch_create_grids(glb_lens *const *lenses, int nlens, const size_t *n1d, const double *centers,
                           const double *ranges, int precision, glb_batch **out) {
  if (!out || !lenses || !n1d || !centers || !ranges || nlens <= 0) return fail(GLB_ERR_ARG, "null argument");
  if (precision != GLB_PREC_FP64 && precision != GLB_PREC_SPLIT) return fail(GLB_ERR_ARG, "unknown precision");
  if (int rc = need_device()) return rc;
  auto b = std::make_unique<glb_batch>();
  CKR(cudaGetDevice(&b->device));
  CKR(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
  CKR(cudaEventCreate(&b->e0));
  CKR(cudaEventCreate(&b->e1));
  b->precision = precision;
  std::vector<LensDev> L(nlens);
  for (int i = 0; i < nlens; ++i) {
    if (!lenses[i]) return fail(GLB_ERR_ARG, "null lens");
    if (lenses[i]->device != b->device) return fail(GLB_ERR_ARG, "all lenses of a batch must be on one device");
    if (n1d[i] < 1 || n1d[i] > 46340) return fail(GLB_ERR_ARG, "grid side must be in [1, 46340]");
    if (!(ranges[i] > 0)) return fail(GLB_ERR_ARG, "GridMap range is <= 0!");
    if (int rc = make_lens_dev(lenses[i], L[i])) return rc;
    b->lenses.push_back(lenses[i]);
    b->n1d.push_back(n1d[i]);
    b->offset.push_back(b->total);
    b->centers.push_back(centers[2 * i]);
    b->centers.push_back(centers[2 * i + 1]);
    b->ranges.push_back(ranges[i]);
    b->total += n1d[i] * n1d[i];
  }
  CKR(b->d_lenses.alloc(nlens));
  CKR(b->y.alloc(2 * b->total));
  CKR(b->A.alloc(4 * b->total));
  CKR(b->counter.alloc(1));
  CKR(cudaMemcpy(b->d_lenses.p, L.data(), nlens * sizeof(LensDev), cudaMemcpyHostToDevice));
  if (int rc = batch_chunks(b.get(), 3)) return rc;
  if (int rc = device_nfw_tables(b->tab)) return rc;
  if (int rc = persistent_grid(b->block, precision, &b->grid)) return rc;
  *out = b.release();
  return 0;
}

int glb_batch_run(glb_batch *b, int use_graph) {
  if (!b) return fail(GLB_ERR_ARG, "null batch");
  if (int rc = set_dev(b->device)) return rc;
  CKR(cudaEventRecord(b->e0, b->stream));
  if (use_graph) {
    if (!b->exec) {
      CKR(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      int rc = batch_enqueue(b);
      cudaGraph_t g = nullptr;
      cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (rc) return rc;
      CKR(e);
      b->graph = g;
      CKR(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    CKR(cudaGraphLaunch(b->exec, b->stream));
  } else {
    if (int rc = batch_enqueue(b)) return rc;
  }
  CKR(cudaEventRecord(b->e1, b->stream));
  CKR(cudaEventSynchronize(b->e1));
  CKR(cudaEventElapsedTime(&b->last_ms, b->e0, b->e1));
  return 0;
}

// Project autotuner, one dimension at a time: the block size (64, 128, 256
// threads, each with its persistent grid) at the current tile, then the warp
// tile (8 x 4, 16 x 2, 32 x 1 rays: the shape of the 32 neighbouring rays a
// warp walks together) at that block size; each candidate timed twice, the
// fastest kept.  The walk keeps no node stack (preorder array with skip
// links), so there is no stack depth to tune.  The graph is rebuilt on the
// next graph run.
int glb_batch_autotune(glb_batch *b, int *best_block, double *best_ms) {
  if (!b) return fail(GLB_ERR_ARG, "null batch");
  if (int rc = set_dev(b->device)) return rc;
  drop_graph(b);
  auto time_it = [&](double *t) -> int {
    *t = 1e300;
    for (int rep = 0; rep < 2; ++rep) {
      if (int rc = glb_batch_run(b, 0)) return rc;
      *t = std::min(*t, (double)b->last_ms);
    }
    return 0;
  };
  double best = 1e300;
  int bb = b->block, bg = b->grid;
  for (int c : {64, 128, 256}) {
    b->block = c;
    if (int rc = persistent_grid(c, b->precision, &b->grid)) return rc;
    double t;
    if (int rc = time_it(&t)) return rc;
    if (t < best) {
      best = t;
      bb = c;
      bg = b->grid;
    }
  }
  b->block = bb;
  b->grid = bg;
  int bt = b->tile_log2w;
  for (int w : {3, 4, 5}) {
    if (w == bt) continue;
    if (int rc = batch_chunks(b, w)) return rc;
    double t;
    if (int rc = time_it(&t)) return rc;
    if (t < best) {
      best = t;
      bt = w;
    }
  }
  if (int rc = batch_chunks(b, bt)) return rc;
  if (best_block) *best_block = bb;
  if (best_ms) *best_ms = best;
  return 0;
}

int glb_batch_tile(glb_batch *b, int *tile_width) {
  if (!b || !tile_width) return fail(GLB_ERR_ARG, "null argument");
  *tile_width = 1 << b->tile_log2w;
  return 0;
}

int glb_batch_set_tile(glb_batch *b, int tile_width) {
  if (!b || (tile_width != 8 && tile_width != 16 && tile_width != 32))
    return fail(GLB_ERR_ARG, "tile width must be 8, 16 or 32");
  if (int rc = set_dev(b->device)) return rc;
  drop_graph(b);
  return batch_chunks(b, tile_width == 8 ? 3 : tile_width == 16 ? 4 : 5);
}

int glb_batch_set_block(glb_batch *b, int block) {
  if (!b || (block != 64 && block != 128 && block != 256)) return fail(GLB_ERR_ARG, "block must be 64, 128 or 256");
  if (int rc = set_dev(b->device)) return rc;
  b->block = block;
  if (int rc = persistent_grid(block, b->precision, &b->grid)) return rc;
  drop_graph(b);
  return 0;
}

int glb_batch_info(glb_batch *b, size_t *total_rays, double *last_ms, int *block) {
  if (!b) return fail(GLB_ERR_ARG, "null batch");
  if (total_rays) *total_rays = b->total;
  if (last_ms) *last_ms = b->last_ms;
  if (block) *block = b->block;
  return 0;
}

int glb_batch_result(glb_batch *b, int i, double *y, double *A) {
  if (!b || i < 0 || i >= (int)b->lenses.size()) return fail(GLB_ERR_ARG, "bad lens index");
  if (int rc = set_dev(b->device)) return rc;
  size_t n = b->n1d[i] * b->n1d[i], o = b->offset[i];
  if (y) CKR(cudaMemcpy(y, b->y.p + 2 * o, 2 * n * sizeof(double), cudaMemcpyDeviceToHost));
  if (A) CKR(cudaMemcpy(A, b->A.p + 4 * o, 4 * n * sizeof(double), cudaMemcpyDeviceToHost));
  return 0;
}

int glb_batch_destroy(glb_batch *b) {
  if (!b) return 0;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->e0) cudaEventDestroy(b->e0);
  if (b->e1) cudaEventDestroy(b->e1);
  cudaStream_t s = b->stream;
  delete b;
  if (s) cudaStreamDestroy(s);
  return 0;
}

}  // extern "C"

// ===================================================================== server
namespace {

__global__ void k_req_keys(const double *x, size_t n, const unsigned *req_of, const double *bbox,
                           unsigned long long *keys, unsigned *idx) {
  size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned r = req_of[i];
  const double *b = bbox + 4 * r;
  double sx = b[2] > b[0] ? 65535.0 / (b[2] - b[0]) : 0.0, sy = b[3] > b[1] ? 65535.0 / (b[3] - b[1]) : 0.0;
  unsigned qx = (unsigned)fmin(fmax((x[2 * i] - b[0]) * sx, 0.0), 65535.0);
  unsigned qy = (unsigned)fmin(fmax((x[2 * i + 1] - b[1]) * sy, 0.0), 65535.0);
  keys[i] = ((unsigned long long)r << 32) | (spread16(qx) | (spread16(qy) << 1));
  idx[i] = (unsigned)i;
}

__global__ void k_gather_sorted(const double *x, const unsigned *perm, size_t n, double *xs) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  unsigned i = perm[k];
  xs[2 * k] = x[2 * (size_t)i];
  xs[2 * k + 1] = x[2 * (size_t)i + 1];
}

constexpr int kMaxReqPerBatch = 65536;

struct Req {
  long long ticket;
  int model;
  size_t n;
  const double *x;
  double zs;
  double *y, *A;
  double bbox[4];
  double t_submit = 0, t_start = 0, t_done = 0;
  std::atomic<int> done{0};
  int status = 0;
};

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Device memory of one batch, in bytes per ray: x, sorted x, y, A (10
// doubles), two 64-bit sort keys, three 32-bit index arrays, the radix sort's
// temporary storage (bounded by kSortBytesPerRay per ray plus a constant), the
// 32-ray chunks and the recursion state of requests that take the per-plane
// kernels (12 doubles).
constexpr size_t kSortBytesPerRay = 32;
constexpr size_t kBatchBytesPerRay = 10 * 8 + 2 * 8 + 3 * 4 + kSortBytesPerRay + 8 + 12 * 8;
// Requests of at least this many rays run through the per-plane kernels
// (one launch per plane over the request's rays, the lens path's kernels,
// which fill the GPU for several waves from this size on); smaller ones go
// through k_batch's 32-ray chunks, whose persistent queue balances uneven
// requests better (a stream of 1e3-5e5-ray requests on light cones at 60
// requests/s: 3.84M rays/s all on k_batch against 3.70M with requests from
// 16,384 rays on per plane).  The choice depends only on the request, so its
// result is the same alone and in any mix.
constexpr size_t kServePerPlaneMin = (size_t)1 << 20;
constexpr size_t kBatchBytesFixed = (size_t)4 << 20;

struct Slot {
  cudaStream_t s = nullptr;
  cudaEvent_t ev = nullptr;
  double *hx = nullptr, *hy = nullptr, *hA = nullptr;  // pinned staging (max_rays_per_batch)
  unsigned *hreq = nullptr;
  // device memory of the batch in flight: taken from the device's stream-
  // ordered pool on the slot's stream when the batch launches and given back
  // on the same stream after its results are copied out
  char *dmem = nullptr;
  size_t dbytes = 0;
  std::vector<std::shared_ptr<Req>> reqs;
  std::vector<size_t> offs;
  size_t n = 0;
};

}  // namespace

struct glb_server {
  int device = 0;
  int precision = GLB_PREC_FP64;
  size_t cap = 0;  // rays per batch at most (max_rays_per_batch; the pinned staging of a slot)
  size_t reserve = 0;  // device bytes admission leaves free for everything else
  size_t total_bytes = 0;
  // the server's own stream-ordered pool: it keeps the memory it has reserved
  // (release threshold at its maximum), so batches reuse it instead of mapping
  // new memory each time; admission counts what it holds unused as free
  cudaMemPool_t pool = nullptr;
  std::vector<glb_lens *> models;
  std::vector<LensDev> h_lenses;  // host copies (source-plane defaults of each model)
  DBuf<LensDev> d_lenses;
  NFWTables tab{};
  int grid = 0;
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv_submit, cv_done;
  std::deque<std::shared_ptr<Req>> pending;
  std::deque<int> free_slots;
  std::deque<int> inflight;  // slot indices in launch order
  std::unordered_map<long long, std::shared_ptr<Req>> all;
  long long next_ticket = 1;
  bool stop = false;
  int error = 0;
  std::string error_msg;
  std::thread dispatcher, completer;
  // statistics
  unsigned long long batches = 0, rays_done = 0, reqs_done = 0;
  unsigned long long memory_waits = 0;  // dispatches held back until batches in flight gave memory back
  double busy_t0 = 0, busy_t1 = 0;
  double min_free_gb = -1;  // least free HBM seen at admission
};

namespace {

size_t batch_bytes(size_t n) { return kBatchBytesFixed + n * kBatchBytesPerRay; }

// Source-plane scalars of a request: zs >= 0 as Lens::FindSourcePlane
// (MultiPlane/lens.cpp:2659-2680, the host twin of k_batch's
// find_source_plane), zs < 0 the model's own source plane.
void request_source(const glb_lens *l, const LensDev &d, double zs, int &jmax, double &dls, double &dds) {
  if (zs < 0) {
    jmax = d.jmax_default;
    dls = d.dls_default;
    dds = d.dds_default;
    return;
  }
  const double Ds = coordist(l->cosmo, zs);
  double Dls;
  if (zs <= l->plane_z[0]) {
    jmax = 0;
    Dls = Ds;
  } else {
    jmax = (int)l->planes.size();
    while (l->plane_z[jmax - 1] > zs) --jmax;
    Dls = coordist2(l->cosmo, l->plane_z[jmax - 1], zs);
  }
  dls = Dls / Ds;
  dds = jmax > 0 ? l->Dl[jmax - 1] / Ds : 0.0;
}

// The recursion state of rays already in sorted order (theta = SumPrevAlphas
// = x, A = SumPrevAG = I; the layout of k_init_state).
__global__ void k_init_sorted(const double *xs, size_t n, double *st) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double t0 = xs[2 * k], t1 = xs[2 * k + 1];
  st[k] = t0;
  st[n + k] = t1;
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
}

// Device memory available to a new batch now: free HBM plus memory the
// stream-ordered pool holds but no allocation uses, less the reserve.
size_t admissible_bytes(glb_server *S) {
  size_t freeb = 0, totb = 0;
  if (cudaMemGetInfo(&freeb, &totb) != cudaSuccess) return 0;
  size_t reserved = 0, used = 0;
  cudaMemPoolGetAttribute(S->pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
  cudaMemPoolGetAttribute(S->pool, cudaMemPoolAttrUsedMemCurrent, &used);
  const size_t avail = freeb + (reserved > used ? reserved - used : 0);
  const double gb = avail / 1e9;
  if (S->min_free_gb < 0 || gb < S->min_free_gb) S->min_free_gb = gb;
  return avail > S->reserve ? avail - S->reserve : 0;
}

int launch_slot(glb_server *S, Slot &sl) {
  cudaStream_t s = sl.s;
  size_t n = 0, nr = sl.reqs.size();
  sl.offs.resize(nr);
  std::vector<double> bb(4 * nr);
  for (size_t r = 0; r < nr; ++r) {
    Req &q = *sl.reqs[r];
    sl.offs[r] = n;
    memcpy(sl.hx + 2 * n, q.x, 2 * q.n * sizeof(double));
    for (size_t i = 0; i < q.n; ++i) sl.hreq[n + i] = (unsigned)r;
    memcpy(&bb[4 * r], q.bbox, 4 * sizeof(double));
    n += q.n;
  }
  sl.n = n;
  // the batch's device memory, carved from one stream-ordered allocation
  std::vector<Chunk> C;
  size_t big_max = 0;
  auto per_plane = [S](const Req &q) { return q.n >= kServePerPlaneMin && !S->models[q.model]->planes.empty(); };
  for (size_t r = 0; r < nr; ++r) {
    Req &q = *sl.reqs[r];
    if (per_plane(q)) {
      big_max = std::max(big_max, q.n);
      continue;
    }
    for (size_t c = 0; c < q.n; c += 32) {
      Chunk k;
      memset(&k, 0, sizeof(k));
      k.lens = q.model;
      k.kind = 1;
      k.lanes = (int)std::min<size_t>(32, q.n - c);
      k.a = (int)(sl.offs[r] + c);
      k.zs = q.zs;
      C.push_back(k);
    }
  }
  int bits = 32;
  while ((1ull << (bits - 32)) < nr + 1 && bits < 64) ++bits;
  size_t tb = 0;
  CKR(cub::DeviceRadixSort::SortPairs(nullptr, tb, (unsigned long long *)nullptr, (unsigned long long *)nullptr,
                                      (unsigned *)nullptr, (unsigned *)nullptr, (int)n, 0, bits, s));
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t o_x = 0, o_xs = o_x + al(16 * n), o_y = o_xs + al(16 * n), o_A = o_y + al(16 * n);
  const size_t o_bb = o_A + al(32 * n), o_k = o_bb + al(32 * nr), o_k2 = o_k + al(8 * n);
  const size_t o_idx = o_k2 + al(8 * n), o_perm = o_idx + al(4 * n), o_req = o_perm + al(4 * n);
  const size_t o_ch = o_req + al(4 * n), o_cnt = o_ch + al(C.size() * sizeof(Chunk)), o_tmp = o_cnt + 256;
  const size_t o_st = o_tmp + al(tb);
  sl.dbytes = o_st + al(12 * big_max * sizeof(double));
  CKR(cudaMallocFromPoolAsync((void **)&sl.dmem, sl.dbytes, S->pool, s));
  char *m = sl.dmem;
  double *dx = (double *)(m + o_x), *dxs = (double *)(m + o_xs), *dy = (double *)(m + o_y), *dA = (double *)(m + o_A);
  double *dbb = (double *)(m + o_bb);
  unsigned long long *keys = (unsigned long long *)(m + o_k), *keys2 = (unsigned long long *)(m + o_k2);
  unsigned *idx = (unsigned *)(m + o_idx), *perm = (unsigned *)(m + o_perm), *req_of = (unsigned *)(m + o_req);
  Chunk *dch = (Chunk *)(m + o_ch);
  int *counter = (int *)(m + o_cnt);
  CKR(cudaMemcpyAsync(dx, sl.hx, 2 * n * sizeof(double), cudaMemcpyHostToDevice, s));
  CKR(cudaMemcpyAsync(req_of, sl.hreq, n * sizeof(unsigned), cudaMemcpyHostToDevice, s));
  CKR(cudaMemcpyAsync(dbb, bb.data(), bb.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  k_req_keys<<<nblk(n, 256), 256, 0, s>>>(dx, n, req_of, dbb, keys, idx);
  CKR(cub::DeviceRadixSort::SortPairs(m + o_tmp, tb, keys, keys2, idx, perm, (int)n, 0, bits, s));
  k_gather_sorted<<<nblk(n, 256), 256, 0, s>>>(dx, perm, n, dxs);
  // chunks: requests stay contiguous in sorted order; 32 rays per chunk
  CKR(cudaMemcpyAsync(dch, C.data(), C.size() * sizeof(Chunk), cudaMemcpyHostToDevice, s));
  CKR(cudaMemsetAsync(counter, 0, sizeof(int), s));
  if (!C.empty()) {
    if (S->precision == GLB_PREC_SPLIT)
      k_batch<GLB_PREC_SPLIT><<<S->grid, 128, batch_smem_bytes(128), s>>>(dch, (int)C.size(), S->d_lenses.p, S->tab,
                                                                         dxs, perm, dy, dA, counter);
    else
      k_batch<GLB_PREC_FP64><<<S->grid, 128, batch_smem_bytes(128), s>>>(dch, (int)C.size(), S->d_lenses.p, S->tab,
                                                                        dxs, perm, dy, dA, counter);
    CKR(cudaGetLastError());
  }
  // large requests: the lens path's per-plane kernels over the request's rays
  // (contiguous in sorted order), results scattered to their batch slots
  double *st = (double *)(m + o_st);
  for (size_t r = 0; r < nr; ++r) {
    Req &q = *sl.reqs[r];
    if (!per_plane(q)) continue;
    const glb_lens *l = S->models[q.model];
    const LensDev &d = S->h_lenses[q.model];
    const size_t nq = q.n, off = sl.offs[r];
    StepArgs a;
    memset(&a, 0, sizeof(a));
    a.planes = d.planes;
    a.halos = d.halos;
    a.tab = S->tab;
    a.st = st;
    a.n = nq;
    a.charge = d.charge;
    request_source(l, d, q.zs, a.jmax, a.dls_ds, a.d_ds);
    k_init_sorted<<<nblk(nq, 256), 256, 0, s>>>(dxs + 2 * off, nq, st);
    if (int rc = launch_plane_steps(l, a, a.jmax, S->precision, s, nullptr)) return rc;
    k_finish<<<nblk(nq, 256), 256, 0, s>>>(st, perm + off, nq, dy, dA);
    CKR(cudaGetLastError());
  }
  CKR(cudaMemcpyAsync(sl.hy, dy, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CKR(cudaMemcpyAsync(sl.hA, dA, 4 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
  CKR(cudaFreeAsync(sl.dmem, s));
  CKR(cudaEventRecord(sl.ev, s));
  return 0;
}

// Continuous batching: whenever a slot is free, every pending request that fits
// the slot's ray budget (in arrival order) is admitted into one batch and
// launched, while earlier batches are still running on the other slots.
void dispatcher_main(glb_server *S) {
  cudaSetDevice(S->device);
  for (;;) {
    int si;
    std::vector<std::shared_ptr<Req>> take;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      for (;;) {
        S->cv_submit.wait(lk, [&] { return S->stop || (!S->pending.empty() && !S->free_slots.empty()); });
        if (S->stop) return;
        // admission by the device memory free now (re-read at every dispatch)
        const size_t avail = admissible_bytes(S);
        size_t budget = avail > kBatchBytesFixed ? (avail - kBatchBytesFixed) / kBatchBytesPerRay : 0;
        budget = std::min(budget, S->cap);
        if (S->pending.front()->n <= budget) {
          size_t used = 0;
          while (!S->pending.empty() && used + S->pending.front()->n <= budget &&
                 (int)take.size() < kMaxReqPerBatch) {
            used += S->pending.front()->n;
            take.push_back(S->pending.front());
            S->pending.pop_front();
          }
          break;
        }
        if (S->inflight.empty()) {
          // nothing will give memory back: the request cannot run now
          auto q = S->pending.front();
          S->pending.pop_front();
          q->status = GLB_ERR_OOM;
          q->t_start = q->t_done = now_s();
          q->done.store(1);
          S->cv_done.notify_all();
          continue;
        }
        // wait for a batch in flight to finish and give its memory back
        ++S->memory_waits;
        const unsigned long long b0 = S->batches;
        S->cv_submit.wait(lk, [&] { return S->stop || S->batches != b0; });
      }
      si = S->free_slots.front();
      S->free_slots.pop_front();
    }
    Slot &sl = *S->slots[si];
    sl.reqs = take;
    double t = now_s();
    for (auto &q : take) q->t_start = t;
    int rc = launch_slot(S, sl);
    std::lock_guard<std::mutex> lk(S->mu);
    if (rc) {
      S->error = rc;
      S->error_msg = t_err;
      for (auto &q : take) {
        q->status = rc;
        q->done.store(1);
      }
      S->free_slots.push_back(si);
      S->cv_done.notify_all();
    } else {
      if (S->busy_t0 == 0) S->busy_t0 = t;
      S->inflight.push_back(si);
      S->cv_done.notify_all();
    }
  }
}

// Completion: waits for batches in launch order and hands results back.
void completer_main(glb_server *S) {
  cudaSetDevice(S->device);
  for (;;) {
    int si;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_done.wait(lk, [&] { return S->stop || !S->inflight.empty(); });
      if (S->inflight.empty() && S->stop) return;
      si = S->inflight.front();
    }
    Slot &sl = *S->slots[si];
    cudaError_t e = cudaEventSynchronize(sl.ev);
    double t = now_s();
    for (size_t r = 0; r < sl.reqs.size(); ++r) {
      Req &q = *sl.reqs[r];
      if (e == cudaSuccess) {
        memcpy(q.y, sl.hy + 2 * sl.offs[r], 2 * q.n * sizeof(double));
        memcpy(q.A, sl.hA + 4 * sl.offs[r], 4 * q.n * sizeof(double));
      } else {
        q.status = GLB_ERR_CUDA;
      }
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->inflight.pop_front();
    for (auto &q : sl.reqs) {
      q->t_done = t;
      q->done.store(1);
      S->rays_done += q->n;
      S->reqs_done += 1;
    }
    S->batches += 1;
    S->busy_t1 = t;
    sl.reqs.clear();
    S->free_slots.push_back(si);
    S->cv_submit.notify_all();
    S->cv_done.notify_all();
  }
}

}  // namespace

extern "C" {

int glb_server_create(glb_lens *const *models, int nmodels, size_t max_rays_per_batch, int precision, int nslots,
                      glb_server **out) {
  if (!out || !models || nmodels <= 0) return fail(GLB_ERR_ARG, "null argument");
  if (precision != GLB_PREC_FP64 && precision != GLB_PREC_SPLIT) return fail(GLB_ERR_ARG, "unknown precision");
  if (nslots < 1 || nslots > 8) return fail(GLB_ERR_ARG, "nslots must be in [1, 8]");
  if (int rc = need_device()) return rc;
  auto S = std::make_unique<glb_server>();
  CKR(cudaGetDevice(&S->device));
  S->precision = precision;
  // rays per batch at most (the pinned host staging of each slot); the device
  // memory of a batch is taken when it launches, against the HBM free then
  S->cap = std::min<size_t>(max_rays_per_batch ? max_rays_per_batch : (size_t)4 << 20, (size_t)1 << 30);
  size_t freeb = 0, totb = 0;
  CKR(cudaMemGetInfo(&freeb, &totb));
  S->reserve = totb / 20;  // 5 % of HBM stays free for other work
  S->total_bytes = totb;
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = S->device;
  CKR(cudaMemPoolCreate(&S->pool, &props));
  unsigned long long keep = ~0ull;  // cudaMemPoolAttrReleaseThreshold is a 64-bit value
  CKR(cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  std::vector<LensDev> L(nmodels);
  for (int i = 0; i < nmodels; ++i) {
    if (!models[i] || models[i]->device != S->device) return fail(GLB_ERR_ARG, "models must be lenses on one device");
    if (int rc = make_lens_dev(models[i], L[i])) return rc;
    S->models.push_back(models[i]);
    S->h_lenses.push_back(L[i]);
  }
  CKR(S->d_lenses.alloc(nmodels));
  CKR(cudaMemcpy(S->d_lenses.p, L.data(), nmodels * sizeof(LensDev), cudaMemcpyHostToDevice));
  if (int rc = device_nfw_tables(S->tab)) return rc;
  if (int rc = persistent_grid(128, precision, &S->grid)) return rc;
  size_t cap = S->cap;
  for (int i = 0; i < nslots; ++i) {
    auto sl = std::make_unique<Slot>();
    CKR(cudaStreamCreateWithFlags(&sl->s, cudaStreamNonBlocking));
    CKR(cudaEventCreateWithFlags(&sl->ev, cudaEventBlockingSync | cudaEventDisableTiming));
    CKR(cudaMallocHost((void **)&sl->hx, 2 * cap * sizeof(double)));
    CKR(cudaMallocHost((void **)&sl->hy, 2 * cap * sizeof(double)));
    CKR(cudaMallocHost((void **)&sl->hA, 4 * cap * sizeof(double)));
    CKR(cudaMallocHost((void **)&sl->hreq, cap * sizeof(unsigned)));
    S->slots.push_back(std::move(sl));
    S->free_slots.push_back(i);
  }
  glb_server *p = S.release();
  p->dispatcher = std::thread(dispatcher_main, p);
  p->completer = std::thread(completer_main, p);
  *out = p;
  return 0;
}

int glb_server_submit(glb_server *S, int model, size_t n, const double *x, double zs, double *y, double *A,
                      long long *ticket) {
  if (!S || !ticket || (n > 0 && (!x || !y || !A))) return fail(GLB_ERR_ARG, "null argument");
  if (model < 0 || model >= (int)S->models.size()) return fail(GLB_ERR_ARG, "unknown model");
  if (n > S->cap) return fail(GLB_ERR_ARG, "request larger than the server's ray budget per batch");
  if (n > 0 && batch_bytes(n) + S->reserve > S->total_bytes)
    return fail(GLB_ERR_OOM, "request larger than the device memory could ever hold");
  auto q = std::make_shared<Req>();
  q->model = model;
  q->n = n;
  q->x = x;
  q->zs = zs;
  q->y = y;
  q->A = A;
  q->bbox[0] = q->bbox[1] = 1e300;
  q->bbox[2] = q->bbox[3] = -1e300;
  for (size_t i = 0; i < n; ++i) {
    q->bbox[0] = std::min(q->bbox[0], x[2 * i]);
    q->bbox[1] = std::min(q->bbox[1], x[2 * i + 1]);
    q->bbox[2] = std::max(q->bbox[2], x[2 * i]);
    q->bbox[3] = std::max(q->bbox[3], x[2 * i + 1]);
  }
  q->t_submit = now_s();
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->stop) return fail(GLB_ERR_ARG, "server stopped");
  q->ticket = S->next_ticket++;
  if (n == 0) {
    q->t_start = q->t_done = q->t_submit;
    q->done.store(1);
  } else {
    S->pending.push_back(q);
    S->cv_submit.notify_all();
  }
  S->all[q->ticket] = q;
  *ticket = q->ticket;
  return 0;
}

int glb_server_wait(glb_server *S, long long ticket, double timeout_s, double *times) {
  if (!S) return fail(GLB_ERR_ARG, "null server");
  std::shared_ptr<Req> q;
  {
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(ticket);
    if (it == S->all.end()) return fail(GLB_ERR_ARG, "unknown ticket");
    q = it->second;
    auto pred = [&] { return q->done.load() != 0; };
    if (timeout_s > 0) {
      if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
        return fail(GLB_ERR_TIMEOUT, "request not finished within the timeout");
    } else {
      S->cv_done.wait(lk, pred);
    }
    S->all.erase(ticket);
  }
  if (times) {
    times[0] = q->t_submit;
    times[1] = q->t_start;
    times[2] = q->t_done;
  }
  if (q->status) return fail(q->status, "request failed on the device");
  return 0;
}

int glb_server_poll(glb_server *S, long long ticket, int *done) {
  if (!S || !done) return fail(GLB_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->all.find(ticket);
  if (it == S->all.end()) return fail(GLB_ERR_ARG, "unknown ticket");
  *done = it->second->done.load();
  return 0;
}

int glb_server_stats(glb_server *S, double *stats) {
  if (!S || !stats) return fail(GLB_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  stats[0] = (double)S->rays_done;
  stats[1] = (double)S->reqs_done;
  stats[2] = (double)S->batches;
  stats[3] = S->busy_t1 - S->busy_t0;
  stats[4] = (double)S->cap;
  stats[5] = (double)S->pending.size();
  return 0;
}

int glb_server_admission(glb_server *S, double *memory_waits, double *min_free_gb) {
  if (!S) return fail(GLB_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lk(S->mu);
  if (memory_waits) *memory_waits = (double)S->memory_waits;
  if (min_free_gb) *min_free_gb = S->min_free_gb;
  return 0;
}

int glb_server_destroy(glb_server *S) {
  if (!S) return 0;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_submit.notify_all();
  S->cv_done.notify_all();
  if (S->dispatcher.joinable()) S->dispatcher.join();
  // let the batches already on the GPU finish before the slots go away
  for (auto &sl : S->slots) cudaStreamSynchronize(sl->s);
  {
    std::lock_guard<std::mutex> lk(S->mu);
  }
  S->cv_done.notify_all();
  if (S->completer.joinable()) S->completer.join();
  cudaSetDevice(S->device);
  for (auto &sl : S->slots) {
    cudaStreamSynchronize(sl->s);
    cudaFreeHost(sl->hx);
    cudaFreeHost(sl->hy);
    cudaFreeHost(sl->hA);
    cudaFreeHost(sl->hreq);
    cudaEventDestroy(sl->ev);
    cudaStreamDestroy(sl->s);
  }
  if (S->pool) cudaMemPoolDestroy(S->pool);
  delete S;
  return 0;
}

}  // extern "C"
