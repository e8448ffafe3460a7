// Adaptive kNN smoothing of particles on the device
// (LensHaloParticles::calculate_smoothing, include/particle_halo.h:683-730).
//
// The reference sets every particle's Size to TreeSimple::NNDistance(x, Nsmooth+1)
// (include/simpleTree.h:483-618): the heap of the query's leaf (or its parent
// when the leaf holds fewer than Nsmooth+1 particles) seeds a bound that a
// full preorder walk of a median-split 3-d tree then tightens, so the value
// returned is the exact (Nsmooth+1)-th smallest distance from the particle
// (itself included), squared distances being summed in double from float
// coordinate differences and the square root rounded to float.  One case is
// not exact: when the node seeding the heap is the tree's top node (only
// possible for N = 2*Nsmooth+1, for queries in the top node's first child) the
// walk revisits the top node's two leaves and pushes their particles again.
//
// Here the answer is computed directly, without the reference's tree:
//   1. particles are sorted along a 63-bit Morton curve of the bounding box
//      and cut into buckets of S..2S-1 consecutive particles
//      (S = 2*Nsmooth rounded up to 32);
//   2. an implicit binary tree over the buckets carries float bounding boxes,
//      and every aligned 32-particle chunk of the sorted array has its box;
//   3. one CTA per bucket: every query first takes the (Nsmooth+1)-th
//      smallest squared distance within its own bucket as a bound; the CTA
//      lists the buckets whose boxes lie within the largest bound of its
//      queries, ordered by a lower bound of their gap to its own box; each
//      warp then scans the list per query until that gap bound passes the
//      query's current bound, and reads the chunks of the buckets within the
//      bound into a shared-memory buffer of squared distances below it,
//      cutting the buffer back to exactly Nsmooth+1 entries (and the bound to
//      their maximum) after each bucket once it holds twice that;
//   4. the (Nsmooth+1)-th smallest entry, selected exactly on its 64-bit
//      pattern, is the answer.
// Box tests use the same float subtraction as the distances, so a box is
// skipped only when every particle in it is at least the bound away in the
// computed arithmetic.  The N = 2*Nsmooth+1 case replays the reference's walk
// for the affected queries (k_knn_top_walk).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "glb_host.h"

namespace glb {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kWarps = 4;         // warps per CTA in k_knn
constexpr int kListCap = 1024;    // candidate buckets listed per CTA
constexpr int kStack = 64;        // per-warp DFS stack (tree depth <= 31)
constexpr int kFront = 512;       // breadth-first frontier of the candidate search

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return Status::err(-2, std::string("CUDA: ") + cudaGetErrorString(e_) + " at " \
                                 + #call);                                           \
  } while (0)

__device__ __forceinline__ unsigned f2ord(float f) {
  unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float ord2f(unsigned u) {
  unsigned b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  float f;
  memcpy(&f, &b, 4);
  return f;
}

// Squared distance as NNDistance sums it: ((dx^2 + dy^2) + dz^2) in double
// from float differences (each square is exact in double).
__device__ __forceinline__ double knn_r2(float px, float py, float pz, float qx, float qy, float qz) {
  const double dx = (double)__fsub_rn(px, qx);
  const double dy = (double)__fsub_rn(py, qy);
  const double dz = (double)__fsub_rn(pz, qz);
  return __fma_rn(dz, dz, __fma_rn(dy, dy, __dmul_rn(dx, dx)));
}

// Lower bound of knn_r2 over a box: per axis the float gap, rounded like the
// particle differences (rounding is monotone, so no particle in the box has a
// smaller computed difference), squared and summed in the same order.
__device__ __forceinline__ float gap1(float q, float lo, float hi) {
  return q < lo ? __fsub_rn(lo, q) : (q > hi ? __fsub_rn(q, hi) : 0.f);
}
__device__ __forceinline__ double gap2_point(float qx, float qy, float qz, float4 lo, float4 hi) {
  const double gx = gap1(qx, lo.x, hi.x), gy = gap1(qy, lo.y, hi.y), gz = gap1(qz, lo.z, hi.z);
  return __fma_rn(gz, gz, __fma_rn(gy, gy, __dmul_rn(gx, gx)));
}
// Between any point of box a and any point of box b.
__device__ __forceinline__ float gapbb(float alo, float ahi, float blo, float bhi) {
  return ahi < blo ? __fsub_rn(blo, ahi) : (bhi < alo ? __fsub_rn(alo, bhi) : 0.f);
}
__device__ __forceinline__ double gap2_box(float4 alo, float4 ahi, float4 blo, float4 bhi) {
  const double gx = gapbb(alo.x, ahi.x, blo.x, bhi.x), gy = gapbb(alo.y, ahi.y, blo.y, bhi.y),
               gz = gapbb(alo.z, ahi.z, blo.z, bhi.z);
  return __fma_rn(gz, gz, __fma_rn(gy, gy, __dmul_rn(gx, gx)));
}

__device__ __forceinline__ unsigned long long warp_max64(unsigned long long v) {
  for (int o = 16; o; o >>= 1) {
    unsigned long long w = __shfl_xor_sync(kFull, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// k-th smallest (1-based) of buf[0, cnt) (non-negative doubles, so the bit
// patterns order like the values), by bitwise radix selection from the
// highest bit in which the entries differ, first on the high 32-bit words and
// then, among the entries sharing the selected high word, on the low words;
// stops as soon as one entry is left.  Exact zeros (a particle's distance to
// itself or to a coincident one) are counted apart, so that the selection
// starts from the highest bit in which the non-zero entries differ.
__device__ __noinline__ double warp_select(const double *buf, int cnt, int k, int lane) {
  unsigned lo = kFull, hi = 0u;
  int zeros = 0;
  for (int i = lane; i < cnt; i += 32) {
    const unsigned h = (unsigned)__double2hiint(buf[i]);
    if (h == 0u && buf[i] == 0.0) {
      ++zeros;
      continue;
    }
    lo = min(lo, h);
    hi = max(hi, h);
  }
  zeros = (int)__reduce_add_sync(kFull, (unsigned)zeros);
  if (k <= zeros) return 0.0;
  k -= zeros;
  lo = __reduce_min_sync(kFull, lo);
  hi = __reduce_max_sync(kFull, hi);
  unsigned hword = lo;
  int act = cnt - zeros;
  if (lo != hi) {
    const int top = 31 - __clz(lo ^ hi);
    unsigned above = top >= 31 ? 0u : ~((2u << top) - 1u);
    unsigned prefix = lo & above;
    for (int b = top; b >= 0; --b) {
      const unsigned bit = 1u << b;
      int c0 = 0;
      for (int i = lane; i < cnt; i += 32) {
        const double v = buf[i];
        const unsigned h = (unsigned)__double2hiint(v);
        c0 += ((h & above) == prefix) && !(h & bit) && v != 0.0;
      }
      c0 = (int)__reduce_add_sync(kFull, (unsigned)c0);
      if (k <= c0) {
        act = c0;
      } else {
        k -= c0;
        prefix |= bit;
        act -= c0;
      }
      above |= bit;
      if (act == 1) {
        unsigned long long f = 0ull;
        for (int i = lane; i < cnt; i += 32) {
          const unsigned long long u = __double_as_longlong(buf[i]);
          if (((unsigned)(u >> 32) & above) == prefix && u != 0ull) f = u;
        }
        return __longlong_as_double(warp_max64(f));
      }
    }
    hword = prefix;
  }
  // act entries share the high word `hword`; rank k among their low words
  unsigned llo = kFull, lhi = 0u;
  for (int i = lane; i < cnt; i += 32) {
    const unsigned long long u = __double_as_longlong(buf[i]);
    if ((unsigned)(u >> 32) == hword) {
      llo = min(llo, (unsigned)u);
      lhi = max(lhi, (unsigned)u);
    }
  }
  llo = __reduce_min_sync(kFull, llo);
  lhi = __reduce_max_sync(kFull, lhi);
  if (llo == lhi) return __hiloint2double((int)hword, (int)llo);
  const int top = 31 - __clz(llo ^ lhi);
  unsigned above = top >= 31 ? 0u : ~((2u << top) - 1u);
  unsigned prefix = llo & above;
  for (int b = top; b >= 0; --b) {
    const unsigned bit = 1u << b;
    int c0 = 0;
    for (int i = lane; i < cnt; i += 32) {
      const unsigned long long u = __double_as_longlong(buf[i]);
      const unsigned l = (unsigned)u;
      c0 += ((unsigned)(u >> 32) == hword) && ((l & above) == prefix) && !(l & bit);
    }
    c0 = (int)__reduce_add_sync(kFull, (unsigned)c0);
    if (k <= c0) {
      act = c0;
    } else {
      k -= c0;
      prefix |= bit;
      act -= c0;
    }
    above |= bit;
    if (act == 1) break;
  }
  if (act == 1) {
    unsigned f = 0u;
    for (int i = lane; i < cnt; i += 32) {
      const unsigned long long u = __double_as_longlong(buf[i]);
      if ((unsigned)(u >> 32) == hword && ((unsigned)u & above) == prefix) f = (unsigned)u;
    }
    return __hiloint2double((int)hword, (int)__reduce_max_sync(kFull, f));
  }
  return __hiloint2double((int)hword, (int)prefix);
}

// Keeps exactly K entries of buf[0, cnt): all below beta (the K-th smallest)
// and as many equal to beta as needed.  Returns K.
__device__ __noinline__ int warp_compact(double *buf, int cnt, int K, double beta, int lane) {
  int nless = 0;
  for (int i = lane; i < cnt; i += 32) nless += buf[i] < beta;
  nless = (int)__reduce_add_sync(kFull, (unsigned)nless);
  const int need = K - nless;
  int w = 0, eq = 0;
  const unsigned lt_mask = (1u << lane) - 1u;
  for (int base = 0; base < cnt; base += 32) {
    const int i = base + lane;
    const double v = i < cnt ? buf[i] : 0.0;
    const bool less = i < cnt && v < beta, equal = i < cnt && v == beta;
    const unsigned em = __ballot_sync(kFull, equal);
    const bool keep = less || (equal && eq + __popc(em & lt_mask) < need);
    const unsigned km = __ballot_sync(kFull, keep);
    __syncwarp();
    if (keep) buf[w + __popc(km & lt_mask)] = v;
    __syncwarp();
    w += __popc(km);
    eq += __popc(em);
  }
  return w;
}

// ------------------------------------------------------------------ build
__global__ void k_bbox3(const glb_particle_rec *p, size_t n, unsigned *mm) {
  unsigned lo[3] = {kFull, kFull, kFull}, hi[3] = {0u, 0u, 0u};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const unsigned o = f2ord(p[i].x[k]);
      lo[k] = min(lo[k], o);
      hi[k] = max(hi[k], o);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    lo[k] = __reduce_min_sync(kFull, lo[k]);
    hi[k] = __reduce_max_sync(kFull, hi[k]);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      atomicMin(&mm[k], lo[k]);
      atomicMax(&mm[3 + k], hi[k]);
    }
  }
}

// 21-bit integer -> every third bit of a 63-bit word.
__device__ __forceinline__ unsigned long long spread3(unsigned v) {
  unsigned long long x = v & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffull;
  x = (x | x << 16) & 0x1f0000ff0000ffull;
  x = (x | x << 8) & 0x100f00f00f00f00full;
  x = (x | x << 4) & 0x10c30c30c30c30c3ull;
  x = (x | x << 2) & 0x1249249249249249ull;
  return x;
}

__global__ void k_morton3(const glb_particle_rec *p, size_t n, const unsigned *mm, unsigned long long *key,
                          unsigned *idx) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned q[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float lo = ord2f(mm[k]), ext = ord2f(mm[3 + k]) - lo;
    const float sc = ext > 0.f && isfinite(ext) ? 2097151.f / ext : 0.f;
    q[k] = (unsigned)fminf(fmaxf((p[i].x[k] - lo) * sc, 0.f), 2097151.f);
  }
  key[i] = spread3(q[0]) | (spread3(q[1]) << 1) | (spread3(q[2]) << 2);
  idx[i] = (unsigned)i;
}

__global__ void k_gather_pos(const glb_particle_rec *p, const unsigned *sidx, size_t n, float4 *pos) {
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const unsigned j = sidx[i];
  pos[i] = make_float4(p[j].x[0], p[j].x[1], p[j].x[2], __uint_as_float(j));
}

__device__ __forceinline__ size_t bucket_start(int b, size_t n, int nb) { return (size_t)b * n / (size_t)nb; }

// One warp per leaf slot of the implicit tree: the bucket's bounding box, or
// an empty box for padding slots.
__global__ void k_bucket_box(const float4 *pos, size_t n, int nb, int P, float4 *blo, float4 *bhi) {
  const int b = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (b >= P) return;
  float lx = INFINITY, ly = INFINITY, lz = INFINITY, hx = -INFINITY, hy = -INFINITY, hz = -INFINITY;
  if (b < nb) {
    const size_t s = bucket_start(b, n, nb), e = bucket_start(b + 1, n, nb);
    for (size_t i = s + lane; i < e; i += 32) {
      const float4 v = pos[i];
      lx = fminf(lx, v.x);
      ly = fminf(ly, v.y);
      lz = fminf(lz, v.z);
      hx = fmaxf(hx, v.x);
      hy = fmaxf(hy, v.y);
      hz = fmaxf(hz, v.z);
    }
  }
  for (int o = 16; o; o >>= 1) {
    lx = fminf(lx, __shfl_xor_sync(kFull, lx, o));
    ly = fminf(ly, __shfl_xor_sync(kFull, ly, o));
    lz = fminf(lz, __shfl_xor_sync(kFull, lz, o));
    hx = fmaxf(hx, __shfl_xor_sync(kFull, hx, o));
    hy = fmaxf(hy, __shfl_xor_sync(kFull, hy, o));
    hz = fmaxf(hz, __shfl_xor_sync(kFull, hz, o));
  }
  if (lane == 0) {
    blo[P + b] = make_float4(lx, ly, lz, 0.f);
    bhi[P + b] = make_float4(hx, hy, hz, 0.f);
  }
}

// One warp per aligned 32-particle chunk of the sorted array: its box.
__global__ void k_chunk_box(const float4 *pos, size_t n, float4 *clo, float4 *chi) {
  const size_t c = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (c >= (n + 31) / 32) return;
  const size_t i = (c << 5) + lane;
  float4 v = pos[i < n ? i : c << 5];
  float lx = v.x, ly = v.y, lz = v.z, hx = v.x, hy = v.y, hz = v.z;
  for (int o = 16; o; o >>= 1) {
    lx = fminf(lx, __shfl_xor_sync(kFull, lx, o));
    ly = fminf(ly, __shfl_xor_sync(kFull, ly, o));
    lz = fminf(lz, __shfl_xor_sync(kFull, lz, o));
    hx = fmaxf(hx, __shfl_xor_sync(kFull, hx, o));
    hy = fmaxf(hy, __shfl_xor_sync(kFull, hy, o));
    hz = fmaxf(hz, __shfl_xor_sync(kFull, hz, o));
  }
  if (lane == 0) {
    clo[c] = make_float4(lx, ly, lz, 0.f);
    chi[c] = make_float4(hx, hy, hz, 0.f);
  }
}

// Internal nodes [w, 2w) of the implicit tree from their children.
__global__ void k_box_up(int w, float4 *blo, float4 *bhi) {
  const int i = w + (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (i >= 2 * w) return;
  const float4 a = blo[2 * i], b = blo[2 * i + 1], c = bhi[2 * i], d = bhi[2 * i + 1];
  blo[i] = make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), 0.f);
  bhi[i] = make_float4(fmaxf(c.x, d.x), fmaxf(c.y, d.y), fmaxf(c.z, d.z), 0.f);
}

// ----------------------------------------------------------------- search
struct KnnArgs {
  const float4 *pos;  // Morton-sorted {x, y, z, original index}
  const float4 *blo, *bhi;
  const float4 *clo, *chi;  // boxes of the aligned 32-particle chunks of pos
  size_t n;
  int nb, P, K, cap;
  int shrink_at;      // buffer size that triggers a shrink after a bucket
  float *size_out;    // indexed by original particle index
  int *flags;         // [0]: CTAs whose candidate list overflowed
};

// Appends the squared distances below beta of bucket c's particles to the
// warp's buffer.  The bucket's aligned 32-particle chunks are tested against
// beta first (one chunk box per lane); only chunks within it are read.  The
// buffer is cut back to K entries (and beta to their largest) whenever the
// next 32 might not fit, and after the bucket once it holds shrink_at entries,
// so that the bound tightens early.
__device__ __forceinline__ void knn_visit(const KnnArgs &a, int c, float qx, float qy, float qz, double *buf,
                                          int &cnt, double &beta, int lane) {
  const size_t s = bucket_start(c, a.n, a.nb), e = bucket_start(c + 1, a.n, a.nb);
  const unsigned lt_mask = (1u << lane) - 1u;
  const size_t ch0 = s >> 5, nch = ((e - 1) >> 5) - ch0 + 1;
  for (size_t cg = 0; cg < nch; cg += 32) {
    const size_t ch = ch0 + cg + lane;
    const bool near = cg + lane < nch && gap2_point(qx, qy, qz, a.clo[ch], a.chi[ch]) < beta;
    unsigned cm = __ballot_sync(kFull, near);
    while (cm) {
      const int l = __ffs(cm) - 1;
      cm &= cm - 1;
      if (cnt + 32 > a.cap) {
        beta = warp_select(buf, cnt, a.K, lane);
        cnt = warp_compact(buf, cnt, a.K, beta, lane);
      }
      const size_t i = ((ch0 + cg + l) << 5) + lane;
      double r2 = 0.0;
      bool keep = false;
      if (i >= s && i < e) {
        const float4 v = a.pos[i];
        r2 = knn_r2(v.x, v.y, v.z, qx, qy, qz);
        keep = r2 < beta;
      }
      const unsigned m = __ballot_sync(kFull, keep);
      if (keep) buf[cnt + __popc(m & lt_mask)] = r2;
      cnt += __popc(m);
      __syncwarp();
    }
  }
  if (cnt >= a.shrink_at) {
    beta = warp_select(buf, cnt, a.K, lane);
    cnt = warp_compact(buf, cnt, a.K, beta, lane);
  }
}

#ifndef GLB_KNN_MIN_BLOCKS
#define GLB_KNN_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(kWarps * 32, GLB_KNN_MIN_BLOCKS) k_knn(KnnArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const size_t s0 = bucket_start(b, a.n, a.nb);
  const int m = (int)(bucket_start(b + 1, a.n, a.nb) - s0);
  const int mmax = (int)((a.n + a.nb - 1) / a.nb);
  float4 *own = reinterpret_cast<float4 *>(smem);
  double *qbeta = reinterpret_cast<double *>(own + mmax);
  double *buf = qbeta + mmax + (size_t)warp * a.cap;
  int *list = reinterpret_cast<int *>(qbeta + mmax + (size_t)kWarps * a.cap);
  int *stack = list + kListCap + warp * kStack;
  int *front = list + kListCap + kWarps * kStack;
  float *lkey = reinterpret_cast<float *>(front + 2 * kFront);  // gap bound of each sorted list entry
  __shared__ unsigned long long s_r2max;
  __shared__ int s_nlist, s_overflow, s_fn[2];

  for (int i = tid; i < m; i += blockDim.x) own[i] = a.pos[s0 + i];
  if (tid == 0) {
    s_r2max = 0ull;
    s_nlist = 0;
    s_overflow = 0;
  }
  __syncthreads();

  // 1. bound of every query from its own bucket (m >= K)
  unsigned long long r2max = 0ull;
  for (int q = warp; q < m; q += kWarps) {
    const float4 x = own[q];
    for (int i = lane; i < m; i += 32) buf[i] = knn_r2(own[i].x, own[i].y, own[i].z, x.x, x.y, x.z);
    __syncwarp();
    const double beta = warp_select(buf, m, a.K, lane);
    if (lane == 0) qbeta[q] = beta;
    const unsigned long long u = __double_as_longlong(beta);
    r2max = u > r2max ? u : r2max;
    __syncwarp();
  }
  if (lane == 0) atomicMax(&s_r2max, r2max);
  __syncthreads();

  // 2. buckets whose box lies within the largest bound of the box of this one,
  //    level by level over the implicit tree by all threads of the CTA
  {
    const double R2 = __longlong_as_double(s_r2max);
    const float4 olo = a.blo[a.P + b], ohi = a.bhi[a.P + b];
    if (tid == 0) {
      s_fn[0] = a.P > 1 ? 1 : 0;
      s_fn[1] = 0;
      front[0] = 1;
    }
    __syncthreads();
    int cur = 0;
    for (;;) {
      const int nf = min(s_fn[cur], kFront);
      __syncthreads();
      if (nf == 0) break;
      for (int i = tid; i < nf; i += blockDim.x) {
        const int node = front[cur * kFront + i];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int ch = 2 * node + h;
          if (!(gap2_box(olo, ohi, a.blo[ch], a.bhi[ch]) < R2)) continue;
          if (ch >= a.P) {
            const int c = ch - a.P;
            if (c == b || c >= a.nb) continue;
            const int k = atomicAdd(&s_nlist, 1);
            if (k < kListCap) list[k] = c;
            else s_overflow = 1;
          } else {
            const int k = atomicAdd(&s_fn[cur ^ 1], 1);
            if (k < kFront) front[(cur ^ 1) * kFront + k] = ch;
            else s_overflow = 1;
          }
        }
      }
      if (tid == 0) s_fn[cur] = 0;
      __syncthreads();
      cur ^= 1;
    }
  }
  if (tid == 0 && s_overflow) atomicAdd(&a.flags[0], 1);
  __syncthreads();
  const int nlist = min(s_nlist, kListCap);
  const bool overflow = s_overflow != 0;
  // near-first order: by a lower bound (rounded down to float) of the gap
  // between this bucket's box and the candidate's, then by the distance
  // between box centres; rank sort in the (still unused) warp buffers.  The
  // gap order lets a query stop at the first entry whose bound is beyond it.
  const float4 olo = a.blo[a.P + b], ohi = a.bhi[a.P + b];
  const bool sorted = !overflow && nlist > 1 && (size_t)nlist * 12 <= (size_t)kWarps * a.cap * sizeof(double);
  if (sorted) {
    const float ox = 0.5f * (olo.x + ohi.x), oy = 0.5f * (olo.y + ohi.y), oz = 0.5f * (olo.z + ohi.z);
    float *k1 = reinterpret_cast<float *>(qbeta + mmax);
    float *k2 = k1 + nlist;
    int *ids = reinterpret_cast<int *>(k2 + nlist);
    for (int i = tid; i < nlist; i += blockDim.x) {
      const int c = list[i];
      const float4 lo = a.blo[a.P + c], hi = a.bhi[a.P + c];
      k1[i] = __double2float_rd(gap2_box(olo, ohi, lo, hi));
      const float dx = 0.5f * (lo.x + hi.x) - ox, dy = 0.5f * (lo.y + hi.y) - oy, dz = 0.5f * (lo.z + hi.z) - oz;
      k2[i] = dx * dx + dy * dy + dz * dz;
    }
    __syncthreads();
    for (int i = tid; i < nlist; i += blockDim.x) {
      const float g = k1[i], d = k2[i];
      int r = 0;
      for (int j = 0; j < nlist; ++j) {
        const float gj = k1[j], dj = k2[j];
        r += (gj < g) || (gj == g && (dj < d || (dj == d && j < i)));
      }
      ids[r] = list[i];
      lkey[r] = g;
    }
    __syncthreads();
    for (int i = tid; i < nlist; i += blockDim.x) list[i] = ids[i];
    __syncthreads();
  }

  // 3. per query: own bucket below its bound, then the candidates
  for (int q = warp; q < m; q += kWarps) {
    const float4 x = own[q];
    double beta = qbeta[q];
    int cnt = 0;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int base = 0; base < m; base += 32) {
      const int i = base + lane;
      double r2 = 0.0;
      bool keep = false;
      if (i < m) {
        r2 = knn_r2(own[i].x, own[i].y, own[i].z, x.x, x.y, x.z);
        keep = r2 <= beta;
      }
      const unsigned msk = __ballot_sync(kFull, keep);
      if (keep) buf[cnt + __popc(msk & lt_mask)] = r2;
      cnt += __popc(msk);
    }
    __syncwarp();
    if (cnt > a.K) cnt = warp_compact(buf, cnt, a.K, beta, lane);
    if (!overflow) {
      // 32 listed boxes tested at once against the current bound
      for (int base = 0; base < nlist; base += 32) {
        // every later entry is at least as far from this bucket's box
        if (sorted && (double)lkey[base] >= beta) break;
        const int li = base + lane;
        const int c = li < nlist ? list[li] : 0;
        const bool near = li < nlist && gap2_point(x.x, x.y, x.z, a.blo[a.P + c], a.bhi[a.P + c]) < beta;
        unsigned msk = __ballot_sync(kFull, near);
        while (msk) {
          const int l = __ffs(msk) - 1;
          msk &= msk - 1;
          knn_visit(a, __shfl_sync(kFull, c, l), x.x, x.y, x.z, buf, cnt, beta, lane);
        }
      }
    } else {
      // the list did not fit: walk the tree for this query
      int sp = 0;
      if (lane == 0) stack[0] = 1;
      sp = 1;
      __syncwarp();
      while (sp > 0) {
        const int node = stack[sp - 1];
        __syncwarp();
        --sp;
        if (gap2_point(x.x, x.y, x.z, a.blo[node], a.bhi[node]) >= beta) continue;
        if (node >= a.P) {
          const int c = node - a.P;
          if (c != b && c < a.nb) knn_visit(a, c, x.x, x.y, x.z, buf, cnt, beta, lane);
          continue;
        }
        const int c0 = 2 * node, c1 = 2 * node + 1;
        const double g0 = gap2_point(x.x, x.y, x.z, a.blo[c0], a.bhi[c0]);
        const double g1 = gap2_point(x.x, x.y, x.z, a.blo[c1], a.bhi[c1]);
        const int far = g0 <= g1 ? c1 : c0, near = g0 <= g1 ? c0 : c1;
        if (lane == 0) {
          stack[sp] = far;
          stack[sp + 1] = near;
        }
        sp += 2;
        __syncwarp();
      }
    }
    const double kth = warp_select(buf, cnt, a.K, lane);
    if (lane == 0) a.size_out[__float_as_uint(x.w)] = __double2float_rn(__dsqrt_rn(kth));
    __syncwarp();
  }
}

// ------------------------------------------- N = 2*Nsmooth+1: the reference's walk
// Stable rank of every particle by x (the top node's sort order).
__global__ void k_rank_x(const glb_particle_rec *p, int n, int *order) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float xi = p[i].x[0];
  int r = 0;
  for (int j = 0; j < n; ++j) {
    const float xj = p[j].x[0];
    r += (xj < xi) || (xj == xi && j < i);
  }
  order[r] = i;
}

__device__ void heap_push_d(double *h, int &n, double v) {
  int i = n++;
  while (i > 0) {
    const int up = (i - 1) / 2;
    if (h[up] >= v) break;
    h[i] = h[up];
    i = up;
  }
  h[i] = v;
}
__device__ void heap_pop_d(double *h, int &n) {
  const double v = h[--n];
  int i = 0;
  for (;;) {
    int c = 2 * i + 1;
    if (c >= n) break;
    if (c + 1 < n && h[c + 1] > h[c]) ++c;
    if (h[c] <= v) break;
    h[i] = h[c];
    i = c;
  }
  if (n) h[i] = v;
}

// One CTA (one thread) per particle of the top node's first child: heap of
// the top node's particles, then its two leaves pushed again in order
// (simpleTree.h:561-615 with pass = top).
__global__ void k_knn_top_walk(const glb_particle_rec *p, int n, int K, const int *order, float *size_out) {
  extern __shared__ double heap[];
  if (threadIdx.x != 0) return;
  const int i = blockIdx.x;
  const int cut = n / 2;
  const float xcut = p[order[cut]].x[0], xmin = p[order[0]].x[0], xmax = p[order[n - 1]].x[0];
  const float qx = p[i].x[0], qy = p[i].x[1], qz = p[i].x[2];
  if (!((double)xcut > (double)qx)) return;  // _findleaf went to the second child
  int hn = 0;
  for (int j = 0; j < n; ++j) {
    const glb_particle_rec &pj = p[order[j]];
    const double r2 = knn_r2(pj.x[0], pj.x[1], pj.x[2], qx, qy, qz);
    if (j < K) {
      heap_push_d(heap, hn, r2);
    } else if (r2 < heap[0]) {
      heap_push_d(heap, hn, r2);
      heap_pop_d(heap, hn);
    }
  }
  double bestr = __dsqrt_rn(heap[0]);
  for (int leaf = 0; leaf < 2; ++leaf) {
    const double lo = leaf == 0 ? (double)xmin : (double)xcut, hi = leaf == 0 ? (double)xcut : (double)xmax;
    if (!(((double)qx + bestr) > lo && ((double)qx - bestr) < hi)) continue;
    const int s = leaf == 0 ? 0 : cut, e = leaf == 0 ? cut : n;
    for (int j = s; j < e; ++j) {
      const glb_particle_rec &pj = p[order[j]];
      const double r2 = knn_r2(pj.x[0], pj.x[1], pj.x[2], qx, qy, qz);
      if (r2 < bestr * bestr) {
        heap_push_d(heap, hn, r2);
        heap_pop_d(heap, hn);
        bestr = __dsqrt_rn(heap[0]);
      }
    }
  }
  size_out[i] = __double2float_rn(bestr);
}

unsigned nblk(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

size_t smoothing_smem_bytes(size_t n, int nsmooth) {
  const int K = nsmooth + 1;
  const int S = ((2 * nsmooth + 31) / 32) * 32;
  const int nb = (int)std::max<size_t>(1, n / (size_t)S);
  const int mmax = (int)((n + nb - 1) / nb);
  int cap = std::max(mmax + 64, 2 * K + 64);
  cap = (cap + 31) / 32 * 32;
  return (size_t)mmax * (sizeof(float4) + sizeof(double)) + (size_t)kWarps * cap * sizeof(double) +
         (size_t)(2 * kListCap + kWarps * kStack + 2 * kFront) * sizeof(int);
}

Status smooth_particles_device(const glb_particle_rec *d_p, size_t n, int nsmooth, float *d_size,
                               cudaStream_t st, float *ms_out) {
  if (nsmooth < 1) return Status::err(-1, "Nsmooth must be >= 1");
  if (n <= (size_t)nsmooth + 1)
    return Status::err(-1, "number of neighbors >= total number of particles (TreeSimple::NNDistance)");
  if (n >= (size_t)1 << 31) return Status::err(-1, "more than 2^31-1 particles");
  const int K = nsmooth + 1;
  const int S = ((2 * nsmooth + 31) / 32) * 32;
  const int nb = (int)std::max<size_t>(1, n / (size_t)S);
  int P = 1;
  while (P < nb) P <<= 1;
  const int mmax = (int)((n + nb - 1) / nb);
  int cap = std::max(mmax + 64, 2 * K + 64);
  cap = (cap + 31) / 32 * 32;
  const size_t smem = smoothing_smem_bytes(n, nsmooth);
  if (smem > 200 * 1024) return Status::err(-6, "Nsmooth too large for the shared-memory search");
  const bool top_walk = n == 2 * (size_t)nsmooth + 1;
  if (top_walk && (size_t)(K + 1) * sizeof(double) > 48 * 1024)
    return Status::err(-6, "Nsmooth too large for the N = 2*Nsmooth+1 walk");

  // scratch kept between calls (grown on demand), one per device; calls on a
  // device are serialised
  struct Workspace {
    std::mutex mu;
    size_t n = 0;
    int P = 0;
    DBuf<unsigned long long> key, key2;
    DBuf<unsigned> idx, sidx, mm;
    size_t nch = 0;
    DBuf<float4> pos, blo, bhi, clo, chi;
    DBuf<int> flags;
    DBuf<unsigned char> tmp;
  };
  static Workspace *wss = new Workspace[64];
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return Status::err(-1, "device index beyond the 64 devices the library supports");
  Workspace &w = wss[dev];
  std::lock_guard<std::mutex> lock(w.mu);
  if (w.n < n) {
    CK(w.key.alloc(n));
    CK(w.key2.alloc(n));
    CK(w.idx.alloc(n));
    CK(w.sidx.alloc(n));
    CK(w.pos.alloc(n));
    w.n = n;
  }
  const size_t nch = (n + 31) / 32;
  if (w.nch < nch) {
    CK(w.clo.alloc(nch));
    CK(w.chi.alloc(nch));
    w.nch = nch;
  }
  if (w.P < P) {
    CK(w.blo.alloc(2 * (size_t)P));
    CK(w.bhi.alloc(2 * (size_t)P));
    w.P = P;
  }
  if (!w.mm.p) CK(w.mm.alloc(6));
  if (!w.flags.p) CK(w.flags.alloc(1));

  cudaEvent_t ev[3];
  for (auto &e : ev) CK(cudaEventCreate(&e));
  struct EvGuard {
    cudaEvent_t *e;
    ~EvGuard() {
      for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]);
    }
  } evg{ev};
  CK(cudaEventRecord(ev[0], st));

  static const unsigned init[6] = {kFull, kFull, kFull, 0u, 0u, 0u};
  CK(cudaMemcpyAsync(w.mm.p, init, sizeof init, cudaMemcpyHostToDevice, st));
  CK(cudaMemsetAsync(w.flags.p, 0, sizeof(int), st));
  k_bbox3<<<std::min<unsigned>(nblk(n, 256), 148 * 8), 256, 0, st>>>(d_p, n, w.mm.p);
  k_morton3<<<nblk(n, 256), 256, 0, st>>>(d_p, n, w.mm.p, w.key.p, w.idx.p);
  size_t tb = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, tb, w.key.p, w.key2.p, w.idx.p, w.sidx.p, (int)n, 0, 63, st));
  if (w.tmp.n < tb) CK(w.tmp.alloc(tb));
  CK(cub::DeviceRadixSort::SortPairs(w.tmp.p, tb, w.key.p, w.key2.p, w.idx.p, w.sidx.p, (int)n, 0, 63, st));
  k_gather_pos<<<nblk(n, 256), 256, 0, st>>>(d_p, w.sidx.p, n, w.pos.p);
  k_bucket_box<<<nblk((size_t)P * 32, 256), 256, 0, st>>>(w.pos.p, n, nb, P, w.blo.p, w.bhi.p);
  k_chunk_box<<<nblk(nch * 32, 256), 256, 0, st>>>(w.pos.p, n, w.clo.p, w.chi.p);
  for (int l = P / 2; l >= 1; l /= 2) k_box_up<<<nblk(l, 256), 256, 0, st>>>(l, w.blo.p, w.bhi.p);
  CK(cudaEventRecord(ev[1], st));

  KnnArgs a;
  a.pos = w.pos.p;
  a.blo = w.blo.p;
  a.bhi = w.bhi.p;
  a.clo = w.clo.p;
  a.chi = w.chi.p;
  a.n = n;
  a.nb = nb;
  a.P = P;
  a.K = K;
  a.cap = cap;
  a.shrink_at = std::min(cap - 32, 2 * K);
  a.size_out = d_size;
  a.flags = w.flags.p;
  CK(cudaFuncSetAttribute(k_knn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_knn<<<nb, kWarps * 32, smem, st>>>(a);
  if (top_walk) {
    DBuf<int> order;
    CK(order.alloc(n));
    k_rank_x<<<nblk(n, 128), 128, 0, st>>>(d_p, (int)n, order.p);
    k_knn_top_walk<<<(unsigned)n, 32, (size_t)(K + 1) * sizeof(double), st>>>(d_p, (int)n, K, order.p, d_size);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(st));
  }
  CK(cudaEventRecord(ev[2], st));
  CK(cudaGetLastError());
  CK(cudaEventSynchronize(ev[2]));
  if (ms_out) {
    CK(cudaEventElapsedTime(&ms_out[0], ev[0], ev[1]));
    CK(cudaEventElapsedTime(&ms_out[1], ev[1], ev[2]));
  }
  return Status::ok();
}

}  // namespace glb
