// Block-level group walk of the split form.  A block holds 128 neighbouring
// rays (one per thread, Morton order).  One warp classifies tree cells
// against the bounding box of the block's rays, 32 cells at a time, one per
// lane:
//   * accepted by all -- the nearest point of the box is outside the cell's
//     opening radius: every ray takes the cell's far field;
//   * opened by all -- the farthest point of the box is inside: every ray
//     opens it (a leaf's particles for every ray; an internal cell's children
//     are classified in turn);
//   * mixed -- the box straddles the opening radius: each ray walks the cell's
//     subtree with its own decisions, as walk_split does.
// A cell reaches classification only when every ray opened its parent, so a
// ray meets exactly the cells its own walk meets and takes the same decision
// at each: the interaction sets are those of the FP64 form.  The box tests
// are FP64 with a relative margin of 1e-12 (far beyond the rounding of the
// per-ray test), on the monotone distances of the box's nearest and farthest
// points (restated and checked in tests/test_group_bounds.py).  All four
// warps then evaluate the shared lists for their rays without opening tests
// or votes, the cells' rows and the leaves' particles read through per-warp
// shared memory; lists that fill up are evaluated and cleared, and a queue
// that would overflow hands its cells to the per-ray walks.  Each ray's terms are summed as by walk_split (FP32 partial sums of
// at most 32 terms, near leaves on their own), in the order of the lists.
#pragma once
#include "walk_split.cuh"

namespace glb {

constexpr int kGQ = 1024;  // classification queue (power of two)
constexpr int kGF = 2048;  // cells accepted by all
constexpr int kGL = 768;   // leaves opened by all
constexpr int kGB = 128;   // internal cells opened by all that carry big particles
constexpr int kGM = 512;   // mixed subtrees

struct GroupLists {
  int q[kGQ];
  int far[kGF];
  int leaf[kGL];
  int big[kGB];
  int mixed[kGM];
  float4 rows[4][96];  // per warp: the three rows of 32 far cells
  int qhead, qtail, nfar, nleaf, nbig, nmixed, done, any;
  double box[4];  // xmin, xmax, ymin, ymax of the block's valid rays
};

// A far-field term into the FP32 partial sums (far_term without the flush
// check: the caller flushes every 32 terms).  Invalid lanes add garbage that
// their caller never reads back (their totals are dropped).
__device__ __forceinline__ void far_sum(const float4 &c1, const float4 &c2, float2 d, bool screen, float ns2l,
                                        float piaf, F32Acc &fa) {
  const float2 dd = __fmul2_rn(d, d);
  const float r2f = dd.x + dd.y;
  const float scr = screen ? ex2_approx(r2f * ns2l) : 1.0f;
  const float ir2 = rcp_approx(r2f);
  const float ms = c1.z * scr;
  const float sir4 = scr * ir2 * ir2;
  const float qx = fmaf(c2.w, d.x, c2.y * d.y), qy = fmaf(c2.x, d.y, c2.y * d.x);
  const float qd = fmaf(qx, d.x, qy * d.y);
  const float t = fmaf(c1.z, piaf, -ms * ir2) + 4.f * qd * sir4 * ir2;
  fa.a = __ffma2_rn(f2(t), d, fa.a);
  fa.a = __ffma2_rn(f2(-sir4), make_float2(qx, qy), fa.a);
  fa.g = __ffma2_rn(f2(-ms * ir2 * ir2), make_float2(dd.x - dd.y, d.x * d.y), fa.g);
}

// Classification by one warp until the queue is empty (returns true) or a
// list has no room for another round (returns false: evaluate, clear, call
// again).
__device__ __forceinline__ bool group_classify(const TreeDev &T, GroupLists &G) {
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  const double xmin = G.box[0], xmax = G.box[1], ymin = G.box[2], ymax = G.box[3];
  int head = G.qhead, tail = G.qtail;
  int nfar = G.nfar, nleaf = G.nleaf, nbig = G.nbig, nmixed = G.nmixed;
  bool done = false;
  for (;;) {
    if (head == tail) {
      done = true;
      break;
    }
    if (nfar + 32 > kGF || nleaf + 32 > kGL || nbig + 32 > kGB || nmixed + 32 > kGM) break;
    const int cnt = min(32, tail - head);
    int node = -1, cat = 0, skipn = 0, bc = 0, nch = 0;  // cat: 1 accept, 2 open leaf, 3 open internal, 4 mixed
    if (lane < cnt) {
      node = G.q[(head + lane) & (kGQ - 1)];
      const GNode &nd = T.nodes[node];
      const double cx = nd.cx, cy = nd.cy, o2 = nd.open2;
      const double nx = cx < xmin ? xmin - cx : (cx > xmax ? cx - xmax : 0.0);
      const double ny = cy < ymin ? ymin - cy : (cy > ymax ? cy - ymax : 0.0);
      const double fx = fmax(fabs(cx - xmin), fabs(cx - xmax)), fy = fmax(fabs(cy - ymin), fabs(cy - ymax));
      const double dmin2 = nx * nx + ny * ny, dmax2 = fx * fx + fy * fy;
      skipn = nd.skip;
      if (dmin2 >= o2 * (1.0 + 1e-12)) {
        cat = 1;
      } else if (dmax2 < o2 * (1.0 - 1e-12)) {
        cat = nd.leaf ? 2 : 3;
        bc = nd.leaf ? 0 : nd.bcount;
        if (cat == 3)
          for (int c = node + 1; c < skipn; c = T.nodes[c].skip) ++nch;
      } else {
        cat = 4;
      }
    }
    head += cnt;
    // children of the cells every ray opens join the queue; if they would
    // overflow it, those cells go to the per-ray walks instead
    int incl = nch;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    const int total = __shfl_sync(kFull, incl, 31);
    if ((tail - head) + total > kGQ) {
      if (cat == 3) cat = 4;
    } else if (cat == 3) {
      int pos = tail + incl - nch;
      for (int c = node + 1; c < skipn; c = T.nodes[c].skip) G.q[(pos++) & (kGQ - 1)] = c;
    }
    if ((tail - head) + total <= kGQ) tail += total;
    unsigned m = __ballot_sync(kFull, cat == 1);
    if (cat == 1) G.far[nfar + __popc(m & lt)] = node;
    nfar += __popc(m);
    m = __ballot_sync(kFull, cat == 2);
    if (cat == 2) G.leaf[nleaf + __popc(m & lt)] = node;
    nleaf += __popc(m);
    m = __ballot_sync(kFull, cat == 3 && bc > 0);
    if (cat == 3 && bc > 0) G.big[nbig + __popc(m & lt)] = node;
    nbig += __popc(m);
    m = __ballot_sync(kFull, cat == 4);
    if (cat == 4) G.mixed[nmixed + __popc(m & lt)] = node;
    nmixed += __popc(m);
  }
  if (lane == 0) {
    G.qhead = head;
    G.qtail = tail;
    G.nfar = nfar;
    G.nleaf = nleaf;
    G.nbig = nbig;
    G.nmixed = nmixed;
  }
  return done;
}

// One ray's per-ray walk of the subtree [node0, end) (walk_split's loop, the
// split form only), adding into fa / acc.
__device__ __forceinline__ void group_subtree(const TreeDev &T, const double *rxy, bool valid, float2 nrh, float2 nrl,
                                              int node0, int end, bool screen, float s2f, float ns2l, float piaf,
                                              bool sheet, F32Acc &fa, double *acc, float4 *wrow) {
  const int lane = threadIdx.x & 31;
  int resume = valid ? node0 : 0x7fffffff;
  int node = node0;
  while (node < end) {
    const float4 *sp = reinterpret_cast<const float4 *>(T.snodes + node);
    const float4 c0 = __ldg(sp), c1 = __ldg(sp + 1);
    const int4 c3 = __ldg(reinterpret_cast<const int4 *>(sp + 3));
    const int skip = c3.x;
    const bool act = node >= resume;
    const float2 d = __fadd2_rn(__fadd2_rn(make_float2(c0.x, c0.y), nrh), __fadd2_rn(make_float2(c0.z, c0.w), nrl));
    const float2 dd = __fmul2_rn(d, d);
    const float r2f = dd.x + dd.y;
    bool open = false;
    if (act) {
      const float e = r2f - c1.x;
      open = e < 0.f;
      if (fabsf(e) <= c1.w) open = node_test_f64(T.nodes + node, rxy[0], rxy[1], 0);
    }
    if (act && !open) {
      far_term(c1, __ldg(sp + 2), d, r2f, screen, ns2l, piaf, fa, acc);
      resume = skip;
    }
    if (!__any_sync(kFull, open)) {
      node = skip;
      continue;
    }
    bool nearc = false;
    if (open && (c3.y || c3.w > 0)) {
      const float e = r2f - c1.y;
      nearc = e < 0.f;
      if (fabsf(e) <= kAmbiguous * c1.y) nearc = node_test_f64(T.nodes + node, rxy[0], rxy[1], 1);
    }
    if (c3.y) {
      const int p0 = c3.z, p1 = p0 + c3.w;
      const float wu = __ldg(sp + 2).z;
      if (open && (nearc ? fa.cnt > 0 : fa.cnt + min(c3.w, 32) > 32)) fa.flush(acc);
      for (int q0 = p0; q0 < p1; q0 += 32) {
        const int q1 = min(q0 + 32, p1);
        // the whole warp is here (some lane opened the leaf): stage its particles
        if (q0 + lane < q1) wrow[lane] = __ldg(T.prel + q0 + lane);
        __syncwarp();
        for (int p = q0; p < q1; ++p) {
          const float4 P = wrow[p - q0];
          if (open) leaf_term(T, P, p, d, rxy, nearc, screen, s2f, ns2l, piaf, sheet, wu, node, fa, acc);
        }
        if (open) {
          fa.cnt += q1 - q0;
          if (nearc || q1 < p1) fa.flush(acc);
        }
        __syncwarp();
      }
      node = skip;
    } else {
      if (c3.w > 0 && __any_sync(kFull, nearc)) {
        for (int b = c3.z; b < c3.z + c3.w; ++b) {
          const float4 P = __ldg(T.bigs + b);
          if (!nearc) continue;
          const double x0 = (double)P.x - rxy[0], x1 = (double)P.y - rxy[1];
          double rcm2 = x0 * x0 + x1 * x1;
          if (rcm2 < 1e-20) rcm2 = 1e-20;
          const double size = (double)P.w;
          if (rcm2 < 4 * size * size) bspline_f64<false>(x0, x1, sqrt(rcm2), (double)P.z, size, 0.0, acc);
        }
      }
      node = node + 1;
    }
  }
}

// The group walk for the block's rays (all 128 threads call it; rxy: this
// thread's ray position in shared memory; acc: its FP64 totals).
__device__ __forceinline__ void walk_group(const TreeDev &T, const double *rxy, bool valid, double *acc,
                                           GroupLists &G) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool screen = T.screen2 != 0.0;
  const float s2f = (float)T.screen2;
  const float ns2l = -s2f * kLog2e;
  const bool closed = T.sheet_closed;
  const bool sheet = T.inv_area != 0.0 && !closed;
  const float piaf = sheet ? (float)(kPi * T.inv_area) : 0.f;
  const double rx = rxy[0], ry = rxy[1];
  const float rxh = (float)rx, ryh = (float)ry;
  const float2 nrh = make_float2(-rxh, -ryh);
  const float2 nrl = make_float2(-(float)(rx - (double)rxh), -(float)(ry - (double)ryh));
  F32Acc fa;
  fa.zero();
  if (T.nnodes > 0) {
    for (;;) {
      if (warp == 0) {
        const bool d = group_classify(T, G);
        if (lane == 0) G.done = d ? 1 : 0;
      }
      __syncthreads();
      const int nfar = G.nfar, nleaf = G.nleaf, nbig = G.nbig, nmixed = G.nmixed;
      const bool done = G.done != 0;
      // cells every ray accepts: far fields, no tests; blocks of 32 cells
      // between flushes, so the inner loop has no branch and unrolls.  Each
      // lane of a warp first copies one cell's three rows into the warp's
      // shared-memory slots, and the loop reads them from there.
      float4 *wrow = G.rows[warp];
      for (int i0 = 0; i0 < nfar; i0 += 32) {
        const int cnt = min(32, nfar - i0);
        if (lane < cnt) {
          const float4 *sp = reinterpret_cast<const float4 *>(T.snodes + G.far[i0 + lane]);
          wrow[3 * lane] = __ldg(sp);
          wrow[3 * lane + 1] = __ldg(sp + 1);
          wrow[3 * lane + 2] = __ldg(sp + 2);
        }
        __syncwarp();
        if (valid && fa.cnt > 0) fa.flush(acc);
#pragma unroll 8  // 638 ms per light-cone step; 4: 644, 2: 651
        for (int j = 0; j < cnt; ++j) {
          const float4 c0 = wrow[3 * j], c1 = wrow[3 * j + 1], c2 = wrow[3 * j + 2];
          const float2 d =
              __fadd2_rn(__fadd2_rn(make_float2(c0.x, c0.y), nrh), __fadd2_rn(make_float2(c0.z, c0.w), nrl));
          far_sum(c1, c2, d, screen, ns2l, piaf, fa);
        }
        if (valid) fa.flush(acc);
        __syncwarp();
      }
      // leaves every ray opens: each ray's near-field test, then the particles
      for (int i = 0; i < nleaf; ++i) {
        const int node = G.leaf[i];
        const float4 *sp = reinterpret_cast<const float4 *>(T.snodes + node);
        const float4 c0 = __ldg(sp), c1 = __ldg(sp + 1);
        const int4 c3 = __ldg(reinterpret_cast<const int4 *>(sp + 3));
        const float wu = __ldg(sp + 2).z;
        const float2 d = __fadd2_rn(__fadd2_rn(make_float2(c0.x, c0.y), nrh), __fadd2_rn(make_float2(c0.z, c0.w), nrl));
        const float2 dd = __fmul2_rn(d, d);
        const float r2f = dd.x + dd.y;
        bool nearc = false;
        if (valid) {
          const float e = r2f - c1.y;
          nearc = e < 0.f;
          if (fabsf(e) <= kAmbiguous * c1.y) nearc = node_test_f64(T.nodes + node, rx, ry, 1);
        }
        const int p0 = c3.z, p1 = p0 + c3.w;
        if (valid && (nearc ? fa.cnt > 0 : fa.cnt + min(c3.w, 32) > 32)) fa.flush(acc);
        for (int q0 = p0; q0 < p1; q0 += 32) {
          const int q1 = min(q0 + 32, p1);
          // the chunk's particles, one per lane, into the warp's rows
          if (q0 + lane < q1) wrow[lane] = __ldg(T.prel + q0 + lane);
          __syncwarp();
          for (int p = q0; p < q1; ++p) {
            const float4 P = wrow[p - q0];
            if (valid) leaf_term(T, P, p, d, rxy, nearc, screen, s2f, ns2l, piaf, sheet, wu, node, fa, acc);
          }
          if (valid) {
            fa.cnt += q1 - q0;
            if (nearc || q1 < p1) fa.flush(acc);
          }
          __syncwarp();
        }
      }
      // internal cells every ray opens that carry big particles
      for (int i = 0; i < nbig; ++i) {
        const int node = G.big[i];
        const float4 *sp = reinterpret_cast<const float4 *>(T.snodes + node);
        const float4 c0 = __ldg(sp), c1 = __ldg(sp + 1);
        const int4 c3 = __ldg(reinterpret_cast<const int4 *>(sp + 3));
        const float2 d = __fadd2_rn(__fadd2_rn(make_float2(c0.x, c0.y), nrh), __fadd2_rn(make_float2(c0.z, c0.w), nrl));
        const float2 dd = __fmul2_rn(d, d);
        const float r2f = dd.x + dd.y;
        bool nearc = false;
        if (valid) {
          const float e = r2f - c1.y;
          nearc = e < 0.f;
          if (fabsf(e) <= kAmbiguous * c1.y) nearc = node_test_f64(T.nodes + node, rx, ry, 1);
        }
        if (__any_sync(kFull, nearc)) {
          for (int b = c3.z; b < c3.z + c3.w; ++b) {
            const float4 P = __ldg(T.bigs + b);
            if (!nearc) continue;
            const double x0 = (double)P.x - rx, x1 = (double)P.y - ry;
            double rcm2 = x0 * x0 + x1 * x1;
            if (rcm2 < 1e-20) rcm2 = 1e-20;
            const double size = (double)P.w;
            if (rcm2 < 4 * size * size) bspline_f64<false>(x0, x1, sqrt(rcm2), (double)P.z, size, 0.0, acc);
          }
        }
      }
      // subtrees the rays disagree on: per-ray walks
      for (int i = 0; i < nmixed; ++i) {
        const int r = G.mixed[i];
        group_subtree(T, rxy, valid, nrh, nrl, r, T.nodes[r].skip, screen, s2f, ns2l, piaf, sheet, fa, acc, wrow);
      }
      __syncthreads();
      if (threadIdx.x == 0) G.nfar = G.nleaf = G.nbig = G.nmixed = 0;
      __syncthreads();
      if (done) break;
    }
  }
  if (valid) {
    fa.flush(acc);
    if (T.inv_area != 0.0 && T.nnodes > 0) {
      const double s = T.inv_area * T.root_mass;
      acc[2] -= s;
      if (closed) {
        acc[0] += s * (T.root_cx - rx);
        acc[1] += s * (T.root_cy - ry);
      }
    }
  }
}

}  // namespace glb
