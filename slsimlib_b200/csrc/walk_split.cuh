// Split-precision form of the warp-cooperative walk (same traversal and the
// same per-ray opening decisions as walk_f64 in walk.cuh):
//   * ray-minus-node-centre offsets and the opening tests stay in FP64, so
//     every ray interacts with exactly the cells and particles of the FP64
//     form;
//   * far-field and leaf-particle terms are evaluated in FP32 from offsets
//     that are exact to FP32 rounding: a leaf particle's offset is
//     (particle - leaf centre of mass, stored in FP32 at build time) +
//     (leaf centre of mass - ray, from FP64);
//   * the sums are compensated by blocking: FP32 partial sums of at most 32
//     terms are flushed into FP64 totals, which bounds the accumulation error
//     by the per-term rounding instead of letting it grow with the ~1e4 terms
//     of a walk;
//   * particles within two softening lengths of the ray, whose point-mass
//     term is cancelled by a B-spline correction, and the B-spline
//     corrections themselves are evaluated entirely in FP64 (the close-range
//     offsets), so no cancellation happens in FP32.
#pragma once
#include "walk.cuh"

namespace glb {

struct F32Acc {
  float a0, a1, k, g0, g1;
  int cnt;
  __device__ inline void zero() {
    a0 = a1 = k = g0 = g1 = 0.f;
    cnt = 0;
  }
  __device__ __forceinline__ void flush(double *acc) {
    acc[0] += (double)a0;
    acc[1] += (double)a1;
    acc[2] += (double)k;
    acc[3] += (double)g0;
    acc[4] += (double)g1;
    zero();
  }
};

__device__ __forceinline__ void walk_split(const TreeDev &T, double rx, double ry, bool valid, double *acc) {
  const float inv_pi = (float)(1.0 / kPi);
  const bool screen = T.screen2 != 0.0;
  const float s2f = (float)T.screen2;
  const float iaf = (float)T.inv_area;
  F32Acc fa;
  fa.zero();
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
    if (act && !open) {
      const GNodeF nf = T.nodesf[node];
      const float dxf = (float)dx, dyf = (float)dy, r2f = (float)r2;
      const float scr = screen ? __expf(-r2f * s2f) : 1.0f;
      const float ir2 = __fdividef(1.0f, r2f);
      const float ir4 = ir2 * ir2;
      const float mass = nf.mass, q0 = nf.q0, q1 = nf.q1, q2 = nf.q2;
      const float ms = mass * inv_pi * scr;
      float t = mass * iaf - ms * ir2;
      const float qd = (q0 * dxf * dxf + q1 * dyf * dyf + 2.f * q2 * dxf * dyf);
      const float qs = inv_pi * scr * ir4;
      const float t4 = 4.f * qd * qs * ir2;
      fa.a0 += (t + t4) * dxf - (q0 * dxf + q2 * dyf) * qs;
      fa.a1 += (t + t4) * dyf - (q1 * dyf + q2 * dxf) * qs;
      t = -2.0f * ms * ir4;
      fa.g0 += 0.5f * (dxf * dxf - dyf * dyf) * t;
      fa.g1 += dxf * dyf * t;
      fa.k -= iaf * mass;
      if (++fa.cnt >= 32) fa.flush(acc);
      resume = skip;
    }
    if (!__any_sync(kFull, open)) {
      node = skip;
      continue;
    }
    const bool nearc = open && (r2 < nd->near2);
    if (nd->leaf) {
      const int p0 = nd->pstart, p1 = p0 + nd->pcount;
      const float dxn = (float)dx, dyn = (float)dy;
      if (open && fa.cnt) fa.flush(acc);
      for (int p = p0; p < p1; ++p) {
        const float4 P = __ldg(T.prel + p);
        if (open) {
          const float x0 = P.x + dxn, x1 = P.y + dyn;
          const float rcm2f = x0 * x0 + x1 * x1;
          if (rcm2f < 4.0001f * P.w * P.w) {
            // within two softening lengths: the point mass and any B-spline
            // correction cancel, so both are done in FP64 exactly as walk_f64
            const float4 Q = __ldg(T.parts + p);
            const double y0 = (double)Q.x - rx, y1 = (double)Q.y - ry;
            double rr = y0 * y0 + y1 * y1;
            const double scr = screen ? exp(-rr * T.screen2) : 1.0;
            if (rr < 1e-20) rr = 1e-20;
            const double m = (double)Q.z, ir2 = 1.0 / rr, prefac = m * scr * ir2 * (1.0 / kPi);
            acc[0] += (T.inv_area * m - prefac) * y0;
            acc[1] += (T.inv_area * m - prefac) * y1;
            const double tmp = -2.0 * prefac * ir2;
            acc[3] += 0.5 * (y0 * y0 - y1 * y1) * tmp;
            acc[4] += y0 * y1 * tmp;
            acc[2] -= m * T.inv_area;
            const double size = (double)Q.w;
            if (nearc && size < nd->width && rr < 4 * size * size)
              bspline_f64<false>(y0, y1, sqrt(rr), m, size, 0.0, acc);
          } else {
            const float scr = screen ? __expf(-rcm2f * s2f) : 1.0f;
            const float m = P.z;
            const float ir2 = __fdividef(1.0f, rcm2f);
            const float prefac = m * scr * ir2 * inv_pi;
            const float ta = iaf * m - prefac;
            fa.a0 += ta * x0;
            fa.a1 += ta * x1;
            // shear terms scaled by 1/r^2 first so that nothing overflows FP32
            fa.g0 -= prefac * ((x0 * x0 - x1 * x1) * ir2);
            fa.g1 -= prefac * (2.0f * x0 * x1 * ir2);
            fa.k -= m * iaf;
          }
        }
        if (((p - p0) & 31) == 31 && open) fa.flush(acc);
      }
      if (open) fa.flush(acc);
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
            if (rcm2 < 4 * size * size) bspline_f64<false>(x0, x1, sqrt(rcm2), (double)P.z, size, 0.0, acc);
          }
        }
      }
      node = node + 1;
    }
  }
  fa.flush(acc);
}

}  // namespace glb
