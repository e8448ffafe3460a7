// Split-precision form of the warp-cooperative walk: the same traversal and
// the same per-ray opening decisions as walk_f64 (walk.cuh), with the
// arithmetic moved to FP32 wherever that keeps FP32 relative precision.
//   * Ray-minus-node offsets are formed from double-float pairs (node centre
//     hi + lo, ray hi + lo), so each offset has FP32 relative error however
//     far the cell is from the origin.
//   * Opening tests are taken in FP32 when the FP32 distance is clearly on
//     one side of the threshold (further than 4e-6 relative, ~8x the FP32
//     error bound); otherwise the test is repeated in FP64 on the exact
//     node, so every ray interacts with exactly the cells of the FP64 form.
//   * Far-field and leaf-particle terms are evaluated in FP32; a leaf
//     particle's offset is (particle - leaf centre of mass, stored in FP32 at
//     build time) + (leaf centre of mass - ray).
//   * Particles within two softening lengths of the ray, whose point-mass term
//     is cancelled by a B-spline correction, and the B-spline corrections
//     themselves, are evaluated entirely in FP64.
//   * Sums are compensated by blocking: FP32 partial sums of at most 32 terms
//     are flushed into FP64 totals, which bounds the accumulation error by the
//     per-term rounding instead of letting it grow with the ~1e4 terms of a
//     walk.
#pragma once
#include "walk.cuh"

namespace glb {

struct F32Acc {
  float a0, a1, k, g0, g1;
  int cnt;
  __device__ __forceinline__ void zero() {
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

constexpr float kAmbiguous = 4e-6f;  // relative band around a threshold decided in FP64

// Exact FP64 threshold test for the rare rays in the ambiguity band.
__device__ __noinline__ bool node_test_f64(const GNode *nd, double rx, double ry, int which) {
  const double dx = nd->cx - rx, dy = nd->cy - ry;
  return (dx * dx + dy * dy) < (which ? nd->near2 : nd->open2);
}

// x-width of a node record (GNodeS.width), read only by the plain FP32 form.
__device__ __forceinline__ float c2w(const float4 *sp) { return __ldg(sp + 2).z; }

struct Near64 {
  double a0, a1, k, g0, g1;
};

// A leaf particle within two softening lengths of the ray: the point mass and
// its B-spline correction in FP64, exactly as walk_f64 evaluates them.
__device__ __noinline__ Near64 near_particle_f64(float4 Q, double rx, double ry, double screen2, double inv_area,
                                                  bool nearc, double width) {
  Near64 o;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const double y0 = (double)Q.x - rx, y1 = (double)Q.y - ry;
  double rr = y0 * y0 + y1 * y1;
  const double scr = screen2 != 0.0 ? exp(-rr * screen2) : 1.0;
  if (rr < 1e-20) rr = 1e-20;
  const double m = (double)Q.z, ir2 = 1.0 / rr, prefac = m * scr * ir2 * (1.0 / kPi);
  acc[0] = (inv_area * m - prefac) * y0;
  acc[1] = (inv_area * m - prefac) * y1;
  const double tmp = -2.0 * prefac * ir2;
  acc[3] = 0.5 * (y0 * y0 - y1 * y1) * tmp;
  acc[4] = y0 * y1 * tmp;
  acc[2] = -m * inv_area;
  const double size = (double)Q.w;
  if (nearc && size < width && rr < 4 * size * size) bspline_f64<false>(y0, y1, sqrt(rr), m, size, 0.0, acc);
  o.a0 = acc[0];
  o.a1 = acc[1];
  o.k = acc[2];
  o.g0 = acc[3];
  o.g1 = acc[4];
  return o;
}

// b_spline_profile (include/quadTree.h:147-190) in FP32, for the plain FP32
// form only.
__device__ __forceinline__ void bspline_f32(float x0, float x1, float r, float Mass, float size, float *f) {
  const float ipi = (float)(1.0 / kPi);
  const float q = r / size;
  float M, sigma;
  if (q > 2.f) {
    sigma = 0.f;
    M = 1.f;
  } else {
    const float q2 = q * q, q3 = q2 * q;
    sigma = (8.f - 12.f * q + 6.f * q2 - q3) / 4.f;
    if (q > 1.f) {
      sigma *= 10.f / size / size / 7.f * ipi;
      M = (-1.f + 20.f * q2 * (1.f - q + 3.f * q2 / 8.f - q3 / 20.f)) / 7.f;
    } else {
      sigma = 10.f * (sigma - 1.f + 3.f * q - 3.f * q2 + q3) / size / size / 7.f * ipi;
      M = 10.f * q2 * (1.f - 3.f * q / 4.f + 3.f * q3 / 10.f) / 7.f;
    }
  }
  const float alpha_r = (M - 1.f) * ipi / r;
  const float gt = alpha_r / r - sigma;
  f[0] -= Mass * alpha_r * x0 / r;
  f[1] -= Mass * alpha_r * x1 / r;
  f[3] -= gt * Mass * (x0 * x0 - x1 * x1) / r / r;
  f[4] -= gt * Mass * 2.f * x0 * x1 / r / r;
  f[2] += Mass * sigma;
}

// PURE = true is the plain FP32 form of the precision sweep: FP32 offsets
// from FP32 coordinates, FP32 opening tests and sums throughout, FP32
// near field; it keeps no FP64 arithmetic and so no guarantee of the FP64
// form's interaction set or precision.
template <bool PURE = false>
__device__ __forceinline__ void walk_split(const TreeDev &T, double rx, double ry, bool valid, double *acc) {
  const float inv_pi = (float)(1.0 / kPi);
  const bool screen = T.screen2 != 0.0;
  const float s2f = (float)T.screen2;
  const float iaf = (float)T.inv_area;
  const float rxh = (float)rx, ryh = (float)ry;
  const float rxl = PURE ? 0.f : (float)(rx - (double)rxh), ryl = PURE ? 0.f : (float)(ry - (double)ryh);
  float pf[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // PURE: the FP32 total
  F32Acc fa;
  fa.zero();
  int resume = valid ? 0 : 0x7fffffff;
  int node = 0;
  const int nn = T.nnodes;
  while (node < nn) {
    const float4 *sp = reinterpret_cast<const float4 *>(T.snodes + node);
    const float4 c0 = __ldg(sp), c1 = __ldg(sp + 1);
    const int4 c3 = __ldg(reinterpret_cast<const int4 *>(sp + 3));
    const int skip = max(c3.x, node + 1);  // forward progress even on a malformed array
    const bool act = node >= resume;
    const float dxf = PURE ? (c0.x - rxh) : (c0.x - rxh) + (c0.z - rxl);
    const float dyf = PURE ? (c0.y - ryh) : (c0.y - ryh) + (c0.w - ryl);
    const float r2f = dxf * dxf + dyf * dyf;
    bool open = false;
    if (act) {
      const float d = r2f - c1.x;
      open = d < 0.f;
      if (!PURE && fabsf(d) <= kAmbiguous * c1.x) open = node_test_f64(T.nodes + node, rx, ry, 0);
    }
    if (act && !open) {
      // far field: monopole + quadrupole (quadTree.h:1090-1123)
      const float4 c2 = __ldg(sp + 2);
      const float scr = screen ? __expf(-r2f * s2f) : 1.0f;
      const float ir2 = __fdividef(1.0f, r2f);
      const float ir4 = ir2 * ir2;
      const float mass = c1.z, q0 = c1.w, q1 = c2.x, q2 = c2.y;
      const float ms = mass * inv_pi * scr;
      const float t = mass * iaf - ms * ir2;
      const float qd = (q0 * dxf * dxf + q1 * dyf * dyf + 2.f * q2 * dxf * dyf);
      const float qs = inv_pi * scr * ir4;
      const float t4 = 4.f * qd * qs * ir2;
      fa.a0 += (t + t4) * dxf - (q0 * dxf + q2 * dyf) * qs;
      fa.a1 += (t + t4) * dyf - (q1 * dyf + q2 * dxf) * qs;
      fa.g0 -= ms * ir2 * ((dxf * dxf - dyf * dyf) * ir2);
      fa.g1 -= ms * ir2 * (2.0f * dxf * dyf * ir2);
      fa.k -= iaf * mass;
      if (PURE) {
        pf[0] += fa.a0; pf[1] += fa.a1; pf[2] += fa.k; pf[3] += fa.g0; pf[4] += fa.g1;
        fa.zero();
      } else if (++fa.cnt >= 32) {
        fa.flush(acc);
      }
      resume = skip;
    }
    if (!__any_sync(kFull, open)) {
      node = skip;
      continue;
    }
    bool nearc = false;
    if (open) {
      const float e = r2f - c1.y;
      nearc = e < 0.f;
      if (!PURE && fabsf(e) <= kAmbiguous * c1.y) nearc = node_test_f64(T.nodes + node, rx, ry, 1);
    }
    if (c3.y) {  // leaf
      const int p0 = c3.z, p1 = p0 + c3.w;
      if (open && fa.cnt) fa.flush(acc);
      // particles in chunks of 32 so that the FP32 partial sums stay short
      for (int q0 = p0; q0 < p1; q0 += 32) {
        const int q1 = min(q0 + 32, p1);
        for (int p = q0; p < q1; ++p) {
          const float4 P = __ldg(T.prel + p);
          if (open) {
            const float x0 = P.x + dxf, x1 = P.y + dyf;
            float rcm2f = x0 * x0 + x1 * x1;
            if (PURE) {
              // plain FP32: point mass, then the B-spline if within two sizes
              const float scr = screen ? __expf(-rcm2f * s2f) : 1.0f;
              const float rr = fmaxf(rcm2f, 1e-20f);
              const float m = P.z, ir2 = __fdividef(1.0f, rr), prefac = m * scr * ir2 * inv_pi;
              pf[0] += (iaf * m - prefac) * x0;
              pf[1] += (iaf * m - prefac) * x1;
              pf[3] -= prefac * ir2 * (x0 * x0 - x1 * x1);
              pf[4] -= prefac * ir2 * (2.0f * x0 * x1);
              pf[2] -= m * iaf;
              if (nearc && P.w < c2w(sp) && rr < 4.f * P.w * P.w) bspline_f32(x0, x1, sqrtf(rr), m, P.w, pf);
            } else if (rcm2f < fmaxf(4.0001f * P.w * P.w, 1e-12f)) {  // near or (unsoftened) coincident
              const Near64 o = near_particle_f64(__ldg(T.parts + p), rx, ry, T.screen2, T.inv_area, nearc,
                                                 T.nodes[node].width);
              acc[0] += o.a0;
              acc[1] += o.a1;
              acc[2] += o.k;
              acc[3] += o.g0;
              acc[4] += o.g1;
            } else {
              const float scr = screen ? __expf(-rcm2f * s2f) : 1.0f;
              const float m = P.z;
              const float ir2 = __fdividef(1.0f, rcm2f);
              const float prefac = m * scr * ir2 * inv_pi;
              const float ta = iaf * m - prefac;
              fa.a0 += ta * x0;
              fa.a1 += ta * x1;
              // shear terms scaled by 1/r^2 first so that nothing overflows FP32
              const float pi2 = prefac * ir2;
              fa.g0 -= pi2 * (x0 * x0 - x1 * x1);
              fa.g1 -= pi2 * (2.0f * x0 * x1);
              fa.k -= m * iaf;
            }
          }
        }
        if (open) fa.flush(acc);
      }
      node = skip;
    } else {
      if (__any_sync(kFull, nearc)) {
        const int b0 = c3.z, b1 = b0 + c3.w;
        for (int b = b0; b < b1; ++b) {
          const float4 P = __ldg(T.bigs + b);
          if (PURE && nearc) {
            const float x0 = P.x - rxh, x1 = P.y - ryh;
            const float rr = fmaxf(x0 * x0 + x1 * x1, 1e-20f);
            if (rr < 4.f * P.w * P.w) bspline_f32(x0, x1, sqrtf(rr), P.z, P.w, pf);
          } else if (nearc) {
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
  if (PURE) {
    for (int c = 0; c < 5; ++c) acc[c] += (double)pf[c];
  } else {
    fa.flush(acc);
  }
}

}  // namespace glb
