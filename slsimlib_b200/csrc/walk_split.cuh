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
//   * Far-field and leaf-particle terms are evaluated in FP32, x/y pairs with
//     the packed FP32x2 instructions of sm_100 (one issue slot per pair); a
//     leaf particle's offset is (particle - leaf centre of mass, stored in
//     FP32 at build time) + (leaf centre of mass - ray).
//   * A leaf particle within two softening lengths whose B-spline correction
//     the reference applies at the same leaf is evaluated as one softened
//     mass: point mass and correction summed analytically, so the two terms
//     that cancel as r -> 0 never meet in floating point.  Particles whose
//     correction is applied at an ancestor node (softening >= leaf width),
//     (nearly) coincident particles and the ancestors' corrections stay in
//     FP64, exactly as walk_f64 evaluates them.
//   * The inv_area sheet is added once per walk in FP64 where that is exact
//     algebra (its kappa always; its deflection for masses of one sign), not
//     as ~1e4 FP32 terms that cancel near the mass centre.
//   * Sums are compensated by blocking: FP32 partial sums of at most 32 terms
//     are flushed into FP64 totals, which bounds the accumulation error by the
//     per-term rounding instead of letting it grow with the ~1e4 terms of a
//     walk.
// Node and particle records of this form carry mass / pi, quadrupole / pi,
// -mass / pi and the squared near-field radius (GNodeS, TreeDev::prel).
#pragma once
#include "walk.cuh"

namespace glb {

// FP32 partial sums of one walk: alpha and gamma as x/y pairs for the packed
// instructions (g.y holds gamma[1] / 2), kappa, and the number of terms
// since the last flush into the FP64 totals.
struct F32Acc {
  float2 a, g;
  float k;
  int cnt;
  __device__ __forceinline__ void zero() {
    a = make_float2(0.f, 0.f);
    g = make_float2(0.f, 0.f);
    k = 0.f;
    cnt = 0;
  }
  __device__ __forceinline__ void flush(double *acc) {
    acc[0] += (double)a.x;
    acc[1] += (double)a.y;
    acc[2] += (double)k;
    acc[3] += (double)g.x;
    acc[4] += 2.0 * (double)g.y;
    zero();
  }
};

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kInvPiF = (float)(1.0 / kPi);

// PTX approximate base-2 exponential and reciprocal (the MUFU unit).
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }

// Exact FP64 threshold test for the rare rays in the ambiguity band.
__device__ __noinline__ bool node_test_f64(const GNode *nd, double rx, double ry, int which) {
  const double dx = nd->cx - rx, dy = nd->cy - ry;
  return (dx * dx + dy * dy) < (which ? nd->near2 : nd->open2);
}

struct Near64 {
  double a0, a1, k, g0, g1;
};

// A leaf particle evaluated in FP64, exactly as walk_f64 does: the point mass
// and, when the leaf applies it, its B-spline correction.  The inv_area
// sheet's deflection is included with inv_area != 0; its kappa never (the
// caller adds the sheet's kappa in closed form).
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
  const double size = (double)Q.w;
  if (nearc && size < width && rr < 4 * size * size) bspline_f64<false>(y0, y1, sqrt(rr), m, size, 0.0, acc);
  o.a0 = acc[0];
  o.a1 = acc[1];
  o.k = acc[2];
  o.g0 = acc[3];
  o.g1 = acc[4];
  return o;
}

// A softened particle at 0 < r < 2 size: the screened point mass of
// quadTree.h:1017-1046 plus the B-spline correction of b_spline_profile
// (quadTree.h:147-190), summed in closed form.  With q = r/size,
// u = 2 - q and c = 10 / (7 pi size^2), the cubic spline's enclosed-mass
// fraction M and surface density sigma give
//   M / (pi r^2)          = c (1 - 3q/4 + 3q^3/10)             (q <= 1)
//                         = (1 - u^4 (5/2 - u) / 7) / (pi r^2)  (1 < q < 2)
//   sigma                 = c (1 - 3q^2/2 + 3q^3/4)             (q <= 1)
//                         = c u^3 / 4                            (1 < q < 2)
//   M/(pi r^2) - sigma    = c q (-3/4 + 3q/2 - 9q^2/20)          (q <= 1)
// and, with E = exp(-r^2 s2) - 1 (screening of the point mass only),
//   alpha += -m (E/(pi r^2) + M/(pi r^2)) x
//   gamma += -m (E/(pi r^2) + M/(pi r^2) - sigma) (x0^2 - x1^2, 2 x0 x1) / r^2
//   kappa +=  m sigma
// which is algebraically the reference's sum but has no cancellation between
// the point mass and its correction (both ~1/r as r -> 0).
__device__ __forceinline__ void softened_f32(float2 x, float r2, float m, float size, float s2, F32Acc &fa) {
  const float r = sqrtf(r2);
  const float is = __fdividef(1.f, size);
  const float q = r * is;
  const float c = (float)(10.0 / 7.0 / kPi) * is * is;
  float Mr, sg, sh;
  if (q <= 1.f) {
    const float q2 = q * q;
    Mr = c * fmaf(q2 * q, 0.3f, fmaf(q, -0.75f, 1.f));
    sg = c * fmaf(q2 * q, 0.75f, fmaf(q2, -1.5f, 1.f));
    sh = c * q * fmaf(q, fmaf(q, -0.45f, 1.5f), -0.75f);
  } else {
    const float u = 2.f - q, u2 = u * u;
    const float M = fmaf(-u2 * u2, (2.5f - u) * (float)(1.0 / 7.0), 1.f);
    Mr = M * kInvPiF * __fdividef(1.f, r2);
    sg = c * u2 * u * 0.25f;
    sh = Mr - sg;
  }
  const float er = s2 != 0.f ? expm1f(-r2 * s2) * __fdividef(1.f, r2) * kInvPiF : 0.f;
  const float ac = -m * (er + Mr);
  const float gc = -m * (er + sh) * __fdividef(1.f, r2);
  fa.a = __ffma2_rn(f2(ac), x, fa.a);
  fa.g = __ffma2_rn(f2(gc), make_float2(x.x * x.x - x.y * x.y, x.x * x.y), fa.g);
  fa.k = fmaf(m, sg, fa.k);
}

// b_spline_profile (include/quadTree.h:147-190) in FP32, for the plain FP32
// form only.
__device__ __forceinline__ void bspline_f32(float x0, float x1, float r, float Mass, float size, float *f) {
  const float ipi = kInvPiF;
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
// from FP32 coordinates, FP32 opening tests and sums throughout, the
// reference's FP32-evaluated B-spline; it keeps no FP64 arithmetic and so no
// guarantee of the FP64 form's interaction set or precision.
// SKIPNEAR: take the near-field test only where it is read (leaves, internal
// nodes with big particles).  Same results; it pays in the batched kernel
// (+1.1 % on 256 uneven lenses) but makes the one-ray plane step spill far
// more (45M -> 27M rays/s on a 512^2 single plane), so only k_batch sets it.
// MERGE: far leaves join the running partial sums (below); without it every
// opened leaf is summed on its own, flushed before and after (the one-ray
// tree-force kernel: merging made it spill 232 / 420 B against 76 / 192 B and
// run 9 % slower at opening angle 0.3).
template <bool PURE = false, bool SKIPNEAR = false, bool MERGE = true>
__device__ __forceinline__ void walk_split(const TreeDev &T, double rx, double ry, bool valid, double *acc) {
  const bool screen = T.screen2 != 0.0;
  const float s2f = (float)T.screen2;
  const float ns2l = -s2f * kLog2e;          // exp(-r2 s2) = 2^(r2 ns2l)
  // inv_area sheet: in closed form at the end (masses of one sign), else term
  // by term; piaf is the sheet per unit of mass/pi
  const bool closed = !PURE && T.sheet_closed;
  const bool sheet = T.inv_area != 0.0 && !closed;
  const float piaf = sheet ? (float)(kPi * T.inv_area) : 0.f;
  const float rxh = (float)rx, ryh = (float)ry;
  const float rxl = PURE ? 0.f : (float)(rx - (double)rxh), ryl = PURE ? 0.f : (float)(ry - (double)ryh);
  const float2 nrh = make_float2(-rxh, -ryh), nrl = make_float2(-rxl, -ryl);  // negated ray, hi and lo
  float pf[5] = {0.f, 0.f, 0.f, 0.f, 0.f};  // PURE: the FP32 total
  F32Acc fa;
  fa.zero();
  int resume = valid ? 0 : 0x7fffffff;
  int node = 0;
  const int nn = T.nnodes;
  while (node < nn) {
    const float4 *sp = reinterpret_cast<const float4 *>(T.snodes + node);
    const float4 c0 = __ldg(sp), c1 = __ldg(sp + 1);  // centre; open2, near2, mass/pi, open band
    const int4 c3 = __ldg(reinterpret_cast<const int4 *>(sp + 3));  // skip, leaf, start, count
    const int skip = c3.x;  // > node: checked once per tree by the build (k_check_skips)
    const bool act = node >= resume;
    const float2 d = PURE ? __fadd2_rn(make_float2(c0.x, c0.y), nrh)
                          : __fadd2_rn(__fadd2_rn(make_float2(c0.x, c0.y), nrh), __fadd2_rn(make_float2(c0.z, c0.w), nrl));
    const float2 dd = __fmul2_rn(d, d);
    const float r2f = dd.x + dd.y;
    bool open = false;
    if (act) {
      const float e = r2f - c1.x;
      open = e < 0.f;
      if (!PURE && fabsf(e) <= c1.w) open = node_test_f64(T.nodes + node, rx, ry, 0);  // c1.w: the band
    }
    if (act && !open) {
      // far field: monopole + quadrupole (quadTree.h:1090-1123); c1.z = mass/pi,
      // c2.w, c2.x, c2.y = quadrupole/pi
      const float4 c2 = __ldg(sp + 2);
      const float scr = screen ? ex2_approx(r2f * ns2l) : 1.0f;
      const float ir2 = rcp_approx(r2f);
      const float ms = c1.z * scr;                 // mass/pi, screened
      const float sir4 = scr * ir2 * ir2;
      const float qx = fmaf(c2.w, d.x, c2.y * d.y), qy = fmaf(c2.x, d.y, c2.y * d.x);
      const float qd = fmaf(qx, d.x, qy * d.y);    // q0 dx^2 + q1 dy^2 + 2 q2 dx dy
      const float t = fmaf(c1.z, piaf, -ms * ir2) + 4.f * qd * sir4 * ir2;
      float2 a = __ffma2_rn(f2(t), d, PURE ? make_float2(0.f, 0.f) : fa.a);
      a = __ffma2_rn(f2(-sir4), make_float2(qx, qy), a);
      float2 g = __ffma2_rn(f2(-ms * ir2 * ir2), make_float2(dd.x - dd.y, d.x * d.y),
                            PURE ? make_float2(0.f, 0.f) : fa.g);
      if (PURE) {  // (the split form adds the sheet's kappa in closed form)
        pf[0] += a.x; pf[1] += a.y; pf[2] -= piaf * c1.z; pf[3] += g.x; pf[4] += 2.f * g.y;
      } else {
        fa.a = a;
        fa.g = g;
        if (++fa.cnt >= 32) fa.flush(acc);
      }
      resume = skip;
    }
    if (!__any_sync(kFull, open)) {
      node = skip;
      continue;
    }
    bool nearc = false;
    if (open && (!SKIPNEAR || c3.y || c3.w > 0)) {
      const float e = r2f - c1.y;
      nearc = e < 0.f;
      if (!PURE && fabsf(e) <= kAmbiguous * c1.y) nearc = node_test_f64(T.nodes + node, rx, ry, 1);
    }
    if (c3.y) {  // leaf
      const int p0 = c3.z, p1 = p0 + c3.w;
      const float wu = __ldg(sp + 2).z;  // leaf width rounded up to FP32: size < wu <=> size < width
      // Outside the near-field radius (point masses only) a leaf's particles
      // join the running FP32 partial sums when these have room for them (at
      // most 32 terms between flushes), else the sums are flushed first; a
      // near leaf (softened terms, which carry kappa) is summed on its own,
      // flushed before and after, so that its large terms never share a
      // partial sum with other leaves' (merging those too raised the kappa
      // p99.9 of a softened, sheeted tree from under 1e-5 to 1.4e-5).
      // Leaves of more than 32 particles go in chunks of 32.
      if (!PURE && open && ((nearc || !MERGE) ? fa.cnt > 0 : fa.cnt + min(c3.w, 32) > 32)) fa.flush(acc);
      for (int q0 = p0; q0 < p1; q0 += 32) {
        const int q1 = min(q0 + 32, p1);
#pragma unroll 2  // two independent particles in flight (measured: 6.6 % faster at 64 registers)
        for (int p = q0; p < q1; ++p) {
          const float4 P = __ldg(T.prel + p);  // {x - cx, y - cy, -mass/pi, near radius^2}
          if (!open) continue;
          const float2 x = __fadd2_rn(make_float2(P.x, P.y), d);
          const float2 xx = __fmul2_rn(x, x);
          const float r2 = xx.x + xx.y;
          if (PURE) {
            // plain FP32: point mass, then the B-spline if within two sizes
            const float scr = screen ? ex2_approx(r2 * ns2l) : 1.0f;
            const float rr = fmaxf(r2, 1e-20f);
            const float ir2 = __fdividef(1.0f, rr);
            const float npre = P.z * scr * ir2;    // -mass scr / (pi r^2)
            const float ta = npre - piaf * P.z;
            pf[0] += ta * x.x;
            pf[1] += ta * x.y;
            pf[3] += npre * ir2 * (xx.x - xx.y);
            pf[4] += npre * ir2 * (2.0f * x.x * x.y);
            pf[2] += piaf * P.z;
            if (nearc && rr < P.w) {
              const float4 Q = __ldg(T.parts + p);
              if (Q.w < wu && rr < 4.f * Q.w * Q.w) bspline_f32(x.x, x.y, sqrtf(rr), Q.z, Q.w, pf);
            }
            continue;
          }
          bool point = true;
          if (r2 < P.w) {  // within two softening lengths (or coincident)
            const float4 Q = __ldg(T.parts + p);
            if (r2 < 1e-12f || !(Q.w < wu)) {
              const Near64 o = near_particle_f64(Q, rx, ry, T.screen2, sheet ? T.inv_area : 0.0, nearc,
                                                 T.nodes[node].width);
              acc[0] += o.a0;
              acc[1] += o.a1;
              acc[2] += o.k;
              acc[3] += o.g0;
              acc[4] += o.g1;
              point = false;
            } else if (nearc && r2 < 4.f * Q.w * Q.w) {
              softened_f32(x, r2, Q.z, Q.w, s2f, fa);
              if (sheet) fa.a = __ffma2_rn(f2(-piaf * P.z), x, fa.a);
              point = false;
            }
          }
          if (point) {
            const float scr = screen ? ex2_approx(r2 * ns2l) : 1.0f;
            const float ir2 = rcp_approx(r2);
            const float npre = P.z * scr * ir2;  // -mass scr / (pi r^2)
            fa.a = __ffma2_rn(f2(npre), x, fa.a);
            fa.g = __ffma2_rn(f2(npre * ir2), make_float2(xx.x - xx.y, x.x * x.y), fa.g);
            if (sheet) fa.a = __ffma2_rn(f2(-piaf * P.z), x, fa.a);  // inv_area * mass * x
          }
        }
        if (!PURE && open) {
          fa.cnt += q1 - q0;
          if (nearc || !MERGE || q1 < p1) fa.flush(acc);
        }
      }
      node = skip;
    } else {
      if ((!SKIPNEAR || c3.w > 0) && __any_sync(kFull, nearc)) {
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
    // the sheet's kappa is -inv_area x (total mass) for every walk (each
    // particle's mass enters exactly once, in a cell or as a leaf particle);
    // its deflection is closed-form for masses of one sign
    if (T.inv_area != 0.0 && nn > 0) {
      const double s = T.inv_area * T.root_mass;
      acc[2] -= s;
      if (closed) {
        acc[0] += s * (T.root_cx - rx);
        acc[1] += s * (T.root_cy - ry);
      }
    }
  }
}

// One far-field term (monopole + quadrupole, quadTree.h:1090-1123) into the
// FP32 partial sums, flushed every 32 terms.
__device__ __forceinline__ void far_term(const float4 &c1, const float4 &c2, float2 d, float r2f, bool screen,
                                         float ns2l, float piaf, F32Acc &fa, double *acc) {
  const float scr = screen ? ex2_approx(r2f * ns2l) : 1.0f;
  const float ir2 = rcp_approx(r2f);
  const float ms = c1.z * scr;
  const float sir4 = scr * ir2 * ir2;
  const float qx = fmaf(c2.w, d.x, c2.y * d.y), qy = fmaf(c2.x, d.y, c2.y * d.x);
  const float qd = fmaf(qx, d.x, qy * d.y);
  const float t = fmaf(c1.z, piaf, -ms * ir2) + 4.f * qd * sir4 * ir2;
  fa.a = __ffma2_rn(f2(t), d, fa.a);
  fa.a = __ffma2_rn(f2(-sir4), make_float2(qx, qy), fa.a);
  const float2 dd = __fmul2_rn(d, d);
  fa.g = __ffma2_rn(f2(-ms * ir2 * ir2), make_float2(dd.x - dd.y, d.x * d.y), fa.g);
  if (++fa.cnt >= 32) fa.flush(acc);
}

// One leaf particle for one ray (the split forms of quadTree.h:1017-1077):
// FP64 where the particle (nearly) coincides with the ray or its correction
// belongs to an ancestor, the closed-form softened mass within two softening
// lengths of a near leaf, else the point mass.
__device__ __forceinline__ void leaf_term(const TreeDev &T, float4 P, int p, float2 d, const double *rxy, bool nearc,
                                          bool screen, float s2f, float ns2l, float piaf, bool sheet, float wu,
                                          int node, F32Acc &fa, double *acc) {
  const float2 x = __fadd2_rn(make_float2(P.x, P.y), d);
  const float2 xx = __fmul2_rn(x, x);
  const float r2 = xx.x + xx.y;
  if (r2 < P.w) {  // within two softening lengths (or coincident)
    const float4 Q = __ldg(T.parts + p);
    if (r2 < 1e-12f || !(Q.w < wu)) {
      const Near64 o = near_particle_f64(Q, rxy[0], rxy[1], T.screen2, sheet ? T.inv_area : 0.0, nearc,
                                         T.nodes[node].width);
      acc[0] += o.a0;
      acc[1] += o.a1;
      acc[2] += o.k;
      acc[3] += o.g0;
      acc[4] += o.g1;
      return;
    }
    if (nearc && r2 < 4.f * Q.w * Q.w) {
      softened_f32(x, r2, Q.z, Q.w, s2f, fa);
      if (sheet) fa.a = __ffma2_rn(f2(-piaf * P.z), x, fa.a);
      return;
    }
  }
  const float scr = screen ? ex2_approx(r2 * ns2l) : 1.0f;
  const float ir2 = rcp_approx(r2);
  const float npre = P.z * scr * ir2;
  fa.a = __ffma2_rn(f2(npre), x, fa.a);
  fa.g = __ffma2_rn(f2(npre * ir2), make_float2(xx.x - xx.y, x.x * x.y), fa.g);
  if (sheet) fa.a = __ffma2_rn(f2(-piaf * P.z), x, fa.a);
}

// The split walk for two rays per lane (a warp walks 64 neighbouring rays):
// each ray keeps its own opening decisions, partial sums and resume point as
// walk_split<false> does for one, while the node rows, the warp vote, the
// loop control and the leaf particles are loaded and executed once for both.
// Each ray forms its own double-float offsets, so its terms, decisions and
// FP64 totals are walk_split<false, false, false>'s: a leaf opened by a ray is
// summed on its own, flushed before and after, and the results are
// bit-identical to the one-ray walk's.  rxy: {rx0, ry0, rx1, ry1} (the rays'
// FP64 positions); acc0 / acc1: the rays' FP64 totals.
__device__ __forceinline__ void walk_split2(const TreeDev &T, const double *rxy, bool valid0, bool valid1,
                                            double *acc0, double *acc1) {
  const bool screen = T.screen2 != 0.0;
  const float s2f = (float)T.screen2;
  const float ns2l = -s2f * kLog2e;
  const bool closed = T.sheet_closed;
  const bool sheet = T.inv_area != 0.0 && !closed;
  const float piaf = sheet ? (float)(kPi * T.inv_area) : 0.f;
  float2 nrh[2], nrl[2];  // negated rays, hi and lo
  for (int r = 0; r < 2; ++r) {
    const double rx = rxy[2 * r], ry = rxy[2 * r + 1];
    const float rxh = (float)rx, ryh = (float)ry;
    nrh[r] = make_float2(-rxh, -ryh);
    nrl[r] = make_float2(-(float)(rx - (double)rxh), -(float)(ry - (double)ryh));
  }
  F32Acc fa0, fa1;
  fa0.zero();
  fa1.zero();
  int resume0 = valid0 ? 0 : 0x7fffffff, resume1 = valid1 ? 0 : 0x7fffffff;
  int node = 0;
  const int nn = T.nnodes;
  while (node < nn) {
    const float4 *sp = reinterpret_cast<const float4 *>(T.snodes + node);
    const float4 c0 = __ldg(sp), c1 = __ldg(sp + 1);
    const int4 c3 = __ldg(reinterpret_cast<const int4 *>(sp + 3));
    const int skip = c3.x;
    const bool act0 = node >= resume0, act1 = node >= resume1;
    const float2 cc = make_float2(c0.x, c0.y), cl = make_float2(c0.z, c0.w);
    const float2 d0 = __fadd2_rn(__fadd2_rn(cc, nrh[0]), __fadd2_rn(cl, nrl[0]));
    const float2 d1 = __fadd2_rn(__fadd2_rn(cc, nrh[1]), __fadd2_rn(cl, nrl[1]));
    const float2 dd0 = __fmul2_rn(d0, d0), dd1 = __fmul2_rn(d1, d1);
    const float r2f0 = dd0.x + dd0.y, r2f1 = dd1.x + dd1.y;
    bool open0 = false, open1 = false;
    if (act0) {
      const float e = r2f0 - c1.x;
      open0 = e < 0.f;
      if (fabsf(e) <= c1.w) open0 = node_test_f64(T.nodes + node, rxy[0], rxy[1], 0);
    }
    if (act1) {
      const float e = r2f1 - c1.x;
      open1 = e < 0.f;
      if (fabsf(e) <= c1.w) open1 = node_test_f64(T.nodes + node, rxy[2], rxy[3], 0);
    }
    const bool far0 = act0 && !open0, far1 = act1 && !open1;
    if (far0 || far1) {
      const float4 c2 = __ldg(sp + 2);
      if (far0) {
        far_term(c1, c2, d0, r2f0, screen, ns2l, piaf, fa0, acc0);
        resume0 = skip;
      }
      if (far1) {
        far_term(c1, c2, d1, r2f1, screen, ns2l, piaf, fa1, acc1);
        resume1 = skip;
      }
    }
    if (!__any_sync(kFull, open0 || open1)) {
      node = skip;
      continue;
    }
    bool nearc0 = false, nearc1 = false;
    // the near-field test matters at a leaf and at an internal node with big
    // particles (c3.w of them) only; skipping it elsewhere measured 1.3 %
    // faster on the light-cone plane step when this walk served it
    const bool need_near = c3.y || c3.w > 0;
    if (open0 && need_near) {
      const float e = r2f0 - c1.y;
      nearc0 = e < 0.f;
      if (fabsf(e) <= kAmbiguous * c1.y) nearc0 = node_test_f64(T.nodes + node, rxy[0], rxy[1], 1);
    }
    if (open1 && need_near) {
      const float e = r2f1 - c1.y;
      nearc1 = e < 0.f;
      if (fabsf(e) <= kAmbiguous * c1.y) nearc1 = node_test_f64(T.nodes + node, rxy[2], rxy[3], 1);
    }
    if (c3.y) {  // leaf
      const int p0 = c3.z, p1 = p0 + c3.w;
      const float wu = __ldg(sp + 2).z;
      if (open0 && fa0.cnt) fa0.flush(acc0);
      if (open1 && fa1.cnt) fa1.flush(acc1);
      for (int q0 = p0; q0 < p1; q0 += 32) {
        const int q1 = min(q0 + 32, p1);
        for (int p = q0; p < q1; ++p) {
          const float4 P = __ldg(T.prel + p);
          if (open0) leaf_term(T, P, p, d0, rxy, nearc0, screen, s2f, ns2l, piaf, sheet, wu, node, fa0, acc0);
          if (open1) leaf_term(T, P, p, d1, rxy + 2, nearc1, screen, s2f, ns2l, piaf, sheet, wu, node, fa1, acc1);
        }
        if (open0) fa0.flush(acc0);
        if (open1) fa1.flush(acc1);
      }
      node = skip;
    } else {
      if (c3.w > 0 && __any_sync(kFull, nearc0 || nearc1)) {
        const int b0 = c3.z, b1 = b0 + c3.w;
        for (int b = b0; b < b1; ++b) {
          const float4 P = __ldg(T.bigs + b);
          for (int r = 0; r < 2; ++r) {
            if (!(r ? nearc1 : nearc0)) continue;
            const double x0 = (double)P.x - rxy[2 * r], x1 = (double)P.y - rxy[2 * r + 1];
            double rcm2 = x0 * x0 + x1 * x1;
            if (rcm2 < 1e-20) rcm2 = 1e-20;
            const double size = (double)P.w;
            if (rcm2 < 4 * size * size) bspline_f64<false>(x0, x1, sqrt(rcm2), (double)P.z, size, 0.0, r ? acc1 : acc0);
          }
        }
      }
      node = node + 1;
    }
  }
  fa0.flush(acc0);
  fa1.flush(acc1);
  if (T.inv_area != 0.0 && nn > 0) {
    const double s = T.inv_area * T.root_mass;
    for (int r = 0; r < 2; ++r) {
      double *acc = r ? acc1 : acc0;
      acc[2] -= s;
      if (closed) {
        acc[0] += s * (T.root_cx - rxy[2 * r]);
        acc[1] += s * (T.root_cy - rxy[2 * r + 1]);
      }
    }
  }
}

}  // namespace glb
