// Analytic halo profiles on the device: NFW (table-interpolated, as the
// reference does) and the non-singular isothermal ellipsoid (Kormann et al.
// 1993 closed forms with complex asinh).  All results accumulate (+=) into
// out[0..5] = {alpha0, alpha1, kappa, gamma0, gamma1, phi} exactly like
// LensHalo::force_halo (MultiPlane/lens_halos.cpp:1528-1546).
#pragma once
#include "glb_internal.h"

namespace glb {

// ------------------------------------------------------------- NFW
// LensHaloNFW profile functions, AnalyticNSIE/nfw_lens.cpp:82-132.
__host__ __device__ __forceinline__ double nfw_g(double x) {
  if (x < 1e-5) x = 1e-5;
  double ans = log(x / 2);
  if (x == 1.0) return ans + 1.0;
  if (x > 1.0) return ans + 2 * atan(sqrt((x - 1) / (x + 1))) / sqrt(x * x - 1);
  return ans + 2 * atanh(sqrt((1 - x) / (x + 1))) / sqrt(1 - x * x);
}
__host__ __device__ __forceinline__ double nfw_f(double x) {
  if (x == 0) x = 1e-5;
  if (x == 1.0) return 1.0 / 3.0;
  if (x > 1.0) return (1 - 2 * atan(sqrt((x - 1) / (x + 1))) / sqrt(x * x - 1)) / (x * x - 1);
  return (1 - 2 * atanh(sqrt((1 - x) / (x + 1))) / sqrt(1 - x * x)) / (x * x - 1);
}
__host__ __device__ __forceinline__ double nfw_g2(double x) {
  if (x == 0) x = 1e-5;
  if (x == 1) return 10 / 3. + 4 * log(0.5);
  double y = x * x - 1;
  double ans = 4 * log(x / 2) / x / x - 2 / y;
  if (x < 1.0) return ans + 4 * (2 / x / x + 1 / y) * atanh(sqrt((1 - x) / (x + 1))) / sqrt(-y);
  return ans + 4 * (2 / x / x + 1 / y) * atan(sqrt((x - 1) / (x + 1))) / sqrt(y);
}
__host__ __device__ __forceinline__ double nfw_h(double x) {
  if (x == 0) x = 1e-5;
  if (x <= 1.0) {
    double a = atanh(sqrt(1. - x * x)), l = log(x / 2.);
    return 2. * (l * l - a * a);
  }
  double a = atan(sqrt(x * x - 1.)), l = log(x / 2.);
  return 2. * (l * l + a * a);
}

constexpr int kNfwTable = 10000;     // LensHaloNFW::NTABLE (lens_halos.cpp:352)
constexpr double kNfwMaxRm = 100.0;  // LensHaloNFW::maxrm (lens_halos.cpp:353)

// LensHaloNFW::InterpolateFromTable (lens_halos.cpp:566-580): linear between
// table nodes, the analytic function in bin 0.  which: 0 f, 1 g, 2 g2, 3 h.
__device__ __forceinline__ double nfw_interp(const NFWTables &T, int which, double y) {
  int j = (int)(y / kNfwMaxRm * kNfwTable);
  if (j <= 0) {
    switch (which) {
      case 0: return nfw_f(y);
      case 1: return nfw_g(y);
      case 2: return nfw_g2(y);
      default: return nfw_h(y);
    }
  }
  if (j > kNfwTable - 2) j = kNfwTable - 2;  // beyond the reference's table
  const double *t = which == 0 ? T.f : which == 1 ? T.g : which == 2 ? T.g2 : T.h;
  double x0 = __ldg(T.x + j), x1 = __ldg(T.x + j + 1);
  double t0 = __ldg(t + j), t1 = __ldg(t + j + 1);
  return (t1 - t0) / (x1 - x0) * (y - x0) + t0;
}

// Point mass of the full halo mass beyond Rmax: LensHalo::force_point,
// lens_halos.cpp:1578-1598 (subtract_point = false).
template <bool PHI>
__host__ __device__ __forceinline__ void point_mass(double mass, double x0, double x1, double rcm2, double *out) {
  double prefac = mass / rcm2 / kPi;
  out[0] += -1.0 * prefac * x0;
  out[1] += -1.0 * prefac * x1;
  double tmp = -2.0 * prefac / rcm2;
  out[3] += 0.5 * (x0 * x0 - x1 * x1) * tmp;
  out[4] += x0 * x1 * tmp;
  if (PHI) out[5] += 0.5 * mass * log(rcm2) / kPi;
}

// LensHalo::force_point with subtract_point = true (lens_halos.cpp:1548-1562):
// inside Rmax (rcm2 < Rmax^2 as floats) the point mass scaled by `screening`
// is added (rcm2 == 0: nothing) and the halo's own terms follow; beyond Rmax
// the halo contributes nothing.  Returns whether the own terms follow.
template <bool PHI>
__host__ __device__ __forceinline__ bool subtract_point_terms(double mass, double Rmax2, double x0, double x1,
                                                              double screening, double *out) {
  const double rcm2 = x0 * x0 + x1 * x1;
  if (!(rcm2 < Rmax2)) return false;
  if (rcm2 == 0) return true;
  double fac = screening * mass / rcm2 / kPi;
  out[0] += fac * x0;
  out[1] += fac * x1;
  fac = 2.0 * fac / rcm2;
  out[3] += 0.5 * (x0 * x0 - x1 * x1) * fac;
  out[4] += x0 * x1 * fac;
  if (PHI) out[5] += -0.5 * mass * log(rcm2) / kPi;
  return true;
}

// LensHalo::force_halo -> force_point / force_halo_sym with LensHaloNFW's
// alpha_h, kappa_h, gamma_h, phi_h (include/lens_halos.h:842-856).  SUB: the
// force_halo_sym terms of subtract_point = true (lens_halos.cpp:1620-1640:
// alpha_h + 1, gamma_h + 2 and -log(rcm2)/2 in the potential, after
// subtract_point_terms; nothing beyond Rmax).
template <bool PHI, bool SUB = false>
__device__ __forceinline__ void nfw_force(const NFWDev &d, const NFWTables &T, double x0, double x1,
                                 double *out) {
  double rcm2 = x0 * x0 + x1 * x1;
  if (!(rcm2 < d.Rmax2)) {
    if (!SUB) point_mass<PHI>(d.mass, x0, x1, rcm2, out);
    return;
  }
  if (rcm2 < 1e-20) rcm2 = 1e-20;
  double prefac = d.mass / rcm2 / kPi;
  double x = sqrt(rcm2) / d.rscale;
  double tmp = (-1.0 * nfw_interp(T, 1, x) / d.gmax + (SUB ? 1.0 : 0.0)) * prefac;
  out[0] += tmp * x0;
  out[1] += tmp * x1;
  out[2] += 0.5 * x * x * nfw_interp(T, 0, x) / d.gmax * prefac;
  tmp = (-0.5 * x * x * nfw_interp(T, 2, x) / d.gmax + (SUB ? 2.0 : 0.0)) * prefac / rcm2;
  out[3] += 0.5 * (x0 * x0 - x1 * x1) * tmp;
  out[4] += x0 * x1 * tmp;
  if (PHI) {
    double phih = 0.25 * (nfw_interp(T, 3, x) - d.h_xmax) / d.gmax + d.log_rsize;
    out[5] += phih * d.mass / kPi;
    if (SUB) out[5] -= 0.5 * log(rcm2) * d.mass / kPi;
  }
}

// ------------------------------------------------------------- NSIE
struct cplx {
  double re, im;
};
__host__ __device__ __forceinline__ cplx c_mul(cplx a, cplx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__host__ __device__ __forceinline__ cplx c_scale(cplx a, double s) { return {a.re * s, a.im * s}; }
__host__ __device__ __forceinline__ cplx c_add(cplx a, cplx b) { return {a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx c_sub(cplx a, cplx b) { return {a.re - b.re, a.im - b.im}; }
// real / complex
__host__ __device__ __forceinline__ cplx c_rdiv(double a, cplx b) {
  // scaled to avoid overflow in |b|^2 (Smith's formulation)
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, den = b.re + b.im * r;
    return {a / den, -a * r / den};
  }
  double r = b.re / b.im, den = b.re * r + b.im;
  return {a * r / den, -a / den};
}
// principal square root (branch cut on the negative real axis; the sign of a
// zero imaginary part selects the side, as in C99 csqrt)
__host__ __device__ __forceinline__ cplx c_sqrt(cplx z) {
  if (z.re == 0.0 && z.im == 0.0) return {0.0, z.im};
  double t = sqrt(0.5 * (fabs(z.re) + hypot(z.re, z.im)));
  if (z.re >= 0.0) return {t, z.im / (2.0 * t)};
  return {fabs(z.im) / (2.0 * t), copysign(t, z.im)};
}
// asinh(z) = log(z + sqrt(z^2 + 1)) for Re z >= 0; odd symmetry otherwise.
// For |z| < 0.5 the logarithm is taken as log1p(z + z^2 / (1 + sqrt(z^2+1)))
// so that small arguments keep full relative precision.
__host__ __device__ __forceinline__ cplx c_asinh(cplx z) {
  bool neg = z.re < 0.0 || (z.re == 0.0 && signbit(z.re));
  if (neg) z = {-z.re, -z.im};
  cplx zz = {z.re * z.re - z.im * z.im, 2.0 * z.re * z.im};
  cplx w = {(1.0 - z.im) * (1.0 + z.im) + z.re * z.re, zz.im};
  cplx s = c_sqrt(w);
  cplx r;
  if (z.re * z.re + z.im * z.im < 0.25) {
    cplx onep = {1.0 + s.re, s.im};
    cplx q = c_mul(zz, c_rdiv(1.0, onep));
    cplx v = c_add(z, q);
    r.re = 0.5 * log1p(2.0 * v.re + v.re * v.re + v.im * v.im);
    r.im = atan2(v.im, 1.0 + v.re);
  } else {
    cplx u = c_add(z, s);
    r.re = log(hypot(u.re, u.im));
    r.im = atan2(u.im, u.re);
  }
  if (neg) r = {-r.re, -r.im};
  return r;
}

// alphaNSIE (AnalyticNSIE/nsie.cpp:14-83); rotation angles precomputed.
__host__ __device__ __forceinline__ void alpha_nsie(const NSIEDev &d, double xt0, double xt1, double *alpha) {
  double r = sqrt(xt0 * xt0 + xt1 * xt1);
  if (r < 1.0e-20 || r > 1.0e20) {
    alpha[0] = alpha[1] = 0.0;
    return;
  }
  if (d.f == 1.0) {
    if (d.bc == 0.0) {
      alpha[0] = -1.0 * xt0 / r;
      alpha[1] = -1.0 * xt1 / r;
    } else {
      double t = sqrt(r * r + d.bc * d.bc) - d.bc;
      alpha[0] = -1.0 * t * xt0 / r / r;
      alpha[1] = -1.0 * t * xt1 / r / r;
    }
    return;
  }
  double x0 = xt0 * d.c1 - xt1 * d.s1, x1 = xt1 * d.c1 + xt0 * d.s1;
  double s;
  if (x0 > 0) {
    s = -1;
    x0 *= -1;
  } else
    s = 1;
  double f = d.f, fp = d.fp, bc = d.bc;
  double b2 = x0 * x0 + f * f * x1 * x1;
  cplx cx = {x0, x1};
  cplx tmp = c_mul(c_scale(cx, f * f), cx);
  tmp.re -= fp * fp * bc * bc;
  cplx xi = c_rdiv(fp, c_sqrt(tmp));
  cplx a1 = c_asinh(c_scale(xi, sqrt(b2 + bc * bc)));
  cplx a2 = c_asinh(c_scale(xi, bc));
  cplx ca = c_sub(a1, a2);
  ca = {d.sqrt_f * ca.re / fp, d.sqrt_f * ca.im / fp};
  double al0 = s * ca.re, al1 = -ca.im;
  alpha[0] = al0 * d.c2 - al1 * d.s2;
  alpha[1] = al1 * d.c2 + al0 * d.s2;
}

// kappaNSIE (nsie.cpp:89-106) on already-rotated or raw coordinates.
__host__ __device__ __forceinline__ double kappa_nsie_rot(double f, double bc, double x0, double x1) {
  double b2 = x0 * x0 + f * f * x1 * x1;
  if ((b2 < 1.0e-20) && (bc < 1.0e-20)) return 1.0e10;
  if (b2 > 1.0e20) return 0.0;
  return 0.5 * sqrt(f / (b2 + bc * bc));
}

__host__ __device__ __forceinline__ double kappa_nsie(const NSIEDev &d, double xt0, double xt1) {
  double x0 = xt0 * d.c1 - xt1 * d.s1, x1 = xt1 * d.c1 + xt0 * d.s1;
  return kappa_nsie_rot(d.f, d.bc, x0, x1);
}

// gammaNSIE (nsie.cpp:112-145)
__host__ __device__ __forceinline__ void gamma_nsie(const NSIEDev &d, double xt0, double xt1, double *gam) {
  double r = sqrt(xt0 * xt0 + xt1 * xt1);
  if (r < 1.0e-20 || r > 1.0e20) {
    gam[0] = gam[1] = 0.0;
    return;
  }
  double x0 = xt0 * d.c1 - xt1 * d.s1, x1 = xt1 * d.c1 + xt0 * d.s1;
  double f = d.f, fp = d.fp, bc = d.bc;
  double b2 = x0 * x0 + f * f * x1 * x1;
  double k0 = kappa_nsie_rot(f, bc, x0 * d.c0 - x1 * d.s0, x1 * d.c0 + x0 * d.s0);
  double fr = f * r, fr2 = fr * fr, fb = fp * bc, fb2 = fb * fb;
  double P = d.sqrt_f *
             (k0 * (x0 * x0 + f * f * f * f * x1 * x1) / d.sqrt_f - 0.5 * (1 + f * f) * sqrt(b2 + bc * bc) +
              f * bc) /
             (fr2 * fr2 - 2 * f * f * fp * fp * bc * bc * (x0 * x0 - x1 * x1) + fb2 * fb2);
  double g0 = (f * f * (x0 * x0 - x1 * x1) - fp * fp * bc * bc) * P;
  double g1 = 2 * f * f * x0 * x1 * P;
  gam[0] = g0 * d.c3 - g1 * d.s3;
  gam[1] = g1 * d.c3 + g0 * d.s3;
}

// LensHaloRealNSIE::force_halo, MultiPlane/lens_halos.cpp:1938-2014.
template <bool PHI>
__host__ __device__ __forceinline__ void nsie_force(const NSIEDev &d, double x0, double x1, double *out) {
  double rcm2 = x0 * x0 + x1 * x1;
  if (!(rcm2 < d.Rmax2)) {
    point_mass<PHI>(d.mass, x0, x1, rcm2, out);
    return;
  }
  if (rcm2 < 1e-20) rcm2 = 1e-20;
  if (rcm2 > d.Rsize2) {
    double r = sqrt(rcm2);
    double f1 = (d.Rmax - r) / d.dRmaxRsize, f2 = (r - d.Rsize) / d.dRmaxRsize;
    double ae[2];
    alpha_nsie(d, x0, x1, ae);
    ae[0] *= d.units;
    ae[1] *= d.units;
    double tmp = d.mass / rcm2 / kPi;
    double ai0 = -1.0 * tmp * x0, ai1 = -1.0 * tmp * x1;
    out[0] += ai0 * f2 + ae[0] * f1;
    out[1] += ai1 * f2 + ae[1] * f1;
    tmp = -2.0 * d.mass / rcm2 / kPi / rcm2;
    out[3] += 0.5 * (x0 * x0 - x1 * x1) * tmp;
    out[4] += x0 * x1 * tmp;
  } else {
    double t[2], g[2];
    alpha_nsie(d, x0, x1, t);
    out[0] += d.units * t[0];
    out[1] += d.units * t[1];
    out[2] += d.units * kappa_nsie(d, x0, x1);
    gamma_nsie(d, x0, x1, g);
    out[3] += d.units * g[0];
    out[4] += d.units * g[1];
  }
}

}  // namespace glb
