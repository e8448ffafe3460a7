// Flat Lambda-CDM distances for the lens set-up (host) and per-ray source
// planes (device).  The reference takes these from CosmoLib's COSMOLOGY
// (coorDist / angDist, used at MultiPlane/lens.cpp:2397-2515,2659-2680 and
// include/lens_halos.h:137-146); CosmoLib is not part of SLsimLib, so this is
// the project's own flat, radiation-free model:
//   D_C(z) = (c/H0) * int_0^z dz' / sqrt(Om (1+z')^3 + Ok (1+z')^2 + OL)
// evaluated with composite 16-point Gauss-Legendre panels of width <= 0.25 in
// z (the integrand is analytic on [0, z], so the rule is converged to double
// precision).
#pragma once
#include <math.h>

#ifdef __CUDACC__
#define GLB_HD __host__ __device__
#else
#define GLB_HD
#endif

namespace glb {

struct Cosmo {
  double om, ol, h;
};

// 16-point Gauss-Legendre abscissae / weights on [-1, 1] (positive half).
GLB_HD inline double gl16_x(int i) {
  const double x[8] = {0.0950125098376374401853193, 0.2816035507792589132304605,
                       0.4580167776572273863424194, 0.6178762444026437484466718,
                       0.7554044083550030338951012, 0.8656312023878317438804679,
                       0.9445750230732325760779884, 0.9894009349916499325961542};
  return x[i];
}
GLB_HD inline double gl16_w(int i) {
  const double w[8] = {0.1894506104550684962853967, 0.1826034150449235888667637,
                       0.1691565193950025381893121, 0.1495959888165767320815017,
                       0.1246289712555338720524763, 0.0951585116824927848099251,
                       0.0622535239386478928628438, 0.0271524594117540948517806};
  return w[i];
}

GLB_HD inline double inv_E(const Cosmo &c, double z) {
  double a = 1.0 + z;
  return 1.0 / sqrt(c.om * a * a * a + (1.0 - c.om - c.ol) * a * a + c.ol);
}

// Comoving distance to redshift z in Mpc (no h factor).
GLB_HD inline double coordist(const Cosmo &c, double z) {
  if (z <= 0.0) return 0.0;
  int panels = (int)ceil(z / 0.25);
  double w = z / panels, sum = 0.0;
  for (int p = 0; p < panels; ++p) {
    double mid = (p + 0.5) * w, half = 0.5 * w, s = 0.0;
    for (int i = 0; i < 8; ++i) {
      double dx = half * gl16_x(i);
      s += gl16_w(i) * (inv_E(c, mid - dx) + inv_E(c, mid + dx));
    }
    sum += s * half;
  }
  return 2.99792458e5 / (100.0 * c.h) * sum;
}

GLB_HD inline double coordist2(const Cosmo &c, double z1, double z2) {
  return coordist(c, z2) - coordist(c, z1);
}
GLB_HD inline double angdist(const Cosmo &c, double z) { return coordist(c, z) / (1.0 + z); }

// Inverse of coordist by bisection (host set-up only).
inline double invcoordist(const Cosmo &c, double d) {
  double lo = 0.0, hi = 1.0;
  while (coordist(c, hi) < d) hi *= 2.0;
  for (int i = 0; i < 200 && hi - lo > 1e-15 * hi; ++i) {
    double mid = 0.5 * (lo + hi);
    if (coordist(c, mid) < d) lo = mid; else hi = mid;
  }
  return 0.5 * (lo + hi);
}

}  // namespace glb
