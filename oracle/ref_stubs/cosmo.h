/* Stand-in for the absent CosmoLib "cosmo.h" (oracle build only).
   Flat LambdaCDM with Omega_r = 0; distances in Mpc (no h factor).
   Only the members used on the ray-shooting path are provided. */
#pragma once
#include <cmath>
#ifndef lightspeed
#define lightspeed 2.99792458e5
#endif
enum class CosmoParamSet { WMAP5yr, Millennium, Planck1yr, Planck, BigMultiDark, Planck18, none };
class COSMOLOGY {
public:
  COSMOLOGY(double om = 0.3, double ol = 0.7, double h = 0.7) : Om(om), Ol(ol), hh(h) {}
  COSMOLOGY(CosmoParamSet) : Om(0.3), Ol(0.7), hh(0.7) {}
  double getOmega_matter() const { return Om; }
  double getOmega_lambda() const { return Ol; }
  double gethubble() const { return hh; }
  double coorDist(double z) const;
  double coorDist(double z1, double z2) const { return coorDist(z2) - coorDist(z1); }
  double angDist(double z) const { return coorDist(z) / (1 + z); }
  double angDist(double z1, double z2) const { return coorDist(z1, z2) / (1 + z2); }
  double radDist(double z) const { return coorDist(z); }
  void PrintCosmology() const {}
  double SigmaCrit(double zl, double zs) const { return 0; }
  double invCoorDist(double d) const;
  /* field-halo mass-function integrals: not on the ray-shooting path */
  template <typename... A> double haloNumberInBufferedCone(A...) const { return 0; }
  template <typename... A> double haloMassInBufferedCone(A...) const { return 0; }
  double radDist(double z1, double z2) const { return coorDist(z1, z2); }
private:
  double Om, Ol, hh;
};
