/* Stand-in for the absent CosmoLib "halo.h" (oracle build only).  These names
   appear only in field-halo generation and file-reading constructors, which
   the ray-shooting path never calls; they do nothing. */
#pragma once
struct NFW_Utility {
  template <typename A, typename B, typename C, typename D, typename E>
  void match_nfw(A, B, C, D, E) {}
};
struct HALOCalculator {
  template <typename... A> HALOCalculator(A...) {}
  template <typename... A> void reset(A...) {}
  double getRvir() const { return 0; }
  double getR200() const { return 0; }
  double getConcentration(int = 0) const { return 1; }
  static double MosterStellarMassFraction(double) { return 0; }
};
inline double ran2(long *) { return 0.5; }
inline double poidev(float, long *) { return 0; }
