/* Empty stand-in for an absent third-party header (oracle build only). */
#pragma once
/* Bisection table search over a 1-indexed ascending table xx[1..n]:
   *j is set so that xx[*j] <= x < xx[*j+1]; 0 or n flag x outside the table.
   Used by Lens::ResetSourcePlane. */
inline void locateD(double *xx, unsigned long n, double x, unsigned long *j) {
  unsigned long ju = n + 1, jl = 0, jm;
  while (ju - jl > 1) { jm = (ju + jl) >> 1; if (x >= xx[jm]) jl = jm; else ju = jm; }
  if (x == xx[1]) *j = 1; else if (x == xx[n]) *j = n - 1; else *j = jl;
}
