/* Stand-in for an absent third-party header (oracle build only): the two NR
 * helpers and the sign function the reference's image finder uses. */
#pragma once
inline double DMIN(double a, double b) { return a < b ? a : b; }
inline double DMAX(double a, double b) { return a > b ? a : b; }
template <class T>
inline int sgn(T v) { return (T(0) < v) - (v < T(0)); }
/* NR's offset vectors (v[nl..nh]) as the reference's sort routines use them. */
inline unsigned long *lvector(long nl, long nh) { return new unsigned long[nh - nl + 1] - nl; }
inline void free_lvector(unsigned long *v, long nl, long) { delete[] (v + nl); }
