/* Stand-in for the absent NR "utilities.h" (oracle build only).
   Only the templates the ray-shooting sources name are provided.  nintegrate
   feeds tables that are not compared (the NFW potential-integral table and the
   NSIE elliptic-integral table); it is an adaptive Simpson rule. */
#pragma once
#include <cstddef>
#include <cmath>
#include <vector>
#include <functional>
#include <algorithm>
using std::min;
using std::max;
namespace Utilities {
template <typename T>
std::size_t closest(const std::vector<T> &v, T x) {
  std::size_t best = 0;
  for (std::size_t i = 1; i < v.size(); ++i) if (std::fabs(v[i] - x) < std::fabs(v[best] - x)) best = i;
  return best;
}
template <typename T>
void fill_linear(std::vector<T> &v, std::size_t n, T lo, T hi) {
  v.resize(n);
  for (std::size_t i = 0; i < n; ++i) v[i] = n > 1 ? lo + (hi - lo) * i / (n - 1) : lo;
}
template <typename F, typename T = double>
T simpson_step_(F &f, T a, T b, T fa, T fm, T fb, T whole, T eps, int depth) {
  T m = (a + b) / 2, lm = (a + m) / 2, rm = (m + b) / 2;
  T flm = f(lm), frm = f(rm);
  T left = (m - a) / 6 * (fa + 4 * flm + fm), right = (b - m) / 6 * (fm + 4 * frm + fb);
  T delta = left + right - whole;
  if (depth <= 0 || !(std::fabs(delta) > 15 * eps)) return left + right + delta / 15;
  return simpson_step_<F, T>(f, a, m, fa, flm, fm, left, eps / 2, depth - 1) +
         simpson_step_<F, T>(f, m, b, fm, frm, fb, right, eps / 2, depth - 1);
}
/* Adaptive Simpson; tol is relative to a first estimate of the integral.
   A NaN integrand stops the refinement at once instead of exhausting it. */
template <typename F, typename T = double>
T nintegrate(F &f, T a, T b, T tol) {
  T fa = f(a), fb = f(b), fm = f((a + b) / 2);
  T whole = (b - a) / 6 * (fa + 4 * fm + fb);
  T eps = tol * (std::fabs(whole) > 0 ? std::fabs(whole) : T(1e-300));
  return simpson_step_<F, T>(f, a, b, fa, fm, fb, whole, eps, 30);
}
template <typename T, typename R, typename C>
long locate(const std::vector<T> &v, R x, C comp) {
  long lo = 0, hi = (long)v.size();
  while (lo < hi) { long mid = (lo + hi) / 2; if (comp(x, v[mid])) hi = mid; else lo = mid + 1; }
  return lo - 1;
}
template <typename T>
long locate(const std::vector<T> &v, T x) {
  long lo = 0, hi = (long)v.size();
  while (lo < hi) { long mid = (lo + hi) / 2; if (x < v[mid]) hi = mid; else lo = mid + 1; }
  return lo - 1;
}
inline double InterpolateYvec(std::vector<double> &x, std::vector<double> &y, double xx) {
  long i = locate(x, xx);
  if (i < 0) return y.front();
  if (i >= (long)x.size() - 1) return y.back();
  return y[i] + (y[i + 1] - y[i]) * (xx - x[i]) / (x[i + 1] - x[i]);
}
}
