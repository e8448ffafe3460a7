/* Stand-in for an absent third-party header (oracle build only): the NR
   factorial that the reference's shapelet source names (never evaluated by the
   oracle's commands). */
#pragma once
#include <cmath>
inline double factrl(int n) { return std::tgamma(n + 1.0); }
