/* Minimal stand-in for boost/variant.hpp (oracle build only): the reference's
   utilities header names boost::variant in a CSV logger that the ray-shooting
   path never uses.  Values are accepted and discarded. */
#pragma once
#include <ostream>
namespace boost {
template <typename... T> class variant {
public:
  variant() {}
  template <typename U> variant(const U &) {}
  template <typename U> variant &operator=(const U &) { return *this; }
};
template <typename... T> std::ostream &operator<<(std::ostream &os, const variant<T...> &) { return os; }
template <typename R, typename... T> R get(const variant<T...> &) { return R(); }
}
