// Minimal stand-in for boost::numeric::bounds, written for the oracle build.
// The reference's TINY library (tiny_constants.h:4,139-143) only needs
// highest() and lowest() of the floating-point types it instantiates.
#ifndef ORACLE_BOOST_SHIM_BOUNDS_HPP
#define ORACLE_BOOST_SHIM_BOUNDS_HPP
#include <limits>
namespace boost { namespace numeric {
template <typename T> struct bounds {
  static T highest() { return std::numeric_limits<T>::max(); }
  static T lowest() {
    return std::numeric_limits<T>::is_integer ? std::numeric_limits<T>::min()
                                              : -std::numeric_limits<T>::max();
  }
  static T smallest() {
    return std::numeric_limits<T>::is_integer ? T(0) : std::numeric_limits<T>::denorm_min();
  }
};
} }
#endif
