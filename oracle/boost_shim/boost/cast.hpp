// Minimal stand-in for boost::numeric_cast, written for the oracle build.
// tiny_constants.h:130-160 uses it only to convert double constants to the
// working floating-point type, where a plain static_cast has the same result.
#ifndef ORACLE_BOOST_SHIM_CAST_HPP
#define ORACLE_BOOST_SHIM_CAST_HPP
namespace boost {
template <typename Target, typename Source>
inline Target numeric_cast(Source const& s) { return static_cast<Target>(s); }
}
#endif
