// Test scaffolding for the oracle build only: boost::math::tgamma via std::tgamma.
#ifndef ORACLE_STANDIN_BOOST_GAMMA_HPP
#define ORACLE_STANDIN_BOOST_GAMMA_HPP
#include <cmath>
namespace boost { namespace math {
template <class T> T tgamma(T x) { return std::tgamma(x); }
}}  // namespace boost::math
#endif
