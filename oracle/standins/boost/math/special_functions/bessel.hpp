// Test scaffolding for the oracle build only: Boost.Math is absent here; C++17's std::cyl_bessel_j stands in for
// boost::math::cyl_bessel_j, which pairstat/StructureFactor.cpp names (its Mtilde; the oracle does not call it).
#pragma once
#include <cmath>

namespace boost {
namespace math {
using std::cyl_bessel_j;
}
}
