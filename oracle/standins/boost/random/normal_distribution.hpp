// Test scaffolding for the oracle build only: forwards to the stand-in boost/random.hpp.
#include "../random.hpp"
