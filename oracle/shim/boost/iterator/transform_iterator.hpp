// Test-infrastructure shim: see boost/cyc_boost_shim.hpp.
#include "../cyc_boost_shim.hpp"
