// Test-infrastructure stub: the engine header includes "Rcpp.h" but only
// needs the standard containers below when built outside R.
#include <set>
#include <map>
#include <list>
