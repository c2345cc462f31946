// Build shim (TEST INFRASTRUCTURE): libstdc++ does not declare std::floorl /
// std::ceill / std::powl, which lib/src/static/modulus_switching.cpp and
// lib/src/operators/lwe_conversion.cpp use.
#include <cmath>
namespace std { using ::floorl; using ::ceill; using ::powl; }
