// Build shim (TEST INFRASTRUCTURE): the reference includes this path for hexl::NTT.
#include "../hexl.hpp"
