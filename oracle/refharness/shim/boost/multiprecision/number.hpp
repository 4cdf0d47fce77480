/* stand-in (TEST INFRASTRUCTURE ONLY) */
#include "cpp_int.hpp"
