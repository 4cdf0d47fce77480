/* stand-in: everything ExArith.cpp uses is in cpp_int.hpp (TEST INFRASTRUCTURE ONLY) */
#include "../cpp_int.hpp"
