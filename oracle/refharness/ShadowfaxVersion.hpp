/* Stand-in for the CMake-generated version header of the reference
 * (src/ShadowfaxVersion.hpp.in); used only by the oracle harness build. */
#ifndef SHADOWFAXVERSION_HPP
#define SHADOWFAXVERSION_HPP
#define GIT_BUILD_STRING "oracle-harness"
#define COMPILE_DATE "n/a"
#define COMPILE_TIME "n/a"
#endif
