/* stand-in for the generated header (TEST INFRASTRUCTURE ONLY): the harnesses build no Ewald table */
#ifndef EWALDTABLELOCATION_HPP
#define EWALDTABLELOCATION_HPP
#define EWALDTABLE_LOCATION "ewald_unused.dat"
#endif
