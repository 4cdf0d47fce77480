/*
 * TimeLine stand-in for the reference harnesses (TEST INFRASTRUCTURE ONLY):
 * one definition per harness program, included by its single translation
 * unit.
 */
#ifndef SFX_REFHARNESS_TIMELINE_STUB_HPP
#define SFX_REFHARNESS_TIMELINE_STUB_HPP

#include "TimeLine.hpp"

/* ------------------------------------------------------------------------ */
/* TimeLine: only the inline getters (src/TimeLine.hpp:145-192) are used by  */
/* VorFace::calculate_flux.  The full TimeLine.cpp drags in snapshot I/O, so */
/* the harness supplies this one constructor.  With _integer_maxtime = 2^60, */
/* _mintime = 0, _tottime = dt and every particle spanning [0, 2^60),        */
/* get_realtime(timestep) == dt exactly and every cell is active.            */
/* ------------------------------------------------------------------------ */
TimeLine::TimeLine(double maxtime, double, double cfl, double,
                   ParticleVector& particlevector, std::string, std::string,
                   UnitSet&, UnitSet&, bool gravity, bool periodic,
                   Cosmology* cosmology, bool treetime, double, double,
                   unsigned int, bool)
        : _particles(particlevector) {
    _maxtime = maxtime;
    _mintime = 0.;
    _tottime = maxtime;
    _integer_maxtime = 1ul << 60;
    _current_time = 0;
    _timestep = 1ul << 60;
    _snaptime = maxtime;
    _snapshotwriter = NULL;
    _cfl = cfl;
    _gravity = gravity;
    _periodic = periodic;
    _cosmology = cosmology;
    _grav_eta = 0.;
    _max_timestep = 0;
    _min_timestep = 0;
    _treetime = treetime;
    _iotimer = NULL;
}

/* TimeLine::set_time(unsigned long) is the other member the harness needs
 * (local time steps start a system step at a given tick); TimeLine.cpp is
 * not linked, so the harness supplies it: the current tick becomes `time`. */
void TimeLine::set_time(unsigned long time) {
    _current_time = time;
}

#endif
