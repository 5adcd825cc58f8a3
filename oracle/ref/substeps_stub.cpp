// src/modules/ephemeris_generator.cpp:303-304: record_substeps returns at once unless a
// combined-integrator subsystem is attached, which never happens through the oracle's entry points;
// the generator translation unit itself is not part of the oracle build.
#include "physics/mass.h"

void msystem::record_substeps(fast_real, bool) {}
