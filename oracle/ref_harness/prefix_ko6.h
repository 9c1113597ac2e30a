/* Forced-include prefix for building the reference's CPU path unchanged:
 * pull in its common.h first, then drop the MPI build and the 4th-difference
 * KO switch so calRHS compiles the 6th-difference (3-ghost) Kreiss-Oliger
 * branch (nuosc_class.cpp:112-117).  common.h is #pragma once, so the later
 * includes from the reference sources are no-ops. */
#include "common.h"
#undef COSENU_MPI
#undef KO_ORD_3
