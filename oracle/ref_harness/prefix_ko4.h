/* As prefix_ko6.h, but keeps KO_ORD_3 (the reference default, common.h:17):
 * 4th-difference (2-ghost) Kreiss-Oliger branch (nuosc_class.cpp:119-123). */
#include "common.h"
#undef COSENU_MPI
