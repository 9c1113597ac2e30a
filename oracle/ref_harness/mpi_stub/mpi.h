/* Empty stand-in for <mpi.h>.  The reference's common.h includes <mpi.h>
 * unconditionally under its own #define COSENU_MPI; the prefix headers in
 * this directory #undef COSENU_MPI right after, so no MPI symbol is used. */
