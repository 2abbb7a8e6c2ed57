/* Sequential OPS stand-in: no MPI layer (test infrastructure only). */
#ifndef OPS_MPI_CORE_H
#define OPS_MPI_CORE_H
#include "ops_lib_core.h"
#endif
