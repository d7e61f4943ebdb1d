/* See petscksp.h: PETSc declarations for compiling the reference as an oracle. */
#include "petscksp.h"
