/* Aborting body of every PETSc stub (see petscksp.h).  Test infrastructure. */
#include "petscksp.h"

#include <cstdio>
#include <cstdlib>

PetscErrorCode oracle_petsc_unreachable(const char* name)
{
    std::fprintf(stderr, "petsc shim: %s reached; the oracle driver runs no PETSc path\n", name);
    std::abort();
}
