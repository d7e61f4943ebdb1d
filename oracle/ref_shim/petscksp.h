/*
 * Declarations that let the reference MSPAI sources compile without PETSc.
 * Only the Matrix Market path of the reference is run by the oracle driver;
 * every PETSc routine here is a stub that aborts if it is ever reached.
 * Test infrastructure only.
 */
#ifndef ORACLE_SHIM_PETSCKSP_H
#define ORACLE_SHIM_PETSCKSP_H

#include "mpi.h"

typedef int PetscErrorCode;
typedef int PetscInt;
typedef int PetscMPIInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;

typedef struct _p_Mat* Mat;
typedef struct _p_Vec* Vec;
typedef struct _p_KSP* KSP;
typedef struct _p_PC* PC;
typedef struct _p_PetscOptionItems PetscOptionItems;

typedef struct {
    double nz_used;
    double nz_allocated;
    double nz_unneeded;
} MatInfo;

typedef enum { MAT_LOCAL = 1, MAT_GLOBAL_MAX = 2, MAT_GLOBAL_SUM = 3 } MatInfoType;
typedef enum { MAT_INITIAL_MATRIX = 0, MAT_REUSE_MATRIX = 1, MAT_INPLACE_MATRIX = 2 } MatReuse;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;

#define PETSC_COMM_WORLD 0
#define PETSC_DEFAULT (-2)
#define PETSC_DECIDE (-1)
#define PETSC_NULL 0
#define MATAIJ "aij"
#define MATSEQAIJ "seqaij"
#define MATMPIAIJ "mpiaij"
#define CHKERRQ(e) \
    do {           \
        (void)(e); \
    } while (0)
#define PetscFunctionBegin \
    do {                   \
    } while (0)
#define PetscFunctionReturn(x) return (x)

PetscErrorCode oracle_petsc_unreachable(const char* name);

#define ORACLE_PETSC_STUB(name) \
    template <class... Args>    \
    inline PetscErrorCode name(Args...) { return oracle_petsc_unreachable(#name); }

ORACLE_PETSC_STUB(MatGetRow)
ORACLE_PETSC_STUB(MatRestoreRow)
ORACLE_PETSC_STUB(MatGetInfo)
ORACLE_PETSC_STUB(MatDestroy)
ORACLE_PETSC_STUB(MatGetSize)
ORACLE_PETSC_STUB(MatGetLocalSize)
ORACLE_PETSC_STUB(MatGetOwnershipRange)
ORACLE_PETSC_STUB(MatTranspose)
ORACLE_PETSC_STUB(MatSetType)
ORACLE_PETSC_STUB(MatSetSizes)
ORACLE_PETSC_STUB(MatCreate)
ORACLE_PETSC_STUB(MatSeqAIJSetPreallocation)
ORACLE_PETSC_STUB(MatMPIAIJSetPreallocation)
ORACLE_PETSC_STUB(MatMatMult)
ORACLE_PETSC_STUB(MatEqual)
ORACLE_PETSC_STUB(MatCreateBAIJ)
ORACLE_PETSC_STUB(MatCreateMPIAIJ)
ORACLE_PETSC_STUB(MatAssemblyBegin)
ORACLE_PETSC_STUB(MatAssemblyEnd)
ORACLE_PETSC_STUB(MatSetValues)
ORACLE_PETSC_STUB(MatSetValuesBlocked)
ORACLE_PETSC_STUB(MatSetUp)
ORACLE_PETSC_STUB(MatSetFromOptions)
ORACLE_PETSC_STUB(MatMult)
ORACLE_PETSC_STUB(VecGetArray)
ORACLE_PETSC_STUB(VecRestoreArray)
ORACLE_PETSC_STUB(PetscFree)
ORACLE_PETSC_STUB(PetscMalloc)
ORACLE_PETSC_STUB(PetscMalloc1)
ORACLE_PETSC_STUB(PetscPrintf)

#endif
