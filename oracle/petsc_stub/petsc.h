/* ORACLE build only: PETSc scalar and handle types, enough for Apollo's equation
 * plugin headers to compile without PETSc.  No PETSc function is declared. */
#ifndef APOLLO_ORACLE_PETSC_STUB_H
#define APOLLO_ORACLE_PETSC_STUB_H
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscInt;
typedef int PetscErrorCode;
typedef struct _p_DM* DM;
typedef struct _p_Vec* Vec;
typedef struct _p_Mat* Mat;
typedef struct _p_TS* TS;
#endif
