/* ORACLE build only.  The PETSc types of ../petsc_stub/petsc.h plus the
 * declarations that Apollo's solver headers, its Euler limiter and its grid
 * boundary conditions name.  ref_limiter.cpp defines the DM and Vec calls the
 * limiter makes, over a plain per-element array; nothing else is defined. */
#ifndef APOLLO_ORACLE_SOLVER_STUB_H
#define APOLLO_ORACLE_SOLVER_STUB_H
#include "../petsc_stub/petsc.h"
typedef struct _p_PetscViewer* PetscViewer;
typedef int MPI_Comm;
#define PETSC_MAX_PATH_LEN 4096
typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;
PetscErrorCode DMPlexGetHeightStratum(DM, PetscInt, PetscInt*, PetscInt*);
PetscErrorCode DMPlexGetHybridBounds(DM, PetscInt*, PetscInt*, PetscInt*, PetscInt*);
PetscErrorCode DMPlexPointLocalRead(DM, PetscInt, const PetscScalar*, void*);
PetscErrorCode DMPlexPointLocalRef(DM, PetscInt, PetscScalar*, void*);
PetscErrorCode DMGetLocalVector(DM, Vec*);
PetscErrorCode DMRestoreLocalVector(DM, Vec*);
PetscErrorCode DMGlobalToLocalBegin(DM, Vec, InsertMode, Vec);
PetscErrorCode DMGlobalToLocalEnd(DM, Vec, InsertMode, Vec);
PetscErrorCode DMLocalToGlobalBegin(DM, Vec, InsertMode, Vec);
PetscErrorCode DMLocalToGlobalEnd(DM, Vec, InsertMode, Vec);
PetscErrorCode VecGetArrayRead(Vec, const PetscScalar**);
PetscErrorCode VecRestoreArrayRead(Vec, const PetscScalar**);
PetscErrorCode VecGetArray(Vec, PetscScalar**);
PetscErrorCode VecRestoreArray(Vec, PetscScalar**);
PetscErrorCode VecDestroy(Vec*);
PetscErrorCode DMDestroy(DM*);
typedef enum { NORM_1 = 0, NORM_2 = 1 } NormType;
PetscErrorCode VecNormBegin(Vec, NormType, PetscReal*);
PetscErrorCode VecNormEnd(Vec, NormType, PetscReal*);
int PetscIsInfOrNanReal(PetscReal);
#endif
