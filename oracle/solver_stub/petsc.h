/* ORACLE build only.  The PETSc types of ../petsc_stub/petsc.h plus the
 * declarations that Apollo's solver headers, its Euler limiter and its grid
 * boundary conditions name.  ref_limiter.cpp defines the DM and Vec calls the
 * limiter makes, over a plain per-element array; nothing else is defined. */
#ifndef APOLLO_ORACLE_SOLVER_STUB_H
#define APOLLO_ORACLE_SOLVER_STUB_H
#include "../petsc_stub/petsc.h"
#include "mpi.h"
typedef struct _p_PetscViewer* PetscViewer;
typedef struct _p_PetscSection* PetscSection;
typedef struct _p_PetscObject* PetscObject;
typedef struct _p_IS* IS;
typedef struct { double fill; } MatFactorInfo;
typedef int PetscMPIInt;
typedef enum { PETSC_FALSE = 0, PETSC_TRUE = 1 } PetscBool;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { MAT_INITIAL_MATRIX = 0, MAT_REUSE_MATRIX = 1, MAT_IGNORE_MATRIX = 2 } MatReuse;
typedef enum { MAT_DO_NOT_COPY_VALUES = 0, MAT_COPY_VALUES = 1, MAT_SHARE_NONZERO_PATTERN = 2 } MatDuplicateOption;
typedef enum { MAT_FACTOR_NONE = 0, MAT_FACTOR_LU = 1 } MatFactorType;
#define PETSC_MAX_PATH_LEN 4096
#define PETSC_NULL 0
#define PETSC_DEFAULT -2
#define PETSC_DECIDE -1
#define PETSC_COMM_SELF MPI_COMM_SELF
#define PETSC_COMM_WORLD MPI_COMM_WORLD
#define PETSC_VIEWER_STDOUT_WORLD ((PetscViewer)0)
#define PETSC_VIEWER_STDOUT_SELF ((PetscViewer)0)
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
/* dense matrices (the node, cubature and connectivity matrices) */
PetscErrorCode MatCreateSeqDense(MPI_Comm, PetscInt, PetscInt, PetscScalar*, Mat*);
PetscErrorCode MatCreateSeqAIJ(MPI_Comm, PetscInt, PetscInt, PetscInt, const PetscInt*, Mat*);
PetscErrorCode MatSetValue(Mat, PetscInt, PetscInt, PetscScalar, InsertMode);
PetscErrorCode MatAssemblyBegin(Mat, MatAssemblyType);
PetscErrorCode MatAssemblyEnd(Mat, MatAssemblyType);
PetscErrorCode MatGetRow(Mat, PetscInt, PetscInt*, const PetscInt**, const PetscScalar**);
PetscErrorCode MatRestoreRow(Mat, PetscInt, PetscInt*, const PetscInt**, const PetscScalar**);
PetscErrorCode MatGetSize(Mat, PetscInt*, PetscInt*);
PetscErrorCode MatDestroy(Mat*);
PetscErrorCode MatView(Mat, PetscViewer);
PetscErrorCode MatZeroEntries(Mat);
PetscErrorCode MatTranspose(Mat, MatReuse, Mat*);
PetscErrorCode MatMatMult(Mat, Mat, MatReuse, PetscReal, Mat*);
PetscErrorCode MatMatTransposeMult(Mat, Mat, MatReuse, PetscReal, Mat*);
PetscErrorCode MatDuplicate(Mat, MatDuplicateOption, Mat*);
PetscErrorCode MatGetFactor(Mat, const char*, MatFactorType, Mat*);
PetscErrorCode MatLUFactorSymbolic(Mat, Mat, IS, IS, const MatFactorInfo*);
PetscErrorCode MatLUFactorNumeric(Mat, Mat, const MatFactorInfo*);
PetscErrorCode MatLUFactor(Mat, IS, IS, const MatFactorInfo*);
PetscErrorCode MatMatSolve(Mat, Mat, Mat);
/* vectors */
PetscErrorCode VecCreateSeq(MPI_Comm, PetscInt, Vec*);
PetscErrorCode VecGetSize(Vec, PetscInt*);
PetscErrorCode VecZeroEntries(Vec);
PetscErrorCode VecDuplicate(Vec, Vec*);
PetscErrorCode VecGetDM(Vec, DM*);
PetscErrorCode VecView(Vec, PetscViewer);
/* the mesh */
PetscErrorCode DMPlexUninterpolate(DM, DM*);
PetscErrorCode DMPlexGetCone(DM, PetscInt, const PetscInt**);
PetscErrorCode DMPlexGetSupport(DM, PetscInt, const PetscInt**);
PetscErrorCode DMPlexGetLabelValue(DM, const char*, PetscInt, PetscInt*);
PetscErrorCode DMPlexGetDepthStratum(DM, PetscInt, PetscInt*, PetscInt*);
PetscErrorCode DMGetCoordinatesLocal(DM, Vec*);
PetscErrorCode DMGetCoordinateSection(DM, PetscSection*);
PetscErrorCode DMGetDefaultSection(DM, PetscSection*);
PetscErrorCode PetscSectionGetOffset(PetscSection, PetscInt, PetscInt*);
PetscErrorCode DMPlexVecGetClosure(DM, PetscSection, Vec, PetscInt, PetscInt*, PetscScalar**);
PetscErrorCode DMPlexVecRestoreClosure(DM, PetscSection, Vec, PetscInt, PetscInt*, PetscScalar**);
PetscErrorCode DMPlexPointGlobalRef(DM, PetscInt, PetscScalar*, void*);
MPI_Comm PetscObjectComm(PetscObject);
PetscErrorCode PetscBarrier(PetscObject);
PetscErrorCode PetscFinalize(void);
#endif
