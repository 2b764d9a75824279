/*
 * Sequential stand-in for the subset of PETSc's Mat/Vec/KSP API that the
 * reference CPU flow solver calls (FlowSolver.hpp:491-527 for creation,
 * FlowSolver.inl:1186-1375 and 2106-2273 for assembly and solves).
 * Test infrastructure only; nothing in the product links it.
 *
 * What it defines, and why:
 *  - Mat keeps an explicit sparse row map, so after assembly it holds exactly
 *    the (row, col) pattern the reference inserted.  That pattern is the golden
 *    sparsity the device CSR is compared with.  MatZeroEntries keeps the
 *    pattern and zeroes the values (PETSc AIJ semantics).
 *  - KSPSolve replaces PETSc's Krylov methods with tight, documented solves,
 *    always from the zero initial guess the reference loads (VecZeroEntries(u)):
 *      KSPBCGS   -> unpreconditioned BiCGStab, ||b - A x||_2 <= rtol ||b||_2
 *      KSPFGMRES -> conjugate gradients on the symmetric, singular
 *                   pure-Neumann pressure-correction matrix: the right-hand
 *                   side is projected onto mean zero first and the solution is
 *                   projected onto mean zero at the end, which selects the
 *                   minimum-norm solution independent of the method.
 *    PETSc/AmgX versions are not pinned by the reference, so these semantics
 *    are the definition the oracle uses (the reference has no solver tests).
 *  - Tolerances come from mcshim_set_tolerances(); defaults are 1e-13.
 */
#pragma once

#include <stddef.h>
#include "mpi.h"

typedef int PetscInt;
typedef double PetscScalar;
typedef double PetscReal;
typedef int PetscErrorCode;
typedef int PetscBool;

typedef struct mcshim_Mat *Mat;
typedef struct mcshim_Vec *Vec;
typedef struct mcshim_KSP *KSP;
typedef struct mcshim_PC *PC;

typedef const char *KSPType;
typedef const char *PCType;
typedef int KSPConvergedReason;

typedef enum { INSERT_VALUES = 1, ADD_VALUES = 2 } InsertMode;
typedef enum { MAT_FLUSH_ASSEMBLY = 1, MAT_FINAL_ASSEMBLY = 0 } MatAssemblyType;
typedef enum { MAT_DO_NOT_COPY_VALUES = 0, MAT_COPY_VALUES = 1 } MatDuplicateOption;

#define KSPBCGS "bcgs"
#define KSPFGMRES "fgmres"
#define KSPCG "cg"
#define PCNONE "none"
#define PCGAMG "gamg"
#define PCJACOBI "jacobi"
#define PETSC_DECIDE (-1)

extern MPI_Comm PETSC_COMM_WORLD;

#ifdef __cplusplus
extern "C" {
#endif

PetscErrorCode PetscInitialize(int *argc, char ***argv, const char *file, const char *help);
PetscErrorCode PetscFinalize(void);

PetscErrorCode MatCreate(MPI_Comm comm, Mat *A);
PetscErrorCode MatSetSizes(Mat A, PetscInt m, PetscInt n, PetscInt M, PetscInt N);
PetscErrorCode MatSetFromOptions(Mat A);
PetscErrorCode MatSeqAIJSetPreallocation(Mat A, PetscInt nz, const PetscInt nnz[]);
PetscErrorCode MatMPIAIJSetPreallocation(Mat A, PetscInt d_nz, const PetscInt d_nnz[], PetscInt o_nz, const PetscInt o_nnz[]);
PetscErrorCode MatSetUp(Mat A);
PetscErrorCode MatDuplicate(Mat A, MatDuplicateOption op, Mat *B);
PetscErrorCode MatZeroEntries(Mat A);
PetscErrorCode MatSetValue(Mat A, PetscInt i, PetscInt j, PetscScalar v, InsertMode mode);
PetscErrorCode MatAssemblyBegin(Mat A, MatAssemblyType t);
PetscErrorCode MatAssemblyEnd(Mat A, MatAssemblyType t);
PetscErrorCode MatGetOwnershipRange(Mat A, PetscInt *first, PetscInt *last);
PetscErrorCode MatDestroy(Mat *A);

PetscErrorCode VecCreate(MPI_Comm comm, Vec *v);
PetscErrorCode VecSetSizes(Vec v, PetscInt n, PetscInt N);
PetscErrorCode VecSetFromOptions(Vec v);
PetscErrorCode VecDuplicate(Vec v, Vec *w);
PetscErrorCode VecZeroEntries(Vec v);
PetscErrorCode VecSetValue(Vec v, PetscInt i, PetscScalar x, InsertMode mode);
PetscErrorCode VecAssemblyBegin(Vec v);
PetscErrorCode VecAssemblyEnd(Vec v);
PetscErrorCode VecGetValues(Vec v, PetscInt n, const PetscInt idx[], PetscScalar y[]);
PetscErrorCode VecDestroy(Vec *v);

PetscErrorCode KSPCreate(MPI_Comm comm, KSP *ksp);
PetscErrorCode KSPSetType(KSP ksp, KSPType type);
PetscErrorCode KSPGetPC(KSP ksp, PC *pc);
PetscErrorCode PCSetType(PC pc, PCType type);
PetscErrorCode KSPSetPC(KSP ksp, PC pc);
PetscErrorCode KSPSetOperators(KSP ksp, Mat A, Mat P);
PetscErrorCode KSPSetFromOptions(KSP ksp);
PetscErrorCode KSPSolve(KSP ksp, Vec b, Vec x);
PetscErrorCode KSPGetConvergedReason(KSP ksp, KSPConvergedReason *reason);
PetscErrorCode KSPGetIterationNumber(KSP ksp, PetscInt *its);
PetscErrorCode KSPDestroy(KSP *ksp);

/* Harness controls (not PETSc API). */
void mcshim_set_tolerances(double bcgs_rtol, double cg_rtol, int max_iters);
/* Copy out the assembled CSR of a matrix: row_ptr[n+1], col[nnz], val[nnz]
 * (columns ascending within a row).  Pass NULL arrays to query n and nnz. */
void mcshim_mat_csr(Mat A, PetscInt *n, PetscInt *nnz, PetscInt *row_ptr, PetscInt *col, double *val);
void mcshim_vec_values(Vec v, PetscInt *n, double *out);
/* Statistics of the most recent KSPSolve. */
void mcshim_last_solve(int *iters, double *rel_residual, int *kind);
/* Count of KSPSolve calls per kind (0: BiCGStab, 1: CG) since load. */
void mcshim_solve_counts(long *bcgs, long *cg);

#ifdef __cplusplus
}
#endif
