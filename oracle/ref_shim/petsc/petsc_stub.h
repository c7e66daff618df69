/*
 * TEST INFRASTRUCTURE ONLY -- never linked into the product library.
 *
 * The few PETSc names the reference's fem.cpp / fem.h / mesh.h mention, as
 * inert stand-ins, so that their element-matrix routines (Cfem::set_gpt_*,
 * set_Phi_dPhiS_*, set_amat_bmat) compile from the reference sources
 * without PETSc (absent from the reference tree). Every PETSc call is a
 * no-op returning 0; nothing here takes part in the element arithmetic.
 */
#ifndef CEP_PETSC_STUB_H
#define CEP_PETSC_STUB_H
/* PETSc's own headers bring in the C string, math and I/O declarations */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef double PetscScalar;
typedef int PetscInt;
typedef int PetscErrorCode;
typedef int MPI_Comm;
typedef struct cep_petsc_obj *Mat, *Vec, *KSP, *PC, *VecScatter;
typedef const char *KSPType, *PCType;
enum InsertMode { INSERT_VALUES, ADD_VALUES };
enum ScatterMode { SCATTER_FORWARD };
enum MatAssemblyType { MAT_FINAL_ASSEMBLY };
enum MatStructure { SAME_NONZERO_PATTERN };
#define PETSC_COMM_WORLD 0
#define PETSC_NULL 0
#define PETSC_DECIDE (-1)
#define KSPCG "cg"
#define PCJACOBI "jacobi"

static inline int PetscPrintf(MPI_Comm, const char *, ...) { return 0; }
#define CEP_PETSC_NOOP(name) \
  template <class... A>      \
  static inline int name(A...) { return 0; }
CEP_PETSC_NOOP(MatCreateMPIAIJ)
CEP_PETSC_NOOP(MatGetOwnershipRange)
CEP_PETSC_NOOP(MatSetValues)
CEP_PETSC_NOOP(MatAssemblyBegin)
CEP_PETSC_NOOP(MatAssemblyEnd)
CEP_PETSC_NOOP(MatMult)
CEP_PETSC_NOOP(VecCreate)
CEP_PETSC_NOOP(VecSetSizes)
CEP_PETSC_NOOP(VecSetFromOptions)
CEP_PETSC_NOOP(VecDuplicate)
CEP_PETSC_NOOP(VecSet)
CEP_PETSC_NOOP(VecScale)
CEP_PETSC_NOOP(VecGetArray)
CEP_PETSC_NOOP(VecScatterCreateToAll)
CEP_PETSC_NOOP(VecScatterBegin)
CEP_PETSC_NOOP(VecScatterEnd)
CEP_PETSC_NOOP(KSPCreate)
CEP_PETSC_NOOP(KSPSetOperators)
CEP_PETSC_NOOP(KSPSetType)
CEP_PETSC_NOOP(KSPGetPC)
CEP_PETSC_NOOP(KSPSetFromOptions)
CEP_PETSC_NOOP(KSPSetUp)
CEP_PETSC_NOOP(KSPSolve)
CEP_PETSC_NOOP(KSPGetIterationNumber)
CEP_PETSC_NOOP(PCSetType)
#undef CEP_PETSC_NOOP
#endif
