// Minimal stand-in for the PETSc calls the device glue uses (PETSc is not installed here): a
// shell Mat with a context and a MATOP_MULT callback, a Vec over a device array (what
// VecCUDAGetArrayRead / VecCUDAGetArrayWrite return for VECCUDA), a shell PC.  Only the
// signatures and the calling convention matter: the glue in cuda_dg_operator.h compiles against
// PETSc's real headers unchanged.
#pragma once

#include <cstdint>

typedef int PetscErrorCode;
typedef int64_t PetscInt;
#define PETSC_SUCCESS 0
#define PETSC_ERR_LIB 76
#define PetscCall(expr)                       \
    do {                                      \
        PetscErrorCode ierr_ = (expr);        \
        if (ierr_ != PETSC_SUCCESS) return ierr_; \
    } while (0)

struct _p_Vec {
    double* array;  // device array of a VECCUDA vector
    PetscInt n;
};
typedef _p_Vec* Vec;

typedef enum { MATOP_MULT = 7 } MatOperation;
struct _p_Mat {
    void* ctx = nullptr;
    PetscErrorCode (*mult)(_p_Mat*, Vec, Vec) = nullptr;
    PetscInt m = 0, bs = 1;
};
typedef _p_Mat* Mat;

struct _p_PC {
    void* ctx = nullptr;
    PetscErrorCode (*apply)(_p_PC*, Vec, Vec) = nullptr;
};
typedef _p_PC* PC;

inline PetscErrorCode VecCUDAGetArrayRead(Vec v, const double** a) { *a = v->array; return PETSC_SUCCESS; }
inline PetscErrorCode VecCUDARestoreArrayRead(Vec, const double** a) { *a = nullptr; return PETSC_SUCCESS; }
inline PetscErrorCode VecCUDAGetArrayWrite(Vec v, double** a) { *a = v->array; return PETSC_SUCCESS; }
inline PetscErrorCode VecCUDARestoreArrayWrite(Vec, double** a) { *a = nullptr; return PETSC_SUCCESS; }
inline PetscErrorCode VecGetLocalSize(Vec v, PetscInt* n) { *n = v->n; return PETSC_SUCCESS; }

inline PetscErrorCode MatCreateShell(PetscInt m, PetscInt bs, void* ctx, Mat* A) {
    *A = new _p_Mat;
    (*A)->ctx = ctx;
    (*A)->m = m;
    (*A)->bs = bs;
    return PETSC_SUCCESS;
}
inline PetscErrorCode MatShellSetOperation(Mat A, MatOperation op, void (*f)(void)) {
    if (op == MATOP_MULT) A->mult = reinterpret_cast<PetscErrorCode (*)(Mat, Vec, Vec)>(f);
    return PETSC_SUCCESS;
}
template <typename T>
inline PetscErrorCode MatShellGetContext(Mat A, T* ctx) {
    *ctx = static_cast<T>(A->ctx);
    return PETSC_SUCCESS;
}
inline PetscErrorCode MatMult(Mat A, Vec x, Vec y) { return A->mult(A, x, y); }
inline PetscErrorCode MatDestroy(Mat* A) {
    delete *A;
    *A = nullptr;
    return PETSC_SUCCESS;
}

inline PetscErrorCode PCCreateShell(void* ctx, PC* pc) {
    *pc = new _p_PC;
    (*pc)->ctx = ctx;
    return PETSC_SUCCESS;
}
inline PetscErrorCode PCShellSetApply(PC pc, PetscErrorCode (*f)(PC, Vec, Vec)) {
    pc->apply = f;
    return PETSC_SUCCESS;
}
template <typename T>
inline PetscErrorCode PCShellGetContext(PC pc, T* ctx) {
    *ctx = static_cast<T>(pc->ctx);
    return PETSC_SUCCESS;
}
inline PetscErrorCode PCApply(PC pc, Vec r, Vec z) { return pc->apply(pc, r, z); }
inline PetscErrorCode PCDestroy(PC* pc) {
    delete *pc;
    *pc = nullptr;
    return PETSC_SUCCESS;
}
