// shim_stubs.cpp — definitions behind the stand-in SUNDIALS headers.
//
// TEST INFRASTRUCTURE ONLY.  The checker library compiles the reference's
// own 2d_i2 sources (RHS wrapper f, JtvProduct, PrecondSetup/PrecondSolve,
// the cuFFT demag module) so that tests can call them on the same inputs as
// libllg.so.  The vector accessors are real (a handle holds a device
// pointer); everything main() would need to run CVODE is a stub that
// reports failure — the checker never runs main().
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#include <cuda_runtime.h>

#include <cvode/cvode.h>
#include <nvector/nvector_cuda.h>
#include <sunlinsol/sunlinsol_spgmr.h>
#include <sunnonlinsol/sunnonlinsol_newton.h>

extern "C" {

sunrealtype* N_VGetDeviceArrayPointer_Cuda(N_Vector v) { return v ? v->dev : nullptr; }
sunrealtype* N_VGetHostArrayPointer_Cuda(N_Vector v) { return v ? v->host : nullptr; }
N_Vector N_VNew_Cuda(sunindextype, SUNContext) { return nullptr; }
void N_VDestroy(N_Vector) {}
void N_VCopyToDevice_Cuda(N_Vector) {}
void N_VCopyFromDevice_Cuda(N_Vector) {}
int N_VEnableFusedOps_Cuda(N_Vector, int) { return -1; }

int SUNContext_Create(int, SUNContext* ctx) { if (ctx) *ctx = nullptr; return -1; }
int SUNContext_Free(SUNContext*) { return 0; }

void* CVodeCreate(int, SUNContext) { return nullptr; }
int CVodeInit(void*, CVRhsFn, sunrealtype, N_Vector) { return -1; }
int CVodeSetUserData(void*, void*) { return -1; }
int CVodeSVtolerances(void*, sunrealtype, N_Vector) { return -1; }
int CVodeSetNonlinearSolver(void*, SUNNonlinearSolver) { return -1; }
int CVodeSetLinearSolver(void*, SUNLinearSolver, void*) { return -1; }
int CVodeSetJacTimes(void*, CVLsJacTimesSetupFn, CVLsJacTimesVecFn) { return -1; }
int CVodeSetPreconditioner(void*, CVLsPrecSetupFn, CVLsPrecSolveFn) { return -1; }
int CVodeSetMaxOrd(void*, int) { return -1; }
int CVode(void*, sunrealtype, N_Vector, sunrealtype*, int) { return -1; }
int CVodeGetNumSteps(void*, long* n) { *n = 0; return -1; }
int CVodeGetNumRhsEvals(void*, long* n) { *n = 0; return -1; }
int CVodeGetNumLinSolvSetups(void*, long* n) { *n = 0; return -1; }
int CVodeGetNumErrTestFails(void*, long* n) { *n = 0; return -1; }
int CVodeGetNumNonlinSolvIters(void*, long* n) { *n = 0; return -1; }
int CVodeGetNumNonlinSolvConvFails(void*, long* n) { *n = 0; return -1; }
int CVodeGetNumGEvals(void*, long* n) { *n = 0; return -1; }
int CVodeGetNumLinIters(void*, long* n) { *n = 0; return -1; }
int CVodeGetNumLinConvFails(void*, long* n) { *n = 0; return -1; }
int CVodeGetNumJtimesEvals(void*, long* n) { *n = 0; return -1; }
void CVodeFree(void**) {}

SUNLinearSolver SUNLinSol_SPGMR(N_Vector, int, int, SUNContext) { return nullptr; }
int SUNLinSol_SPGMRSetGSType(SUNLinearSolver, int) { return -1; }
int SUNLinSolFree(SUNLinearSolver) { return 0; }
SUNNonlinearSolver SUNNonlinSol_Newton(N_Vector, SUNContext) { return nullptr; }
int SUNNonlinSolFree(SUNNonlinearSolver) { return 0; }

// host dot product of two device vectors (the slot's generic fallback)
sunrealtype N_VDotProd(N_Vector x, N_Vector y) {
  std::vector<double> a((size_t)x->n), b((size_t)y->n);
  cudaMemcpy(a.data(), x->dev, a.size() * sizeof(double), cudaMemcpyDeviceToHost);
  cudaMemcpy(b.data(), y->dev, b.size() * sizeof(double), cudaMemcpyDeviceToHost);
  double s = 0.0;
  for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
  return s;
}

// clone: a new device vector of the same length sharing the operation table
N_Vector llg_shim_nv_clone(N_Vector w) {
  N_Vector v = (N_Vector)calloc(1, sizeof(*v));
  if (!v) return nullptr;
  v->n = w->n;
  v->ops = w->ops;
  if (cudaMalloc(&v->dev, (size_t)w->n * sizeof(double)) != cudaSuccess) { free(v); return nullptr; }
  return v;
}
void llg_shim_nv_free(N_Vector v) {
  if (!v) return;
  cudaFree(v->dev);
  free(v);
}

}  // extern "C"
