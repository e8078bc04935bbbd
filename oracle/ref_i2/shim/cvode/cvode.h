/* Stand-in for the CVODE interface the reference's main() calls.  Only
 * declarations: the checker never runs main(); every function is a stub
 * that reports failure (oracle/ref_i2/shim_stubs.cpp).  TEST
 * INFRASTRUCTURE ONLY. */
#ifndef LLG_SHIM_CVODE_H
#define LLG_SHIM_CVODE_H
#include <sundials/sundials_types.h>
#include <sundials/sundials_nvector.h>
#include <sundials/sundials_iterative.h>
#define CV_BDF 2
#define CV_NORMAL 1
#define CV_SUCCESS 0
typedef struct llg_shim_linsol* SUNLinearSolver;
typedef struct llg_shim_nonlinsol* SUNNonlinearSolver;
typedef int (*CVRhsFn)(sunrealtype, N_Vector, N_Vector, void*);
typedef int (*CVLsJacTimesSetupFn)(sunrealtype, N_Vector, N_Vector, void*);
typedef int (*CVLsJacTimesVecFn)(N_Vector, N_Vector, sunrealtype, N_Vector, N_Vector, void*, N_Vector);
typedef int (*CVLsPrecSetupFn)(sunrealtype, N_Vector, N_Vector, sunbooleantype, sunbooleantype*, sunrealtype, void*);
typedef int (*CVLsPrecSolveFn)(sunrealtype, N_Vector, N_Vector, N_Vector, N_Vector, sunrealtype, sunrealtype, int,
                               void*);
#ifdef __cplusplus
extern "C" {
#endif
void* CVodeCreate(int lmm, SUNContext ctx);
int CVodeInit(void* mem, CVRhsFn f, sunrealtype t0, N_Vector y0);
int CVodeSetUserData(void* mem, void* ud);
int CVodeSVtolerances(void* mem, sunrealtype rtol, N_Vector atol);
int CVodeSetNonlinearSolver(void* mem, SUNNonlinearSolver nls);
int CVodeSetLinearSolver(void* mem, SUNLinearSolver ls, void* A);
int CVodeSetJacTimes(void* mem, CVLsJacTimesSetupFn setup, CVLsJacTimesVecFn jtv);
int CVodeSetPreconditioner(void* mem, CVLsPrecSetupFn psetup, CVLsPrecSolveFn psolve);
int CVodeSetMaxOrd(void* mem, int maxord);
int CVode(void* mem, sunrealtype tout, N_Vector yout, sunrealtype* tret, int itask);
int CVodeGetNumSteps(void* mem, long* n);
int CVodeGetNumRhsEvals(void* mem, long* n);
int CVodeGetNumLinSolvSetups(void* mem, long* n);
int CVodeGetNumErrTestFails(void* mem, long* n);
int CVodeGetNumNonlinSolvIters(void* mem, long* n);
int CVodeGetNumNonlinSolvConvFails(void* mem, long* n);
int CVodeGetNumGEvals(void* mem, long* n);
int CVodeGetNumLinIters(void* mem, long* n);
int CVodeGetNumLinConvFails(void* mem, long* n);
int CVodeGetNumJtimesEvals(void* mem, long* n);
void CVodeFree(void** mem);
#ifdef __cplusplus
}
#endif
#endif
