/* Stand-in: the Newton solver constructor.  TEST INFRASTRUCTURE ONLY. */
#ifndef LLG_SHIM_SUNNONLINSOL_NEWTON_H
#define LLG_SHIM_SUNNONLINSOL_NEWTON_H
#include <cvode/cvode.h>
#ifdef __cplusplus
extern "C" {
#endif
SUNNonlinearSolver SUNNonlinSol_Newton(N_Vector y, SUNContext ctx);
int SUNNonlinSolFree(SUNNonlinearSolver nls);
#ifdef __cplusplus
}
#endif
#endif
