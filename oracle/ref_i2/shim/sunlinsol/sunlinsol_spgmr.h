/* Stand-in: the SPGMR constructor the reference's main() calls.  TEST
 * INFRASTRUCTURE ONLY. */
#ifndef LLG_SHIM_SUNLINSOL_SPGMR_H
#define LLG_SHIM_SUNLINSOL_SPGMR_H
#include <cvode/cvode.h>
#ifdef __cplusplus
extern "C" {
#endif
SUNLinearSolver SUNLinSol_SPGMR(N_Vector y, int pretype, int maxl, SUNContext ctx);
int SUNLinSol_SPGMRSetGSType(SUNLinearSolver ls, int gstype);
int SUNLinSolFree(SUNLinearSolver ls);
#ifdef __cplusplus
}
#endif
#endif
