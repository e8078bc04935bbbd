/* Stand-in: the vector handle type and the two operation slots the
 * reference's fused-vector layer replaces (nvclone, nvdotprodmulti).  TEST
 * INFRASTRUCTURE ONLY. */
#ifndef LLG_SHIM_SUNDIALS_NVECTOR_H
#define LLG_SHIM_SUNDIALS_NVECTOR_H
#include <sundials/sundials_types.h>
#define SUN_SUCCESS 0
struct llg_shim_nvector;
typedef struct llg_shim_nvector* N_Vector;
struct llg_shim_nvector_ops {
  N_Vector (*nvclone)(N_Vector);
  SUNErrCode (*nvdotprodmulti)(int, N_Vector, N_Vector*, sunrealtype*);
};
typedef struct llg_shim_nvector_ops* N_Vector_Ops;
/* a device array of n doubles, its host mirror and its operation table */
struct llg_shim_nvector {
  double* dev;
  double* host;
  long n;
  N_Vector_Ops ops;
};
#ifdef __cplusplus
extern "C" {
#endif
sunrealtype N_VDotProd(N_Vector x, N_Vector y);
#ifdef __cplusplus
}
#endif
#endif
