/* Stand-in: the vector handle type (see nvector/nvector_cuda.h).  TEST
 * INFRASTRUCTURE ONLY. */
#ifndef LLG_SHIM_SUNDIALS_NVECTOR_H
#define LLG_SHIM_SUNDIALS_NVECTOR_H
#include <sundials/sundials_types.h>
/* a device array of n doubles and its host mirror */
struct llg_shim_nvector {
  double* dev;
  double* host;
  long n;
};
typedef struct llg_shim_nvector* N_Vector;
#endif
