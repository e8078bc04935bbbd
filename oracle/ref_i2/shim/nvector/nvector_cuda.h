/* Stand-in for the CUDA vector module: the accessors the reference's
 * callbacks use on a vector handle.  TEST INFRASTRUCTURE ONLY. */
#ifndef LLG_SHIM_NVECTOR_CUDA_H
#define LLG_SHIM_NVECTOR_CUDA_H
#include <sundials/sundials_nvector.h>
#ifdef __cplusplus
extern "C" {
#endif
sunrealtype* N_VGetDeviceArrayPointer_Cuda(N_Vector v);
sunrealtype* N_VGetHostArrayPointer_Cuda(N_Vector v);
N_Vector N_VNew_Cuda(sunindextype n, SUNContext ctx);
void N_VDestroy(N_Vector v);
void N_VCopyToDevice_Cuda(N_Vector v);
void N_VCopyFromDevice_Cuda(N_Vector v);
int N_VEnableFusedOps_Cuda(N_Vector v, int on);
#ifdef __cplusplus
}
#endif
#endif
