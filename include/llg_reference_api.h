/*
 * llg_reference_api.h — the reference's own module entry points, exported by
 * libllg.so with the reference's names and argument meaning, so a caller
 * written against the reference links unchanged.
 *
 *   Demag_Init            src/irregular/2d_fft/2d_i2/demag_fft.h:29
 *   Demag_Apply           src/irregular/2d_fft/2d_i2/demag_fft.h:33
 *   Demag_Destroy         src/irregular/2d_fft/2d_i2/demag_fft.h:35
 *   Demag_GetSelfCoupling src/irregular/2d_fft/2d_i2/demag_fft.h:39-42
 *   Demag_ApplyWindowed   src/irregular/2d_fft/2d_i3/demag_fft.h:36-40
 *   Demag_SetStream       src/irregular/2d_fft/2d_i3/demag_fft.h:43
 *   Precond_Create        src/irregular/2d_fft/2d_i2/precond.h:28
 *   Precond_Destroy       src/irregular/2d_fft/2d_i2/precond.h:29
 *
 * Demag_Init(nx, ny, …) takes the cell grid (the reference passes ng) and
 * uses periodic, un-padded boundaries like the reference; Demag_InitOpen is
 * the zero-padded (open-boundary) twin with no reference counterpart.
 *
 * The SUNDIALS-signature callbacks (f, JtvProduct, PrecondSetup,
 * PrecondSolve; 2d_i2/2d_fft.cu:366, jtv.h:26-27, precond.h:31-38) and the
 * N_Vector multi-dot installer are compiled into libllg.so only when the
 * SUNDIALS headers are present at build time (LLG_HAVE_SUNDIALS); their
 * user_data argument is an llg_ctx*.
 */
#ifndef LLG_REFERENCE_API_H
#define LLG_REFERENCE_API_H

#include "llg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct DemagData DemagData;
typedef struct PrecondData PrecondData;
struct CUstream_st; /* cudaStream_t */

DemagData* Demag_Init(int nx, int ny, double thick, double demag_strength);
DemagData* Demag_InitOpen(int nx, int ny, double thick, double demag_strength);
void Demag_Apply(DemagData* d, const double* y_dev, double* h_out_dev);
void Demag_ApplyWindowed(DemagData* d, const double* y_dev, const double* w_dev, double* h_out_dev);
void Demag_SetStream(DemagData* d, struct CUstream_st* stream);
void Demag_GetSelfCoupling(DemagData* d, double* nxx0_scaled, double* nyy0_scaled, double* nzz0_scaled);
void Demag_Destroy(DemagData* d);

PrecondData* Precond_Create(int ng, int ny, int ncell);
void Precond_Destroy(PrecondData* pd);

#ifdef LLG_HAVE_SUNDIALS
#include <cvode/cvode.h>
#include <nvector/nvector_cuda.h>
int f(sunrealtype t, N_Vector y, N_Vector ydot, void* user_data);
int JtvProduct(N_Vector v, N_Vector Jv, sunrealtype t, N_Vector y, N_Vector fy, void* user_data, N_Vector tmp);
int PrecondSetup(sunrealtype t, N_Vector y, N_Vector fy, sunbooleantype jok, sunbooleantype* jcurPtr,
                 sunrealtype gamma, void* user_data);
int PrecondSolve(sunrealtype t, N_Vector y, N_Vector fy, N_Vector r, N_Vector z, sunrealtype gamma,
                 sunrealtype delta, int lr, void* user_data);
void FusedNVec_InitCtx(N_Vector v, llg_ctx* ctx);
void FusedNVec_FreePool(void);
#endif

#ifdef __cplusplus
}
#endif
#endif
