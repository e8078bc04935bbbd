// sundials_adapter.cpp — SUNDIALS-signature callbacks over libllg.so.
//
// These are the four callbacks CVODE's linear-solver interface calls in the
// reference (src/irregular/2d_fft/2d_i2/2d_fft.cu:366, 2d_i2/jtv.h:26-27,
// 2d_i2/precond.h:31-38) plus the nvdotprodmulti slot installer
// (2d_i2/deferred_nvector.cu:146-235).  user_data is an llg_ctx* (the one
// change a caller makes: it replaces the byte-mirrored UserData struct).
// They are compiled only where the SUNDIALS headers exist, so a reference
// main() can link against libllg.so; this build environment has no SUNDIALS,
// and the translation unit is then empty.
#if defined(__has_include)
#if __has_include(<cvode/cvode.h>) && __has_include(<nvector/nvector_cuda.h>)
#define LLG_HAVE_SUNDIALS 1
#endif
#endif

#ifdef LLG_HAVE_SUNDIALS
#include <cvode/cvode.h>
#include <nvector/nvector_cuda.h>
#include <sundials/sundials_nvector.h>

#include "../../include/llg.h"

extern "C" {

int f(sunrealtype t, N_Vector y, N_Vector ydot, void* user_data) {
  return llg_rhs((llg_ctx*)user_data, t, N_VGetDeviceArrayPointer_Cuda(y), N_VGetDeviceArrayPointer_Cuda(ydot));
}

int JtvProduct(N_Vector v, N_Vector Jv, sunrealtype t, N_Vector y, N_Vector fy, void* user_data, N_Vector tmp) {
  (void)tmp;
  return llg_jtv((llg_ctx*)user_data, N_VGetDeviceArrayPointer_Cuda(v), N_VGetDeviceArrayPointer_Cuda(Jv), t,
                 N_VGetDeviceArrayPointer_Cuda(y), N_VGetDeviceArrayPointer_Cuda(fy));
}

int PrecondSetup(sunrealtype t, N_Vector y, N_Vector fy, sunbooleantype jok, sunbooleantype* jcurPtr,
                 sunrealtype gamma, void* user_data) {
  int jcur = 0;
  const int rc = llg_psetup((llg_ctx*)user_data, t, N_VGetDeviceArrayPointer_Cuda(y),
                            N_VGetDeviceArrayPointer_Cuda(fy), jok, &jcur, gamma);
  *jcurPtr = jcur ? SUNTRUE : SUNFALSE;
  return rc;
}

int PrecondSolve(sunrealtype t, N_Vector y, N_Vector fy, N_Vector r, N_Vector z, sunrealtype gamma,
                 sunrealtype delta, int lr, void* user_data) {
  return llg_psolve((llg_ctx*)user_data, t, N_VGetDeviceArrayPointer_Cuda(y), N_VGetDeviceArrayPointer_Cuda(fy),
                    N_VGetDeviceArrayPointer_Cuda(r), N_VGetDeviceArrayPointer_Cuda(z), gamma, delta, lr);
}

static llg_ctx* g_dot_ctx = nullptr;
static N_Vector (*g_clone)(N_Vector) = nullptr;

static SUNErrCode llg_nv_dotprodmulti(int nvec, N_Vector x, N_Vector* Y, sunrealtype* out) {
  if (nvec > 16 || !g_dot_ctx) {
    for (int j = 0; j < nvec; j++) out[j] = N_VDotProd(x, Y[j]);
    return SUN_SUCCESS;
  }
  const double* ys[16];
  for (int j = 0; j < nvec; j++) ys[j] = N_VGetDeviceArrayPointer_Cuda(Y[j]);
  return llg_dot_multi(g_dot_ctx, nvec, N_VGetDeviceArrayPointer_Cuda(x), ys, out) == 0 ? SUN_SUCCESS : -1;
}

static N_Vector llg_nv_clone(N_Vector w) {
  N_Vector v = g_clone(w);
  if (!v) return nullptr;
  N_VEnableFusedOps_Cuda(v, 1);
  v->ops->nvdotprodmulti = llg_nv_dotprodmulti;
  v->ops->nvclone = llg_nv_clone;
  return v;
}

// FusedNVec_Init(v) of the reference with the context that owns the stream.
void FusedNVec_InitCtx(N_Vector v, llg_ctx* ctx) {
  if (!v) return;
  g_dot_ctx = ctx;
  if (!g_clone) g_clone = v->ops->nvclone;
  N_VEnableFusedOps_Cuda(v, 1);
  v->ops->nvdotprodmulti = llg_nv_dotprodmulti;
  v->ops->nvclone = llg_nv_clone;
}

void FusedNVec_FreePool(void) { g_dot_ctx = nullptr; }

}  // extern "C"
#endif
