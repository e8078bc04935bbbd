// ref_i6_f.cu — the reference's compact (active-cell) RHS wrapper f, its
// zero_inactive_kernel / f_kernel_compact and the host-side ellipse builder
// BuildEllipticalActiveLists, compiled from
// src/irregular/2d_fft/2d_i6/2d_i6.cu where it lies (the include path points
// at the reference tree; nothing is copied), with C entry points for tests.
//
// TEST INFRASTRUCTURE ONLY.  Built with DEMAG_STRENGTH > 0 so that f takes its
// demag branch whenever a DemagData (Demag_Init of ref_i6_demag.cu) is given.
#define main llg_ref_i6_main_not_run
#include "2d_i6.cu"
#undef main

// the reference's fused-vector layer (deferred_nvector.cu) is not compiled
// here: only main() installs it
extern "C" void FusedNVec_Init(N_Vector) {}
extern "C" void FusedNVec_FreePool(void) {}

extern "C" int ref_i6_set_rhs_consts(const double* msk3, double chk, double che, double alpha, double chg) {
  cudaError_t e = cudaMemcpyToSymbol(c_msk, msk3, 3 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_chk, &chk, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_che, &che, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_alpha, &alpha, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_chg, &chg, sizeof(double));
  return e == cudaSuccess ? 0 : -1;
}

// The ellipse lists (host only).  Returns the counts; the id arrays are
// copied into the caller's buffers of ncell entries each.
extern "C" int ref_i6_ellipse_lists(int ng, int ny, int* active_out, int* n_active, int* inactive_out,
                                    int* n_inactive) {
  int *ha = nullptr, *hi = nullptr;
  BuildEllipticalActiveLists(ng, ny, &ha, &hi, n_active, n_inactive);
  memcpy(active_out, ha, (size_t)*n_active * sizeof(int));
  memcpy(inactive_out, hi, (size_t)*n_inactive * sizeof(int));
  free(ha);
  free(hi);
  return 0;
}

// f(t, y, ydot, user_data) on device arrays; demag may be NULL (field zero)
extern "C" int ref_i6_rhs(double t, double* d_y, double* d_ydot, double* d_hdmag, int* d_active, int n_active,
                          int* d_inactive, int n_inactive, int ng, int ny, void* demag) {
  UserData ud;
  memset(&ud, 0, sizeof(ud));
  ud.demag = (DemagData*)demag;
  ud.d_hdmag = d_hdmag;
  ud.d_active_ids = d_active;
  ud.d_inactive_ids = d_inactive;
  ud.n_active = n_active;
  ud.n_inactive = n_inactive;
  ud.nx = 3 * ng;
  ud.ny = ny;
  ud.ng = ng;
  ud.ncell = ng * ny;
  ud.neq = 3 * ng * ny;
  llg_shim_nvector yv = {d_y, nullptr, 3L * ng * ny}, ydv = {d_ydot, nullptr, 3L * ng * ny};
  const int rc = f(t, &yv, &ydv, &ud);
  return (cudaDeviceSynchronize() == cudaSuccess) ? rc : -1;
}
