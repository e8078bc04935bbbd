// ref_i1_f.cu — the reference's full-grid RHS wrapper f with linear
// anisotropy and interfacial DMI (normalize_m_kernel,
// f_kernel_unified_soa_periodic), compiled from
// src/irregular/2d_fft/2d_i1/2d_fft.cu where it lies (the include path points
// at the reference tree; nothing is copied), with C entry points for tests.
//
// TEST INFRASTRUCTURE ONLY.  Built with DEMAG_STRENGTH > 0 so that f takes its
// demag branch whenever a DemagData (Demag_Init of ref_i1_demag.cu) is given.
#define main llg_ref_i1_main_not_run
#include "2d_fft.cu"
#undef main

// the reference's fused-vector layer (deferred_nvector.cu) is not compiled
// here: only main() installs it
extern "C" void FusedNVec_Init(N_Vector) {}
extern "C" void FusedNVec_FreePool(void) {}

extern "C" int ref_i1_set_rhs_consts(const double* msk3, const double* nsk3, double chk, double che, double alpha,
                                     double chg, double cha, double chb) {
  cudaError_t e = cudaMemcpyToSymbol(c_msk, msk3, 3 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_nsk, nsk3, 3 * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_chk, &chk, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_che, &che, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_alpha, &alpha, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_chg, &chg, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_cha, &cha, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_chb, &chb, sizeof(double));
  return e == cudaSuccess ? 0 : -1;
}

// f(t, y, ydot, user_data) on device arrays; demag may be NULL (field zero)
extern "C" int ref_i1_rhs(double t, double* d_y, double* d_ydot, double* d_hdmag, int ng, int ny, void* demag) {
  UserData ud;
  memset(&ud, 0, sizeof(ud));
  ud.demag = (DemagData*)demag;
  ud.d_hdmag = d_hdmag;
  ud.nx = 3 * ng;
  ud.ny = ny;
  ud.ng = ng;
  ud.ncell = ng * ny;
  ud.neq = 3 * ng * ny;
  llg_shim_nvector yv = {d_y, nullptr, 3L * ng * ny}, ydv = {d_ydot, nullptr, 3L * ng * ny};
  const int rc = f(t, &yv, &ydv, &ud);
  return (cudaDeviceSynchronize() == cudaSuccess) ? rc : -1;
}
