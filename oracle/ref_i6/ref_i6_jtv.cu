// ref_i6_jtv.cu — the reference's compact JtvProduct (jtv_zero_inactive_kernel,
// jtv_kernel_compact), compiled from src/irregular/2d_fft/2d_i6/jtv.cu where
// it lies.  TEST INFRASTRUCTURE ONLY.
#include <string.h>

#include "jtv.cu"

extern "C" int ref_i6_set_jtv_consts(double chk, double che, double alpha, double chg) {
  cudaError_t e = cudaMemcpyToSymbol(jc_chk, &chk, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(jc_che, &che, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(jc_alpha, &alpha, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(jc_chg, &chg, sizeof(double));
  return e == cudaSuccess ? 0 : -1;
}

extern "C" int ref_i6_jtv(double* d_v, double* d_Jv, double* d_y, int* d_active, int n_active, int* d_inactive,
                          int n_inactive, int ng, int ny) {
  JtvUserData ud;
  memset(&ud, 0, sizeof(ud));
  ud.d_active_ids = d_active;
  ud.d_inactive_ids = d_inactive;
  ud.n_active = n_active;
  ud.n_inactive = n_inactive;
  ud.nx = 3 * ng;
  ud.ny = ny;
  ud.ng = ng;
  ud.ncell = ng * ny;
  ud.neq = 3 * ng * ny;
  const long n3 = 3L * ng * ny;
  llg_shim_nvector v = {d_v, nullptr, n3}, jv = {d_Jv, nullptr, n3}, y = {d_y, nullptr, n3};
  const int rc = JtvProduct(&v, &jv, 0.0, &y, nullptr, &ud, nullptr);
  return (cudaDeviceSynchronize() == cudaSuccess) ? rc : -1;
}
