// ref_i1_jtv.cu — the reference's JtvProduct / jtv_kernel with linear
// anisotropy and DMI, compiled from src/irregular/2d_fft/2d_i1/jtv.cu where it
// lies.  TEST INFRASTRUCTURE ONLY.
#include <string.h>

#include "jtv.cu"

extern "C" int ref_i1_set_jtv_consts(double chk, double che, double alpha, double chg, double cha, double chb) {
  cudaError_t e = cudaMemcpyToSymbol(jc_chk, &chk, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(jc_che, &che, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(jc_alpha, &alpha, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(jc_chg, &chg, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(jc_cha, &cha, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(jc_chb, &chb, sizeof(double));
  return e == cudaSuccess ? 0 : -1;
}

extern "C" int ref_i1_jtv(double* d_v, double* d_Jv, double* d_y, int ng, int ny) {
  JtvUserData ud;
  memset(&ud, 0, sizeof(ud));
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
