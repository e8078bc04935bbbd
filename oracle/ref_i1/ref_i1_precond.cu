// ref_i1_precond.cu — the reference's block-Jacobi PrecondSetup /
// PrecondSolve with linear anisotropy and DMI (build_J_kernel,
// apply_P_kernel), compiled from src/irregular/2d_fft/2d_i1/precond.cu where
// it lies.  TEST INFRASTRUCTURE ONLY.
#include <string.h>

#include "precond.cu"

extern "C" int ref_i1_set_precond_consts(double chk, double che, double alpha, double chg, double cha, double chb) {
  cudaError_t e = cudaMemcpyToSymbol(pc_chk, &chk, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(pc_che, &che, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(pc_alpha, &alpha, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(pc_chg, &chg, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(pc_cha, &cha, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(pc_chb, &chb, sizeof(double));
  return e == cudaSuccess ? 0 : -1;
}

static PcUserData ref_ud(void* pd, double* d_hdmag, int ng, int ny, const double* n0) {
  PcUserData ud;
  memset(&ud, 0, sizeof(ud));
  ud.pd_opaque = pd;
  ud.d_hdmag = d_hdmag;
  ud.nx = 3 * ng;
  ud.ny = ny;
  ud.ng = ng;
  ud.ncell = ng * ny;
  ud.neq = 3 * ng * ny;
  if (n0) { ud.nxx0 = n0[0]; ud.nyy0 = n0[1]; ud.nzz0 = n0[2]; }
  return ud;
}

// PrecondSetup at y with the demag field d_hdmag and self-coupling n0[3]
extern "C" int ref_i1_psetup(void* pd, double* d_y, double* d_hdmag, const double* n0, double gamma, int ng, int ny) {
  PcUserData ud = ref_ud(pd, d_hdmag, ng, ny, n0);
  llg_shim_nvector y = {d_y, nullptr, 3L * ng * ny};
  sunbooleantype jcur = 0;
  const int rc = PrecondSetup(0.0, &y, nullptr, 0, &jcur, gamma, &ud);
  return (cudaDeviceSynchronize() == cudaSuccess && jcur) ? rc : -1;
}

extern "C" int ref_i1_psolve(void* pd, double* d_r, double* d_z, int ng, int ny) {
  PcUserData ud = ref_ud(pd, nullptr, ng, ny, nullptr);
  const long n3 = 3L * ng * ny;
  llg_shim_nvector r = {d_r, nullptr, n3}, z = {d_z, nullptr, n3};
  const int rc = PrecondSolve(0.0, nullptr, nullptr, &r, &z, 0.0, 0.0, 1, &ud);
  return (cudaDeviceSynchronize() == cudaSuccess) ? rc : -1;
}
