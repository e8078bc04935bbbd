// ref_i6_precond.cu — the reference's compact block-Jacobi PrecondSetup /
// PrecondSolve (build_J_kernel_compact, apply_P_kernel_compact,
// pc_zero_inactive_kernel), compiled from src/irregular/2d_fft/2d_i6/precond.cu
// where it lies.  TEST INFRASTRUCTURE ONLY.
#include <string.h>

#include "precond.cu"

extern "C" int ref_i6_set_precond_consts(double chk, double che, double alpha, double chg) {
  cudaError_t e = cudaMemcpyToSymbol(pc_chk, &chk, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(pc_che, &che, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(pc_alpha, &alpha, sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(pc_chg, &chg, sizeof(double));
  return e == cudaSuccess ? 0 : -1;
}

static PcUserData ref_ud(void* pd, double* d_hdmag, int* d_active, int n_active, int* d_inactive, int n_inactive,
                         int ng, int ny, const double* n0) {
  PcUserData ud;
  memset(&ud, 0, sizeof(ud));
  ud.pd_opaque = pd;
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
  if (n0) { ud.nxx0 = n0[0]; ud.nyy0 = n0[1]; ud.nzz0 = n0[2]; }
  return ud;
}

// PrecondSetup at y with the demag field d_hdmag and self-coupling n0[3]
extern "C" int ref_i6_psetup(void* pd, double* d_y, double* d_hdmag, const double* n0, double gamma,
                             int* d_active, int n_active, int* d_inactive, int n_inactive, int ng, int ny) {
  PcUserData ud = ref_ud(pd, d_hdmag, d_active, n_active, d_inactive, n_inactive, ng, ny, n0);
  llg_shim_nvector y = {d_y, nullptr, 3L * ng * ny};
  sunbooleantype jcur = 0;
  const int rc = PrecondSetup(0.0, &y, nullptr, 0, &jcur, gamma, &ud);
  return (cudaDeviceSynchronize() == cudaSuccess && jcur) ? rc : -1;
}

extern "C" int ref_i6_psolve(void* pd, double* d_r, double* d_z, int* d_active, int n_active, int* d_inactive,
                             int n_inactive, int ng, int ny) {
  PcUserData ud = ref_ud(pd, nullptr, d_active, n_active, d_inactive, n_inactive, ng, ny, nullptr);
  const long n3 = 3L * ng * ny;
  llg_shim_nvector r = {d_r, nullptr, n3}, z = {d_z, nullptr, n3};
  const int rc = PrecondSolve(0.0, nullptr, nullptr, &r, &z, 0.0, 0.0, 1, &ud);
  return (cudaDeviceSynchronize() == cudaSuccess) ? rc : -1;
}
