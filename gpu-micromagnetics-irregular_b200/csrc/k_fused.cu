// k_fused.cu — integrator-specific fused passes, sm_100a.
//
// CVODE drives the reference's callbacks through chains of N_Vector calls
// (linear sums, scalings, dot products; src/irregular/2d_fft/2d_i2/2d_fft.cu
// :648-724 and the SUNDIALS NVECTOR_CUDA kernels that show up as ~45 % of its
// kernel time).  Each function here is one HBM pass that applies, element by
// element, the same operations as a chain of those calls:
//
//   fused_ewt_wrms        ewt = 1/(rtol|y|+atol)  +  ||y||_wrms(ewt)
//   fused_lin_normalize   y = zn0 + ycor, then the RHS's normalisation
//   fused_field           the RHS's demag field for y (or zero)
//   fused_resid           RHS f(y) and the Newton residual
//                         −(−γ f + (rl1 zn1 + ycor)) in the epilogue
//   fused_psolve_scale_dot  V0 = ewt ⊙ P⁻¹ r  +  V0·V0
//   fused_lincomb_norm    z = Σ c_k X_k  +  z·z           (classical GS)
//   fused_lincomb_div     z = (Σ c_k X_k) / w             (GMRES correction)
//   fused_update_wrms2    ycor += del  +  ||del||, ||ycor|| (Newton test)
//   fused_wrms2           ||x1||  and  ||a x2 + b x3||     (order selection)
//
// Reductions use the deterministic partition of dev_reduce.cuh; results land
// in c->d_scal as raw sums (the host takes sqrt(s/neq)).
#include <math.h>

#include "dev_physics.cuh"
#include "dev_reduce.cuh"
#include "llg_internal.h"
#include "launch.h"
#include "dev_integ.h"

namespace {

constexpr int FV = 17;
struct CPack {
  double c[FV];
};
struct XPack {
  const double* p[FV];
};
// Krylov basis vectors stored as VT (double, or float for the FP32-basis solver)
template <typename T>
struct XPackT {
  const T* p[FV];
};
struct ZPack {
  double* p[8];
};

int cell_blocks(int ncell) { return red_blocks(ncell); }

__global__ void __launch_bounds__(RT) k_ewt_wrms(double rtol, double atol, const double* __restrict__ y,
                                                 double* __restrict__ ewt, long long n, double* partials,
                                                 unsigned int* counter, double* out, const DevArgs* da) {
  pdl_entry();
  if (da && !da->run_ewt) return;
  __shared__ double sm[2 * (RT / 32)];
  double acc[2] = {0.0, 0.0};
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double yi = y[i];
    const double t = rtol * fabs(yi) + atol;
    if (t <= 0.0) acc[0] += 1.0;   // (a NaN state is left to the norm check)
    const double w = 1.0 / t;
    ewt[i] = w;
    const double p = yi * w;
    acc[1] += p * p;
  }
  block_sum<2>(acc, sm);
  finalize<2>(partials, gridDim.x, counter, out, 0, 1.0, acc);
}

// A null ycor stands for the zero vector (the Newton iteration's first
// iterate); 1*x + 1*0 is x exactly, so the result is the same either way.
__device__ __forceinline__ double ycor_at(const double* ycor, int i) { return ycor ? ycor[i] : 0.0; }

__global__ void k_lin_normalize(const double* __restrict__ zn0, const double* __restrict__ ycor,
                                double* __restrict__ y, int n, int kind, double eps, const DevArgs* da) {
  pdl_entry();
  if (da && da->ycor_zero) ycor = nullptr;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double m1 = 1.0 * zn0[k] + 1.0 * ycor_at(ycor, k);
    const double m2 = 1.0 * zn0[n + k] + 1.0 * ycor_at(ycor, n + k);
    const double m3 = 1.0 * zn0[2 * n + k] + 1.0 * ycor_at(ycor, 2 * n + k);
    double o1 = m1, o2 = m2, o3 = m3;
    if (kind != LLG_NORM_NONE) {
      const double ymp = sqrt(m1 * m1 + m2 * m2 + m3 * m3);
      if (kind == LLG_NORM_REG) {
        const double inv = 1.0 / (ymp + eps);
        o1 = m1 * inv; o2 = m2 * inv; o3 = m3 * inv;
      } else if (ymp > 1.0e-30) {
        const double inv = 1.0 / ymp;
        o1 = m1 * inv; o2 = m2 * inv; o3 = m3 * inv;
      }
    }
    y[k] = o1; y[n + k] = o2; y[2 * n + k] = o3;
  }
}

// RHS at y with the Newton residual epilogue; writes −res (the Newton
// iteration's negated right-hand side) and no ydot.
__global__ void __launch_bounds__(TX * TY) k_rhs_resid_tile(DevProblem P, const double* __restrict__ y,
                                                            const double* __restrict__ hd,
                                                            const double* __restrict__ zn1,
                                                            const double* __restrict__ ycor, double rl1,
                                                            double gamma, double* __restrict__ negres,
                                                            const DevArgs* da) {
  pdl_entry();
  __shared__ Tile<1> T;
  if (da) {
    rl1 = da->rl1;
    gamma = da->gamma;
    if (da->ycor_zero) ycor = nullptr;
  }
  const double* f[1] = {y};
  load_tile<1>(P, T, f);
  const int gi = blockIdx.x * TX + threadIdx.x, gj = blockIdx.y * TY + threadIdx.y;
  if (gi >= P.ng || gj >= P.ny) return;
  const int n = P.ncell, cell = gj * P.ng + gi;
  const double m[3] = {y[cell], y[n + cell], y[2 * n + cell]};
  double msk[3], nsk[3];
  cell_axes(P, cell, msk, nsk);
  double h[3];
  tile_field(P, T.v[0], threadIdx.x + 1, threadIdx.y + 1, m, msk, nsk, h);
#pragma unroll
  for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + happ_at(P, a, gi);
  double o[3];
  llg_torque(P, alpha_at(P, gi), m, h, gate_of(P, cell), o);
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int i = a * n + cell;
    const double t = rl1 * zn1[i] + 1.0 * ycor_at(ycor, i);
    const double r = (-gamma) * o[a] + 1.0 * t;
    negres[i] = -1.0 * r;
  }
}

__global__ void k_rhs_resid_compact(DevProblem P, const double* __restrict__ y, const double* __restrict__ hd,
                                    const int32_t* __restrict__ act_ids, int na,
                                    const int32_t* __restrict__ inact_ids, int ni,
                                    const double* __restrict__ zn1, const double* __restrict__ ycor, double rl1,
                                    double gamma, double* __restrict__ negres, const DevArgs* da) {
  pdl_entry();
  const int n = P.ncell;
  if (da) {
    rl1 = da->rl1;
    gamma = da->gamma;
    if (da->ycor_zero) ycor = nullptr;
  }
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na + ni; t += gridDim.x * blockDim.x) {
    double o[3] = {0.0, 0.0, 0.0};
    int cell;
    if (t >= na) {
      cell = inact_ids[t - na];
    } else {
      cell = act_ids[t];
      const int gi = cell % P.ng, gj = cell / P.ng;
      const double m[3] = {y[cell], y[n + cell], y[2 * n + cell]};
      double msk[3], nsk[3];
      cell_axes(P, cell, msk, nsk);
      double h[3];
      gather_field(P, y, gi, gj, m, msk, nsk, h);
#pragma unroll
      for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + happ_at(P, a, gi);
      llg_torque(P, alpha_at(P, gi), m, h, 1.0, o);
    }
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int i = a * n + cell;
      const double tt = rl1 * zn1[i] + 1.0 * ycor_at(ycor, i);
      const double r = (-gamma) * o[a] + 1.0 * tt;
      negres[i] = -1.0 * r;
    }
  }
}

// (streams at HBM speed, so it rebuilds the block from the frozen (m, h),
// 48 B/cell, rather than reading the 72 B/cell FP64 inverse that psetup
// stores; pinvf non-null: the FP32 inverse stored for an FP32 Krylov basis,
// 36 B/cell, which the Arnoldi operator applies too, is read instead)
template <typename VT = double>
__global__ void __launch_bounds__(RT) k_psolve_scale_dot(DevProblem P, const double* __restrict__ pm,
                                                         const double* __restrict__ ph,
                                                         const float* __restrict__ pinvf,
                                                         const double* __restrict__ r,
                                                         const double* __restrict__ ewt, VT* __restrict__ v0,
                                                         double gamma, double* partials, unsigned int* counter,
                                                         double* out, const DevArgs* da, double* aout) {
  pdl_entry();
  __shared__ double sm[RT / 32];
  double acc[1] = {0.0};
  const int n = P.ncell;
  if (da) gamma = da->gamma_setup;
  for (int k = blockIdx.x * RT + threadIdx.x; k < n; k += gridDim.x * RT) {
    const double rr[3] = {r[k], r[n + k], r[2 * n + k]};
    double Pi[9];
    if (pinvf) {
      load_pinv(pinvf, n, k, Pi);
    } else {
      const double m[3] = {pm[k], pm[n + k], pm[2 * n + k]};
      const double h[3] = {ph[k], ph[n + k], ph[2 * n + k]};
      double msk[3], nsk[3];
      cell_axes(P, k, msk, nsk);
      const double ws = P.windowed ? P.w[k] : 1.0;
      block_inverse(P, m, h, msk, ws, gamma, Pi);
    }
    double g = 1.0;
    if (!P.windowed && P.act) g = P.act[k] ? 1.0 : 0.0;
    const double z0 = g * (Pi[0] * rr[0] + Pi[1] * rr[1] + Pi[2] * rr[2]);
    const double z1 = g * (Pi[3] * rr[0] + Pi[4] * rr[1] + Pi[5] * rr[2]);
    const double z2 = g * (Pi[6] * rr[0] + Pi[7] * rr[1] + Pi[8] * rr[2]);
    const VT a0 = (VT)(ewt[k] * z0), a1 = (VT)(ewt[n + k] * z1), a2 = (VT)(ewt[2 * n + k] * z2);
    v0[k] = a0; v0[n + k] = a1; v0[2 * n + k] = a2;
    acc[0] += (double)a0 * (double)a0;
    acc[0] += (double)a1 * (double)a1;
    acc[0] += (double)a2 * (double)a2;
  }
  block_sum<1>(acc, sm);
  const bool last = finalize<1>(partials, gridDim.x, counter, out, 0, 1.0, acc);
  if (last && aout && threadIdx.x == 0) *aout = gs_scale_of(out[0], nullptr);   // 1 / ||V0||
}

// z = c0 X0; z = c_k X_k + z (z may alias X0), and sum z^2
template <typename VT = double>
__global__ void __launch_bounds__(RT) k_lincomb_norm(int nv, CPack c, XPackT<VT> X, VT* z, long long n,
                                                     double* partials, unsigned int* counter, double* out,
                                                     KScale ks) {
  pdl_entry();
  __shared__ double sm[RT / 32];
  __shared__ double xs[FV];   // scales of the X vectors, staged once (see k_lincomb_update)
  if (threadIdx.x < nv) xs[threadIdx.x] = kscale_of(ks.a[threadIdx.x]);
  __syncthreads();
  double acc[1] = {0.0};
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    double s = c.c[0] * (xs[0] * (double)X.p[0][i]);
    for (int k = 1; k < nv; k++) s = c.c[k] * (xs[k] * (double)X.p[k][i]) + s;
    const VT sv = (VT)s;
    z[i] = sv;
    acc[0] += (double)sv * (double)sv;
  }
  block_sum<1>(acc, sm);
  finalize<1>(partials, gridDim.x, counter, out, 0, 1.0, acc);
}

template <typename VT = double>
__global__ void k_lincomb_div(int nv, CPack c, XPackT<VT> X, const double* __restrict__ w, double* __restrict__ z,
                              long long n, KScale ks) {
  pdl_entry();
  __shared__ double xs[FV];   // scales of the X vectors, staged once (see k_lincomb_update)
  if (threadIdx.x < nv) xs[threadIdx.x] = kscale_of(ks.a[threadIdx.x]);
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double s = c.c[0] * (xs[0] * (double)X.p[0][i]);
    for (int k = 1; k < nv; k++) s = c.c[k] * (xs[k] * (double)X.p[k][i]) + s;
    z[i] = s / w[i];
  }
}

// ycor = 1*ycor + 1*del (ycor_in null: zero); sums (del*w)^2 and (ycor*w)^2
__global__ void __launch_bounds__(RT) k_update_wrms2(const double* ycor_in, double* ycor, const double* __restrict__ del,
                                                     const double* __restrict__ w, long long n, double* partials,
                                                     unsigned int* counter, double* out, const DevArgs* da, Pub pub) {
  pdl_entry();
  __shared__ double sm[2 * (RT / 32)];
  double acc[2] = {0.0, 0.0};
  if (da) {
    if (!da->run_update) return;
    ycor_in = da->ycor_zero ? nullptr : ycor;
  }
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double d = del[i];
    const double yc = 1.0 * (ycor_in ? ycor_in[i] : 0.0) + 1.0 * d;
    ycor[i] = yc;
    const double wi = w[i];
    const double p = d * wi, q = yc * wi;
    acc[0] += p * p;
    acc[1] += q * q;
  }
  block_sum<2>(acc, sm);
  if (finalize<2>(partials, gridDim.x, counter, out, 0, 1.0, acc)) publish_carried(pub);
}

// GMRES correction and Newton update in one pass: d = (sum_k c_k X_k) / w
// (the correction, stored only when del is non-null), ycor = 1*ycor + 1*d
// (ycor_in null: zero), and the sums (d*w)^2, (ycor*w)^2 — per element the
// arithmetic of k_lincomb_div followed by k_update_wrms2, with the latter's
// reduction partition
template <typename VT = double>
__global__ void __launch_bounds__(RT) k_lincomb_update(int nv, CPack c, XPackT<VT> X, const double* __restrict__ w,
                                                       double* del, const double* ycor_in, double* ycor, long long n,
                                                       double* partials, unsigned int* counter, double* out,
                                                       KScale ks, Pub pub) {
  pdl_entry();
  __shared__ double sm[2 * (RT / 32)];
  // scales of the X vectors (1 when stored normalised), staged once: read
  // through pointers they would be reloaded after every store (aliasing)
  __shared__ double xs[FV];
  if (threadIdx.x < nv) xs[threadIdx.x] = kscale_of(ks.a[threadIdx.x]);
  __syncthreads();
  const double xa0 = xs[0];
  double acc[2] = {0.0, 0.0};
  const long long st = (long long)gridDim.x * RT;
  for (long long i0 = blockIdx.x * (long long)RT + threadIdx.x; i0 < n; i0 += UB * st) {
    double s[UB], wv[UB], yv[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const long long i = i0 + u * st;
      const bool in = i < n;
      s[u] = in ? c.c[0] * (xa0 * (double)X.p[0][i]) : 0.0;
      wv[u] = in ? w[i] : 1.0;
      yv[u] = (in && ycor_in) ? ycor_in[i] : 0.0;
    }
    for (int k = 1; k < nv; k++) {
      const double xa = xs[k];
      double xv[UB];
#pragma unroll
      for (int u = 0; u < UB; u++) xv[u] = (i0 + u * st < n) ? xa * (double)X.p[k][i0 + u * st] : 0.0;
#pragma unroll
      for (int u = 0; u < UB; u++) s[u] = c.c[k] * xv[u] + s[u];
    }
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const long long i = i0 + u * st;
      if (i >= n) continue;
      const double wi = wv[u];
      const double d = s[u] / wi;
      if (del) del[i] = d;
      const double yc = 1.0 * yv[u] + 1.0 * d;
      ycor[i] = yc;
      const double p = d * wi, q = yc * wi;
      acc[0] += p * p;
      acc[1] += q * q;
    }
  }
  block_sum<2>(acc, sm);
  if (finalize<2>(partials, gridDim.x, counter, out, 0, 1.0, acc)) publish_carried(pub);
}

// k_lincomb_update with the vector count NV fixed at compile time: the loads
// of all NV vectors (and of w, ycor) for the UB slice elements are issued
// before any of them is used.  Per element the same operations in the same
// order, so the vectors are bitwise those of k_lincomb_update; it runs on one
// resident wave of blocks (red_blocks_resident), so its two sums are added in
// another partition.
template <int NV, typename VT>
__global__ void __launch_bounds__(RT) k_lincomb_update_k(CPack c, XPackT<VT> X, const double* __restrict__ w,
                                                         double* del, const double* ycor_in, double* ycor,
                                                         long long n, double* partials, unsigned int* counter,
                                                         double* out, KScale ks, Pub pub) {
  pdl_entry();
  __shared__ double sm[2 * (RT / 32)];
  __shared__ double xs[NV];
  if (threadIdx.x < NV) xs[threadIdx.x] = kscale_of(ks.a[threadIdx.x]);
  __syncthreads();
  double cf[NV], xa[NV];
#pragma unroll
  for (int k = 0; k < NV; k++) {
    cf[k] = c.c[k];
    xa[k] = xs[k];
  }
  double acc[2] = {0.0, 0.0};
  const long long st = (long long)gridDim.x * RT;
  for (long long i0 = blockIdx.x * (long long)RT + threadIdx.x; i0 < n; i0 += UB * st) {
    VT xr[NV][UB];
    double wv[UB], yv[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const long long i = i0 + u * st;
      const bool in = i < n;
#pragma unroll
      for (int k = 0; k < NV; k++) xr[k][u] = in ? X.p[k][i] : VT(0);
      wv[u] = in ? w[i] : 1.0;
      yv[u] = (in && ycor_in) ? ycor_in[i] : 0.0;
    }
    double s[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) s[u] = cf[0] * (xa[0] * (double)xr[0][u]);
#pragma unroll
    for (int k = 1; k < NV; k++)
#pragma unroll
      for (int u = 0; u < UB; u++) s[u] = cf[k] * (xa[k] * (double)xr[k][u]) + s[u];
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const long long i = i0 + u * st;
      if (i >= n) continue;
      const double wi = wv[u];
      const double d = s[u] / wi;
      if (del) del[i] = d;
      const double yc = 1.0 * yv[u] + 1.0 * d;
      ycor[i] = yc;
      const double p = d * wi, q = yc * wi;
      acc[0] += p * p;
      acc[1] += q * q;
    }
  }
  block_sum<2>(acc, sm);
  if (finalize<2>(partials, gridDim.x, counter, out, 0, 1.0, acc)) publish_carried(pub);
}

// sums (x1*w)^2 and ((a x2 + b x3)*w)^2
__global__ void __launch_bounds__(RT) k_wrms2(const double* __restrict__ x1, double a, const double* __restrict__ x2,
                                              double b, const double* __restrict__ x3, const double* __restrict__ w,
                                              long long n, double* partials, unsigned int* counter, double* out) {
  pdl_entry();
  __shared__ double sm[2 * (RT / 32)];
  double acc[2] = {0.0, 0.0};
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double wi = w[i];
    const double p = x1[i] * wi;
    const double v = a * x2[i] + b * x3[i];
    const double q = v * wi;
    acc[0] += p * p;
    acc[1] += q * q;
  }
  block_sum<2>(acc, sm);
  finalize<2>(partials, gridDim.x, counter, out, 0, 1.0, acc);
}

// Start of a BDF attempt, one pass per cell: (new step only) the tolerance
// weights of zn0 with their bad-weight count and ||zn0||^2; (when pending)
// zn[j] *= f_j, j = 1..Q; the Nordsieck predictor (Pascal triangle); and y =
// normalise(zn0 + 0), the first Newton iterate's state.  Per element the
// arithmetic of k_ewt_wrms, k_scale_cols, k_nordsieck and k_lin_normalize.
// Every load of a cell is issued before its first store.
template <int Q>
__global__ void __launch_bounds__(RT) k_predict_fused(ZPack zn, CPack f, int pend, int do_ewt, double rtol,
                                                      double atol, double* __restrict__ ewt, double* __restrict__ y,
                                                      int n, int kind, double eps, double* partials,
                                                      unsigned int* counter, double* out, int lazy, CPack lc,
                                                      const double* __restrict__ acor, double* zsave) {
  pdl_entry();
  __shared__ double sm[2 * (RT / 32)];
  double acc[2] = {0.0, 0.0};
  for (int cell = blockIdx.x * RT + threadIdx.x; cell < n; cell += gridDim.x * RT) {
    double v[3][Q + 1];
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int j = 0; j <= Q; j++) v[a][j] = zn.p[j][(long long)a * n + cell];
    double xc[3] = {0.0, 0.0, 0.0};
    if (lazy) {
#pragma unroll
      for (int a = 0; a < 3; a++) xc[a] = acor[(long long)a * n + cell];
    }
    double m[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const long long i = (long long)a * n + cell;
      if (lazy) {   // the previous step's completion (k_complete_norms' arithmetic)
#pragma unroll
        for (int j = 0; j <= Q; j++) v[a][j] = lc.c[j] * xc[a] + v[a][j];
        if (zsave) zsave[i] = 1.0 * xc[a];
      }
      if (do_ewt) {
        const double t = rtol * fabs(v[a][0]) + atol;
        if (t <= 0.0) acc[0] += 1.0;   // (a NaN state is left to the norm check)
        const double w = 1.0 / t;
        ewt[i] = w;
        const double p = v[a][0] * w;
        acc[1] += p * p;
      }
      if (pend) {
#pragma unroll
        for (int j = 1; j <= Q; j++) v[a][j] = f.c[j] * v[a][j];
      }
#pragma unroll
      for (int k = 1; k <= Q; k++)
#pragma unroll
        for (int j = Q; j >= k; j--) v[a][j - 1] = v[a][j - 1] + v[a][j];
#pragma unroll
      for (int j = 0; j < Q; j++) zn.p[j][i] = v[a][j];
      if (pend || lazy) zn.p[Q][i] = v[a][Q];
      m[a] = 1.0 * v[a][0] + 1.0 * 0.0;
    }
    double o[3] = {m[0], m[1], m[2]};
    if (kind != LLG_NORM_NONE) {
      const double ymp = sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
      if (kind == LLG_NORM_REG) {
        const double inv = 1.0 / (ymp + eps);
        o[0] = m[0] * inv; o[1] = m[1] * inv; o[2] = m[2] * inv;
      } else if (ymp > 1.0e-30) {
        const double inv = 1.0 / ymp;
        o[0] = m[0] * inv; o[1] = m[1] * inv; o[2] = m[2] * inv;
      }
    }
    y[cell] = o[0]; y[n + cell] = o[1]; y[2 * n + cell] = o[2];
  }
  if (do_ewt) {
    block_sum<2>(acc, sm);
    finalize<2>(partials, gridDim.x, counter, out, 0, 1.0, acc);
  }
}

// complete_step and the order-selection norms in one pass: zn[j] = l_j acor +
// zn[j] (j = 0..Q); zn[qmax] = 1 * acor when save; when norms, the sums
// (zn[Q] w)^2 and ((-cquot zn[qmax] + 1 acor) w)^2 of the updated vectors —
// the arithmetic of k_scale_add_multi, k_scale and k_wrms2, with k_wrms2's
// reduction partition.  Every load of an element is issued before its stores.
// (store 0: the norms alone, of the completed values, nothing written — the
// completion itself is then applied by the next predict pass)
template <int Q>
__global__ void __launch_bounds__(RT) k_complete_norms(int qmax, CPack l, const double* __restrict__ acor, ZPack zn,
                                                       double* zmaxp, int save, int norms, double a2,
                                                       const double* __restrict__ w,
                                                       long long n, double* partials, unsigned int* counter,
                                                       double* out, int store) {
  pdl_entry();
  __shared__ double sm[2 * (RT / 32)];
  double acc[2] = {0.0, 0.0};
  const bool far = norms && !save && qmax > Q;   // zn[qmax] is read, not updated
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double xi = acor[i];
    double v[Q + 1];
    if (store) {
#pragma unroll
      for (int j = 0; j <= Q; j++) v[j] = zn.p[j][i];
    } else {
      v[Q] = zn.p[Q][i];
    }
    const double zfar = far ? zmaxp[i] : 0.0;
    const double wi = norms ? w[i] : 0.0;
    if (store) {
#pragma unroll
      for (int j = 0; j <= Q; j++) {
        v[j] = l.c[j] * xi + v[j];
        zn.p[j][i] = v[j];
      }
    } else {
      v[Q] = l.c[Q] * xi + v[Q];
    }
    double zmax = (qmax == Q) ? v[Q] : zfar;
    if (save) {
      const double z = 1.0 * xi;
      if (store) zmaxp[i] = z;
      zmax = z;
    }
    if (norms) {
      const double p = v[Q] * wi;
      const double u = a2 * zmax + 1.0 * xi;
      const double qq = u * wi;
      acc[0] += p * p;
      acc[1] += qq * qq;
    }
  }
  if (norms) {
    block_sum<2>(acc, sm);
    finalize<2>(partials, gridDim.x, counter, out, 0, 1.0, acc);
  }
}

int ew_blocks(const llg_ctx* c, long long n) {
  long long g = (n + 255) / 256;
  const long long cap = (long long)c->num_sms * 8;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

int fused_ewt_wrms(llg_ctx* c, double rtol, double atol, const double* y, double* ewt, int slot, const DevArgs* da) {
  LLG_COUNT(KID_REDUCE);
  klaunch(k_ewt_wrms, red_blocks(c->neq), RT, 0, c->stream, rtol, atol, y, ewt, c->neq, c->d_red, c->d_counter,
                                                       c->d_scal + slot, da);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int fused_lin_normalize(llg_ctx* c, const double* zn0, const double* ycor, double* y, const DevArgs* da) {
  LLG_COUNT(KID_NORM);
  klaunch(k_lin_normalize, ew_blocks(c, c->ncell), 256, 0, c->stream, zn0, ycor, y, c->ncell, c->p.norm_kind,
                                                                c->p.norm_eps, da);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int fused_field(llg_ctx* c, const double* y) {
  if (c->demag) {
    const int rc = demag_apply(c, y, c->d_hd);
    if (rc) return rc;
    c->nfe_demag++;
    return 0;
  }
  // no demag: the field buffer was cleared when the context was made and
  // nothing else writes it
  return 0;
}

int fused_resid(llg_ctx* c, const double* y, const double* zn1, const double* ycor, double rl1, double gamma,
                double* negres, const DevArgs* da) {
  LLG_COUNT(KID_RHS);
  if (c->p.exec_model == LLG_EXEC_COMPACT) {
    const int tot = c->n_active + c->n_inactive;
    klaunch(k_rhs_resid_compact, ew_blocks(c, tot), 256, 0, c->stream, c->dp, y, c->d_hd, c->d_active_ids, c->n_active,
                                                                   c->d_inactive_ids, c->n_inactive, zn1, ycor, rl1,
                                                                   gamma, negres, da);
  } else {
    dim3 g((c->p.ng + TX - 1) / TX, (c->p.ny + TY - 1) / TY);
    klaunch(k_rhs_resid_tile, g, dim3(TX, TY), 0, c->stream, c->dp, y, c->d_hd, zn1, ycor, rl1, gamma, negres, da);
  }
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

template <typename VT>
static int psolve_scale_dot_impl(llg_ctx* c, const double* r, const double* ewt, VT* v0, int slot, const DevArgs* da,
                                 int slot_aout) {
  if (!c->have_setup && !da) { llg_set_error("psolve before psetup"); return LLG_ERR_STATE; }
  LLG_COUNT(KID_PSOLVE);
  const float* pinvf = (sizeof(VT) == sizeof(float) && c->pinv_f32 && !da) ? reinterpret_cast<const float*>(c->d_pinv)
                                                                          : nullptr;
  klaunch(k_psolve_scale_dot<VT>, cell_blocks(c->ncell), RT, 0, c->stream, c->dp, c->d_pm, c->d_ph, pinvf, r, ewt,
          v0, c->gamma_setup, c->d_red, c->d_counter, c->d_scal + slot, da,
          slot_aout >= 0 ? c->d_scal + slot_aout : nullptr);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int fused_psolve_scale_dot(llg_ctx* c, const double* r, const double* ewt, double* v0, int slot, const DevArgs* da,
                           int slot_aout) {
  return psolve_scale_dot_impl<double>(c, r, ewt, v0, slot, da, slot_aout);
}
int fused_psolve_scale_dot_f(llg_ctx* c, const double* r, const double* ewt, float* v0, int slot, int slot_aout) {
  return psolve_scale_dot_impl<float>(c, r, ewt, v0, slot, nullptr, slot_aout);
}

template <typename VT>
static int lincomb_norm_impl(llg_ctx* c, int nv, const double* coef, const VT* const* X, VT* z, int slot,
                             const KScale* ks) {
  if (nv < 1 || nv > FV) { llg_set_error("lincomb_norm: bad nvec"); return LLG_ERR_ARG; }
  CPack cp{};
  XPackT<VT> xp{};
  for (int k = 0; k < nv; k++) { cp.c[k] = coef[k]; xp.p[k] = X[k]; }
  const KScale kz{};
  LLG_COUNT(KID_REDUCE);
  klaunch(k_lincomb_norm<VT>, red_blocks(c->neq), RT, 0, c->stream, nv, cp, xp, z, c->neq, c->d_red, c->d_counter,
          c->d_scal + slot, ks ? *ks : kz);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int fused_lincomb_norm(llg_ctx* c, int nv, const double* coef, const double* const* X, double* z, int slot,
                       const KScale* ks) {
  return lincomb_norm_impl<double>(c, nv, coef, X, z, slot, ks);
}
int fused_lincomb_norm_f(llg_ctx* c, int nv, const double* coef, const float* const* X, float* z, int slot,
                         const KScale* ks) {
  return lincomb_norm_impl<float>(c, nv, coef, X, z, slot, ks);
}

template <typename VT>
static int lincomb_div_impl(llg_ctx* c, int nv, const double* coef, const VT* const* X, const double* w, double* z,
                            const KScale* ks) {
  if (nv < 1 || nv > FV) { llg_set_error("lincomb_div: bad nvec"); return LLG_ERR_ARG; }
  CPack cp{};
  XPackT<VT> xp{};
  for (int k = 0; k < nv; k++) { cp.c[k] = coef[k]; xp.p[k] = X[k]; }
  const KScale kz{};
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_lincomb_div<VT>, ew_blocks(c, c->neq), 256, 0, c->stream, nv, cp, xp, w, z, c->neq, ks ? *ks : kz);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int fused_lincomb_div(llg_ctx* c, int nv, const double* coef, const double* const* X, const double* w, double* z,
                      const KScale* ks) {
  return lincomb_div_impl<double>(c, nv, coef, X, w, z, ks);
}
int fused_lincomb_div_f(llg_ctx* c, int nv, const double* coef, const float* const* X, const double* w, double* z,
                        const KScale* ks) {
  return lincomb_div_impl<float>(c, nv, coef, X, w, z, ks);
}

int fused_update_wrms2(llg_ctx* c, bool ycor_zero, double* ycor, const double* del, const double* w, int slot,
                       const DevArgs* da) {
  LLG_COUNT(KID_REDUCE);
  // (the device-resident form reads nothing back through the mailbox)
  const Pub pub = da ? Pub{} : take_publish(c);
  klaunch(k_update_wrms2, red_blocks(c->neq), RT, 0, c->stream, ycor_zero ? nullptr : ycor, ycor, del, w, c->neq, c->d_red, c->d_counter,
                                                           c->d_scal + slot, da, pub);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int fused_wrms2(llg_ctx* c, const double* x1, double a, const double* x2, double b, const double* x3,
                const double* w, int slot) {
  LLG_COUNT(KID_REDUCE);
  klaunch(k_wrms2, red_blocks(c->neq), RT, 0, c->stream, x1, a, x2, b, x3, w, c->neq, c->d_red, c->d_counter,
                                                    c->d_scal + slot);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

template <typename VT>
static int lincomb_update_impl(llg_ctx* c, int nv, const double* coef, const VT* const* X, const double* w,
                               double* del, bool ycor_zero, double* ycor, int slot, const KScale* ks) {
  if (nv < 1 || nv > FV) { llg_set_error("lincomb_update: bad nvec"); return LLG_ERR_ARG; }
  CPack cp{};
  XPackT<VT> xp{};
  for (int k = 0; k < nv; k++) { cp.c[k] = coef[k]; xp.p[k] = X[k]; }
  const KScale kz{};
  const KScale kk = ks ? *ks : kz;
  LLG_COUNT(KID_REDUCE);
  const int nb = red_blocks(c->neq);
  const double* yin = ycor_zero ? nullptr : ycor;
  double* out = c->d_scal + slot;
  const Pub pub = take_publish(c);
#define LU_K(NV)                                                                                                   \
  klaunch(k_lincomb_update_k<NV, VT>, red_blocks_resident(c->neq, LLG_PER_SM((k_lincomb_update_k<NV, VT>)), c->num_sms), \
          RT, 0, c->stream, cp, xp, w, del, yin, ycor, c->neq, c->d_red, c->d_counter, out, kk, pub)
  switch (nv) {
    case 1: LU_K(1); break;
    case 2: LU_K(2); break;
    case 3: LU_K(3); break;
    case 4: LU_K(4); break;
    case 5: LU_K(5); break;
    case 6: LU_K(6); break;
    case 7: LU_K(7); break;
    case 8: LU_K(8); break;
    default:
      klaunch(k_lincomb_update<VT>, nb, RT, 0, c->stream, nv, cp, xp, w, del, yin, ycor, c->neq, c->d_red,
              c->d_counter, out, kk, pub);
  }
#undef LU_K
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int fused_lincomb_update(llg_ctx* c, int nv, const double* coef, const double* const* X, const double* w,
                         double* del, bool ycor_zero, double* ycor, int slot, const KScale* ks) {
  return lincomb_update_impl<double>(c, nv, coef, X, w, del, ycor_zero, ycor, slot, ks);
}
int fused_lincomb_update_f(llg_ctx* c, int nv, const double* coef, const float* const* X, const double* w,
                           double* del, bool ycor_zero, double* ycor, int slot, const KScale* ks) {
  return lincomb_update_impl<float>(c, nv, coef, X, w, del, ycor_zero, ycor, slot, ks);
}

int fused_predict(llg_ctx* c, int q, double* const* zn, const double* f, bool pend, bool do_ewt, double rtol,
                  double atol, double* ewt, double* y, int slot, const double* lazy_l, const double* acor,
                  double* zsave) {
  if (q < 1 || q > 5) { llg_set_error("predict: bad order"); return LLG_ERR_ARG; }
  ZPack zp{};
  CPack fp{}, lp{};
  for (int j = 0; j <= q; j++) { zp.p[j] = zn[j]; fp.c[j] = f ? f[j] : 1.0; lp.c[j] = lazy_l ? lazy_l[j] : 0.0; }
  const int lz = lazy_l ? 1 : 0;
  LLG_COUNT(KID_ELEMWISE);
  long long nbl = (c->ncell + RT - 1) / RT;   // ~one cell per thread, up to the partials' capacity
  if (nbl > RMAXB) nbl = RMAXB;
  if (nbl < 1) nbl = 1;
  const int nb = (int)nbl;
  const int pe = pend ? 1 : 0, de = do_ewt ? 1 : 0;
  double* out = c->d_scal + slot;
#define PRED(Q)                                                                                                \
  klaunch(k_predict_fused<Q>, cap_resident(nb, LLG_PER_SM((k_predict_fused<Q>)), c->num_sms), RT, 0, c->stream,  \
          zp, fp, pe, de, rtol, atol, ewt, y, c->ncell, c->p.norm_kind,                                          \
                                               c->p.norm_eps, c->d_red, c->d_counter, out, lz, lp, acor,         \
                                               lz ? zsave : nullptr)
  switch (q) {
    case 1: PRED(1); break;
    case 2: PRED(2); break;
    case 3: PRED(3); break;
    case 4: PRED(4); break;
    default: PRED(5); break;
  }
#undef PRED
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int fused_complete(llg_ctx* c, int q, int qmax, const double* l, const double* acor, double* const* zn, bool save,
                   bool norms, double cquot, const double* w, int slot, bool store) {
  if (!store && !norms) return 0;
  if (q < 0 || q > 5 || qmax < q || qmax > 5) { llg_set_error("complete: bad order"); return LLG_ERR_ARG; }
  ZPack zp{};
  CPack lp{};
  for (int j = 0; j <= qmax; j++) zp.p[j] = zn[j];
  for (int j = 0; j <= q; j++) lp.c[j] = l[j];
  LLG_COUNT(KID_ELEMWISE);
  const int sv = save ? 1 : 0, nm = norms ? 1 : 0, st = store ? 1 : 0;
#define COMP(Q)                                                                                    \
  klaunch(k_complete_norms<Q>, red_blocks_resident(c->neq, LLG_PER_SM((k_complete_norms<Q>)), c->num_sms), RT, 0, \
          c->stream, qmax, lp, acor, zp, zn[qmax], sv, nm, -cquot,                                                   \
                                                                w, c->neq, c->d_red, c->d_counter,             \
                                                                c->d_scal + slot, st)
  switch (q) {
    case 0: COMP(0); break;
    case 1: COMP(1); break;
    case 2: COMP(2); break;
    case 3: COMP(3); break;
    case 4: COMP(4); break;
    default: COMP(5); break;
  }
#undef COMP
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
