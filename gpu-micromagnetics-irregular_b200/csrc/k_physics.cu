// k_physics.cu — per-cell LLG operators for sm_100a.
//
// Reference formulas (restated, one source of truth in DevProblem):
//   normalise   2d_i2/2d_fft.cu:262-282 (m/(|m|+eps)), 2d_i1/2d_fft.cu:253-275 (m/|m|)
//   RHS         2d_i2/2d_fft.cu:300-357 (+happ 2d_i4/2d_fft.cu:309-311,
//               linear+DMI 2d_i1/2d_fft.cu:344-367, windowed 2d_i3/2d_fft.cu:451-627,
//               compact 2d_i6/2d_i6.cu:250-343)
//   Jv          2d_i2/jtv.cu:49-122, 2d_i1/jtv.cu:43-96, 2d_i6/jtv.cu:47-130
//   P setup     2d_i2/precond.cu:119-251      P solve 2d_i2/precond.cu:254-285
//
// B200 mapping.  Every stencil kernel works on a 32x8 cell tile: the 3 (or 6)
// SoA components of the tile plus a one-cell halo are staged in shared memory
// with coalesced 256-byte row loads (boundary rule applied per slot: wrap or
// zero), so each input byte is fetched from HBM once per tile instead of five
// times per cell.  The grids are sized from the problem (ceil(ng/32) x
// ceil(ny/8) CTAs of 256 threads); at 1536x512 that is 3072 CTAs, ~21 waves
// of 148 SMs.  Compact (EXEC_COMPACT) kernels launch one thread per listed
// cell and read neighbours through L1.
//
// Preconditioner.  psetup stores the frozen cell state (m, h) and the 3x3
// block inverse (I - gamma_setup J)^-1 of every cell (9 planes, 72 B/cell),
// as the reference keeps its P^-1 array.  The Arnoldi operator reads the
// inverse: rebuilding it costs ~230 FP64 operations per cell, about half of
// that kernel's arithmetic, which bounds it once its loads are pipelined.
// psolve, a plain stream at HBM speed, rebuilds the block from (m, h) in
// registers instead (48 B/cell read rather than 72); both forms give the same
// bits (the same block_inverse on the same inputs).
#include <math.h>

#include <algorithm>

#include <map>
#include <mutex>
#include <tuple>

#include "llg_internal.h"
#include "launch.h"
#include "dev_physics.cuh"

namespace {

// ── kernels ────────────────────────────────────────────────────────────
__global__ void k_normalize(double* __restrict__ y, int n, int kind, double eps) {
  pdl_entry();
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double m1 = y[k], m2 = y[n + k], m3 = y[2 * n + k];
    const double ymp = sqrt(m1 * m1 + m2 * m2 + m3 * m3);
    if (kind == LLG_NORM_REG) {
      const double inv = 1.0 / (ymp + eps);
      y[k] = m1 * inv; y[n + k] = m2 * inv; y[2 * n + k] = m3 * inv;
    } else if (ymp > 1.0e-30) {
      const double inv = 1.0 / ymp;
      y[k] = m1 * inv; y[n + k] = m2 * inv; y[2 * n + k] = m3 * inv;
    }
  }
}

__global__ void __launch_bounds__(TX * TY) k_rhs_tile(DevProblem P, const double* __restrict__ y,
                                                      const double* __restrict__ hd,
                                                      double* __restrict__ ydot) {
  pdl_entry();
  __shared__ Tile<1> T;
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
  ydot[cell] = o[0]; ydot[n + cell] = o[1]; ydot[2 * n + cell] = o[2];
}

__global__ void k_rhs_compact(DevProblem P, const double* __restrict__ y, const double* __restrict__ hd,
                              double* __restrict__ ydot, const int32_t* __restrict__ act_ids, int na,
                              const int32_t* __restrict__ inact_ids, int ni) {
  pdl_entry();
  const int n = P.ncell;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na + ni; t += gridDim.x * blockDim.x) {
    if (t >= na) {
      const int cell = inact_ids[t - na];
      ydot[cell] = 0.0; ydot[n + cell] = 0.0; ydot[2 * n + cell] = 0.0;
      continue;
    }
    const int cell = act_ids[t];
    const int gi = cell % P.ng, gj = cell / P.ng;
    const double m[3] = {y[cell], y[n + cell], y[2 * n + cell]};
    double msk[3], nsk[3];
    cell_axes(P, cell, msk, nsk);
    double h[3];
    gather_field(P, y, gi, gj, m, msk, nsk, h);
#pragma unroll
    for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + happ_at(P, a, gi);
    double o[3];
    llg_torque(P, alpha_at(P, gi), m, h, 1.0, o);
    ydot[cell] = o[0]; ydot[n + cell] = o[1]; ydot[2 * n + cell] = o[2];
  }
}

__global__ void __launch_bounds__(TX * TY) k_jtv_tile(DevProblem P, const double* __restrict__ v,
                                                      double* __restrict__ Jv, const double* __restrict__ y,
                                                      const double* __restrict__ hd) {
  pdl_entry();
  __shared__ Tile<2> T;
  const double* f[2] = {y, v};
  load_tile<2>(P, T, f);
  const int gi = blockIdx.x * TX + threadIdx.x, gj = blockIdx.y * TY + threadIdx.y;
  if (gi >= P.ng || gj >= P.ny) return;
  const int n = P.ncell, cell = gj * P.ng + gi;
  const int sx = threadIdx.x + 1, sy = threadIdx.y + 1;
  const double m[3] = {y[cell], y[n + cell], y[2 * n + cell]};
  const double vv[3] = {v[cell], v[n + cell], v[2 * n + cell]};
  double msk[3], nsk[3];
  cell_axes(P, cell, msk, nsk);
  double h[3];
  tile_field(P, T.v[0], sx, sy, m, msk, nsk, h);
  if (P.jv_full) {
#pragma unroll
    for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + happ_at(P, a, gi);
  }
  double K[3][3];
  aniso_jac(P, m, msk, K);
  double dh[3];
#pragma unroll
  for (int a = 0; a < 3; a++)
    dh_from(P, T.v[1][a][sy][sx - 1], T.v[1][a][sy][sx + 1], T.v[1][a][sy - 1][sx], T.v[1][a][sy + 1][sx], a, K,
            vv, nsk, dh[a]);
  if (P.jv_hv) {
#pragma unroll
    for (int a = 0; a < 3; a++) dh[a] = dh[a] + P.jv_hv[a * n + cell];
  }
  double o[3];
  jv_cell(P, m, vv, h, dh, gate_of(P, cell), o);
  Jv[cell] = o[0]; Jv[n + cell] = o[1]; Jv[2 * n + cell] = o[2];
}

__global__ void k_jtv_compact(DevProblem P, const double* __restrict__ v, double* __restrict__ Jv,
                              const double* __restrict__ y, const double* __restrict__ hd,
                              const int32_t* __restrict__ act_ids, int na, const int32_t* __restrict__ inact_ids,
                              int ni) {
  pdl_entry();
  const int n = P.ncell;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na + ni; t += gridDim.x * blockDim.x) {
    if (t >= na) {
      const int cell = inact_ids[t - na];
      Jv[cell] = 0.0; Jv[n + cell] = 0.0; Jv[2 * n + cell] = 0.0;
      continue;
    }
    const int cell = act_ids[t];
    const int gi = cell % P.ng, gj = cell / P.ng;
    const double m[3] = {y[cell], y[n + cell], y[2 * n + cell]};
    const double vv[3] = {v[cell], v[n + cell], v[2 * n + cell]};
    double msk[3], nsk[3];
    cell_axes(P, cell, msk, nsk);
    double h[3];
    gather_field(P, y, gi, gj, m, msk, nsk, h);
    if (P.jv_full) {
#pragma unroll
      for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + happ_at(P, a, gi);
    }
    double K[3][3];
    aniso_jac(P, m, msk, K);
    double dh[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
      dh_from(P, gather_nb(P, v, a, gi - 1, gj), gather_nb(P, v, a, gi + 1, gj), gather_nb(P, v, a, gi, gj - 1),
              gather_nb(P, v, a, gi, gj + 1), a, K, vv, nsk, dh[a]);
    if (P.jv_hv) {
#pragma unroll
      for (int a = 0; a < 3; a++) dh[a] = dh[a] + P.jv_hv[a * n + cell];
    }
    double o[3];
    jv_cell(P, m, vv, h, dh, 1.0, o);
    Jv[cell] = o[0]; Jv[n + cell] = o[1]; Jv[2 * n + cell] = o[2];
  }
}

// psetup: freeze (m, h_total) per cell
__global__ void __launch_bounds__(TX * TY) k_psetup_tile(DevProblem P, const double* __restrict__ y,
                                                         const double* __restrict__ hd, double* __restrict__ pm,
                                                         double* __restrict__ ph, double* __restrict__ pinv,
                                                         double gamma, const DevArgs* da, int pinv_f32) {
  pdl_entry();
  if (da && !da->run_setup) return;
  if (da) gamma = da->gamma_setup;
  __shared__ Tile<1> T;
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
  for (int a = 0; a < 3; a++) {
    h[a] = h[a] + hd[a * n + cell] + happ_at(P, a, gi);
    pm[a * n + cell] = m[a];
    ph[a * n + cell] = h[a];
  }
  const double ws = P.windowed ? P.w[cell] : 1.0;
  double Pi[9];
  block_inverse(P, m, h, msk, ws, gamma, Pi);
  if (pinv_f32) {
    float* pf = reinterpret_cast<float*>(pinv);
#pragma unroll
    for (int k = 0; k < 9; k++) pf[(long long)k * n + cell] = (float)Pi[k];
  } else {
#pragma unroll
    for (int k = 0; k < 9; k++) pinv[(long long)k * n + cell] = Pi[k];
  }
}


__global__ void k_psolve(DevProblem P, const double* __restrict__ pm, const double* __restrict__ ph,
                         const double* __restrict__ r, double* __restrict__ z, double gamma, const DevArgs* da) {
  pdl_entry();
  const int n = P.ncell;
  if (da) gamma = da->gamma_setup;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const double m[3] = {pm[k], pm[n + k], pm[2 * n + k]};
    const double h[3] = {ph[k], ph[n + k], ph[2 * n + k]};
    const double rr[3] = {r[k], r[n + k], r[2 * n + k]};
    double msk[3], nsk[3];
    cell_axes(P, k, msk, nsk);
    const double ws = P.windowed ? P.w[k] : 1.0;
    double Pi[9];
    block_inverse(P, m, h, msk, ws, gamma, Pi);
    double g = 1.0;
    if (!P.windowed && P.act) g = P.act[k] ? 1.0 : 0.0;
    z[k] = g * (Pi[0] * rr[0] + Pi[1] * rr[1] + Pi[2] * rr[2]);
    z[n + k] = g * (Pi[3] * rr[0] + Pi[4] * rr[1] + Pi[5] * rr[2]);
    z[2 * n + k] = g * (Pi[6] * rr[0] + Pi[7] * rr[1] + Pi[8] * rr[2]);
  }
}

// Fused Arnoldi operator of left-preconditioned, ewt-scaled GMRES:
//   vt = in / s ;  u = vt − γ J(y) vt ;  out = s ⊙ P^-1 u
// One pass: reads in (stencil), s (stencil), y (stencil), pm/ph, writes out.
template <typename VT = double>
__global__ void __launch_bounds__(TX * TY, 4) k_arnoldi_tile(DevProblem P, const VT* __restrict__ in,
                                                          const double* __restrict__ s,
                                                          VT* __restrict__ out, const double* __restrict__ y,
                                                          const double* __restrict__ hd,
                                                          const VT* __restrict__ pinv, double gamma,
                                                          int scale_out, const DevArgs* da, const double* in_a) {
  pdl_entry();
  __shared__ Tile<2> T;
  if constexpr (sizeof(VT) == sizeof(double)) {
    if (da) {
      in = da->arn_in;
      out = da->arn_out;
      gamma = da->gamma;
    }
  }
  const double ain = kscale_of(in_a);   // the input is read as ain * in
  // stage y and vt = in/s (windowed: w·) with halo
  {
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int tid = threadIdx.y * TX + threadIdx.x;
    const int n = P.ncell;
    constexpr int ROWSLOTS = (TY + 2) * TX;
    constexpr int COLSLOTS = (TY + 2) * 2;
    for (int q = tid; q < ROWSLOTS + COLSLOTS; q += TX * TY) {
      int sx, sy;
      if (q < ROWSLOTS) { sy = q / TX; sx = 1 + (q % TX); }
      else { const int r2 = q - ROWSLOTS; sy = r2 >> 1; sx = (r2 & 1) ? (TX + 1) : 0; }
      int gi = x0 - 1 + sx, gj = y0 - 1 + sy;
      const bool ok = map_nb(gi, gj, P.ng, P.ny, P.bc);
      const int cell = gj * P.ng + gi;
      const double ww = (ok && P.windowed) ? P.w[cell] : 1.0;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        T.v[0][a][sy][sx] = ok ? ww * y[a * n + cell] : 0.0;
        T.v[1][a][sy][sx] = ok ? ww * ((ain * (double)in[a * n + cell]) / s[a * n + cell]) : 0.0;
      }
    }
    __syncthreads();
  }
  const int gi = blockIdx.x * TX + threadIdx.x, gj = blockIdx.y * TY + threadIdx.y;
  if (gi >= P.ng || gj >= P.ny) return;
  const int n = P.ncell, cell = gj * P.ng + gi;
  const int sx = threadIdx.x + 1, sy = threadIdx.y + 1;
  const double ss[3] = {s[cell], s[n + cell], s[2 * n + cell]};
  double m[3], vv[3];
  if (!P.windowed) {   // the staged centre holds y and in/s themselves (window 1)
#pragma unroll
    for (int a = 0; a < 3; a++) {
      m[a] = T.v[0][a][sy][sx];
      vv[a] = T.v[1][a][sy][sx];
    }
  } else {
#pragma unroll
    for (int a = 0; a < 3; a++) {
      m[a] = y[a * n + cell];
      vv[a] = (ain * (double)in[a * n + cell]) / ss[a];
    }
  }
  double msk[3], nsk[3];
  cell_axes(P, cell, msk, nsk);
  double h[3];
  tile_field(P, T.v[0], sx, sy, m, msk, nsk, h);
  if (P.jv_full) {
#pragma unroll
    for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + happ_at(P, a, gi);
  }
  double K[3][3];
  aniso_jac(P, m, msk, K);
  double dh[3];
#pragma unroll
  for (int a = 0; a < 3; a++)
    dh_from(P, T.v[1][a][sy][sx - 1], T.v[1][a][sy][sx + 1], T.v[1][a][sy - 1][sx], T.v[1][a][sy + 1][sx], a, K,
            vv, nsk, dh[a]);
  if (P.jv_hv) {
#pragma unroll
    for (int a = 0; a < 3; a++) dh[a] = dh[a] + P.jv_hv[a * n + cell];
  }
  const double g = gate_of(P, cell);
  double jv[3];
  jv_cell(P, m, vv, h, dh, g, jv);
  double u[3];
#pragma unroll
  for (int a = 0; a < 3; a++) u[a] = 1.0 * vv[a] + (-gamma) * jv[a];
  double Pi[9];
  load_pinv(pinv, n, cell, Pi);
  double gz = 1.0;
  if (!P.windowed && P.act) gz = P.act[cell] ? 1.0 : 0.0;
  const double z0 = gz * (Pi[0] * u[0] + Pi[1] * u[1] + Pi[2] * u[2]);
  const double z1 = gz * (Pi[3] * u[0] + Pi[4] * u[1] + Pi[5] * u[2]);
  const double z2 = gz * (Pi[6] * u[0] + Pi[7] * u[1] + Pi[8] * u[2]);
  if (scale_out) {
    out[cell] = (VT)(ss[0] * z0);
    out[n + cell] = (VT)(ss[1] * z1);
    out[2 * n + cell] = (VT)(ss[2] * z2);
  } else {  // block-Jacobi output for a further preconditioning stage
    out[cell] = (VT)z0;
    out[n + cell] = (VT)z1;
    out[2 * n + cell] = (VT)z2;
  }
}

// ── persistent, double-buffered Arnoldi operator (unwindowed problems) ──
// The same per-cell arithmetic as k_arnoldi_tile.  Each CTA walks tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... and, while it computes one tile,
// cp.async streams the next tile's inputs into the other shared-memory
// buffer: the y, in and s stencils (tile + one-cell halo, zero outside a
// free edge, wrapped on a periodic one) and, when the Jacobian uses the full
// field, the demag field of the centre cells.  The HBM reads of one tile
// therefore overlap the FP64 work of the previous one instead of alternating
// with it.  The gate of a cell is read ahead of the stencil wait, its stored
// block inverse ahead of the stencil arithmetic.
constexpr int AP_SLOTS = (TY + 2) * TX + (TY + 2) * 2;   // staged stencil slots per component
constexpr int AP_PLANE = (TY + 2) * (TX + 2);            // doubles per stencil component
constexpr int AP_CELLS = TX * TY;
constexpr int AP_NT = TX * TY;
__host__ __device__ constexpr int ap_buf_doubles(int jv_full, int f32 = 0) {
  // (an FP32 basis stages its input in a float plane after the doubles)
  return 9 * AP_PLANE + (jv_full ? 3 : 0) * AP_CELLS + (f32 ? (3 * AP_PLANE + 1) / 2 : 0);
}

__device__ __forceinline__ void cp_async8(void* dst, const void* src, bool ok) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  const int sz = ok ? 8 : 0;   // 0: zero-fill, nothing read
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src, bool ok) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  const int sz = ok ? 4 : 0;   // 0: zero-fill, nothing read
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ void ap_slot(int q, int& sx, int& sy) {
  if (q < (TY + 2) * TX) { sy = q / TX; sx = 1 + (q % TX); }
  else { const int r2 = q - (TY + 2) * TX; sy = r2 >> 1; sx = (r2 & 1) ? (TX + 1) : 0; }
}

template <typename VT = double>
__global__ void __launch_bounds__(AP_NT, 3) k_arnoldi_pipe(DevProblem P, const VT* __restrict__ in,
                                                           const double* __restrict__ s,
                                                           VT* __restrict__ out, const double* __restrict__ y,
                                                           const double* __restrict__ hd,
                                                           const VT* __restrict__ pinv, double gamma,
                                                           int scale_out, const DevArgs* da, const double* in_a) {
  pdl_entry();
  extern __shared__ __align__(16) double apsm[];
  constexpr bool F32 = sizeof(VT) != sizeof(double);
  if constexpr (!F32) {
    if (da) {
      in = da->arn_in;
      out = da->arn_out;
      gamma = da->gamma;
    }
  }
  const double ain = kscale_of(in_a);   // the input is read as ain * in
  const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
  const int n = P.ncell, ng = P.ng, ny = P.ny;
  const int gx = (ng + TX - 1) / TX, ntiles = gx * ((ny + TY - 1) / TY);
  const int bufd = ap_buf_doubles(P.jv_full, F32 ? 1 : 0);
  const int foff = ap_buf_doubles(P.jv_full);   // the float staging plane (FP32 basis)
  typedef double Plane[TY + 2][TX + 2];
  typedef float FPlane[TY + 2][TX + 2];

  auto issue = [&](int t, double* B) {
    const int x0 = (t % gx) * TX, y0 = (t / gx) * TY;
    Plane* Y = reinterpret_cast<Plane*>(B);
    Plane* V = Y + 3;
    Plane* S = Y + 6;
    for (int q = tid; q < AP_SLOTS; q += AP_NT) {
      int sx, sy;
      ap_slot(q, sx, sy);
      int gi = x0 - 1 + sx, gj = y0 - 1 + sy;
      const bool ok = map_nb(gi, gj, ng, ny, P.bc);
      const long long cell = ok ? (long long)gj * ng + gi : 0;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        cp_async8(&Y[a][sy][sx], y + a * (long long)n + cell, ok);
        if constexpr (F32) {
          FPlane* Fv = reinterpret_cast<FPlane*>(B + foff);
          cp_async4(&Fv[a][sy][sx], in + a * (long long)n + cell, ok);
        } else {
          cp_async8(&V[a][sy][sx], in + a * (long long)n + cell, ok);
        }
        cp_async8(&S[a][sy][sx], s + a * (long long)n + cell, ok);
      }
    }
    if (P.jv_full) {
      double* C = B + 9 * AP_PLANE;
      const int cx = x0 + tx, cy = y0 + ty;
      const bool cok = cx < ng && cy < ny;
      const long long cell = cok ? (long long)cy * ng + cx : 0;
#pragma unroll
      for (int a = 0; a < 3; a++) cp_async8(&C[a * AP_CELLS + tid], hd + a * (long long)n + cell, cok);
    }
  };

  int t = blockIdx.x, b = 0;
  if (t < ntiles) issue(t, apsm);
  cp_async_commit();
  for (; t < ntiles; t += gridDim.x, b ^= 1) {
    double* B = apsm + b * bufd;
    const int tn = t + gridDim.x;
    if (tn < ntiles) issue(tn, apsm + (b ^ 1) * bufd);
    cp_async_commit();
    const int x0 = (t % gx) * TX, y0 = (t / gx) * TY;
    const int gi = x0 + tx, gj = y0 + ty;
    const bool cok = gi < ng && gj < ny;
    const int cell = gj * ng + gi;
    const double g = (cok && P.act) ? (P.act[cell] ? 1.0 : 0.0) : 1.0;   // gate, loaded while the tile lands
    cp_async_wait1();
    __syncthreads();
    Plane* Y = reinterpret_cast<Plane*>(B);
    Plane* V = Y + 3;
    Plane* S = Y + 6;
    // vt = (ain in) / s on every staged slot (0 outside a free edge)
    for (int q = tid; q < AP_SLOTS; q += AP_NT) {
      int sx, sy;
      ap_slot(q, sx, sy);
      int ii = x0 - 1 + sx, jj = y0 - 1 + sy;
      const bool ok = map_nb(ii, jj, ng, ny, P.bc);
      if constexpr (F32) {
        const FPlane* Fv = reinterpret_cast<const FPlane*>(B + foff);
#pragma unroll
        for (int a = 0; a < 3; a++)
          V[a][sy][sx] = ok ? 1.0 * ((ain * (double)Fv[a][sy][sx]) / S[a][sy][sx]) : 0.0;
      } else {
#pragma unroll
        for (int a = 0; a < 3; a++) V[a][sy][sx] = ok ? 1.0 * ((ain * V[a][sy][sx]) / S[a][sy][sx]) : 0.0;
      }
    }
    __syncthreads();
    if (cok) {
      double Pi[9];
      load_pinv(pinv, n, cell, Pi);   // first use after the stencil arithmetic below
      const double* C = B + 9 * AP_PLANE;
      const int sx = tx + 1, sy = ty + 1;
      double m[3], vv[3], ss[3];
#pragma unroll
      for (int a = 0; a < 3; a++) {
        m[a] = Y[a][sy][sx];
        vv[a] = V[a][sy][sx];
        ss[a] = S[a][sy][sx];
      }
      double msk[3], nsk[3];
      cell_axes(P, cell, msk, nsk);
      double h[3];
      tile_field(P, Y, sx, sy, m, msk, nsk, h);
      if (P.jv_full) {
#pragma unroll
        for (int a = 0; a < 3; a++) h[a] = h[a] + C[a * AP_CELLS + tid] + happ_at(P, a, P.src_on ? gi : -1);
      }
      double K[3][3];
      aniso_jac(P, m, msk, K);
      double dh[3];
#pragma unroll
      for (int a = 0; a < 3; a++)
        dh_from(P, V[a][sy][sx - 1], V[a][sy][sx + 1], V[a][sy - 1][sx], V[a][sy + 1][sx], a, K, vv, nsk, dh[a]);
      if (P.jv_hv) {
#pragma unroll
        for (int a = 0; a < 3; a++) dh[a] = dh[a] + P.jv_hv[a * (long long)n + cell];
      }
      double jv[3];
      jv_cell(P, m, vv, h, dh, g, jv);
      double u[3];
#pragma unroll
      for (int a = 0; a < 3; a++) u[a] = 1.0 * vv[a] + (-gamma) * jv[a];
      const double z0 = g * (Pi[0] * u[0] + Pi[1] * u[1] + Pi[2] * u[2]);
      const double z1 = g * (Pi[3] * u[0] + Pi[4] * u[1] + Pi[5] * u[2]);
      const double z2 = g * (Pi[6] * u[0] + Pi[7] * u[1] + Pi[8] * u[2]);
      if (scale_out) {
        out[cell] = (VT)(ss[0] * z0);
        out[n + cell] = (VT)(ss[1] * z1);
        out[2 * n + cell] = (VT)(ss[2] * z2);
      } else {
        out[cell] = (VT)z0;
        out[n + cell] = (VT)z1;
        out[2 * n + cell] = (VT)z2;
      }
    }
    __syncthreads();   // buffer b is refilled by the next iteration's issue
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");   // (only empty groups remain)
}

// the Arnoldi operator's input vt = (a in) / s, for the demag derivative of
// LLG_JV_FULL_DEMAG (the same arithmetic as the operator's staging)
template <typename VT = double>
__global__ void k_arnoldi_input(const VT* __restrict__ in, const double* __restrict__ s, const double* in_a,
                                double* __restrict__ vt, long long n3) {
  pdl_entry();
  const double ain = kscale_of(in_a);
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n3; i += (long long)gridDim.x * blockDim.x)
    vt[i] = 1.0 * ((ain * (double)in[i]) / s[i]);
}

int grid_1d(const llg_ctx* c, long long work, int block) {
  long long g = (work + block - 1) / block;
  const long long cap = (long long)c->num_sms * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

int launch_normalize(llg_ctx* c, double* y) {
  if (c->p.norm_kind == LLG_NORM_NONE) return 0;
  LLG_COUNT(KID_NORM);
  klaunch(k_normalize, grid_1d(c, c->ncell, 256), 256, 0, c->stream, y, c->ncell, c->p.norm_kind, c->p.norm_eps);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

static dim3 tile_grid(const llg_ctx* c) { return dim3((c->p.ng + TX - 1) / TX, (c->p.ny + TY - 1) / TY); }

int launch_rhs(llg_ctx* c, const double* y, const double* hd, double* ydot) {
  if (c->p.exec_model == LLG_EXEC_COMPACT) {
    const int tot = c->n_active + c->n_inactive;
    LLG_COUNT(KID_RHS);
    klaunch(k_rhs_compact, grid_1d(c, tot, 256), 256, 0, c->stream, c->dp, y, hd, ydot, c->d_active_ids, c->n_active,
                                                               c->d_inactive_ids, c->n_inactive);
  } else {
    LLG_COUNT(KID_RHS);
    klaunch(k_rhs_tile, tile_grid(c), dim3(TX, TY), 0, c->stream, c->dp, y, hd, ydot);
  }
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int launch_jtv(llg_ctx* c, const double* v, double* Jv, const double* y) {
  DevProblem P = c->dp;
  if (c->d_hv) {   // LLG_JV_FULL_DEMAG: the demag field of v enters the field derivative
    const int rc = demag_apply(c, v, c->d_hv);
    if (rc) return rc;
    P.jv_hv = c->d_hv;
  }
  if (c->p.exec_model == LLG_EXEC_COMPACT) {
    const int tot = c->n_active + c->n_inactive;
    LLG_COUNT(KID_JTV);
    klaunch(k_jtv_compact, grid_1d(c, tot, 256), 256, 0, c->stream, P, v, Jv, y, c->d_hd, c->d_active_ids,
                                                               c->n_active, c->d_inactive_ids, c->n_inactive);
  } else {
    LLG_COUNT(KID_JTV);
    klaunch(k_jtv_tile, tile_grid(c), dim3(TX, TY), 0, c->stream, P, v, Jv, y, c->d_hd);
  }
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int launch_psetup(llg_ctx* c, const double* y, double gamma, const DevArgs* da) {
  LLG_COUNT(KID_PSETUP);
  klaunch(k_psetup_tile, tile_grid(c), dim3(TX, TY), 0, c->stream, c->dp, y, c->d_hd, c->d_pm, c->d_ph, c->d_pinv,
          gamma, da, c->pinv_f32);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  c->gamma_setup = gamma;
  c->have_setup = 1;
  return 0;
}

int launch_psolve(llg_ctx* c, const double* r, double* z, const DevArgs* da) {
  if (!c->have_setup && !da) { llg_set_error("psolve before psetup"); return LLG_ERR_STATE; }
  LLG_COUNT(KID_PSOLVE);
  klaunch(k_psolve, grid_1d(c, c->ncell, 256), 256, 0, c->stream, c->dp, c->d_pm, c->d_ph, r, z, c->gamma_setup, da);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int arnoldi_setup(llg_ctx* c) {
  const size_t smax = 2 * sizeof(double) * ap_buf_doubles(1);
  const size_t smaxf = 2 * sizeof(double) * ap_buf_doubles(1, 1);
  if (cudaFuncSetAttribute((const void*)k_arnoldi_pipe<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smax) != cudaSuccess ||
      cudaFuncSetAttribute((const void*)k_arnoldi_pipe<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smaxf) != cudaSuccess) {
    llg_set_error("arnoldi operator: shared-memory opt-in failed");
    return LLG_ERR_CUDA;
  }
  const long long ntiles = (long long)((c->p.ng + TX - 1) / TX) * ((c->p.ny + TY - 1) / TY);
  for (int jf = 0; jf < 2; jf++) {
    int per_sm = 0, per_sm_f = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_arnoldi_pipe<double>, AP_NT,
                                                      2 * sizeof(double) * ap_buf_doubles(jf)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_f, k_arnoldi_pipe<float>, AP_NT,
                                                      2 * sizeof(double) * ap_buf_doubles(jf, 1)) != cudaSuccess ||
        per_sm < 1 || per_sm_f < 1) {
      llg_set_error("arnoldi operator: occupancy query failed");
      return LLG_ERR_CUDA;
    }
    c->arn_grid[jf] = (int)std::min<long long>(ntiles, (long long)per_sm * c->num_sms);
    c->arn_grid_f[jf] = (int)std::min<long long>(ntiles, (long long)per_sm_f * c->num_sms);
  }
  return 0;
}

// Autotune of the persistent operator's grid: the first launch of a (grid
// size, staged field, basis precision) shape times the kernel at 1, 2, ...
// CTAs per SM up to the occupancy limit on the live buffers (each candidate
// twice, the second timing kept) and keeps the fastest, process-wide.  The
// grid does not change any cell's arithmetic; the candidates' outputs are
// overwritten by the launch that follows.
static std::mutex g_arn_mu;
static std::map<std::tuple<int, int, int, int>, int> g_arn_tuned;

template <typename VT>
static int arnoldi_tune(llg_ctx* c, const DevProblem& P, int jf, const VT* in, const double* ewt, VT* out,
                        const double* y, double gamma, int scale_out, const double* in_a, int* grid) {
  constexpr int f32 = sizeof(VT) != sizeof(double) ? 1 : 0;
  const auto key = std::make_tuple(c->p.ng, c->p.ny, jf, f32);
  {
    std::lock_guard<std::mutex> g(g_arn_mu);
    auto it = g_arn_tuned.find(key);
    if (it != g_arn_tuned.end()) { *grid = it->second; return 0; }
  }
  const long long ntiles = (long long)((c->p.ng + TX - 1) / TX) * ((c->p.ny + TY - 1) / TY);
  const int gmax = *grid;
  const size_t smem = 2 * sizeof(double) * ap_buf_doubles(jf, f32);
  cudaEvent_t e0, e1;
  LLG_CUDA_TRY(cudaEventCreate(&e0));
  LLG_CUDA_TRY(cudaEventCreate(&e1));
  int best = gmax;
  float best_ms = 1e30f;
  for (int per = 1; per * c->num_sms <= gmax + c->num_sms - 1; per++) {
    const int gsz = (int)std::min<long long>({ntiles, (long long)per * c->num_sms, (long long)gmax});
    float ms = 0.f;
    for (int rep = 0; rep < 2; rep++) {
      cudaEventRecord(e0, c->stream);
      k_arnoldi_pipe<VT><<<gsz, AP_NT, smem, c->stream>>>(P, in, ewt, out, y, c->d_hd,
                                                          reinterpret_cast<const VT*>(c->d_pinv), gamma, scale_out,
                                                          nullptr, in_a);
      cudaEventRecord(e1, c->stream);
    }
    if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      LLG_CUDA_TRY(cudaGetLastError());
      return LLG_ERR_CUDA;
    }
    if (ms < best_ms) { best_ms = ms; best = gsz; }
    if (gsz >= gmax) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  pdl_break();
  *grid = best;
  std::lock_guard<std::mutex> g(g_arn_mu);
  g_arn_tuned[key] = best;
  return 0;
}

template <typename VT>
static int arnoldi_op_impl(llg_ctx* c, const VT* in, const double* ewt, VT* out, const double* y, double gamma,
                           int scale_out, const DevArgs* da, const double* in_a) {
  if (!c->have_setup && !da) { llg_set_error("arnoldi operator before psetup"); return LLG_ERR_STATE; }
  DevProblem P = c->dp;
  if (c->d_hv) {   // LLG_JV_FULL_DEMAG: demag field of the operator's input vt = (a in) / s
    if (da) { llg_set_error("the demag-derivative Jacobian runs on the host-driven integrator"); return LLG_ERR_NOTSUP; }
    LLG_COUNT(KID_ELEMWISE);
    klaunch(k_arnoldi_input<VT>, grid_1d(c, c->neq, 256), 256, 0, c->stream, in, ewt, in_a, c->d_vt,
            (long long)c->neq);
    LLG_CUDA_TRY(cudaPeekAtLastError());
    const int rc = demag_apply(c, c->d_vt, c->d_hv);
    if (rc) return rc;
    P.jv_hv = c->d_hv;
  }
  constexpr int f32 = sizeof(VT) != sizeof(double) ? 1 : 0;
  if (f32 != c->pinv_f32) {
    llg_set_error("arnoldi operator: block inverse stored in the other precision (psetup first)");
    return LLG_ERR_STATE;
  }
  LLG_COUNT(KID_ARNOLDI);
  ktimer_mark(c, KID_ARNOLDI, true);
  if (c->dp.windowed) {
    klaunch(k_arnoldi_tile<VT>, tile_grid(c), dim3(TX, TY), 0, c->stream, P, in, ewt, out, y, c->d_hd,
            reinterpret_cast<const VT*>(c->d_pinv), gamma, scale_out, da, in_a);
  } else {
    const int jf = c->dp.jv_full ? 1 : 0;
    int& grid = f32 ? c->arn_grid_f[jf] : c->arn_grid[jf];
    if (!da && !c->capturing && !(f32 ? c->arn_tuned_f[jf] : c->arn_tuned[jf])) {
      const int rc = arnoldi_tune<VT>(c, P, jf, in, ewt, out, y, gamma, scale_out, in_a, &grid);
      if (rc) return rc;
      (f32 ? c->arn_tuned_f[jf] : c->arn_tuned[jf]) = 1;
    }
    klaunch(k_arnoldi_pipe<VT>, grid, AP_NT,
            2 * sizeof(double) * ap_buf_doubles(jf, f32), c->stream, P, in, ewt, out, y, c->d_hd,
            reinterpret_cast<const VT*>(c->d_pinv), gamma, scale_out, da, in_a);
  }
  ktimer_mark(c, KID_ARNOLDI, false);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int launch_arnoldi_op(llg_ctx* c, const double* in, const double* ewt, double* out, const double* y,
                      double gamma, int scale_out, const DevArgs* da, const double* in_a) {
  return arnoldi_op_impl<double>(c, in, ewt, out, y, gamma, scale_out, da, in_a);
}

int launch_arnoldi_op_f(llg_ctx* c, const float* in, const double* ewt, float* out, const double* y, double gamma,
                        const double* in_a) {
  return arnoldi_op_impl<float>(c, in, ewt, out, y, gamma, 1, nullptr, in_a);
}

int rhs_full(llg_ctx* c, double t, double* y, double* ydot) {
  set_source_time(c, t);
  int rc = launch_normalize(c, y);
  if (rc) return rc;
  if (c->demag) {   // (without demag the field buffer stays as cleared at creation)
    rc = demag_apply(c, y, c->d_hd);
    if (rc) return rc;
    c->nfe_demag++;
  }
  return launch_rhs(c, y, c->d_hd, ydot);
}
