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
// Preconditioner.  psetup stores the frozen cell state (m, h) — 48 B/cell —
// instead of the 72 B/cell inverse; psolve rebuilds the 3x3 block and its
// adjugate inverse in registers.  The FP64 work (~200 flop/cell) hides under
// the memory time, so each psolve moves 96 B/cell instead of 120 B/cell.
#include <math.h>

#include "llg_internal.h"

namespace {

constexpr int TX = 32;
constexpr int TY = 8;

// Logical slot -> grid cell.  Tile slots can lie up to a tile width past the
// edge (grids narrower than a tile), so the periodic wrap is a full modulo.
__device__ __forceinline__ bool map_nb(int& i, int& j, int ng, int ny, int bc) {
  if (bc == LLG_BC_FREE) return (i >= 0 && i < ng && j >= 0 && j < ny);
  i %= ng;
  if (i < 0) i += ng;
  j %= ny;
  if (j < 0) j += ny;
  return true;
}

__device__ __forceinline__ double gate_of(const DevProblem& P, int cell) {
  if (P.windowed) return P.w[cell];
  if (P.act) return P.act[cell] ? 1.0 : 0.0;
  return 1.0;
}

__device__ __forceinline__ void cell_axes(const DevProblem& P, int cell, double msk[3], double nsk[3]) {
  if (P.windowed) {
    const int n = P.ncell;
    msk[0] = P.msk3[cell]; msk[1] = P.msk3[n + cell]; msk[2] = P.msk3[2 * n + cell];
    nsk[0] = P.nsk3[cell]; nsk[1] = P.nsk3[n + cell]; nsk[2] = P.nsk3[2 * n + cell];
  } else {
    msk[0] = P.msk[0]; msk[1] = P.msk[1]; msk[2] = P.msk[2];
    nsk[0] = P.nsk[0]; nsk[1] = P.nsk[1]; nsk[2] = P.nsk[2];
  }
}

__device__ __forceinline__ void aniso_field(const DevProblem& P, const double m[3], const double msk[3],
                                            double an[3]) {
  if (P.aniso == LLG_ANISO_CUBIC) {
#pragma unroll
    for (int a = 0; a < 3; a++) an[a] = msk[a] * P.chk * m[a] * (m[a] * m[a] - 1.0);
  } else {
    const double md = m[0] * msk[0] + m[1] * msk[1] + m[2] * msk[2];
    const double fac = P.chk * md + P.cha;
#pragma unroll
    for (int a = 0; a < 3; a++) an[a] = msk[a] * fac;
  }
}

// symmetric local dh/dm of the anisotropy (+ window-scaled demag self term)
__device__ __forceinline__ void aniso_jac(const DevProblem& P, const double m[3], const double msk[3],
                                          double K[3][3]) {
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int b = 0; b < 3; b++) K[a][b] = 0.0;
  if (P.aniso == LLG_ANISO_CUBIC) {
#pragma unroll
    for (int a = 0; a < 3; a++) K[a][a] = msk[a] * P.chk * (3.0 * m[a] * m[a] - 1.0);
  } else {
#pragma unroll
    for (int a = 0; a < 3; a++)
#pragma unroll
      for (int b = 0; b < 3; b++) K[a][b] = P.chk * msk[a] * msk[b];
  }
}

__device__ __forceinline__ void llg_torque(const DevProblem& P, const double m[3], const double h[3],
                                           double g, double out[3]) {
  const double m1 = m[0], m2 = m[1], m3 = m[2], h1 = h[0], h2 = h[1], h3 = h[2];
  const double mh = m1 * h1 + m2 * h2 + m3 * h3;
  out[0] = g * (P.chg * (m3 * h2 - m2 * h3) + P.alpha * (h1 - mh * m1));
  out[1] = g * (P.chg * (m1 * h3 - m3 * h1) + P.alpha * (h2 - mh * m2));
  out[2] = g * (P.chg * (m2 * h1 - m1 * h2) + P.alpha * (h3 - mh * m3));
}

// (I - gamma*ws*J)^-1 at frozen (m, h); closed form of 2d_i2/precond.cu:186-250
__device__ __forceinline__ void block_inverse(const DevProblem& P, const double m[3], const double h[3],
                                              const double msk[3], double ws, double gamma, double Pi[9]) {
  double K[3][3];
  aniso_jac(P, m, msk, K);
#pragma unroll
  for (int a = 0; a < 3; a++) K[a][a] += ws * P.n0[a];
  const double mh = m[0] * h[0] + m[1] * h[1] + m[2] * h[2];
  double e[3];
#pragma unroll
  for (int b = 0; b < 3; b++) e[b] = h[b] + (K[b][0] * m[0] + K[b][1] * m[1] + K[b][2] * m[2]);
  double A[3][3];
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const double kb0 = K[0][b], kb1 = K[1][b], kb2 = K[2][b];
    const double kxm[3] = {kb1 * m[2] - kb2 * m[1], kb2 * m[0] - kb0 * m[2], kb0 * m[1] - kb1 * m[0]};
    double hxe[3] = {0.0, 0.0, 0.0};
    if (b == 0) { hxe[1] = h[2]; hxe[2] = -h[1]; }
    if (b == 1) { hxe[0] = -h[2]; hxe[2] = h[0]; }
    if (b == 2) { hxe[0] = h[1]; hxe[1] = -h[0]; }
    const double kb[3] = {kb0, kb1, kb2};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const double dm = P.alpha * (kb[a] - e[b] * m[a] - (a == b ? mh : 0.0));
      const double J = ws * (P.chg * (kxm[a] + hxe[a]) + dm);
      A[a][b] = (a == b ? 1.0 : 0.0) - gamma * J;
    }
  }
  const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
  const double c10 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
  const double c20 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
  const double det = A[0][0] * c00 + A[0][1] * c10 + A[0][2] * c20;
  if (!(fabs(det) > 1e-30)) {
#pragma unroll
    for (int k = 0; k < 9; k++) Pi[k] = (k % 4 == 0) ? 1.0 : 0.0;
    return;
  }
  const double id = 1.0 / det;
  Pi[0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id;
  Pi[1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
  Pi[2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
  Pi[3] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * id;
  Pi[4] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
  Pi[5] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
  Pi[6] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id;
  Pi[7] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
  Pi[8] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
}

// ── shared-memory tile of NF SoA fields (3 comps each) with 1-cell halo ──
template <int NF>
struct Tile {
  double v[NF][3][TY + 2][TX + 2];
};

// Stage fields f[k] (windowed: w·f) of the tile into shared memory.
// Slot (sx, sy) holds logical cell (x0-1+sx, y0-1+sy) with the boundary rule.
template <int NF>
__device__ __forceinline__ void load_tile(const DevProblem& P, Tile<NF>& T, const double* const* f) {
  const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
  const int tid = threadIdx.y * TX + threadIdx.x;
  const int n = P.ncell;
  // interior + halo rows: (TY+2) rows of TX slots; halo cols: (TY+2) x 2 slots
  constexpr int ROWSLOTS = (TY + 2) * TX;
  constexpr int COLSLOTS = (TY + 2) * 2;
  for (int s = tid; s < ROWSLOTS + COLSLOTS; s += TX * TY) {
    int sx, sy;
    if (s < ROWSLOTS) { sy = s / TX; sx = 1 + (s % TX); }
    else { const int q = s - ROWSLOTS; sy = q >> 1; sx = (q & 1) ? (TX + 1) : 0; }
    int gi = x0 - 1 + sx, gj = y0 - 1 + sy;
    const bool ok = map_nb(gi, gj, P.ng, P.ny, P.bc);
    const int cell = gj * P.ng + gi;
    const double ww = (ok && P.windowed) ? P.w[cell] : 1.0;
#pragma unroll
    for (int k = 0; k < NF; k++) {
#pragma unroll
      for (int a = 0; a < 3; a++) T.v[k][a][sy][sx] = ok ? ww * f[k][a * n + cell] : 0.0;
    }
  }
  __syncthreads();
}

// ── kernels ────────────────────────────────────────────────────────────
__global__ void k_normalize(double* __restrict__ y, int n, int kind, double eps) {
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

// field at a tile cell from the staged neighbours (exchange + aniso + DMI)
__device__ __forceinline__ void tile_field(const DevProblem& P, const double (*F)[TY + 2][TX + 2],
                                           int sx, int sy, const double m[3], const double msk[3],
                                           const double nsk[3], double h[3]) {
  double an[3];
  aniso_field(P, m, msk, an);
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double L = F[a][sy][sx - 1], R = F[a][sy][sx + 1];
    const double U = F[a][sy - 1][sx], D = F[a][sy + 1][sx];
    h[a] = P.che * (L + R + U + D) + an[a] + P.chb * nsk[a] * (L + R);
  }
}

__global__ void __launch_bounds__(TX * TY) k_rhs_tile(DevProblem P, const double* __restrict__ y,
                                                      const double* __restrict__ hd,
                                                      double* __restrict__ ydot) {
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
  for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + P.happ[a];
  double o[3];
  llg_torque(P, m, h, gate_of(P, cell), o);
  ydot[cell] = o[0]; ydot[n + cell] = o[1]; ydot[2 * n + cell] = o[2];
}

__device__ __forceinline__ double gather_nb(const DevProblem& P, const double* f, int a, int i, int j) {
  if (!map_nb(i, j, P.ng, P.ny, P.bc)) return 0.0;
  return f[a * P.ncell + j * P.ng + i];
}

__device__ __forceinline__ void gather_field(const DevProblem& P, const double* y, int gi, int gj,
                                             const double m[3], const double msk[3], const double nsk[3],
                                             double h[3]) {
  double an[3];
  aniso_field(P, m, msk, an);
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const double L = gather_nb(P, y, a, gi - 1, gj), R = gather_nb(P, y, a, gi + 1, gj);
    const double U = gather_nb(P, y, a, gi, gj - 1), D = gather_nb(P, y, a, gi, gj + 1);
    h[a] = P.che * (L + R + U + D) + an[a] + P.chb * nsk[a] * (L + R);
  }
}

__global__ void k_rhs_compact(DevProblem P, const double* __restrict__ y, const double* __restrict__ hd,
                              double* __restrict__ ydot, const int32_t* __restrict__ act_ids, int na,
                              const int32_t* __restrict__ inact_ids, int ni) {
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
    for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + P.happ[a];
    double o[3];
    llg_torque(P, m, h, 1.0, o);
    ydot[cell] = o[0]; ydot[n + cell] = o[1]; ydot[2 * n + cell] = o[2];
  }
}

// J(m)·v at one cell given field h, the staged/gathered dh pieces.
__device__ __forceinline__ void jv_cell(const DevProblem& P, const double m[3], const double v[3],
                                        const double h[3], const double dh[3], double g, double o[3]) {
  const double m1 = m[0], m2 = m[1], m3 = m[2], v1 = v[0], v2 = v[1], v3 = v[2];
  const double h1 = h[0], h2 = h[1], h3 = h[2];
  const double mh = m1 * h1 + m2 * h2 + m3 * h3;
  const double dmh = (v1 * h1 + v2 * h2 + v3 * h3) + (m1 * dh[0] + m2 * dh[1] + m3 * dh[2]);
  o[0] = g * (P.chg * (v3 * h2 + m3 * dh[1] - v2 * h3 - m2 * dh[2]) + P.alpha * (dh[0] - dmh * m1 - mh * v1));
  o[1] = g * (P.chg * (v1 * h3 + m1 * dh[2] - v3 * h1 - m3 * dh[0]) + P.alpha * (dh[1] - dmh * m2 - mh * v2));
  o[2] = g * (P.chg * (v2 * h1 + m2 * dh[0] - v1 * h2 - m1 * dh[1]) + P.alpha * (dh[2] - dmh * m3 - mh * v3));
}

__device__ __forceinline__ void dh_from(const DevProblem& P, double L, double R, double U, double D, int a,
                                        const double K[3][3], const double v[3], const double nsk[3],
                                        double& out) {
  const double kv = K[a][0] * v[0] + K[a][1] * v[1] + K[a][2] * v[2];
  out = P.che * (L + R + U + D) + kv + P.chb * nsk[a] * (L + R);
}

__global__ void __launch_bounds__(TX * TY) k_jtv_tile(DevProblem P, const double* __restrict__ v,
                                                      double* __restrict__ Jv, const double* __restrict__ y,
                                                      const double* __restrict__ hd) {
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
    for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + P.happ[a];
  }
  double K[3][3];
  aniso_jac(P, m, msk, K);
  double dh[3];
#pragma unroll
  for (int a = 0; a < 3; a++)
    dh_from(P, T.v[1][a][sy][sx - 1], T.v[1][a][sy][sx + 1], T.v[1][a][sy - 1][sx], T.v[1][a][sy + 1][sx], a, K,
            vv, nsk, dh[a]);
  double o[3];
  jv_cell(P, m, vv, h, dh, gate_of(P, cell), o);
  Jv[cell] = o[0]; Jv[n + cell] = o[1]; Jv[2 * n + cell] = o[2];
}

__global__ void k_jtv_compact(DevProblem P, const double* __restrict__ v, double* __restrict__ Jv,
                              const double* __restrict__ y, const double* __restrict__ hd,
                              const int32_t* __restrict__ act_ids, int na, const int32_t* __restrict__ inact_ids,
                              int ni) {
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
      for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + P.happ[a];
    }
    double K[3][3];
    aniso_jac(P, m, msk, K);
    double dh[3];
#pragma unroll
    for (int a = 0; a < 3; a++)
      dh_from(P, gather_nb(P, v, a, gi - 1, gj), gather_nb(P, v, a, gi + 1, gj), gather_nb(P, v, a, gi, gj - 1),
              gather_nb(P, v, a, gi, gj + 1), a, K, vv, nsk, dh[a]);
    double o[3];
    jv_cell(P, m, vv, h, dh, 1.0, o);
    Jv[cell] = o[0]; Jv[n + cell] = o[1]; Jv[2 * n + cell] = o[2];
  }
}

// psetup: freeze (m, h_total) per cell
__global__ void __launch_bounds__(TX * TY) k_psetup_tile(DevProblem P, const double* __restrict__ y,
                                                         const double* __restrict__ hd, double* __restrict__ pm,
                                                         double* __restrict__ ph) {
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
    h[a] = h[a] + hd[a * n + cell] + P.happ[a];
    pm[a * n + cell] = m[a];
    ph[a * n + cell] = h[a];
  }
}

__global__ void k_psolve(DevProblem P, const double* __restrict__ pm, const double* __restrict__ ph,
                         const double* __restrict__ r, double* __restrict__ z, double gamma) {
  const int n = P.ncell;
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
__global__ void __launch_bounds__(TX * TY) k_arnoldi_tile(DevProblem P, const double* __restrict__ in,
                                                          const double* __restrict__ s,
                                                          double* __restrict__ out, const double* __restrict__ y,
                                                          const double* __restrict__ hd,
                                                          const double* __restrict__ pm,
                                                          const double* __restrict__ ph, double gamma,
                                                          double gamma_p) {
  __shared__ Tile<2> T;
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
        T.v[1][a][sy][sx] = ok ? ww * (in[a * n + cell] / s[a * n + cell]) : 0.0;
      }
    }
    __syncthreads();
  }
  const int gi = blockIdx.x * TX + threadIdx.x, gj = blockIdx.y * TY + threadIdx.y;
  if (gi >= P.ng || gj >= P.ny) return;
  const int n = P.ncell, cell = gj * P.ng + gi;
  const int sx = threadIdx.x + 1, sy = threadIdx.y + 1;
  const double m[3] = {y[cell], y[n + cell], y[2 * n + cell]};
  const double ss[3] = {s[cell], s[n + cell], s[2 * n + cell]};
  const double vv[3] = {in[cell] / ss[0], in[n + cell] / ss[1], in[2 * n + cell] / ss[2]};
  double msk[3], nsk[3];
  cell_axes(P, cell, msk, nsk);
  double h[3];
  tile_field(P, T.v[0], sx, sy, m, msk, nsk, h);
  if (P.jv_full) {
#pragma unroll
    for (int a = 0; a < 3; a++) h[a] = h[a] + hd[a * n + cell] + P.happ[a];
  }
  double K[3][3];
  aniso_jac(P, m, msk, K);
  double dh[3];
#pragma unroll
  for (int a = 0; a < 3; a++)
    dh_from(P, T.v[1][a][sy][sx - 1], T.v[1][a][sy][sx + 1], T.v[1][a][sy - 1][sx], T.v[1][a][sy + 1][sx], a, K,
            vv, nsk, dh[a]);
  const double g = gate_of(P, cell);
  double jv[3];
  jv_cell(P, m, vv, h, dh, g, jv);
  double u[3];
#pragma unroll
  for (int a = 0; a < 3; a++) u[a] = 1.0 * vv[a] + (-gamma) * jv[a];
  // P^-1 from the frozen state
  const double fm[3] = {pm[cell], pm[n + cell], pm[2 * n + cell]};
  const double fh[3] = {ph[cell], ph[n + cell], ph[2 * n + cell]};
  const double ws = P.windowed ? P.w[cell] : 1.0;
  double Pi[9];
  block_inverse(P, fm, fh, msk, ws, gamma_p, Pi);
  double gz = 1.0;
  if (!P.windowed && P.act) gz = P.act[cell] ? 1.0 : 0.0;
  const double z0 = gz * (Pi[0] * u[0] + Pi[1] * u[1] + Pi[2] * u[2]);
  const double z1 = gz * (Pi[3] * u[0] + Pi[4] * u[1] + Pi[5] * u[2]);
  const double z2 = gz * (Pi[6] * u[0] + Pi[7] * u[1] + Pi[8] * u[2]);
  out[cell] = ss[0] * z0;
  out[n + cell] = ss[1] * z1;
  out[2 * n + cell] = ss[2] * z2;
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
  k_normalize<<<grid_1d(c, c->ncell, 256), 256, 0, c->stream>>>(y, c->ncell, c->p.norm_kind, c->p.norm_eps);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

static dim3 tile_grid(const llg_ctx* c) { return dim3((c->p.ng + TX - 1) / TX, (c->p.ny + TY - 1) / TY); }

int launch_rhs(llg_ctx* c, const double* y, const double* hd, double* ydot) {
  if (c->p.exec_model == LLG_EXEC_COMPACT) {
    const int tot = c->n_active + c->n_inactive;
    LLG_COUNT(KID_RHS);
    k_rhs_compact<<<grid_1d(c, tot, 256), 256, 0, c->stream>>>(c->dp, y, hd, ydot, c->d_active_ids, c->n_active,
                                                               c->d_inactive_ids, c->n_inactive);
  } else {
    LLG_COUNT(KID_RHS);
    k_rhs_tile<<<tile_grid(c), dim3(TX, TY), 0, c->stream>>>(c->dp, y, hd, ydot);
  }
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int launch_jtv(llg_ctx* c, const double* v, double* Jv, const double* y) {
  if (c->p.exec_model == LLG_EXEC_COMPACT) {
    const int tot = c->n_active + c->n_inactive;
    LLG_COUNT(KID_JTV);
    k_jtv_compact<<<grid_1d(c, tot, 256), 256, 0, c->stream>>>(c->dp, v, Jv, y, c->d_hd, c->d_active_ids,
                                                               c->n_active, c->d_inactive_ids, c->n_inactive);
  } else {
    LLG_COUNT(KID_JTV);
    k_jtv_tile<<<tile_grid(c), dim3(TX, TY), 0, c->stream>>>(c->dp, v, Jv, y, c->d_hd);
  }
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int launch_psetup(llg_ctx* c, const double* y, double gamma) {
  LLG_COUNT(KID_PSETUP);
  k_psetup_tile<<<tile_grid(c), dim3(TX, TY), 0, c->stream>>>(c->dp, y, c->d_hd, c->d_pm, c->d_ph);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  c->gamma_setup = gamma;
  c->have_setup = 1;
  return 0;
}

int launch_psolve(llg_ctx* c, const double* r, double* z) {
  if (!c->have_setup) { llg_set_error("psolve before psetup"); return LLG_ERR_STATE; }
  LLG_COUNT(KID_PSOLVE);
  k_psolve<<<grid_1d(c, c->ncell, 256), 256, 0, c->stream>>>(c->dp, c->d_pm, c->d_ph, r, z, c->gamma_setup);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int launch_arnoldi_op(llg_ctx* c, const double* in, const double* ewt, double* out, const double* y,
                      double gamma) {
  if (!c->have_setup) { llg_set_error("arnoldi operator before psetup"); return LLG_ERR_STATE; }
  LLG_COUNT(KID_ARNOLDI);
  k_arnoldi_tile<<<tile_grid(c), dim3(TX, TY), 0, c->stream>>>(c->dp, in, ewt, out, y, c->d_hd, c->d_pm, c->d_ph,
                                                               gamma, c->gamma_setup);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int rhs_full(llg_ctx* c, double t, double* y, double* ydot) {
  (void)t;
  int rc = launch_normalize(c, y);
  if (rc) return rc;
  if (c->demag) {
    rc = demag_apply(c, y, c->d_hd);
    if (rc) return rc;
    c->nfe_demag++;
  } else {
    LLG_CUDA_TRY(cudaMemsetAsync(c->d_hd, 0, sizeof(double) * 3 * (size_t)c->ncell, c->stream));
  }
  return launch_rhs(c, y, c->d_hd, ydot);
}
