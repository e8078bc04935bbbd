// dev_physics.cuh — per-cell LLG device helpers shared by the stencil kernels
// (k_physics.cu) and the fused integrator kernels (k_fused.cu).  Formulas and
// reference citations: see the header of k_physics.cu.
#pragma once
#include <math.h>
#include "llg_internal.h"

namespace {


constexpr int TX = 32;
constexpr int TY = 8;

// Logical slot -> grid cell.  Tile slots can lie up to a tile width past the
// edge (grids narrower than a tile), so the periodic wrap is a full modulo.
// Periodic wrap without integer division: the tile loaders ask for indices
// one cell outside the grid (and, in a tile that overhangs a small grid,
// further out, where only the remainder's range matters), so one add or
// subtract covers the common case and the division is the rare fallback.
__device__ __forceinline__ int wrap_idx(int i, int n) {
  if (i < 0) i += n;
  else if (i >= n) i -= n;
  if ((unsigned)i >= (unsigned)n) {   // more than one period out
    i %= n;
    if (i < 0) i += n;
  }
  return i;
}
__device__ __forceinline__ bool map_nb(int& i, int& j, int ng, int ny, int bc) {
  if (bc == LLG_BC_FREE) return (i >= 0 && i < ng && j >= 0 && j < ny);
  i = wrap_idx(i, ng);
  j = wrap_idx(j, ny);
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

// Damping of the RHS at column gi: uniform, or ramped up towards the x edges
// in the absorbing layers (src/slit/2d_slit.cu:297-315, same expression)
__device__ __forceinline__ double alpha_at(const DevProblem& P, int gi) {
  if (P.pml_cells <= 0) return P.alpha;
  const int pml = P.pml_cells;
  double s = 0.0;
  if (gi < pml) s = 1.0 - (double)gi / (double)pml;
  else if (gi >= P.ng - pml) s = (double)(gi - (P.ng - pml)) / (double)pml;
  return P.alpha + (P.pml_alpha_max - P.alpha) * s * s * s;
}

// Uniform applied field, plus the soft spin-wave source's value for the
// current evaluation on its column (x component, src/slit/2d_slit.cu:331-349)
__device__ __forceinline__ double happ_at(const DevProblem& P, int a, int gi) {
  return (a == 0 && P.src_on && gi == P.src_col) ? P.happ[0] + P.src_h : P.happ[a];
}

__device__ __forceinline__ void llg_torque(const DevProblem& P, double alpha, const double m[3], const double h[3],
                                           double g, double out[3]) {
  const double m1 = m[0], m2 = m[1], m3 = m[2], h1 = h[0], h2 = h[1], h3 = h[2];
  const double mh = m1 * h1 + m2 * h2 + m3 * h3;
  out[0] = g * (P.chg * (m3 * h2 - m2 * h3) + alpha * (h1 - mh * m1));
  out[1] = g * (P.chg * (m1 * h3 - m3 * h1) + alpha * (h2 - mh * m2));
  out[2] = g * (P.chg * (m2 * h1 - m1 * h2) + alpha * (h3 - mh * m3));
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

// the block inverse of one cell stored by psetup (9 planes of n doubles)
// (the FP32-basis Krylov solver stores it in FP32)
__device__ __forceinline__ void load_pinv(const float* __restrict__ pinv, int n, int cell, double Pi[9]) {
#pragma unroll
  for (int k = 0; k < 9; k++) Pi[k] = (double)pinv[(long long)k * n + cell];
}
__device__ __forceinline__ void load_pinv(const double* __restrict__ pinv, int n, int cell, double Pi[9]) {
#pragma unroll
  for (int k = 0; k < 9; k++) Pi[k] = pinv[(long long)k * n + cell];
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

}  // namespace
