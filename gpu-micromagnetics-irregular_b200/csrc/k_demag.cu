// k_demag.cu — FFT demagnetising field for sm_100a, FP64.
//
// Reference chain (src/irregular/2d_fft/2d_i2/demag_fft.cu:325-363, windowed
// 2d_i3/demag_fft.cu:371-419):  gather (× w) → cufftExecD2Z (batch 3) →
// Ĥ_a = Σ_b N̂_ab M̂_b → cufftExecZ2D (batch 3) → FFT-shift, × strength/(nx·ny),
// scatter to SoA.  Tensor: 81-point face average of the closed-form Newell
// integrals (demag_fft.cu:27-91) computed once at init.
//
// Here the chain is three hand-written kernels and no library FFT:
//   K1 rows_fwd : SoA y (× w) → real FFT along x of each data row (two real
//                 rows packed into one complex transform) → spectrum S written
//                 column-major [comp][kx][y] so K2 reads whole columns.
//   K2 cols     : per x-frequency column, all three components: FFT along y
//                 (zero-padded rows in open mode) → 3x3 tensor multiply →
//                 inverse FFT along y → S (only the data rows are kept).
//   K3 rows_inv : inverse real FFT along x → h, × strength/(Px·Py) folded into
//                 the tensor, written SoA for the first ng columns only.
// Every transform is a Stockham autosort FFT in shared memory (natural order
// in and out, no reordering tables): each pass stages the thread's radix-R
// butterflies in registers, synchronises, and scatters the results in place.
// The lengths 1024/2048/3072/4096 run a compile-time plan (radix 16 first,
// then one 12/8/6/4/2 pass; the kernels are instantiated per length, FIX),
// every other length a runtime plan (radix 8/4/2/3/5, any other prime through
// a generic path).  A CTA row of threads owns one transform; HBM sees each
// element of y, S and h once per kernel.
// The tensor is stored wrapped at displacement d mod P (d in [-P/2, P-1-P/2]),
// which equals the reference's centring + output shift; the open-boundary
// tensor has its unused d = -P/2 lines zeroed, so its spectra are real.  Only
// xx, yy, zz (real) and xy = yx (complex) are kept: for the single-layer film
// (field point in the mid-plane) the xz, yz, zx, zy integrals cancel; init
// verifies this numerically and refuses the plan otherwise.
#include <math.h>
#include <string.h>
#include <stdio.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "dev_fft.cuh"
#include "llg_internal.h"
#include "launch.h"

namespace {

using FftPlan = FftPlanT<double>;

// 16-byte (cg) or 8-byte (ca) asynchronous global->shared copy
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (BYTES == 16) asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
  else asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// ── K1: forward real transform of data rows along x ─────────────────────
// CTA = (component c, 2*NB rows); threadIdx.y = packed transform (rows ya, ya+1).
// The FP64 input is rounded to R on load (R = float: mixed chain).  FIX > 0:
// the compile-time plan of that length, whose first pass reads its inputs
// from HBM directly and, for an open-boundary row (row_len <= n/2), skips the
// zero-padded upper half of every butterfly; FIX = 0: the runtime plan.
template <typename R, int NB, int EPT, int FIX>
__global__ void k_rows_fwd(FftPlanT<R> pl, const double* __restrict__ in, long long comp_stride, int row_len,
                           int nrows, const double* __restrict__ w, cx_t<R>* __restrict__ S, int ld, int Hx) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  cx_t<R>* sm = reinterpret_cast<cx_t<R>*>(smraw);
  const int c = blockIdx.y;
  const int y0 = blockIdx.x * (2 * NB);
  const int n = FIX > 0 ? FIX : pl.n;
  const int b = threadIdx.y;
  const int np = padded_len<R>(n);
  cx_t<R>* buf = sm + b * np;
  const double* src = in + (long long)c * comp_stride;
  const int ya = y0 + 2 * b, yb = ya + 1;
  // packed input element i: rows ya (real part) and yb (imaginary part)
  auto load_in = [&](int i) -> cx_t<R> {
    double va = 0.0, vb = 0.0;
    if (i < row_len) {
      if (ya < nrows) {
        const long long q = (long long)ya * row_len + i;
        va = src[q] * (w ? w[q] : 1.0);
      }
      if (yb < nrows) {
        const long long q = (long long)yb * row_len + i;
        vb = src[q] * (w ? w[q] : 1.0);
      }
    }
    return mk<R>((R)va, (R)vb);
  };
  if constexpr (FIX > 0) {
    constexpr RadixList L = fixed_radices(FIX);
    constexpr int R0 = L.r[0];
    if constexpr (R0 % 2 == 0) {
      if (2 * row_len <= FIX) stockham_first_pass_ld<R, R0, -1, EPT, true, true>(buf, FIX, load_in);
      else stockham_first_pass_ld<R, R0, -1, EPT, true, false>(buf, FIX, load_in);
    } else {
      stockham_first_pass_ld<R, R0, -1, EPT, true, false>(buf, FIX, load_in);
    }
    fft_fixed<R, -1, EPT, true, FIX, 1, L.nr, R0>(buf, pl);
  } else {
    for (int i = threadIdx.x; i < n; i += blockDim.x) buf[fpad<R, true>(i)] = load_in(i);
    __syncthreads();
    fft_stockham<R, -1, EPT, true>(buf, pl);
  }
  const int T = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
  for (int e = tid; e < Hx * 2 * NB; e += T) {
    const int kx = e / (2 * NB), r = e - kx * (2 * NB);
    const int bb = r >> 1, which = r & 1;
    const int y = y0 + r;
    if (y >= nrows) continue;
    const cx_t<R> zk = sm[bb * np + fpad<R, true>(kx)];
    const cx_t<R> zm = sm[bb * np + fpad<R, true>(kx == 0 ? 0 : n - kx)];   // (n - kx) mod n
    cx_t<R> out;
    if (!which) out = mk<R>(R(0.5) * (zk.x + zm.x), R(0.5) * (zk.y - zm.y));
    else out = mk<R>(R(0.5) * (zk.y + zm.y), R(-0.5) * (zk.x - zm.x));
    S[((long long)c * Hx + kx) * ld + y] = out;
  }
}

// the column transform of one CTA row (a runtime or a compile-time plan)
template <typename R, int SIGN, int EPT, int FIX>
__device__ __forceinline__ void col_fft(cx_t<R>* buf, const FftPlanT<R>& pl) {
  if constexpr (FIX > 0) fft_fixed<R, SIGN, EPT, false, FIX, 0, fixed_radices(FIX).nr, 1>(buf, pl);
  else fft_stockham<R, SIGN, EPT>(buf, pl);
}

// ── K2: column transform + tensor multiply + inverse column transform ─────
// CTA = one x-frequency column.  The three spectrum columns and (STAGE) this
// column's tensor spectra are fetched with asynchronous copies (cp.async) at
// entry, so the tensor read overlaps the forward transform instead of
// stalling the multiply.
template <typename R, int EPT, bool STAGE, int FIX>
__device__ __forceinline__ void cols_conv_concurrent(FftPlanT<R> pl, cx_t<R>* __restrict__ S, int ld, int nrows, int Hx,
                            const R* __restrict__ txx, const R* __restrict__ tyy, const R* __restrict__ tzz,
                            const cx_t<R>* __restrict__ txy) {
  using C = cx_t<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int kx = blockIdx.x;
  const int n = FIX > 0 ? FIX : pl.n;
  const int c = threadIdx.y;
  C* buf = sm + c * n;
  C* col = S + ((long long)c * Hx + kx) * ld;
  const int T = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
  const long long tb = (long long)kx * n;
  R* sxx = reinterpret_cast<R*>(sm + 3 * n);
  R* syy = sxx + n;
  R* szz = syy + n;
  C* sxy = reinterpret_cast<C*>(szz + n);
  for (int yy = threadIdx.x; yy < n; yy += blockDim.x) {
    if (yy < nrows) cp_async<sizeof(C)>(&buf[yy], &col[yy]);
    else buf[yy] = mk<R>(R(0), R(0));
  }
  cp_async_commit();
  if (STAGE) {
    constexpr int PR = 16 / sizeof(R), PC = 16 / sizeof(C);  // elements per 16-byte copy
    const int hr = n / PR, hc = n / PC;
    for (int e = tid; e < 3 * hr + hc; e += T) {
      if (e < hr) cp_async<16>(&sxx[PR * e], &txx[tb + PR * e]);
      else if (e < 2 * hr) cp_async<16>(&syy[PR * (e - hr)], &tyy[tb + PR * (e - hr)]);
      else if (e < 3 * hr) cp_async<16>(&szz[PR * (e - 2 * hr)], &tzz[tb + PR * (e - 2 * hr)]);
      else cp_async<16>(&sxy[PC * (e - 3 * hr)], &txy[tb + PC * (e - 3 * hr)]);
    }
  }
  cp_async_commit();
  cp_async_wait<1>();
  __syncthreads();
  col_fft<R, -1, EPT, FIX>(buf, pl);
  cp_async_wait<0>();
  __syncthreads();
  for (int ky = tid; ky < n; ky += T) {
    const C mx = sm[ky], my = sm[n + ky], mz = sm[2 * n + ky];
    R a, b, d;
    C xy;
    if (STAGE) { a = sxx[ky]; b = syy[ky]; d = szz[ky]; xy = sxy[ky]; }
    else { a = __ldg(&txx[tb + ky]); b = __ldg(&tyy[tb + ky]); d = __ldg(&tzz[tb + ky]); xy = __ldg(&txy[tb + ky]); }
    const C hxy = cmul<R>(xy, my), hyx = cmul<R>(xy, mx);
    sm[ky] = mk<R>(a * mx.x + hxy.x, a * mx.y + hxy.y);
    sm[n + ky] = mk<R>(hyx.x + b * my.x, hyx.y + b * my.y);
    sm[2 * n + ky] = mk<R>(d * mz.x, d * mz.y);
  }
  __syncthreads();
  col_fft<R, +1, EPT, FIX>(buf, pl);
  for (int yy = threadIdx.x; yy < nrows; yy += blockDim.x) col[yy] = buf[yy];
}

template <typename R, int EPT, bool STAGE, int FIX>
__device__ __forceinline__ void cols_conv_in_turn(FftPlanT<R> pl, cx_t<R>* __restrict__ S, int ld, int nrows, int Hx,
                            const R* __restrict__ txx, const R* __restrict__ tyy, const R* __restrict__ tzz,
                            const cx_t<R>* __restrict__ txy) {
  using C = cx_t<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int kx = blockIdx.x;
  const int n = FIX > 0 ? FIX : pl.n;
  const int T = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
  const long long tb = (long long)kx * n;
  R* sxx = reinterpret_cast<R*>(sm + 3 * n);
  R* syy = sxx + n;
  R* szz = syy + n;
  C* sxy = reinterpret_cast<C*>(szz + n);
  for (int c = threadIdx.y; c < 3; c += blockDim.y) {
    C* buf = sm + c * n;
    const C* col = S + ((long long)c * Hx + kx) * ld;
    for (int yy = threadIdx.x; yy < n; yy += blockDim.x) {
      if (yy < nrows) cp_async<sizeof(C)>(&buf[yy], &col[yy]);
      else buf[yy] = mk<R>(R(0), R(0));
    }
  }
  cp_async_commit();
  if (STAGE) {
    constexpr int PR = 16 / sizeof(R), PC = 16 / sizeof(C);  // elements per 16-byte copy
    const int hr = n / PR, hc = n / PC;
    for (int e = tid; e < 3 * hr + hc; e += T) {
      if (e < hr) cp_async<16>(&sxx[PR * e], &txx[tb + PR * e]);
      else if (e < 2 * hr) cp_async<16>(&syy[PR * (e - hr)], &tyy[tb + PR * (e - hr)]);
      else if (e < 3 * hr) cp_async<16>(&szz[PR * (e - 2 * hr)], &tzz[tb + PR * (e - 2 * hr)]);
      else cp_async<16>(&sxy[PC * (e - 3 * hr)], &txy[tb + PC * (e - 3 * hr)]);
    }
  }
  cp_async_commit();
  cp_async_wait<1>();
  __syncthreads();
  for (int c = threadIdx.y; c < 3; c += blockDim.y) col_fft<R, -1, EPT, FIX>(sm + c * n, pl);   // uniform trip count
  cp_async_wait<0>();
  __syncthreads();
  for (int ky = tid; ky < n; ky += T) {
    const C mx = sm[ky], my = sm[n + ky], mz = sm[2 * n + ky];
    R a, b, d;
    C xy;
    if (STAGE) { a = sxx[ky]; b = syy[ky]; d = szz[ky]; xy = sxy[ky]; }
    else { a = __ldg(&txx[tb + ky]); b = __ldg(&tyy[tb + ky]); d = __ldg(&tzz[tb + ky]); xy = __ldg(&txy[tb + ky]); }
    const C hxy = cmul<R>(xy, my), hyx = cmul<R>(xy, mx);
    sm[ky] = mk<R>(a * mx.x + hxy.x, a * mx.y + hxy.y);
    sm[n + ky] = mk<R>(hyx.x + b * my.x, hyx.y + b * my.y);
    sm[2 * n + ky] = mk<R>(d * mz.x, d * mz.y);
  }
  __syncthreads();
  for (int c = threadIdx.y; c < 3; c += blockDim.y) {
    C* buf = sm + c * n;
    col_fft<R, +1, EPT, FIX>(buf, pl);
    C* col = S + ((long long)c * Hx + kx) * ld;
    for (int yy = threadIdx.x; yy < nrows; yy += blockDim.x) col[yy] = buf[yy];
  }
}

// The kernel: CY = 3 transforms the three components concurrently (one CTA
// row each), CY = 1 in turn with one row of threads (long FP64 columns,
// whose registers allow only a third of the threads).  The two bodies are
// separate so that the common form keeps its straight-line code.
template <typename R, int EPT, bool STAGE, int FIX, int CY>
__global__ void k_cols_conv(FftPlanT<R> pl, cx_t<R>* __restrict__ S, int ld, int nrows, int Hx,
                            const R* __restrict__ txx, const R* __restrict__ tyy, const R* __restrict__ tzz,
                            const cx_t<R>* __restrict__ txy) {
  pdl_entry();
  if constexpr (CY == 3) cols_conv_concurrent<R, EPT, STAGE, FIX>(pl, S, ld, nrows, Hx, txx, tyy, tzz, txy);
  else cols_conv_in_turn<R, EPT, STAGE, FIX>(pl, S, ld, nrows, Hx, txx, tyy, tzz, txy);
}

// forward column transform only (tensor spectra at init, FP64)
template <int EPT, int FIX>
__global__ void k_cols_fwd(FftPlan pl, double2* __restrict__ S, int ld, int nrows, int Hx) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* sm = reinterpret_cast<double2*>(smraw);
  const int kx = blockIdx.x;
  const int n = FIX > 0 ? FIX : pl.n;
  double2* col = S + (long long)kx * ld;
  for (int yy = threadIdx.x; yy < n; yy += blockDim.x) sm[yy] = (yy < nrows) ? col[yy] : make_double2(0.0, 0.0);
  __syncthreads();
  col_fft<double, -1, EPT, FIX>(sm, pl);
  for (int yy = threadIdx.x; yy < n; yy += blockDim.x) col[yy] = sm[yy];
}

// ── K3: inverse real transform along x, scatter to SoA h (FP64) ──────────
// FIX > 0: the compile-time plan of that length, whose last pass writes the
// kept outputs i < ng to HBM directly (an open-boundary row, ng <= n/2,
// forms only the lower half of every butterfly); FIX = 0: the runtime plan.
template <typename R, int NB, int EPT, int FIX>
__global__ void k_rows_inv(FftPlanT<R> pl, const cx_t<R>* __restrict__ S, int ld, int nrows, int Hx,
                           double* __restrict__ h, long long comp_stride, int ng) {
  pdl_entry();
  using C = cx_t<R>;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int c = blockIdx.y;
  const int y0 = blockIdx.x * (2 * NB);
  const int n = FIX > 0 ? FIX : pl.n;
  const int b = threadIdx.y;
  const bool even = (n % 2) == 0;
  const int np = padded_len<R>(n);
  // Load the CTA's 2*NB rows of every spectrum column once, with lanes laid
  // out (column, row): the rows of one column are adjacent in memory, so a
  // warp load covers whole sectors.  The pair partner (row 2p+1 of pair p)
  // comes from the next lane; the even lane forms entry kk of pair p's
  // packed transform and, for kk in [1, n - Hx], the mirrored entry n - kk
  // (conjugated spectrum), exactly as entry k would be formed from kk = n - k.
  {
    constexpr int RW = 2 * NB;   // rows per column in this CTA (divides 32)
    const int T = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int total = Hx * RW;
    for (int base = 0; base < total; base += T) {
      const int e = base + tid;
      const int kk = e / RW, r = e - kk * RW, y = y0 + r;
      C v = mk<R>(R(0), R(0));
      if (e < total && y < nrows) v = S[((long long)c * Hx + kk) * ld + y];
      C w;
      w.x = __shfl_down_sync(0xffffffffu, v.x, 1);
      w.y = __shfl_down_sync(0xffffffffu, v.y, 1);
      if (e < total && (r & 1) == 0) {
        C* bp = sm + (r >> 1) * np;
        C A = v, B = w;
        if (kk == 0 || (even && kk == n / 2)) { A.y = R(0); B.y = R(0); }
        bp[fpad<R, true>(kk)] = mk<R>(A.x - B.y, A.y + B.x);
        if (kk >= 1 && kk <= n - Hx) {
          A.y = -A.y;
          B.y = -B.y;
          bp[fpad<R, true>(n - kk)] = mk<R>(A.x - B.y, A.y + B.x);
        }
      }
    }
  }
  __syncthreads();
  C* buf = sm + b * np;
  double* dst = h + (long long)c * comp_stride;
  if constexpr (FIX > 0) {
    // rows ya (real part) and yb (imaginary part), kept outputs i < ng
    const int ya = y0 + 2 * b, yb = ya + 1;
    auto st = [&](int i, C z) {
      if (i < ng) {
        if (ya < nrows) dst[(long long)ya * ng + i] = (double)z.x;
        if (yb < nrows) dst[(long long)yb * ng + i] = (double)z.y;
      }
    };
    constexpr RadixList L = fixed_radices(FIX);
    constexpr int RL = L.r[L.nr - 1];
    fft_fixed<R, +1, EPT, true, FIX, 0, L.nr - 1, 1>(buf, pl);
    if constexpr (RL % 2 == 0) {
      if (2 * ng <= FIX) stockham_last_pass_st<R, RL, +1, EPT, true, true>(buf, pl, FIX, st);
      else stockham_last_pass_st<R, RL, +1, EPT, true, false>(buf, pl, FIX, st);
    } else {
      stockham_last_pass_st<R, RL, +1, EPT, true, false>(buf, pl, FIX, st);
    }
  } else {
    fft_stockham<R, +1, EPT, true>(buf, pl);
    const int T = blockDim.x * blockDim.y, tid = threadIdx.y * blockDim.x + threadIdx.x;
#pragma unroll
    for (int r = 0; r < NB * 2; r++) {
      const int y = y0 + r;
      if (y >= nrows) break;
      for (int i = tid; i < ng; i += T) {
        const C z = sm[(r >> 1) * np + fpad<R, true>(i)];
        dst[(long long)y * ng + i] = (double)((r & 1) ? z.y : z.x);
      }
    }
  }
}

// ── Newell tensor (81-point average of the closed-form integrals) ────────
// Same term grouping as the reference's ctt/calt (demag_fft.cu:27-91).
__device__ void newell_point(double thick, double sx, double sy, double out[9]) {
  const double a = 0.49999, bb = 0.5 * thick, sz = 0.0;
  const double X[2] = {sx - a, sx + a};
  const double Y[2] = {sy - a, sy + a};
  const double Z[2] = {sz - bb, sz + bb};
  double r[2][2][2];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int k = 0; k < 2; k++) r[i][j][k] = sqrt(X[i] * X[i] + Y[j] * Y[j] + Z[k] * Z[k]);
  double xx = 0.0, yy = 0.0, zz = 0.0;
  bool first = true;
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int k = 0; k < 2; k++) {
        const double tm = atan(Z[k] * Y[j] / (X[i] * r[i][j][k]));
        const double sg = ((i + j + k) & 1) ? -1.0 : 1.0;
        xx = first ? tm : xx + sg * tm;
        first = false;
      }
  first = true;
#pragma unroll
  for (int j = 0; j < 2; j++)
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
      for (int k = 0; k < 2; k++) {
        const double tm = atan(Z[k] * X[i] / (Y[j] * r[i][j][k]));
        const double sg = ((i + j + k) & 1) ? -1.0 : 1.0;
        yy = first ? tm : yy + sg * tm;
        first = false;
      }
  first = true;
#pragma unroll
  for (int k = 0; k < 2; k++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const double tm = atan(X[i] * Y[j] / (Z[k] * r[i][j][k]));
        const double sg = ((i + j + k) & 1) ? -1.0 : 1.0;
        zz = first ? tm : zz + sg * tm;
        first = false;
      }
#define LZ(i, j) log((r[i][j][0] - Z[0]) / (r[i][j][1] - Z[1]))
#define LY(i, k) log((r[i][0][k] - Y[0]) / (r[i][1][k] - Y[1]))
#define LX(j, k) log((r[0][j][k] - X[0]) / (r[1][j][k] - X[1]))
  out[0] = xx;
  out[1] = LZ(0, 0) - LZ(1, 0) - LZ(0, 1) + LZ(1, 1);
  out[2] = LY(0, 0) - LY(1, 0) - LY(0, 1) + LY(1, 1);
  out[3] = LZ(0, 0) - LZ(0, 1) - LZ(1, 0) + LZ(1, 1);
  out[4] = yy;
  out[5] = LX(0, 0) - LX(1, 0) - LX(0, 1) + LX(1, 1);
  out[6] = LY(0, 0) - LY(0, 1) - LY(1, 0) + LY(1, 1);
  out[7] = LX(0, 0) - LX(0, 1) - LX(1, 0) + LX(1, 1);
  out[8] = zz;
#undef LZ
#undef LY
#undef LX
}

__device__ __forceinline__ int rep_disp(int i, int n) {
  const int hi = n - 1 - n / 2;
  return (i <= hi) ? i : i - n;
}

// T[c][j*px + i] for c < 9; open: the d = -P/2 lines are zeroed (never used
// by the zero-padded linear convolution).
__global__ void k_newell(double* __restrict__ T, int px, int py, double thick, int open) {
  pdl_entry();
  const long long np = (long long)px * py;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < np;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % px), j = (int)(e / px);
    double acc[9];
#pragma unroll
    for (int c = 0; c < 9; c++) acc[c] = 0.0;
    const bool dead = open && (i == px / 2 || j == py / 2);
    if (!dead) {
      const int dx = rep_disp(i, px), dy = rep_disp(j, py);
      double dm[9];
      for (int jy = -4; jy <= 4; jy++) {
        const double sy = (double)dy + 0.1 * (double)jy;
        for (int ix = -4; ix <= 4; ix++) {
          const double sx = (double)dx + 0.1 * (double)ix;
          newell_point(thick, sx, sy, dm);
#pragma unroll
          for (int c = 0; c < 9; c++) acc[c] += dm[c];
        }
      }
#pragma unroll
      for (int c = 0; c < 9; c++) acc[c] = acc[c] / 81.;
    }
#pragma unroll
    for (int c = 0; c < 9; c++) T[c * np + e] = acc[c];
  }
}

// spectra: out arrays [kx*Py + ky]; S_c holds component c's spectrum (col-major, ld = Py)
__global__ void k_tensor_finish(const double2* __restrict__ Sxx, const double2* __restrict__ Syy,
                                const double2* __restrict__ Szz, const double2* __restrict__ Sxy,
                                const double2* __restrict__ Syx, const double2* __restrict__ Sxz,
                                const double2* __restrict__ Syz, const double2* __restrict__ Szx,
                                const double2* __restrict__ Szy, long long total, double scale,
                                double* __restrict__ txx, double* __restrict__ tyy, double* __restrict__ tzz,
                                double2* __restrict__ txy, double* __restrict__ stats) {
  pdl_entry();
  // stats (per block partial max): [0] max|diag|, [1] max imag diag, [2] max |xz family|, [3] max |xy-yx|
  __shared__ double red[4][256];
  double m0 = 0, m1 = 0, m2 = 0, m3 = 0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const double2 a = Sxx[e], b = Syy[e], d = Szz[e], p = Sxy[e], q = Syx[e];
    m0 = fmax(m0, fmax(fabs(a.x), fmax(fabs(b.x), fabs(d.x))));
    m1 = fmax(m1, fmax(fabs(a.y), fmax(fabs(b.y), fabs(d.y))));
    const double2 u = Sxz[e], v = Syz[e], s = Szx[e], t = Szy[e];
    m2 = fmax(m2, fmax(fmax(fabs(u.x), fabs(u.y)), fmax(fabs(v.x), fabs(v.y))));
    m2 = fmax(m2, fmax(fmax(fabs(s.x), fabs(s.y)), fmax(fabs(t.x), fabs(t.y))));
    m3 = fmax(m3, fmax(fabs(p.x - q.x), fabs(p.y - q.y)));
    txx[e] = a.x * scale;
    tyy[e] = b.x * scale;
    tzz[e] = d.x * scale;
    txy[e] = make_double2(0.5 * (p.x + q.x) * scale, 0.5 * (p.y + q.y) * scale);
  }
  red[0][threadIdx.x] = m0; red[1][threadIdx.x] = m1; red[2][threadIdx.x] = m2; red[3][threadIdx.x] = m3;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 4; k++) red[k][threadIdx.x] = fmax(red[k][threadIdx.x], red[k][threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) stats[blockIdx.x * 4 + k] = red[k][0];
}

}  // namespace

// ── host side ───────────────────────────────────────────────────────────
static constexpr int kRowsNB = 1;  // packed transforms per row-CTA at init (tensor spectra)

// radices with an in-register DFT (stockham_pass); any other prime takes
// the generic pass, one thread per butterfly
static bool fixed_radix(int r) {
  return r == 2 || r == 3 || r == 4 || r == 5 || r == 6 || r == 8 || r == 12 || r == 16;
}

struct HostFft {
  int n = 0, tx = 32, ept = 8;
  int fix = 0;   // n when the compile-time plan runs (fixed_length), else 0
  std::vector<int> radix;
  double2* d_tw = nullptr;
  float2* d_twf = nullptr;   // FP32 twiddles (mixed chain)
  int4* d_pass = nullptr;
  // threads per transform for EPT elements per thread: n/EPT covers the
  // fixed radices; a generic radix R needs one thread per butterfly (n/R)
  int tx_for(int e) const {
    int need = (n + e - 1) / e;
    if (!fix)
      for (int r : radix)
        if (!fixed_radix(r)) need = std::max(need, n / r);
    return ((std::max(need, 32) + 31) / 32) * 32;
  }
  template <typename R>
  FftPlanT<R> dev() const {
    FftPlanT<R> p{};
    p.n = n;
    p.nr = (int)radix.size();
    p.tx = tx;
    p.pass = d_pass;
    if constexpr (sizeof(R) == 8) p.tw = d_tw;
    else p.tw = d_twf;
    return p;
  }
};

// Launch shape of one transform kernel, picked per plan by timing (autotune):
// nb packed transforms per CTA (rows), ept elements per thread, stage =
// tensor column prefetched into shared memory (columns).
struct LaunchCfg {
  int nb = 1, ept = 8;
  bool stage = false;
  int cy = 3;   // columns: components transformed concurrently (3) or in turn (1)
};

struct DemagPlan {
  int px = 0, py = 0, hx = 0, ng = 0, ny = 0;
  int open = 0;
  double strength = 0.0;
  double n0[3] = {0, 0, 0};      // unscaled N(0)
  HostFft fx, fy;
  double2* d_S = nullptr;        // 3*hx*ny
  double* d_txx = nullptr;
  double* d_tyy = nullptr;
  double* d_tzz = nullptr;
  double2* d_txy = nullptr;
  double* d_T = nullptr;         // 9 real tensor components (kept for host queries)
  // mixed-precision chain (LLG_DEMAG_MIXED): FP32 spectrum and tensor spectra
  int mixed = 0;
  float2* d_Sf = nullptr;
  float* d_txxf = nullptr;
  float* d_tyyf = nullptr;
  float* d_tzzf = nullptr;
  float2* d_txyf = nullptr;
  LaunchCfg rows[2], cols[2];    // [0] FP64 chain, [1] FP32 chain (autotuned)
  int* d_err = nullptr;          // wait-ran-out flag of the tensor-core column stage (the context's SLOT_TCERR)
  DemagTc* tc = nullptr;         // tensor-core column stage (k_demag_tc.cu), when the shape allows
  cudaGraphExec_t gexec = nullptr;   // captured chain for gkey = (y, w, h) on the context's own stream
  const void* gkey[3] = {nullptr, nullptr, nullptr};
};

// the runtime pass table of length n (runtime_radices), or -1
static int factorize(int n, std::vector<int>& rad) {
  rad.clear();
  const RadixList L = runtime_radices(n);
  if (L.nr < 0) return -1;
  for (int i = 0; i < L.nr; i++) rad.push_back(L.r[i]);
  return 0;
}

// n if length n has a compile-time plan (kFixedLengths), else 0
static int fixed_length(int n) {
  for (int f : kFixedLengths)
    if (f == n && fixed_radices(n).nr > 0) return n;
  return 0;
}

static int fft_init(HostFft& f, int n, int batch) {
  f.n = n;
  f.fix = fixed_length(n);
  if (factorize(n, f.radix) != 0) {
    llg_set_error("FFT length " + std::to_string(n) + " has a prime factor > 64");
    return LLG_ERR_NOTSUP;
  }
  // threads per transform: n/16 covers the fixed radices (<= 16/R butterflies
  // per thread); a generic radix R needs one thread per butterfly (n/R).
  f.ept = (((n + 7) / 8 + 31) / 32 * 32 * batch <= 1024) ? 8 : 16;
  int need = (n + f.ept - 1) / f.ept;
  for (int r : f.radix)
    if (!fixed_radix(r)) need = std::max(need, n / r);
  f.tx = ((std::max(need, 32) + 31) / 32) * 32;
  std::vector<double2> tw(n);
  std::vector<float2> twf(n);
  for (int k = 0; k < n; k++) {
    const long double ang = 2.0L * 3.14159265358979323846264338327950288L * (long double)k / (long double)n;
    tw[k] = make_double2((double)cosl(ang), (double)-sinl(ang));
    twf[k] = make_float2((float)cosl(ang), (float)-sinl(ang));
  }
  LLG_CUDA_TRY(cudaMalloc(&f.d_tw, sizeof(double2) * n));
  LLG_CUDA_TRY(cudaMemcpy(f.d_tw, tw.data(), sizeof(double2) * n, cudaMemcpyHostToDevice));
  LLG_CUDA_TRY(cudaMalloc(&f.d_twf, sizeof(float2) * n));
  LLG_CUDA_TRY(cudaMemcpy(f.d_twf, twf.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
  std::vector<int4> ps(std::max<size_t>(f.radix.size(), 1));
  int ns = 1;
  for (size_t i = 0; i < f.radix.size(); i++) {
    ps[i] = make_int4(f.radix[i], ns, ((ns & (ns - 1)) == 0) ? __builtin_ctz((unsigned)ns) : -1, 0);
    ns *= f.radix[i];
  }
  LLG_CUDA_TRY(cudaMalloc(&f.d_pass, sizeof(int4) * ps.size()));
  LLG_CUDA_TRY(cudaMemcpy(f.d_pass, ps.data(), sizeof(int4) * ps.size(), cudaMemcpyHostToDevice));
  return 0;
}

static void fft_free(HostFft& f) {
  cudaFree(f.d_tw);
  cudaFree(f.d_twf);
  cudaFree(f.d_pass);
  f.d_twf = nullptr;
  f.d_tw = nullptr;
  f.d_pass = nullptr;
}

void demag_destroy(DemagPlan* d) {
  if (!d) return;
  fft_free(d->fx);
  fft_free(d->fy);
  cudaFree(d->d_S);
  cudaFree(d->d_txx);
  cudaFree(d->d_tyy);
  cudaFree(d->d_tzz);
  cudaFree(d->d_txy);
  cudaFree(d->d_T);
  cudaFree(d->d_Sf);
  cudaFree(d->d_txxf);
  cudaFree(d->d_tyyf);
  cudaFree(d->d_tzzf);
  cudaFree(d->d_txyf);
  demag_tc_destroy(d->tc);
  if (d->gexec) cudaGraphExecDestroy(d->gexec);
  delete d;
}

static int set_smem(const void* fn, size_t bytes) {
  if (bytes > 48 * 1024) {
    LLG_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  }
  return 0;
}

// ── launch helpers (elements-per-thread dispatch) ─────────────────────────
template <typename R>
static constexpr int kp() { return sizeof(R) == 8 ? 0 : 1; }

// Kernel of each launch shape: nb packed transforms per CTA, ept elements
// per thread, and the compile-time plan of the transform length when it has
// one (HostFft::fix).
template <typename R>
using RowsFwdFn = void (*)(FftPlanT<R>, const double*, long long, int, int, const double*, cx_t<R>*, int, int);
template <typename R>
using RowsInvFn = void (*)(FftPlanT<R>, const cx_t<R>*, int, int, int, double*, long long, int);
template <typename R>
using ColsFn = void (*)(FftPlanT<R>, cx_t<R>*, int, int, int, const R*, const R*, const R*, const cx_t<R>*);
using ColsFwdFn = void (*)(FftPlan, double2*, int, int, int);

#define LLG_FIX_SWITCH(fix, EXPR_OF)                                          \
  switch (fix) {                                                              \
    case 1024: return EXPR_OF(1024);                                          \
    case 2048: return EXPR_OF(2048);                                          \
    case 3072: return EXPR_OF(3072);                                          \
    case 4096: return EXPR_OF(4096);                                          \
    default: return EXPR_OF(0);                                               \
  }
template <typename R, int NB, int EPT>
static RowsFwdFn<R> rows_fwd_fn_t(int fix) {
#define K_OF(F) k_rows_fwd<R, NB, EPT, F>
  LLG_FIX_SWITCH(fix, K_OF)
#undef K_OF
}
template <typename R, int NB, int EPT>
static RowsInvFn<R> rows_inv_fn_t(int fix) {
#define K_OF(F) k_rows_inv<R, NB, EPT, F>
  LLG_FIX_SWITCH(fix, K_OF)
#undef K_OF
}
template <typename R, int EPT, bool ST, int CY>
static ColsFn<R> cols_fn_t(int fix) {
#define K_OF(F) k_cols_conv<R, EPT, ST, F, CY>
  LLG_FIX_SWITCH(fix, K_OF)
#undef K_OF
}
template <int EPT>
static ColsFwdFn cols_fwd_fn_t(int fix) {
#define K_OF(F) k_cols_fwd<EPT, F>
  LLG_FIX_SWITCH(fix, K_OF)
#undef K_OF
}
#undef LLG_FIX_SWITCH
template <typename R>
static RowsFwdFn<R> rows_fwd_fn(int fix, int nb, int ept) {
  if (nb == 1) return ept == 8 ? rows_fwd_fn_t<R, 1, 8>(fix) : rows_fwd_fn_t<R, 1, 16>(fix);
  return ept == 8 ? rows_fwd_fn_t<R, 2, 8>(fix) : rows_fwd_fn_t<R, 2, 16>(fix);
}
template <typename R>
static RowsInvFn<R> rows_inv_fn(int fix, int nb, int ept) {
  if (nb == 1) return ept == 8 ? rows_inv_fn_t<R, 1, 8>(fix) : rows_inv_fn_t<R, 1, 16>(fix);
  return ept == 8 ? rows_inv_fn_t<R, 2, 8>(fix) : rows_inv_fn_t<R, 2, 16>(fix);
}
template <typename R, int CY>
static ColsFn<R> cols_fn_cy(int fix, int ept, bool stage) {
  if (ept == 8) return stage ? cols_fn_t<R, 8, true, CY>(fix) : cols_fn_t<R, 8, false, CY>(fix);
  return stage ? cols_fn_t<R, 16, true, CY>(fix) : cols_fn_t<R, 16, false, CY>(fix);
}
template <typename R>
static ColsFn<R> cols_fn(int fix, int ept, bool stage, int cy = 3) {
  return cy == 3 ? cols_fn_cy<R, 3>(fix, ept, stage) : cols_fn_cy<R, 1>(fix, ept, stage);
}
static ColsFwdFn cols_fwd_fn(int fix, int ept) { return ept == 8 ? cols_fwd_fn_t<8>(fix) : cols_fwd_fn_t<16>(fix); }

// threads per block a kernel can be launched with (its register use)
static int max_threads(const void* fn) {
  cudaFuncAttributes at{};
  if (cudaFuncGetAttributes(&at, fn) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return at.maxThreadsPerBlock;
}

template <typename R>
static int launch_rows_fwd(const DemagPlan* d, cudaStream_t s, const double* in, long long cs, int row_len,
                           int nrows, const double* w, cx_t<R>* S, int ld, int ncomp, const LaunchCfg& k) {
  const FftPlanT<R> pl = d->fx.dev<R>();
  const size_t sm = sizeof(cx_t<R>) * (size_t)k.nb * padded_len<R>(d->px);
  const dim3 g((nrows + 2 * k.nb - 1) / (2 * k.nb), ncomp), b(d->fx.tx_for(k.ept), k.nb);
  klaunch(rows_fwd_fn<R>(d->fx.fix, k.nb, k.ept), g, b, sm, s, pl, in, cs, row_len, nrows, w, S, ld, d->hx);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

template <typename R>
static int launch_rows_inv(const DemagPlan* d, cudaStream_t s, const cx_t<R>* S, double* h, long long cs,
                           const LaunchCfg& k) {
  const FftPlanT<R> pl = d->fx.dev<R>();
  const size_t sm = sizeof(cx_t<R>) * (size_t)k.nb * padded_len<R>(d->px);
  const dim3 g((d->ny + 2 * k.nb - 1) / (2 * k.nb), 3), b(d->fx.tx_for(k.ept), k.nb);
  klaunch(rows_inv_fn<R>(d->fx.fix, k.nb, k.ept), g, b, sm, s, pl, S, d->ny, d->ny, d->hx, h, cs, d->ng);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

template <typename R>
static int launch_cols_conv(const DemagPlan* d, cudaStream_t s, cx_t<R>* S, const R* txx, const R* tyy,
                            const R* tzz, const cx_t<R>* txy, const LaunchCfg& k) {
  const FftPlanT<R> pl = d->fy.dev<R>();
  const dim3 b(d->fy.tx_for(k.ept), k.cy);
  const size_t base = sizeof(cx_t<R>) * 3 * (size_t)d->py;
  const size_t sm = k.stage ? base + (sizeof(R) * 3 + sizeof(cx_t<R>)) * (size_t)d->py : base;
  klaunch(cols_fn<R>(d->fy.fix, k.ept, k.stage, k.cy), d->hx, b, sm, s, pl, S, d->ny, d->ny, d->hx, txx, tyy, tzz,
          txy);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

static int launch_cols_fwd(const DemagPlan* d, cudaStream_t s, double2* S) {
  const FftPlan pl = d->fy.dev<double>();
  const size_t sm = sizeof(double2) * (size_t)d->py;
  klaunch(cols_fwd_fn(d->fy.fix, d->fy.ept), d->hx, dim3(d->fy.tx_for(d->fy.ept), 1), sm, s, pl, S, d->py, d->py,
          d->hx);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

template <typename R>
static bool rows_ok(const DemagPlan* d, int nb, int ept) {
  const int threads = d->fx.tx_for(ept) * nb;
  return threads <= 1024 && sizeof(cx_t<R>) * (size_t)nb * padded_len<R>(d->px) <= 227 * 1024 &&
         threads <= max_threads((const void*)rows_fwd_fn<R>(d->fx.fix, nb, ept)) &&
         threads <= max_threads((const void*)rows_inv_fn<R>(d->fx.fix, nb, ept));
}
template <typename R>
static size_t cols_smem(const DemagPlan* d, bool stage) {
  const size_t base = sizeof(cx_t<R>) * 3 * (size_t)d->py;
  return stage ? base + (sizeof(R) * 3 + sizeof(cx_t<R>)) * (size_t)d->py : base;
}
template <typename R>
static bool cols_ok(const DemagPlan* d, int ept, bool stage, int cy = 3) {
  const int threads = d->fy.tx_for(ept) * cy;
  if (threads > 1024 || threads > max_threads((const void*)cols_fn<R>(d->fy.fix, ept, stage, cy))) return false;
  if (!stage) return cols_smem<R>(d, false) <= 227 * 1024;
  return d->py % (int)(16 / sizeof(R)) == 0 && cols_smem<R>(d, true) <= 200 * 1024;
}

// opt in to the dynamic shared memory of every launch shape that fits
template <typename R>
static int set_smem_all(DemagPlan* d) {
  int rc;
  const size_t r1 = sizeof(cx_t<R>) * (size_t)padded_len<R>(d->px), r2 = 2 * r1;
  for (int nb = 1; nb <= 2; nb++)
    for (int ept = 8; ept <= 16; ept *= 2) {
      const size_t r = nb == 1 ? r1 : r2;
      if (r > 227 * 1024) continue;
      if ((rc = set_smem((const void*)rows_fwd_fn<R>(d->fx.fix, nb, ept), r)) ||
          (rc = set_smem((const void*)rows_inv_fn<R>(d->fx.fix, nb, ept), r)))
        return rc;
    }
  const size_t c0 = cols_smem<R>(d, false), c1 = cols_smem<R>(d, true);
  for (int ept = 8; ept <= 16; ept *= 2) {
    for (int cy = 3; cy >= 1; cy -= 2) {
      if ((rc = set_smem((const void*)cols_fn<R>(d->fy.fix, ept, false, cy), c0))) return rc;
      if (c1 <= 200 * 1024 && (rc = set_smem((const void*)cols_fn<R>(d->fy.fix, ept, true, cy), c1))) return rc;
    }
  }
  // default shapes (before tuning): one transform per CTA, fewest elements
  // per thread that the kernel's registers allow
  LaunchCfg& rw = d->rows[kp<R>()];
  LaunchCfg& cl = d->cols[kp<R>()];
  rw.nb = 1;
  rw.ept = rows_ok<R>(d, 1, 8) ? 8 : 16;
  cl.cy = 3;
  if (!cols_ok<R>(d, 8, false) && !cols_ok<R>(d, 16, false)) cl.cy = 1;   // long FP64 columns
  cl.ept = cols_ok<R>(d, 8, false, cl.cy) ? 8 : 16;
  cl.stage = cols_ok<R>(d, cl.ept, true, cl.cy);
  if (!rows_ok<R>(d, rw.nb, rw.ept) || !cols_ok<R>(d, cl.ept, false, cl.cy)) {
    llg_set_error("demag grid too large for the shared-memory transform");
    return LLG_ERR_NOTSUP;
  }
  return 0;
}

// ── autotuner: time every valid pair of row-transform and column launch
// shapes as the three-kernel chain on this plan's buffers, keep the fastest.
// All shapes compute bitwise-identical results (same butterflies, same
// operation order per element), so tuning never changes numerics.  Results
// are cached per (precision, transform size, grid) for later plans.
struct TuneKey {
  int prec, px, py, ny, ng;
  bool operator<(const TuneKey& o) const {
    return std::tie(prec, px, py, ny, ng) < std::tie(o.prec, o.px, o.py, o.ny, o.ng);
  }
};
static std::mutex g_tune_mu;
static std::map<TuneKey, std::pair<LaunchCfg, LaunchCfg>> g_tune;

template <typename R>
static int demag_autotune(llg_ctx* c, DemagPlan* d, cx_t<R>* S, const R* txx, const R* tyy, const R* tzz,
                          const cx_t<R>* txy, bool tune_cols) {
  const TuneKey key{kp<R>(), d->px, d->py, d->ny, d->ng};
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) {
      d->rows[kp<R>()] = it->second.first;
      if (tune_cols) d->cols[kp<R>()] = it->second.second;
      return 0;
    }
  }
  cudaStream_t s = c->stream;
  const long long cs = (long long)c->ncell;
  cudaEvent_t e0, e1;
  LLG_CUDA_TRY(cudaEventCreate(&e0));
  LLG_CUDA_TRY(cudaEventCreate(&e1));
  LaunchCfg best_r = d->rows[kp<R>()], best_c = d->cols[kp<R>()];
  std::vector<LaunchCfg> rcand, ccand;
  for (int nb = 1; nb <= 2; nb++)
    for (int ept = 8; ept <= 16; ept *= 2) {
      if (!rows_ok<R>(d, nb, ept)) continue;
      LaunchCfg k;
      k.nb = nb;
      k.ept = ept;
      rcand.push_back(k);
    }
  if (tune_cols) {
    // components in turn (cy = 1) only where no concurrent shape fits: it
    // ran slower in the stream for 1024-point FP64 columns
    const bool any3 = cols_ok<R>(d, 8, false) || cols_ok<R>(d, 16, false);
    for (int cy = 3; cy >= 1; cy -= 2)
      for (int ept = 8; ept <= 16; ept *= 2)
        for (int st = 0; st <= 1; st++) {
          if ((cy == 1 && any3) || !cols_ok<R>(d, ept, st != 0, cy)) continue;
          LaunchCfg k;
          k.ept = ept;
          k.stage = st != 0;
          k.cy = cy;
          ccand.push_back(k);
        }
  } else {
    ccand.push_back(best_c);   // (the tensor-core column stage, or the fixed shape)
  }
  // Every (rows, columns) pair is timed as the integrator issues it: the
  // three kernels back to back under programmatic dependent launch, so that
  // neighbours which cannot share an SM, or slow each other in the stream,
  // are seen (isolated per-kernel times picked shapes that ran slower there).
  auto chain = [&](const LaunchCfg& kr, const LaunchCfg& kc) -> int {
    int rc = launch_rows_fwd<R>(d, s, c->d_hd, cs, d->ng, d->ny, nullptr, S, d->ny, 3, kr);
    if (!rc) {
      if (!tune_cols && d->tc && sizeof(R) == 4) rc = demag_tc_cols(c, d->tc, reinterpret_cast<float2*>(S));
      else rc = launch_cols_conv<R>(d, s, S, txx, tyy, tzz, txy, kc);
    }
    return rc ? rc : launch_rows_inv<R>(d, s, S, c->d_pm, cs, kr);
  };
  float tbest = 1e30f;
  for (const LaunchCfg& kr : rcand)
    for (const LaunchCfg& kc : ccand) {
      if (chain(kr, kc)) continue;   // warm-up (plain launches)
      cudaEventRecord(e0, s);
      int bad = 0;
      {
        PdlScope pdl(true);
        for (int k = 0; k < 3 && !bad; k++) bad = chain(kr, kc);
      }
      cudaEventRecord(e1, s);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (!bad && ms < tbest) {
        tbest = ms;
        best_r = kr;
        best_c = kc;
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  LLG_CUDA_TRY(cudaGetLastError());
  d->rows[kp<R>()] = best_r;
  if (tune_cols) d->cols[kp<R>()] = best_c;
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune[key] = {best_r, tune_cols ? best_c : d->cols[kp<R>()]};
  return 0;
}

// FP64 tensor spectra -> FP32 copies for the mixed chain
__global__ void k_tensor_to_f32(const double* __restrict__ a, const double* __restrict__ b,
                                const double* __restrict__ c, const double2* __restrict__ xy, long long n,
                                float* __restrict__ af, float* __restrict__ bf, float* __restrict__ cf,
                                float2* __restrict__ xyf) {
  pdl_entry();
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
    af[e] = (float)a[e];
    bf[e] = (float)b[e];
    cf[e] = (float)c[e];
    xyf[e] = make_float2((float)xy[e].x, (float)xy[e].y);
  }
}

int demag_create(llg_ctx* c) {
  const llg_params& p = c->p;
  DemagPlan* d = new DemagPlan();
  d->ng = p.ng;
  d->ny = p.ny;
  d->open = (p.demag_mode == LLG_DEMAG_OPEN);
  d->px = d->open ? 2 * p.ng : p.ng;
  d->py = d->open ? 2 * p.ny : p.ny;
  d->hx = d->px / 2 + 1;
  d->strength = p.demag_strength;
  d->d_err = reinterpret_cast<int*>(c->d_scal + SLOT_TCERR);
  int rc = fft_init(d->fx, d->px, kRowsNB);
  if (!rc) rc = fft_init(d->fy, d->py, 3);
  if (rc) { demag_destroy(d); return rc; }
  d->mixed = (p.demag_precision == LLG_DEMAG_MIXED);
  if (d->fx.tx * kRowsNB > 1024 || sizeof(double2) * (size_t)d->py > 227 * 1024) {
    llg_set_error("demag grid too large for the shared-memory transform");
    demag_destroy(d);
    return LLG_ERR_NOTSUP;
  }
  if ((rc = set_smem_all<double>(d)) || (d->mixed && (rc = set_smem_all<float>(d))) ||
      (rc = set_smem((const void*)cols_fwd_fn(d->fy.fix, 8), sizeof(double2) * (size_t)d->py)) ||
      (rc = set_smem((const void*)cols_fwd_fn(d->fy.fix, 16), sizeof(double2) * (size_t)d->py))) {
    demag_destroy(d);
    return rc;
  }
  const long long np = (long long)d->px * d->py;
  const long long nspec = (long long)d->hx * d->py;
  LLG_CUDA_TRY(cudaMalloc(&d->d_S, sizeof(double2) * 3 * (size_t)d->hx * d->ny));
  LLG_CUDA_TRY(cudaMalloc(&d->d_txx, sizeof(double) * nspec));
  LLG_CUDA_TRY(cudaMalloc(&d->d_tyy, sizeof(double) * nspec));
  LLG_CUDA_TRY(cudaMalloc(&d->d_tzz, sizeof(double) * nspec));
  LLG_CUDA_TRY(cudaMalloc(&d->d_txy, sizeof(double2) * nspec));
  LLG_CUDA_TRY(cudaMalloc(&d->d_T, sizeof(double) * 9 * np));

  cudaStream_t s = c->stream;
  klaunch(k_newell, c->num_sms * 8, 128, 0, s, d->d_T, d->px, d->py, p.demag_thick, d->open);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  // N(0) (wrapped index 0)
  double n0[9];
  for (int k = 0; k < 9; k++)
    LLG_CUDA_TRY(cudaMemcpyAsync(&n0[k], d->d_T + k * np, sizeof(double), cudaMemcpyDeviceToHost, s));
  LLG_CUDA_TRY(cudaStreamSynchronize(s));
  d->n0[0] = n0[0];
  d->n0[1] = n0[4];
  d->n0[2] = n0[8];

  // spectra of all 9 components (real 2-D FFT: rows then columns)
  double2* spec = nullptr;
  LLG_CUDA_TRY(cudaMalloc(&spec, sizeof(double2) * 9 * (size_t)nspec));
  for (int k = 0; k < 9; k++) {
    LaunchCfg k1 = d->rows[kp<double>()];   // the default FP64 shape (one transform per CTA)
    if ((rc = launch_rows_fwd<double>(d, s, d->d_T + k * np, 0, d->px, d->py, nullptr, spec + k * nspec, d->py, 1,
                                      k1)) ||
        (rc = launch_cols_fwd(d, s, spec + k * nspec))) {
      cudaFree(spec);
      demag_destroy(d);
      return rc;
    }
  }
  const int nblk = 256;
  double* d_stats = nullptr;
  LLG_CUDA_TRY(cudaMalloc(&d_stats, sizeof(double) * 4 * nblk));
  const double scale = d->strength / (double)np;
  klaunch(k_tensor_finish, nblk, 256, 0, s, spec + 0 * nspec, spec + 4 * nspec, spec + 8 * nspec, spec + 1 * nspec,
                                       spec + 3 * nspec, spec + 2 * nspec, spec + 5 * nspec, spec + 6 * nspec,
                                       spec + 7 * nspec, nspec, scale, d->d_txx, d->d_tyy, d->d_tzz, d->d_txy,
                                       d_stats);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  std::vector<double> st(4 * nblk);
  LLG_CUDA_TRY(cudaMemcpyAsync(st.data(), d_stats, sizeof(double) * 4 * nblk, cudaMemcpyDeviceToHost, s));
  LLG_CUDA_TRY(cudaStreamSynchronize(s));
  cudaFree(d_stats);
  cudaFree(spec);
  double mx[4] = {0, 0, 0, 0};
  for (int b = 0; b < nblk; b++)
    for (int k = 0; k < 4; k++) mx[k] = std::max(mx[k], st[4 * b + k]);
  const double tol = 1e-10 * std::max(mx[0], 1e-300);
  if (mx[1] > tol || mx[2] > tol || mx[3] > tol) {
    char buf[256];
    snprintf(buf, sizeof buf,
             "demag tensor outside the film form: max|diag|=%.3e imag(diag)=%.3e |xz..|=%.3e |xy-yx|=%.3e", mx[0],
             mx[1], mx[2], mx[3]);
    llg_set_error(buf);
    c->demag = d;
    return LLG_ERR_NOTSUP;
  }
  if (d->mixed) {
    LLG_CUDA_TRY(cudaMalloc(&d->d_Sf, sizeof(float2) * 3 * (size_t)d->hx * d->ny));
    LLG_CUDA_TRY(cudaMalloc(&d->d_txxf, sizeof(float) * nspec));
    LLG_CUDA_TRY(cudaMalloc(&d->d_tyyf, sizeof(float) * nspec));
    LLG_CUDA_TRY(cudaMalloc(&d->d_tzzf, sizeof(float) * nspec));
    LLG_CUDA_TRY(cudaMalloc(&d->d_txyf, sizeof(float2) * nspec));
    klaunch(k_tensor_to_f32, c->num_sms * 4, 256, 0, s, d->d_txx, d->d_tyy, d->d_tzz, d->d_txy, nspec, d->d_txxf,
                                                   d->d_tyyf, d->d_tzzf, d->d_txyf);
    LLG_CUDA_TRY(cudaPeekAtLastError());
    // tensor-core column stage where the column shape allows it (else FP32 Stockham columns)
    if ((rc = demag_tc_create(c, d->px, d->py, d->hx, d->ny, d->d_txxf, d->d_tyyf, d->d_tzzf, d->d_txyf, &d->tc))) {
      c->demag = d;
      return rc;
    }
    if ((rc = demag_autotune<float>(c, d, d->d_Sf, d->d_txxf, d->d_tyyf, d->d_tzzf, d->d_txyf, d->tc == nullptr))) {
      c->demag = d;
      return rc;
    }
  } else if ((rc = demag_autotune<double>(c, d, d->d_S, d->d_txx, d->d_tyy, d->d_tzz, d->d_txy, true))) {
    c->demag = d;
    return rc;
  }
  c->demag = d;
  return 0;
}

// stage 0 rows_fwd, 1 column convolution, 2 rows_inv; FP64 or mixed chain
static int demag_run_stage_raw(llg_ctx* c, DemagPlan* d, int stage, const double* y, const double* w, double* h) {
  const long long cs = (long long)c->ncell;
  if (stage == 0) {
    LLG_COUNT(KID_DEMAG_ROWS_FWD);
    if (d->mixed) return launch_rows_fwd<float>(d, c->stream, y, cs, d->ng, d->ny, w, d->d_Sf, d->ny, 3, d->rows[1]);
    return launch_rows_fwd<double>(d, c->stream, y, cs, d->ng, d->ny, w, d->d_S, d->ny, 3, d->rows[0]);
  }
  if (stage == 1) {
    LLG_COUNT(KID_DEMAG_COLS);
    if (d->mixed) {
      if (d->tc) return demag_tc_cols(c, d->tc, d->d_Sf);
      return launch_cols_conv<float>(d, c->stream, d->d_Sf, d->d_txxf, d->d_tyyf, d->d_tzzf, d->d_txyf, d->cols[1]);
    }
    return launch_cols_conv<double>(d, c->stream, d->d_S, d->d_txx, d->d_tyy, d->d_tzz, d->d_txy, d->cols[0]);
  }
  LLG_COUNT(KID_DEMAG_ROWS_INV);
  if (d->mixed) return launch_rows_inv<float>(d, c->stream, d->d_Sf, h, cs, d->rows[1]);
  return launch_rows_inv<double>(d, c->stream, d->d_S, h, cs, d->rows[0]);
}

// (timed when the family's live kernel timer is on)
static int demag_run_stage(llg_ctx* c, DemagPlan* d, int stage, const double* y, const double* w, double* h) {
  const int kid = (stage == 0) ? KID_DEMAG_ROWS_FWD : (stage == 1) ? KID_DEMAG_COLS : KID_DEMAG_ROWS_INV;
  ktimer_mark(c, kid, true);
  const int rc = demag_run_stage_raw(c, d, stage, y, w, h);
  ktimer_mark(c, kid, false);
  return rc;
}

int demag_apply(llg_ctx* c, const double* y, double* h) {
  return demag_apply_w(c, y, c->p.windowed ? c->d_w : nullptr, h);
}

int demag_apply_w(llg_ctx* c, const double* y, const double* w, double* h) {
  DemagPlan* d = c->demag;
  if (!d) {
    LLG_CUDA_TRY(cudaMemsetAsync(h, 0, sizeof(double) * 3 * (size_t)c->ncell, c->stream));
    return 0;
  }
  int rc;
  // legacy default stream, or inside the device-resident step graph's capture:
  // launch the stages directly
  if (c->stream == nullptr || c->capturing) {
    for (int stage = 0; stage < 3; stage++)
      if ((rc = demag_run_stage(c, d, stage, y, w, h))) return rc;
    return 0;
  }
  // On a context's own stream the three-kernel chain runs as one CUDA graph,
  // captured on first use for these (y, w, h) buffers and replayed after.
  if (!(d->gexec && d->gkey[0] == y && d->gkey[1] == w && d->gkey[2] == h)) {
    if (d->gexec) { cudaGraphExecDestroy(d->gexec); d->gexec = nullptr; }
    cudaGraph_t graph = nullptr;
    LLG_CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    rc = 0;
    const int pdl_saved = g_no_pdl;
    g_no_pdl = 1;
    for (int stage = 0; stage < 3 && rc == 0; stage++) rc = demag_run_stage(c, d, stage, y, w, h);
    g_no_pdl = pdl_saved;
    const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
    // the capture launched nothing; the replay below is counted instead
    g_kcount[KID_DEMAG_ROWS_FWD].fetch_sub(1);
    g_kcount[KID_DEMAG_COLS].fetch_sub(1);
    g_kcount[KID_DEMAG_ROWS_INV].fetch_sub(1);
    if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
    LLG_CUDA_TRY(ce);
    const cudaError_t ie = cudaGraphInstantiate(&d->gexec, graph, 0);
    cudaGraphDestroy(graph);
    LLG_CUDA_TRY(ie);
    d->gkey[0] = y;
    d->gkey[1] = w;
    d->gkey[2] = h;
  }
  LLG_COUNT(KID_DEMAG_ROWS_FWD);
  LLG_COUNT(KID_DEMAG_COLS);
  LLG_COUNT(KID_DEMAG_ROWS_INV);
  LLG_CUDA_TRY(cudaGraphLaunch(d->gexec, c->stream));
  return 0;
}

// one stage of the chain alone (profiling): 0 rows_fwd, 1 cols_conv, 2 rows_inv
int demag_stage(llg_ctx* c, int stage, const double* y, double* h) {
  DemagPlan* d = c->demag;
  if (!d) return LLG_ERR_STATE;
  return demag_run_stage(c, d, stage, y, c->p.windowed ? c->d_w : nullptr, h);
}

// a plan whose kernels wait on asynchronous completions (the tensor-core
// column stage) can have set the flag
static bool demag_waits(const DemagPlan* d) { return d && d->tc; }

int demag_check(llg_ctx* c) {
  if (!demag_waits(c->demag)) return 0;
  int f = 0;
  cudaMemcpyAsync(&f, c->demag->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  cudaStreamSynchronize(c->stream);
  if (f) {
    llg_set_error("demag: a tensor-core completion wait ran out (results invalid)");
    return LLG_ERR_TIMEOUT;
  }
  return 0;
}

int demag_check_last(llg_ctx* c) {
  if (!demag_waits(c->demag)) return 0;
  int f = 0;
  memcpy(&f, c->h_scal + SLOT_TCERR, sizeof(int));
  if (f) {
    llg_set_error("demag: a tensor-core completion wait ran out (results invalid)");
    return LLG_ERR_TIMEOUT;
  }
  return 0;
}

int demag_dims(llg_ctx* c, int out[4]) {
  DemagPlan* d = c->demag;
  if (!d) return LLG_ERR_STATE;
  out[0] = d->px; out[1] = d->py; out[2] = d->hx; out[3] = d->ny;
  return 0;
}

int demag_self(llg_ctx* c, double out3[3]) {
  if (!c->demag) { out3[0] = out3[1] = out3[2] = 0.0; return 0; }
  for (int a = 0; a < 3; a++) out3[a] = c->demag->n0[a] * c->demag->strength;
  return 0;
}

int demag_tensor_host(llg_ctx* c, int comp, int dx, int dy, double* out) {
  DemagPlan* d = c->demag;
  if (!d || comp < 0 || comp > 8) { *out = 0.0; return d ? LLG_ERR_ARG : 0; }
  const int wx = ((dx % d->px) + d->px) % d->px, wy = ((dy % d->py) + d->py) % d->py;
  const long long np = (long long)d->px * d->py;
  LLG_CUDA_TRY(cudaMemcpy(out, d->d_T + comp * np + (long long)wy * d->px + wx, sizeof(double),
                          cudaMemcpyDeviceToHost));
  return 0;
}
