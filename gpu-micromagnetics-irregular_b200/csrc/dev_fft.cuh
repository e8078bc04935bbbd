// dev_fft.cuh — shared-memory Stockham FFT core, templated on the real type
// (double for the FP64 demag chain, float for the mixed-precision chain).
//
// Natural order in and out, no reordering tables: each pass stages the
// thread's radix-R butterflies (R = 8/4/2/3/5; any other prime through a
// generic path) in registers, synchronises, applies twiddles and the
// in-register DFT, and scatters to (j / Ns)·Ns·R + j % Ns + r·Ns.
#pragma once
#include <cuda_runtime.h>

namespace {

constexpr int MAXR = 24;  // passes

template <typename R> struct Cx;
template <> struct Cx<double> { using T = double2; };
template <> struct Cx<float> { using T = float2; };
template <typename R> using cx_t = typename Cx<R>::T;

template <typename R>
__device__ __forceinline__ cx_t<R> mk(R a, R b) {
  cx_t<R> v;
  v.x = a;
  v.y = b;
  return v;
}

// Stockham plan for one transform length n.  Radices in pass order
// (8/4/2 first so every power-of-two pass sees a power-of-two span Ns, then
// 3, 5 and any other prime).  tx = threads per transform.
template <typename R>
struct FftPlanT {
  int n, nr, tx;
  const int4* pass;     // per pass: (radix R, span Ns before the pass, log2 Ns or -1, 0)
  const cx_t<R>* tw;    // tw[k] = exp(-2 pi i k / n)
};

// Padded transform buffers (PAD = true): one unused element after every 128
// bytes, so the small-span Stockham scatters (stride R or R*Ns elements
// across a warp) spread over all banks instead of a few.
template <typename R, bool PAD>
__device__ __forceinline__ int fpad(int i) {
  if constexpr (PAD) return i + (i >> (sizeof(R) == 8 ? 3 : 4));
  else return i;
}
template <typename R>
__host__ __device__ constexpr int padded_len(int n) { return n + (n >> (sizeof(R) == 8 ? 3 : 4)) + 1; }

template <typename R>
__device__ __forceinline__ cx_t<R> cmul(cx_t<R> a, cx_t<R> b) {
  return mk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename R>
__device__ __forceinline__ cx_t<R> cadd(cx_t<R> a, cx_t<R> b) { return mk<R>(a.x + b.x, a.y + b.y); }
template <typename R>
__device__ __forceinline__ cx_t<R> csub(cx_t<R> a, cx_t<R> b) { return mk<R>(a.x - b.x, a.y - b.y); }
// v * (SIGN < 0 ? -i : +i)
template <typename R, int SIGN>
__device__ __forceinline__ cx_t<R> rot90(cx_t<R> v) {
  return (SIGN < 0) ? mk<R>(v.y, -v.x) : mk<R>(-v.y, v.x);
}

template <typename R, int SIGN>
__device__ __forceinline__ cx_t<R> twid(const FftPlanT<R>& pl, int idx) {
  cx_t<R> w = __ldg(&pl.tw[idx]);
  if (SIGN > 0) w.y = -w.y;
  return w;
}

// in-register DFTs, out[q] = sum_r v[r] exp(SIGN 2 pi i r q / R)
template <typename R, int SIGN>
__device__ __forceinline__ void dft2(cx_t<R>* v) {
  const cx_t<R> a = v[0], b = v[1];
  v[0] = cadd<R>(a, b);
  v[1] = csub<R>(a, b);
}
template <typename R, int SIGN>
__device__ __forceinline__ void dft4(cx_t<R>* v) {
  const cx_t<R> a0 = cadd<R>(v[0], v[2]), a1 = csub<R>(v[0], v[2]);
  const cx_t<R> b0 = cadd<R>(v[1], v[3]), b1 = rot90<R, SIGN>(csub<R>(v[1], v[3]));
  v[0] = cadd<R>(a0, b0);
  v[2] = csub<R>(a0, b0);
  v[1] = cadd<R>(a1, b1);
  v[3] = csub<R>(a1, b1);
}
template <typename R, int SIGN>
__device__ __forceinline__ void dft3(cx_t<R>* v) {
  const R c = R(-0.5), s = R(SIGN) * R(0.86602540378443864676);  // sin(2pi/3)
  const cx_t<R> t1 = cadd<R>(v[1], v[2]), t2 = csub<R>(v[1], v[2]);
  const cx_t<R> a = mk<R>(v[0].x + c * t1.x, v[0].y + c * t1.y);
  const cx_t<R> b = mk<R>(-s * t2.y, s * t2.x);  // i*s*t2
  v[0] = cadd<R>(v[0], t1);
  v[1] = cadd<R>(a, b);
  v[2] = csub<R>(a, b);
}
template <typename R, int SIGN>
__device__ __forceinline__ void dft5(cx_t<R>* v) {
  const R c1 = R(0.30901699437494742410), c2 = R(-0.80901699437494742410);
  const R s1 = R(SIGN) * R(0.95105651629515357212), s2 = R(SIGN) * R(0.58778525229247312917);
  const cx_t<R> t1 = cadd<R>(v[1], v[4]), t2 = cadd<R>(v[2], v[3]);
  const cx_t<R> t3 = csub<R>(v[1], v[4]), t4 = csub<R>(v[2], v[3]);
  const cx_t<R> a1 = mk<R>(v[0].x + c1 * t1.x + c2 * t2.x, v[0].y + c1 * t1.y + c2 * t2.y);
  const cx_t<R> a2 = mk<R>(v[0].x + c2 * t1.x + c1 * t2.x, v[0].y + c2 * t1.y + c1 * t2.y);
  const cx_t<R> b1 = mk<R>(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
  const cx_t<R> b2 = mk<R>(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
  v[0] = mk<R>(v[0].x + t1.x + t2.x, v[0].y + t1.y + t2.y);
  v[1] = mk<R>(a1.x - b1.y, a1.y + b1.x);
  v[4] = mk<R>(a1.x + b1.y, a1.y - b1.x);
  v[2] = mk<R>(a2.x - b2.y, a2.y + b2.x);
  v[3] = mk<R>(a2.x + b2.y, a2.y - b2.x);
}
template <typename R, int SIGN>
__device__ __forceinline__ void dft8(cx_t<R>* v) {
  const R h = R(0.70710678118654752440);
  cx_t<R> e[4] = {v[0], v[2], v[4], v[6]};
  cx_t<R> o[4] = {v[1], v[3], v[5], v[7]};
  dft4<R, SIGN>(e);
  dft4<R, SIGN>(o);
  const cx_t<R> o1 = mk<R>(h * (o[1].x - SIGN * o[1].y), h * (o[1].y + SIGN * o[1].x));
  const cx_t<R> o2 = rot90<R, SIGN>(o[2]);
  const cx_t<R> o3 = mk<R>(-h * (o[3].x + SIGN * o[3].y), h * (SIGN * o[3].x - o[3].y));
  v[0] = cadd<R>(e[0], o[0]);
  v[4] = csub<R>(e[0], o[0]);
  v[1] = cadd<R>(e[1], o1);
  v[5] = csub<R>(e[1], o1);
  v[2] = cadd<R>(e[2], o2);
  v[6] = csub<R>(e[2], o2);
  v[3] = cadd<R>(e[3], o3);
  v[7] = csub<R>(e[3], o3);
}
template <typename R, int RAD, int SIGN>
__device__ __forceinline__ void dft_fixed(cx_t<R>* v) {
  if constexpr (RAD == 2) dft2<R, SIGN>(v);
  else if constexpr (RAD == 3) dft3<R, SIGN>(v);
  else if constexpr (RAD == 4) dft4<R, SIGN>(v);
  else if constexpr (RAD == 5) dft5<R, SIGN>(v);
  else if constexpr (RAD == 8) dft8<R, SIGN>(v);
}

// One Stockham pass of one transform held in buf[0..n).  All threads of the
// row stage their butterflies in registers, the block synchronises, then
// twiddle + DFT_R + scatter to (j / Ns)·Ns·R + j % Ns + r·Ns.
// A row of tx threads covers n/R butterflies with at most MB each
// (tx >= n/EPT is guaranteed by the plan).
template <typename R, int RAD, int SIGN, int EPT, bool PAD>
__device__ __forceinline__ void stockham_pass(cx_t<R>* buf, const FftPlanT<R>& pl, int4 ps) {
  constexpr int MB = (EPT + RAD - 1) / RAD;
  const int n = pl.n, nb = n / RAD, Ns = ps.y, lg = ps.z;
  const int tstride = n / (Ns * RAD);
  cx_t<R> v[MB][RAD];
#pragma unroll
  for (int u = 0; u < MB; u++) {
    const int j = threadIdx.x + u * blockDim.x;
    if (j < nb) {
#pragma unroll
      for (int r = 0; r < RAD; r++) v[u][r] = buf[fpad<R, PAD>(j + r * nb)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < MB; u++) {
    const int j = threadIdx.x + u * blockDim.x;
    if (j < nb) {
      int q, jm;
      if (lg >= 0) { q = j >> lg; jm = j & (Ns - 1); }
      else { q = j / Ns; jm = j - q * Ns; }
      if (Ns > 1 && jm != 0) {
        // one table load per butterfly; higher powers in registers
        const cx_t<R> w1 = twid<R, SIGN>(pl, jm * tstride);
        cx_t<R> wr = w1;
#pragma unroll
        for (int r = 1; r < RAD; r++) {
          v[u][r] = cmul<R>(v[u][r], wr);
          if (r + 1 < RAD) wr = cmul<R>(wr, w1);
        }
      }
      dft_fixed<R, RAD, SIGN>(v[u]);
      const int ob = q * Ns * RAD + jm;
#pragma unroll
      for (int r = 0; r < RAD; r++) buf[fpad<R, PAD>(ob + r * Ns)] = v[u][r];
    }
  }
  __syncthreads();
}

// Any other radix (small primes, test sizes only): one butterfly per thread
// (the plan sizes tx >= n/R), R <= 64, O(R^2).
template <typename R, int SIGN, bool PAD>
__device__ void stockham_pass_generic(cx_t<R>* buf, const FftPlanT<R>& pl, int4 ps) {
  const int RAD = ps.x;
  const int n = pl.n, nb = n / RAD, Ns = ps.y;
  const int tstride = n / (Ns * RAD), rstride = n / RAD;
  const int j = threadIdx.x;
  cx_t<R> v[64];
  if (j < nb) {
    for (int r = 0; r < RAD; r++) v[r] = buf[fpad<R, PAD>(j + r * nb)];
  }
  __syncthreads();
  if (j < nb) {
    const int q = j / Ns, jm = j - q * Ns;
    for (int r = 1; r < RAD; r++) v[r] = cmul<R>(v[r], twid<R, SIGN>(pl, jm * r * tstride));
    const int ob = q * Ns * RAD + jm;
    for (int k = 0; k < RAD; k++) {
      cx_t<R> acc = v[0];
      for (int r = 1; r < RAD; r++) acc = cadd<R>(acc, cmul<R>(v[r], twid<R, SIGN>(pl, ((r * k) % RAD) * rstride)));
      buf[fpad<R, PAD>(ob + k * Ns)] = acc;
    }
  }
  __syncthreads();
}

// Natural-order in, natural-order out, in place in buf (this row's transform).
// Every thread of the block must call it (it synchronises).  The passes run
// as straight-line regions in factorisation order (8s, one 4, one 2, 3s, 5s,
// other primes): a runtime switch over radices inside one loop makes the
// register allocator keep every variant's state live at once.
template <typename R, int SIGN, int EPT, bool PAD = false>
__device__ void fft_stockham(cx_t<R>* buf, const FftPlanT<R>& pl) {
  int p = 0;
  for (; p < pl.nr && __ldg(&pl.pass[p].x) == 8; p++) stockham_pass<R, 8, SIGN, EPT, PAD>(buf, pl, __ldg(&pl.pass[p]));
  if (p < pl.nr && __ldg(&pl.pass[p].x) == 4) { stockham_pass<R, 4, SIGN, EPT, PAD>(buf, pl, __ldg(&pl.pass[p])); p++; }
  if (p < pl.nr && __ldg(&pl.pass[p].x) == 2) { stockham_pass<R, 2, SIGN, EPT, PAD>(buf, pl, __ldg(&pl.pass[p])); p++; }
  for (; p < pl.nr && __ldg(&pl.pass[p].x) == 3; p++) stockham_pass<R, 3, SIGN, EPT, PAD>(buf, pl, __ldg(&pl.pass[p]));
  for (; p < pl.nr && __ldg(&pl.pass[p].x) == 5; p++) stockham_pass<R, 5, SIGN, EPT, PAD>(buf, pl, __ldg(&pl.pass[p]));
  for (; p < pl.nr; p++) stockham_pass_generic<R, SIGN, PAD>(buf, pl, __ldg(&pl.pass[p]));
}

}  // namespace
