// dev_fft.cuh — shared-memory Stockham FFT core, templated on the real type
// (double for the FP64 demag chain, float for the mixed-precision chain).
//
// Natural order in and out, no reordering tables: each pass stages the
// thread's radix-R butterflies (R = 16/8/4/2, 12/6, 3, 5; any other prime
// through a generic path) in registers, synchronises, applies twiddles and the
// in-register DFT, and scatters to (j / Ns)·Ns·R + j % Ns + r·Ns.  A length
// runs either a runtime plan (pass table in device memory) or, for the
// lengths of kFixedLengths, a compile-time plan whose passes, spans and
// shifts are constants of its kernel.
#pragma once
#include <cuda_runtime.h>

namespace {

constexpr int MAXR = 24;  // passes

template <typename R> struct Cx;
template <> struct Cx<double> { using T = double2; };
template <> struct Cx<float> { using T = float2; };
template <typename R> using cx_t = typename Cx<R>::T;

#define FFT_HD __host__ __device__ __forceinline__

template <typename R>
FFT_HD cx_t<R> mk(R a, R b) {
  cx_t<R> v;
  v.x = a;
  v.y = b;
  return v;
}

// Stockham plan for one transform length n: the runtime pass table
// (runtime_radices: 8/4/2 first so every power-of-two pass sees a
// power-of-two span Ns, then 3, 5 and any other prime) and the twiddles, which
// a compile-time plan uses too.  tx = threads per transform.
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
FFT_HD cx_t<R> cmul(cx_t<R> a, cx_t<R> b) {
  return mk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename R>
FFT_HD cx_t<R> cadd(cx_t<R> a, cx_t<R> b) { return mk<R>(a.x + b.x, a.y + b.y); }
template <typename R>
FFT_HD cx_t<R> csub(cx_t<R> a, cx_t<R> b) { return mk<R>(a.x - b.x, a.y - b.y); }
// v * (SIGN < 0 ? -i : +i)
template <typename R, int SIGN>
FFT_HD cx_t<R> rot90(cx_t<R> v) {
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
FFT_HD void dft2(cx_t<R>* v) {
  const cx_t<R> a = v[0], b = v[1];
  v[0] = cadd<R>(a, b);
  v[1] = csub<R>(a, b);
}
template <typename R, int SIGN>
FFT_HD void dft4(cx_t<R>* v) {
  const cx_t<R> a0 = cadd<R>(v[0], v[2]), a1 = csub<R>(v[0], v[2]);
  const cx_t<R> b0 = cadd<R>(v[1], v[3]), b1 = rot90<R, SIGN>(csub<R>(v[1], v[3]));
  v[0] = cadd<R>(a0, b0);
  v[2] = csub<R>(a0, b0);
  v[1] = cadd<R>(a1, b1);
  v[3] = csub<R>(a1, b1);
}
template <typename R, int SIGN>
FFT_HD void dft3(cx_t<R>* v) {
  const R c = R(-0.5), s = R(SIGN) * R(0.86602540378443864676);  // sin(2pi/3)
  const cx_t<R> t1 = cadd<R>(v[1], v[2]), t2 = csub<R>(v[1], v[2]);
  const cx_t<R> a = mk<R>(v[0].x + c * t1.x, v[0].y + c * t1.y);
  const cx_t<R> b = mk<R>(-s * t2.y, s * t2.x);  // i*s*t2
  v[0] = cadd<R>(v[0], t1);
  v[1] = cadd<R>(a, b);
  v[2] = csub<R>(a, b);
}
template <typename R, int SIGN>
FFT_HD void dft5(cx_t<R>* v) {
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
FFT_HD void dft8(cx_t<R>* v) {
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
// v * (c + SIGN i s), a constant rotation
template <typename R, int SIGN>
FFT_HD cx_t<R> crot(cx_t<R> v, R c, R s) {
  const R ss = R(SIGN) * s;
  return mk<R>(v.x * c - v.y * ss, v.x * ss + v.y * c);
}
// Composite radices as two in-register stages (Cooley-Tukey, R = A x B):
// index r = B n1 + n2, frequency q = k1 + A k2; the inner DFT_A runs over n1
// for every n2, the products take the constant twiddles w_R^(n2 k1), the
// outer DFT_B runs over n2 for every k1.
template <typename R, int SIGN>
FFT_HD void dft6(cx_t<R>* v) {   // 6 = 2 x 3
  const R h = R(0.5), t = R(0.86602540378443864676);   // cos, sin of 2 pi / 6
  cx_t<R> a[3][2];
#pragma unroll
  for (int n2 = 0; n2 < 3; n2++) {
    a[n2][0] = v[n2];
    a[n2][1] = v[3 + n2];
    dft2<R, SIGN>(a[n2]);
  }
  a[1][1] = crot<R, SIGN>(a[1][1], h, t);      // w6^1
  a[2][1] = crot<R, SIGN>(a[2][1], -h, t);     // w6^2
#pragma unroll
  for (int k1 = 0; k1 < 2; k1++) {
    cx_t<R> b[3] = {a[0][k1], a[1][k1], a[2][k1]};
    dft3<R, SIGN>(b);
#pragma unroll
    for (int k2 = 0; k2 < 3; k2++) v[k1 + 2 * k2] = b[k2];
  }
}
template <typename R, int SIGN>
FFT_HD void dft12(cx_t<R>* v) {  // 12 = 4 x 3
  const R h = R(0.5), t = R(0.86602540378443864676);   // cos, sin of 2 pi / 6
  cx_t<R> a[3][4];
#pragma unroll
  for (int n2 = 0; n2 < 3; n2++) {
#pragma unroll
    for (int n1 = 0; n1 < 4; n1++) a[n2][n1] = v[3 * n1 + n2];
    dft4<R, SIGN>(a[n2]);
  }
  a[1][1] = crot<R, SIGN>(a[1][1], t, h);      // w12^1
  a[1][2] = crot<R, SIGN>(a[1][2], h, t);      // w12^2
  a[1][3] = rot90<R, SIGN>(a[1][3]);           // w12^3
  a[2][1] = crot<R, SIGN>(a[2][1], h, t);      // w12^2
  a[2][2] = crot<R, SIGN>(a[2][2], -h, t);     // w12^4
  a[2][3] = mk<R>(-a[2][3].x, -a[2][3].y);     // w12^6
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    cx_t<R> b[3] = {a[0][k1], a[1][k1], a[2][k1]};
    dft3<R, SIGN>(b);
#pragma unroll
    for (int k2 = 0; k2 < 3; k2++) v[k1 + 4 * k2] = b[k2];
  }
}
template <typename R, int SIGN>
FFT_HD void dft16(cx_t<R>* v) {  // 16 = 4 x 4
  const R c1 = R(0.92387953251128675613), s1 = R(0.38268343236508977173);   // cos, sin of pi / 8
  const R h = R(0.70710678118654752440);
  cx_t<R> a[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; n2++) {
#pragma unroll
    for (int n1 = 0; n1 < 4; n1++) a[n2][n1] = v[4 * n1 + n2];
    dft4<R, SIGN>(a[n2]);
  }
  a[1][1] = crot<R, SIGN>(a[1][1], c1, s1);    // w16^1
  a[1][2] = crot<R, SIGN>(a[1][2], h, h);      // w16^2
  a[1][3] = crot<R, SIGN>(a[1][3], s1, c1);    // w16^3
  a[2][1] = crot<R, SIGN>(a[2][1], h, h);      // w16^2
  a[2][2] = rot90<R, SIGN>(a[2][2]);           // w16^4
  a[2][3] = crot<R, SIGN>(a[2][3], -h, h);     // w16^6
  a[3][1] = crot<R, SIGN>(a[3][1], s1, c1);    // w16^3
  a[3][2] = crot<R, SIGN>(a[3][2], -h, h);     // w16^6
  a[3][3] = crot<R, SIGN>(a[3][3], -c1, -s1);  // w16^9
#pragma unroll
  for (int k1 = 0; k1 < 4; k1++) {
    cx_t<R> b[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
    dft4<R, SIGN>(b);
#pragma unroll
    for (int k2 = 0; k2 < 4; k2++) v[k1 + 4 * k2] = b[k2];
  }
}
template <typename R, int RAD, int SIGN>
FFT_HD void dft_fixed(cx_t<R>* v) {
  if constexpr (RAD == 2) dft2<R, SIGN>(v);
  else if constexpr (RAD == 3) dft3<R, SIGN>(v);
  else if constexpr (RAD == 4) dft4<R, SIGN>(v);
  else if constexpr (RAD == 5) dft5<R, SIGN>(v);
  else if constexpr (RAD == 6) dft6<R, SIGN>(v);
  else if constexpr (RAD == 8) dft8<R, SIGN>(v);
  else if constexpr (RAD == 12) dft12<R, SIGN>(v);
  else if constexpr (RAD == 16) dft16<R, SIGN>(v);
}

// v[r] *= w^(r * jm * tstride), r = 1..RAD-1 (the twiddles of butterfly jm
// of a pass with span Ns; r * jm * tstride < n for r < RAD)
template <typename R, int RAD, int SIGN>
__device__ __forceinline__ void apply_twiddles(cx_t<R>* v, const FftPlanT<R>& pl, int jm, int tstride) {
  if constexpr (RAD <= 8) {
    // one table load per butterfly; higher powers in registers
    const cx_t<R> w1 = twid<R, SIGN>(pl, jm * tstride);
    cx_t<R> wr = w1;
#pragma unroll
    for (int r = 1; r < RAD; r++) {
      v[r] = cmul<R>(v[r], wr);
      if (r + 1 < RAD) wr = cmul<R>(wr, w1);
    }
  } else {
    // w^1, w^2, w^4, w^8 from the table; every other power is a product of
    // at most three of them, so no power carries a long chain of roundings
    const int b = jm * tstride;
    const cx_t<R> w1 = twid<R, SIGN>(pl, b), w2 = twid<R, SIGN>(pl, 2 * b);
    const cx_t<R> w4 = twid<R, SIGN>(pl, 4 * b), w8 = twid<R, SIGN>(pl, 8 * b);
#pragma unroll
    for (int r = 1; r < RAD; r++) {
      cx_t<R> wr;
      bool have = false;
      if (r & 1) { wr = w1; have = true; }
      if (r & 2) { wr = have ? cmul<R>(wr, w2) : w2; have = true; }
      if (r & 4) { wr = have ? cmul<R>(wr, w4) : w4; have = true; }
      if (r & 8) { wr = have ? cmul<R>(wr, w8) : w8; }
      v[r] = cmul<R>(v[r], wr);
    }
  }
}

// One Stockham pass of one transform of length n held in buf[0..n), span Ns
// (lg = log2 Ns, or -1).  All threads of the row stage their butterflies in
// registers, the block synchronises, then twiddle + DFT_R + scatter to
// (j / Ns)·Ns·R + j % Ns + r·Ns.  A row of tx threads covers n/R butterflies
// with at most MB each (tx >= n/EPT is guaranteed by the plan).  n, Ns and
// lg are arguments so that a compile-time plan (fft_fixed) folds them.
template <typename R, int RAD, int SIGN, int EPT, bool PAD>
__device__ __forceinline__ void stockham_pass_n(cx_t<R>* buf, const FftPlanT<R>& pl, int n, int Ns, int lg,
                                                int tx = threadIdx.x) {
  constexpr int MB = (EPT + RAD - 1) / RAD;
  const int nb = n / RAD;
  const int tstride = n / (Ns * RAD);
  cx_t<R> v[MB][RAD];
#pragma unroll
  for (int u = 0; u < MB; u++) {
    const int j = tx + u * blockDim.x;
    if (j < nb) {
#pragma unroll
      for (int r = 0; r < RAD; r++) v[u][r] = buf[fpad<R, PAD>(j + r * nb)];
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < MB; u++) {
    const int j = tx + u * blockDim.x;
    if (j < nb) {
      int q, jm;
      if (lg >= 0) { q = j >> lg; jm = j & (Ns - 1); }
      else { q = j / Ns; jm = j - q * Ns; }
      if (Ns > 1 && jm != 0) apply_twiddles<R, RAD, SIGN>(v[u], pl, jm, tstride);
      dft_fixed<R, RAD, SIGN>(v[u]);
      const int ob = q * Ns * RAD + jm;
#pragma unroll
      for (int r = 0; r < RAD; r++) buf[fpad<R, PAD>(ob + r * Ns)] = v[u][r];
    }
  }
  __syncthreads();
}
template <typename R, int RAD, int SIGN, int EPT, bool PAD>
__device__ __forceinline__ void stockham_pass(cx_t<R>* buf, const FftPlanT<R>& pl, int4 ps) {
  stockham_pass_n<R, RAD, SIGN, EPT, PAD>(buf, pl, pl.n, ps.y, ps.z);
}

// The first pass (span 1: no twiddles, butterfly j writes j·R .. j·R + R-1)
// with its inputs taken from ld(i) instead of from buf, so the input never
// makes a round trip through shared memory.  HALF: the inputs i >= n/2 are
// known to be zero (an open-boundary row, zero-padded to twice its length)
// and the butterflies' upper halves are not loaded or computed.
template <typename R, int RAD, int SIGN, int EPT, bool PAD, bool HALF, typename LD>
__device__ __forceinline__ void stockham_first_pass_ld(cx_t<R>* buf, int n, LD&& ld, int tx = threadIdx.x) {
  constexpr int MB = (EPT + RAD - 1) / RAD;
  static_assert(!HALF || RAD % 2 == 0, "HALF needs an even radix");
  const int nb = n / RAD;
#pragma unroll
  for (int u = 0; u < MB; u++) {
    const int j = tx + u * blockDim.x;
    if (j < nb) {
      cx_t<R> v[RAD];
#pragma unroll
      for (int r = 0; r < RAD; r++) v[r] = (HALF && 2 * r >= RAD) ? mk<R>(R(0), R(0)) : ld(j + r * nb);
      dft_fixed<R, RAD, SIGN>(v);
#pragma unroll
      for (int r = 0; r < RAD; r++) buf[fpad<R, PAD>(j * RAD + r)] = v[r];
    }
  }
  __syncthreads();
}

// The last pass (span n/R: butterfly j = jm writes jm + r·n/R) with its
// outputs handed to st(i, value) instead of written back to buf.  HALF: only
// the outputs i < n/2 are wanted (the kept half of an open-boundary row), so
// the upper half of every butterfly is not stored.  buf is only read: no
// barrier follows.
template <typename R, int RAD, int SIGN, int EPT, bool PAD, bool HALF, typename ST>
__device__ __forceinline__ void stockham_last_pass_st(const cx_t<R>* buf, const FftPlanT<R>& pl, int n, ST&& st,
                                                      int tx = threadIdx.x) {
  constexpr int MB = (EPT + RAD - 1) / RAD;
  static_assert(!HALF || RAD % 2 == 0, "HALF needs an even radix");
  const int nb = n / RAD;   // = the span of the last pass
#pragma unroll
  for (int u = 0; u < MB; u++) {
    const int j = tx + u * blockDim.x;
    if (j < nb) {
      cx_t<R> v[RAD];
#pragma unroll
      for (int r = 0; r < RAD; r++) v[r] = buf[fpad<R, PAD>(j + r * nb)];
      if (nb > 1 && j != 0) apply_twiddles<R, RAD, SIGN>(v, pl, j, 1);
      dft_fixed<R, RAD, SIGN>(v);
#pragma unroll
      for (int r = 0; r < RAD; r++)
        if (!HALF || 2 * r < RAD) st(j + r * nb, v[r]);
    }
  }
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

// ── the two factorisations ──────────────────────────────────────────────
// A runtime plan (any length; its pass table lives in device memory) runs 8s,
// one 4, one 2, 3s, 5s and any other prime <= 64 (fft_stockham).  A
// compile-time plan (fft_fixed, the lengths of kFixedLengths) runs 16s, the
// rest of the power of two as one 8, 4 or 2 — or, with a factor 3, one 12
// or 6 — then 3s and 5s: 3072 = 16.16.12 is three shared-memory passes.
// Each length has exactly one plan, so results never depend on launch shape.
struct RadixList {
  int r[MAXR];
  int nr;   // -1: not factorable (a prime factor > 64, or too many passes)
};
__host__ __device__ constexpr RadixList runtime_radices(int n) {
  RadixList L{};
  int m = n, k = 0;
  // (after the 8s at most one 4 and one 2 remain)
  const int small[5] = {8, 4, 2, 3, 5};
  for (int s = 0; s < 5; s++) {
    const int r = small[s];
    while (m % r == 0) {
      if (k >= MAXR) { L.nr = -1; return L; }
      L.r[k++] = r;
      m /= r;
    }
  }
  for (int p = 7; m > 1; p += 2) {
    while (m % p == 0) {
      if (p > 64 || k >= MAXR) { L.nr = -1; return L; }
      L.r[k++] = p;
      m /= p;
    }
    if (p * p > m && m > 1) {
      if (m > 64 || k >= MAXR) { L.nr = -1; return L; }
      L.r[k++] = m;
      m = 1;
    }
  }
  L.nr = k;
  return L;
}
__host__ __device__ constexpr RadixList fixed_radices(int n) {
  RadixList L{};
  int m = n, k = 0;
  while (m % 16 == 0) { L.r[k++] = 16; m /= 16; }
  int p2 = 1;
  while (m % 2 == 0) { p2 *= 2; m /= 2; }
  if ((p2 == 2 || p2 == 4) && m % 3 == 0) {
    L.r[k++] = 3 * p2;
    m /= 3;
  } else if (p2 > 1) {
    L.r[k++] = p2;
  }
  while (m % 3 == 0) { L.r[k++] = 3; m /= 3; }
  while (m % 5 == 0) { L.r[k++] = 5; m /= 5; }
  L.nr = (m == 1) ? k : -1;
  return L;
}
__host__ __device__ constexpr int ilog2_or_neg(int x) {
  if (x <= 0 || (x & (x - 1))) return -1;
  int l = 0;
  while ((1 << l) < x) l++;
  return l;
}

// Natural-order in, natural-order out, in place in buf (this row's transform),
// runtime plan.  Every thread of the block must call it (it synchronises).
// The passes run as straight-line regions in factorisation order: a runtime
// switch over radices inside one loop makes the register allocator keep every
// variant's state live at once.
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

// Compile-time plan of length N (fixed_radices): passes [P, PE) with span NS
// at pass P, every size, span and shift folded into the code.  pl supplies
// the twiddle table only.
template <typename R, int SIGN, int EPT, bool PAD, int N, int P, int PE, int NS>
__device__ __forceinline__ void fft_fixed(cx_t<R>* buf, const FftPlanT<R>& pl, int tx = threadIdx.x) {
  if constexpr (P < PE) {
    constexpr RadixList L = fixed_radices(N);
    constexpr int RAD = L.r[P];
    stockham_pass_n<R, RAD, SIGN, EPT, PAD>(buf, pl, N, NS, ilog2_or_neg(NS), tx);
    fft_fixed<R, SIGN, EPT, PAD, N, P + 1, PE, NS * RAD>(buf, pl, tx);
  }
}

// the lengths with a compile-time plan (their kernels are instantiated per
// length); every other length takes the runtime plan
constexpr int kFixedLengths[] = {1024, 2048, 3072, 4096};

}  // namespace
