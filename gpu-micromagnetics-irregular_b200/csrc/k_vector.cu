// k_vector.cu — NVector-style vector operations for the integrator, sm_100a.
//
// Replaces the reference's SUNDIALS NVECTOR_CUDA kernels and its fused
// multi-dot (src/irregular/2d_fft/2d_i2/deferred_nvector.cu:95-180).
//
// Reductions are deterministic: the block partition depends only on the
// vector length (never on the SM count), each thread accumulates its grid-
// stride slice in a fixed order, blocks reduce with warp shuffles in a fixed
// tree, and the last block to finish (an atomic ticket, not an atomic add)
// sums the per-block partials in block order.  The reference's multi_dot adds
// block partials with atomicAdd (deferred_nvector.cu:127-129), which makes its
// dot products depend on scheduling; here repeated runs are bitwise equal.
//
// Element-wise integrator updates that CVODE issues as chains of
// N_VLinearSum calls (Nordsieck predictor/restore, column rescale, the
// l_j·Δ corrector update) are single passes that apply the same per-element
// operation sequence in registers, so they give the same bits as the chains
// while moving each vector once.
#include <math.h>
#include <string.h>

#include <atomic>
#include <chrono>

#include "llg_internal.h"
#include "launch.h"
#include "dev_reduce.cuh"

namespace {

constexpr int MAXV = 17;        // vectors per fused op

struct PtrPack {
  const double* p[MAXV];
};
struct MPtrPack {
  double* p[MAXV];
};
struct CoefPack {
  double c[MAXV];
};

// Krylov basis vectors stored as VT (double, or float for the FP32-basis
// Krylov solver); arithmetic and accumulation stay FP64
template <typename T>
struct VPack {
  const T* p[MAXV];
};

template <int K, typename VT = double>
__global__ void __launch_bounds__(RT) k_dot_multi(const VT* __restrict__ x, VPack<VT> Y, long long n,
                                                  double* partials, unsigned int* counter, double* out,
                                                  KScale ks) {
  pdl_entry();
  __shared__ double sm[K * (RT / 32)];
  double ya[K];   // scales of the Y vectors (1 when stored normalised)
#pragma unroll
  for (int k = 0; k < K; k++) ya[k] = kscale_of(ks.a[k]);
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.0;
  const long long st = (long long)gridDim.x * RT;
  for (long long i0 = blockIdx.x * (long long)RT + threadIdx.x; i0 < n; i0 += UB * st) {
    double xv[UB], yv[UB][K];
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const long long i = i0 + u * st;
      xv[u] = (i < n) ? (double)x[i] : 0.0;
#pragma unroll
      for (int k = 0; k < K; k++) yv[u][k] = (i < n) ? ya[k] * (double)Y.p[k][i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < UB; u++)
      if (i0 + u * st < n) {
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] += xv[u] * yv[u][k];
      }
  }
  block_sum<K>(acc, sm);
  finalize<K>(partials, gridDim.x, counter, out, 0, 1.0, acc);
}

__global__ void __launch_bounds__(RT) k_wrms(const double* __restrict__ x, const double* __restrict__ w,
                                             long long n, double* partials, unsigned int* counter, double* out) {
  pdl_entry();
  __shared__ double sm[RT / 32];
  double acc[1] = {0.0};
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double p = x[i] * w[i];
    acc[0] += p * p;
  }
  block_sum<1>(acc, sm);
  finalize<1>(partials, gridDim.x, counter, out, 1, (double)n, acc);
}

// wrms of (a x + b y) with weights w
__global__ void __launch_bounds__(RT) k_wrms_lin(double a, const double* __restrict__ x, double b,
                                                 const double* __restrict__ y, const double* __restrict__ w,
                                                 long long n, double* partials, unsigned int* counter,
                                                 double* out) {
  pdl_entry();
  __shared__ double sm[RT / 32];
  double acc[1] = {0.0};
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double v = a * x[i] + b * y[i];
    const double p = v * w[i];
    acc[0] += p * p;
  }
  block_sum<1>(acc, sm);
  finalize<1>(partials, gridDim.x, counter, out, 1, (double)n, acc);
}

// ewt = 1/(rtol|y| + atol); out = max(bad flag) (1 if any denominator <= 0 or NaN)
__global__ void __launch_bounds__(RT) k_set_ewt(double rtol, double atol, const double* __restrict__ y,
                                                double* __restrict__ ewt, long long n, double* partials,
                                                unsigned int* counter, double* out) {
  pdl_entry();
  double bad[1] = {0.0};
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double t = rtol * fabs(y[i]) + atol;
    if (t <= 0.0) bad[0] = 1.0;   // (a NaN state is left to the norm check)
    ewt[i] = 1.0 / t;
  }
  const double wm = warp_max(bad[0]);
  __shared__ double sm[RT / 32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = wm;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = (threadIdx.x < RT / 32) ? sm[threadIdx.x] : 0.0;
    bad[0] = warp_max(s);
  }
  finalize<1>(partials, gridDim.x, counter, out, 2, 1.0, bad);
}

// hub_inv = max |f0| / (0.1|y0| + 1/(1/(rtol|y0|+atol)))   (cvUpperBoundH0)
__global__ void __launch_bounds__(RT) k_hin_bound(double rtol, double atol, const double* __restrict__ y,
                                                  const double* __restrict__ f, long long n, double* partials,
                                                  unsigned int* counter, double* out) {
  pdl_entry();
  double m[1] = {0.0};
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double ay = fabs(y[i]);
    const double t1 = 1.0 / (1.0 / (rtol * ay + atol));
    const double den = 0.1 * ay + 1.0 * t1;
    m[0] = fmax(m[0], fabs(f[i]) / den);
  }
  const double wm = warp_max(m[0]);
  __shared__ double sm[RT / 32];
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = wm;
  __syncthreads();
  if (threadIdx.x < 32) {
    double s = (threadIdx.x < RT / 32) ? sm[threadIdx.x] : 0.0;
    m[0] = warp_max(s);
  }
  finalize<1>(partials, gridDim.x, counter, out, 2, 1.0, m);
}

__global__ void k_lin(double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                      double* __restrict__ z, long long n) {
  pdl_entry();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = a * x[i] + b * y[i];
}
template <typename VT = double>
__global__ void k_scale(double a, const VT* __restrict__ x, VT* __restrict__ z, long long n) {
  pdl_entry();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = (VT)(a * (double)x[i]);
}
__global__ void k_const(double a, double* __restrict__ z, long long n) {
  pdl_entry();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = a;
}
__global__ void k_prod(const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ z,
                       long long n) {
  pdl_entry();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = x[i] * y[i];
}
__global__ void k_div(const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ z,
                      long long n) {
  pdl_entry();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = x[i] / y[i];
}
// z = c0 X0; z = c_k X_k + z   (z may alias X0)
__global__ void k_lincomb(int nv, CoefPack c, PtrPack X, double* z, long long n) {
  pdl_entry();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double s = c.c[0] * X.p[0][i];
    for (int k = 1; k < nv; k++) s = c.c[k] * X.p[k][i] + s;
    z[i] = s;
  }
}
// Z_j = a_j x + Y_j
__global__ void k_scale_add_multi(int nv, CoefPack a, const double* __restrict__ x, PtrPack Y, MPtrPack Z,
                                  long long n) {
  pdl_entry();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double xi = x[i];
    for (int k = 0; k < nv; k++) Z.p[k][i] = a.c[k] * xi + Y.p[k][i];
  }
}
// Pascal triangle (sign +1: predictor, -1: restore) over zn[0..Q], in registers
template <int Q>
__global__ void k_nordsieck(MPtrPack zn, int sign, long long n) {
  pdl_entry();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    double v[Q + 1];
#pragma unroll
    for (int j = 0; j <= Q; j++) v[j] = zn.p[j][i];
#pragma unroll
    for (int k = 1; k <= Q; k++)
#pragma unroll
      for (int j = Q; j >= k; j--) v[j - 1] = (sign > 0) ? v[j - 1] + v[j] : v[j - 1] - v[j];
#pragma unroll
    for (int j = 0; j < Q; j++) zn.p[j][i] = v[j];
  }
}
// zn[j] *= f_j for j = 1..q
__global__ void k_scale_cols(int q, CoefPack f, MPtrPack zn, long long n) {
  pdl_entry();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    for (int j = 1; j <= q; j++) zn.p[j][i] = f.c[j] * zn.p[j][i];
  }
}

// classical Gram-Schmidt update with the dots read on the device:
// z = 1 z + sum_{i<k} (-dots_i) X_i, and sum z^2 (the arithmetic of
// k_lincomb_norm with coefficients {1, -dots_0, ..., -dots_{k-1}})
// (VT float: the stored, rounded values are what the norm sums)
template <typename VT = double>
__global__ void __launch_bounds__(RT) k_gs_update(int k, VPack<VT> X, const double* __restrict__ dots, VT* z,
                                                  long long n, double* partials, unsigned int* counter,
                                                  double* out, KScale ks, double* aout, Pub pub) {
  pdl_entry();
  __shared__ double sm[RT / 32];
  // scales of the X vectors, staged once: read through pointers, they would be
  // reloaded after every store to z (the compiler cannot rule out aliasing)
  __shared__ double xs[MAXV - 1];
  if (threadIdx.x < k) xs[threadIdx.x] = kscale_of(ks.a[threadIdx.x]);
  __syncthreads();
  double cf[MAXV - 1];
#pragma unroll
  for (int j = 0; j < MAXV - 1; j++) cf[j] = (j < k) ? -dots[j] : 0.0;
  double acc[1] = {0.0};
  const long long st = (long long)gridDim.x * RT;
  for (long long i0 = blockIdx.x * (long long)RT + threadIdx.x; i0 < n; i0 += UB * st) {
    double s[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) s[u] = (i0 + u * st < n) ? 1.0 * (double)z[i0 + u * st] : 0.0;
#pragma unroll
    for (int j = 0; j < MAXV - 1; j++)
      if (j < k) {
        double xv[UB];
        const double xa = xs[j];   // the scale of X_j (1 when stored normalised)
#pragma unroll
        for (int u = 0; u < UB; u++) xv[u] = (i0 + u * st < n) ? xa * (double)X.p[j][i0 + u * st] : 0.0;
#pragma unroll
        for (int u = 0; u < UB; u++) s[u] = cf[j] * xv[u] + s[u];
      }
#pragma unroll
    for (int u = 0; u < UB; u++)
      if (i0 + u * st < n) {
        const VT sv = (VT)s[u];
        z[i0 + u * st] = sv;
        acc[0] += (double)sv * (double)sv;
      }
  }
  block_sum<1>(acc, sm);
  const bool last = finalize<1>(partials, gridDim.x, counter, out, 0, 1.0, acc);
  // the updated vector's scale; dots[k] is its sum of squares before the update
  if (last && aout && threadIdx.x == 0) *aout = gs_scale_of(out[0], dots + k);
  if (last) publish_carried(pub);
}

// k_gs_update with the vector count K fixed at compile time: the loads of
// all K basis vectors (and of z) for the UB slice elements are issued before
// any of them is used, where the runtime-k loop waits on one vector at a
// time.  Per element the same operations in the same order, so z is bitwise
// that of k_gs_update; it runs on one resident wave of blocks
// (red_blocks_resident), so its sum of squares is added in another partition.
template <int K, typename VT>
__global__ void __launch_bounds__(RT) k_gs_update_k(VPack<VT> X, const double* __restrict__ dots, VT* z, long long n,
                                                    double* partials, unsigned int* counter, double* out, KScale ks,
                                                    double* aout, Pub pub) {
  pdl_entry();
  __shared__ double sm[RT / 32];
  __shared__ double xs[K];
  if (threadIdx.x < K) xs[threadIdx.x] = kscale_of(ks.a[threadIdx.x]);
  __syncthreads();
  double cf[K], xa[K];
#pragma unroll
  for (int j = 0; j < K; j++) {
    cf[j] = -dots[j];
    xa[j] = xs[j];
  }
  double acc[1] = {0.0};
  const long long st = (long long)gridDim.x * RT;
  for (long long i0 = blockIdx.x * (long long)RT + threadIdx.x; i0 < n; i0 += UB * st) {
    VT zr[UB], xr[K][UB];
#pragma unroll
    for (int u = 0; u < UB; u++) {
      const long long i = i0 + u * st;
      const bool in = i < n;
      zr[u] = in ? z[i] : VT(0);
#pragma unroll
      for (int j = 0; j < K; j++) xr[j][u] = in ? X.p[j][i] : VT(0);
    }
    double s[UB];
#pragma unroll
    for (int u = 0; u < UB; u++) s[u] = 1.0 * (double)zr[u];
#pragma unroll
    for (int j = 0; j < K; j++)
#pragma unroll
      for (int u = 0; u < UB; u++) s[u] = cf[j] * (xa[j] * (double)xr[j][u]) + s[u];
#pragma unroll
    for (int u = 0; u < UB; u++)
      if (i0 + u * st < n) {
        const VT sv = (VT)s[u];
        z[i0 + u * st] = sv;
        acc[0] += (double)sv * (double)sv;
      }
  }
  block_sum<1>(acc, sm);
  const bool last = finalize<1>(partials, gridDim.x, counter, out, 0, 1.0, acc);
  if (last && aout && threadIdx.x == 0) *aout = gs_scale_of(out[0], dots + K);
  if (last) publish_carried(pub);
}

// one warp copies d_scal[lo, hi) into the mapped host mailbox, makes the
// copies visible to the host, then writes the sequence word last
__global__ void k_publish(const double* __restrict__ src, int lo, int hi, double* mail,
                          unsigned long long seq) {
  pdl_entry();
  for (int i = lo + (int)threadIdx.x; i < hi; i += 32) mail[i] = src[i];
  __threadfence_system();
  __syncwarp();
  if (threadIdx.x == 0) {
    volatile unsigned long long* flag = reinterpret_cast<volatile unsigned long long*>(mail + NSCAL);
    *flag = seq;
  }
}

int ew_grid(const llg_ctx* c, long long n) {
  long long g = (n + 255) / 256;
  const long long cap = (long long)c->num_sms * 8;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace

int reductions_init(llg_ctx* c) {
  c->red_blocks_max = RMAXB;
  LLG_CUDA_TRY(cudaMalloc(&c->d_red, sizeof(double) * MAXV * RMAXB));
  LLG_CUDA_TRY(cudaMalloc(&c->d_scal, sizeof(double) * NSCAL));
  LLG_CUDA_TRY(cudaMalloc(&c->d_counter, sizeof(unsigned int) * 4));
  LLG_CUDA_TRY(cudaMemset(c->d_counter, 0, sizeof(unsigned int) * 4));
  LLG_CUDA_TRY(cudaMemset(c->d_scal, 0, sizeof(double) * NSCAL));
  LLG_CUDA_TRY(cudaMallocHost(&c->h_scal, sizeof(double) * NSCAL));
  memset(c->h_scal, 0, sizeof(double) * NSCAL);
  LLG_CUDA_TRY(cudaHostAlloc(&c->h_mail, sizeof(double) * (NSCAL + 1), cudaHostAllocMapped));
  memset(c->h_mail, 0, sizeof(double) * (NSCAL + 1));
  LLG_CUDA_TRY(cudaHostGetDevicePointer((void**)&c->d_mail, c->h_mail, 0));
  c->mail_seq = 0;
  return 0;
}

void reductions_free(llg_ctx* c) {
  cudaFree(c->d_red);
  cudaFree(c->d_scal);
  cudaFree(c->d_counter);
  if (c->h_scal) cudaFreeHost(c->h_scal);
  if (c->h_mail) cudaFreeHost(c->h_mail);
  c->d_red = c->d_scal = nullptr;
  c->d_counter = nullptr;
  c->h_scal = nullptr;
  c->h_mail = c->d_mail = nullptr;
}

template <typename VT>
static int vdot_multi_impl(llg_ctx* c, int nvec, const VT* x, const VT* const* Y, int slot, const KScale* ks) {
  const KScale kz{};
  const KScale& kk = ks ? *ks : kz;
  if (nvec <= 0) return 0;
  if (nvec > 16) { llg_set_error("dot_multi: nvec > 16"); return LLG_ERR_ARG; }
  VPack<VT> pk{};
  for (int k = 0; k < nvec; k++) pk.p[k] = Y[k];
  const long long n = c->neq;
  const int nb = red_blocks(n);
  double* out = c->d_scal + slot;
  switch (nvec) {
#define DOTK(K) \
  case K: LLG_COUNT(KID_REDUCE); klaunch(k_dot_multi<K, VT>, nb, RT, 0, c->stream, x, pk, n, c->d_red, c->d_counter, out, kk); break;
    DOTK(1) DOTK(2) DOTK(3) DOTK(4) DOTK(5) DOTK(6) DOTK(7) DOTK(8)
    DOTK(9) DOTK(10) DOTK(11) DOTK(12) DOTK(13) DOTK(14) DOTK(15) DOTK(16)
#undef DOTK
  }
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int vdot_multi_dev(llg_ctx* c, int nvec, const double* x, const double* const* Y, int slot, const KScale* ks) {
  return vdot_multi_impl<double>(c, nvec, x, Y, slot, ks);
}
int vdot_multi_dev_f(llg_ctx* c, int nvec, const float* x, const float* const* Y, int slot, const KScale* ks) {
  return vdot_multi_impl<float>(c, nvec, x, Y, slot, ks);
}

int vwrms_dev(llg_ctx* c, const double* x, const double* w, int slot) {
  const long long n = c->neq;
  LLG_COUNT(KID_REDUCE);
  klaunch(k_wrms, red_blocks(n), RT, 0, c->stream, x, w, n, c->d_red, c->d_counter, c->d_scal + slot);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

int vwrms_diff_dev(llg_ctx* c, double a, const double* x, double b, const double* y, const double* w, int slot) {
  const long long n = c->neq;
  LLG_COUNT(KID_REDUCE);
  klaunch(k_wrms_lin, red_blocks(n), RT, 0, c->stream, a, x, b, y, w, n, c->d_red, c->d_counter, c->d_scal + slot);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

void arm_publish(llg_ctx* c, int lo, int hi) {
  c->pub_armed = Pub{};
  if (lo < 0 || hi > NSCAL || hi <= lo) return;   // fetch_range reports it
  c->pub_armed = Pub{c->d_scal, c->d_mail, lo, hi, ++c->mail_seq};
}

Pub take_publish(llg_ctx* c) {
  const Pub p = c->pub_armed;
  c->pub_armed = Pub{};
  if (p.seq) c->pub_carried = p;
  return p;
}

// Read-back of d_scal[lo, hi) into h_scal: the publish kernel runs after the
// producing kernels (stream order) and the host polls the mailbox's sequence
// word, instead of a device-to-host copy plus a stream synchronisation (the
// copy engine's start-up and the wake-up were most of a read-back's cost).
// When the last launch carried a request for this range (arm_publish), its
// last block has published and only the poll remains.
// The poll is bounded by wall time; past it (or after a launch error) the
// stream is synchronised, which reports any device-side failure.
int fetch_range(llg_ctx* c, int lo, int hi) {
  const Pub carried = c->pub_carried;
  c->pub_carried = Pub{};
  c->pub_armed = Pub{};
  if (lo < 0 || hi > NSCAL || hi <= lo) { llg_set_error("fetch_range: bad slots"); return LLG_ERR_ARG; }
  unsigned long long seq;
  if (carried.seq && carried.lo == lo && carried.hi == hi) {
    seq = carried.seq;
  } else {
    seq = ++c->mail_seq;
    klaunch(k_publish, 1, 32, 0, c->stream, c->d_scal, lo, hi, c->d_mail, seq);
    LLG_CUDA_TRY(cudaPeekAtLastError());
  }
  volatile unsigned long long* flag = reinterpret_cast<volatile unsigned long long*>(c->h_mail + NSCAL);
  bool seen = false;
  const auto t0 = std::chrono::steady_clock::now();
  for (unsigned long it = 0;; it++) {
    if (*flag >= seq) { seen = true; break; }
    if ((it & 1023) == 1023) {
      if (std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(200)) break;
      if (cudaStreamQuery(c->stream) == cudaSuccess && *flag >= seq) { seen = true; break; }
    }
  }
  if (!seen) {
    LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (*flag < seq) { llg_set_error("fetch_range: read-back did not arrive"); return LLG_ERR_CUDA; }
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  const volatile double* mail = c->h_mail;
  for (int i = lo; i < hi; i++) c->h_scal[i] = mail[i];
  return 0;
}

template <typename VT>
static int vgs_update_impl(llg_ctx* c, int k, VT* const* V, int slot_dots, int slot_ss, const KScale* ks,
                           int slot_aout) {
  if (k < 1 || k > MAXV - 1) { llg_set_error("gs_update: bad k"); return LLG_ERR_ARG; }
  VPack<VT> pk{};
  for (int j = 0; j < k; j++) pk.p[j] = V[j];
  const KScale kz{};
  LLG_COUNT(KID_REDUCE);
  const int nb = red_blocks(c->neq);
  const double* dots = c->d_scal + slot_dots;
  double* ss = c->d_scal + slot_ss;
  double* aout = slot_aout >= 0 ? c->d_scal + slot_aout : nullptr;
  const KScale kk = ks ? *ks : kz;
  const Pub pub = take_publish(c);
#define GS_K(K)                                                                                                  \
  klaunch(k_gs_update_k<K, VT>, red_blocks_resident(c->neq, LLG_PER_SM((k_gs_update_k<K, VT>)), c->num_sms), RT, \
          0, c->stream, pk, dots, V[k], c->neq, c->d_red, c->d_counter, ss, kk, aout, pub)
  switch (k) {
    case 1: GS_K(1); break;
    case 2: GS_K(2); break;
    case 3: GS_K(3); break;
    case 4: GS_K(4); break;
    case 5: GS_K(5); break;
    case 6: GS_K(6); break;
    case 7: GS_K(7); break;
    case 8: GS_K(8); break;
    default:
      klaunch(k_gs_update<VT>, nb, RT, 0, c->stream, k, pk, dots, V[k], c->neq, c->d_red, c->d_counter, ss, kk, aout,
              pub);
  }
#undef GS_K
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vgs_update_dev(llg_ctx* c, int k, double* const* V, int slot_dots, int slot_ss, const KScale* ks,
                   int slot_aout) {
  return vgs_update_impl<double>(c, k, V, slot_dots, slot_ss, ks, slot_aout);
}
int vgs_update_dev_f(llg_ctx* c, int k, float* const* V, int slot_dots, int slot_ss, const KScale* ks,
                     int slot_aout) {
  return vgs_update_impl<float>(c, k, V, slot_dots, slot_ss, ks, slot_aout);
}

int fetch_scalars(llg_ctx* c, int slot, int n, double* out) {
  const int rc = fetch_range(c, slot, slot + n);
  if (rc) return rc;
  for (int k = 0; k < n; k++) out[k] = c->h_scal[slot + k];
  return 0;
}

int vlin(llg_ctx* c, double a, const double* x, double b, const double* y, double* z) {
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_lin, ew_grid(c, c->neq), 256, 0, c->stream, a, x, b, y, z, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vscale_f(llg_ctx* c, double a, const float* x, float* z) {
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_scale<float>, ew_grid(c, c->neq), 256, 0, c->stream, a, x, z, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vscale(llg_ctx* c, double a, const double* x, double* z) {
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_scale<double>, ew_grid(c, c->neq), 256, 0, c->stream, a, x, z, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vconst(llg_ctx* c, double a, double* z) {
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_const, ew_grid(c, c->neq), 256, 0, c->stream, a, z, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vprod(llg_ctx* c, const double* x, const double* y, double* z) {
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_prod, ew_grid(c, c->neq), 256, 0, c->stream, x, y, z, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vdiv(llg_ctx* c, const double* x, const double* y, double* z) {
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_div, ew_grid(c, c->neq), 256, 0, c->stream, x, y, z, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vlincomb(llg_ctx* c, int nvec, const double* coef, const double* const* X, double* z) {
  if (nvec < 1 || nvec > MAXV) { llg_set_error("lincomb: bad nvec"); return LLG_ERR_ARG; }
  CoefPack cp{};
  PtrPack pk{};
  for (int k = 0; k < nvec; k++) { cp.c[k] = coef[k]; pk.p[k] = X[k]; }
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_lincomb, ew_grid(c, c->neq), 256, 0, c->stream, nvec, cp, pk, z, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vscale_add_multi(llg_ctx* c, int nvec, const double* a, const double* x, double* const* Y, double* const* Z) {
  if (nvec <= 0) return 0;
  if (nvec > MAXV) { llg_set_error("scale_add_multi: bad nvec"); return LLG_ERR_ARG; }
  CoefPack cp{};
  PtrPack yp{};
  MPtrPack zp{};
  for (int k = 0; k < nvec; k++) { cp.c[k] = a[k]; yp.p[k] = Y[k]; zp.p[k] = Z[k]; }
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_scale_add_multi, ew_grid(c, c->neq), 256, 0, c->stream, nvec, cp, x, yp, zp, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vnordsieck_shift(llg_ctx* c, int q, double* const* zn, int sign) {
  if (q < 1) return 0;
  MPtrPack zp{};
  for (int j = 0; j <= q; j++) zp.p[j] = zn[j];
  LLG_COUNT(KID_ELEMWISE);
  const int g = ew_grid(c, c->neq);
  switch (q) {
    case 1: klaunch(k_nordsieck<1>, g, 256, 0, c->stream, zp, sign, c->neq); break;
    case 2: klaunch(k_nordsieck<2>, g, 256, 0, c->stream, zp, sign, c->neq); break;
    case 3: klaunch(k_nordsieck<3>, g, 256, 0, c->stream, zp, sign, c->neq); break;
    case 4: klaunch(k_nordsieck<4>, g, 256, 0, c->stream, zp, sign, c->neq); break;
    default: klaunch(k_nordsieck<5>, g, 256, 0, c->stream, zp, sign, c->neq); break;
  }
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vscale_columns(llg_ctx* c, int q, double eta, double* const* zn) {
  if (q < 1) return 0;
  CoefPack f{};
  MPtrPack zp{};
  double factor = eta;
  for (int j = 1; j <= q; j++) { f.c[j] = factor; factor *= eta; zp.p[j] = zn[j]; }
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_scale_cols, ew_grid(c, c->neq), 256, 0, c->stream, q, f, zp, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vscale_columns_f(llg_ctx* c, int q, const double* f, double* const* zn) {
  if (q < 1) return 0;
  CoefPack fp{};
  MPtrPack zp{};
  for (int j = 1; j <= q; j++) { fp.c[j] = f[j]; zp.p[j] = zn[j]; }
  LLG_COUNT(KID_ELEMWISE);
  klaunch(k_scale_cols, ew_grid(c, c->neq), 256, 0, c->stream, q, fp, zp, c->neq);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vset_ewt(llg_ctx* c, double rtol, double atol, const double* y, double* ewt, int slot) {
  const long long n = c->neq;
  LLG_COUNT(KID_REDUCE);
  klaunch(k_set_ewt, red_blocks(n), RT, 0, c->stream, rtol, atol, y, ewt, n, c->d_red, c->d_counter, c->d_scal + slot);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
int vhin_bound(llg_ctx* c, double rtol, double atol, const double* y0, const double* f0, double* tmp) {
  (void)tmp;
  const long long n = c->neq;
  LLG_COUNT(KID_REDUCE);
  klaunch(k_hin_bound, red_blocks(n), RT, 0, c->stream, rtol, atol, y0, f0, n, c->d_red, c->d_counter, c->d_scal + 40);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
