// k_noalloc.cu — the Gram–Schmidt multi-dot without any device allocation.
//
// Who needs it: some callers cannot let a library allocate device memory at
// the moment they need K dot products.  An application whose device memory
// is owned by another allocator (a framework's caching pool that has
// reserved the GPU) would see a cudaMalloc fail or fragment its pool; a
// solver loop with a fixed memory budget, or one with real-time limits,
// allows no allocation after set-up because cudaMalloc/cudaFree can
// synchronise the device.  llg_dot_multi works through an llg_ctx, and
// creating one allocates; this entry point needs only the caller's input
// and output buffers.
//
// Its reduction scratch — the per-block partial sums and the last-block
// ticket — is one file-scope device array of LLG_NOALLOC_MAX_VECS x
// LLG_NOALLOC_MAX_BLOCKS doubles plus a ticket word (about 128 KiB).  Every
// GPU that loads libllg.so holds that array until the process exits.  Host
// code cannot pass the array's name to a kernel (in host code the name is a
// host-side stand-in, not a device address), so the first call on each
// device looks up the device address with cudaGetSymbolAddress, with that
// device current, and caches it per device ordinal; that first call makes
// this one synchronous runtime call, later calls make none.  The cached address belongs to the CUDA
// runtime's primary context of the device: callers that make another
// driver-API context current on the same device must not use this entry
// point from it.  All calls share the array and it keeps the last call's
// contents: the ticket is cleared on the caller's stream at the start of
// every call, and calls that overlap on the GPU (different streams, no
// ordering between them) race on the array.
//
// The partition of the vector into blocks, the per-thread accumulation order
// and the reduction tree are those of llg_dot_multi, so both give the same
// deterministic result.
#include <math.h>

#include <mutex>

#include "llg_internal.h"

namespace {

constexpr int NA_T = 256;
constexpr int NA_MAXV = LLG_NOALLOC_MAX_VECS;
constexpr int NA_MAXB = LLG_NOALLOC_MAX_BLOCKS;
constexpr int NA_MAXDEV = 64;

// partials[k * nb + b] for k < NA_MAXV, b < NA_MAXB; the last 32 doubles
// hold the ticket word (unsigned int at the first of them).
static __device__ __align__(256) double g_noalloc_scratch[NA_MAXV * NA_MAXB + 32];

struct YPack {
  const double* p[NA_MAXV];
};

__device__ __forceinline__ double na_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

template <int K>
__device__ __forceinline__ void na_block_sum(double (&v)[K], double* sm) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const double s = na_warp_sum(v[k]);
    if (lane == 0) sm[k * (NA_T / 32) + wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      double s = (lane < NA_T / 32) ? sm[k * (NA_T / 32) + lane] : 0.0;
      v[k] = na_warp_sum(s);
    }
  }
}

template <int K>
__global__ void __launch_bounds__(NA_T) k_dot_multi_noalloc(const double* __restrict__ x, YPack Y, long long n,
                                                            double* scratch, double* __restrict__ out) {
  __shared__ double sm[K * (NA_T / 32)];
  __shared__ double sm2[K * (NA_T / 32)];
  __shared__ bool last;
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; k++) acc[k] = 0.0;
  for (long long i = blockIdx.x * (long long)NA_T + threadIdx.x; i < n; i += (long long)gridDim.x * NA_T) {
    const double xi = x[i];
#pragma unroll
    for (int k = 0; k < K; k++) acc[k] += xi * Y.p[k][i];
  }
  na_block_sum<K>(acc, sm);
  const int nb = gridDim.x;
  unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + NA_MAXV * NA_MAXB);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) scratch[k * nb + blockIdx.x] = acc[k];
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += NA_T) s += ((volatile double*)scratch)[k * nb + b];
    v[k] = s;
  }
  na_block_sum<K>(v, sm2);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) out[k] = v[k];
    *ticket = 0u;
  }
}

int na_blocks(long long n) {
  long long b = (n + NA_T * 8 - 1) / (NA_T * 8);
  if (b > NA_MAXB) b = NA_MAXB;
  if (b < 1) b = 1;
  return (int)b;
}

std::mutex g_na_mu;
double* g_na_addr[NA_MAXDEV] = {};

// Device address of g_noalloc_scratch on the current device (looked up once).
int na_scratch_ptr(double** out) {
  int dev = 0;
  LLG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAXDEV) {
    llg_set_error("llg_dot_multi_noalloc: device ordinal beyond 64");
    return LLG_ERR_NOTSUP;
  }
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      llg_set_error(std::string("llg_dot_multi_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return LLG_ERR_CUDA;
    }
    g_na_addr[dev] = static_cast<double*>(p);
  }
  *out = g_na_addr[dev];
  return 0;
}

}  // namespace

extern "C" int llg_dot_multi_noalloc(int nvec, const double* d_x, const double* const* d_Y, int64_t n,
                                     double* d_out, void* cuda_stream) {
  if (nvec < 1 || nvec > NA_MAXV) {
    llg_set_error("llg_dot_multi_noalloc: nvec must be 1..LLG_NOALLOC_MAX_VECS (16), got " + std::to_string(nvec));
    return LLG_ERR_ARG;
  }
  if (!d_x || !d_Y || !d_out || n < 0) {
    llg_set_error("llg_dot_multi_noalloc: null pointer or negative length");
    return LLG_ERR_ARG;
  }
  for (int k = 0; k < nvec; k++)
    if (!d_Y[k]) { llg_set_error("llg_dot_multi_noalloc: null vector pointer"); return LLG_ERR_ARG; }
  double* scratch = nullptr;
  int rc = na_scratch_ptr(&scratch);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)cuda_stream;
  LLG_CUDA_TRY(cudaMemsetAsync(scratch + NA_MAXV * NA_MAXB, 0, sizeof(double), s));
  YPack pk{};
  for (int k = 0; k < nvec; k++) pk.p[k] = d_Y[k];
  const int nb = na_blocks(n);
  LLG_COUNT(KID_REDUCE);
  switch (nvec) {
#define NAK(K) \
  case K: k_dot_multi_noalloc<K><<<nb, NA_T, 0, s>>>(d_x, pk, (long long)n, scratch, d_out); break;
    NAK(1) NAK(2) NAK(3) NAK(4) NAK(5) NAK(6) NAK(7) NAK(8)
    NAK(9) NAK(10) NAK(11) NAK(12) NAK(13) NAK(14) NAK(15) NAK(16)
#undef NAK
  }
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}
