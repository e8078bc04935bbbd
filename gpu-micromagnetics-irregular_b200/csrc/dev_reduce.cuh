// dev_reduce.cuh — deterministic block/grid reductions shared by the vector
// kernels (k_vector.cu) and the fused integrator kernels (k_fused.cu).
// The block partition depends only on the vector length; blocks reduce with
// warp shuffles in a fixed tree; the last block (atomic ticket) sums the
// per-block partials in block order.
#pragma once
#include <math.h>
#include "llg_internal.h"

namespace {

constexpr int RT = 256;         // threads per reduction block
// Streaming kernels keep UB elements of their grid-stride slice in flight:
// the loads of UB consecutive slice elements (i, i + stride, ...) are issued
// before any of them is used or stored, then the elements are finished in
// slice order, so per-element arithmetic and per-thread summation order are
// those of the one-element loop.
constexpr int UB = 4;
constexpr int RMAXB = 1024;     // max reduction blocks

int red_blocks(long long n) {
  long long b = (n + RT * 8 - 1) / (RT * 8);
  if (b > RMAXB) b = RMAXB;
  if (b < 1) b = 1;
  return (int)b;
}

// red_blocks(n) capped at the blocks that are resident at once (per_sm of
// the kernel times the SMs): for kernels whose registers leave fewer than
// red_blocks' count resident, each thread then takes more slice elements
// instead of a second, partly filled wave running after the first.  The
// partition still depends only on n, the kernel and the device.
template <typename KernelT>
int occ_per_sm(KernelT kernel) {
  int p = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p, kernel, RT, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    p = 0;
  }
  return p;
}
inline int cap_resident(int b, int per_sm, int num_sms) {
  if (per_sm <= 0) return b;
  const long long cap = (long long)per_sm * num_sms;
  return (int)(b < cap ? b : cap);
}
inline int red_blocks_resident(long long n, int per_sm, int num_sms) {
  return cap_resident(red_blocks(n), per_sm, num_sms);
}
// per_sm of one kernel, queried once per process (each expansion is its own
// function-local static)
#define LLG_PER_SM(kern) ([]() { static const int p_ = occ_per_sm(kern); return p_; }())

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

// block sum of K values per thread; result valid in thread 0
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* sm /* [K][RT/32] */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; k++) {
    const double s = warp_sum(v[k]);
    if (lane == 0) sm[k * (RT / 32) + wid] = s;
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) {
      double s = (lane < RT / 32) ? sm[k * (RT / 32) + lane] : 0.0;
      s = warp_sum(s);
      v[k] = s;
    }
  }
}

// Last-block finalisation: partials[k*nb + b]; out[k] = sum_b partials (fixed tree).
// Returns true in the last block (where thread 0 wrote out).
template <int K>
__device__ __forceinline__ bool finalize(double* partials, int nb, unsigned int* counter, double* out,
                                         int mode /*0 sum, 1 wrms with n, 2 max*/, double nrm,
                                         const double (&mine)[K]) {
  __shared__ bool last;
  __shared__ double sm[K * (RT / 32)];
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) partials[k * nb + blockIdx.x] = mine[k];
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  double v[K];
#pragma unroll
  for (int k = 0; k < K; k++) {
    double s = (mode == 2) ? 0.0 : 0.0;
    for (int b = threadIdx.x; b < nb; b += RT) {
      const double pv = ((volatile double*)partials)[k * nb + b];
      s = (mode == 2) ? fmax(s, pv) : s + pv;
    }
    v[k] = s;
  }
  if (mode == 2) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < K; k++) {
      const double s = warp_max(v[k]);
      if (lane == 0) sm[k * (RT / 32) + wid] = s;
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
      for (int k = 0; k < K; k++) {
        double s = (lane < RT / 32) ? sm[k * (RT / 32) + lane] : 0.0;
        v[k] = warp_max(s);
      }
    }
  } else {
    block_sum<K>(v, sm);
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; k++) out[k] = (mode == 1) ? sqrt(v[k] / nrm) : v[k];
    *counter = 0u;
  }
  return true;
}

// Called by every thread of a reduction's last block once its results are
// stored: warp 0 carries out the read-back request p (Pub).  __syncwarp
// orders thread 0's stores of the results before the other lanes' loads; the
// loads are volatile so that they come from L2, where the earlier kernels'
// values are.
__device__ __forceinline__ void publish_carried(const Pub& p) {
  if (p.seq == 0 || threadIdx.x >= 32) return;
  __syncwarp();
  for (int i = p.lo + (int)threadIdx.x; i < p.hi; i += 32) p.mail[i] = ((const volatile double*)p.scal)[i];
  __threadfence_system();
  __syncwarp();
  if (threadIdx.x == 0) *reinterpret_cast<volatile unsigned long long*>(p.mail + NSCAL) = p.seq;
}

}  // namespace
