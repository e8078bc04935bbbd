// k_learned.cu — learned preconditioner: a 3-layer 3x3 convolutional network
// applied on top of block-Jacobi, its training on the GPU (hand-written
// forward, backward and Adam kernels), and the harvesting of training pairs
// from the integrator's own SPGMR solves.  No counterpart in the reference.
//
// The network is linear in the residual, so within one setup it is a fixed
// linear left preconditioner for GMRES:
//   u = P_BJ^-1 r                         (3x3 block-Jacobi, frozen m, h, gamma)
//   F = [u, m x u, m x (m x u)] * mask    (9 channels, m frozen at psetup)
//   z = (u + gamma * W3 * W2 * W1 * F) * mask
// with * a 3x3 cross-correlation, zero padding, no bias, no activation,
// channels 9 -> 16 -> 16 -> 3.  Inference uses BF16-rounded weights with FP32
// accumulation; training keeps FP32 master weights.  The gamma factor lets
// the layers learn the gamma-free part of (I - gamma J)^-1 - P_BJ^-1, whose
// leading term is gamma P_BJ^-1 J_exchange P_BJ^-1 (the exchange coupling
// that block-Jacobi leaves out).
//
// Training target: the solver's own SPGMR solutions x of (I - gamma J) x = r,
// harvested from block-Jacobi solves; loss per patch
//   sum_interior (ewt (z - x))^2 / sum_interior (ewt x)^2
// over random PxP patches (3-cell border excluded, as the patch's zero
// padding is not the grid's).  Layout of every activation: [batch][channel]
// [row][col] FP32.
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <random>
#include <vector>

#include "dev_reduce.cuh"
#include "dev_tc.cuh"
#include "llg_internal.h"

namespace {

constexpr int CIN0 = 9, CH = 16, COUT3 = 3;
constexpr int NW1 = CH * CIN0 * 9, NW2 = CH * CH * 9, NW3 = COUT3 * CH * 9;
constexpr int NWT = NW1 + NW2 + NW3;   // 4032
constexpr int TW = 32, TH = 8;         // conv tile (threads)
constexpr int BORDER = 3;

// ── convolution kernels (grid: x tiles, y tiles, batch; block 32 x 8) ──
template <int CIN, int COUT>
__global__ void __launch_bounds__(TW * TH) k_conv3(const float* __restrict__ in, const float* __restrict__ w,
                                                   float* __restrict__ out, int H, int W) {
  __shared__ float sw[COUT * CIN * 9];
  __shared__ float st[CIN][TH + 2][TW + 2];
  const int b = blockIdx.z, x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const int tid = threadIdx.y * TW + threadIdx.x;
  const size_t plane = (size_t)H * W;
  for (int i = tid; i < COUT * CIN * 9; i += TW * TH) sw[i] = w[i];
  const float* src = in + (size_t)b * CIN * plane;
  for (int i = tid; i < CIN * (TH + 2) * (TW + 2); i += TW * TH) {
    const int c = i / ((TH + 2) * (TW + 2)), r = i % ((TH + 2) * (TW + 2));
    const int yy = r / (TW + 2), xx = r % (TW + 2);
    const int gy = y0 + yy - 1, gx = x0 + xx - 1;
    st[c][yy][xx] = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? src[c * plane + (size_t)gy * W + gx] : 0.f;
  }
  __syncthreads();
  const int gx = x0 + threadIdx.x, gy = y0 + threadIdx.y;
  if (gx >= W || gy >= H) return;
  float acc[COUT];
#pragma unroll
  for (int o = 0; o < COUT; o++) acc[o] = 0.f;
  for (int c = 0; c < CIN; c++)
#pragma unroll
    for (int t = 0; t < 9; t++) {
      const float v = st[c][threadIdx.y + t / 3][threadIdx.x + t % 3];
#pragma unroll
      for (int o = 0; o < COUT; o++) acc[o] = fmaf(sw[(o * CIN + c) * 9 + t], v, acc[o]);
    }
  float* dst = out + (size_t)b * COUT * plane + (size_t)gy * W + gx;
#pragma unroll
  for (int o = 0; o < COUT; o++) dst[o * plane] = acc[o];
}

// din[c][y][x] = sum_o sum_t w[o][c][t] dout[o][y - dy + 1][x - dx + 1]
template <int CIN, int COUT>
__global__ void __launch_bounds__(TW * TH) k_conv3_bwd_data(const float* __restrict__ dout,
                                                            const float* __restrict__ w, float* __restrict__ din,
                                                            int H, int W) {
  __shared__ float sw[COUT * CIN * 9];
  __shared__ float sd[COUT][TH + 2][TW + 2];
  const int b = blockIdx.z, x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const int tid = threadIdx.y * TW + threadIdx.x;
  const size_t plane = (size_t)H * W;
  for (int i = tid; i < COUT * CIN * 9; i += TW * TH) sw[i] = w[i];
  const float* src = dout + (size_t)b * COUT * plane;
  for (int i = tid; i < COUT * (TH + 2) * (TW + 2); i += TW * TH) {
    const int o = i / ((TH + 2) * (TW + 2)), r = i % ((TH + 2) * (TW + 2));
    const int yy = r / (TW + 2), xx = r % (TW + 2);
    const int gy = y0 + yy - 1, gx = x0 + xx - 1;
    sd[o][yy][xx] = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? src[o * plane + (size_t)gy * W + gx] : 0.f;
  }
  __syncthreads();
  const int gx = x0 + threadIdx.x, gy = y0 + threadIdx.y;
  if (gx >= W || gy >= H) return;
  float acc[CIN];
#pragma unroll
  for (int c = 0; c < CIN; c++) acc[c] = 0.f;
  for (int o = 0; o < COUT; o++)
#pragma unroll
    for (int t = 0; t < 9; t++) {
      const float v = sd[o][threadIdx.y + 2 - t / 3][threadIdx.x + 2 - t % 3];
#pragma unroll
      for (int c = 0; c < CIN; c++) acc[c] = fmaf(sw[(o * CIN + c) * 9 + t], v, acc[c]);
    }
  float* dst = din + (size_t)b * CIN * plane + (size_t)gy * W + gx;
#pragma unroll
  for (int c = 0; c < CIN; c++) dst[c * plane] = acc[c];
}

// per-block partial weight gradients: part[block][o][c][t] = sum over the
// block's pixels of dout[o][p] in[c][p + t - (1,1)]
template <int CIN, int COUT>
__global__ void __launch_bounds__(TW * TH) k_conv3_bwd_w(const float* __restrict__ in, const float* __restrict__ dout,
                                                         float* __restrict__ part, int H, int W) {
  __shared__ float st[CIN][TH + 2][TW + 2];
  __shared__ float sd[COUT][TH][TW];
  const int b = blockIdx.z, x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const int tid = threadIdx.y * TW + threadIdx.x;
  const size_t plane = (size_t)H * W;
  const float* si = in + (size_t)b * CIN * plane;
  const float* so = dout + (size_t)b * COUT * plane;
  for (int i = tid; i < CIN * (TH + 2) * (TW + 2); i += TW * TH) {
    const int c = i / ((TH + 2) * (TW + 2)), r = i % ((TH + 2) * (TW + 2));
    const int yy = r / (TW + 2), xx = r % (TW + 2);
    const int gy = y0 + yy - 1, gx = x0 + xx - 1;
    st[c][yy][xx] = (gy >= 0 && gy < H && gx >= 0 && gx < W) ? si[c * plane + (size_t)gy * W + gx] : 0.f;
  }
  for (int i = tid; i < COUT * TH * TW; i += TW * TH) {
    const int o = i / (TH * TW), r = i % (TH * TW);
    const int yy = r / TW, xx = r % TW;
    const int gy = y0 + yy, gx = x0 + xx;
    sd[o][yy][xx] = (gy < H && gx < W) ? so[o * plane + (size_t)gy * W + gx] : 0.f;
  }
  __syncthreads();
  const size_t blk = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
  for (int e = tid; e < COUT * CIN * 9; e += TW * TH) {
    const int o = e / (CIN * 9), c = (e / 9) % CIN, t = e % 9, dy = t / 3, dx = t % 3;
    float acc = 0.f;
    for (int py = 0; py < TH; py++)
#pragma unroll 8
      for (int px = 0; px < TW; px++) acc = fmaf(sd[o][py][px], st[c][py + dy][px + dx], acc);
    part[blk * (COUT * CIN * 9) + e] = acc;
  }
}

// out[e] = sum over blocks (fixed order) of part[block][e]
__global__ void k_sum_parts(const float* __restrict__ part, int nblk, int n, float* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  double acc = 0.0;
  for (int k = 0; k < nblk; k++) acc += part[(size_t)k * n + e];
  out[e] = (float)acc;
}

// ── training: features, loss, gradient of the output, Adam ──
// patch planes: u, m, ewt, x [b][3][P][P], mask [b][P][P], gamma[b]
__global__ void k_feat_patch(const float* __restrict__ u, const float* __restrict__ m,
                             const float* __restrict__ mask, float* __restrict__ f, int nb, int P) {
  const size_t plane = (size_t)P * P;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nb * plane; i += (size_t)gridDim.x * blockDim.x) {
    const size_t b = i / plane, p = i % plane;
    const float* ub = u + b * 3 * plane;
    const float* mb = m + b * 3 * plane;
    const float k = mask[i];
    const float u0 = ub[p], u1 = ub[plane + p], u2 = ub[2 * plane + p];
    const float m0 = mb[p], m1 = mb[plane + p], m2 = mb[2 * plane + p];
    const float a0 = m1 * u2 - m2 * u1, a1 = m2 * u0 - m0 * u2, a2 = m0 * u1 - m1 * u0;   // m x u
    const float b0 = m1 * a2 - m2 * a1, b1 = m2 * a0 - m0 * a2, b2 = m0 * a1 - m1 * a0;   // m x (m x u)
    float* fb = f + b * 9 * plane;
    fb[p] = u0 * k; fb[plane + p] = u1 * k; fb[2 * plane + p] = u2 * k;
    fb[3 * plane + p] = a0 * k; fb[4 * plane + p] = a1 * k; fb[5 * plane + p] = a2 * k;
    fb[6 * plane + p] = b0 * k; fb[7 * plane + p] = b1 * k; fb[8 * plane + p] = b2 * k;
  }
}

// one block per patch: num[b] = sum_int (ewt (z - x))^2, den[b] = sum_int (ewt x)^2
__global__ void __launch_bounds__(256) k_loss_terms(const float* __restrict__ u, const float* __restrict__ y3,
                                                    const float* __restrict__ mask, const float* __restrict__ ewt,
                                                    const float* __restrict__ x, const float* __restrict__ gam,
                                                    int P, double* __restrict__ num, double* __restrict__ den) {
  const int b = blockIdx.x;
  const size_t plane = (size_t)P * P;
  double a[2] = {0.0, 0.0};
  for (size_t i = threadIdx.x; i < 3 * plane; i += blockDim.x) {
    const size_t p = i % plane;
    const int yy = (int)(p / P), xx = (int)(p % P);
    if (yy < BORDER || yy >= P - BORDER || xx < BORDER || xx >= P - BORDER) continue;
    const size_t g = b * 3 * plane + i;
    const float z = (u[g] + gam[b] * y3[g]) * mask[b * plane + p];
    const double e = (double)ewt[g] * ((double)z - x[g]);
    const double r = (double)ewt[g] * x[g];
    a[0] += e * e;
    a[1] += r * r;
  }
  __shared__ double sm[2 * (RT / 32)];
  block_sum<2>(a, sm);
  if (threadIdx.x == 0) { num[b] = a[0]; den[b] = a[1] > 0.0 ? a[1] : 1.0; }
}

// d loss / d y3 = gamma mask 2 ewt^2 (z - x) interior / den[b] / nb
__global__ void k_loss_grad(const float* __restrict__ u, const float* __restrict__ y3, const float* __restrict__ mask,
                            const float* __restrict__ ewt, const float* __restrict__ x,
                            const float* __restrict__ gam, const double* __restrict__ den, int nb, int P,
                            float* __restrict__ dy3) {
  const size_t plane = (size_t)P * P;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nb * 3 * plane;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t b = i / (3 * plane), p = i % plane;
    const int yy = (int)(p / P), xx = (int)(p % P);
    float g = 0.f;
    if (!(yy < BORDER || yy >= P - BORDER || xx < BORDER || xx >= P - BORDER)) {
      const float k = mask[b * plane + p];
      const float z = (u[i] + gam[b] * y3[i]) * k;
      const float e = ewt[i] * ewt[i] * (z - x[i]);
      g = (float)(2.0 * e / den[b] / nb) * gam[b] * k;
    }
    dy3[i] = g;
  }
}

__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                       float* __restrict__ m2, int n, float lr, float b1, float b2, float c1, float c2, float eps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi;
  const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = v;
  w[i] -= lr * (a / c1) / (sqrtf(v / c2) + eps);
}

// patch extraction from harvested whole-grid samples (FP64 SoA) into FP32 planes
struct PatchSrc {
  const double* u;
  const double* m;
  const double* ewt;
  const double* x;
};
__global__ void k_extract(const PatchSrc* __restrict__ src, const int4* __restrict__ off, const uint8_t* __restrict__ act,
                          int ng, int ny, int P, float* __restrict__ u, float* __restrict__ m,
                          float* __restrict__ ewt, float* __restrict__ x, float* __restrict__ mask, int nb) {
  const size_t plane = (size_t)P * P;
  const size_t ncell = (size_t)ng * ny;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < nb * plane; i += (size_t)gridDim.x * blockDim.x) {
    const size_t b = i / plane, p = i % plane;
    const int4 o = off[b];   // sample, y0, x0
    const int yy = o.y + (int)(p / P), xx = o.z + (int)(p % P);
    const size_t cell = (size_t)yy * ng + xx;
    const PatchSrc s = src[o.x];
    mask[i] = act ? (float)act[cell] : 1.f;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const size_t d = (b * 3 + a) * plane + p, q = a * ncell + cell;
      u[d] = (float)s.u[q];
      m[d] = (float)s.m[q];
      ewt[d] = (float)s.ewt[q];
      x[d] = (float)s.x[q];
    }
  }
}

// ── inference on the whole grid ──
__global__ void k_feat_grid(const double* __restrict__ z, const double* __restrict__ pm,
                            const uint8_t* __restrict__ act, int n, float* __restrict__ f) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float kk = act ? (float)act[k] : 1.f;
    const float u0 = (float)z[k], u1 = (float)z[n + k], u2 = (float)z[2 * n + k];
    const float m0 = (float)pm[k], m1 = (float)pm[n + k], m2 = (float)pm[2 * n + k];
    const float a0 = m1 * u2 - m2 * u1, a1 = m2 * u0 - m0 * u2, a2 = m0 * u1 - m1 * u0;
    const float b0 = m1 * a2 - m2 * a1, b1 = m2 * a0 - m0 * a2, b2 = m0 * a1 - m1 * a0;
    f[k] = u0 * kk; f[n + k] = u1 * kk; f[2 * n + k] = u2 * kk;
    f[3 * n + k] = a0 * kk; f[4 * n + k] = a1 * kk; f[5 * n + k] = a2 * kk;
    f[6 * n + k] = b0 * kk; f[7 * n + k] = b1 * kk; f[8 * n + k] = b2 * kk;
  }
}

// out = ewt (z + gamma y3) mask; optional sum of out^2 (deterministic partition)
__global__ void __launch_bounds__(RT) k_combine(const double* __restrict__ z, const float* __restrict__ y3,
                                                const double* __restrict__ ewt, const uint8_t* __restrict__ act,
                                                double gamma, int n, double* __restrict__ out, double* partials,
                                                unsigned int* counter, double* res) {
  __shared__ double sm[RT / 32];
  double acc[1] = {0.0};
  for (int k = blockIdx.x * RT + threadIdx.x; k < n; k += gridDim.x * RT) {
    const double kk = act ? (double)act[k] : 1.0;
#pragma unroll
    for (int a = 0; a < 3; a++) {
      const int i = a * n + k;
      const double v = ewt[i] * ((z[i] + gamma * (double)y3[i]) * kk);
      out[i] = v;
      acc[0] += v * v;
    }
  }
  if (res) {
    block_sum<1>(acc, sm);
    finalize<1>(partials, gridDim.x, counter, res, 0, 1.0, acc);
  }
}

__global__ void k_round_bf16(const float* __restrict__ w, float* __restrict__ wq, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) wq[i] = __bfloat162float(__float2bfloat16_rn(w[i]));
}

dim3 conv_grid(int H, int W, int B) { return dim3((W + TW - 1) / TW, (H + TH - 1) / TH, B); }

// ── fused inference on the tensor cores (tcgen05, BF16 operands, FP32 accumulation) ──
// One CTA computes a 32x16 tile of outputs.  The three layers run over the
// tile's 38x22 input region (3-cell halo) held in shared memory as BF16
// activations, laid out [channel chunk of 8][pixel] with one 16-byte row per
// pixel and chunk; that is the K-major operand layout (8-pixel core matrices,
// SBO = 128 B, LBO = one chunk), so the operand of 3x3 tap (dy, dx) for 128
// consecutive pixels is the same layout started dy*38 + dx pixels later: each
// layer is 9 MMAs (M = 128 pixels, N = 16 channels, K = 16) per 128-pixel
// block, accumulated in tensor memory.  Pixels whose taps wrap across the
// region's rows sit in its outer ring, which the next layer's valid outputs
// never read; cells outside the grid are zeroed after every layer (the
// layer-wise zero padding of the network).
constexpr int FO_W = 32, FO_H = 16;
constexpr int FS_W = FO_W + 6, FS_H = FO_H + 6, FNPIX = FS_W * FS_H;   // 38 x 22 = 836
constexpr int FNBLK = (FNPIX + 127) / 128, FNPP = FNBLK * 128;          // 7 blocks, 896
constexpr int FMG = 40;                                                 // zero margin >= 38 + 1
constexpr int FCHUNK = (FNPP + 2 * FMG) * 16;                           // bytes per 8-channel chunk
constexpr int FBUF = 2 * FCHUNK;                                        // 16 channels
constexpr int FWB = 27 * 512;                                           // 3 layers x 9 taps x (16x16 BF16)
constexpr int FSMEM = FWB + 2 * FBUF;
constexpr uint32_t FTMEM = 128;

struct InferArgs {
  const double* z;
  const double* pm;
  const uint8_t* act;
  const double* ewt;
  double* out;
  const uint4* wpack;
  double gamma;
  int ng, ny, ntx, ntiles;
  double* partials;
  unsigned int* counter;
  double* res;
  int* err;
};

union B8 {
  __nv_bfloat16 h[8];
  uint4 u;
};

constexpr int FNT = 512;   // 16 warps: 4 lane quarters x 4 block groups

__global__ void __launch_bounds__(FNT, 2) k_learned_fused(InferArgs a) {
  extern __shared__ __align__(1024) unsigned char smf[];
  unsigned char* sW = smf;
  unsigned char* const buf0 = smf + FWB;
  unsigned char* const buf1 = smf + FWB + FBUF;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  __shared__ int s_fail;
  __shared__ double red[FNT / 32];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, q = warp & 3, hs = warp >> 2;
  const int n = a.ng * a.ny;
  for (int i = tid; i < FWB / 16; i += FNT) reinterpret_cast<uint4*>(sW)[i] = a.wpack[i];
  for (int i = tid; i < 2 * FBUF / 16; i += FNT) reinterpret_cast<uint4*>(buf0)[i] = make_uint4(0, 0, 0, 0);
  if (warp == 0) tmem_alloc(&tslot, FTMEM);
  if (tid == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
    s_fail = 0;
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tslot;
  uint32_t phase = 0;
  double acc[1] = {0.0};
  bool good = true;
  for (int tile = blockIdx.x; tile < a.ntiles && good; tile += gridDim.x) {
    const int x0 = (tile % a.ntx) * FO_W - 3, y0 = (tile / a.ntx) * FO_H - 3;
    // features -> buf0
    for (int p = tid; p < FNPP; p += FNT) {
      float f[16];
#pragma unroll
      for (int k = 0; k < 16; k++) f[k] = 0.f;
      const int gx = x0 + p % FS_W, gy = y0 + p / FS_W;
      if (p < FNPIX && gx >= 0 && gx < a.ng && gy >= 0 && gy < a.ny) {
        const int cell = gy * a.ng + gx;
        if (!a.act || a.act[cell]) {
          const float u0 = (float)a.z[cell], u1 = (float)a.z[n + cell], u2 = (float)a.z[2 * n + cell];
          const float m0 = (float)a.pm[cell], m1 = (float)a.pm[n + cell], m2 = (float)a.pm[2 * n + cell];
          const float a0 = m1 * u2 - m2 * u1, a1 = m2 * u0 - m0 * u2, a2 = m0 * u1 - m1 * u0;
          f[0] = u0; f[1] = u1; f[2] = u2; f[3] = a0; f[4] = a1; f[5] = a2;
          f[6] = m1 * a2 - m2 * a1; f[7] = m2 * a0 - m0 * a2; f[8] = m0 * a1 - m1 * a0;
        }
      }
      B8 c0, c1;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        c0.h[k] = __float2bfloat16_rn(f[k]);
        c1.h[k] = __float2bfloat16_rn(f[8 + k]);
      }
      *reinterpret_cast<uint4*>(buf0 + (FMG + p) * 16) = c0.u;
      *reinterpret_cast<uint4*>(buf0 + FCHUNK + (FMG + p) * 16) = c1.u;
    }
    for (int l = 0; l < 3 && good; l++) {
      unsigned char* src = (l & 1) ? buf1 : buf0;
      unsigned char* dst = (l & 1) ? buf0 : buf1;
      fence_proxy_async_smem();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t idesc = idesc_bf16_f32(128, 16, 0, 0);
        for (int b = 0; b < FNBLK; b++)
          for (int t = 0; t < 9; t++) {
            const int sh = (t / 3 - 1) * FS_W + (t % 3 - 1);
            const uint32_t A = smem_u32(src) + (uint32_t)((FMG + 128 * b + sh) * 16);
            tc_mma_f16(tbase + 16 * b, smem_desc(A, FCHUNK, 128), smem_desc(smem_u32(sW) + (l * 9 + t) * 512, 128, 256),
                       idesc, t > 0 ? 1u : 0u);
          }
        tc_commit(&mbar);
      }
      const bool ok = mbar_wait(&mbar, phase, 1u << 22);
      if (!ok) atomicExch(&s_fail, 1);
      __syncthreads();
      if (s_fail) { good = false; break; }
      phase ^= 1u;
      tc_fence_after();
      for (int b = hs; b < FNBLK; b += FNT / 128) {
        float v[16];
        tmem_ld16(tbase + ((uint32_t)(32 * q) << 16) + 16 * b, v);
        const int p = 128 * b + 32 * q + lane;
        const int ix = p % FS_W, jy = p / FS_W;
        const int gx = x0 + ix, gy = y0 + jy;
        const bool inside = p < FNPIX && gx >= 0 && gx < a.ng && gy >= 0 && gy < a.ny;
        if (l < 2) {
          B8 c0, c1;
#pragma unroll
          for (int k = 0; k < 8; k++) {
            c0.h[k] = __float2bfloat16_rn(inside ? v[k] : 0.f);
            c1.h[k] = __float2bfloat16_rn(inside ? v[8 + k] : 0.f);
          }
          *reinterpret_cast<uint4*>(dst + (FMG + p) * 16) = c0.u;
          *reinterpret_cast<uint4*>(dst + FCHUNK + (FMG + p) * 16) = c1.u;
        } else if (inside && ix >= 3 && ix < FS_W - 3 && jy >= 3 && jy < FS_H - 3) {
          const int cell = gy * a.ng + gx;
          const double k = (!a.act || a.act[cell]) ? 1.0 : 0.0;
#pragma unroll
          for (int c = 0; c < 3; c++) {
            const int i = c * n + cell;
            const double o = a.ewt[i] * ((a.z[i] + a.gamma * (double)v[c]) * k);
            a.out[i] = o;
            acc[0] += o * o;
          }
        }
      }
    }
  }
  if (!good) {
    if (tid == 0) atomicExch(a.err, 1);
    mbar_wait(&mbar, phase, 1u << 22);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, FTMEM);
  }
  if (a.res && good) {
    // deterministic sum of out^2: warp trees, warps in order, CTAs in order
    // by the last CTA to finish (ticket), counter reset for the next use
    __shared__ bool last;
    const double v = warp_sum(acc[0]);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int w = 0; w < FNT / 32; w++) t += red[w];
      a.partials[blockIdx.x] = t;
      __threadfence();
      last = (atomicAdd(a.counter, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (last && tid == 0) {
      __threadfence();
      double t = 0.0;
      for (int k = 0; k < (int)gridDim.x; k++) t += ((volatile double*)a.partials)[k];
      *a.res = t;
      *a.counter = 0u;
    }
  }
}

// FP32 weights -> BF16 B operands: layer l, tap t: (n = out channel, k = in
// channel) K-major, 16 x 16, LBO 128, SBO 256; absent channels zero
__global__ void k_pack_weights(const float* __restrict__ w, uint16_t* __restrict__ pk) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;   // over 27 * 256 entries
  if (e >= 27 * 256) return;
  const int lt = e / 256, l = lt / 9, t = lt % 9, nn = (e % 256) / 16, kk = e % 16;
  const int cin = (l == 0) ? CIN0 : CH, cout = (l == 2) ? COUT3 : CH;
  const int base = (l == 0) ? 0 : (l == 1 ? NW1 : NW1 + NW2);
  float v = 0.f;
  if (nn < cout && kk < cin) v = w[base + (nn * cin + kk) * 9 + t];
  const __nv_bfloat16 h = __float2bfloat16_rn(v);
  pk[(lt * 512 + off_kmajor(nn, kk, 128, 256)) / 2] = *reinterpret_cast<const uint16_t*>(&h);
}

}  // namespace

// ── host side ──────────────────────────────────────────────────────────
struct Learned {
  // weights
  float* d_w = nullptr;      // FP32 master (training)
  float* d_wq = nullptr;     // BF16-rounded copy (FP32 reference inference path)
  uint16_t* d_wpack = nullptr;  // BF16 tensor-core operands of the fused inference kernel
  int* d_err = nullptr;
  bool fused = true;         // fused tensor-core inference (else the FP32 layer-by-layer path)
  float* d_g = nullptr;
  float* d_m1 = nullptr;
  float* d_m2 = nullptr;
  bool have_weights = false;
  int fell_back = 0;         // block-Jacobi fallback: 1 failed solve, 2 not worth its cost
  double pol_it_learned = -1.0, pol_it_bj = -1.0, pol_kappa = -1.0;   // last policy judgement
  int policy = 1;            // 1: cost-aware probing, 0: learned on every solve
  long long napply = 0;
  // inference scratch (whole grid)
  float* d_f = nullptr;      // 9N
  float* d_a1 = nullptr;     // 16N
  float* d_a2 = nullptr;     // 16N
  float* d_y3 = nullptr;     // 3N
  double* d_z = nullptr;     // 3N block-Jacobi output
  // harvest
  int max_samples = 0, stride = 1, nsamples = 0, seen = 0;
  std::vector<double*> hu, hx, hew, hm;
  std::vector<double> hgam;
};

static void lfree(Learned* l) {
  float* fs[] = {l->d_w, l->d_wq, l->d_g, l->d_m1, l->d_m2, l->d_f, l->d_a1, l->d_a2, l->d_y3};
  for (float* p : fs) cudaFree(p);
  cudaFree(l->d_wpack);
  cudaFree(l->d_err);
  cudaFree(l->d_z);
  for (auto* p : l->hu) cudaFree(p);
  for (auto* p : l->hx) cudaFree(p);
  for (auto* p : l->hew) cudaFree(p);
  for (auto* p : l->hm) cudaFree(p);
}

void learned_destroy(Learned* l) {
  if (!l) return;
  lfree(l);
  delete l;
}

static int learned_get(llg_ctx* c, Learned** out) {
  if (!c->learned) {
    Learned* l = new Learned();
    const size_t wb = sizeof(float) * NWT;
    if (cudaMalloc(&l->d_w, wb) != cudaSuccess || cudaMalloc(&l->d_wq, wb) != cudaSuccess ||
        cudaMalloc(&l->d_g, wb) != cudaSuccess || cudaMalloc(&l->d_m1, wb) != cudaSuccess ||
        cudaMalloc(&l->d_m2, wb) != cudaSuccess || cudaMalloc(&l->d_wpack, FWB) != cudaSuccess ||
        cudaMalloc(&l->d_err, sizeof(int)) != cudaSuccess) {
      learned_destroy(l);
      llg_set_error("learned: weight allocation failed");
      return LLG_ERR_NOMEM;
    }
    cudaMemset(l->d_w, 0, wb);
    cudaMemset(l->d_wq, 0, wb);
    cudaMemset(l->d_wpack, 0, FWB);
    cudaMemset(l->d_err, 0, sizeof(int));
    if (cudaFuncSetAttribute((const void*)k_learned_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, FSMEM) !=
        cudaSuccess) {
      learned_destroy(l);
      llg_set_error("learned: shared-memory opt-in failed");
      return LLG_ERR_CUDA;
    }
    c->learned = l;
  }
  *out = c->learned;
  return 0;
}

static int ensure_infer_scratch(llg_ctx* c, Learned* l) {
  if (l->d_f) return 0;
  const size_t n = (size_t)c->ncell;
  if (cudaMalloc(&l->d_f, sizeof(float) * 9 * n) != cudaSuccess ||
      cudaMalloc(&l->d_a1, sizeof(float) * 16 * n) != cudaSuccess ||
      cudaMalloc(&l->d_a2, sizeof(float) * 16 * n) != cudaSuccess ||
      cudaMalloc(&l->d_y3, sizeof(float) * 3 * n) != cudaSuccess ||
      cudaMalloc(&l->d_z, sizeof(double) * 3 * n) != cudaSuccess) {
    llg_set_error("learned: inference scratch allocation failed");
    return LLG_ERR_NOMEM;
  }
  return 0;
}

// network forward on [B][CIN0][H][W] features f -> y3 [B][3][H][W]
static int net_forward(cudaStream_t s, const float* w, const float* f, float* a1, float* a2, float* y3, int B, int H,
                       int W) {
  const dim3 g = conv_grid(H, W, B), b(TW, TH);
  LLG_COUNT(KID_LEARNED);
  k_conv3<CIN0, CH><<<g, b, 0, s>>>(f, w, a1, H, W);
  LLG_COUNT(KID_LEARNED);
  k_conv3<CH, CH><<<g, b, 0, s>>>(a1, w + NW1, a2, H, W);
  LLG_COUNT(KID_LEARNED);
  k_conv3<CH, COUT3><<<g, b, 0, s>>>(a2, w + NW1 + NW2, y3, H, W);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

// learned preconditioner on the whole grid: out = ewt (z + gamma Net(z; pm)) mask,
// z = block-Jacobi solve already in l->d_z; optional sum of out^2 -> d_scal[slot]
int learned_apply(llg_ctx* c, const double* ewt, double* out, int slot) {
  Learned* l = c->learned;
  if (!l || !l->have_weights) { llg_set_error("learned preconditioner has no weights"); return LLG_ERR_STATE; }
  int rc = ensure_infer_scratch(c, l);
  if (rc) return rc;
  const int n = c->ncell;
  if (l->fused) {
    InferArgs a{};
    a.z = l->d_z; a.pm = c->d_pm; a.act = c->d_act; a.ewt = ewt; a.out = out;
    a.wpack = reinterpret_cast<const uint4*>(l->d_wpack);
    a.gamma = c->gamma_setup;
    a.ng = c->p.ng; a.ny = c->p.ny;
    a.ntx = (c->p.ng + FO_W - 1) / FO_W;
    a.ntiles = a.ntx * ((c->p.ny + FO_H - 1) / FO_H);
    a.partials = c->d_red; a.counter = c->d_counter;
    a.res = slot >= 0 ? c->d_scal + slot : nullptr;
    a.err = l->d_err;
    const int grid = std::min(a.ntiles, 2 * c->num_sms);
    LLG_COUNT(KID_LEARNED);
    k_learned_fused<<<grid, FNT, FSMEM, c->stream>>>(a);
    LLG_CUDA_TRY(cudaPeekAtLastError());
    l->napply++;
    return 0;
  }
  LLG_COUNT(KID_LEARNED);
  k_feat_grid<<<c->num_sms * 8, 256, 0, c->stream>>>(l->d_z, c->d_pm, c->d_act, n, l->d_f);
  if ((rc = net_forward(c->stream, l->d_wq, l->d_f, l->d_a1, l->d_a2, l->d_y3, 1, c->p.ny, c->p.ng))) return rc;
  LLG_COUNT(KID_LEARNED);
  k_combine<<<red_blocks(n), RT, 0, c->stream>>>(l->d_z, l->d_y3, ewt, c->d_act, c->gamma_setup, n, out, c->d_red,
                                                c->d_counter, slot >= 0 ? c->d_scal + slot : nullptr);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  l->napply++;
  return 0;
}

double* learned_zbuf(llg_ctx* c) {
  Learned* l = c->learned;
  if (!l || ensure_infer_scratch(c, l)) return nullptr;
  return l->d_z;
}

bool learned_active(llg_ctx* c) {
  return c->p.precond_kind == LLG_PREC_LEARNED && c->learned && c->learned->have_weights && !c->learned->fell_back;
}

void learned_fall_back(llg_ctx* c, int reason) {
  if (c->learned) c->learned->fell_back = reason;
}

bool learned_policy_on(llg_ctx* c) { return c->learned && c->learned->policy; }

void learned_policy_record(llg_ctx* c, double it_learned, double it_bj, double kappa) {
  if (!c->learned) return;
  c->learned->pol_it_learned = it_learned;
  c->learned->pol_it_bj = it_bj;
  c->learned->pol_kappa = kappa;
}

// ── harvesting (called by the integrator after a converged block-Jacobi solve) ──
bool learned_harvest_wanted(llg_ctx* c) {
  Learned* l = c->learned;
  return l && l->max_samples > 0 && l->nsamples < l->max_samples;
}

// u = P_BJ^-1 r (already computed into u_src), x solution, ewt, frozen m
int learned_harvest(llg_ctx* c, const double* u_src, const double* x, const double* ewt, double gamma) {
  Learned* l = c->learned;
  if (!learned_harvest_wanted(c)) return 0;
  if ((l->seen++ % l->stride) != 0) return 0;
  const size_t vb = sizeof(double) * 3 * (size_t)c->ncell;
  double *u = nullptr, *xx = nullptr, *e = nullptr, *m = nullptr;
  if (cudaMalloc(&u, vb) != cudaSuccess || cudaMalloc(&xx, vb) != cudaSuccess || cudaMalloc(&e, vb) != cudaSuccess ||
      cudaMalloc(&m, vb) != cudaSuccess) {
    cudaFree(u); cudaFree(xx); cudaFree(e); cudaFree(m);
    l->max_samples = l->nsamples;   // out of memory: stop harvesting
    return 0;
  }
  LLG_CUDA_TRY(cudaMemcpyAsync(u, u_src, vb, cudaMemcpyDeviceToDevice, c->stream));
  LLG_CUDA_TRY(cudaMemcpyAsync(xx, x, vb, cudaMemcpyDeviceToDevice, c->stream));
  LLG_CUDA_TRY(cudaMemcpyAsync(e, ewt, vb, cudaMemcpyDeviceToDevice, c->stream));
  LLG_CUDA_TRY(cudaMemcpyAsync(m, c->d_pm, vb, cudaMemcpyDeviceToDevice, c->stream));
  l->hu.push_back(u); l->hx.push_back(xx); l->hew.push_back(e); l->hm.push_back(m);
  l->hgam.push_back(gamma);
  l->nsamples++;
  return 0;
}

// ── training ──
struct TrainBuf {
  float *u = nullptr, *m = nullptr, *ewt = nullptr, *x = nullptr, *mask = nullptr, *gam = nullptr;
  float *f = nullptr, *a1 = nullptr, *a2 = nullptr, *y3 = nullptr;
  float *d3 = nullptr, *d2 = nullptr, *d1 = nullptr, *part = nullptr;
  double *num = nullptr, *den = nullptr;
  PatchSrc* src = nullptr;
  int4* off = nullptr;
  void release() {
    float* fs[] = {u, m, ewt, x, mask, gam, f, a1, a2, y3, d3, d2, d1, part};
    for (float* p : fs) cudaFree(p);
    cudaFree(num); cudaFree(den); cudaFree(src); cudaFree(off);
  }
};

static int train_alloc(TrainBuf& t, int nb, int P) {
  const size_t pl = (size_t)nb * P * P;
  const int nblk = ((P + TW - 1) / TW) * ((P + TH - 1) / TH) * nb;
  bool ok = cudaMalloc(&t.u, 4 * 3 * pl) == cudaSuccess && cudaMalloc(&t.m, 4 * 3 * pl) == cudaSuccess &&
            cudaMalloc(&t.ewt, 4 * 3 * pl) == cudaSuccess && cudaMalloc(&t.x, 4 * 3 * pl) == cudaSuccess &&
            cudaMalloc(&t.mask, 4 * pl) == cudaSuccess && cudaMalloc(&t.gam, 4 * nb) == cudaSuccess &&
            cudaMalloc(&t.f, 4 * 9 * pl) == cudaSuccess && cudaMalloc(&t.a1, 4 * 16 * pl) == cudaSuccess &&
            cudaMalloc(&t.a2, 4 * 16 * pl) == cudaSuccess && cudaMalloc(&t.y3, 4 * 3 * pl) == cudaSuccess &&
            cudaMalloc(&t.d3, 4 * 3 * pl) == cudaSuccess && cudaMalloc(&t.d2, 4 * 16 * pl) == cudaSuccess &&
            cudaMalloc(&t.d1, 4 * 16 * pl) == cudaSuccess &&
            cudaMalloc(&t.part, 4 * (size_t)nblk * NW2) == cudaSuccess &&
            cudaMalloc(&t.num, 8 * nb) == cudaSuccess && cudaMalloc(&t.den, 8 * nb) == cudaSuccess;
  if (!ok) {
    t.release();
    llg_set_error("learned: training buffer allocation failed");
    return LLG_ERR_NOMEM;
  }
  return 0;
}

// loss (mean over patches, read back only if want_loss) and gradient d_g for
// the batch already in t (u, m, ewt, x, mask, gam)
static int train_fwd_bwd(cudaStream_t s, const float* w, float* g, TrainBuf& t, int nb, int P, double* loss) {
  const dim3 cg = conv_grid(P, P, nb), cb(TW, TH);
  const int nblk = cg.x * cg.y * cg.z;
  const size_t pl = (size_t)nb * P * P;
  const int eg = (int)std::min<size_t>((pl + 255) / 256, 4096);
  LLG_COUNT(KID_LEARNED);
  k_feat_patch<<<eg, 256, 0, s>>>(t.u, t.m, t.mask, t.f, nb, P);
  int rc = net_forward(s, w, t.f, t.a1, t.a2, t.y3, nb, P, P);
  if (rc) return rc;
  LLG_COUNT(KID_LEARNED);
  k_loss_terms<<<nb, 256, 0, s>>>(t.u, t.y3, t.mask, t.ewt, t.x, t.gam, P, t.num, t.den);
  LLG_COUNT(KID_LEARNED);
  k_loss_grad<<<eg, 256, 0, s>>>(t.u, t.y3, t.mask, t.ewt, t.x, t.gam, t.den, nb, P, t.d3);
  // layer 3
  LLG_COUNT(KID_LEARNED);
  k_conv3_bwd_w<CH, COUT3><<<cg, cb, 0, s>>>(t.a2, t.d3, t.part, P, P);
  LLG_COUNT(KID_LEARNED);
  k_sum_parts<<<(NW3 + 255) / 256, 256, 0, s>>>(t.part, nblk, NW3, g + NW1 + NW2);
  LLG_COUNT(KID_LEARNED);
  k_conv3_bwd_data<CH, COUT3><<<cg, cb, 0, s>>>(t.d3, w + NW1 + NW2, t.d2, P, P);
  // layer 2
  LLG_COUNT(KID_LEARNED);
  k_conv3_bwd_w<CH, CH><<<cg, cb, 0, s>>>(t.a1, t.d2, t.part, P, P);
  LLG_COUNT(KID_LEARNED);
  k_sum_parts<<<(NW2 + 255) / 256, 256, 0, s>>>(t.part, nblk, NW2, g + NW1);
  LLG_COUNT(KID_LEARNED);
  k_conv3_bwd_data<CH, CH><<<cg, cb, 0, s>>>(t.d2, w + NW1, t.d1, P, P);
  // layer 1
  LLG_COUNT(KID_LEARNED);
  k_conv3_bwd_w<CIN0, CH><<<cg, cb, 0, s>>>(t.f, t.d1, t.part, P, P);
  LLG_COUNT(KID_LEARNED);
  k_sum_parts<<<(NW1 + 255) / 256, 256, 0, s>>>(t.part, nblk, NW1, g);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  if (loss) {
    std::vector<double> num(nb), den(nb);
    LLG_CUDA_TRY(cudaMemcpyAsync(num.data(), t.num, 8 * nb, cudaMemcpyDeviceToHost, s));
    LLG_CUDA_TRY(cudaMemcpyAsync(den.data(), t.den, 8 * nb, cudaMemcpyDeviceToHost, s));
    LLG_CUDA_TRY(cudaStreamSynchronize(s));
    double L = 0.0;
    for (int b = 0; b < nb; b++) L += num[b] / den[b];
    *loss = L / nb;
  }
  return 0;
}

extern "C" {

int llg_learned_harvest(llg_ctx* c, int32_t max_samples, int32_t stride) {
  if (!c || max_samples < 0 || stride < 1) { llg_set_error("llg_learned_harvest: bad argument"); return LLG_ERR_ARG; }
  Learned* l;
  int rc = learned_get(c, &l);
  if (rc) return rc;
  l->max_samples = max_samples;
  l->stride = stride;
  return 0;
}

int llg_learned_num_samples(llg_ctx* c) { return (c && c->learned) ? c->learned->nsamples : 0; }

int llg_learned_set_weights(llg_ctx* c, const float* h_w, int32_t n) {
  if (!c || !h_w || n != NWT) { llg_set_error("llg_learned_set_weights: need 4032 weights"); return LLG_ERR_ARG; }
  Learned* l;
  int rc = learned_get(c, &l);
  if (rc) return rc;
  LLG_CUDA_TRY(cudaMemcpy(l->d_w, h_w, sizeof(float) * NWT, cudaMemcpyHostToDevice));
  k_round_bf16<<<(NWT + 255) / 256, 256, 0, c->stream>>>(l->d_w, l->d_wq, NWT);
  k_pack_weights<<<(27 * 256 + 255) / 256, 256, 0, c->stream>>>(l->d_w, l->d_wpack);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  l->have_weights = true;
  l->fell_back = 0;
  return 0;
}

int llg_learned_get_weights(llg_ctx* c, float* h_w, int32_t n) {
  if (!c || !h_w || n != NWT || !c->learned) { llg_set_error("llg_learned_get_weights: no weights"); return LLG_ERR_ARG; }
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  LLG_CUDA_TRY(cudaMemcpy(h_w, c->learned->d_w, sizeof(float) * NWT, cudaMemcpyDeviceToHost));
  return 0;
}

int llg_learned_policy(llg_ctx* c, double* it_learned, double* it_bj, double* kappa) {
  if (!c) return LLG_ERR_ARG;
  const Learned* l = c->learned;
  if (it_learned) *it_learned = l ? l->pol_it_learned : -1.0;
  if (it_bj) *it_bj = l ? l->pol_it_bj : -1.0;
  if (kappa) *kappa = l ? l->pol_kappa : -1.0;
  return 0;
}

int llg_learned_set_policy(llg_ctx* c, int32_t cost_aware) {
  if (!c) return LLG_ERR_ARG;
  Learned* l;
  int rc = learned_get(c, &l);
  if (rc) return rc;
  l->policy = cost_aware != 0;
  return 0;
}

int llg_learned_set_fused(llg_ctx* c, int32_t fused) {
  if (!c) return LLG_ERR_ARG;
  Learned* l;
  int rc = learned_get(c, &l);
  if (rc) return rc;
  l->fused = fused != 0;
  return 0;
}

// out = ewt (z + gamma Net(z; pm)) on active cells for caller-given z, frozen
// m (pm) and gamma (checker entry point of the inference kernels); writes
// sum out^2 to *norm2 when it is not null
int llg_learned_apply(llg_ctx* c, const double* d_z, const double* d_pm, const double* d_ewt, double gamma,
                      double* d_out, double* norm2) {
  if (!c || !d_z || !d_pm || !d_ewt || !d_out) return LLG_ERR_ARG;
  if (!c->learned || !c->learned->have_weights) { llg_set_error("llg_learned_apply: no weights"); return LLG_ERR_STATE; }
  int rc = ensure_infer_scratch(c, c->learned);
  if (rc) return rc;
  const size_t vb = sizeof(double) * 3 * (size_t)c->ncell;
  LLG_CUDA_TRY(cudaMemcpyAsync(c->learned->d_z, d_z, vb, cudaMemcpyDeviceToDevice, c->stream));
  LLG_CUDA_TRY(cudaMemcpyAsync(c->d_pm, d_pm, vb, cudaMemcpyDeviceToDevice, c->stream));
  const double g0 = c->gamma_setup;
  c->gamma_setup = gamma;
  rc = learned_apply(c, d_ewt, d_out, 60);
  c->gamma_setup = g0;
  if (rc) return rc;
  double s = 0.0;
  LLG_CUDA_TRY(cudaMemcpyAsync(&s, c->d_scal + 60, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  int fail = 0;
  LLG_CUDA_TRY(cudaMemcpy(&fail, c->learned->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (fail) { llg_set_error("learned inference: a tensor-core completion wait ran out"); return LLG_ERR_TIMEOUT; }
  if (norm2) *norm2 = s;
  return 0;
}

int llg_learned_status(llg_ctx* c, int32_t* active, int32_t* fell_back, int64_t* napply) {
  if (!c) return LLG_ERR_ARG;
  if (active) *active = learned_active(c) ? 1 : 0;
  if (fell_back) *fell_back = c->learned ? c->learned->fell_back : 0;
  if (napply) *napply = c->learned ? c->learned->napply : 0;
  return 0;
}

int llg_learned_train(llg_ctx* c, const llg_train_opts* o, double* loss_first, double* loss_last) {
  if (!c || !o || o->iters < 1 || o->batch < 1 || o->patch < 2 * BORDER + 2 || !(o->lr > 0.0)) {
    llg_set_error("llg_learned_train: bad options");
    return LLG_ERR_ARG;
  }
  Learned* l;
  int rc = learned_get(c, &l);
  if (rc) return rc;
  if (l->nsamples < 1) { llg_set_error("llg_learned_train: no harvested samples"); return LLG_ERR_STATE; }
  const int P = std::min(o->patch, std::min(c->p.ng, c->p.ny));
  const int nb = o->batch;
  cudaStream_t s = c->stream;
  TrainBuf t;
  if ((rc = train_alloc(t, nb, P))) return rc;
  std::vector<PatchSrc> src(l->nsamples);
  for (int k = 0; k < l->nsamples; k++) src[k] = PatchSrc{l->hu[k], l->hm[k], l->hew[k], l->hx[k]};
  if (cudaMalloc(&t.src, sizeof(PatchSrc) * src.size()) != cudaSuccess ||
      cudaMalloc(&t.off, sizeof(int4) * nb) != cudaSuccess) {
    t.release();
    llg_set_error("learned: allocation failed");
    return LLG_ERR_NOMEM;
  }
  LLG_CUDA_TRY(cudaMemcpy(t.src, src.data(), sizeof(PatchSrc) * src.size(), cudaMemcpyHostToDevice));
  // initial weights: small seeded values unless weights are already present
  std::mt19937_64 rng((uint64_t)o->seed);
  if (!l->have_weights) {
    std::vector<float> w0(NWT);
    std::normal_distribution<float> nd(0.f, 1.f);
    const float s1 = (float)o->init_scale / sqrtf(9.f * CIN0), s2 = (float)o->init_scale / sqrtf(9.f * CH);
    for (int i = 0; i < NWT; i++) w0[i] = nd(rng) * (i < NW1 ? s1 : s2);
    LLG_CUDA_TRY(cudaMemcpy(l->d_w, w0.data(), sizeof(float) * NWT, cudaMemcpyHostToDevice));
  }
  LLG_CUDA_TRY(cudaMemsetAsync(l->d_m1, 0, sizeof(float) * NWT, s));
  LLG_CUDA_TRY(cudaMemsetAsync(l->d_m2, 0, sizeof(float) * NWT, s));
  std::vector<int4> off(nb);
  std::vector<float> gam(nb);
  std::uniform_int_distribution<int> ds(0, l->nsamples - 1), dy(0, c->p.ny - P), dx(0, c->p.ng - P);
  const float b1 = 0.9f, b2 = 0.999f;
  float c1 = 1.f, c2 = 1.f;
  const size_t pl = (size_t)nb * P * P;
  const int eg = (int)std::min<size_t>((pl + 255) / 256, 4096);
  for (int it = 0; it < o->iters; it++) {
    for (int b = 0; b < nb; b++) {
      const int k = ds(rng);
      off[b] = make_int4(k, dy(rng), dx(rng), 0);
      gam[b] = (float)l->hgam[k];
    }
    LLG_CUDA_TRY(cudaMemcpyAsync(t.off, off.data(), sizeof(int4) * nb, cudaMemcpyHostToDevice, s));
    LLG_CUDA_TRY(cudaMemcpyAsync(t.gam, gam.data(), sizeof(float) * nb, cudaMemcpyHostToDevice, s));
    LLG_COUNT(KID_LEARNED);
    k_extract<<<eg, 256, 0, s>>>(t.src, t.off, c->d_act, c->p.ng, c->p.ny, P, t.u, t.m, t.ewt, t.x, t.mask, nb);
    double L = 0.0;
    const bool want = (it == 0 && loss_first) || (it == o->iters - 1 && loss_last);
    if ((rc = train_fwd_bwd(s, l->d_w, l->d_g, t, nb, P, want ? &L : nullptr))) { t.release(); return rc; }
    if (it == 0 && loss_first) *loss_first = L;
    if (it == o->iters - 1 && loss_last) *loss_last = L;
    c1 *= b1;
    c2 *= b2;
    LLG_COUNT(KID_LEARNED);
    k_adam<<<(NWT + 255) / 256, 256, 0, s>>>(l->d_w, l->d_g, l->d_m1, l->d_m2, NWT, (float)o->lr, b1, b2, 1.f - c1,
                                             1.f - c2, 1e-8f);
    LLG_CUDA_TRY(cudaPeekAtLastError());
  }
  k_round_bf16<<<(NWT + 255) / 256, 256, 0, s>>>(l->d_w, l->d_wq, NWT);
  k_pack_weights<<<(27 * 256 + 255) / 256, 256, 0, s>>>(l->d_w, l->d_wpack);
  LLG_CUDA_TRY(cudaStreamSynchronize(s));
  t.release();
  l->have_weights = true;
  l->fell_back = 0;
  return 0;
}

// Loss, gradient and network output for host-provided FP32 patches (checker
// entry point for the training kernels; no context needed).
int llg_learned_loss_grad(const float* h_w, int32_t nb, int32_t P, const float* h_u, const float* h_m,
                          const float* h_mask, const float* h_ewt, const float* h_x, const float* h_gamma,
                          double* loss, float* h_grad, float* h_z) {
  if (!h_w || nb < 1 || P < 2 * BORDER + 2 || !h_u || !h_m || !h_mask || !h_ewt || !h_x || !h_gamma || !loss ||
      !h_grad) {
    llg_set_error("llg_learned_loss_grad: bad argument");
    return LLG_ERR_ARG;
  }
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
    llg_set_error("no CUDA device: libllg.so has no CPU path");
    return LLG_ERR_CUDA;
  }
  TrainBuf t;
  int rc = train_alloc(t, nb, P);
  if (rc) return rc;
  float *w = nullptr, *g = nullptr;
  const size_t pl = (size_t)nb * P * P;
  auto done = [&](int r) { t.release(); cudaFree(w); cudaFree(g); return r; };
  if (cudaMalloc(&w, sizeof(float) * NWT) != cudaSuccess || cudaMalloc(&g, sizeof(float) * NWT) != cudaSuccess)
    return done(LLG_ERR_NOMEM);
  if (cudaMemcpy(w, h_w, sizeof(float) * NWT, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t.u, h_u, 12 * pl, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t.m, h_m, 12 * pl, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t.ewt, h_ewt, 12 * pl, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t.x, h_x, 12 * pl, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t.mask, h_mask, 4 * pl, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t.gam, h_gamma, 4 * nb, cudaMemcpyHostToDevice) != cudaSuccess) {
    llg_set_error("llg_learned_loss_grad: upload failed");
    return done(LLG_ERR_CUDA);
  }
  if ((rc = train_fwd_bwd(0, w, g, t, nb, P, loss))) return done(rc);
  if (cudaMemcpy(h_grad, g, sizeof(float) * NWT, cudaMemcpyDeviceToHost) != cudaSuccess) return done(LLG_ERR_CUDA);
  if (h_z) {
    // z = (u + gamma y3) mask, assembled on the host from the device y3
    std::vector<float> y3(3 * pl), u(h_u, h_u + 3 * pl);
    if (cudaMemcpy(y3.data(), t.y3, 12 * pl, cudaMemcpyDeviceToHost) != cudaSuccess) return done(LLG_ERR_CUDA);
    const size_t plane = (size_t)P * P;
    for (int b = 0; b < nb; b++)
      for (int a = 0; a < 3; a++)
        for (size_t p = 0; p < plane; p++) {
          const size_t i = ((size_t)b * 3 + a) * plane + p;
          h_z[i] = (u[i] + h_gamma[b] * y3[i]) * h_mask[b * plane + p];
        }
  }
  return done(0);
}

}  // extern "C"
