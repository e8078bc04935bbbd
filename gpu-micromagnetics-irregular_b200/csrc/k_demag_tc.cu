// k_demag_tc.cu — tensor-core column stage of the mixed-precision demag chain
// (sm_100a: tcgen05.mma from shared-memory descriptors into TMEM).
//
// The FP64 chain's column stage (k_demag.cu, K2) transforms each x-frequency
// column of the row spectrum along y, multiplies by the tensor spectra and
// transforms back (the reference's cufftExecD2Z/Z2D column half and
// multiply_kernel, src/irregular/2d_fft/2d_i2/demag_fft.cu:106-141, :342-353).
// Here, for transform length P = 1024 = 32 x 32 with ny = 512 (open film,
// zero-padded) or 1024 data rows, the column transform is a four-step DFT
// whose two 32-point stages are real-ified complex GEMMs on the tensor cores:
//
//   forward  n = 32 n1 + n2,  k = k1 + 32 k2
//     F1: Y[k1; n2]  = sum_{n1 < D1} x[32 n1 + n2] w32^(n1 k1)     (GEMM, K = 2 D1)
//         Y'         = Y * w1024^(n2 k1)                          (epilogue, FP32)
//     F2: X[k1 + 32 k2] = sum_{n2} Y'[k1; n2] w32^(n2 k2)         (GEMM, K = 64)
//   multiply  H = N X (3x3 film tensor: xx, yy, zz, xy = yx), FP32, in registers
//   inverse (as conj o forward o conj, so the same DFT matrices serve)
//     G2: conj Z[k1; n2] = sum_{k2} conj H[k1 + 32 k2] w32^(n2 k2)
//         epilogue: * w1024^(n2 k1)
//     G1: conj x[32 n1 + n2] = sum_{k1} (...) w32^(n1 k1),  n1 < D1 only
//
// Operands are FP16: every FP32 value v is split into hi = fp16(v) and
// lo' = fp16(2^11 (v - hi)) (scaled so it stays a normal FP16 number); each
// GEMM accumulates Ahi*Bhi into one FP32 tensor-memory accumulator and
// Alo'*Bhi + Ahi*Blo' into a second, and the epilogue forms hi + 2^-11 lo
// (the lo*lo term, ~2^-22 relative, is dropped).  Exact
// power-of-two scalings keep every FP16 operand within [-1, 1]: per
// (component, column) the input is scaled by its own 2^-e (warp max), the
// tensor by a global 2^e_t, and each 32-term stage by 2^-5 (2^-6 after the
// 2-term tensor sum); the final store undoes them exactly.
//
// CTA: 12 warps, one group of 4 x-frequency columns at a time (persistent
// over groups).  Warp w handles component c = w/4 and TMEM lane quarter
// q = w%4, i.e. column 4g+q: GEMM rows are (column, 32 indices), one
// 128-row M tile per component, so the tensor multiply finds the three
// components of one (column, frequency) in the same thread.  Tensor memory:
// component c uses columns [128c, 128c+64) (hi) and [128c+64, 128c+128) (lo)
// in every stage; a stage's accumulators are read back before the next
// stage's MMAs are issued.
#include <cuda_fp16.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "dev_tc.cuh"
#include "llg_internal.h"
#include "launch.h"

namespace {

constexpr int P = 1024;
constexpr int NCOL = 4;                           // x-frequency columns per group
constexpr int NWARP = 12, NT = NWARP * 32;
constexpr int kTcWpr = 2;                         // warps per (component, lane quarter) role
constexpr int LBO_K = 128;                        // K-major: K-adjacent core matrices
constexpr int SBO_MN = 128, LBO_MN = 16 * 128 + 16;  // MN-major, M = 128 (16 B pad per K group)
constexpr int AMAT = 8 * LBO_MN;                  // one 128 x 64 FP16 operand, either layout
constexpr int ACOMP = 2 * AMAT;                   // hi + lo
constexpr uint32_t TMEM_COLS = 512;
constexpr uint32_t WAIT_LIMIT = 1u << 22;

__host__ __device__ constexpr int bbytes_for(int D1) { return 1024 * D1 + 16384; }

struct TcArgs {
  float2* S;
  int hx, ld, ngroups;
  const float* txx;
  const float* tyy;
  const float* tzz;
  const float2* txy;
  const float2* tw;     // exp(-2 pi i j / 1024), j < 1024
  const uint4* bmat;    // B operands, in their shared-memory layout
  float s_t;            // 2^e_t * 2^-6
  int e_t;
  int* err;
};

union H8 {
  __half h[8];
  __half2 h2[4];
  uint4 u;
};

// split products over `ksteps` K=16 steps: D_hi = Ahi Bhi, D_lo = Alo' Bhi + Ahi Blo'
__device__ __forceinline__ void issue3(uint32_t d, uint32_t aH, uint32_t aL, uint32_t bH, uint32_t bL, int ksteps,
                                       uint32_t a_step, uint32_t alb, uint32_t asb, uint32_t bsb, uint32_t idesc) {
#pragma unroll 1
  for (int p = 0; p < 3; p++) {
    const uint32_t A = (p == 1) ? aL : aH;
    const uint32_t B = (p == 2) ? bL : bH;
    const uint32_t dd = (p == 0) ? d : d + 64;
#pragma unroll 1
    for (int s = 0; s < ksteps; s++)
      tc_mma_f16(dd, smem_desc(A + s * a_step, alb, asb), smem_desc(B + s * 256, LBO_K, bsb), idesc,
                 (p == 2 || s > 0) ? 1u : 0u);
  }
}

// hi + 2^-11 lo of 16 accumulator columns starting at column `col` of this warp's lanes
__device__ __forceinline__ void acc_ld16(uint32_t tl, uint32_t col, float (&v)[16]) {
  float lo[16];
  tmem_ld16x2(tl + col, tl + col + 64, v, lo);
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = fmaf(lo[i], LO_UNSCALE, v[i]);
}
// the same for 8 columns
__device__ __forceinline__ void acc_ld8(uint32_t tl, uint32_t col, float (&v)[8]) {
  float lo[8];
  tmem_ld8x2(tl + col, tl + col + 64, v, lo);
#pragma unroll
  for (int i = 0; i < 8; i++) v[i] = fmaf(lo[i], LO_UNSCALE, v[i]);
}

template <int D1, int WPR>
__global__ void __launch_bounds__(NT * WPR, 1) k_cols_tc(TcArgs a) {
  pdl_entry();
  constexpr int NTW = NT * WPR;
  constexpr int K1 = 2 * D1;
  constexpr int oF1h = 0, oF1l = 128 * K1, oF2h = 256 * K1, oF2l = oF2h + 8192, oG1h = oF2h + 16384,
                oG1l = oG1h + 256 * D1;
  constexpr int BB = bbytes_for(D1);
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* Ab = sm + BB;
  __shared__ uint64_t mbar[2];    // per team: the MMA completion of its stage
  __shared__ uint32_t tmem_slot;
  __shared__ int s_fail[2];
  __shared__ int s_e[3][NCOL];    // per (component, column) input exponent
  __shared__ int s_eo[3][NCOL];   // exponent carried by the tensor product
  __shared__ float2 s_tw[32][32]; // w1024^(k l) at [k][l]: lane l reads [k][l], no bank conflicts

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // WPR warps share each (component, TMEM lane quarter) role, each taking
  // its share of the accumulator column blocks in every epilogue
  const int q = warp & 3, role = warp >> 2, c = role / WPR, h = role - c * WPR;
  // Two teams run the stage sequence independently: warps 0-7 the coupled x
  // and y components, warps 8-11 the z component.  Each has its own named
  // barrier, MMA-issuing thread and completion mbarrier, so one team's
  // epilogue (CUDA cores, TMEM read-back) overlaps the other's MMAs and
  // neither waits at the other's barriers.
  const int team = (c < 2) ? 0 : 1;
  const int team_lead = team ? 256 * WPR : 0, team_threads = team ? 128 * WPR : 256 * WPR;
  const int c_lo = team ? 2 : 0, c_hi = team ? 3 : 2;
  auto team_sync = [&]() {
    asm volatile("bar.sync %0, %1;\n" ::"r"(1 + team), "r"(team_threads) : "memory");
  };

  for (int i = tid; i < BB / 16; i += NTW) reinterpret_cast<uint4*>(sm)[i] = a.bmat[i];
  for (int i = tid; i < 32 * 32; i += NTW) s_tw[i >> 5][i & 31] = a.tw[((i >> 5) * (i & 31)) & (P - 1)];
  if (warp == 0) tmem_alloc(&tmem_slot, TMEM_COLS);
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    mbar_init_fence();
    s_fail[0] = 0;
    s_fail[1] = 0;
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmem_slot;
  const uint32_t tl = tbase + ((uint32_t)(32 * q) << 16);
  const uint32_t sA = smem_u32(Ab), sB = smem_u32(sm);
  unsigned char* Ah = Ab + c * ACOMP;
  unsigned char* Al = Ah + AMAT;
  uint32_t phase = 0;

  // team barrier + the team's lead thread issues the stage's MMAs for the
  // team's components + the team waits for them
  auto run_stage = [&](int st) -> bool {
    fence_proxy_async_smem();
    tc_fence_before();
    team_sync();
    if (tid == team_lead) {
      tc_fence_after();
      for (int cc = c_lo; cc < c_hi; cc++) {
        const uint32_t aH = sA + cc * ACOMP, aL = aH + AMAT;
        if (st == 0)
          issue3(tbase + 128 * cc, aH, aL, sB + oF1h, sB + oF1l, K1 / 16, 2 * LBO_K, LBO_K, K1 * 16, K1 * 16,
                 idesc_f16_f32(128, 64, 0, 0));
        else if (st == 1)
          issue3(tbase + 128 * cc, aH, aL, sB + oF2h, sB + oF2l, 4, 2 * LBO_MN, LBO_MN, SBO_MN, 1024,
                 idesc_f16_f32(128, 64, 1, 0));
        else if (st == 2)
          issue3(tbase + 128 * cc, aH, aL, sB + oF2h, sB + oF2l, 4, 2 * LBO_K, LBO_K, 1024, 1024,
                 idesc_f16_f32(128, 64, 0, 0));
        else
          issue3(tbase + 128 * cc, aH, aL, sB + oG1h, sB + oG1l, 4, 2 * LBO_MN, LBO_MN, SBO_MN, 1024,
                 idesc_f16_f32(128, 2 * D1, 1, 0));
      }
      tc_commit(&mbar[team]);
    }
    const bool ok = mbar_wait(&mbar[team], phase, WAIT_LIMIT);
    if (!ok) atomicExch(&s_fail[team], 1);
    team_sync();
    if (s_fail[team]) return false;   // phase left pending for the bounded drain below
    phase ^= 1u;
    tc_fence_after();
    return true;
  };

  // L2 prefetch of one group's tensor columns (and, for a later group, its
  // spectrum columns): the tensor multiply and the next group's F1 loads then
  // read L2 instead of waiting on HBM
  auto prefetch_group = [&](int gg, bool spectrum) {
    if (tid != 0 || gg >= a.ngroups) return;
    for (int qq = 0; qq < NCOL; qq++) {
      const int k2 = gg * NCOL + qq;
      if (k2 >= a.hx) break;
      const long long tb = (long long)k2 * P;
      prefetch_l2_bulk(a.txx + tb, P * sizeof(float));
      prefetch_l2_bulk(a.tyy + tb, P * sizeof(float));
      prefetch_l2_bulk(a.tzz + tb, P * sizeof(float));
      prefetch_l2_bulk(a.txy + tb, P * sizeof(float2));
      if (spectrum)
        for (int cc = 0; cc < 3; cc++)
          prefetch_l2_bulk(a.S + ((long long)cc * a.hx + k2) * a.ld, (uint32_t)(a.ld * sizeof(float2)));
    }
  };
  prefetch_group(blockIdx.x, false);
  bool good = true;
  for (int g = blockIdx.x; g < a.ngroups && good; g += gridDim.x) {
    prefetch_group(g + gridDim.x, true);
    const int kx = g * NCOL + q;
    const bool colok = kx < a.hx;
    // ── F1 operand: rows 32q + n2, K = (n1, re/im), this warp's own row ──
    {
      const float2* src = a.S + ((long long)c * a.hx + (colok ? kx : 0)) * a.ld;
      float2 v[D1];
      float mx = 0.f;
#pragma unroll
      for (int n1 = 0; n1 < D1; n1++) {
        v[n1] = colok ? src[32 * n1 + lane] : make_float2(0.f, 0.f);
        mx = fmaxf(mx, fmaxf(fabsf(v[n1].x), fabsf(v[n1].y)));
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      int e = 0;
      if (mx > 0.f) frexpf(mx, &e);   // mx < 2^e
      e = max(e, -127);               // 2^-e stays a finite float (subnormal-only columns)
      if (lane == 0 && h == 0) s_e[c][q] = e;
      const float sc = ldexpf(1.f, -e);   // v * 2^-e: exact, or rounded as ldexpf rounds
      const int r = 32 * q + lane;
#pragma unroll
      for (int j = 0; j < K1 / 8; j++) {
        if (j / (K1 / 8 / WPR) != h) continue;   // this warp's share of the K chunks
        H8 hh, ll;
#pragma unroll
        for (int t = 0; t < 4; t++) split_h2(v[4 * j + t].x * sc, v[4 * j + t].y * sc, hh.h2[t], ll.h2[t]);
        const uint32_t o = off_kmajor(r, 8 * j, LBO_K, K1 * 16);
        *reinterpret_cast<uint4*>(Ah + o) = hh.u;
        *reinterpret_cast<uint4*>(Al + o) = ll.u;
      }
    }
    if (!(good = run_stage(0))) break;
    // ── F1 epilogue: twiddle w1024^(n2 k1), 2^-5 -> F2 operand (MN-major) ──
#pragma unroll 1
    for (int j = h * (4 / WPR); j < (h + 1) * (4 / WPR); j++) {
      float v[16];
      acc_ld16(tl, 128 * c + 16 * j, v);
      H8 hr, lr, hi, li;
#pragma unroll
      for (int t = 0; t < 8; t += 2) {
        float re[2], im[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const float2 w = s_tw[8 * j + t + u][lane];   // w1024^(n2 k1), n2 = lane
          const float yr = v[2 * (t + u)], yi = v[2 * (t + u) + 1];
          re[u] = (yr * w.x - yi * w.y) * 0.03125f;
          im[u] = (yr * w.y + yi * w.x) * 0.03125f;
        }
        split_h2(re[0], re[1], hr.h2[t / 2], lr.h2[t / 2]);
        split_h2(im[0], im[1], hi.h2[t / 2], li.h2[t / 2]);
      }
      const int m0 = 32 * q + 8 * j;
      const uint32_t ore = off_mnmajor(m0, 2 * lane, LBO_MN, SBO_MN), oim = off_mnmajor(m0, 2 * lane + 1, LBO_MN, SBO_MN);
      *reinterpret_cast<uint4*>(Ah + ore) = hr.u;
      *reinterpret_cast<uint4*>(Al + ore) = lr.u;
      *reinterpret_cast<uint4*>(Ah + oim) = hi.u;
      *reinterpret_cast<uint4*>(Al + oim) = li.u;
    }
    if (!(good = run_stage(1))) break;
    // ── F2 epilogue: tensor multiply, conj, 2^(e_t-6) -> G2 operand (K-major) ──
    {
      // (the z team reads only its own exponent: the x/y ones may already be the next group's)
      const int ex = (c < 2) ? s_e[0][q] : 0, ey = (c < 2) ? s_e[1][q] : 0;
      const int em = (c == 2) ? s_e[2][q] : max(ex, ey);
      const float fx = ldexpf(1.f, ex - em), fy = ldexpf(1.f, ey - em);
      const long long tb = (long long)(colok ? kx : 0) * P + lane;
      const int r = 32 * q + lane;
      const float* tdiag = (c == 0) ? a.txx : ((c == 1) ? a.tyy : a.tzz);
      // tensor entries of frequency block j (8 frequencies), loaded one block
      // ahead so their latency overlaps the previous block's arithmetic
      float tn[8];
      float2 tq[8];
      auto load_t = [&](int j, float(&n)[8], float2(&x)[8]) {
#pragma unroll
        for (int i = 0; i < 8; i++) {
          const long long e = tb + 32LL * (8 * j + i);
          n[i] = colok ? __ldg(&tdiag[e]) : 0.f;
          x[i] = (colok && c < 2) ? __ldg(&a.txy[e]) : make_float2(0.f, 0.f);
        }
      };
      // (with two warps per role the other warps hide the tensor loads, and the
      // next block's entries would not fit in the register budget)
      constexpr bool AHEAD = WPR == 1;
      const int j0 = h * (4 / WPR), j1 = j0 + 4 / WPR;
      if constexpr (AHEAD) load_t(j0, tn, tq);
#pragma unroll 1
      for (int j = j0; j < j1; j++) {
        float nn[8];
        float2 nq[8];
        if constexpr (AHEAD) {
          if (j + 1 < j1) load_t(j + 1, nn, nq);
        } else {
          load_t(j, tn, tq);
        }
        // the accumulator block: all 16 columns at once, or (two warps per
        // role, tighter register budget) 8 columns per half
        constexpr int XW = (WPR == 1) ? 16 : 8;
        float X0[XW], X1[XW];
        auto ld_x = [&](int col0) {
          if constexpr (XW == 16) {
            if (c < 2) {
              acc_ld16(tl, col0, X0);
              acc_ld16(tl, 128 + col0, X1);
            } else {
              acc_ld16(tl, 256 + col0, X0);
            }
          } else {
            if (c < 2) {
              acc_ld8(tl, col0, X0);
              acc_ld8(tl, 128 + col0, X1);
            } else {
              acc_ld8(tl, 256 + col0, X0);
            }
          }
        };
        if constexpr (XW == 16) ld_x(16 * j);
#pragma unroll
        for (int half = 0; half < 2; half++) {
          if constexpr (XW == 8) ld_x(16 * j + 8 * half);
          H8 hh, ll;
#pragma unroll
          for (int t = 0; t < 4; t++) {
            const int i = 4 * half + t;
            const int xi2 = (XW == 16) ? 2 * i : 2 * t;   // this frequency's (re, im) in X
            float hr = 0.f, hm = 0.f;
            if (colok) {
              const float n = tn[i];
              const float2 nxy = tq[i];
              if (c == 0) {
                const float xr = X0[xi2] * fx, xi = X0[xi2 + 1] * fx;
                const float yr = X1[xi2] * fy, yi = X1[xi2 + 1] * fy;
                hr = n * xr + (nxy.x * yr - nxy.y * yi);
                hm = n * xi + (nxy.x * yi + nxy.y * yr);
              } else if (c == 1) {
                const float xr = X0[xi2] * fx, xi = X0[xi2 + 1] * fx;
                const float yr = X1[xi2] * fy, yi = X1[xi2 + 1] * fy;
                hr = (nxy.x * xr - nxy.y * xi) + n * yr;
                hm = (nxy.x * xi + nxy.y * xr) + n * yi;
              } else {
                hr = n * X0[xi2];
                hm = n * X0[xi2 + 1];
              }
            }
            split_h2(hr * a.s_t, -hm * a.s_t, hh.h2[t], ll.h2[t]);
          }
          const uint32_t o = off_kmajor(r, 8 * (2 * j + half), LBO_K, 1024);
          *reinterpret_cast<uint4*>(Ah + o) = hh.u;
          *reinterpret_cast<uint4*>(Al + o) = ll.u;
        }
        if (AHEAD && j + 1 < j1) {
#pragma unroll
          for (int i = 0; i < 8; i++) {
            tn[i] = nn[i];
            tq[i] = nq[i];
          }
        }
      }
      if (lane == 0 && h == 0) s_eo[c][q] = em;
    }
    if (!(good = run_stage(2))) break;
    // ── G2 epilogue: twiddle w1024^(n2 k1), 2^-5 -> G1 operand (MN-major) ──
#pragma unroll 1
    for (int j = h * (4 / WPR); j < (h + 1) * (4 / WPR); j++) {
      float v[16];
      acc_ld16(tl, 128 * c + 16 * j, v);
      H8 hr, lr, hi, li;
#pragma unroll
      for (int t = 0; t < 8; t += 2) {
        float re[2], im[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
          const float2 w = s_tw[8 * j + t + u][lane];   // w1024^(n2 k1), k1 = lane
          const float zr = v[2 * (t + u)], zi = v[2 * (t + u) + 1];
          re[u] = (zr * w.x - zi * w.y) * 0.03125f;
          im[u] = (zr * w.y + zi * w.x) * 0.03125f;
        }
        split_h2(re[0], re[1], hr.h2[t / 2], lr.h2[t / 2]);
        split_h2(im[0], im[1], hi.h2[t / 2], li.h2[t / 2]);
      }
      const int m0 = 32 * q + 8 * j;
      const uint32_t ore = off_mnmajor(m0, 2 * lane, LBO_MN, SBO_MN), oim = off_mnmajor(m0, 2 * lane + 1, LBO_MN, SBO_MN);
      *reinterpret_cast<uint4*>(Ah + ore) = hr.u;
      *reinterpret_cast<uint4*>(Al + ore) = lr.u;
      *reinterpret_cast<uint4*>(Ah + oim) = hi.u;
      *reinterpret_cast<uint4*>(Al + oim) = li.u;
    }
    if (!(good = run_stage(3))) break;
    // ── G1 epilogue: conj, undo the scalings, store FP32 column ──
    {
      const float so = ldexpf(1.f, s_eo[c][q] + 16 - a.e_t);
      float2* dst = a.S + ((long long)c * a.hx + (colok ? kx : 0)) * a.ld;
#pragma unroll 1
      for (int j = h * (D1 / 8 / WPR); j < (h + 1) * (D1 / 8 / WPR); j++) {
        float v[16];
        acc_ld16(tl, 128 * c + 16 * j, v);
        if (colok) {
#pragma unroll
          for (int t = 0; t < 8; t++) dst[32 * (8 * j + t) + lane] = make_float2(v[2 * t] * so, -v[2 * t + 1] * so);
        }
      }
    }
  }
  if (!good) {
    if (tid == team_lead) atomicExch(a.err, 1);
    // let the team's MMAs still in flight finish (bounded) before tensor memory is freed
    mbar_wait(&mbar[team], phase, WAIT_LIMIT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, TMEM_COLS);
  }
}

// max |x| over the four FP32 tensor spectra (positive floats order as their bits)
__global__ void k_absmax4(const float* __restrict__ a, const float* __restrict__ b, const float* __restrict__ c,
                          const float2* __restrict__ d, long long n, unsigned int* out) {
  pdl_entry();
  float m = 0.f;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    m = fmaxf(m, fmaxf(fmaxf(fabsf(a[e]), fabsf(b[e])), fmaxf(fabsf(c[e]), fmaxf(fabsf(d[e].x), fabsf(d[e].y)))));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// ── self-test GEMM: D (128 x 64) = A (128 x 64) * B (64 x 64)^T, FP16 in, FP32 out ──
__global__ void __launch_bounds__(128, 1) k_tc_selftest(const uint4* __restrict__ ops, int abytes, int bbytes,
                                                        int a_mn, float* __restrict__ D, int* err) {
  pdl_entry();
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < (abytes + bbytes) / 16; i += blockDim.x) reinterpret_cast<uint4*>(sm)[i] = ops[i];
  if (warp == 0) tmem_alloc(&tmem_slot, 64);
  if (tid == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tmem_slot;
  const uint32_t sA = smem_u32(sm), sB = sA + abytes;
  if (tid == 0) {
    for (int s = 0; s < 4; s++) {
      const uint64_t ad = a_mn ? smem_desc(sA + s * 2 * LBO_MN, LBO_MN, SBO_MN) : smem_desc(sA + s * 256, LBO_K, 1024);
      tc_mma_f16(tbase, ad, smem_desc(sB + s * 256, LBO_K, 1024), idesc_f16_f32(128, 64, a_mn, 0), s > 0);
    }
    tc_commit(&mbar);
  }
  const bool ok = mbar_wait(&mbar, 0, WAIT_LIMIT);
  if (!ok && tid == 0) atomicExch(err, 1);
  tc_fence_after();
  if (ok) {
    for (int j = 0; j < 4; j++) {
      float v[16];
      tmem_ld16(tbase + ((uint32_t)(32 * warp) << 16) + 16 * j, v);
      for (int t = 0; t < 16; t++) D[(32 * warp + (tid & 31)) * 64 + 16 * j + t] = v[t];
    }
  } else {
    mbar_wait(&mbar, 0, WAIT_LIMIT);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, 64);
  }
}

}  // namespace

struct DemagTc {
  int D1 = 0, hx = 0, ny = 0, ngroups = 0, grid = 0;
  size_t smem = 0;
  int e_t = 0;
  float s_t = 0.f;
  uint4* d_bmat = nullptr;
  float2* d_tw = nullptr;
  int* d_err = nullptr;
  const float *txx = nullptr, *tyy = nullptr, *tzz = nullptr;
  const float2* txy = nullptr;
};

// real-ified complex W[o][i] = exp(-2 pi i o i / 32) (no x ni), K-major FP16
// hi/lo at byte offsets oh/ol:  B[2o+po][2i+pi] = [[Re, -Im], [Im, Re]]
static void put_dft(std::vector<unsigned char>& buf, int oh, int ol, int no, int ni, int sbo) {
  for (int o = 0; o < no; o++)
    for (int i = 0; i < ni; i++) {
      const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)((o * i) % 32) / 32.0L;
      const float wr = (float)cosl(ang), wi = (float)sinl(ang);
      const float ent[2][2] = {{wr, -wi}, {wi, wr}};
      for (int po = 0; po < 2; po++)
        for (int pi = 0; pi < 2; pi++) {
          const float v = ent[po][pi];
          const __half h = __float2half_rn(v);
          const __half l = __float2half_rn((v - __half2float(h)) * 2048.f);   // scaled remainder
          const uint32_t off = off_kmajor(2 * o + po, 2 * i + pi, LBO_K, sbo);
          memcpy(&buf[oh + off], &h, 2);
          memcpy(&buf[ol + off], &l, 2);
        }
    }
}

int demag_tc_create(llg_ctx* c, int px, int py, int hx, int ny, const float* txx, const float* tyy, const float* tzz,
                    const float2* txy, DemagTc** out) {
  (void)px;
  *out = nullptr;
  if (py != P || !(ny == 512 || ny == 1024)) return 0;   // other shapes: FP32 Stockham columns
  DemagTc* t = new DemagTc();
  t->D1 = ny / 32;
  t->hx = hx;
  t->ny = ny;
  t->ngroups = (hx + NCOL - 1) / NCOL;
  t->grid = std::min(t->ngroups, c->num_sms);
  t->txx = txx; t->tyy = tyy; t->tzz = tzz; t->txy = txy;
  const int D1 = t->D1, K1 = 2 * D1, BB = bbytes_for(D1);
  t->smem = (size_t)BB + 3 * (size_t)ACOMP;
  // B operands: F1 (64 x K1), F2 (64 x 64), G1 (2 D1 x 64), hi then lo each
  std::vector<unsigned char> b(BB, 0);
  const int oF1h = 0, oF1l = 128 * K1, oF2h = 256 * K1, oF2l = oF2h + 8192, oG1h = oF2h + 16384, oG1l = oG1h + 256 * D1;
  put_dft(b, oF1h, oF1l, 32, D1, K1 * 16);   // W[k1][n1], n1 < D1
  put_dft(b, oF2h, oF2l, 32, 32, 1024);      // W[k2][n2]
  put_dft(b, oG1h, oG1l, D1, 32, 1024);      // W[n1][k1], n1 < D1
  std::vector<float2> tw(P);
  for (int j = 0; j < P; j++) {
    const long double ang = -2.0L * 3.14159265358979323846264338327950288L * (long double)j / (long double)P;
    tw[j] = make_float2((float)cosl(ang), (float)sinl(ang));
  }
  auto fail = [&](int rc) { demag_tc_destroy(t); return rc; };
  // the timeout flag (and, during this set-up, the tensor scan's maximum) lives
  // in the context's scalar slots, so the integrator's read-backs carry it home
  t->d_err = reinterpret_cast<int*>(c->d_scal + SLOT_TCERR);
  if (cudaMalloc(&t->d_bmat, BB) != cudaSuccess || cudaMalloc(&t->d_tw, sizeof(float2) * P) != cudaSuccess) {
    llg_set_error("demag_tc_create: device allocation failed");
    return fail(LLG_ERR_NOMEM);
  }
  if (cudaMemcpy(t->d_bmat, b.data(), BB, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(t->d_tw, tw.data(), sizeof(float2) * P, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(t->d_err, 0, sizeof(int) * 2) != cudaSuccess) {
    llg_set_error("demag_tc_create: upload failed");
    return fail(LLG_ERR_CUDA);
  }
  // global tensor scale 2^e_t with max|N| 2^e_t < 1
  unsigned int* d_mx = reinterpret_cast<unsigned int*>(t->d_err + 1);
  klaunch(k_absmax4, c->num_sms * 4, 256, 0, c->stream, txx, tyy, tzz, txy, (long long)hx * P, d_mx);
  unsigned int mxb = 0;
  if (cudaMemcpyAsync(&mxb, d_mx, sizeof(unsigned int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess ||
      cudaStreamSynchronize(c->stream) != cudaSuccess) {
    llg_set_error("demag_tc_create: tensor scan failed");
    return fail(LLG_ERR_CUDA);
  }
  float mx;
  memcpy(&mx, &mxb, sizeof mx);
  int e = 0;
  if (mx > 0.f) frexpf(mx, &e);
  t->e_t = -e;
  t->s_t = ldexpf(1.f, t->e_t - 6);
  const void* fn = (D1 == 16) ? (const void*)k_cols_tc<16, kTcWpr> : (const void*)k_cols_tc<32, kTcWpr>;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)t->smem) != cudaSuccess) {
    llg_set_error("demag_tc_create: shared-memory opt-in failed");
    return fail(LLG_ERR_CUDA);
  }
  *out = t;
  return 0;
}

void demag_tc_destroy(DemagTc* t) {
  if (!t) return;
  cudaFree(t->d_bmat);
  cudaFree(t->d_tw);
  delete t;
}

int demag_tc_cols(llg_ctx* c, DemagTc* t, float2* Sf) {
  TcArgs a{};
  a.S = Sf;
  a.hx = t->hx;
  a.ld = t->ny;
  a.ngroups = t->ngroups;
  a.txx = t->txx; a.tyy = t->tyy; a.tzz = t->tzz; a.txy = t->txy;
  a.tw = t->d_tw;
  a.bmat = t->d_bmat;
  a.s_t = t->s_t;
  a.e_t = t->e_t;
  a.err = t->d_err;
  if (t->D1 == 16) klaunch(k_cols_tc<16, kTcWpr>, t->grid, NT * kTcWpr, t->smem, c->stream, a);
  else klaunch(k_cols_tc<32, kTcWpr>, t->grid, NT * kTcWpr, t->smem, c->stream, a);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

// 1 if a tensor-core wait ran out since the plan was made (reads back a flag)
int demag_tc_failed(llg_ctx* c, DemagTc* t) {
  int f = 0;
  if (!t) return 0;
  cudaMemcpyAsync(&f, t->d_err, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
  cudaStreamSynchronize(c->stream);
  return f;
}

extern "C" int llg_selftest_tcgen05(int flags, double* max_rel_err) {
  if (!max_rel_err || flags < 0 || flags > 3) return LLG_ERR_ARG;
  *max_rel_err = -1.0;
  const int a_mn_major = flags & 1;
  const float a_scale = (flags & 2) ? ldexpf(1.f, -20) : 1.f;   // bit 1: FP16-subnormal A values
  // random FP16 operands (exact), host double reference
  const int M = 128, N = 64, K = 64;
  const int abytes = a_mn_major ? AMAT : M * K * 2, bbytes = N * K * 2;
  std::vector<unsigned char> buf(abytes + bbytes, 0);
  std::vector<float> A(M * K), B(N * K);
  uint32_t s = 12345u;
  auto rnd = [&]() { s = s * 1664525u + 1013904223u; return ((s >> 8) & 0xFFFF) / 32768.0f - 1.0f; };
  for (int i = 0; i < M * K; i++) A[i] = __half2float(__float2half_rn(rnd() * a_scale));
  for (int i = 0; i < N * K; i++) B[i] = __half2float(__float2half_rn(rnd()));
  for (int m = 0; m < M; m++)
    for (int k = 0; k < K; k++) {
      const __half h = __float2half_rn(A[m * K + k]);
      const uint32_t off = a_mn_major ? off_mnmajor(m, k, LBO_MN, SBO_MN) : off_kmajor(m, k, LBO_K, 1024);
      memcpy(&buf[off], &h, 2);
    }
  for (int n = 0; n < N; n++)
    for (int k = 0; k < K; k++) {
      const __half h = __float2half_rn(B[n * K + k]);
      memcpy(&buf[abytes + off_kmajor(n, k, LBO_K, 1024)], &h, 2);
    }
  uint4* d_ops = nullptr;
  float* d_D = nullptr;
  int* d_err = nullptr;
  LLG_CUDA_TRY(cudaMalloc(&d_ops, buf.size()));
  LLG_CUDA_TRY(cudaMalloc(&d_D, sizeof(float) * M * N));
  LLG_CUDA_TRY(cudaMalloc(&d_err, sizeof(int)));
  LLG_CUDA_TRY(cudaMemcpy(d_ops, buf.data(), buf.size(), cudaMemcpyHostToDevice));
  LLG_CUDA_TRY(cudaMemset(d_err, 0, sizeof(int)));
  LLG_CUDA_TRY(cudaMemset(d_D, 0, sizeof(float) * M * N));
  const size_t smem = buf.size();
  LLG_CUDA_TRY(cudaFuncSetAttribute((const void*)k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_tc_selftest<<<1, 128, smem>>>(d_ops, abytes, bbytes, a_mn_major, d_D, d_err);
  LLG_CUDA_TRY(cudaGetLastError());
  LLG_CUDA_TRY(cudaDeviceSynchronize());
  std::vector<float> D(M * N);
  int err = 0;
  LLG_CUDA_TRY(cudaMemcpy(D.data(), d_D, sizeof(float) * M * N, cudaMemcpyDeviceToHost));
  LLG_CUDA_TRY(cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
  cudaFree(d_ops);
  cudaFree(d_D);
  cudaFree(d_err);
  if (err) { llg_set_error("tcgen05 self-test: MMA completion wait ran out"); return LLG_ERR_TIMEOUT; }
  double worst = 0.0;
  for (int m = 0; m < M; m++)
    for (int n = 0; n < N; n++) {
      double ref = 0.0, mag = 0.0;
      for (int k = 0; k < K; k++) {
        ref += (double)A[m * K + k] * B[n * K + k];
        mag += fabs((double)A[m * K + k] * B[n * K + k]);
      }
      worst = std::max(worst, fabs((double)D[m * N + n] - ref) / std::max(mag, 1e-30));
    }
  *max_rel_err = worst;
  return 0;
}
