// k_geometry.cu — geometry builders on the device (llg_build_geometry_device).
//
// The reference builds every mask on the host, and its polycrystal builder is
// the slow part of a run's set-up: nearest_grain scans every grain and its 8
// periodic images for every cell (src/irregular/2d_fft/2d_i3/2d_fft.cu:300-315,
// O(N·G·9)) and the tanh window measures every cell's distance to every hole
// cell (:346-371, O(N·N_hole)).  Here:
//   * grain sites and axes come from the host (the reference's rand() order,
//     O(G), geometry.cpp), then one thread per cell finds the nearest grain
//     with the host's arithmetic (no FMA contraction: rounded products and
//     sums, so ties break as on the host and grain ids are identical);
//   * the distance of every cell to the nearest dead-grain cell is an exact
//     separable transform on the periodic grid: a column pass (one thread per
//     column sweeps 3·ny rows: distance to the nearest hole above / below
//     with the minimum-image convention) and a row pass (one block per row,
//     the row staged in shared memory, each cell the minimum over the row of
//     dx² + g²(x')) — every value is a small integer, so the result equals the
//     brute-force minimum bit for bit;
//   * the window, active flags and per-cell axes follow per cell.
// The other geometries are per-cell predicates with the host's arithmetic.
// Initial states are not built here: they follow the C library's rand()
// sequence on the host (llg_build_geometry).
#include <math.h>

#include <vector>

#include "llg_internal.h"

int geom_grains(const llg_geom_spec* g, std::vector<double>& d8, std::vector<int>& dead);

namespace {

constexpr int GT = 256;

__global__ void k_nearest_grain(const double* __restrict__ gr8, int NG, int ng, int ny, int32_t* __restrict__ gid) {
  const int n = ng * ny;
  for (int cell = blockIdx.x * GT + threadIdx.x; cell < n; cell += gridDim.x * GT) {
    const double x = (double)(cell % ng) + 0.5, y = (double)(cell / ng) + 0.5;
    int best = 0;
    double bd = 1.0e30;
    for (int k = 0; k < NG; k++) {
      const double sx = gr8[8 * k], sy = gr8[8 * k + 1];
      for (int dyp = -1; dyp <= 1; dyp++)
        for (int dxp = -1; dxp <= 1; dxp++) {
          const double dx = __dsub_rn(x, __dadd_rn(sx, (double)dxp * (double)ng));
          const double dy = __dsub_rn(y, __dadd_rn(sy, (double)dyp * (double)ny));
          const double d2 = __dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy));
          if (d2 < bd) { bd = d2; best = k; }
        }
    }
    gid[cell] = best;
  }
}

// column pass: g2[y][x] = squared distance (in y, periodic) to the nearest
// hole cell of column x, INF when the column has none
__global__ void k_hole_cols(const int32_t* __restrict__ gid, const int* __restrict__ dead, int ng, int ny,
                            double* __restrict__ g2) {
  const int x = blockIdx.x * GT + threadIdx.x;
  if (x >= ng) return;
  const double INF = __longlong_as_double(0x7ff0000000000000ll);
  const int H = 3 * ny;
  long long last = -1;
  for (int t = 0; t < H; t++) {
    const int row = t % ny;
    if (dead[gid[(long long)row * ng + x]]) last = t;
    if (t >= ny && t < 2 * ny) g2[(long long)(t - ny) * ng + x] = (last < 0) ? INF : (double)(t - last);
  }
  last = -1;
  for (int t = H - 1; t >= 0; t--) {
    const int row = t % ny;
    if (dead[gid[(long long)row * ng + x]]) last = t;
    if (t >= ny && t < 2 * ny) {
      const long long i = (long long)(t - ny) * ng + x;
      const double fw = g2[i];
      const double bw = (last < 0) ? INF : (double)(last - t);
      const double d = fmin(fw, bw);
      g2[i] = (d == INF) ? INF : d * d;
    }
  }
}

// row pass + window + flags + axes: one block per row y
__global__ void k_hole_rows_window(const double* __restrict__ g2, const int32_t* __restrict__ gid,
                                   const int* __restrict__ dead, const double* __restrict__ gr8, int ng, int ny,
                                   double eps, uint8_t* act, double* w, double* msk3, double* nsk3,
                                   unsigned int* nact, int any_hole) {
  extern __shared__ double row[];
  const int y = blockIdx.x;
  for (int x = threadIdx.x; x < ng; x += blockDim.x) row[x] = g2[(long long)y * ng + x];
  __syncthreads();
  const int n = ng * ny;
  unsigned int cnt = 0;
  for (int x = threadIdx.x; x < ng; x += blockDim.x) {
    const long long cell = (long long)y * ng + x;
    const int g = gid[cell];
    double ww = 1.0;
    if (any_hole) {
      if (dead[g]) {
        ww = 0.0;
      } else {
        double best = __longlong_as_double(0x7ff0000000000000ll);
        for (int X = 0; X < ng; X++) {
          const int ad = abs(x - X);
          const double dd = (double)min(ad, ng - ad);
          best = fmin(best, dd * dd + row[X]);   // small integers: exact
        }
        const double d = sqrt(best) - 0.5;
        ww = 0.5 * (1.0 + tanh(d / eps));
        if (ww < 1.0e-3) ww = 0.0;
        if (ww > 1.0 - 1.0e-3) ww = 1.0;
      }
    }
    const uint8_t a = (ww > 1.0e-3) ? 1 : 0;
    cnt += a;
    if (act) act[cell] = a;
    if (w) w[cell] = ww;
    if (msk3) { msk3[cell] = gr8[8 * g + 2]; msk3[n + cell] = gr8[8 * g + 3]; msk3[2 * n + cell] = gr8[8 * g + 4]; }
    if (nsk3) { nsk3[cell] = gr8[8 * g + 5]; nsk3[n + cell] = gr8[8 * g + 6]; nsk3[2 * n + cell] = gr8[8 * g + 7]; }
  }
  atomicAdd(nact, cnt);
}

struct ShapeArgs {
  int kind, ng, ny;
  double hx, hy, hs;                // square hole: centre, half side
  double hwo, hho, hwi, hhi;        // ring
  double irx2, iry2;                // ellipse
  double rin, rout;                 // annulus
  int screen_col, slit_lo, slit_hi; // slit
};

__global__ void k_shape(ShapeArgs s, uint8_t* act, double* w, double* msk3, double* nsk3, unsigned int* nact) {
  const int n = s.ng * s.ny;
  const double cxc = 0.5 * s.ng, cyc = 0.5 * s.ny;
  unsigned int cnt = 0;
  for (int cell = blockIdx.x * GT + threadIdx.x; cell < n; cell += gridDim.x * GT) {
    const int i = cell % s.ng, j = cell / s.ng;
    uint8_t a = 1;
    switch (s.kind) {
      case LLG_GEOM_HOLE_SQUARE:
        a = (fabs((double)i - s.hx) <= s.hs && fabs((double)j - s.hy) <= s.hs) ? 0 : 1;
        break;
      case LLG_GEOM_RING: {
        const double dx = fabs(__dsub_rn(__dadd_rn((double)i, 0.5), cxc));
        const double dy = fabs(__dsub_rn(__dadd_rn((double)j, 0.5), cyc));
        const bool in_o = (dx <= s.hwo && dy <= s.hho), in_i = (dx < s.hwi && dy < s.hhi);
        a = (in_o && !in_i) ? 1 : 0;
        break;
      }
      case LLG_GEOM_ELLIPSE: {
        const double dx = __dsub_rn(__dadd_rn((double)i, 0.5), cxc), dy = __dsub_rn(__dadd_rn((double)j, 0.5), cyc);
        const double q = __dadd_rn(__dmul_rn(__dmul_rn(dx, dx), s.irx2), __dmul_rn(__dmul_rn(dy, dy), s.iry2));
        a = (q <= 1.0) ? 1 : 0;
        break;
      }
      case LLG_GEOM_ANNULUS: {
        const double dx = __dsub_rn(__dadd_rn((double)i, 0.5), cxc), dy = __dsub_rn(__dadd_rn((double)j, 0.5), cyc);
        const double r = __dsqrt_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));
        a = (r >= s.rin && r <= s.rout) ? 1 : 0;
        break;
      }
      case LLG_GEOM_SLIT:
        a = (i == s.screen_col && !(j >= s.slit_lo && j < s.slit_hi)) ? 0 : 1;
        break;
      default:
        break;
    }
    cnt += a;
    if (act) act[cell] = a;
    if (w) w[cell] = a ? 1.0 : 0.0;
    if (msk3) { msk3[cell] = 0.0; msk3[n + cell] = 0.0; msk3[2 * n + cell] = 0.0; }
    if (nsk3) { nsk3[cell] = 0.0; nsk3[n + cell] = 0.0; nsk3[2 * n + cell] = 0.0; }
  }
  atomicAdd(nact, cnt);
}

__global__ void k_fill_i32(int32_t* p, int n, int v) {
  for (int i = blockIdx.x * GT + threadIdx.x; i < n; i += gridDim.x * GT) p[i] = v;
}

int grid_for(long long n) {
  long long b = (n + GT - 1) / GT;
  if (b > 148 * 16) b = 148 * 16;
  return (int)(b < 1 ? 1 : b);
}

struct DevBufs {
  std::vector<void*> p;
  ~DevBufs() {
    for (void* q : p) cudaFree(q);
  }
  template <class T>
  cudaError_t get(T** out, size_t bytes) {
    void* q = nullptr;
    const cudaError_t e = cudaMalloc(&q, bytes);
    if (e == cudaSuccess) p.push_back(q);
    *out = static_cast<T*>(q);
    return e;
  }
};

}  // namespace

extern "C" int llg_build_geometry_device(const llg_geom_spec* g, uint8_t* d_active, double* d_w, double* d_msk3,
                                         double* d_nsk3, int32_t* d_grain_id, void* cuda_stream) {
  if (!g || g->ng <= 0 || g->ny <= 0) { llg_set_error("llg_build_geometry_device: bad spec"); return LLG_ERR_ARG; }
  if ((long long)g->ng * g->ny > (1ll << 31) - 1) { llg_set_error("llg_build_geometry_device: grid too large"); return LLG_ERR_ARG; }
  const int ng = g->ng, ny = g->ny, n = ng * ny;
  cudaStream_t st = (cudaStream_t)cuda_stream;
  DevBufs tmp;
  unsigned int* d_cnt = nullptr;
  LLG_CUDA_TRY(tmp.get(&d_cnt, sizeof(unsigned int)));
  LLG_CUDA_TRY(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned int), st));
  if (g->geometry_kind == LLG_GEOM_POLYCRYSTAL) {
    if (!(g->mask_eps_cells > 0.0)) { llg_set_error("llg_build_geometry_device: mask_eps_cells must be > 0"); return LLG_ERR_ARG; }
    std::vector<double> d8;
    std::vector<int> dead;
    const int rc = geom_grains(g, d8, dead);
    if (rc) { llg_set_error("llg_build_geometry_device: num_grains must be > 0"); return rc; }
    const int NG = (int)dead.size();
    int any = 0;
    for (int v : dead) any |= v;
    double* d_gr = nullptr;
    int* d_dead = nullptr;
    int32_t* gid = d_grain_id;
    double* g2 = nullptr;
    LLG_CUDA_TRY(tmp.get(&d_gr, d8.size() * sizeof(double)));
    LLG_CUDA_TRY(tmp.get(&d_dead, dead.size() * sizeof(int)));
    if (!gid) LLG_CUDA_TRY(tmp.get(&gid, (size_t)n * sizeof(int32_t)));
    LLG_CUDA_TRY(tmp.get(&g2, (size_t)n * sizeof(double)));
    LLG_CUDA_TRY(cudaMemcpyAsync(d_gr, d8.data(), d8.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    LLG_CUDA_TRY(cudaMemcpyAsync(d_dead, dead.data(), dead.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    LLG_COUNT(KID_OTHER);
    k_nearest_grain<<<grid_for(n), GT, 0, st>>>(d_gr, NG, ng, ny, gid);
    LLG_CUDA_TRY(cudaPeekAtLastError());
    if (any) {
      LLG_COUNT(KID_OTHER);
      k_hole_cols<<<(ng + GT - 1) / GT, GT, 0, st>>>(gid, d_dead, ng, ny, g2);
      LLG_CUDA_TRY(cudaPeekAtLastError());
    }
    const size_t smem = (size_t)ng * sizeof(double);
    if (smem > 227 * 1024) { llg_set_error("llg_build_geometry_device: rows longer than 29056 cells"); return LLG_ERR_NOTSUP; }
    if (smem > 48 * 1024)
      LLG_CUDA_TRY(cudaFuncSetAttribute(k_hole_rows_window, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LLG_COUNT(KID_OTHER);
    k_hole_rows_window<<<ny, GT, smem, st>>>(g2, gid, d_dead, d_gr, ng, ny, g->mask_eps_cells, d_active, d_w,
                                             d_msk3, d_nsk3, d_cnt, any);
    LLG_CUDA_TRY(cudaPeekAtLastError());
  } else {
    ShapeArgs s{};
    s.kind = g->geometry_kind;
    s.ng = ng;
    s.ny = ny;
    switch (g->geometry_kind) {
      case LLG_GEOM_BULK:
      case LLG_GEOM_CUSTOM:
        s.kind = LLG_GEOM_BULK;
        break;
      case LLG_GEOM_HOLE_SQUARE:
        s.hx = g->hole_center_x_frac * (double)(ng - 1);
        s.hy = g->hole_center_y_frac * (double)(ny - 1);
        s.hs = g->hole_radius_frac_y * (double)ny;
        break;
      case LLG_GEOM_RING:
        s.hwo = 0.5 * g->outer_w_frac * ng;
        s.hho = 0.5 * g->outer_h_frac * ny;
        s.hwi = s.hwo * g->inner_w_frac_of_outer;
        s.hhi = s.hho * g->inner_h_frac_of_outer;
        break;
      case LLG_GEOM_ELLIPSE: {
        const double rx = g->active_rx_frac * ng, ry = g->active_ry_frac * ny;
        if (!(rx > 0.0) || !(ry > 0.0)) { llg_set_error("llg_build_geometry_device: bad ellipse"); return LLG_ERR_ARG; }
        s.irx2 = 1.0 / (rx * rx);
        s.iry2 = 1.0 / (ry * ry);
        break;
      }
      case LLG_GEOM_ANNULUS: {
        const double nmin = (double)(ng < ny ? ng : ny);
        s.rin = g->annulus_r_in_frac * nmin;
        s.rout = g->annulus_r_out_frac * nmin;
        break;
      }
      case LLG_GEOM_SLIT: {
        s.screen_col = (int)(g->screen_x_frac * (double)ng + 0.5);
        const int slit_w = (int)(g->slit_w_frac * (double)ny + 0.5);
        s.slit_lo = ny / 2 - slit_w / 2;
        s.slit_hi = s.slit_lo + slit_w;
        break;
      }
      default:
        llg_set_error("llg_build_geometry_device: unknown geometry kind");
        return LLG_ERR_ARG;
    }
    LLG_COUNT(KID_OTHER);
    k_shape<<<grid_for(n), GT, 0, st>>>(s, d_active, d_w, d_msk3, d_nsk3, d_cnt);
    LLG_CUDA_TRY(cudaPeekAtLastError());
    if (d_grain_id) {
      LLG_COUNT(KID_OTHER);
      k_fill_i32<<<grid_for(n), GT, 0, st>>>(d_grain_id, n, 0);
      LLG_CUDA_TRY(cudaPeekAtLastError());
    }
  }
  unsigned int nact = 0;
  LLG_CUDA_TRY(cudaMemcpyAsync(&nact, d_cnt, sizeof(nact), cudaMemcpyDeviceToHost, st));
  LLG_CUDA_TRY(cudaStreamSynchronize(st));
  return (int)nact;
}
