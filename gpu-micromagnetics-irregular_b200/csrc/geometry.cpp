// geometry.cpp — host-side geometry / initial-condition builders and the
// KEY=VALUE knob parser of libllg.so.
//
// Builders (same predicates and C-library rand() call order as the
// reference, so a seed gives the same mask and state):
//   square hole     src/irregular/2d_fft/2d_i2/2d_fft.cu:544-566
//   ring / rect     src/irregular/2d_fft/2d_i5/2d_fft.cu:512-545 + configs/sim_config.h
//                   GEOMETRY_RING (outer rect minus inner rect; i5 = no inner rect)
//   ellipse         src/irregular/2d_fft/2d_i6/2d_i6.cu:462-533
//   polycrystal     src/irregular/2d_fft/2d_i3/2d_fft.cu:255-387
//   annulus         circular ring r_in <= r <= r_out (no reference twin)
//   IC uniform      2d_i2/2d_fft.cu:610-639;  stripes 2d_i1/2d_fft.cu:540-541, 625-657
//   IC two-domain   2d_i4/2d_fft.cu:562-595;  grain bumps 2d_i3/2d_fft.cu:916-984
// The polycrystal tanh window is O(N x N_hole) in the reference; here it is a
// two-pass exact Euclidean distance transform on the periodic grid, O(N).
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <functional>
#include <limits>
#include <map>
#include <string>
#include <vector>

#include "../../include/llg.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

struct Grain {
  double sx, sy, ax, ay, az, nx, ny, nz;
  int dead;
};

double runit() { return (double)rand() / (double)RAND_MAX; }

std::vector<Grain> make_grains(const llg_geom_spec& g) {
  const int ng = g.ng, ny = g.ny, NG = g.num_grains;
  std::vector<Grain> gr(NG);
  srand((unsigned)g.hole_seed);
  int gx = (int)ceil(sqrt((double)NG * (double)ng / (double)ny));
  if (gx < 1) gx = 1;
  const int gy = (NG + gx - 1) / gx;
  const double dxs = (double)ng / gx, dys = (double)ny / gy;
  int idx = 0;
  for (int j = 0; j < gy && idx < NG; j++)
    for (int i = 0; i < gx && idx < NG; i++, idx++) {
      double sx = ((double)i + 0.15 + 0.7 * runit()) * dxs;
      double sy = ((double)j + 0.15 + 0.7 * runit()) * dys;
      while (sx < 0.0) sx += ng;
      while (sx >= (double)ng) sx -= ng;
      while (sy < 0.0) sy += ny;
      while (sy >= (double)ny) sy -= ny;
      gr[idx].sx = sx;
      gr[idx].sy = sy;
    }
  for (; idx < NG; idx++) {
    gr[idx].sx = runit() * (double)ng;
    gr[idx].sy = runit() * (double)ny;
  }
  for (auto& q : gr) {
    const double u = runit();
    const double sign = (runit() < 0.5) ? -1.0 : 1.0;
    const double z = sign * pow(u, 1.0 / g.grain_z_bias);
    const double phi = 2.0 * kPi * runit();
    const double rxy = sqrt(std::max(0.0, 1.0 - z * z));
    q.ax = rxy * cos(phi);
    q.ay = rxy * sin(phi);
    q.az = z;
    const double psi = 2.0 * kPi * runit();
    q.nx = cos(psi);
    q.ny = sin(psi);
    q.nz = 0.0;
    q.dead = (runit() < g.dead_grain_frac) ? 1 : 0;
  }
  return gr;
}

int nearest_grain(const std::vector<Grain>& gr, double x, double y, int ng, int ny) {
  int best = 0;
  double bd = 1.0e30;
  for (int k = 0; k < (int)gr.size(); k++)
    for (int dyp = -1; dyp <= 1; dyp++)
      for (int dxp = -1; dxp <= 1; dxp++) {
        const double dx = x - (gr[k].sx + dxp * (double)ng);
        const double dy = y - (gr[k].sy + dyp * (double)ny);
        const double d2 = dx * dx + dy * dy;
        if (d2 < bd) { bd = d2; best = k; }
      }
  return best;
}

// Squared distance to the nearest hole cell on the periodic grid using the
// reference's minimum-image convention (|dx| = min(|d|, ng-|d|) per axis).
// Exact separable distance transform (Felzenszwalb–Huttenlocher): a periodic
// 1-D sweep along y, then the lower envelope of parabolas along x over three
// periodic copies.  All intermediate values are small integers, so the result
// equals the brute-force minimum bit for bit.
std::vector<double> hole_dist2(const std::vector<uint8_t>& hole, int ng, int ny) {
  const double INF = std::numeric_limits<double>::infinity();
  std::vector<double> g2((size_t)ng * ny, INF);
  const int H = 3 * ny;
  std::vector<double> dfw(H), dbw(H);
  for (int x = 0; x < ng; x++) {
    long last = -1;
    for (int t = 0; t < H; t++) {
      if (hole[(size_t)(t % ny) * ng + x]) last = t;
      dfw[t] = (last < 0) ? INF : (double)(t - last);
    }
    last = -1;
    for (int t = H - 1; t >= 0; t--) {
      if (hole[(size_t)(t % ny) * ng + x]) last = t;
      dbw[t] = (last < 0) ? INF : (double)(last - t);
    }
    for (int t = ny; t < 2 * ny; t++) {
      const double d = std::min(dfw[t], dbw[t]);
      g2[(size_t)(t - ny) * ng + x] = (d == INF) ? INF : d * d;
    }
  }
  std::vector<double> out((size_t)ng * ny, INF);
  const int W = 3 * ng;
  std::vector<double> f(W), z(W + 1);
  std::vector<int> v(W);
  for (int y = 0; y < ny; y++) {
    for (int X = 0; X < W; X++) f[X] = g2[(size_t)y * ng + (X % ng)];
    int k = -1;
    for (int q = 0; q < W; q++) {
      if (f[q] == INF) continue;
      if (k < 0) { k = 0; v[0] = q; z[0] = -INF; z[1] = INF; continue; }
      double s = ((f[q] + (double)q * q) - (f[v[k]] + (double)v[k] * v[k])) / (2.0 * q - 2.0 * v[k]);
      while (s <= z[k]) {
        k--;
        s = ((f[q] + (double)q * q) - (f[v[k]] + (double)v[k] * v[k])) / (2.0 * q - 2.0 * v[k]);
      }
      k++;
      v[k] = q;
      z[k] = s;
      z[k + 1] = INF;
    }
    if (k < 0) continue;
    int kk = 0;
    for (int X = 0; X < W; X++) {
      while (z[kk + 1] < X) kk++;
      if (X >= ng && X < 2 * ng) {
        const double dd = (double)(X - v[kk]);
        out[(size_t)y * ng + (X - ng)] = dd * dd + f[v[kk]];
      }
    }
  }
  return out;
}

}  // namespace

// Grains of a polycrystal spec in the reference's rand() order (the device
// builder, k_geometry.cu, takes its sites and axes from here): per grain
// sx, sy, ax, ay, az, nx, ny, nz and the dead flag.
int geom_grains(const llg_geom_spec* g, std::vector<double>& d8, std::vector<int>& dead) {
  if (!g || g->num_grains <= 0) return LLG_ERR_ARG;
  const std::vector<Grain> gr = make_grains(*g);
  d8.resize(gr.size() * 8);
  dead.resize(gr.size());
  for (size_t k = 0; k < gr.size(); k++) {
    const double v[8] = {gr[k].sx, gr[k].sy, gr[k].ax, gr[k].ay, gr[k].az, gr[k].nx, gr[k].ny, gr[k].nz};
    for (int q = 0; q < 8; q++) d8[k * 8 + q] = v[q];
    dead[k] = gr[k].dead;
  }
  return 0;
}

extern "C" int llg_default_geom_spec(llg_geom_spec* g) {
  if (!g) return LLG_ERR_ARG;
  memset(g, 0, sizeof(*g));
  g->ng = 128; g->ny = 64;
  g->geometry_kind = LLG_GEOM_BULK;
  g->ic_kind = LLG_IC_UNIFORM;
  g->hole_center_x_frac = 0.5; g->hole_center_y_frac = 0.5; g->hole_radius_frac_y = 0.22;
  g->outer_w_frac = 0.5; g->outer_h_frac = 0.5; g->inner_w_frac_of_outer = 0.5; g->inner_h_frac_of_outer = 0.5;
  g->active_rx_frac = 0.25; g->active_ry_frac = 0.25;
  g->annulus_r_in_frac = 0.15; g->annulus_r_out_frac = 0.35;
  g->num_grains = 72; g->hole_seed = 20251104; g->dead_grain_frac = 0.16; g->mask_eps_cells = 2.2;
  g->grain_z_bias = 1.6;
  g->init_m[0] = 1.0; g->init_m[1] = 0.0; g->init_m[2] = 0.0;
  g->init_random_seed = 12345; g->init_random_eps = 0.01;
  g->stripe_left_frac = 0.25; g->stripe_right_frac = 0.75;
  g->two_domain_split_frac = 0.875; g->two_domain_tail_my = -0.0175;
  g->ic_core_mz = 0.95; g->ic_jitter_eps = 0.0;
  // src/2d_fft/2d_fft.cu:94-120 and src/slit/2d_slit.cu:80-90 defaults
  g->texture_core_mz = -0.998; g->texture_outer_mz = 0.998; g->texture_width_frac = 0.35; g->texture_eps = 1.0e-12;
  g->circle_cx_frac = 0.5; g->circle_cy_frac = 0.5; g->circle_r_frac_y = 0.22;
  g->screen_x_frac = 0.5; g->slit_w_frac = 0.10;
  return 0;
}

extern "C" int llg_build_geometry(const llg_geom_spec* g, uint8_t* active_out, double* w_out, double* msk3,
                                  double* nsk3, int32_t* gid_out, double* y0) {
  if (!g || g->ng <= 0 || g->ny <= 0) return LLG_ERR_ARG;
  const int ng = g->ng, ny = g->ny;
  const size_t n = (size_t)ng * ny;
  std::vector<uint8_t> act(n, 1);
  std::vector<double> w(n, 1.0);
  std::vector<int32_t> gid(n, 0);
  std::vector<Grain> gr;
  const double cxc = 0.5 * ng, cyc = 0.5 * ny;
  switch (g->geometry_kind) {
    case LLG_GEOM_BULK:
    case LLG_GEOM_CUSTOM:
      break;
    case LLG_GEOM_HOLE_SQUARE: {
      const double cx = g->hole_center_x_frac * (double)(ng - 1);
      const double cy = g->hole_center_y_frac * (double)(ny - 1);
      const double hs = g->hole_radius_frac_y * (double)ny;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++)
          act[(size_t)j * ng + i] = (fabs((double)i - cx) <= hs && fabs((double)j - cy) <= hs) ? 0 : 1;
      break;
    }
    case LLG_GEOM_RING: {
      const double hwo = 0.5 * g->outer_w_frac * ng, hho = 0.5 * g->outer_h_frac * ny;
      const double hwi = hwo * g->inner_w_frac_of_outer, hhi = hho * g->inner_h_frac_of_outer;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++) {
          const double dx = fabs((double)i + 0.5 - cxc), dy = fabs((double)j + 0.5 - cyc);
          const bool in_o = (dx <= hwo && dy <= hho), in_i = (dx < hwi && dy < hhi);
          act[(size_t)j * ng + i] = (in_o && !in_i) ? 1 : 0;
        }
      break;
    }
    case LLG_GEOM_ELLIPSE: {
      const double rx = g->active_rx_frac * ng, ry = g->active_ry_frac * ny;
      if (!(rx > 0.0) || !(ry > 0.0)) return LLG_ERR_ARG;
      const double irx2 = 1.0 / (rx * rx), iry2 = 1.0 / (ry * ry);
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++) {
          const double dx = (double)i + 0.5 - cxc, dy = (double)j + 0.5 - cyc;
          act[(size_t)j * ng + i] = (dx * dx * irx2 + dy * dy * iry2 <= 1.0) ? 1 : 0;
        }
      break;
    }
    case LLG_GEOM_ANNULUS: {
      const double nmin = (double)std::min(ng, ny);
      const double rin = g->annulus_r_in_frac * nmin, rout = g->annulus_r_out_frac * nmin;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++) {
          const double dx = (double)i + 0.5 - cxc, dy = (double)j + 0.5 - cyc;
          const double r = sqrt(dx * dx + dy * dy);
          act[(size_t)j * ng + i] = (r >= rin && r <= rout) ? 1 : 0;
        }
      break;
    }
    case LLG_GEOM_POLYCRYSTAL: {
      if (g->num_grains <= 0 || !(g->mask_eps_cells > 0.0)) return LLG_ERR_ARG;
      gr = make_grains(*g);
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++) gid[(size_t)j * ng + i] = nearest_grain(gr, i + 0.5, j + 0.5, ng, ny);
      std::vector<uint8_t> hole(n, 0);
      size_t nh = 0;
      for (size_t k = 0; k < n; k++) { hole[k] = (uint8_t)gr[gid[k]].dead; nh += hole[k]; }
      if (nh > 0) {
        const auto d2 = hole_dist2(hole, ng, ny);
        for (size_t k = 0; k < n; k++) {
          if (hole[k]) { w[k] = 0.0; continue; }
          const double d = sqrt(d2[k]) - 0.5;
          double ww = 0.5 * (1.0 + tanh(d / g->mask_eps_cells));
          if (ww < 1.0e-3) ww = 0.0;
          if (ww > 1.0 - 1.0e-3) ww = 1.0;
          w[k] = ww;
        }
      }
      for (size_t k = 0; k < n; k++) act[k] = (w[k] > 1.0e-3) ? 1 : 0;
      if (msk3)
        for (size_t k = 0; k < n; k++) { msk3[k] = gr[gid[k]].ax; msk3[n + k] = gr[gid[k]].ay; msk3[2 * n + k] = gr[gid[k]].az; }
      if (nsk3)
        for (size_t k = 0; k < n; k++) { nsk3[k] = gr[gid[k]].nx; nsk3[n + k] = gr[gid[k]].ny; nsk3[2 * n + k] = gr[gid[k]].nz; }
      break;
    }
    case LLG_GEOM_SLIT: {   // src/slit/2d_slit.cu:482-486, 541-560
      const int screen_col = (int)(g->screen_x_frac * (double)ng + 0.5);
      const int slit_w = (int)(g->slit_w_frac * (double)ny + 0.5);
      const int lo = ny / 2 - slit_w / 2, hi = lo + slit_w;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++)
          act[(size_t)j * ng + i] = (i == screen_col && !(j >= lo && j < hi)) ? 0 : 1;
      break;
    }
    default:
      return LLG_ERR_ARG;
  }
  if (g->geometry_kind != LLG_GEOM_POLYCRYSTAL) {
    for (size_t k = 0; k < n; k++) w[k] = act[k] ? 1.0 : 0.0;
    if (msk3) std::fill(msk3, msk3 + 3 * n, 0.0);
    if (nsk3) std::fill(nsk3, nsk3 + 3 * n, 0.0);
  }
  long nact = 0;
  for (size_t k = 0; k < n; k++) nact += act[k];

  if (y0) {
    std::fill(y0, y0 + 3 * n, 0.0);
    srand((unsigned)g->init_random_seed);
    auto put = [&](size_t k, double a, double b, double cc) { y0[k] = a; y0[n + k] = b; y0[2 * n + k] = cc; };
    switch (g->ic_kind) {
      case LLG_IC_UNIFORM:
      case LLG_IC_CUSTOM: {
        double m0 = g->init_m[0], m1 = g->init_m[1], m2 = g->init_m[2];
        const double n0 = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
        if (n0 > 1.0e-30) { m0 /= n0; m1 /= n0; m2 /= n0; }
        for (size_t k = 0; k < n; k++)
          if (act[k]) put(k, m0, m1, m2);
        break;
      }
      case LLG_IC_HEAD_ON_STRIPES: {
        const int q1 = (int)(g->stripe_left_frac * (double)ng + 0.5);
        const int q3 = (int)(g->stripe_right_frac * (double)ng + 0.5);
        const double eps = g->init_random_eps;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const size_t k = (size_t)j * ng + i;
            double a = (i >= q1 && i < q3) ? 1.0 : -1.0;
            double b = eps * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
            double cc = eps * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
            const double nn = sqrt(a * a + b * b + cc * cc);
            if (act[k]) put(k, a / nn, b / nn, cc / nn);
          }
        break;
      }
      case LLG_IC_TWO_DOMAIN: {
        const int js = (int)floor(g->two_domain_split_frac * (double)ny);
        const double tail = g->two_domain_tail_my;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const size_t k = (size_t)j * ng + i;
            if (!act[k]) continue;
            double a, b;
            if (j >= js) { a = -1.0; b = 0.0; }
            else { a = 1.0; b = (i < ng / 2) ? -tail : tail; }
            const double nn = sqrt(a * a + b * b);
            put(k, a / nn, b / nn, 0.0);
          }
        break;
      }
      case LLG_IC_TWO_DOMAIN_X:
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const size_t k = (size_t)j * ng + i;
            if (act[k]) put(k, (i < ng / 2) ? 1.0 : -1.0, 0.0, 0.0);
          }
        break;
      case LLG_IC_VORTEX:
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const size_t k = (size_t)j * ng + i;
            if (!act[k]) continue;
            const double x = (double)i + 0.5 - cxc, yv = (double)j + 0.5 - cyc;
            const double a = -yv, b = x, cc = 0.1;
            const double nn = sqrt(a * a + b * b + cc * cc);
            put(k, a / nn, b / nn, cc / nn);
          }
        break;
      case LLG_IC_NEEL: {   // src/2d_fft/2d_fft.cu:460-463, 533-580
        const double cx = g->circle_cx_frac * (double)(ng - 1), cy = g->circle_cy_frac * (double)(ny - 1);
        const double radius = g->circle_r_frac_y * (double)ny;
        const double core = g->texture_core_mz, outer = g->texture_outer_mz;
        double width = g->texture_width_frac * radius;
        if (width < 1.0) width = 1.0;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const size_t k = (size_t)j * ng + i;
            if (!act[k]) continue;
            const double ddx = (double)i - cx, ddy = (double)j - cy;
            const double rho = sqrt(ddx * ddx + ddy * ddy);
            const double u = (rho - radius) / width;
            const double sw = 0.5 * (1.0 - tanh(u));
            double mz0 = outer + (core - outer) * sw;
            if (mz0 > 1.0) mz0 = 1.0;
            if (mz0 < -1.0) mz0 = -1.0;
            const double mperp = sqrt(fmax(0.0, 1.0 - mz0 * mz0));
            double mx0 = 0.0, my0 = 0.0;
            if (rho > g->texture_eps) { mx0 = mperp * (ddx / rho); my0 = mperp * (ddy / rho); }
            put(k, mx0, my0, mz0);
          }
        break;
      }
      case LLG_IC_GRAIN_BUMPS: {
        if (gr.empty()) break;
        const double core = g->ic_core_mz, epsn = 0.05;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const size_t k = (size_t)j * ng + i;
            const Grain& G = gr[gid[k]];
            if (w[k] <= 1.0e-3) continue;
            double ddx = (double)i + 0.5 - G.sx, ddy = (double)j + 0.5 - G.sy;
            if (ddx > ng / 2.0) ddx -= ng;
            if (ddx < -ng / 2.0) ddx += ng;
            if (ddy > ny / 2.0) ddy -= ny;
            if (ddy < -ny / 2.0) ddy += ny;
            const double r = sqrt(ddx * ddx + ddy * ddy);
            const double s = std::min(1.0, r / 14.0);
            double sgz = (G.az >= 0.0) ? 1.0 : -1.0;
            if (fabs(G.az) < 0.05) sgz = 0.0;
            double mz0 = sgz * core * (1.0 - s * s);
            const double mperp = sqrt(std::max(0.0, 1.0 - mz0 * mz0));
            double tx = -ddy, ty = ddx;
            const double tn = sqrt(tx * tx + ty * ty);
            if (tn > 1.0e-12) { tx /= tn; ty /= tn; } else { tx = 1.0; ty = 0.0; }
            const double bn = sqrt(G.ax * G.ax + G.ay * G.ay);
            const double ex = (bn > 1.0e-6) ? G.ax / bn : 1.0, ey = (bn > 1.0e-6) ? G.ay / bn : 0.0;
            double px = (1.0 - s) * tx + s * ex, py = (1.0 - s) * ty + s * ey;
            const double pn = sqrt(px * px + py * py);
            if (pn > 1.0e-12) { px /= pn; py /= pn; }
            double a = mperp * px + epsn * (2.0 * runit() - 1.0);
            double b = mperp * py + epsn * (2.0 * runit() - 1.0);
            mz0 += epsn * (2.0 * runit() - 1.0);
            const double nn = sqrt(a * a + b * b + mz0 * mz0);
            if (nn > 1.0e-12) { a /= nn; b /= nn; mz0 /= nn; }
            put(k, a, b, mz0);
          }
        break;
      }
      default:
        break;
    }
    if (g->ic_jitter_eps > 0.0) {
      const double e = g->ic_jitter_eps;
      for (size_t k = 0; k < n; k++) {
        if (!act[k]) continue;
        double a = y0[k] + e * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
        double b = y0[n + k] + e * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
        double cc = y0[2 * n + k] + e * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
        const double nn = sqrt(a * a + b * b + cc * cc);
        if (nn > 1.0e-30) { a /= nn; b /= nn; cc /= nn; }
        put(k, a, b, cc);
      }
    }
  }
  if (active_out) memcpy(active_out, act.data(), n);
  if (w_out) memcpy(w_out, w.data(), n * sizeof(double));
  if (gid_out) memcpy(gid_out, gid.data(), n * sizeof(int32_t));
  return (int)nact;
}

// ── KEY=VALUE knob parser (configs/sim_config.h names) ──────────────────
extern "C" int llg_parse_config(const char* text, llg_params* p, llg_geom_spec* g, llg_solver_opts* o) {
  if (!text || !p || !g || !o) return LLG_ERR_ARG;
  std::string s(text);
  size_t pos = 0;
  int count = 0;
  auto trim = [](std::string v) {
    while (!v.empty() && isspace((unsigned char)v.back())) v.pop_back();
    size_t a = 0;
    while (a < v.size() && isspace((unsigned char)v[a])) a++;
    return v.substr(a);
  };
  // knob name -> setter
  std::map<std::string, std::function<bool(const std::string&)>> set;
  auto dbl = [](double* dst) {
    return [dst](const std::string& v) {
      char* e = nullptr;
      const double x = strtod(v.c_str(), &e);
      if (e == v.c_str() || *e) return false;
      *dst = x;
      return true;
    };
  };
  auto i32 = [](int32_t* dst) {
    return [dst](const std::string& v) {
      char* e = nullptr;
      const long x = strtol(v.c_str(), &e, 10);
      if (e == v.c_str() || *e) return false;
      *dst = (int32_t)x;
      return true;
    };
  };
  auto u32 = [](uint32_t* dst) {
    return [dst](const std::string& v) {
      char* e = nullptr;
      const unsigned long x = strtoul(v.c_str(), &e, 10);
      if (e == v.c_str() || *e) return false;
      *dst = (uint32_t)x;
      return true;
    };
  };
  auto enm = [](int32_t* dst, std::map<std::string, int> names) {
    return [dst, names](const std::string& v) {
      auto it = names.find(v);
      if (it != names.end()) { *dst = it->second; return true; }
      char* e = nullptr;
      const long x = strtol(v.c_str(), &e, 10);
      if (e == v.c_str() || *e) return false;
      *dst = (int32_t)x;
      return true;
    };
  };
  int32_t nx_val = -1, ny_val = -1;
  set["NX_VAL"] = i32(&nx_val);  // reference slots: ng = NX_VAL / 3 (sim_config.h:56)
  set["NY_VAL"] = i32(&ny_val);
  set["NG"] = i32(&p->ng);
  set["NY"] = i32(&p->ny);
  set["EXECUTION_MODEL"] = enm(&p->exec_model, {{"EXEC_YMSK", 0}, {"EXEC_COMPACT", 1}});
  set["BOUNDARY"] = enm(&p->bc, {{"BC_PERIODIC", 0}, {"BC_FREE", 1}});
  set["NORMALIZE"] = enm(&p->norm_kind, {{"NORM_NONE", 0}, {"NORM_EXACT", 1}, {"NORM_REG", 2}});
  set["NORM_EPS"] = dbl(&p->norm_eps);
  set["ANISO_KIND"] = enm(&p->aniso_kind, {{"ANISO_LINEAR", 0}, {"ANISO_CUBIC", 1}});
  set["PHYS_C_CHG"] = dbl(&p->chg);
  set["PHYS_C_ALPHA"] = dbl(&p->alpha);
  set["PHYS_C_CHE"] = dbl(&p->che);
  set["PHYS_C_CHK"] = dbl(&p->chk);
  set["PHYS_C_CHA"] = dbl(&p->cha);
  set["PHYS_C_CHB"] = dbl(&p->chb);
  set["PHYS_MSK_X"] = dbl(&p->msk[0]);
  set["PHYS_MSK_Y"] = dbl(&p->msk[1]);
  set["PHYS_MSK_Z"] = dbl(&p->msk[2]);
  set["PHYS_NSK_X"] = dbl(&p->nsk[0]);
  set["PHYS_NSK_Y"] = dbl(&p->nsk[1]);
  set["PHYS_NSK_Z"] = dbl(&p->nsk[2]);
  static int32_t happ_enable = -1;
  happ_enable = -1;
  double happ[3] = {p->happ[0], p->happ[1], p->happ[2]};
  set["HAPP_ENABLE"] = i32(&happ_enable);
  set["HAPP_X"] = dbl(&happ[0]);
  set["HAPP_Y"] = dbl(&happ[1]);
  set["HAPP_Z"] = dbl(&happ[2]);
  set["DEMAG_STRENGTH"] = dbl(&p->demag_strength);
  set["DEMAG_THICK"] = dbl(&p->demag_thick);
  set["DEMAG_MODE"] = enm(&p->demag_mode, {{"DEMAG_OFF", 0}, {"DEMAG_PERIODIC", 1}, {"DEMAG_OPEN", 2}});
  set["DEMAG_WINDOWED"] = i32(&p->windowed);
  set["DEMAG_PRECISION"] = enm(&p->demag_precision, {{"DEMAG_FP64", 0}, {"DEMAG_MIXED", 1}});
  set["JV_MODE"] = enm(&p->jv_mode, {{"JV_REFERENCE", 0}, {"JV_FULL_FIELD", 1}});
  set["PRECOND"] = enm(&p->precond_kind, {{"PREC_BLOCK_JACOBI", 0}, {"PREC_LEARNED", 1}});
  set["GEOMETRY_KIND"] = enm(&g->geometry_kind, {{"GEOMETRY_BULK", 0}, {"GEOMETRY_HOLE_SQUARE", 1},
                                                 {"GEOMETRY_RING", 2}, {"GEOMETRY_POLYCRYSTAL", 3},
                                                 {"GEOMETRY_CUSTOM", 4}, {"GEOMETRY_ELLIPSE", 5},
                                                 {"GEOMETRY_ANNULUS", 6}, {"GEOMETRY_SLIT", 7}});
  set["HOLE_CENTER_X_FRAC"] = dbl(&g->hole_center_x_frac);
  set["HOLE_CENTER_Y_FRAC"] = dbl(&g->hole_center_y_frac);
  set["HOLE_RADIUS_FRAC_Y"] = dbl(&g->hole_radius_frac_y);
  set["OUTER_W_FRAC"] = dbl(&g->outer_w_frac);
  set["OUTER_H_FRAC"] = dbl(&g->outer_h_frac);
  set["INNER_W_FRAC_OF_OUTER"] = dbl(&g->inner_w_frac_of_outer);
  set["INNER_H_FRAC_OF_OUTER"] = dbl(&g->inner_h_frac_of_outer);
  set["NUM_GRAINS"] = i32(&g->num_grains);
  set["DEAD_GRAIN_FRAC"] = dbl(&g->dead_grain_frac);
  set["HOLE_SEED"] = u32(&g->hole_seed);
  set["MASK_EPS_CELLS"] = dbl(&g->mask_eps_cells);
  set["GRAIN_Z_BIAS"] = dbl(&g->grain_z_bias);
  set["ACTIVE_RX_FRAC"] = dbl(&g->active_rx_frac);
  set["ACTIVE_RY_FRAC"] = dbl(&g->active_ry_frac);
  set["ANNULUS_R_IN_FRAC"] = dbl(&g->annulus_r_in_frac);
  set["ANNULUS_R_OUT_FRAC"] = dbl(&g->annulus_r_out_frac);
  set["IC_KIND"] = enm(&g->ic_kind, {{"IC_UNIFORM", 0}, {"IC_HEAD_ON_STRIPES", 1}, {"IC_TWO_DOMAIN", 2},
                                     {"IC_GRAIN_BUMPS", 3}, {"IC_CUSTOM", 4}, {"IC_TWO_DOMAIN_X", 5},
                                     {"IC_VORTEX", 6}, {"IC_NEEL", 7}});
  // Néel texture (src/2d_fft/2d_fft.cu:94-120) and slit knobs (src/slit/2d_slit.cu:80-135)
  set["TEXTURE_CORE_MZ"] = dbl(&g->texture_core_mz);
  set["TEXTURE_OUTER_MZ"] = dbl(&g->texture_outer_mz);
  set["TEXTURE_WIDTH_FRAC"] = dbl(&g->texture_width_frac);
  set["TEXTURE_EPS"] = dbl(&g->texture_eps);
  set["CIRCLE_CENTER_X_FRAC"] = dbl(&g->circle_cx_frac);
  set["CIRCLE_CENTER_Y_FRAC"] = dbl(&g->circle_cy_frac);
  set["CIRCLE_RADIUS_FRAC_Y"] = dbl(&g->circle_r_frac_y);
  set["SCREEN_X_FRAC"] = dbl(&g->screen_x_frac);
  set["SLIT_W_FRAC"] = dbl(&g->slit_w_frac);
  double src_x_frac = -1.0, drive_freq = -1.0;
  set["SRC_X_FRAC"] = dbl(&src_x_frac);
  set["DRIVE_FREQ"] = dbl(&drive_freq);
  set["H_DRIVE"] = dbl(&p->src_amp);
  set["RAMP_TIME"] = dbl(&p->src_ramp);
  set["PML_CELLS"] = i32(&p->pml_cells);
  set["PML_ALPHA_MAX"] = dbl(&p->pml_alpha_max);
  set["INIT_MX"] = dbl(&g->init_m[0]);
  set["INIT_MY"] = dbl(&g->init_m[1]);
  set["INIT_MZ"] = dbl(&g->init_m[2]);
  set["STRIPE_LEFT_FRAC"] = dbl(&g->stripe_left_frac);
  set["STRIPE_RIGHT_FRAC"] = dbl(&g->stripe_right_frac);
  set["INIT_RANDOM_EPS"] = dbl(&g->init_random_eps);
  set["INIT_RANDOM_SEED"] = u32(&g->init_random_seed);
  set["TWO_DOMAIN_SPLIT_FRAC"] = dbl(&g->two_domain_split_frac);
  set["TWO_DOMAIN_TAIL_MY"] = dbl(&g->two_domain_tail_my);
  set["IC_CORE_MZ"] = dbl(&g->ic_core_mz);
  set["IC_JITTER_EPS"] = dbl(&g->ic_jitter_eps);
  set["RTOL_VAL"] = dbl(&o->rtol);
  set["ATOL_VAL"] = dbl(&o->atol);
  set["KRYLOV_DIM"] = i32(&o->maxl);
  set["MAX_BDF_ORDER"] = i32(&o->maxord);
  set["GS_KIND"] = enm(&o->gs_type, {{"GS_KIND_AUTO", 0}, {"GS_KIND_CGS", 1}, {"GS_KIND_MGS", 2}});
  set["MXSTEP"] = i32(&o->mxstep);
  set["DEVICE_RESIDENT"] = i32(&o->device_resident);
  while (pos < s.size()) {
    size_t e = s.find_first_of("\n;", pos);
    if (e == std::string::npos) e = s.size();
    std::string line = s.substr(pos, e - pos);
    pos = e + 1;
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    // allow whitespace-separated KEY=VALUE tokens on one line
    size_t tp = 0;
    while (tp < line.size()) {
      while (tp < line.size() && isspace((unsigned char)line[tp])) tp++;
      if (tp >= line.size()) break;
      size_t te = tp;
      while (te < line.size() && !isspace((unsigned char)line[te])) te++;
      std::string tok = line.substr(tp, te - tp);
      tp = te;
      const size_t eq = tok.find('=');
      if (eq == std::string::npos) return LLG_ERR_ARG;
      std::string key = trim(tok.substr(0, eq)), val = trim(tok.substr(eq + 1));
      if (!key.empty() && key[0] == '-' && key.size() > 1 && key[1] == 'D') key = key.substr(2);
      auto it = set.find(key);
      if (it == set.end()) return LLG_ERR_ARG;
      if (!it->second(val)) return LLG_ERR_ARG;
      count++;
    }
  }
  if (nx_val > 0) {
    if (nx_val % 3) return LLG_ERR_ARG;
    p->ng = nx_val / 3;
  }
  if (ny_val > 0) p->ny = ny_val;
  if (src_x_frac >= 0.0) p->src_col = (int32_t)(src_x_frac * (double)p->ng + 0.5);
  if (drive_freq >= 0.0) p->src_omega = 2.0 * 3.14159265358979323846 * drive_freq;
  g->ng = p->ng;
  g->ny = p->ny;
  if (happ_enable == 0) { p->happ[0] = p->happ[1] = p->happ[2] = 0.0; }
  else { p->happ[0] = happ[0]; p->happ[1] = happ[1]; p->happ[2] = happ[2]; }
  return count;
}
