/*
 * or_geometry.c — CPU restatement of the host-side geometry and initial-
 * condition builders.  TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 *   square hole     src/irregular/2d_fft/2d_i2/2d_fft.cu:544-566
 *   rectangle/ring  src/irregular/2d_fft/2d_i5/2d_fft.cu:512-545 (outer rect;
 *                   the inner rect of configs/sim_config.h GEOMETRY_RING is cut out)
 *   ellipse         src/irregular/2d_fft/2d_i6/2d_i6.cu:462-533
 *   polycrystal     src/irregular/2d_fft/2d_i3/2d_fft.cu:255-387
 *                   (generate_grains, nearest_grain, tanh window, axes)
 *   IC uniform      2d_i2/2d_fft.cu:610-639
 *   IC stripes      2d_i1/2d_fft.cu:540-541, 625-657
 *   IC two-domain   2d_i4/2d_fft.cu:562-595
 *   IC grain bumps  2d_i3/2d_fft.cu:916-984
 *   slit screen     src/slit/2d_slit.cu:482-486, 541-560
 *   IC Néel texture src/2d_fft/2d_fft.cu:460-463, 533-580
 * Random numbers come from the C library srand/rand in the reference's
 * call order, so the same seed gives the same geometry and state.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "or_internal.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct { double sx, sy, ax, ay, az, nx, ny, nz; int dead; } grain;

static double runit(void) { return (double)rand() / (double)RAND_MAX; }

static void gen_grains(const llg_geom_spec* g, grain* gr) {
  const int ng = g->ng, ny = g->ny, NG = g->num_grains;
  srand((unsigned)g->hole_seed);
  int gx = (int)ceil(sqrt((double)NG * (double)ng / (double)ny));
  if (gx < 1) gx = 1;
  const int gy = (NG + gx - 1) / gx;
  const double dxs = (double)ng / (double)gx, dys = (double)ny / (double)gy;
  int idx = 0;
  for (int j = 0; j < gy && idx < NG; j++)
    for (int i = 0; i < gx && idx < NG; i++) {
      gr[idx].sx = ((double)i + 0.15 + 0.7 * runit()) * dxs;
      gr[idx].sy = ((double)j + 0.15 + 0.7 * runit()) * dys;
      while (gr[idx].sx < 0.0) gr[idx].sx += (double)ng;
      while (gr[idx].sx >= (double)ng) gr[idx].sx -= (double)ng;
      while (gr[idx].sy < 0.0) gr[idx].sy += (double)ny;
      while (gr[idx].sy >= (double)ny) gr[idx].sy -= (double)ny;
      idx++;
    }
  while (idx < NG) { gr[idx].sx = runit() * (double)ng; gr[idx].sy = runit() * (double)ny; idx++; }
  for (int k = 0; k < NG; k++) {
    const double u = runit();
    const double sign = (runit() < 0.5) ? -1.0 : 1.0;
    const double z = sign * pow(u, 1.0 / g->grain_z_bias);
    const double phi = 2.0 * M_PI * runit();
    const double rxy = sqrt(fmax(0.0, 1.0 - z * z));
    gr[k].ax = rxy * cos(phi);
    gr[k].ay = rxy * sin(phi);
    gr[k].az = z;
    const double psi = 2.0 * M_PI * runit();
    gr[k].nx = cos(psi);
    gr[k].ny = sin(psi);
    gr[k].nz = 0.0;
    gr[k].dead = (runit() < g->dead_grain_frac) ? 1 : 0;
  }
}

static int nearest(const grain* gr, int NG, double x, double y, int ng, int ny) {
  int best = 0;
  double bd = 1.0e30;
  for (int k = 0; k < NG; k++)
    for (int dyp = -1; dyp <= 1; dyp++)
      for (int dxp = -1; dxp <= 1; dxp++) {
        const double sx = gr[k].sx + (double)dxp * (double)ng;
        const double sy = gr[k].sy + (double)dyp * (double)ny;
        const double dx = x - sx, dy = y - sy;
        const double d2 = dx * dx + dy * dy;
        if (d2 < bd) { bd = d2; best = k; }
      }
  return best;
}

int or_build_geometry(const llg_geom_spec* g, uint8_t* active_out, double* w_out, double* msk3,
                      double* nsk3, int32_t* gid_out, double* y0) {
  if (!g || g->ng <= 0 || g->ny <= 0) return LLG_ERR_ARG;
  const int ng = g->ng, ny = g->ny;
  const long n = (long)ng * ny;
  uint8_t* act = (uint8_t*)malloc((size_t)n);
  double* w = (double*)malloc((size_t)n * sizeof(double));
  int32_t* gid = (int32_t*)calloc((size_t)n, sizeof(int32_t));
  grain* gr = NULL;
  if (!act || !w || !gid) { free(act); free(w); free(gid); return LLG_ERR_NOMEM; }
  for (long k = 0; k < n; k++) { act[k] = 1; w[k] = 1.0; }

  switch (g->geometry_kind) {
    case LLG_GEOM_BULK:
    case LLG_GEOM_CUSTOM:
      break;
    case LLG_GEOM_HOLE_SQUARE: {
      const double cx = g->hole_center_x_frac * (double)(ng - 1);
      const double cy = g->hole_center_y_frac * (double)(ny - 1);
      const double hs = g->hole_radius_frac_y * (double)ny;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++) {
          const double ddx = fabs((double)i - cx), ddy = fabs((double)j - cy);
          act[(long)j * ng + i] = (ddx <= hs && ddy <= hs) ? 0 : 1;
        }
      break;
    }
    case LLG_GEOM_RING: {
      const double cx = 0.5 * (double)ng, cy = 0.5 * (double)ny;
      const double hwo = 0.5 * g->outer_w_frac * (double)ng, hho = 0.5 * g->outer_h_frac * (double)ny;
      const double hwi = hwo * g->inner_w_frac_of_outer, hhi = hho * g->inner_h_frac_of_outer;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++) {
          const double dx = fabs((double)i + 0.5 - cx), dy = fabs((double)j + 0.5 - cy);
          const int in_o = (dx <= hwo && dy <= hho);
          const int in_i = (dx < hwi && dy < hhi);
          act[(long)j * ng + i] = (in_o && !in_i) ? 1 : 0;
        }
      break;
    }
    case LLG_GEOM_ELLIPSE: {
      const double cx = 0.5 * (double)ng, cy = 0.5 * (double)ny;
      const double rx = g->active_rx_frac * (double)ng, ry = g->active_ry_frac * (double)ny;
      if (rx <= 0.0 || ry <= 0.0) { free(act); free(w); free(gid); return LLG_ERR_ARG; }
      const double irx2 = 1.0 / (rx * rx), iry2 = 1.0 / (ry * ry);
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++) {
          const double dx = (double)i + 0.5 - cx, dy = (double)j + 0.5 - cy;
          const double q = dx * dx * irx2 + dy * dy * iry2;
          act[(long)j * ng + i] = (q <= 1.0) ? 1 : 0;
        }
      break;
    }
    case LLG_GEOM_ANNULUS: {
      const double cx = 0.5 * (double)ng, cy = 0.5 * (double)ny;
      const double nmin = (double)(ng < ny ? ng : ny);
      const double rin = g->annulus_r_in_frac * nmin, rout = g->annulus_r_out_frac * nmin;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++) {
          const double dx = (double)i + 0.5 - cx, dy = (double)j + 0.5 - cy;
          const double r = sqrt(dx * dx + dy * dy);
          act[(long)j * ng + i] = (r >= rin && r <= rout) ? 1 : 0;
        }
      break;
    }
    case LLG_GEOM_SLIT: {
      const int screen_col = (int)(g->screen_x_frac * (double)ng + 0.5);
      const int slit_w = (int)(g->slit_w_frac * (double)ny + 0.5);
      const int lo = ny / 2 - slit_w / 2, hi = lo + slit_w;
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++) {
          const int in_screen = (i == screen_col) && !((j >= lo) && (j < hi));
          act[(long)j * ng + i] = in_screen ? 0 : 1;
        }
      break;
    }
    case LLG_GEOM_POLYCRYSTAL: {
      const int NG = g->num_grains;
      if (NG <= 0) { free(act); free(w); free(gid); return LLG_ERR_ARG; }
      gr = (grain*)calloc((size_t)NG, sizeof(grain));
      gen_grains(g, gr);
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < ng; i++)
          gid[(long)j * ng + i] = nearest(gr, NG, (double)i + 0.5, (double)j + 0.5, ng, ny);
      long nh = 0;
      for (long k = 0; k < n; k++) if (gr[gid[k]].dead) nh++;
      if (nh > 0) {
        int* hx = (int*)malloc((size_t)nh * sizeof(int));
        int* hy = (int*)malloc((size_t)nh * sizeof(int));
        long q = 0;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++)
            if (gr[gid[(long)j * ng + i]].dead) { hx[q] = i; hy[q] = j; q++; }
#pragma omp parallel for schedule(dynamic, 4)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const long cell = (long)j * ng + i;
            if (gr[gid[cell]].dead) { w[cell] = 0.0; continue; }
            double d2m = 1.0e30;
            for (long k = 0; k < nh; k++) {
              int ddx = i - hx[k], ddy = j - hy[k];
              if (ddx > ng / 2) ddx -= ng;
              if (ddx < -ng / 2) ddx += ng;
              if (ddy > ny / 2) ddy -= ny;
              if (ddy < -ny / 2) ddy += ny;
              const double d2 = (double)(ddx * ddx + ddy * ddy);
              if (d2 < d2m) d2m = d2;
            }
            const double d = sqrt(d2m) - 0.5;
            double ww = 0.5 * (1.0 + tanh(d / g->mask_eps_cells));
            if (ww < 1.0e-3) ww = 0.0;
            if (ww > 1.0 - 1.0e-3) ww = 1.0;
            w[cell] = ww;
          }
        free(hx); free(hy);
      }
      for (long k = 0; k < n; k++) act[k] = (w[k] > 1.0e-3) ? 1 : 0;
      if (msk3)
        for (long k = 0; k < n; k++) { msk3[k] = gr[gid[k]].ax; msk3[n + k] = gr[gid[k]].ay; msk3[2 * n + k] = gr[gid[k]].az; }
      if (nsk3)
        for (long k = 0; k < n; k++) { nsk3[k] = gr[gid[k]].nx; nsk3[n + k] = gr[gid[k]].ny; nsk3[2 * n + k] = gr[gid[k]].nz; }
      break;
    }
    default:
      free(act); free(w); free(gid);
      return LLG_ERR_ARG;
  }
  if (g->geometry_kind != LLG_GEOM_POLYCRYSTAL) {
    for (long k = 0; k < n; k++) w[k] = act[k] ? 1.0 : 0.0;
  }

  long nact = 0;
  for (long k = 0; k < n; k++) nact += act[k];

  if (y0) {
    memset(y0, 0, sizeof(double) * 3 * (size_t)n);
    srand((unsigned)g->init_random_seed);
    switch (g->ic_kind) {
      case LLG_IC_UNIFORM:
      case LLG_IC_CUSTOM: {
        double m0 = g->init_m[0], m1 = g->init_m[1], m2 = g->init_m[2];
        const double n0 = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
        if (n0 > 1.0e-30) { m0 /= n0; m1 /= n0; m2 /= n0; }
        for (long k = 0; k < n; k++)
          if (act[k]) { y0[k] = m0; y0[n + k] = m1; y0[2 * n + k] = m2; }
        break;
      }
      case LLG_IC_HEAD_ON_STRIPES: {
        const int q1 = (int)(g->stripe_left_frac * (double)ng + 0.5);
        const int q3 = (int)(g->stripe_right_frac * (double)ng + 0.5);
        const double eps = g->init_random_eps;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const long cell = (long)j * ng + i;
            double mx0 = (i >= q1 && i < q3) ? 1.0 : -1.0;
            double my0 = eps * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
            double mz0 = eps * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
            const double nn = sqrt(mx0 * mx0 + my0 * my0 + mz0 * mz0);
            mx0 /= nn; my0 /= nn; mz0 /= nn;
            if (act[cell]) { y0[cell] = mx0; y0[n + cell] = my0; y0[2 * n + cell] = mz0; }
          }
        break;
      }
      case LLG_IC_TWO_DOMAIN: {
        const int jsplit = (int)floor(g->two_domain_split_frac * (double)ny);
        const double tail = g->two_domain_tail_my;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const long cell = (long)j * ng + i;
            if (!act[cell]) continue;
            double mx0, my0, mz0 = 0.0;
            if (j >= jsplit) { mx0 = -1.0; my0 = 0.0; }
            else { mx0 = 1.0; my0 = (i < ng / 2) ? -tail : tail; }
            const double nn = sqrt(mx0 * mx0 + my0 * my0 + mz0 * mz0);
            if (nn > 1e-30) { mx0 /= nn; my0 /= nn; mz0 /= nn; }
            y0[cell] = mx0; y0[n + cell] = my0; y0[2 * n + cell] = mz0;
          }
        break;
      }
      case LLG_IC_TWO_DOMAIN_X: {
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const long cell = (long)j * ng + i;
            if (!act[cell]) continue;
            y0[cell] = (i < ng / 2) ? 1.0 : -1.0;
          }
        break;
      }
      case LLG_IC_VORTEX: {
        const double cx = 0.5 * (double)ng, cy = 0.5 * (double)ny;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const long cell = (long)j * ng + i;
            if (!act[cell]) continue;
            const double x = (double)i + 0.5 - cx, y = (double)j + 0.5 - cy;
            double mx0 = -y, my0 = x, mz0 = 0.1;
            const double nn = sqrt(mx0 * mx0 + my0 * my0 + mz0 * mz0);
            mx0 /= nn; my0 /= nn; mz0 /= nn;
            y0[cell] = mx0; y0[n + cell] = my0; y0[2 * n + cell] = mz0;
          }
        break;
      }
      case LLG_IC_NEEL: {
        const double cx = g->circle_cx_frac * (double)(ng - 1);
        const double cy = g->circle_cy_frac * (double)(ny - 1);
        const double radius = g->circle_r_frac_y * (double)ny;
        double width = g->texture_width_frac * radius;
        if (width < 1.0) width = 1.0;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const long cell = (long)j * ng + i;
            if (!act[cell]) continue;
            const double ddx = (double)i - cx, ddy = (double)j - cy;
            const double rho = sqrt(ddx * ddx + ddy * ddy);
            const double s = 0.5 * (1.0 - tanh((rho - radius) / width));
            double mz0 = g->texture_outer_mz + (g->texture_core_mz - g->texture_outer_mz) * s;
            if (mz0 > 1.0) mz0 = 1.0;
            if (mz0 < -1.0) mz0 = -1.0;
            const double mperp = sqrt(fmax(0.0, 1.0 - mz0 * mz0));
            y0[cell] = (rho > g->texture_eps) ? mperp * (ddx / rho) : 0.0;
            y0[n + cell] = (rho > g->texture_eps) ? mperp * (ddy / rho) : 0.0;
            y0[2 * n + cell] = mz0;
          }
        break;
      }
      case LLG_IC_GRAIN_BUMPS: {
        if (!gr) break;
        const double core = g->ic_core_mz, epsn = 0.05;
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < ng; i++) {
            const long k = (long)j * ng + i;
            const int gg = gid[k];
            if (w[k] <= 1.0e-3) continue;
            double ddx = (double)i + 0.5 - gr[gg].sx, ddy = (double)j + 0.5 - gr[gg].sy;
            if (ddx > ng / 2.0) ddx -= ng;
            if (ddx < -ng / 2.0) ddx += ng;
            if (ddy > ny / 2.0) ddy -= ny;
            if (ddy < -ny / 2.0) ddy += ny;
            const double r = sqrt(ddx * ddx + ddy * ddy);
            double s = r / 14.0;
            if (s > 1.0) s = 1.0;
            double sgz = (gr[gg].az >= 0.0) ? 1.0 : -1.0;
            if (fabs(gr[gg].az) < 0.05) sgz = 0.0;
            double mz0 = sgz * core * (1.0 - s * s);
            const double mperp = sqrt(fmax(0.0, 1.0 - mz0 * mz0));
            double tx = -ddy, ty = ddx;
            const double tn = sqrt(tx * tx + ty * ty);
            if (tn > 1.0e-12) { tx /= tn; ty /= tn; } else { tx = 1.0; ty = 0.0; }
            const double bx = gr[gg].ax, by = gr[gg].ay;
            const double bn = sqrt(bx * bx + by * by);
            double ex, ey;
            if (bn > 1.0e-6) { ex = bx / bn; ey = by / bn; } else { ex = 1.0; ey = 0.0; }
            double pxx = (1.0 - s) * tx + s * ex, pyy = (1.0 - s) * ty + s * ey;
            const double pn = sqrt(pxx * pxx + pyy * pyy);
            if (pn > 1.0e-12) { pxx /= pn; pyy /= pn; }
            double mx0 = mperp * pxx + epsn * (2.0 * runit() - 1.0);
            double my0 = mperp * pyy + epsn * (2.0 * runit() - 1.0);
            mz0 += epsn * (2.0 * runit() - 1.0);
            const double nn = sqrt(mx0 * mx0 + my0 * my0 + mz0 * mz0);
            if (nn > 1.0e-12) { mx0 /= nn; my0 /= nn; mz0 /= nn; }
            y0[k] = mx0; y0[n + k] = my0; y0[2 * n + k] = mz0;
          }
        break;
      }
      default:
        break;
    }
    if (g->ic_jitter_eps > 0.0) {
      const double e = g->ic_jitter_eps;
      for (long k = 0; k < n; k++) {
        if (!act[k]) continue;
        double m0 = y0[k] + e * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
        double m1 = y0[n + k] + e * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
        double m2 = y0[2 * n + k] + e * (2.0 * (double)rand() / (double)RAND_MAX - 1.0);
        const double nn = sqrt(m0 * m0 + m1 * m1 + m2 * m2);
        if (nn > 1.0e-30) { m0 /= nn; m1 /= nn; m2 /= nn; }
        y0[k] = m0; y0[n + k] = m1; y0[2 * n + k] = m2;
      }
    }
  }

  if (active_out) memcpy(active_out, act, (size_t)n);
  if (w_out) memcpy(w_out, w, (size_t)n * sizeof(double));
  if (gid_out) memcpy(gid_out, gid, (size_t)n * sizeof(int32_t));
  if (g->geometry_kind != LLG_GEOM_POLYCRYSTAL) {
    if (msk3) for (long k = 0; k < 3 * n; k++) msk3[k] = 0.0;
    if (nsk3) for (long k = 0; k < 3 * n; k++) nsk3[k] = 0.0;
  }
  free(gr);
  free(act); free(w); free(gid);
  return (int)nact;
}
