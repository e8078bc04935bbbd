/*
 * or_demag.c — CPU restatement of the FFT demagnetisation chain.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 *   or_newell_point  ctt(): closed-form Newell integrals,
 *                    src/irregular/2d_fft/2d_i2/demag_fft.cu:27-61.  The nine
 *                    terms are evaluated with the reference's own grouping
 *                    (log of ratios, same term order) because the tensor is
 *                    pinned against the reference's printed N(0).
 *   or_newell_avg    calt(): 9x9-point average over the cell face, offsets
 *                    0.1·{-4..4}, demag_fft.cu:64-91.
 *   tensor placement demag_fft.cu:69-80 centres the tensor at (nx/2, ny/2) and
 *                    scatter_real_kernel (:143-161) undoes it with an FFT
 *                    shift; storing N at the wrapped displacement d mod P
 *                    (d in [-P/2, P-1-P/2]) gives the same circular sums.
 *   or_demag_apply   gather → forward FFT → Ĥ_a = Σ_b N̂_ab M̂_b → inverse FFT
 *                    → scale strength/(Px·Py), demag_fft.cu:325-363; the
 *                    windowed gather multiplies by w (2d_i3/demag_fft.cu:125-139).
 *   or_demag_direct  the same convolution as an O(N^2) sum (the reference's
 *                    demag_direct.cu cross-check, 2d_i1/demag_direct.cu).
 * Open boundaries (LLG_DEMAG_OPEN) run the same chain on a zero-padded
 * 2ng x 2ny grid; |d| <= ng-1 is all a linear convolution touches.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "or_internal.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ── Newell tensor ─────────────────────────────────────────────────── */
void or_newell_point(double thick, double sx, double sy, double out9[9]) {
  const double a = 0.49999, b = 0.5 * thick, sz = 0.0;
  const double X[2] = {sx - a, sx + a};
  const double Y[2] = {sy - a, sy + a};
  const double Z[2] = {sz - b, sz + b};
  double r[2][2][2]; /* r[ix][iy][iz] */
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++)
      for (int k = 0; k < 2; k++)
        r[i][j][k] = sqrt(X[i] * X[i] + Y[j] * Y[j] + Z[k] * Z[k]);
  /* sign (-1)^(number of '+a' coordinates) */
#define SG(i, j, k) ((((i) + (j) + (k)) & 1) ? -1.0 : 1.0)
  double xx = 0.0, yy = 0.0, zz = 0.0;
  int first = 1;
  /* xx: x outer, y middle, z inner; atan(Z·Y / (X·r)) */
  for (int i = 0; i < 2; i++)
    for (int j = 0; j < 2; j++)
      for (int k = 0; k < 2; k++) {
        const double tm = atan(Z[k] * Y[j] / (X[i] * r[i][j][k]));
        xx = first ? tm : xx + SG(i, j, k) * tm;
        first = 0;
      }
  first = 1;
  /* yy: y outer, x middle, z inner; atan(Z·X / (Y·r)) */
  for (int j = 0; j < 2; j++)
    for (int i = 0; i < 2; i++)
      for (int k = 0; k < 2; k++) {
        const double tm = atan(Z[k] * X[i] / (Y[j] * r[i][j][k]));
        yy = first ? tm : yy + SG(i, j, k) * tm;
        first = 0;
      }
  first = 1;
  /* zz: z outer, y middle, x inner; atan(X·Y / (Z·r)) */
  for (int k = 0; k < 2; k++)
    for (int j = 0; j < 2; j++)
      for (int i = 0; i < 2; i++) {
        const double tm = atan(X[i] * Y[j] / (Z[k] * r[i][j][k]));
        zz = first ? tm : zz + SG(i, j, k) * tm;
        first = 0;
      }
  /* off-diagonal terms: log of ratios over the pair of the third coordinate */
#define LZ(i, j) log((r[i][j][0] - Z[0]) / (r[i][j][1] - Z[1]))
#define LY(i, k) log((r[i][0][k] - Y[0]) / (r[i][1][k] - Y[1]))
#define LX(j, k) log((r[0][j][k] - X[0]) / (r[1][j][k] - X[1]))
  const double xy = LZ(0, 0) - LZ(1, 0) - LZ(0, 1) + LZ(1, 1); /* y outer, x inner */
  const double yx = LZ(0, 0) - LZ(0, 1) - LZ(1, 0) + LZ(1, 1); /* x outer, y inner */
  const double xz = LY(0, 0) - LY(1, 0) - LY(0, 1) + LY(1, 1); /* z outer, x inner */
  const double zx = LY(0, 0) - LY(0, 1) - LY(1, 0) + LY(1, 1); /* x outer, z inner */
  const double yz = LX(0, 0) - LX(1, 0) - LX(0, 1) + LX(1, 1); /* z outer, y inner */
  const double zy = LX(0, 0) - LX(0, 1) - LX(1, 0) + LX(1, 1); /* y outer, z inner */
#undef LZ
#undef LY
#undef LX
#undef SG
  out9[0] = xx; out9[1] = xy; out9[2] = xz;
  out9[3] = yx; out9[4] = yy; out9[5] = yz;
  out9[6] = zx; out9[7] = zy; out9[8] = zz;
}

void or_newell_avg(double thick, int dx, int dy, double out9[9]) {
  double acc[9] = {0};
  double dm[9];
  for (int jy = -4; jy <= 4; jy++) {
    const double sy = (double)dy + 0.1 * (double)jy;
    for (int ix = -4; ix <= 4; ix++) {
      const double sx = (double)dx + 0.1 * (double)ix;
      or_newell_point(thick, sx, sy, dm);
      for (int k = 0; k < 9; k++) acc[k] += dm[k];
    }
  }
  for (int k = 0; k < 9; k++) out9[k] = acc[k] / 81.;
}

/* representative displacement of wrapped index i on a grid of n points:
 * d in [-n/2, n-1-n/2] exactly as the reference's centring (i - n/2). */
static inline int rep_disp(int i, int n) {
  const int hi = n - 1 - n / 2;
  return (i <= hi) ? i : i - n;
}

/* ── FFT (mixed radix, recursive, complex interleaved) ──────────────── */
typedef struct { int n; int nf; int fac[64]; double* tw; } fft_plan;

static int fft_factor(int n, int* fac) {
  int nf = 0, m = n;
  while (m % 4 == 0) { fac[nf++] = 4; m /= 4; }
  while (m % 2 == 0) { fac[nf++] = 2; m /= 2; }
  for (int p = 3; m > 1; p += 2) {
    while (m % p == 0) { fac[nf++] = p; m /= p; }
    if ((long)p * p > m && m > 1) { fac[nf++] = m; m = 1; }
  }
  return nf;
}

static void fft_plan_init(fft_plan* pl, int n, int sign) {
  pl->n = n;
  pl->nf = fft_factor(n, pl->fac);
  pl->tw = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  for (int k = 0; k < n; k++) {
    const double ang = 2.0 * M_PI * (double)k / (double)n;
    pl->tw[2 * k] = cos(ang);
    pl->tw[2 * k + 1] = (sign < 0 ? -1.0 : 1.0) * sin(ang);
  }
}

static void fft_work(const fft_plan* pl, double* out, const double* in, int fstride, int istride,
                     int lvl, int nrem) {
  const int p = pl->fac[lvl];
  const int m = nrem / p;
  if (m == 1) {
    for (int q = 0; q < p; q++) {
      out[2 * q] = in[2 * (size_t)q * fstride * istride];
      out[2 * q + 1] = in[2 * (size_t)q * fstride * istride + 1];
    }
  } else {
    for (int q = 0; q < p; q++)
      fft_work(pl, out + 2 * (size_t)q * m, in + 2 * (size_t)q * fstride * istride, fstride * p,
               istride, lvl + 1, m);
  }
  /* generic butterfly with combined twiddles W_N^(fstride·k·q) */
  double scr[2 * 64];
  double* big = NULL;
  double* s = scr;
  if (p > 64) { big = (double*)malloc(sizeof(double) * 2 * (size_t)p); s = big; }
  const int N = pl->n;
  for (int u = 0; u < m; u++) {
    for (int q = 0; q < p; q++) {
      s[2 * q] = out[2 * (u + (size_t)q * m)];
      s[2 * q + 1] = out[2 * (u + (size_t)q * m) + 1];
    }
    for (int q1 = 0; q1 < p; q1++) {
      const int k = u + q1 * m;
      double re = s[0], im = s[1];
      long tw = 0;
      for (int q = 1; q < p; q++) {
        tw += (long)fstride * k;
        tw %= N;
        const double wr = pl->tw[2 * tw], wi = pl->tw[2 * tw + 1];
        re += s[2 * q] * wr - s[2 * q + 1] * wi;
        im += s[2 * q] * wi + s[2 * q + 1] * wr;
      }
      out[2 * (size_t)k] = re;
      out[2 * (size_t)k + 1] = im;
    }
  }
  free(big);
}

static void fft_exec(const fft_plan* pl, double* data, double* tmp) {
  if (pl->n == 1) return;
  fft_work(pl, tmp, data, 1, 1, 0, pl->n);
  memcpy(data, tmp, sizeof(double) * 2 * (size_t)pl->n);
}

int or_fft(int n, double* data, int sign) {
  if (n <= 0) return -1;
  fft_plan pl;
  fft_plan_init(&pl, n, sign);
  double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)n);
  fft_exec(&pl, data, tmp);
  free(tmp);
  free(pl.tw);
  return 0;
}

/* 2-D FFT of a px*py complex array (row-major, x fastest). */
static void fft2(double* a, int px, int py, int sign) {
  fft_plan prow, pcol;
  fft_plan_init(&prow, px, sign);
  fft_plan_init(&pcol, py, sign);
#pragma omp parallel
  {
    double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)(px > py ? px : py));
    double* col = (double*)malloc(sizeof(double) * 2 * (size_t)py);
#pragma omp for schedule(static)
    for (int j = 0; j < py; j++) fft_exec(&prow, a + 2 * (size_t)j * px, tmp);
#pragma omp for schedule(static)
    for (int i = 0; i < px; i++) {
      for (int j = 0; j < py; j++) {
        col[2 * j] = a[2 * ((size_t)j * px + i)];
        col[2 * j + 1] = a[2 * ((size_t)j * px + i) + 1];
      }
      fft_exec(&pcol, col, tmp);
      for (int j = 0; j < py; j++) {
        a[2 * ((size_t)j * px + i)] = col[2 * j];
        a[2 * ((size_t)j * px + i) + 1] = col[2 * j + 1];
      }
    }
    free(tmp);
    free(col);
  }
  free(prow.tw);
  free(pcol.tw);
}

/* ── demag context ─────────────────────────────────────────────────── */
or_demag* or_demag_create(const llg_params* p) {
  or_demag* d = (or_demag*)calloc(1, sizeof(or_demag));
  if (!d) return NULL;
  if (p->demag_mode == LLG_DEMAG_OPEN) { d->px = 2 * p->ng; d->py = 2 * p->ny; }
  else { d->px = p->ng; d->py = p->ny; }
  d->strength = p->demag_strength;
  d->thick = p->demag_thick;
  const size_t np = (size_t)d->px * d->py;
  for (int c = 0; c < 9; c++) {
    d->t[c] = (double*)malloc(np * sizeof(double));
    d->that[c] = (double*)malloc(2 * np * sizeof(double));
    if (!d->t[c] || !d->that[c]) { or_demag_free(d); return NULL; }
  }
  const int px = d->px, py = d->py;
#pragma omp parallel for schedule(dynamic, 4)
  for (int j = 0; j < py; j++) {
    for (int i = 0; i < px; i++) {
      double v[9];
      or_newell_avg(d->thick, rep_disp(i, px), rep_disp(j, py), v);
      for (int c = 0; c < 9; c++) d->t[c][(size_t)j * px + i] = v[c];
    }
  }
  d->n0[0] = d->t[0][0];
  d->n0[1] = d->t[4][0];
  d->n0[2] = d->t[8][0];
  for (int c = 0; c < 9; c++) {
    for (size_t k = 0; k < np; k++) { d->that[c][2 * k] = d->t[c][k]; d->that[c][2 * k + 1] = 0.0; }
    fft2(d->that[c], px, py, -1);
  }
  return d;
}

void or_demag_free(or_demag* d) {
  if (!d) return;
  for (int c = 0; c < 9; c++) { free(d->t[c]); free(d->that[c]); }
  free(d);
}

int or_demag_run(const or_ctx* c, const double* y, double* h) {
  const or_demag* d = c->dm;
  if (!d) { memset(h, 0, sizeof(double) * 3 * (size_t)c->ncell); return 0; }
  const int px = d->px, py = d->py, ng = c->p.ng, ny = c->p.ny;
  const size_t np = (size_t)px * py;
  const long n = c->ncell;
  double* M[3];
  double* H = (double*)malloc(2 * np * sizeof(double));
  for (int b = 0; b < 3; b++) {
    M[b] = (double*)calloc(2 * np, sizeof(double));
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < ng; i++) {
        const long cell = (long)j * ng + i;
        const double v = y[b * n + cell];
        M[b][2 * ((size_t)j * px + i)] = c->w ? c->w[cell] * v : v;
      }
    fft2(M[b], px, py, -1);
  }
  const double scale = d->strength / (double)np;
  for (int a = 0; a < 3; a++) {
#pragma omp parallel for schedule(static)
    for (size_t k = 0; k < np; k++) {
      double re = 0.0, im = 0.0;
      for (int b = 0; b < 3; b++) {
        const double* F = d->that[3 * a + b];
        re += F[2 * k] * M[b][2 * k] - F[2 * k + 1] * M[b][2 * k + 1];
        im += F[2 * k] * M[b][2 * k + 1] + F[2 * k + 1] * M[b][2 * k];
      }
      H[2 * k] = re;
      H[2 * k + 1] = im;
    }
    fft2(H, px, py, +1);
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < ng; i++) h[a * n + (long)j * ng + i] = H[2 * ((size_t)j * px + i)] * scale;
  }
  for (int b = 0; b < 3; b++) free(M[b]);
  free(H);
  return 0;
}

int or_demag_apply(or_ctx* c, const double* y, double* h) { return or_demag_run(c, y, h); }

int or_demag_direct(or_ctx* c, const double* y, double* h) {
  const or_demag* d = c->dm;
  const long n = c->ncell;
  if (!d) { memset(h, 0, sizeof(double) * 3 * (size_t)n); return 0; }
  const int px = d->px, py = d->py, ng = c->p.ng, ny = c->p.ny;
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < ng; i++) {
      double acc[3] = {0.0, 0.0, 0.0};
      for (int jj = 0; jj < ny; jj++) {
        const int wy = ((j - jj) % py + py) % py;
        for (int ii = 0; ii < ng; ii++) {
          const int wx = ((i - ii) % px + px) % px;
          const size_t t = (size_t)wy * px + wx;
          const long src = (long)jj * ng + ii;
          const double ww = c->w ? c->w[src] : 1.0;
          const double m0 = ww * y[src], m1 = ww * y[n + src], m2 = ww * y[2 * n + src];
          for (int a = 0; a < 3; a++)
            acc[a] += d->t[3 * a][t] * m0 + d->t[3 * a + 1][t] * m1 + d->t[3 * a + 2][t] * m2;
        }
      }
      const long cell = (long)j * ng + i;
      for (int a = 0; a < 3; a++) h[a * n + cell] = d->strength * acc[a];
    }
  }
  return 0;
}

int or_demag_self(or_ctx* c, double out3[3]) {
  if (!c->dm) { out3[0] = out3[1] = out3[2] = 0.0; return 0; }
  for (int a = 0; a < 3; a++) out3[a] = c->dm->n0[a] * c->dm->strength;
  return 0;
}

double or_demag_tensor(or_ctx* c, int comp, int dx, int dy) {
  if (!c->dm || comp < 0 || comp > 8) return 0.0;
  const int px = c->dm->px, py = c->dm->py;
  const int wx = ((dx % px) + px) % px, wy = ((dy % py) + py) % py;
  return c->dm->t[comp][(size_t)wy * px + wx];
}
