/*
 * or_physics.c — CPU restatement of the per-cell LLG operators.
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 *   or_normalize  2d_i2/2d_fft.cu:262-282 (regularised, eps = 1e-3)
 *                 2d_i1/2d_fft.cu:253-275 (exact, skipped for |m| <= 1e-30)
 *   or_rhs        2d_i2/2d_fft.cu:300-357 + 366-411 (dense mask, cubic)
 *                 2d_i4/2d_fft.cu:309-311 (+ uniform applied field)
 *                 2d_i1/2d_fft.cu:296-368 (linear anisotropy + DMI)
 *                 2d_i6/2d_i6.cu:250-343 (compact: inactive entries zeroed)
 *                 2d_i3/2d_fft.cu:451-627 (windowed neighbours w·m, per-cell
 *                 axes, output gated by w_self)
 *                 src/slit/2d_slit.cu:236-240, 297-349 (soft source on one
 *                 column, damping ramped up in the absorbing edge columns)
 *   or_jtv        2d_i2/jtv.cu:49-122, 2d_i1/jtv.cu:43-96, 2d_i6/jtv.cu:47-130
 *                 (+ the demag derivative the reference omits, 2d_i2/jtv.h:9-13,
 *                 in LLG_JV_FULL_DEMAG)
 *   or_psetup     2d_i2/precond.cu:119-251, 2d_i1/precond.cu:108-241
 *   or_psolve     2d_i2/precond.cu:254-285 (z = ymsk · P^-1 r)
 *
 * SoA index: component a of cell c lives at a*ncell + c.  All paths use
 * the same formula: yd = gate · (chg (h × m) + alpha (h − (m·h) m)),
 * gate = 1/0 by the active flag (dense mask and compact lists give the same
 * numbers), or w_self when windowed.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "or_internal.h"

static inline int wrapi(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

/* Neighbour value of component a at (i + di, j + dj) for the stencil:
 * periodic wrap or, with free edges, 0 outside the grid (the same trick the
 * reference uses for hole neighbours, which hold m = 0).  Windowed runs
 * read w·m (2d_i3/2d_fft.cu:492-506).                                     */
static inline double nbv(const or_ctx* c, const double* y, int a, int i, int j) {
  const int ng = c->p.ng, ny = c->p.ny;
  if (c->p.bc == LLG_BC_FREE) {
    if (i < 0 || i >= ng || j < 0 || j >= ny) return 0.0;
  } else {
    i = wrapi(i, ng);
    j = wrapi(j, ny);
  }
  const long cell = (long)j * ng + i;
  const double v = y[a * c->ncell + cell];
  return c->w ? c->w[cell] * v : v;
}

static inline double cell_axis(const or_ctx* c, const double* arr3, const double* uni, int a, long cell) {
  return arr3 ? arr3[a * c->ncell + cell] : uni[a];
}

static inline double gate_of(const or_ctx* c, long cell) {
  if (c->w) return c->w[cell];
  if (c->active) return c->active[cell] ? 1.0 : 0.0;
  return 1.0;
}

void or_normalize(or_ctx* c, double* y) {
  const long n = c->ncell;
  if (c->p.norm_kind == LLG_NORM_NONE) return;
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n; k++) {
    const double m1 = y[k], m2 = y[n + k], m3 = y[2 * n + k];
    const double ymp = sqrt(m1 * m1 + m2 * m2 + m3 * m3);
    if (c->p.norm_kind == LLG_NORM_REG) {
      const double inv = 1.0 / (ymp + c->p.norm_eps);
      y[k] = m1 * inv; y[n + k] = m2 * inv; y[2 * n + k] = m3 * inv;
    } else if (ymp > 1.0e-30) {
      const double inv = 1.0 / ymp;
      y[k] = m1 * inv; y[n + k] = m2 * inv; y[2 * n + k] = m3 * inv;
    }
  }
}

/* Soft source h_x(t) = H ramp(t) sin(omega t), smoothstep ramp
 * (src/slit/2d_slit.cu:236-240, 331-340).                                 */
static double source_at(const llg_params* p, double t) {
  if (p->src_amp == 0.0 || p->src_col < 0 || p->src_col >= p->ng) return 0.0;
  double ramp = 1.0;
  if (p->src_ramp > 0.0 && t < p->src_ramp) {
    const double x = t / p->src_ramp;
    ramp = x * x * (3.0 - 2.0 * x);
  }
  return p->src_amp * ramp * sin(p->src_omega * t);
}

/* RHS damping of column i: cubic ramp in the absorbing layers
 * (src/slit/2d_slit.cu:297-315).                                          */
static double alpha_at(const llg_params* p, int i) {
  if (p->pml_cells <= 0) return p->alpha;
  const int pml = p->pml_cells;
  double s = 0.0;
  if (i < pml) s = 1.0 - (double)i / (double)pml;
  else if (i >= p->ng - pml) s = (double)(i - (p->ng - pml)) / (double)pml;
  return p->alpha + (p->pml_alpha_max - p->alpha) * s * s * s;
}

/* Local field pieces shared by f, Jv and P.  exch_a = che·Σ4 nbrs,
 * dmi_a = chb·nsk_a·(L + R) (2d_i1/2d_fft.cu:344-360).                    */
typedef struct { double h[3]; double msk[3]; double nsk[3]; } local_field;

static void field_at(const or_ctx* c, const double* y, int i, int j, int with_demag_app,
                     local_field* lf) {
  const long n = c->ncell;
  const long cell = (long)j * c->p.ng + i;
  const double m[3] = {y[cell], y[n + cell], y[2 * n + cell]};
  for (int a = 0; a < 3; a++) {
    lf->msk[a] = cell_axis(c, c->msk3, c->p.msk, a, cell);
    lf->nsk[a] = cell_axis(c, c->nsk3, c->p.nsk, a, cell);
  }
  double aniso[3];
  if (c->p.aniso_kind == LLG_ANISO_CUBIC) {
    for (int a = 0; a < 3; a++) aniso[a] = lf->msk[a] * c->p.chk * m[a] * (m[a] * m[a] - 1.0);
  } else {
    const double md = m[0] * lf->msk[0] + m[1] * lf->msk[1] + m[2] * lf->msk[2];
    const double fac = c->p.chk * md + c->p.cha;
    for (int a = 0; a < 3; a++) aniso[a] = lf->msk[a] * fac;
  }
  for (int a = 0; a < 3; a++) {
    const double L = nbv(c, y, a, i - 1, j), R = nbv(c, y, a, i + 1, j);
    const double U = nbv(c, y, a, i, j - 1), D = nbv(c, y, a, i, j + 1);
    double h = c->p.che * (L + R + U + D) + aniso[a] + c->p.chb * lf->nsk[a] * (L + R);
    if (with_demag_app) {
      const int src = (a == 0 && c->p.src_amp != 0.0 && c->p.src_col >= 0 && c->p.src_col < c->p.ng &&
                       i == c->p.src_col);
      h = h + c->hd[a * n + cell] + (src ? c->p.happ[0] + c->src_h : c->p.happ[a]);
    }
    lf->h[a] = h;
  }
}

int or_rhs(or_ctx* c, double t, double* y, double* ydot) {
  c->src_h = source_at(&c->p, t);
  const long n = c->ncell;
  const int ng = c->p.ng, ny = c->p.ny;
  or_normalize(c, y);
  if (c->p.demag_mode != LLG_DEMAG_OFF && c->p.demag_strength > 0.0) {
    if (or_demag_run(c, y, c->hd) != 0) return -1;
  } else {
    memset(c->hd, 0, sizeof(double) * 3 * n);
  }
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < ng; i++) {
      const long cell = (long)j * ng + i;
      if (c->active && !c->active[cell] && !c->w) {
        ydot[cell] = 0.0; ydot[n + cell] = 0.0; ydot[2 * n + cell] = 0.0;
        continue;
      }
      local_field lf;
      field_at(c, y, i, j, 1, &lf);
      const double m1 = y[cell], m2 = y[n + cell], m3 = y[2 * n + cell];
      const double h1 = lf.h[0], h2 = lf.h[1], h3 = lf.h[2];
      const double mh = m1 * h1 + m2 * h2 + m3 * h3;
      const double g = gate_of(c, cell);
      const double al = alpha_at(&c->p, i);
      ydot[cell]         = g * (c->p.chg * (m3 * h2 - m2 * h3) + al * (h1 - mh * m1));
      ydot[n + cell]     = g * (c->p.chg * (m1 * h3 - m3 * h1) + al * (h2 - mh * m2));
      ydot[2 * n + cell] = g * (c->p.chg * (m2 * h1 - m1 * h2) + al * (h3 - mh * m3));
    }
  }
  return 0;
}

/* dh/dm of the local anisotropy, K (symmetric 3x3): cubic diag(msk_a chk (3m_a^2-1))
 * (2d_i2/precond.cu:177-179), linear chk·msk msk^T (2d_i1/precond.cu:163).  */
static void aniso_jac(const or_ctx* c, const double m[3], const double msk[3], double K[3][3]) {
  for (int a = 0; a < 3; a++)
    for (int b = 0; b < 3; b++) K[a][b] = 0.0;
  if (c->p.aniso_kind == LLG_ANISO_CUBIC) {
    for (int a = 0; a < 3; a++) K[a][a] = msk[a] * c->p.chk * (3.0 * m[a] * m[a] - 1.0);
  } else {
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) K[a][b] = c->p.chk * msk[a] * msk[b];
  }
}

/* LLG_JV_FULL_DEMAG: the field derivative also carries the demag term
 * N ⊛ (w v) (strength-scaled), the part the reference's Jv omits
 * (2d_i2/jtv.h:9-13); h is the full field as in LLG_JV_FULL_FIELD.          */
int or_jtv(or_ctx* c, const double* v, double* Jv, const double* y) {
  const long n = c->ncell;
  const int ng = c->p.ng, ny = c->p.ny;
  const int full = (c->p.jv_mode == LLG_JV_FULL_FIELD || c->p.jv_mode == LLG_JV_FULL_DEMAG);
  double* hv = NULL;
  if (c->p.jv_mode == LLG_JV_FULL_DEMAG && c->dm) {
    hv = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    if (!hv || or_demag_run(c, v, hv) != 0) { free(hv); return -1; }
  }
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < ng; i++) {
      const long cell = (long)j * ng + i;
      if (c->active && !c->active[cell] && !c->w) {
        Jv[cell] = 0.0; Jv[n + cell] = 0.0; Jv[2 * n + cell] = 0.0;
        continue;
      }
      local_field lf;
      field_at(c, y, i, j, full, &lf);
      const double m[3] = {y[cell], y[n + cell], y[2 * n + cell]};
      const double vv[3] = {v[cell], v[n + cell], v[2 * n + cell]};
      double K[3][3];
      aniso_jac(c, m, lf.msk, K);
      double dh[3];
      for (int a = 0; a < 3; a++) {
        const double L = nbv(c, v, a, i - 1, j), R = nbv(c, v, a, i + 1, j);
        const double U = nbv(c, v, a, i, j - 1), D = nbv(c, v, a, i, j + 1);
        const double kv = K[a][0] * vv[0] + K[a][1] * vv[1] + K[a][2] * vv[2];
        dh[a] = c->p.che * (L + R + U + D) + kv + c->p.chb * lf.nsk[a] * (L + R);
        if (hv) dh[a] = dh[a] + hv[a * n + cell];
      }
      const double h1 = lf.h[0], h2 = lf.h[1], h3 = lf.h[2];
      const double m1 = m[0], m2 = m[1], m3 = m[2];
      const double v1 = vv[0], v2 = vv[1], v3 = vv[2];
      const double mh = m1 * h1 + m2 * h2 + m3 * h3;
      const double dmh = (v1 * h1 + v2 * h2 + v3 * h3) + (m1 * dh[0] + m2 * dh[1] + m3 * dh[2]);
      const double g = gate_of(c, cell);
      const double chg = c->p.chg, al = c->p.alpha;
      Jv[cell]         = g * (chg * (v3 * h2 + m3 * dh[1] - v2 * h3 - m2 * dh[2]) + al * (dh[0] - dmh * m1 - mh * v1));
      Jv[n + cell]     = g * (chg * (v1 * h3 + m1 * dh[2] - v3 * h1 - m3 * dh[0]) + al * (dh[1] - dmh * m2 - mh * v2));
      Jv[2 * n + cell] = g * (chg * (v2 * h1 + m2 * dh[0] - v1 * h2 - m1 * dh[1]) + al * (dh[2] - dmh * m3 - mh * v3));
    }
  }
  free(hv);
  return 0;
}

/* Local 3x3 Jacobian of f w.r.t. the cell's own m (neighbours held fixed):
 *   J·d = chg (K d × m + h × d) + alpha (K d − (d·h + m·K d) m − (m·h) d)
 * which for diagonal K is the closed form of 2d_i2/precond.cu:39-50.      */
int or_psetup(or_ctx* c, const double* y, double gamma) {
  const long n = c->ncell;
  const int ng = c->p.ng, ny = c->p.ny;
  double n0[3] = {0.0, 0.0, 0.0};
  or_demag_self(c, n0);
#pragma omp parallel for schedule(static)
  for (int j = 0; j < ny; j++) {
    for (int i = 0; i < ng; i++) {
      const long cell = (long)j * ng + i;
      local_field lf;
      field_at(c, y, i, j, 1, &lf);
      const double m[3] = {y[cell], y[n + cell], y[2 * n + cell]};
      double K[3][3];
      aniso_jac(c, m, lf.msk, K);
      const double ws = c->w ? c->w[cell] : 1.0;
      for (int a = 0; a < 3; a++) K[a][a] += ws * n0[a];
      const double* h = lf.h;
      const double mh = m[0] * h[0] + m[1] * h[1] + m[2] * h[2];
      double e[3];
      for (int b = 0; b < 3; b++) e[b] = h[b] + (K[b][0] * m[0] + K[b][1] * m[1] + K[b][2] * m[2]);
      double J[3][3];
      for (int b = 0; b < 3; b++) {
        const double kb[3] = {K[0][b], K[1][b], K[2][b]};
        /* (K[:,b] × m) and (h × e_b) */
        const double kxm[3] = {kb[1] * m[2] - kb[2] * m[1], kb[2] * m[0] - kb[0] * m[2],
                               kb[0] * m[1] - kb[1] * m[0]};
        double hxe[3] = {0.0, 0.0, 0.0};
        if (b == 0) { hxe[1] = h[2]; hxe[2] = -h[1]; }
        if (b == 1) { hxe[0] = -h[2]; hxe[2] = h[0]; }
        if (b == 2) { hxe[0] = h[1]; hxe[1] = -h[0]; }
        for (int a = 0; a < 3; a++) {
          double dm = c->p.alpha * (kb[a] - e[b] * m[a] - (a == b ? mh : 0.0));
          J[a][b] = ws * (c->p.chg * (kxm[a] + hxe[a]) + dm);
        }
      }
      double A[3][3];
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) A[a][b] = (a == b ? 1.0 : 0.0) - gamma * J[a][b];
      const double c00 = A[1][1] * A[2][2] - A[1][2] * A[2][1];
      const double c10 = A[1][2] * A[2][0] - A[1][0] * A[2][2];
      const double c20 = A[1][0] * A[2][1] - A[1][1] * A[2][0];
      const double det = A[0][0] * c00 + A[0][1] * c10 + A[0][2] * c20;
      double P[9];
      if (!(fabs(det) > 1e-30)) {
        for (int k = 0; k < 9; k++) P[k] = (k % 4 == 0) ? 1.0 : 0.0;
      } else {
        const double id = 1.0 / det;
        P[0] = (A[1][1] * A[2][2] - A[1][2] * A[2][1]) * id;
        P[1] = (A[0][2] * A[2][1] - A[0][1] * A[2][2]) * id;
        P[2] = (A[0][1] * A[1][2] - A[0][2] * A[1][1]) * id;
        P[3] = (A[1][2] * A[2][0] - A[1][0] * A[2][2]) * id;
        P[4] = (A[0][0] * A[2][2] - A[0][2] * A[2][0]) * id;
        P[5] = (A[0][2] * A[1][0] - A[0][0] * A[1][2]) * id;
        P[6] = (A[1][0] * A[2][1] - A[1][1] * A[2][0]) * id;
        P[7] = (A[0][1] * A[2][0] - A[0][0] * A[2][1]) * id;
        P[8] = (A[0][0] * A[1][1] - A[0][1] * A[1][0]) * id;
      }
      for (int k = 0; k < 9; k++) c->pinv[k * n + cell] = P[k];
    }
  }
  return 0;
}

int or_psolve(or_ctx* c, const double* r, double* z) {
  const long n = c->ncell;
  const double* P = c->pinv;
#pragma omp parallel for schedule(static)
  for (long k = 0; k < n; k++) {
    const double r0 = r[k], r1 = r[n + k], r2 = r[2 * n + k];
    double g = 1.0;
    if (c->active && !c->w) g = c->active[k] ? 1.0 : 0.0;
    z[k]         = g * (P[0 * n + k] * r0 + P[1 * n + k] * r1 + P[2 * n + k] * r2);
    z[n + k]     = g * (P[3 * n + k] * r0 + P[4 * n + k] * r1 + P[5 * n + k] * r2);
    z[2 * n + k] = g * (P[6 * n + k] * r0 + P[7 * n + k] * r1 + P[8 * n + k] * r2);
  }
  return 0;
}

const double* or_hdemag(or_ctx* c) { return c->hd; }
const double* or_pinv(or_ctx* c) { return c->pinv; }

or_ctx* or_create(const llg_params* p) {
  if (!p || p->ng <= 0 || p->ny <= 0) return NULL;
  or_ctx* c = (or_ctx*)calloc(1, sizeof(or_ctx));
  if (!c) return NULL;
  c->p = *p;
  c->ncell = (long)p->ng * p->ny;
  c->neq = 3 * c->ncell;
  c->hd = (double*)calloc((size_t)c->neq, sizeof(double));
  c->pinv = (double*)calloc((size_t)9 * c->ncell, sizeof(double));
  if (!c->hd || !c->pinv) { or_destroy(c); return NULL; }
  if (p->demag_mode != LLG_DEMAG_OFF && p->demag_strength > 0.0) {
    c->dm = or_demag_create(p);
    if (!c->dm) { or_destroy(c); return NULL; }
  }
  return c;
}

void or_destroy(or_ctx* c) {
  if (!c) return;
  free(c->active); free(c->w); free(c->msk3); free(c->nsk3);
  free(c->hd); free(c->pinv);
  or_demag_free(c->dm);
  extern void or_bdf_free(or_bdf*);
  or_bdf_free(c->bdf);
  free(c);
}

int or_set_active(or_ctx* c, const uint8_t* active) {
  free(c->active);
  c->active = NULL;
  if (!active) return 0;
  c->active = (uint8_t*)malloc((size_t)c->ncell);
  if (!c->active) return -1;
  memcpy(c->active, active, (size_t)c->ncell);
  return 0;
}

int or_set_window(or_ctx* c, const double* w, const double* msk3, const double* nsk3) {
  free(c->w); free(c->msk3); free(c->nsk3);
  c->w = c->msk3 = c->nsk3 = NULL;
  const size_t n = (size_t)c->ncell;
  if (w) { c->w = (double*)malloc(n * sizeof(double)); memcpy(c->w, w, n * sizeof(double)); }
  if (msk3) { c->msk3 = (double*)malloc(3 * n * sizeof(double)); memcpy(c->msk3, msk3, 3 * n * sizeof(double)); }
  if (nsk3) { c->nsk3 = (double*)malloc(3 * n * sizeof(double)); memcpy(c->nsk3, nsk3, 3 * n * sizeof(double)); }
  return 0;
}

#ifdef _OPENMP
#include <omp.h>
int or_set_threads(int n) { if (n > 0) omp_set_num_threads(n); return omp_get_max_threads(); }
#else
int or_set_threads(int n) { (void)n; return 1; }
#endif
