/*
 * or_bdf.c — CPU restatement of the integrator the reference drives its
 * operators with: SUNDIALS CVODE (BDF, Nordsieck form, orders 1..maxord,
 * variable step), SUNNonlinSol_Newton (max 3 iterations) and SUNLinSol_SPGMR
 * (left preconditioning, maxl Krylov vectors, no restarts), configured as
 * in src/irregular/2d_fft/2d_i2/2d_fft.cu:648-681:
 *     CVodeCreate(CV_BDF); CVodeSVtolerances(rtol, atol); SPGMR(PREC_LEFT,
 *     KRYLOV_DIM); classical Gram–Schmidt if neq < 500000 (else modified);
 *     CVodeSetMaxOrd(MAX_BDF_ORDER); CVode(..., tout, ..., CV_NORMAL).
 * TEST INFRASTRUCTURE ONLY (see oracle.h).
 *
 * SUNDIALS itself is a third-party dependency that is not in the reference
 * tree and is not installed here; its version is not pinned by the
 * reference (Makefile:2 points at /usr/local/sundials; the SUNErrCode return
 * type at deferred_nvector.cu:146 implies SUNDIALS >= 7.0).  The algorithm
 * below follows the published CVODE description (Hindmarsh et al., ACM TOMS
 * 31(3), 2005; CVODE user guide "Mathematical considerations"): fixed-
 * leading-coefficient BDF, local error test with tq[2], order selection
 * from the q-1 / q+1 estimates, Newton convergence rate test (CRDOWN 0.3,
 * RDIV 2), preconditioner refresh every 20 steps or on |gamma ratio-1|>0.3,
 * GMRES tolerance 0.05·tq[4]·sqrt(neq) with ewt scaling on both sides.
 *
 * The RHS may rescale y in place (normalisation inside f); it is always
 * called on the same work vector CVODE passes: zn[0] at start-up and after
 * repeated error-test failures, the y scratch vector otherwise.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "or_internal.h"

#define QMAXL 5
#define MAXLL 16

/* CVODE constants */
#define UROUND      DBL_EPSILON
#define FUZZ_FACTOR 100.0
#define HLB_FACTOR  100.0
#define HUB_FACTOR  0.1
#define H_BIAS      0.5
#define MAX_ITERS   4
#define CORTES      0.1
#define THRESH      1.5
#define ETAMX1      10000.0
#define ETAMX2      10.0
#define ETAMX3      10.0
#define ETAMXF      0.2
#define ETAMIN      0.1
#define ETACF       0.25
#define ADDON       1.0e-6
#define BIAS1       6.0
#define BIAS2       6.0
#define BIAS3       10.0
#define ONEPSM      1.000001
#define SMALL_NST   10
#define MXNCF       10
#define MXNEF       7
#define MXNEF1      3
#define SMALL_NEF   2
#define LONG_WAIT   10
#define NLS_MAXCOR  3
#define CRDOWN      0.3
#define DGMAX       0.3
#define RDIV        2.0
#define MSBP        20
#define LS_EPLIN    0.05
#define LS_MSBJ     51
#define LS_DGMAX    0.2
#define GS_FACTOR   1000.0

/* internal flags */
#define FIRST_CALL      0
#define PREV_CONV_FAIL  1
#define PREV_ERR_FAIL   2
#define DO_ERROR_TEST   3
#define PREDICT_AGAIN   4
#define TRY_AGAIN       5
#define NLS_CONTINUE    901
#define NLS_CONV_RECVR  902
#define CV_NO_FAILURES  0
#define CV_FAIL_BAD_J   1
#define CV_FAIL_OTHER   2
#define LS_SUCCESS      0
#define LS_RES_REDUCED  1
#define LS_CONV_FAIL    2
#define LS_QRSOL_FAIL   3

struct or_bdf {
  or_ctx* c;
  long neq;
  int qmax, maxl, classical_gs, mxstep;
  double rtol, atol;
  double* zn[QMAXL + 1];
  double *ewt, *acor, *y, *tempv, *ftemp, *delta, *lsx;
  double* V[MAXLL + 1];
  double *xcor, *vtemp;
  double Hes[MAXLL + 1][MAXLL], givens[2 * MAXLL], yg[MAXLL + 1];
  double tn, h, hscale, hprime, next_h, eta, etamax, hu, hmin, hmax_inv;
  double etaq, etaqm1, etaqp1;
  int q, qprime, next_q, qwait, L, qu, indx_acor;
  double l[QMAXL + 2], tq[6], tau[QMAXL + 2];
  double gamma, gammap, gamrat, rl1, crate, delp, acnrm, saved_tq5;
  int jcur_nls, jcur, convfail, started, ls_curiter, jbad_ls;
  long nst, nfe, nsetups, nni, ncfn, netf, nli, nlcf, njv, nps, npe, nstlp, nstlj, nscon;
};

/* ── deterministic vector kernels (blocked sums, fixed order) ─────── */
#define RBLK 4096

double or_dot(const double* x, const double* y, long n) {
  const long nb = (n + RBLK - 1) / RBLK;
  double* part = (double*)malloc(sizeof(double) * (size_t)(nb > 0 ? nb : 1));
#pragma omp parallel for schedule(static)
  for (long b = 0; b < nb; b++) {
    double s = 0.0;
    const long e = (b + 1) * RBLK < n ? (b + 1) * RBLK : n;
    for (long i = b * RBLK; i < e; i++) s += x[i] * y[i];
    part[b] = s;
  }
  double s = 0.0;
  for (long b = 0; b < nb; b++) s += part[b];
  free(part);
  return s;
}

double or_wrms(const double* x, const double* w, long n) {
  const long nb = (n + RBLK - 1) / RBLK;
  double* part = (double*)malloc(sizeof(double) * (size_t)(nb > 0 ? nb : 1));
#pragma omp parallel for schedule(static)
  for (long b = 0; b < nb; b++) {
    double s = 0.0;
    const long e = (b + 1) * RBLK < n ? (b + 1) * RBLK : n;
    for (long i = b * RBLK; i < e; i++) { const double p = x[i] * w[i]; s += p * p; }
    part[b] = s;
  }
  double s = 0.0;
  for (long b = 0; b < nb; b++) s += part[b];
  free(part);
  return sqrt(s / (double)n);
}

static void vlin(double a, const double* x, double b, const double* y, double* z, long n) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) z[i] = a * x[i] + b * y[i];
}
static void vscale(double a, const double* x, double* z, long n) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) z[i] = a * x[i];
}
static void vconst(double a, double* z, long n) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) z[i] = a;
}
static void vprod(const double* x, const double* y, double* z, long n) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) z[i] = x[i] * y[i];
}
static void vdiv(const double* x, const double* y, double* z, long n) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) z[i] = x[i] / y[i];
}
/* z = c[0] X[0]; z = c[k] X[k] + z (N_VLinearCombination without a fused op) */
static void vlincomb(int nv, const double* c, double* const* X, double* z, long n) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++) {
    double s = c[0] * X[0][i];
    for (int k = 1; k < nv; k++) s = c[k] * X[k][i] + s;
    z[i] = s;
  }
}
static double vmaxnorm(const double* x, long n) {
  double m = 0.0;
  for (long i = 0; i < n; i++) { const double a = fabs(x[i]); if (a > m) m = a; }
  return m;
}

static double powi(double b, int e) {
  double p = 1.0;
  for (int i = 1; i <= (e < 0 ? -e : e); i++) p *= b;
  return e < 0 ? 1.0 / p : p;
}
static double powr(double b, double e) { return (b <= 0.0) ? 0.0 : pow(b, e); }

/* ewt = 1/(rtol |y| + atol); -1 if any denominator <= 0 (cvEwtSetSV) */
static int set_ewt(or_bdf* b, const double* ycur) {
  const long n = b->neq;
  int bad = 0;
  for (long i = 0; i < n; i++) {
    const double t = b->rtol * fabs(ycur[i]) + b->atol;
    if (t <= 0.0) bad = 1;   /* a NaN state is left to the WRMS-norm check */
    b->ewt[i] = 1.0 / t;
  }
  return bad ? -1 : 0;
}

/* ── physics bridge ─────────────────────────────────────────────────── */
static int call_f(or_bdf* b, double t, double* y, double* ydot) {
  b->nfe++;
  return or_rhs(b->c, t, y, ydot);
}

/* ── SPGMR (left preconditioning, s1 = s2 = ewt, no restarts) ───────── */
static int atimes(or_bdf* b, const double* v, double* z) {
  or_jtv(b->c, v, z, b->y);
  b->njv++;
  vlin(1.0, v, -b->gamma, z, z, b->neq);
  return 0;
}
static int psolve(or_bdf* b, const double* r, double* z) {
  b->nps++;
  return or_psolve(b->c, r, z);
}

static int qr_fact(int n, double (*h)[MAXLL], double* q) {
  const int n1 = n - 1;
  int code = 0;
  for (int k = 0; k < n1; k++) {
    const int i = 2 * k;
    const double t1 = h[k][n1], t2 = h[k + 1][n1];
    const double c = q[i], s = q[i + 1];
    h[k][n1] = c * t1 - s * t2;
    h[k + 1][n1] = s * t1 + c * t2;
  }
  const double t1 = h[n1][n1], t2 = h[n][n1];
  double c, s;
  if (t2 == 0.0) { c = 1.0; s = 0.0; }
  else if (fabs(t2) >= fabs(t1)) { const double t3 = t1 / t2; s = -1.0 / sqrt(1.0 + t3 * t3); c = -s * t3; }
  else { const double t3 = t2 / t1; c = 1.0 / sqrt(1.0 + t3 * t3); s = -c * t3; }
  q[2 * n1] = c;
  q[2 * n1 + 1] = s;
  if ((h[n1][n1] = c * t1 - s * t2) == 0.0) code = n;
  return code;
}

static int qr_sol(int n, double (*h)[MAXLL], const double* q, double* bb) {
  int code = 0;
  for (int k = 0; k < n; k++) {
    const double c = q[2 * k], s = q[2 * k + 1];
    const double t1 = bb[k], t2 = bb[k + 1];
    bb[k] = c * t1 - s * t2;
    bb[k + 1] = s * t1 + c * t2;
  }
  for (int k = n - 1; k >= 0; k--) {
    if (h[k][k] == 0.0) { code = k + 1; break; }
    bb[k] /= h[k][k];
    for (int i = 0; i < k; i++) bb[i] -= bb[k] * h[i][k];
  }
  return code;
}

/* Gram–Schmidt of V[k] against V[0..k-1]; returns the new norm. */
static double gram_schmidt(or_bdf* b, int k) {
  const long n = b->neq;
  double** V = b->V;
  if (b->classical_gs) {
    double dots[MAXLL + 1];
    for (int i = 0; i <= k; i++) dots[i] = or_dot(V[k], V[i], n);
    const double vk_norm = sqrt(dots[k]);
    double cf[MAXLL + 1];
    double* X[MAXLL + 1];
    cf[0] = 1.0; X[0] = V[k];
    for (int i = 0; i < k; i++) { b->Hes[i][k - 1] = dots[i]; cf[i + 1] = -dots[i]; X[i + 1] = V[i]; }
    vlincomb(k + 1, cf, X, V[k], n);
    double nrm = sqrt(or_dot(V[k], V[k], n));
    if (GS_FACTOR * nrm < vk_norm) {
      for (int i = 0; i < k; i++) dots[i] = or_dot(V[k], V[i], n);
      cf[0] = 1.0; X[0] = V[k];
      for (int i = 0; i < k; i++) { b->Hes[i][k - 1] += dots[i]; cf[i + 1] = -dots[i]; X[i + 1] = V[i]; }
      vlincomb(k + 1, cf, X, V[k], n);
      nrm = sqrt(or_dot(V[k], V[k], n));
    }
    return nrm;
  }
  const double vk_norm = sqrt(or_dot(V[k], V[k], n));
  for (int i = 0; i < k; i++) {
    b->Hes[i][k - 1] = or_dot(V[i], V[k], n);
    vlin(1.0, V[k], -b->Hes[i][k - 1], V[i], V[k], n);
  }
  double nrm = sqrt(or_dot(V[k], V[k], n));
  double temp = GS_FACTOR * vk_norm;
  if ((temp + nrm) != temp) return nrm;
  double nn2 = 0.0;
  for (int i = 0; i < k; i++) {
    const double np = or_dot(V[i], V[k], n);
    temp = GS_FACTOR * b->Hes[i][k - 1];
    if ((temp + np) == temp) continue;
    b->Hes[i][k - 1] += np;
    vlin(1.0, V[k], -np, V[i], V[k], n);
    nn2 += np * np;
  }
  if (nn2 != 0.0) {
    const double t = nrm * nrm - nn2;
    nrm = (t > 0.0) ? sqrt(t) : 0.0;
  }
  return nrm;
}

/* Solve (I - gamma J) x = rhs; x returned in rhs.  Returns LS_* code and
 * adds the iteration count to nli. */
static int spgmr(or_bdf* b, double* rhs, double delta) {
  const long n = b->neq;
  double** V = b->V;
  const int lmax = b->maxl;
  int nli = 0, krydim = 0, converged = 0;
  /* r0 = b (zero guess) */
  memcpy(V[0], rhs, sizeof(double) * (size_t)n);
  psolve(b, V[0], b->vtemp);
  vprod(b->ewt, b->vtemp, V[0], n);
  const double beta = sqrt(or_dot(V[0], V[0], n));
  double rnorm = beta, rho = beta;
  if (rnorm <= delta) { vconst(0.0, rhs, n); return LS_SUCCESS; }
  vconst(0.0, b->xcor, n);
  for (int i = 0; i <= lmax; i++)
    for (int j = 0; j < lmax; j++) b->Hes[i][j] = 0.0;
  double rot = 1.0;
  vscale(1.0 / rnorm, V[0], V[0], n);
  for (int l = 0; l < lmax; l++) {
    nli++;
    krydim = l + 1;
    vdiv(V[l], b->ewt, b->vtemp, n);
    atimes(b, b->vtemp, V[l + 1]);
    psolve(b, V[l + 1], b->vtemp);
    vprod(b->ewt, b->vtemp, V[l + 1], n);
    b->Hes[l + 1][l] = gram_schmidt(b, l + 1);
    if (qr_fact(krydim, b->Hes, b->givens) != 0) { b->nli += nli; return LS_CONV_FAIL; }
    rot *= b->givens[2 * l + 1];
    rho = fabs(rot * rnorm);
    if (rho <= delta) { converged = 1; break; }
    vscale(1.0 / b->Hes[l + 1][l], V[l + 1], V[l + 1], n);
  }
  b->nli += nli;
  b->yg[0] = rnorm;
  for (int i = 1; i <= krydim; i++) b->yg[i] = 0.0;
  if (qr_sol(krydim, b->Hes, b->givens, b->yg) != 0) return LS_QRSOL_FAIL;
  {
    double cf[MAXLL + 1];
    double* X[MAXLL + 1];
    cf[0] = 1.0; X[0] = b->xcor;
    for (int k = 0; k < krydim; k++) { cf[k + 1] = b->yg[k]; X[k + 1] = V[k]; }
    vlincomb(krydim + 1, cf, X, b->xcor, n);
  }
  if (converged || rho < beta) {
    vdiv(b->xcor, b->ewt, rhs, n);
    return converged ? LS_SUCCESS : LS_RES_REDUCED;
  }
  return LS_CONV_FAIL;
}

/* ── CVODE pieces ───────────────────────────────────────────────────── */
static void set_bdf(or_bdf* b) {
  double alpha0, alpha0_hat, xi_inv, xistar_inv, hsum;
  const int q = b->q;
  b->l[0] = b->l[1] = xi_inv = xistar_inv = 1.0;
  for (int i = 2; i <= q; i++) b->l[i] = 0.0;
  alpha0 = alpha0_hat = -1.0;
  hsum = b->h;
  if (q > 1) {
    for (int j = 2; j < q; j++) {
      hsum += b->tau[j - 1];
      xi_inv = b->h / hsum;
      alpha0 -= 1.0 / j;
      for (int i = j; i >= 1; i--) b->l[i] += b->l[i - 1] * xi_inv;
    }
    alpha0 -= 1.0 / q;
    xistar_inv = -b->l[1] - alpha0;
    hsum += b->tau[q - 1];
    xi_inv = b->h / hsum;
    alpha0_hat = -b->l[1] - xi_inv;
    for (int i = q; i >= 1; i--) b->l[i] += b->l[i - 1] * xistar_inv;
  }
  /* test quantities */
  const double A1 = 1.0 - alpha0_hat + alpha0;
  const double A2 = 1.0 + q * A1;
  b->tq[2] = fabs(A1 / (alpha0 * A2));
  b->tq[5] = fabs(A2 * xistar_inv / (b->l[q] * xi_inv));
  if (b->qwait == 1) {
    if (q > 1) {
      const double C = xistar_inv / b->l[q];
      const double A3 = alpha0 + 1.0 / q;
      const double A4 = alpha0_hat + xi_inv;
      const double Cpinv = (1.0 - A4 + A3) / A3;
      b->tq[1] = fabs(C * Cpinv);
    } else {
      b->tq[1] = 1.0;
    }
    hsum += b->tau[q];
    xi_inv = b->h / hsum;
    const double A5 = alpha0 - (1.0 / (q + 1));
    const double A6 = alpha0_hat - xi_inv;
    const double Cppinv = (1.0 - A6 + A5) / A2;
    b->tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
  }
  b->tq[4] = CORTES / b->tq[2];
}

static void cv_set(or_bdf* b) {
  set_bdf(b);
  b->rl1 = 1.0 / b->l[1];
  b->gamma = b->h * b->rl1;
  if (b->nst == 0) b->gammap = b->gamma;
  b->gamrat = (b->nst > 0) ? b->gamma / b->gammap : 1.0;
}

/* Pascal-triangle predictor, element by element (same operations as the
 * q(q+1)/2 sequential N_VLinearSum calls). */
static void predict(or_bdf* b) {
  b->tn += b->h;
  const int q = b->q;
  const long n = b->neq;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++)
    for (int k = 1; k <= q; k++)
      for (int j = q; j >= k; j--) b->zn[j - 1][i] = b->zn[j - 1][i] + b->zn[j][i];
}

static void restore(or_bdf* b, double saved_t) {
  b->tn = saved_t;
  const int q = b->q;
  const long n = b->neq;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; i++)
    for (int k = 1; k <= q; k++)
      for (int j = q; j >= k; j--) b->zn[j - 1][i] = b->zn[j - 1][i] - b->zn[j][i];
}

static void rescale(or_bdf* b) {
  double factor = b->eta;
  for (int j = 1; j <= b->q; j++) {
    vscale(factor, b->zn[j], b->zn[j], b->neq);
    factor *= b->eta;
  }
  b->h = b->hscale * b->eta;
  b->next_h = b->h;
  b->hscale = b->h;
  b->nscon = 0;
}

static void increase_bdf(or_bdf* b) {
  double alpha0, alpha1, prod, xi, xiold, hsum, A1;
  for (int i = 0; i <= b->qmax; i++) b->l[i] = 0.0;
  b->l[2] = alpha1 = prod = xiold = 1.0;
  alpha0 = -1.0;
  hsum = b->hscale;
  if (b->q > 1) {
    for (int j = 1; j < b->q; j++) {
      hsum += b->tau[j + 1];
      xi = hsum / b->hscale;
      prod *= xi;
      alpha0 -= 1.0 / (j + 1);
      alpha1 += 1.0 / xi;
      for (int i = j + 2; i >= 2; i--) b->l[i] = b->l[i] * xiold + b->l[i - 1];
      xiold = xi;
    }
  }
  A1 = (-alpha0 - alpha1) / prod;
  const long n = b->neq;
  vscale(A1, b->zn[b->indx_acor], b->zn[b->L], n);
  for (int j = 2; j <= b->q; j++) vlin(b->l[j], b->zn[b->L], 1.0, b->zn[j], b->zn[j], n);
}

static void decrease_bdf(or_bdf* b) {
  double hsum, xi;
  for (int i = 0; i <= b->qmax; i++) b->l[i] = 0.0;
  b->l[2] = 1.0;
  hsum = 0.0;
  for (int j = 1; j <= b->q - 2; j++) {
    hsum += b->tau[j];
    xi = hsum / b->hscale;
    for (int i = j + 2; i >= 2; i--) b->l[i] = b->l[i] * xi + b->l[i - 1];
  }
  for (int j = 2; j < b->q; j++) vlin(-b->l[j], b->zn[b->q], 1.0, b->zn[j], b->zn[j], b->neq);
}

static void adjust_order(or_bdf* b, int dq) {
  if (b->q == 2 && dq != 1) return;
  if (dq == 1) increase_bdf(b);
  else if (dq == -1) decrease_bdf(b);
}

static void adjust_params(or_bdf* b) {
  if (b->qprime != b->q) {
    adjust_order(b, b->qprime - b->q);
    b->q = b->qprime;
    b->L = b->q + 1;
    b->qwait = b->L;
  }
  rescale(b);
}

/* Newton residual: y = zn0 + ycor; ftemp = f(tn, y); res = rl1 zn1 + ycor - gamma ftemp */
static int nls_residual(or_bdf* b, const double* ycor, double* res) {
  const long n = b->neq;
  vlin(1.0, b->zn[0], 1.0, ycor, b->y, n);
  const int r = call_f(b, b->tn, b->y, b->ftemp);
  if (r < 0) return LLG_CV_RHSFUNC_FAIL;
  if (r > 0) return 1;
  vlin(b->rl1, b->zn[1], 1.0, ycor, res, n);
  vlin(-b->gamma, b->ftemp, 1.0, res, res, n);
  return 0;
}

static int nls_lsetup(or_bdf* b, int jbad) {
  if (jbad) b->convfail = CV_FAIL_BAD_J;
  /* cvLsSetup: jbad heuristics for the (matrix-free) preconditioner */
  const double dgamma = fabs(b->gamma / b->gammap - 1.0);
  const int ls_jbad = (b->nst == 0) || (b->nst >= b->nstlj + LS_MSBJ) ||
                      ((b->convfail == CV_FAIL_BAD_J) && (dgamma < LS_DGMAX)) ||
                      (b->convfail == CV_FAIL_OTHER);
  b->jbad_ls = ls_jbad;
  int jcur = ls_jbad;
  const int r = or_psetup(b->c, b->y, b->gamma); /* block-Jacobi always rebuilds */
  jcur = 1;
  b->npe++;
  b->nstlj = b->nst;
  b->jcur = jcur;
  b->nsetups++;
  b->jcur_nls = b->jcur;
  b->gamrat = 1.0;
  b->gammap = b->gamma;
  b->crate = 1.0;
  b->nstlp = b->nst;
  if (r < 0) return LLG_CV_LSETUP_FAIL;
  if (r > 0) return 1;
  return 0;
}

static int nls_lsolve(or_bdf* b, double* del) {
  const double deltar = LS_EPLIN * b->tq[4];
  const double delta = deltar * sqrt((double)b->neq);
  const int r = spgmr(b, del, delta);
  if (r != LS_SUCCESS) b->nlcf++;
  if (r == LS_SUCCESS) return 0;
  if (r == LS_RES_REDUCED) return (b->ls_curiter == 0) ? 0 : 1;
  return 1;
}

static int nls_ctest(or_bdf* b, const double* ycor, const double* del, double tol, int m) {
  const double dn = or_wrms(del, b->ewt, b->neq);
  if (m > 0) {
    const double r = dn / b->delp;
    b->crate = (CRDOWN * b->crate > r) ? CRDOWN * b->crate : r;
  }
  const double dcon = dn * (b->crate < 1.0 ? b->crate : 1.0) / tol;
  if (dcon <= 1.0) {
    b->acnrm = (m == 0) ? dn : or_wrms(ycor, b->ewt, b->neq);
    return 0;
  }
  if ((m >= 1) && (dn > RDIV * b->delp)) return NLS_CONV_RECVR;
  b->delp = dn;
  return NLS_CONTINUE;
}

static int newton(or_bdf* b, int call_setup) {
  double* ycor = b->acor;
  double* del = b->delta;
  int jbad = 0, retval = 0;
  for (;;) {
    retval = nls_residual(b, ycor, del);
    if (retval != 0) break;
    if (call_setup) {
      retval = nls_lsetup(b, jbad);
      if (retval != 0) break;
    }
    int m = 0;
    for (;;) {
      b->nni++;
      vscale(-1.0, del, del, b->neq);
      b->ls_curiter = m;
      retval = nls_lsolve(b, del);
      if (retval != 0) break;
      vlin(1.0, ycor, 1.0, del, ycor, b->neq);
      retval = nls_ctest(b, ycor, del, b->tq[4], m);
      if (retval == 0) { b->jcur_nls = 0; return 0; }
      if (retval != NLS_CONTINUE) break;
      m++;
      if (m >= NLS_MAXCOR) { retval = NLS_CONV_RECVR; break; }
      retval = nls_residual(b, ycor, del);
      if (retval != 0) break;
    }
    if (retval > 0 && !b->jcur_nls) {
      call_setup = 1;
      jbad = 1;
      vconst(0.0, ycor, b->neq);
      continue;
    }
    break;
  }
  return retval;
}

static int cv_nls(or_bdf* b, int nflag) {
  b->convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL)) ? CV_NO_FAILURES : CV_FAIL_OTHER;
  const int call_setup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL) || (b->nst == 0) ||
                         (b->nst >= b->nstlp + MSBP) || (fabs(b->gamrat - 1.0) > DGMAX);
  vconst(0.0, b->acor, b->neq);
  const int flag = newton(b, call_setup);
  vlin(1.0, b->zn[0], 1.0, b->acor, b->y, b->neq);
  if (flag != 0) return flag;
  b->jcur = 0;
  return 0;
}

static int handle_nflag(or_bdf* b, int* nflag, double saved_t, int* ncf) {
  if (*nflag == 0) return DO_ERROR_TEST;
  b->ncfn++;
  restore(b, saved_t);
  if (*nflag < 0) return *nflag;
  (*ncf)++;
  b->etamax = 1.0;
  if ((fabs(b->h) <= b->hmin * ONEPSM) || (*ncf == MXNCF)) return LLG_CV_CONV_FAILURE;
  b->eta = (ETACF > b->hmin / fabs(b->h)) ? ETACF : b->hmin / fabs(b->h);
  *nflag = PREV_CONV_FAIL;
  rescale(b);
  return PREDICT_AGAIN;
}

static int error_test(or_bdf* b, int* nflag, double saved_t, int* nef, double* dsmp) {
  const double dsm = b->acnrm * b->tq[2];
  *dsmp = dsm;
  if (dsm <= 1.0) return 0;
  (*nef)++;
  b->netf++;
  *nflag = PREV_ERR_FAIL;
  restore(b, saved_t);
  if ((fabs(b->h) <= b->hmin * ONEPSM) || (*nef == MXNEF)) return LLG_CV_ERR_FAILURE;
  b->etamax = 1.0;
  if (*nef <= MXNEF1) {
    double eta = 1.0 / (powr(BIAS2 * dsm, 1.0 / b->L) + ADDON);
    const double lo = b->hmin / fabs(b->h);
    eta = (eta > lo) ? eta : lo;
    eta = (eta > ETAMIN) ? eta : ETAMIN;
    if (*nef >= SMALL_NEF) eta = (eta < ETAMXF) ? eta : ETAMXF;
    b->eta = eta;
    rescale(b);
    return TRY_AGAIN;
  }
  if (b->q > 1) {
    b->eta = (ETAMIN > b->hmin / fabs(b->h)) ? ETAMIN : b->hmin / fabs(b->h);
    adjust_order(b, -1);
    b->L = b->q;
    b->q--;
    b->qwait = b->L;
    rescale(b);
    return TRY_AGAIN;
  }
  b->eta = (ETAMIN > b->hmin / fabs(b->h)) ? ETAMIN : b->hmin / fabs(b->h);
  b->h *= b->eta;
  b->next_h = b->h;
  b->hscale = b->h;
  b->qwait = LONG_WAIT;
  b->nscon = 0;
  const int r = call_f(b, b->tn, b->zn[0], b->tempv);
  if (r < 0) return LLG_CV_RHSFUNC_FAIL;
  vscale(b->h, b->tempv, b->zn[1], b->neq);
  return TRY_AGAIN;
}

static void complete_step(or_bdf* b) {
  b->nst++;
  b->nscon++;
  b->hu = b->h;
  b->qu = b->q;
  for (int i = b->q; i >= 2; i--) b->tau[i] = b->tau[i - 1];
  if ((b->q == 1) && (b->nst > 1)) b->tau[2] = b->tau[1];
  b->tau[1] = b->h;
  const long n = b->neq;
  for (int j = 0; j <= b->q; j++) vlin(b->l[j], b->acor, 1.0, b->zn[j], b->zn[j], n);
  b->qwait--;
  if ((b->qwait == 1) && (b->q != b->qmax)) {
    memcpy(b->zn[b->qmax], b->acor, sizeof(double) * (size_t)n);
    b->saved_tq5 = b->tq[5];
    b->indx_acor = b->qmax;
  }
}

static void set_eta(or_bdf* b) {
  if (b->eta < THRESH) {
    b->eta = 1.0;
    b->hprime = b->h;
  } else {
    b->eta = (b->eta < b->etamax) ? b->eta : b->etamax;
    const double d = fabs(b->h) * b->hmax_inv * b->eta;
    b->eta /= (d > 1.0 ? d : 1.0);
    b->hprime = b->h * b->eta;
    if (b->qprime < b->q) b->nscon = 0;
  }
}

static double eta_qm1(or_bdf* b) {
  if (b->q > 1) {
    const double ddn = or_wrms(b->zn[b->q], b->ewt, b->neq) * b->tq[1];
    return 1.0 / (powr(BIAS1 * ddn, 1.0 / b->q) + ADDON);
  }
  return 0.0;
}

static double eta_qp1(or_bdf* b) {
  if (b->q != b->qmax) {
    if (b->saved_tq5 == 0.0) return 0.0;
    const double cquot = (b->tq[5] / b->saved_tq5) * powi(b->h / b->tau[2], b->L);
    vlin(-cquot, b->zn[b->qmax], 1.0, b->acor, b->tempv, b->neq);
    const double dup = or_wrms(b->tempv, b->ewt, b->neq) * b->tq[3];
    return 1.0 / (powr(BIAS3 * dup, 1.0 / (b->L + 1)) + ADDON);
  }
  return 0.0;
}

static void choose_eta(or_bdf* b) {
  double etam = b->etaqm1 > b->etaq ? b->etaqm1 : b->etaq;
  etam = etam > b->etaqp1 ? etam : b->etaqp1;
  if (etam < THRESH) { b->eta = 1.0; b->qprime = b->q; return; }
  if (etam == b->etaq) { b->eta = b->etaq; b->qprime = b->q; }
  else if (etam == b->etaqm1) { b->eta = b->etaqm1; b->qprime = b->q - 1; }
  else {
    b->eta = b->etaqp1;
    b->qprime = b->q + 1;
    memcpy(b->zn[b->qmax], b->acor, sizeof(double) * (size_t)b->neq);
  }
}

static void prepare_next(or_bdf* b, double dsm) {
  if (b->etamax == 1.0) {
    b->qwait = b->qwait > 2 ? b->qwait : 2;
    b->qprime = b->q;
    b->hprime = b->h;
    b->eta = 1.0;
    return;
  }
  b->etaq = 1.0 / (powr(BIAS2 * dsm, 1.0 / b->L) + ADDON);
  if (b->qwait != 0) {
    b->eta = b->etaq;
    b->qprime = b->q;
    set_eta(b);
    return;
  }
  b->qwait = 2;
  b->etaqm1 = eta_qm1(b);
  b->etaqp1 = eta_qp1(b);
  choose_eta(b);
  set_eta(b);
}

static int cv_step(or_bdf* b) {
  const double saved_t = b->tn;
  int ncf = 0, nef = 0, nflag = FIRST_CALL;
  double dsm = 0.0;
  if ((b->nst > 0) && (b->hprime != b->h)) adjust_params(b);
  for (;;) {
    predict(b);
    cv_set(b);
    nflag = cv_nls(b, nflag);
    const int kflag = handle_nflag(b, &nflag, saved_t, &ncf);
    if (kflag == PREDICT_AGAIN) continue;
    if (kflag != DO_ERROR_TEST) return kflag;
    const int eflag = error_test(b, &nflag, saved_t, &nef, &dsm);
    if (eflag == TRY_AGAIN) continue;
    if (eflag != 0) return eflag;
    break;
  }
  complete_step(b);
  prepare_next(b, dsm);
  b->etamax = (b->nst <= SMALL_NST) ? ETAMX2 : ETAMX3;
  vscale(b->tq[2], b->acor, b->acor, b->neq);
  return 0;
}

/* y(t) = sum_{j=q..0} s^j zn[j], s = (t - tn)/h (CVodeGetDky, k = 0) */
static int get_dky(or_bdf* b, double t, double* dky) {
  double tfuzz = FUZZ_FACTOR * UROUND * (fabs(b->tn) + fabs(b->hu));
  if (b->hu < 0.0) tfuzz = -tfuzz;
  const double tp = b->tn - b->hu - tfuzz;
  const double tn1 = b->tn + tfuzz;
  if ((t - tp) * (t - tn1) > 0.0) return LLG_CV_ILL_INPUT;
  const double s = (t - b->tn) / b->h;
  double cf[QMAXL + 1];
  double* X[QMAXL + 1];
  int nv = 0;
  for (int j = b->q; j >= 0; j--) {
    double cc = 1.0;
    for (int i = 0; i < j; i++) cc *= s;
    cf[nv] = cc;
    X[nv] = b->zn[j];
    nv++;
  }
  vlincomb(nv, cf, X, dky, b->neq);
  return 0;
}

static int y_dd_norm(or_bdf* b, double hg, double* yddnrm) {
  const long n = b->neq;
  vlin(hg, b->zn[1], 1.0, b->zn[0], b->y, n);
  const int r = call_f(b, b->tn + hg, b->y, b->tempv);
  if (r < 0) return LLG_CV_RHSFUNC_FAIL;
  if (r > 0) return 1;
  vlin(1.0, b->tempv, -1.0, b->zn[1], b->tempv, n);
  vscale(1.0 / hg, b->tempv, b->tempv, n);
  *yddnrm = or_wrms(b->tempv, b->ewt, n);
  return 0;
}

static double upper_bound_h0(or_bdf* b, double tdist) {
  const long n = b->neq;
  double* t1 = b->tempv;
  double* t2 = b->acor;
  for (long i = 0; i < n; i++) t2[i] = fabs(b->zn[0][i]);
  for (long i = 0; i < n; i++) t1[i] = 1.0 / (1.0 / (b->rtol * fabs(b->zn[0][i]) + b->atol));
  vlin(HUB_FACTOR, t2, 1.0, t1, t1, n);
  for (long i = 0; i < n; i++) t2[i] = fabs(b->zn[1][i]);
  vdiv(t2, t1, t1, n);
  const double hub_inv = vmaxnorm(t1, n);
  double hub = HUB_FACTOR * tdist;
  if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
  return hub;
}

static int h_in(or_bdf* b, double tout) {
  const double tdiff = tout - b->tn;
  if (tdiff == 0.0) return LLG_CV_TOO_CLOSE;
  const int sign = (tdiff > 0.0) ? 1 : -1;
  const double tdist = fabs(tdiff);
  const double tround = UROUND * (fabs(b->tn) > fabs(tout) ? fabs(b->tn) : fabs(tout));
  if (tdist < 2.0 * tround) return LLG_CV_TOO_CLOSE;
  const double hlb = HLB_FACTOR * tround;
  const double hub = upper_bound_h0(b, tdist);
  double hg = sqrt(hlb * hub);
  if (hub < hlb) { b->h = (sign == -1) ? -hg : hg; return 0; }
  double hnew = hg;
  for (int count1 = 1; count1 <= MAX_ITERS; count1++) {
    int hgok = 0;
    double yddnrm = 0.0;
    for (int count2 = 1; count2 <= MAX_ITERS; count2++) {
      const double hgs = hg * sign;
      const int r = y_dd_norm(b, hgs, &yddnrm);
      if (r < 0) return r;
      if (r == 0) { hgok = 1; break; }
      hg *= 0.2;
    }
    if (!hgok) { if (count1 <= 2) return LLG_CV_RHSFUNC_FAIL; hnew = hg; break; }
    hnew = (yddnrm * hub * hub > 2.0) ? sqrt(2.0 / yddnrm) : sqrt(hg * hub);
    if (count1 == MAX_ITERS) break;
    const double hrat = hnew / hg;
    if ((hrat > 0.5) && (hrat < 2.0)) break;
    if ((count1 > 1) && (hrat > 2.0)) { hnew = hg; break; }
    hg = hnew;
  }
  double h0 = H_BIAS * hnew;
  if (h0 < hlb) h0 = hlb;
  if (h0 > hub) h0 = hub;
  if (sign == -1) h0 = -h0;
  b->h = h0;
  return 0;
}

void or_bdf_free(or_bdf* b) {
  if (!b) return;
  for (int j = 0; j <= QMAXL; j++) free(b->zn[j]);
  free(b->ewt); free(b->acor); free(b->y); free(b->tempv); free(b->ftemp); free(b->delta);
  for (int j = 0; j <= MAXLL; j++) free(b->V[j]);
  free(b->xcor); free(b->vtemp);
  free(b);
}

int or_integrator_init(or_ctx* c, double t0, const double* y0, const llg_solver_opts* o) {
  if (!c || !y0 || !o) return LLG_ERR_ARG;
  or_bdf_free(c->bdf);
  or_bdf* b = (or_bdf*)calloc(1, sizeof(or_bdf));
  if (!b) return LLG_ERR_NOMEM;
  b->c = c;
  b->neq = c->neq;
  b->qmax = (o->maxord >= 1 && o->maxord <= QMAXL) ? o->maxord : QMAXL;
  b->maxl = (o->maxl > 0) ? o->maxl : 5;
  if (b->maxl > MAXLL) b->maxl = MAXLL;
  b->classical_gs = (o->gs_type == LLG_GS_CLASSICAL) || (o->gs_type == LLG_GS_AUTO && b->neq < 500000);
  b->mxstep = (o->mxstep > 0) ? o->mxstep : 500;
  b->rtol = o->rtol;
  b->atol = o->atol;
  const size_t vb = sizeof(double) * (size_t)b->neq;
  for (int j = 0; j <= b->qmax; j++) b->zn[j] = (double*)calloc(1, vb);
  b->ewt = (double*)calloc(1, vb); b->acor = (double*)calloc(1, vb); b->y = (double*)calloc(1, vb);
  b->tempv = (double*)calloc(1, vb); b->ftemp = (double*)calloc(1, vb); b->delta = (double*)calloc(1, vb);
  for (int j = 0; j <= b->maxl; j++) b->V[j] = (double*)calloc(1, vb);
  b->xcor = (double*)calloc(1, vb); b->vtemp = (double*)calloc(1, vb);
  memcpy(b->zn[0], y0, vb);
  b->tn = t0;
  b->q = 1; b->L = 2; b->qwait = b->L; b->etamax = ETAMX1;
  b->qu = 0; b->hu = 0.0; b->hmin = 0.0; b->hmax_inv = 0.0;
  b->crate = 1.0; b->indx_acor = b->qmax;
  c->bdf = b;
  return 0;
}

int or_integrate(or_ctx* c, double tout, double* yout, double* tret) {
  or_bdf* b = c ? c->bdf : NULL;
  if (!b) return LLG_ERR_STATE;
  const long n = b->neq;
  if (!b->started) {
    if (set_ewt(b, b->zn[0]) != 0) return LLG_CV_ILL_INPUT;
    const int r = call_f(b, b->tn, b->zn[0], b->zn[1]);
    if (r != 0) return LLG_CV_RHSFUNC_FAIL;
    const int hr = h_in(b, tout);
    if (hr != 0) return hr;
    b->hscale = b->h;
    b->hprime = b->h;
    vscale(b->h, b->zn[1], b->zn[1], n);
    b->started = 1;
  } else {
    if ((b->tn - tout) * b->h >= 0.0) {
      *tret = tout;
      return get_dky(b, tout, yout);
    }
  }
  int nstloc = 0;
  for (;;) {
    b->next_h = b->h;
    b->next_q = b->q;
    if (b->nst > 0) {
      if (set_ewt(b, b->zn[0]) != 0) {
        memcpy(yout, b->zn[0], sizeof(double) * (size_t)n);
        *tret = b->tn;
        return LLG_CV_ILL_INPUT;
      }
    }
    if ((b->mxstep > 0) && (nstloc >= b->mxstep)) {
      memcpy(yout, b->zn[0], sizeof(double) * (size_t)n);
      *tret = b->tn;
      return LLG_CV_TOO_MUCH_WORK;
    }
    const double nrm = or_wrms(b->zn[0], b->ewt, n);
    if (!isfinite(nrm)) {
      memcpy(yout, b->zn[0], sizeof(double) * (size_t)n);
      *tret = b->tn;
      return LLG_CV_BAD_STATE;
    }
    if (UROUND * nrm > 1.0) {
      memcpy(yout, b->zn[0], sizeof(double) * (size_t)n);
      *tret = b->tn;
      return LLG_CV_TOO_MUCH_ACC;
    }
    const int kflag = cv_step(b);
    if (kflag != 0) {
      memcpy(yout, b->zn[0], sizeof(double) * (size_t)n);
      *tret = b->tn;
      return kflag;
    }
    nstloc++;
    if ((b->tn - tout) * b->h >= 0.0) {
      *tret = tout;
      get_dky(b, tout, yout);
      b->next_q = b->qprime;
      b->next_h = b->hprime;
      break;
    }
  }
  return 0;
}

int or_get_stats(or_ctx* c, llg_stats* st) {
  if (!c || !st) return LLG_ERR_ARG;
  memset(st, 0, sizeof(*st));
  or_bdf* b = c->bdf;
  if (!b) return 0;
  st->nst = b->nst; st->nfe = b->nfe; st->nsetups = b->nsetups; st->nni = b->nni;
  st->ncfn = b->ncfn; st->netf = b->netf; st->nli = b->nli; st->nlcf = b->nlcf;
  st->njvevals = b->njv; st->npsolves = b->nps; st->npe = b->npe;
  st->qlast = b->qu; st->qcur = b->next_q; st->hlast = b->hu; st->hcur = b->next_h; st->tcur = b->tn;
  return 0;
}
