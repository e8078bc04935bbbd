// integrator.cu — BDF (Nordsieck, orders 1..5) + Newton + left-preconditioned
// SPGMR over device-resident vectors.
//
// This is the integrator the reference drives its callbacks with, SUNDIALS
// CVODE configured as in src/irregular/2d_fft/2d_i2/2d_fft.cu:648-681
// (CV_BDF, SV tolerances, Newton, SPGMR(PREC_LEFT, KRYLOV_DIM), classical GS
// below 500000 unknowns, MaxOrd, CV_NORMAL output).  SUNDIALS is not part of
// the reference tree; the step/order/convergence logic follows the published
// CVODE algorithm (Hindmarsh et al., ACM TOMS 31(3) 2005) with CVODE's
// default constants, so the step sequence matches a CVODE run.
//
// All vectors live in HBM; every vector update is one kernel on the
// context's stream.  Scalars (norms, Gram–Schmidt coefficients) come back
// through one pinned copy per decision point.  The Arnoldi step
// (ewt-scaling, Jv, subtraction, block-Jacobi solve, rescaling) is one fused
// kernel (launch_arnoldi_op) instead of the five separate passes of the
// reference's SPGMR + callbacks; the Newton residual, the first Krylov
// vector, the Gram–Schmidt update, the correction update and the
// tolerance weights each carry their norm in the same pass (k_fused.cu).
// The Newton correction starts as an implicit zero (ycor_zero) instead of a
// cleared vector.
#include <float.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "llg_internal.h"
#include "launch.h"

#include "cvode_consts.h"

namespace {
double powi(double b, int e) {
  double p = 1.0;
  for (int i = 1; i <= (e < 0 ? -e : e); i++) p *= b;
  return e < 0 ? 1.0 / p : p;
}
double powr(double b, double e) { return (b <= 0.0) ? 0.0 : pow(b, e); }
}  // namespace

struct Integrator {
  llg_ctx* c = nullptr;
  long long neq = 0;
  int qmax = 5, maxl = 5, classical_gs = 1, mxstep = 500;
  // LLG_KRYLOV_FP32: the basis V[0..maxl] holds floats (the same allocations);
  // the read-back-light SPGMR then calls the float variants of its kernels.
  // kf32_req: requested; kf32: in use (a learned-preconditioner context
  // keeps FP64 until the network is off, then switches in cv_nls)
  bool kf32_req = false, kf32 = false;
  float* Vf(int i) const { return reinterpret_cast<float*>(V[i]); }
  double rtol = 1e-4, atol = 1e-6;
  double* zn[QMAXL + 1] = {};
  double *ewt = nullptr, *acor = nullptr, *y = nullptr, *tempv = nullptr, *delta = nullptr;
  double* V[MAXLL + 1] = {};
  double Hes[MAXLL + 1][MAXLL] = {}, givens[2 * MAXLL] = {}, yg[MAXLL + 1] = {};
  double tn = 0, h = 0, hscale = 0, hprime = 0, next_h = 0, eta = 1, etamax = ETAMX1, hu = 0, hmin = 0,
         hmax_inv = 0;
  double etaq = 0, etaqm1 = 0, etaqp1 = 0;
  int q = 1, qprime = 1, next_q = 1, qwait = 2, L = 2, qu = 0, indx_acor = 5;
  double l[QMAXL + 2] = {}, tq[6] = {}, tau[QMAXL + 2] = {};
  double gamma = 0, gammap = 0, gamrat = 1, rl1 = 1, crate = 1, delp = 0, acnrm = 0, saved_tq5 = 0;
  int jcur_nls = 0, jcur = 0, convfail = 0, started = 0, ls_curiter = 0;
  long long nst = 0, nfe = 0, nsetups = 0, nni = 0, ncfn = 0, netf = 0, nli = 0, nlcf = 0, njv = 0, nps = 0,
            npe = 0, nstlp = 0, nstlj = 0, nscon = 0;
  int err = 0;  // sticky CUDA/launch failure
  bool ycor_zero = false;  // acor holds the zero vector implicitly (not yet written)
  // learned-preconditioner policy: every PROBE_EVERY-th solve runs block-
  // Jacobi; once both sides have enough solves, the learned path stays only
  // if its iterations are cheaper than block-Jacobi's at the measured cost
  // ratio kappa = (learned application) / (fused Arnoldi operator)
  static constexpr int PROBE_EVERY = 8, MIN_LEARNED = 24, MIN_PROBES = 4;
  long long pol_solves = 0, nsl = 0, nil = 0, nsb = 0, nib = 0;
  double kappa = -1.0;
  // device-resident form (integrator_dev.cu): graph + device copy of this state
  int device_resident = 0;
  bool ewt_pending = false;   // weights launched, their checks not yet read
  static constexpr int SLOT_EWT = 4;
  // CVODE's pre-step checks: weights well defined, ||y|| finite and above the
  // accuracy floor
  int state_check(double bad, double nrm) {
    if (bad != 0.0) { llg_set_error("a tolerance weight is not positive"); return LLG_CV_ILL_INPUT; }
    if (!isfinite(nrm)) { llg_set_error("non-finite state (WRMS norm of y is not finite)"); return LLG_CV_BAD_STATE; }
    if (UROUND * nrm > 1.0) return LLG_CV_TOO_MUCH_ACC;
    return 0;
  }
  bool ewt_fresh = false;     // h_scal holds this step's weight checks
  int ewt_checked() {
    // the first read-back of spgmr_spec covers SLOT_EWT; other paths read it here
    if (!ewt_fresh) ok(fetch_range(c, SLOT_EWT, SLOT_EWT + 2));
    ewt_fresh = false;
    return state_check(c->h_scal[SLOT_EWT], wrms_of(c->h_scal[SLOT_EWT + 1]));
  }
  DevInteg* dev = nullptr;
  bool dev_current = false;   // the device copy holds the latest state

  // Step-sequence record / replay.  Recording appends the (h, q) of every
  // accepted step; replaying makes step n use the recorded (h_n, q_n): the
  // order changes and the Nordsieck rescale are CVODE's own, the error test
  // is evaluated but does not reject (replay_forced counts the steps it
  // would have rejected), the Newton iteration may take up to REPLAY_MAXCOR
  // iterations without the divergence test, and a Newton failure retries the
  // same step with a fresh preconditioner setup (twice at most) instead of
  // shrinking h.
  std::vector<double> rec_h, rp_h;
  std::vector<int> rec_q, rp_q;
  int rec_cap = 0;
  bool replay = false;
  long long replay_forced = 0;
  static constexpr int REPLAY_MAXCOR = 10;   // Newton iterations per attempt while replaying

  void export_state(DState& s) const {
    memset(&s, 0, sizeof(s));
#define LLG_CP_OUT(f) s.f = f;
    LLG_DS_DOUBLES(LLG_CP_OUT)
    LLG_DS_INTS(LLG_CP_OUT)
    LLG_DS_LLS(LLG_CP_OUT)
#undef LLG_CP_OUT
    memcpy(s.l, l, sizeof(s.l));
    memcpy(s.tq, tq, sizeof(s.tq));
    memcpy(s.tau, tau, sizeof(s.tau));
    for (int j = 0; j <= QMAXL; j++) s.zn[j] = zn[j];
    for (int j = 0; j <= MAXLL; j++) s.V[j] = V[j];
    s.ewt = ewt; s.acor = acor; s.y = y; s.tempv = tempv; s.delta = delta;
  }
  void import_state(const DState& s) {
#define LLG_CP_IN(f) f = s.f;
    LLG_DS_DOUBLES(LLG_CP_IN)
    LLG_DS_INTS(LLG_CP_IN)
    LLG_DS_LLS(LLG_CP_IN)
#undef LLG_CP_IN
    memcpy(l, s.l, sizeof(s.l));
    memcpy(tq, s.tq, sizeof(s.tq));
    memcpy(tau, s.tau, sizeof(s.tau));
  }
  // the device form covers classical Gram-Schmidt with block-Jacobi; the
  // learned preconditioner and training-pair harvesting stay on the host path
  bool device_applies() {
    return device_resident && started && classical_gs && maxl <= MAXLL - 1 && !learned_active(c) &&
           !learned_harvest_wanted(c) && !replay && rec_cap == 0 && !c->dp.src_on && !c->d_hv && !kf32;
  }
  int integrate_device(double tout, double* yout, double* tret) {
    materialise();
    if (!dev) {
      const int rc = devint_create(c, &dev);
      if (rc) return rc;
    }
    if (!dev_current) {
      DState hs;
      export_state(hs);
      const int rc = devint_upload(dev, hs, c);
      if (rc) return rc;
      dev_current = true;
    }
    DState hs;
    y_ready = false;
    const int rc = devint_run(dev, c, tout, yout, hs);
    if (rc) { dev_current = false; return rc; }
    import_state(hs);
    *tret = hs.tret;
    return hs.status;
  }

  // ── helpers ──
  bool ok(int rc) {
    if (rc != 0 && !err) err = rc;
    return rc == 0;
  }
  double wrms(const double* x) {
    double r = 0.0;
    if (ok(vwrms_dev(c, x, ewt, SLOT_A))) ok(fetch_scalars(c, SLOT_A, 1, &r));
    return r;
  }
  // sqrt(s/neq) of raw sums: the same arithmetic as the device-side wrms
  double wrms_of(double s) const { return sqrt(s / (double)neq); }
  void materialise_acor() {
    if (ycor_zero) { ok(vconst(c, 0.0, acor)); ycor_zero = false; }
  }
  double dot(const double* x, const double* yv) {
    double r = 0.0;
    const double* Y[1] = {yv};
    if (ok(vdot_multi_dev(c, 1, x, Y, SLOT_DOTS))) ok(fetch_scalars(c, SLOT_DOTS, 1, &r));
    return r;
  }
  // a failure planted by llg_inject_rhs_failure (host side, nothing launched)
  bool rhs_injected() {
    if (c->inject_rhs_after < 0 || c->inject_rhs_seen++ < c->inject_rhs_after) return false;
    llg_set_error("RHS evaluation failed (injected)");
    err = LLG_ERR_LAUNCH;
    return true;
  }
  int call_f(double t, double* yv, double* ydot) {
    nfe++;
    if (rhs_injected()) return LLG_ERR_LAUNCH;
    const int r = rhs_full(c, t, yv, ydot);
    if (r) err = r;
    return r;
  }
  int set_ewt(const double* ycur) {
    double bad = 0.0;
    if (ok(vset_ewt(c, rtol, atol, ycur, ewt, SLOT_A + 1))) ok(fetch_scalars(c, SLOT_A + 1, 1, &bad));
    return bad != 0.0 ? -1 : 0;
  }

  // ── SPGMR ──
  double gram_schmidt(int k) {
    if (classical_gs) {
      std::vector<const double*> Y(k + 1);
      for (int i = 0; i <= k; i++) Y[i] = V[i];
      double dots[MAXLL + 1];
      if (ok(vdot_multi_dev(c, k + 1, V[k], Y.data(), SLOT_DOTS))) ok(fetch_scalars(c, SLOT_DOTS, k + 1, dots));
      const double vk_norm = sqrt(dots[k]);
      double cf[MAXLL + 1];
      const double* X[MAXLL + 1];
      cf[0] = 1.0;
      X[0] = V[k];
      for (int i = 0; i < k; i++) { Hes[i][k - 1] = dots[i]; cf[i + 1] = -dots[i]; X[i + 1] = V[i]; }
      double ss = 0.0;
      if (ok(fused_lincomb_norm(c, k + 1, cf, X, V[k], SLOT_DOTS))) ok(fetch_scalars(c, SLOT_DOTS, 1, &ss));
      double nrm = sqrt(ss);
      if (GS_FACTOR * nrm < vk_norm) {
        if (ok(vdot_multi_dev(c, k, V[k], Y.data(), SLOT_DOTS))) ok(fetch_scalars(c, SLOT_DOTS, k, dots));
        cf[0] = 1.0;
        X[0] = V[k];
        for (int i = 0; i < k; i++) { Hes[i][k - 1] += dots[i]; cf[i + 1] = -dots[i]; X[i + 1] = V[i]; }
        if (ok(fused_lincomb_norm(c, k + 1, cf, X, V[k], SLOT_DOTS))) ok(fetch_scalars(c, SLOT_DOTS, 1, &ss));
        nrm = sqrt(ss);
      }
      return nrm;
    }
    const double vk_norm = sqrt(dot(V[k], V[k]));
    for (int i = 0; i < k; i++) {
      Hes[i][k - 1] = dot(V[i], V[k]);
      ok(vlin(c, 1.0, V[k], -Hes[i][k - 1], V[i], V[k]));
    }
    double nrm = sqrt(dot(V[k], V[k]));
    double temp = GS_FACTOR * vk_norm;
    if ((temp + nrm) != temp) return nrm;
    double nn2 = 0.0;
    for (int i = 0; i < k; i++) {
      const double np = dot(V[i], V[k]);
      temp = GS_FACTOR * Hes[i][k - 1];
      if ((temp + np) == temp) continue;
      Hes[i][k - 1] += np;
      ok(vlin(c, 1.0, V[k], -np, V[i], V[k]));
      nn2 += np * np;
    }
    if (nn2 != 0.0) {
      const double t = nrm * nrm - nn2;
      nrm = (t > 0.0) ? sqrt(t) : 0.0;
    }
    return nrm;
  }

  int qr_fact(int n) {
    const int n1 = n - 1;
    int code = 0;
    for (int k = 0; k < n1; k++) {
      const int i = 2 * k;
      const double t1 = Hes[k][n1], t2 = Hes[k + 1][n1];
      const double cc = givens[i], s = givens[i + 1];
      Hes[k][n1] = cc * t1 - s * t2;
      Hes[k + 1][n1] = s * t1 + cc * t2;
    }
    const double t1 = Hes[n1][n1], t2 = Hes[n][n1];
    double cc, s;
    if (t2 == 0.0) { cc = 1.0; s = 0.0; }
    else if (fabs(t2) >= fabs(t1)) { const double t3 = t1 / t2; s = -1.0 / sqrt(1.0 + t3 * t3); cc = -s * t3; }
    else { const double t3 = t2 / t1; cc = 1.0 / sqrt(1.0 + t3 * t3); s = -cc * t3; }
    givens[2 * n1] = cc;
    givens[2 * n1 + 1] = s;
    if ((Hes[n1][n1] = cc * t1 - s * t2) == 0.0) code = n;
    return code;
  }

  int qr_sol(int n, double* bb) {
    int code = 0;
    for (int k = 0; k < n; k++) {
      const double cc = givens[2 * k], s = givens[2 * k + 1];
      const double t1 = bb[k], t2 = bb[k + 1];
      bb[k] = cc * t1 - s * t2;
      bb[k + 1] = s * t1 + cc * t2;
    }
    for (int k = n - 1; k >= 0; k--) {
      if (Hes[k][k] == 0.0) { code = k + 1; break; }
      bb[k] /= Hes[k][k];
      for (int i = 0; i < k; i++) bb[i] -= bb[k] * Hes[i][k];
    }
    return code;
  }

  bool fuse_update = false, update_done = false;   // see nls_lsolve / newton
  double upd_s[2] = {0.0, 0.0};

  // ── read-back-light SPGMR (classical Gram-Schmidt, block-Jacobi) ──
  // The Arnoldi iterations of one solve are enqueued with every coefficient
  // formed on the device (V0 / ||V0||, the Gram-Schmidt update from its own
  // dots, V[k] / ||V[k]||), and the first two are enqueued before any read-
  // back: the second is dropped, unused, when the first converges or needs a
  // second Gram-Schmidt pass.  One read-back then returns ||r||, the dots and
  // the norms of both iterations.  Same kernels, same arithmetic, same
  // decisions as spgmr() below.
  static int slot_it(int l) { return 64 + 24 * l; }       // dots of iteration l (l + 2 values)
  static int slot_ss(int l) { return 64 + 24 * l + 20; }  // sum of squares after its update
  static int slot_sc(int l) { return 64 + 24 * l + 21; }  // scale of the vector it produces
  static constexpr int SLOT_V0SC = 62;                    // scale of V0
  // The basis vectors stay unnormalised in memory; every kernel that reads
  // V[i] reads it as a_i V[i] (KScale, llg_internal.h).  a_0 = 1/||V0|| is
  // written by the kernel that forms ||V0||, a_k = 1/||V[k]|| (1 when a second
  // Gram-Schmidt pass is due; the host then normalises V[k] itself) by the
  // Gram-Schmidt update that forms ||V[k]||.  This replaces a normalising pass
  // over each vector with a multiply where it is read; the values used are
  // the ones that pass would have stored.
  const double* ka[MAXLL + 1] = {};
  KScale basis_scales(int k0, int k1, int at) const {   // entries at.. for V[k0..k1)
    KScale s{};
    for (int i = k0; i < k1; i++) s.a[at + i - k0] = ka[i];
    return s;
  }
  // pub_lo >= 0: the Gram-Schmidt update, the iteration's last kernel,
  // carries the read-back of d_scal[pub_lo, slot_ss(l)] (arm_publish)
  void enqueue_iter(int l, int pub_lo) {
    const int k = l + 1;
    const KScale ys = basis_scales(0, k, 0);   // V[k] itself: the fresh operator output, unscaled
    if (kf32) {
      ok(launch_arnoldi_op_f(c, Vf(l), ewt, Vf(k), y, gamma, ka[l]));
      const float* Y[MAXLL + 1];
      float* W[MAXLL + 1];
      for (int i = 0; i <= k; i++) { Y[i] = Vf(i); W[i] = Vf(i); }
      ok(vdot_multi_dev_f(c, k + 1, Vf(k), Y, slot_it(l), &ys));
      if (pub_lo >= 0) arm_publish(c, pub_lo, slot_ss(l) + 1);
      ok(vgs_update_dev_f(c, k, W, slot_it(l), slot_ss(l), &ys, slot_sc(l)));
    } else {
      ok(launch_arnoldi_op(c, V[l], ewt, V[k], y, gamma, 1, nullptr, ka[l]));
      const double* Y[MAXLL + 1];
      for (int i = 0; i <= k; i++) Y[i] = V[i];
      ok(vdot_multi_dev(c, k + 1, V[k], Y, slot_it(l), &ys));
      if (pub_lo >= 0) arm_publish(c, pub_lo, slot_ss(l) + 1);
      ok(vgs_update_dev(c, k, V, slot_it(l), slot_ss(l), &ys, slot_sc(l)));
    }
    ka[k] = c->d_scal + slot_sc(l);
  }
  int spgmr_spec(double* rhs, double delta_tol, bool harvest, double* zb) {
    const int lmax = maxl;
    int nl = 0, krydim = 0, converged = 0;
    nps++;
    if (harvest) ok(launch_psolve(c, rhs, zb));   // u = P_BJ^-1 r, kept with the solution
    if (!ok(kf32 ? fused_psolve_scale_dot_f(c, rhs, ewt, Vf(0), SLOT_A, SLOT_V0SC)
                 : fused_psolve_scale_dot(c, rhs, ewt, V[0], SLOT_A, nullptr, SLOT_V0SC)))
      return LS_CONV_FAIL;
    ka[0] = c->d_scal + SLOT_V0SC;
    // one Arnoldi iteration before the first read-back: enqueuing two saved
    // a read-back when GMRES needs a second iteration but wasted an operator
    // step, a Gram-Schmidt pass and their dots whenever one sufficed, which
    // cost more (measured at 1536x512: 397 -> 386 us per BDF step)
    int queued = 1;
    for (int l = 0; l < queued; l++) enqueue_iter(l, l == queued - 1 ? 0 : -1);
    ok(fetch_range(c, 0, slot_ss(queued - 1) + 1));
    if (err) return LS_CONV_FAIL;
    ewt_fresh = ewt_pending;
    const double* hsc = c->h_scal;
    const double beta = sqrt(hsc[SLOT_A]);
    double rnorm = beta, rho = beta;
    if (rnorm <= delta_tol) { ok(vconst(c, 0.0, rhs)); return LS_SUCCESS; }
    for (int i = 0; i <= lmax; i++)
      for (int j = 0; j < lmax; j++) Hes[i][j] = 0.0;
    double rot = 1.0;
    for (int l = 0; l < lmax; l++) {
      if (l >= queued) {
        enqueue_iter(l, slot_it(l));
        queued = l + 1;
        ok(fetch_range(c, slot_it(l), slot_ss(l) + 1));
        if (err) return LS_CONV_FAIL;
      }
      nl++;
      krydim = l + 1;
      njv++;
      nps++;
      const int k = l + 1;
      const double* d = hsc + slot_it(l);
      const double vk_norm = sqrt(d[k]);
      for (int i = 0; i < k; i++) Hes[i][l] = d[i];
      double nrm = sqrt(hsc[slot_ss(l)]);
      bool second = false;
      if (GS_FACTOR * nrm < vk_norm) {
        // second pass; V[k]'s scale is 1 (the device made the same test),
        // so later queued iterations are void and are enqueued again
        second = true;
        queued = k;
        double dots[MAXLL + 1], cf[MAXLL + 1], ss = 0.0;
        const KScale ys = basis_scales(0, k, 0), xs = basis_scales(0, k, 1);
        if (kf32) {
          const float* Y[MAXLL + 1];
          for (int i = 0; i < k; i++) Y[i] = Vf(i);
          if (ok(vdot_multi_dev_f(c, k, Vf(k), Y, SLOT_DOTS, &ys))) ok(fetch_scalars(c, SLOT_DOTS, k, dots));
        } else {
          const double* Y[MAXLL + 1];
          for (int i = 0; i < k; i++) Y[i] = V[i];
          if (ok(vdot_multi_dev(c, k, V[k], Y, SLOT_DOTS, &ys))) ok(fetch_scalars(c, SLOT_DOTS, k, dots));
        }
        cf[0] = 1.0;
        for (int i = 0; i < k; i++) { Hes[i][l] += dots[i]; cf[i + 1] = -dots[i]; }
        if (kf32) {
          const float* X[MAXLL + 1];
          X[0] = Vf(k);
          for (int i = 0; i < k; i++) X[i + 1] = Vf(i);
          if (ok(fused_lincomb_norm_f(c, k + 1, cf, X, Vf(k), SLOT_DOTS, &xs))) ok(fetch_scalars(c, SLOT_DOTS, 1, &ss));
        } else {
          const double* X[MAXLL + 1];
          X[0] = V[k];
          for (int i = 0; i < k; i++) X[i + 1] = V[i];
          if (ok(fused_lincomb_norm(c, k + 1, cf, X, V[k], SLOT_DOTS, &xs))) ok(fetch_scalars(c, SLOT_DOTS, 1, &ss));
        }
        nrm = sqrt(ss);
      }
      Hes[k][l] = nrm;
      if (qr_fact(krydim) != 0) { nli += nl; return LS_CONV_FAIL; }
      rot *= givens[2 * l + 1];
      rho = fabs(rot * rnorm);
      if (rho <= delta_tol) { converged = 1; break; }
      if (second) ok(kf32 ? vscale_f(c, 1.0 / Hes[k][l], Vf(k), Vf(k)) : vscale(c, 1.0 / Hes[k][l], V[k], V[k]));
    }
    nli += nl;
    yg[0] = rnorm;
    for (int i = 1; i <= krydim; i++) yg[i] = 0.0;
    if (qr_sol(krydim, yg) != 0) return LS_QRSOL_FAIL;
    if (converged || rho < beta) {
      const double* X[MAXLL + 1];
      const float* Xf[MAXLL + 1];
      for (int k = 0; k < krydim; k++) { X[k] = V[k]; Xf[k] = Vf(k); }
      const KScale xs = basis_scales(0, krydim, 0);
      const bool taken = converged || ls_curiter == 0;
      if (taken && fuse_update) {
        arm_publish(c, SLOT_A, SLOT_A + 2);
        ok(kf32 ? fused_lincomb_update_f(c, krydim, yg, Xf, ewt, harvest ? rhs : nullptr, ycor_zero, acor, SLOT_A, &xs)
                : fused_lincomb_update(c, krydim, yg, X, ewt, harvest ? rhs : nullptr, ycor_zero, acor, SLOT_A, &xs));
        ok(fetch_scalars(c, SLOT_A, 2, upd_s));
        update_done = true;
      } else {
        ok(kf32 ? fused_lincomb_div_f(c, krydim, yg, Xf, ewt, rhs, &xs)
                : fused_lincomb_div(c, krydim, yg, X, ewt, rhs, &xs));
      }
      if (converged && harvest) ok(learned_harvest(c, zb, rhs, ewt, c->gamma_setup));
      return converged ? LS_SUCCESS : LS_RES_REDUCED;
    }
    return LS_CONV_FAIL;
  }

  int spgmr(double* rhs, double delta_tol, bool learned) {
    const int lmax = maxl;
    int nl = 0, krydim = 0, converged = 0;
    const bool harvest = !learned && learned_harvest_wanted(c);
    double* zb = (learned || harvest) ? learned_zbuf(c) : nullptr;
    if ((learned || harvest) && !zb) return LS_CONV_FAIL;
    if (!learned && classical_gs) return spgmr_spec(rhs, delta_tol, harvest, zb);
    if (kf32) { llg_set_error("FP32 Krylov basis: the learned / modified Gram-Schmidt solver keeps FP64"); err = LLG_ERR_NOTSUP; return LS_CONV_FAIL; }
    nps++;
    double ss = 0.0;
    if (harvest) ok(launch_psolve(c, rhs, zb));   // u = P_BJ^-1 r, kept with the solution
    if (learned) {
      // V0 = ewt (I + gamma Net) P_BJ^-1 r, and its norm
      if (!ok(launch_psolve(c, rhs, zb)) || !ok(learned_apply(c, ewt, V[0], SLOT_A))) return LS_CONV_FAIL;
    } else if (!ok(fused_psolve_scale_dot(c, rhs, ewt, V[0], SLOT_A))) {
      return LS_CONV_FAIL;
    }
    ok(fetch_scalars(c, SLOT_A, 1, &ss));
    const double beta = sqrt(ss);
    double rnorm = beta, rho = beta;
    if (rnorm <= delta_tol) { ok(vconst(c, 0.0, rhs)); return LS_SUCCESS; }
    for (int i = 0; i <= lmax; i++)
      for (int j = 0; j < lmax; j++) Hes[i][j] = 0.0;
    double rot = 1.0;
    ok(vscale(c, 1.0 / rnorm, V[0], V[0]));
    for (int l = 0; l < lmax; l++) {
      nl++;
      krydim = l + 1;
      njv++;
      nps++;
      if (learned && kappa < 0.0) {
        // one-time cost ratio of the learned application to the Arnoldi operator
        cudaEvent_t e[3];
        for (auto& ev : e) cudaEventCreate(&ev);
        cudaEventRecord(e[0], c->stream);
        ok(launch_arnoldi_op(c, V[l], ewt, zb, y, gamma, 0));
        cudaEventRecord(e[1], c->stream);
        ok(learned_apply(c, ewt, V[l + 1], -1));
        cudaEventRecord(e[2], c->stream);
        cudaEventSynchronize(e[2]);
        float ta = 0.f, tl = 0.f;
        cudaEventElapsedTime(&ta, e[0], e[1]);
        cudaEventElapsedTime(&tl, e[1], e[2]);
        for (auto& ev : e) cudaEventDestroy(ev);
        kappa = (ta > 0.f) ? (double)tl / ta : 1.0;
      } else if (learned) {
        ok(launch_arnoldi_op(c, V[l], ewt, zb, y, gamma, 0));
        ok(learned_apply(c, ewt, V[l + 1], -1));
      } else {
        ok(launch_arnoldi_op(c, V[l], ewt, V[l + 1], y, gamma));
      }
      Hes[l + 1][l] = gram_schmidt(l + 1);
      if (qr_fact(krydim) != 0) { nli += nl; return LS_CONV_FAIL; }
      rot *= givens[2 * l + 1];
      rho = fabs(rot * rnorm);
      if (rho <= delta_tol) { converged = 1; break; }
      ok(vscale(c, 1.0 / Hes[l + 1][l], V[l + 1], V[l + 1]));
    }
    nli += nl;
    yg[0] = rnorm;
    for (int i = 1; i <= krydim; i++) yg[i] = 0.0;
    if (qr_sol(krydim, yg) != 0) return LS_QRSOL_FAIL;
    if (converged || rho < beta) {
      // x = 0 + sum_k yg_k V_k, then x / ewt; 0 + a*b is a*b exactly, so the
      // zero initial guess needs no pass of its own
      const double* X[MAXLL + 1];
      for (int k = 0; k < krydim; k++) X[k] = V[k];
      // when the Newton iteration will take this correction (nls_lsolve
      // returns 0), apply it to the correction vector in the same pass
      const bool taken = converged || ls_curiter == 0;
      if (taken && fuse_update) {
        arm_publish(c, SLOT_A, SLOT_A + 2);
        ok(fused_lincomb_update(c, krydim, yg, X, ewt, harvest ? rhs : nullptr, ycor_zero, acor, SLOT_A));
        ok(fetch_scalars(c, SLOT_A, 2, upd_s));
        update_done = true;
      } else {
        ok(fused_lincomb_div(c, krydim, yg, X, ewt, rhs));
      }
      if (converged && harvest) ok(learned_harvest(c, zb, rhs, ewt, c->gamma_setup));
      return converged ? LS_SUCCESS : LS_RES_REDUCED;
    }
    return LS_CONV_FAIL;
  }

  // ── CVODE pieces ──
  void set_bdf() {
    double alpha0, alpha0_hat, xi_inv, xistar_inv, hsum;
    l[0] = l[1] = xi_inv = xistar_inv = 1.0;
    for (int i = 2; i <= q; i++) l[i] = 0.0;
    alpha0 = alpha0_hat = -1.0;
    hsum = h;
    if (q > 1) {
      for (int j = 2; j < q; j++) {
        hsum += tau[j - 1];
        xi_inv = h / hsum;
        alpha0 -= 1.0 / j;
        for (int i = j; i >= 1; i--) l[i] += l[i - 1] * xi_inv;
      }
      alpha0 -= 1.0 / q;
      xistar_inv = -l[1] - alpha0;
      hsum += tau[q - 1];
      xi_inv = h / hsum;
      alpha0_hat = -l[1] - xi_inv;
      for (int i = q; i >= 1; i--) l[i] += l[i - 1] * xistar_inv;
    }
    const double A1 = 1.0 - alpha0_hat + alpha0;
    const double A2 = 1.0 + q * A1;
    tq[2] = fabs(A1 / (alpha0 * A2));
    tq[5] = fabs(A2 * xistar_inv / (l[q] * xi_inv));
    if (qwait == 1) {
      if (q > 1) {
        const double C = xistar_inv / l[q];
        const double A3 = alpha0 + 1.0 / q;
        const double A4 = alpha0_hat + xi_inv;
        const double Cpinv = (1.0 - A4 + A3) / A3;
        tq[1] = fabs(C * Cpinv);
      } else {
        tq[1] = 1.0;
      }
      hsum += tau[q];
      xi_inv = h / hsum;
      const double A5 = alpha0 - (1.0 / (q + 1));
      const double A6 = alpha0_hat - xi_inv;
      const double Cppinv = (1.0 - A6 + A5) / A2;
      tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
    }
    tq[4] = CORTES / tq[2];
  }

  void cv_set() {
    set_bdf();
    rl1 = 1.0 / l[1];
    gamma = h * rl1;
    if (nst == 0) gammap = gamma;
    gamrat = (nst > 0) ? gamma / gammap : 1.0;
  }

  // The weights of a new step and a rescale of zn are not separate passes:
  // predict() applies them (fused_predict), together with the first Newton
  // iterate y = normalise(zn0) that nls_residual then reuses.
  bool ewt_due = false;       // this step's weights still to be formed
  bool resc_pending = false;  // zn[j] *= resc_f[j] still to be applied
  double resc_f[QMAXL + 1] = {};
  bool y_ready = false;       // y = normalise(zn0) for the current zn0
  // Lazy completion: complete_step records zn[j] += l_j acor (j = 0..q, and
  // zn[qmax] = acor when saving) instead of running it, and the next predict
  // pass applies it first, element by element with the same arithmetic, so
  // the Nordsieck array is read and written once per step instead of twice.
  // Anything that reads zn between the two (order change, output
  // interpolation, state export, a copy of zn0 to the caller) materialises it
  // first with the eager pass.
  bool lazy = false;
  int lazy_q = 0;
  bool lazy_save = false;
  double lazy_l[QMAXL + 2] = {};
  void materialise() {
    if (!lazy) return;
    ok(fused_complete(c, lazy_q, qmax, lazy_l, acor, zn, lazy_save, false, 0.0, ewt, SLOT_A, true));
    lazy = false;
  }
  void predict() {
    tn += h;
    const bool lz = lazy && lazy_q == q;
    if (lazy && !lz) materialise();
    ok(fused_predict(c, q, zn, resc_f, resc_pending, ewt_due, rtol, atol, ewt, y, SLOT_EWT, lz ? lazy_l : nullptr,
                     acor, lazy_save ? zn[qmax] : nullptr));
    lazy = false;
    if (ewt_due) ewt_pending = true;
    ewt_due = false;
    resc_pending = false;
    y_ready = true;
  }
  void restore(double saved_t) {
    materialise();   // (nothing is pending after a predict)
    tn = saved_t;
    ok(vnordsieck_shift(c, q, zn, -1));
    y_ready = false;
  }
  void rescale() {
    if (resc_pending) ok(vscale_columns_f(c, q, resc_f, zn));   // (not reached: a predict follows every rescale)
    double factor = eta;
    for (int j = 1; j <= q; j++) { resc_f[j] = factor; factor *= eta; }
    resc_pending = true;
    h = hscale * eta;
    next_h = h;
    hscale = h;
    nscon = 0;
  }
  void increase_bdf() {
    double alpha0, alpha1, prod, xi, xiold, hsum, A1;
    for (int i = 0; i <= qmax; i++) l[i] = 0.0;
    l[2] = alpha1 = prod = xiold = 1.0;
    alpha0 = -1.0;
    hsum = hscale;
    if (q > 1) {
      for (int j = 1; j < q; j++) {
        hsum += tau[j + 1];
        xi = hsum / hscale;
        prod *= xi;
        alpha0 -= 1.0 / (j + 1);
        alpha1 += 1.0 / xi;
        for (int i = j + 2; i >= 2; i--) l[i] = l[i] * xiold + l[i - 1];
        xiold = xi;
      }
    }
    A1 = (-alpha0 - alpha1) / prod;
    ok(vscale(c, A1, zn[indx_acor], zn[L]));
    for (int j = 2; j <= q; j++) ok(vlin(c, l[j], zn[L], 1.0, zn[j], zn[j]));
  }
  void decrease_bdf() {
    double hsum, xi;
    for (int i = 0; i <= qmax; i++) l[i] = 0.0;
    l[2] = 1.0;
    hsum = 0.0;
    for (int j = 1; j <= q - 2; j++) {
      hsum += tau[j];
      xi = hsum / hscale;
      for (int i = j + 2; i >= 2; i--) l[i] = l[i] * xi + l[i - 1];
    }
    for (int j = 2; j < q; j++) ok(vlin(c, -l[j], zn[q], 1.0, zn[j], zn[j]));
  }
  void adjust_order(int dq) {
    if (q == 2 && dq != 1) return;
    if (dq == 1) increase_bdf();
    else if (dq == -1) decrease_bdf();
  }
  void adjust_params() {
    if (qprime != q) {
      materialise();
      adjust_order(qprime - q);
      q = qprime;
      L = q + 1;
      qwait = L;
    }
    rescale();
  }

  // y = zn0 + ycor, f(y) (normalising y in place), and the NEGATED Newton
  // residual  -(rl1 zn1 + ycor - gamma f(y))  in the RHS kernel's epilogue.
  int nls_residual(const double* ycor, double* negres) {
    nfe++;
    if (rhs_injected()) return LLG_CV_RHSFUNC_FAIL;
    const double* yc = ycor_zero ? nullptr : ycor;
    set_source_time(c, tn);
    int r = (ycor_zero && y_ready) ? 0 : fused_lin_normalize(c, zn[0], yc, y);
    y_ready = false;
    if (!r) r = fused_field(c, y);
    if (!r) r = fused_resid(c, y, zn[1], yc, rl1, gamma, negres);
    if (r) { err = r; return LLG_CV_RHSFUNC_FAIL; }
    return 0;
  }
  int nls_lsetup(int jbad) {
    if (jbad) convfail = CV_FAIL_BAD_J;
    const double dgamma = fabs(gamma / gammap - 1.0);
    (void)dgamma;
    const int r = launch_psetup(c, y, gamma);
    npe++;
    nstlj = nst;
    jcur = 1;
    nsetups++;
    jcur_nls = jcur;
    gamrat = 1.0;
    gammap = gamma;
    crate = 1.0;
    nstlp = nst;
    if (r < 0) { err = r; return LLG_CV_LSETUP_FAIL; }
    return 0;
  }
  int nls_lsolve(double* del) {
    const double deltar = LS_EPLIN * tq[4];
    const double dtol = deltar * sqrt((double)neq);
    bool learned = learned_active(c);
    bool probe = false;
    if (learned && learned_policy_on(c) && (pol_solves++ % PROBE_EVERY) == PROBE_EVERY - 1) {
      learned = false;
      probe = true;
    }
    const long long nli0 = nli;
    fuse_update = true;
    update_done = false;
    const int r = spgmr(del, dtol, learned);
    fuse_update = false;
    if (err) return LLG_CV_LSOLVE_FAIL;
    if (learned) { nsl++; nil += nli - nli0; }
    if (probe) { nsb++; nib += nli - nli0; }
    if ((learned || probe) && nsl >= MIN_LEARNED && nsb >= MIN_PROBES && kappa >= 0.0) {
      // per solve, in Arnoldi-operator units: each iteration costs the operator
      // plus ~0.6 for Gram-Schmidt; the learned path adds kappa per application
      // (one per iteration plus the first Krylov vector)
      const double itl = (double)nil / nsl, itb = (double)nib / nsb;
      const double cost_l = itl * 1.6 + (itl + 1.0) * kappa, cost_b = itb * 1.6;
      learned_policy_record(c, itl, itb, kappa);
      if (cost_l >= cost_b) learned_fall_back(c, 2);
      nsl = nil = nsb = nib = 0;   // judge again on fresh counts if it stays
    }
    // GMRES convergence judges the learned preconditioner: a failed solve
    // switches this context back to block-Jacobi (the Newton iteration then
    // recovers as after any linear-solver failure)
    if (learned && (r == LS_CONV_FAIL || r == LS_QRSOL_FAIL)) learned_fall_back(c, 1);
    if (r != LS_SUCCESS) nlcf++;
    if (r == LS_SUCCESS) return 0;
    if (r == LS_RES_REDUCED) return (ls_curiter == 0) ? 0 : 1;
    return 1;
  }
  // s[0], s[1]: raw weighted sums of squares of del and of the updated ycor
  int nls_ctest(const double s[2], double tol, int m) {
    const double dn = wrms_of(s[0]);
    if (m > 0) {
      const double r = dn / delp;
      crate = (CRDOWN * crate > r) ? CRDOWN * crate : r;
    }
    const double dcon = dn * (crate < 1.0 ? crate : 1.0) / tol;
    if (dcon <= 1.0) {
      acnrm = (m == 0) ? dn : wrms_of(s[1]);
      return 0;
    }
    // (a replay keeps its recorded step size, so it lets the iteration run
    // on past a slow start instead of declaring divergence)
    if (!replay && (m >= 1) && (dn > RDIV * delp)) return NLS_CONV_RECVR;
    delp = dn;
    return NLS_CONTINUE;
  }
  int newton(int call_setup) {
    double* ycor = acor;
    double* del = delta;
    int jbad = 0, retval = 0;
    for (;;) {
      retval = nls_residual(ycor, del);
      if (retval != 0) break;
      if (call_setup) {
        retval = nls_lsetup(jbad);
        if (retval != 0) break;
      }
      int m = 0;
      for (;;) {
        nni++;
        ls_curiter = m;
        retval = nls_lsolve(del);
        if (retval != 0) break;
        double s[2] = {0.0, 0.0};
        if (update_done) {   // the GMRES solution pass already applied it
          s[0] = upd_s[0];
          s[1] = upd_s[1];
        } else {
          arm_publish(c, SLOT_A, SLOT_A + 2);
          if (ok(fused_update_wrms2(c, ycor_zero, ycor, del, ewt, SLOT_A))) ok(fetch_scalars(c, SLOT_A, 2, s));
        }
        update_done = false;
        ycor_zero = false;
        retval = nls_ctest(s, tq[4], m);
        if (err) return LLG_CV_LSOLVE_FAIL;
        if (retval == 0) { jcur_nls = 0; return 0; }
        if (retval != NLS_CONTINUE) break;
        m++;
        if (m >= (replay ? REPLAY_MAXCOR : NLS_MAXCOR)) { retval = NLS_CONV_RECVR; break; }
        retval = nls_residual(ycor, del);
        if (retval != 0) break;
      }
      if (retval > 0 && !jcur_nls) {
        call_setup = 1;
        jbad = 1;
        ycor_zero = true;
        continue;
      }
      break;
    }
    return retval;
  }
  int cv_nls(int nflag) {
    convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL)) ? CV_NO_FAILURES : CV_FAIL_OTHER;
    if (kf32_req && !kf32 && !learned_active(c)) {
      // the learned preconditioner is off for good: block-Jacobi continues on
      // the FP32 basis, whose operator reads an FP32 block inverse (a fresh
      // setup below)
      kf32 = true;
      c->pinv_f32 = 1;
      c->have_setup = 0;
    }
    const int call_setup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL) || (nst == 0) ||
                           (nst >= nstlp + MSBP) || (fabs(gamrat - 1.0) > DGMAX) || !c->have_setup;
    ycor_zero = true;
    const int flag = newton(call_setup);
    // (CVODE also forms y = zn0 + acor here; nothing in this integrator reads it)
    if (flag != 0) { materialise_acor(); return flag; }
    jcur = 0;
    return 0;
  }
  int handle_nflag(int* nflag, double saved_t, int* ncf) {
    if (*nflag == 0) return DO_ERROR_TEST;
    ncfn++;
    restore(saved_t);
    if (*nflag < 0) return *nflag;
    (*ncf)++;
    etamax = 1.0;
    if (replay) {   // the step size is fixed: retry with a fresh setup
      if (*ncf > 2) { llg_set_error("replay: Newton iteration failed on a recorded step"); return LLG_CV_CONV_FAILURE; }
      *nflag = PREV_CONV_FAIL;
      return PREDICT_AGAIN;
    }
    if ((fabs(h) <= hmin * ONEPSM) || (*ncf == MXNCF)) return LLG_CV_CONV_FAILURE;
    eta = (ETACF > hmin / fabs(h)) ? ETACF : hmin / fabs(h);
    *nflag = PREV_CONV_FAIL;
    rescale();
    return PREDICT_AGAIN;
  }
  int error_test(int* nflag, double saved_t, int* nef, double* dsmp) {
    const double dsm = acnrm * tq[2];
    *dsmp = dsm;
    if (dsm <= 1.0) return 0;
    if (replay) { replay_forced++; return 0; }
    (*nef)++;
    netf++;
    *nflag = PREV_ERR_FAIL;
    restore(saved_t);
    if ((fabs(h) <= hmin * ONEPSM) || (*nef == MXNEF)) return LLG_CV_ERR_FAILURE;
    etamax = 1.0;
    if (*nef <= MXNEF1) {
      double e = 1.0 / (powr(BIAS2 * dsm, 1.0 / L) + ADDON);
      const double lo = hmin / fabs(h);
      e = (e > lo) ? e : lo;
      e = (e > ETAMIN) ? e : ETAMIN;
      if (*nef >= SMALL_NEF) e = (e < ETAMXF) ? e : ETAMXF;
      eta = e;
      rescale();
      return TRY_AGAIN;
    }
    if (q > 1) {
      eta = (ETAMIN > hmin / fabs(h)) ? ETAMIN : hmin / fabs(h);
      adjust_order(-1);
      L = q;
      q--;
      qwait = L;
      rescale();
      return TRY_AGAIN;
    }
    eta = (ETAMIN > hmin / fabs(h)) ? ETAMIN : hmin / fabs(h);
    h *= eta;
    next_h = h;
    hscale = h;
    qwait = LONG_WAIT;
    nscon = 0;
    const int r = call_f(tn, zn[0], tempv);
    if (r < 0) return LLG_CV_RHSFUNC_FAIL;
    ok(vscale(c, h, tempv, zn[1]));
    return TRY_AGAIN;
  }
  // complete_step; when prepare_next will select the order, the norms it needs
  // are summed in the same pass (one read-back there)
  bool norms_ready = false;
  void complete_step() {
    if ((int)rec_h.size() < rec_cap) { rec_h.push_back(h); rec_q.push_back(q); }
    nst++;
    nscon++;
    hu = h;
    qu = q;
    for (int i = q; i >= 2; i--) tau[i] = tau[i - 1];
    if ((q == 1) && (nst > 1)) tau[2] = tau[1];
    tau[1] = h;
    qwait--;
    const bool save = (qwait == 1) && (q != qmax);
    if (save) {
      saved_tq5 = tq[5];
      indx_acor = qmax;
    }
    norms_ready = (etamax != 1.0) && (qwait == 0);
    const double cquot =
        (norms_ready && q != qmax && saved_tq5 != 0.0) ? (tq[5] / saved_tq5) * powi(h / tau[2], L) : 0.0;
    // the norms (of the completed values) now; the completion itself with the next predict
    ok(fused_complete(c, q, qmax, l, acor, zn, save, norms_ready, cquot, ewt, SLOT_A, false));
    lazy = true;
    lazy_q = q;
    lazy_save = save;
    for (int j = 0; j <= q; j++) lazy_l[j] = l[j];
    y_ready = false;
  }
  void set_eta() {
    if (eta < THRESH) {
      eta = 1.0;
      hprime = h;
    } else {
      eta = (eta < etamax) ? eta : etamax;
      const double d = fabs(h) * hmax_inv * eta;
      eta /= (d > 1.0 ? d : 1.0);
      hprime = h * eta;
      if (qprime < q) nscon = 0;
    }
  }
  void choose_eta() {
    double etam = etaqm1 > etaq ? etaqm1 : etaq;
    etam = etam > etaqp1 ? etam : etaqp1;
    if (etam < THRESH) { eta = 1.0; qprime = q; return; }
    if (etam == etaq) { eta = etaq; qprime = q; }
    else if (etam == etaqm1) { eta = etaqm1; qprime = q - 1; }
    else {
      eta = etaqp1;
      qprime = q + 1;
      ok(vscale(c, 1.0, acor, zn[qmax]));
    }
  }
  void prepare_next(double dsm) {
    if (etamax == 1.0) {
      qwait = qwait > 2 ? qwait : 2;
      qprime = q;
      hprime = h;
      eta = 1.0;
      return;
    }
    etaq = 1.0 / (powr(BIAS2 * dsm, 1.0 / L) + ADDON);
    if (qwait != 0) {
      eta = etaq;
      qprime = q;
      set_eta();
      return;
    }
    qwait = 2;
    // ||zn[q]|| and ||acor - cquot zn[qmax]||, summed by complete_step's pass
    double s[2] = {0.0, 0.0};
    if (!norms_ready) materialise();
    if (norms_ready) ok(fetch_scalars(c, SLOT_A, 2, s));
    else if (ok(fused_wrms2(c, zn[q], -((q != qmax && saved_tq5 != 0.0) ? (tq[5] / saved_tq5) * powi(h / tau[2], L)
                                                                          : 0.0),
                            zn[qmax], 1.0, acor, ewt, SLOT_A)))
      ok(fetch_scalars(c, SLOT_A, 2, s));
    norms_ready = false;
    etaqm1 = 0.0;
    if (q > 1) {
      const double ddn = wrms_of(s[0]) * tq[1];
      etaqm1 = 1.0 / (powr(BIAS1 * ddn, 1.0 / q) + ADDON);
    }
    etaqp1 = 0.0;
    if (q != qmax && saved_tq5 != 0.0) {
      const double dup = wrms_of(s[1]) * tq[3];
      etaqp1 = 1.0 / (powr(BIAS3 * dup, 1.0 / (L + 1)) + ADDON);
    }
    choose_eta();
    set_eta();
  }
  int cv_step() {
    const double saved_t = tn;
    int ncf = 0, nef = 0, nflag = FIRST_CALL;
    double dsm = 0.0;
    if (replay) {
      if (nst >= (long long)rp_h.size()) {
        llg_set_error("replay: the recorded step sequence ends before tout");
        return LLG_ERR_STATE;
      }
      if (nst > 0) {
        const int qt = rp_q[nst];
        const double ht = rp_h[nst];
        if (qt < 1 || qt > qmax || qt > q + 1 || qt < q - 1 || !(ht * h > 0.0)) {
          llg_set_error("replay: recorded step is not reachable from the current order");
          return LLG_ERR_ARG;
        }
        // an order increase builds the new column from the last correction,
        // which CVODE's order selection stores in zn[qmax] when it picks q + 1
        if (qt == q + 1) ok(vscale(c, 1.0, acor, zn[qmax]));
        qprime = qt;
        hprime = ht;
        if (qprime != q || hprime != h) {
          eta = hprime / h;
          adjust_params();
          h = hscale = next_h = ht;
        }
      }
    } else if ((nst > 0) && (hprime != h)) {
      adjust_params();
    }
    for (;;) {
      predict();
      cv_set();
      nflag = cv_nls(nflag);
      if (err) return LLG_CV_RHSFUNC_FAIL;
      if (ewt_pending) {   // the checks CVODE makes before a step, on this step's weights
        ewt_pending = false;
        const int e = ewt_checked();
        if (e) { restore(saved_t); return e; }
      }
      const int kflag = handle_nflag(&nflag, saved_t, &ncf);
      if (kflag == PREDICT_AGAIN) continue;
      if (kflag != DO_ERROR_TEST) return kflag;
      const int eflag = error_test(&nflag, saved_t, &nef, &dsm);
      if (eflag == TRY_AGAIN) continue;
      if (eflag != 0) return eflag;
      break;
    }
    complete_step();
    prepare_next(dsm);
    etamax = (nst <= SMALL_NST) ? ETAMX2 : ETAMX3;
    // (CVODE scales acor by tq[2] here for CVodeGetEstLocalErrors; not exposed)
    return err ? LLG_CV_RHSFUNC_FAIL : 0;
  }
  int get_dky(double t, double* dky) {
    materialise();
    double tfuzz = FUZZ_FACTOR * UROUND * (fabs(tn) + fabs(hu));
    if (hu < 0.0) tfuzz = -tfuzz;
    const double tp = tn - hu - tfuzz;
    const double tn1 = tn + tfuzz;
    if ((t - tp) * (t - tn1) > 0.0) { llg_set_error("get_dky: t outside the last step"); return LLG_CV_ILL_INPUT; }
    const double s = (t - tn) / h;
    double cf[QMAXL + 1];
    const double* X[QMAXL + 1];
    int nv = 0;
    for (int j = q; j >= 0; j--) {
      double cc = 1.0;
      for (int i = 0; i < j; i++) cc *= s;
      cf[nv] = cc;
      X[nv] = zn[j];
      nv++;
    }
    ok(vlincomb(c, nv, cf, X, dky));
    return err ? LLG_CV_RHSFUNC_FAIL : 0;
  }
  int y_dd_norm(double hg, double* yddnrm) {
    ok(vlin(c, hg, zn[1], 1.0, zn[0], y));
    const int r = call_f(tn + hg, y, tempv);
    if (r < 0) return LLG_CV_RHSFUNC_FAIL;
    if (r > 0) return 1;
    ok(vlin(c, 1.0, tempv, -1.0, zn[1], tempv));
    ok(vscale(c, 1.0 / hg, tempv, tempv));
    *yddnrm = wrms(tempv);
    return err ? LLG_CV_RHSFUNC_FAIL : 0;
  }
  int h_in(double tout) {
    const double tdiff = tout - tn;
    if (tdiff == 0.0) return LLG_CV_TOO_CLOSE;
    const int sign = (tdiff > 0.0) ? 1 : -1;
    const double tdist = fabs(tdiff);
    const double tround = UROUND * (fabs(tn) > fabs(tout) ? fabs(tn) : fabs(tout));
    if (tdist < 2.0 * tround) return LLG_CV_TOO_CLOSE;
    const double hlb = HLB_FACTOR * tround;
    double hub_inv = 0.0;
    if (ok(vhin_bound(c, rtol, atol, zn[0], zn[1], tempv))) ok(fetch_scalars(c, 40, 1, &hub_inv));
    double hub = HUB_FACTOR * tdist;
    if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
    double hg = sqrt(hlb * hub);
    if (hub < hlb) { h = (sign == -1) ? -hg : hg; return 0; }
    double hnew = hg;
    for (int count1 = 1; count1 <= MAX_ITERS; count1++) {
      int hgok = 0;
      double yddnrm = 0.0;
      for (int count2 = 1; count2 <= MAX_ITERS; count2++) {
        const double hgs = hg * sign;
        const int r = y_dd_norm(hgs, &yddnrm);
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
    h = h0;
    return 0;
  }

  int integrate(double tout, double* yout, double* tret) {
    if (device_applies()) return integrate_device(tout, yout, tret);
    // programmatic dependent launch: legacy default stream (the demag chain
    // launched kernel by kernel), block-Jacobi path (no harvest copies)
    const PdlScope pdl(c->stream == nullptr && !learned_active(c) && !learned_harvest_wanted(c));
    dev_current = false;   // the host path moves the state on
    const size_t vb = sizeof(double) * (size_t)neq;
    if (!started) {
      if (set_ewt(zn[0]) != 0) return LLG_CV_ILL_INPUT;
      const int r = call_f(tn, zn[0], zn[1]);
      if (r != 0) return LLG_CV_RHSFUNC_FAIL;
      const int hr = h_in(tout);
      if (hr != 0) return hr;
      if (replay) {
        if (rp_h.empty() || !(rp_h[0] * (tout - tn) > 0.0)) {
          llg_set_error("replay: empty or wrongly directed step sequence");
          return LLG_ERR_ARG;
        }
        h = rp_h[0];
      }
      hscale = h;
      hprime = h;
      ok(vscale(c, h, zn[1], zn[1]));
      started = 1;
    } else {
      if ((tn - tout) * h >= 0.0) {
        *tret = tout;
        return get_dky(tout, yout);
      }
    }
    int nstloc = 0;
    for (;;) {
      next_h = h;
      next_q = q;
      double nrm = 0.0;
      if (nst > 0) {
        // new weights and ||zn0||: formed by the step's first predict pass;
        // their checks are read with the step's first read-back (ewt_checked)
        ewt_due = true;
      }
      if ((mxstep > 0) && (nstloc >= mxstep)) {
        materialise();
        cudaMemcpyAsync(yout, zn[0], vb, cudaMemcpyDeviceToDevice, c->stream);
        pdl_break();
        *tret = tn;
        llg_set_error("mxstep reached before tout");
        return LLG_CV_TOO_MUCH_WORK;
      }
      if (nst == 0) {
        nrm = wrms(zn[0]);
        if (err) return LLG_CV_RHSFUNC_FAIL;
        const int e = state_check(0.0, nrm);
        if (e) {
          cudaMemcpyAsync(yout, zn[0], vb, cudaMemcpyDeviceToDevice, c->stream);
          pdl_break();
          *tret = tn;
          return e;
        }
      }
      const int kflag = cv_step();
      if (kflag != 0) {
        materialise();
        cudaMemcpyAsync(yout, zn[0], vb, cudaMemcpyDeviceToDevice, c->stream);
        pdl_break();
        *tret = tn;
        return kflag;
      }
      nstloc++;
      if ((tn - tout) * h >= 0.0) {
        *tret = tout;
        const int r = get_dky(tout, yout);
        next_q = qprime;
        next_h = hprime;
        if (r) return r;
        break;
      }
    }
    return err ? LLG_CV_RHSFUNC_FAIL : 0;
  }

  void free_all() {
    devint_destroy(dev);
    dev = nullptr;
    dev_current = false;
    for (auto& p : zn) { cudaFree(p); p = nullptr; }
    for (auto& p : V) { cudaFree(p); p = nullptr; }
    double** vs[] = {&ewt, &acor, &y, &tempv, &delta};
    for (auto pp : vs) { cudaFree(*pp); *pp = nullptr; }
  }
};

int integrator_create(llg_ctx* c, double t0, const double* y0, const llg_solver_opts* o) {
  Integrator* b = new Integrator();
  b->c = c;
  b->neq = c->neq;
  b->qmax = (o->maxord >= 1 && o->maxord <= QMAXL) ? o->maxord : QMAXL;
  b->maxl = (o->maxl > 0) ? o->maxl : 5;
  if (b->maxl > MAXLL - 1) b->maxl = MAXLL - 1;
  b->classical_gs = (o->gs_type == LLG_GS_CLASSICAL) || (o->gs_type == LLG_GS_AUTO && b->neq < 500000);
  b->mxstep = (o->mxstep > 0) ? o->mxstep : 500;
  b->rtol = o->rtol;
  b->atol = o->atol;
  b->device_resident = o->device_resident ? 1 : 0;
  b->kf32_req = (o->krylov_precision == LLG_KRYLOV_FP32);
  b->kf32 = b->kf32_req && c->p.precond_kind != LLG_PREC_LEARNED;
  if (o->krylov_precision != LLG_KRYLOV_FP64 && o->krylov_precision != LLG_KRYLOV_FP32) {
    delete b;
    llg_set_error("krylov_precision must be LLG_KRYLOV_FP64 or LLG_KRYLOV_FP32");
    return LLG_ERR_ARG;
  }
  if (b->kf32_req && !b->classical_gs) {
    delete b;
    llg_set_error("FP32 Krylov basis needs classical Gram-Schmidt");
    return LLG_ERR_NOTSUP;
  }
  const size_t vb = sizeof(double) * (size_t)b->neq;
  auto alloc = [&](double** p) -> int {
    LLG_CUDA_TRY(cudaMalloc(p, vb));
    LLG_CUDA_TRY(cudaMemsetAsync(*p, 0, vb, c->stream));
    return 0;
  };
  int rc = 0;
  for (int j = 0; j <= b->qmax && !rc; j++) rc = alloc(&b->zn[j]);
  for (int j = 0; j <= b->maxl && !rc; j++) rc = alloc(&b->V[j]);
  double** vs[] = {&b->ewt, &b->acor, &b->y, &b->tempv, &b->delta};
  for (auto pp : vs)
    if (!rc) rc = alloc(pp);
  if (rc) { b->free_all(); delete b; return rc; }
  if (y0 && cudaMemcpyAsync(b->zn[0], y0, vb, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess) {
    b->free_all();
    delete b;
    llg_set_error("integrator_init: copy of y0 failed");
    return LLG_ERR_CUDA;
  }
  b->tn = t0;
  b->q = 1;
  b->L = 2;
  b->qwait = b->L;
  b->etamax = ETAMX1;
  b->indx_acor = b->qmax;
  if (c->integ) { c->integ->free_all(); delete c->integ; }
  c->integ = b;
  // the FP32-basis operator reads an FP32 block inverse: psetup stores that
  // precision from now on (every step sequence starts with a setup)
  if (c->pinv_f32 != (b->kf32 ? 1 : 0)) {
    c->pinv_f32 = b->kf32 ? 1 : 0;
    c->have_setup = 0;
  }
  return 0;
}

void integrator_destroy(Integrator* b) {
  if (!b) return;
  b->free_all();
  delete b;
}

int integrator_run(llg_ctx* c, double tout, double* yout, double* tret) {
  if (!c->integ) { llg_set_error("llg_integrate before llg_integrator_init"); return LLG_ERR_STATE; }
  return c->integ->integrate(tout, yout, tret);
}

// Time one kernel family on the integrator's live buffers (profiling only;
// clobbers scratch vectors, never the Nordsieck history).
int integrator_time_kernel(llg_ctx* c, int kid, int iters, double* avg_ms) {
  Integrator* b = c->integ;
  if (!b) { llg_set_error("time_kernel needs an initialised integrator"); return LLG_ERR_STATE; }
  cudaEvent_t e0, e1;
  LLG_CUDA_TRY(cudaEventCreate(&e0));
  LLG_CUDA_TRY(cudaEventCreate(&e1));
  const double* Y6[6] = {b->zn[0], b->zn[1], b->V[0], b->V[1], b->ewt, b->y};
  double cf[6] = {1.0, 0.5, -0.25, 0.125, 1.0, 2.0};
  auto once = [&]() -> int {
    switch (kid) {
      case KID_RHS: return launch_rhs(c, b->y, c->d_hd, b->tempv);
      case KID_JTV: return launch_jtv(c, b->V[0], b->tempv, b->y);
      case KID_ARNOLDI:
        if (!c->have_setup) return LLG_ERR_STATE;
        return b->kf32 ? launch_arnoldi_op_f(c, b->Vf(0), b->ewt, b->Vf(1), b->y, b->gamma, nullptr)
                       : launch_arnoldi_op(c, b->V[0], b->ewt, b->tempv, b->y, b->gamma);
      case KID_PSETUP: return launch_psetup(c, b->y, c->gamma_setup);
      case KID_PSOLVE: return c->have_setup ? launch_psolve(c, b->V[0], b->tempv) : LLG_ERR_STATE;
      case KID_NORM: return launch_normalize(c, b->tempv);
      case KID_DEMAG_ROWS_FWD: return demag_stage(c, 0, b->y, b->tempv);
      case KID_DEMAG_COLS: return demag_stage(c, 1, b->y, b->tempv);
      case KID_DEMAG_ROWS_INV: return demag_stage(c, 2, b->y, b->tempv);
      case KID_REDUCE: return vdot_multi_dev(c, 6, b->V[0], Y6, 8);
      case KID_ELEMWISE: return vlincomb(c, 6, cf, Y6, b->tempv);
      default: return LLG_ERR_NOTSUP;
    }
  };
  int rc = once();  // warm-up
  if (rc) { cudaEventDestroy(e0); cudaEventDestroy(e1); return rc; }
  cudaEventRecord(e0, c->stream);
  for (int i = 0; i < iters && !rc; i++) rc = once();
  cudaEventRecord(e1, c->stream);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *avg_ms = (double)ms / iters;
  return rc;
}

int integrator_stats(llg_ctx* c, llg_stats* st) {
  memset(st, 0, sizeof(*st));
  st->nfe_demag = c->nfe_demag;
  Integrator* b = c->integ;
  if (!b) return 0;
  st->nst = b->nst; st->nfe = b->nfe; st->nsetups = b->nsetups; st->nni = b->nni;
  st->ncfn = b->ncfn; st->netf = b->netf; st->nli = b->nli; st->nlcf = b->nlcf;
  st->njvevals = b->njv; st->npsolves = b->nps; st->npe = b->npe;
  st->qlast = b->qu; st->qcur = b->next_q; st->hlast = b->hu; st->hcur = b->next_h; st->tcur = b->tn;
  return 0;
}

int devint_trace(DevInteg* d, llg_ctx* c, unsigned long long* dbuf, int cap);
int devint_trace_count(DevInteg* d);

int integrator_trace(llg_ctx* c, unsigned long long* buf, int cap) {
  Integrator* b = c->integ;
  if (!b || !b->dev || !b->dev_current) {
    llg_set_error("trace_control needs a device-resident integrator that has run once");
    return LLG_ERR_STATE;
  }
  return devint_trace(b->dev, c, buf, cap);
}

int integrator_trace_count(llg_ctx* c) {
  Integrator* b = c->integ;
  return (b && b->dev) ? devint_trace_count(b->dev) : 0;
}

// ── step-sequence record / replay ───────────────────────────────────────
int integrator_record_steps(llg_ctx* c, int cap) {
  Integrator* b = c->integ;
  if (!b) { llg_set_error("record_steps needs llg_integrator_init first"); return LLG_ERR_STATE; }
  b->rec_cap = cap > 0 ? cap : 0;
  b->rec_h.clear();
  b->rec_q.clear();
  if (cap > 0) { b->rec_h.reserve(cap); b->rec_q.reserve(cap); }
  return 0;
}

int integrator_recorded_steps(llg_ctx* c, double* h, int32_t* q, int cap) {
  Integrator* b = c->integ;
  if (!b) { llg_set_error("recorded_steps needs llg_integrator_init first"); return LLG_ERR_STATE; }
  const int n = (int)b->rec_h.size();
  for (int i = 0; i < n && i < cap; i++) {
    if (h) h[i] = b->rec_h[i];
    if (q) q[i] = b->rec_q[i];
  }
  return n;
}

int integrator_replay_steps(llg_ctx* c, const double* h, const int32_t* q, int n) {
  Integrator* b = c->integ;
  if (!b) { llg_set_error("replay_steps needs llg_integrator_init first"); return LLG_ERR_STATE; }
  if (n <= 0) { b->replay = false; b->rp_h.clear(); b->rp_q.clear(); return 0; }
  if (!h || !q) { llg_set_error("replay_steps: null sequence"); return LLG_ERR_ARG; }
  if (b->started || b->nst != 0) {
    llg_set_error("replay_steps must be set before the first llg_integrate call");
    return LLG_ERR_STATE;
  }
  if (q[0] != 1) { llg_set_error("replay_steps: the first step of a BDF run has order 1"); return LLG_ERR_ARG; }
  for (int i = 0; i < n; i++) {
    if (!(h[i] != 0.0) || !isfinite(h[i]) || q[i] < 1 || q[i] > b->qmax || (i > 0 && abs(q[i] - q[i - 1]) > 1)) {
      llg_set_error("replay_steps: entry " + std::to_string(i) + " is not a valid (h, q) step");
      return LLG_ERR_ARG;
    }
  }
  b->rp_h.assign(h, h + n);
  b->rp_q.assign(q, q + n);
  b->replay = true;
  b->replay_forced = 0;
  return 0;
}

int integrator_replay_status(llg_ctx* c, int32_t* position, int64_t* forced) {
  Integrator* b = c->integ;
  if (!b) { llg_set_error("replay_status needs llg_integrator_init first"); return LLG_ERR_STATE; }
  if (position) *position = (int32_t)b->nst;
  if (forced) *forced = b->replay_forced;
  return 0;
}

// ── checkpoint / restart ────────────────────────────────────────────────
// Blob: CkptHeader | CkptScalars | FP64 vectors, each neq long, in this order:
// zn[0..qmax], acor, h_demag, and when a preconditioner setup exists the
// frozen m, h and the 9 planes of the stored block inverse (3 vectors).  The
// header's checksum covers everything after the header.
namespace {
constexpr char CKPT_MAGIC[8] = {'L', 'L', 'G', 'C', 'K', 'P', 'T', '1'};
constexpr uint32_t CKPT_VERSION = 1;

struct CkptScalars {
#define LLG_CK_D(f) double f;
#define LLG_CK_I(f) int f;
#define LLG_CK_LL(f) long long f;
  LLG_DS_DOUBLES(LLG_CK_D)
  LLG_DS_INTS(LLG_CK_I)
  LLG_DS_LLS(LLG_CK_LL)
#undef LLG_CK_D
#undef LLG_CK_I
#undef LLG_CK_LL
  double l[QMAXL + 2], tq[6], tau[QMAXL + 2];
};

uint64_t ckpt_hash(const unsigned char* p, uint64_t n) {
  // FNV-1a over 8-byte words (then the tail bytes)
  uint64_t hsh = 1469598103934665603ull;
  uint64_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t w;
    memcpy(&w, p + i, 8);
    hsh = (hsh ^ w) * 1099511628211ull;
  }
  for (; i < n; i++) hsh = (hsh ^ p[i]) * 1099511628211ull;
  return hsh;
}

uint64_t ckpt_nvec(const llg_ckpt_info& h) { return (uint64_t)h.qmax + 1 + 2 + (h.have_setup ? 5 : 0); }

int ckpt_check(const void* buf, uint64_t n, llg_ckpt_info* out) {
  if (!buf || n < sizeof(llg_ckpt_info)) {
    llg_set_error("checkpoint: buffer shorter than its header");
    return LLG_ERR_ARG;
  }
  llg_ckpt_info hd;
  memcpy(&hd, buf, sizeof(hd));
  if (memcmp(hd.magic, CKPT_MAGIC, 8) != 0) { llg_set_error("checkpoint: bad magic"); return LLG_ERR_ARG; }
  if (hd.version != CKPT_VERSION || hd.header_bytes != sizeof(llg_ckpt_info) ||
      hd.scalar_bytes != sizeof(CkptScalars)) {
    llg_set_error("checkpoint: version or layout of another build");
    return LLG_ERR_ARG;
  }
  if (hd.ng <= 0 || hd.ny <= 0 || hd.neq != 3ll * hd.ng * hd.ny || hd.qmax < 1 || hd.qmax > QMAXL ||
      hd.maxl < 1 || hd.maxl > MAXLL - 1) {
    llg_set_error("checkpoint: inconsistent header");
    return LLG_ERR_ARG;
  }
  const uint64_t payload = sizeof(CkptScalars) + ckpt_nvec(hd) * 8ull * (uint64_t)hd.neq;
  if (hd.payload_bytes != payload || n < sizeof(hd) + payload) {
    llg_set_error("checkpoint: truncated or wrongly sized buffer");
    return LLG_ERR_ARG;
  }
  const unsigned char* p = static_cast<const unsigned char*>(buf) + sizeof(hd);
  if (ckpt_hash(p, payload) != hd.checksum) { llg_set_error("checkpoint: checksum mismatch"); return LLG_ERR_ARG; }
  if (out) *out = hd;
  return 0;
}
}  // namespace

extern "C" int llg_checkpoint_inspect(const void* buf, uint64_t n, llg_ckpt_info* info) {
  return ckpt_check(buf, n, info);
}

int integrator_checkpoint_size(llg_ctx* c, uint64_t* bytes) {
  Integrator* b = c->integ;
  if (!b) { llg_set_error("checkpoint needs llg_integrator_init first"); return LLG_ERR_STATE; }
  llg_ckpt_info hd{};
  hd.qmax = b->qmax;
  hd.have_setup = c->have_setup;
  *bytes = sizeof(llg_ckpt_info) + sizeof(CkptScalars) + ckpt_nvec(hd) * 8ull * (uint64_t)b->neq;
  return 0;
}

int integrator_checkpoint_save(llg_ctx* c, void* buf, uint64_t cap, uint64_t* written) {
  Integrator* b = c->integ;
  if (!b) { llg_set_error("checkpoint needs llg_integrator_init first"); return LLG_ERR_STATE; }
  b->materialise();
  if (b->err) { llg_set_error("checkpoint: the integrator is in an error state"); return LLG_ERR_STATE; }
  if (learned_active(c)) {
    llg_set_error("checkpoint: a learned-preconditioner context is not checkpointed (save its weights instead)");
    return LLG_ERR_NOTSUP;
  }
  uint64_t need = 0;
  integrator_checkpoint_size(c, &need);
  if (!buf || cap < need) { llg_set_error("checkpoint: buffer too small"); return LLG_ERR_ARG; }
  llg_ckpt_info hd{};
  memcpy(hd.magic, CKPT_MAGIC, 8);
  hd.version = CKPT_VERSION;
  hd.header_bytes = sizeof(llg_ckpt_info);
  hd.scalar_bytes = sizeof(CkptScalars);
  hd.krylov_precision = b->kf32 ? LLG_KRYLOV_FP32 : LLG_KRYLOV_FP64;
  hd.ng = c->p.ng;
  hd.ny = c->p.ny;
  hd.neq = b->neq;
  hd.qmax = b->qmax;
  hd.maxl = b->maxl;
  hd.classical_gs = b->classical_gs;
  hd.mxstep = b->mxstep;
  hd.device_resident = b->device_resident;
  hd.have_setup = c->have_setup;
  hd.rtol = b->rtol;
  hd.atol = b->atol;
  hd.gamma_setup = c->gamma_setup;
  hd.tn = b->tn;
  hd.nst = b->nst;
  hd.nfe_demag = c->nfe_demag;
  hd.params = c->p;
  CkptScalars sc{};
#define LLG_CK_OUT(f) sc.f = b->f;
  LLG_DS_DOUBLES(LLG_CK_OUT)
  LLG_DS_INTS(LLG_CK_OUT)
  LLG_DS_LLS(LLG_CK_OUT)
#undef LLG_CK_OUT
  memcpy(sc.l, b->l, sizeof(sc.l));
  memcpy(sc.tq, b->tq, sizeof(sc.tq));
  memcpy(sc.tau, b->tau, sizeof(sc.tau));
  unsigned char* p = static_cast<unsigned char*>(buf);
  unsigned char* q = p + sizeof(hd);
  memcpy(q, &sc, sizeof(sc));
  q += sizeof(sc);
  const size_t vb = 8ull * (size_t)b->neq;
  b->materialise_acor();
  std::vector<const double*> src;
  for (int j = 0; j <= b->qmax; j++) src.push_back(b->zn[j]);
  src.push_back(b->acor);
  src.push_back(c->d_hd);
  if (c->have_setup) {
    src.push_back(c->d_pm);
    src.push_back(c->d_ph);
    for (int k = 0; k < 3; k++) src.push_back(c->d_pinv + (size_t)k * b->neq);
  }
  for (const double* d : src) {
    LLG_CUDA_TRY(cudaMemcpyAsync(q, d, vb, cudaMemcpyDeviceToHost, c->stream));
    q += vb;
  }
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  hd.payload_bytes = (uint64_t)(q - p) - sizeof(hd);
  hd.checksum = ckpt_hash(p + sizeof(hd), hd.payload_bytes);
  memcpy(p, &hd, sizeof(hd));
  if (written) *written = (uint64_t)(q - p);
  return 0;
}

int integrator_checkpoint_load(llg_ctx* c, const void* buf, uint64_t n) {
  llg_ckpt_info hd;
  int rc = ckpt_check(buf, n, &hd);
  if (rc) return rc;
  if (hd.ng != c->p.ng || hd.ny != c->p.ny) {
    llg_set_error("checkpoint: grid of another problem");
    return LLG_ERR_ARG;
  }
  if (memcmp(&hd.params, &c->p, sizeof(llg_params)) != 0) {
    llg_set_error("checkpoint: physics parameters differ from this context's");
    return LLG_ERR_ARG;
  }
  llg_solver_opts o{};
  o.rtol = hd.rtol;
  o.atol = hd.atol;
  o.maxl = hd.maxl;
  o.maxord = hd.qmax;
  o.gs_type = hd.classical_gs ? LLG_GS_CLASSICAL : LLG_GS_MODIFIED;
  o.mxstep = hd.mxstep;
  o.device_resident = hd.device_resident;
  o.krylov_precision = (int32_t)hd.krylov_precision;
  rc = integrator_create(c, hd.tn, nullptr, &o);
  if (rc) return rc;
  Integrator* b = c->integ;
  const unsigned char* q = static_cast<const unsigned char*>(buf) + sizeof(hd);
  CkptScalars sc;
  memcpy(&sc, q, sizeof(sc));
  q += sizeof(sc);
#define LLG_CK_IN(f) b->f = sc.f;
  LLG_DS_DOUBLES(LLG_CK_IN)
  LLG_DS_INTS(LLG_CK_IN)
  LLG_DS_LLS(LLG_CK_IN)
#undef LLG_CK_IN
  memcpy(b->l, sc.l, sizeof(sc.l));
  memcpy(b->tq, sc.tq, sizeof(sc.tq));
  memcpy(b->tau, sc.tau, sizeof(sc.tau));
  const size_t vb = 8ull * (size_t)b->neq;
  std::vector<double*> dst;
  for (int j = 0; j <= b->qmax; j++) dst.push_back(b->zn[j]);
  dst.push_back(b->acor);
  dst.push_back(c->d_hd);
  if (hd.have_setup) {
    dst.push_back(c->d_pm);
    dst.push_back(c->d_ph);
    for (int k = 0; k < 3; k++) dst.push_back(c->d_pinv + (size_t)k * b->neq);
  }
  for (double* d : dst) {
    LLG_CUDA_TRY(cudaMemcpyAsync(d, q, vb, cudaMemcpyHostToDevice, c->stream));
    q += vb;
  }
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  // (a learned-preconditioner context restarts on the FP64 basis: an FP32
  // block inverse saved after its hand-over is not used, the next step sets up)
  c->have_setup = (c->pinv_f32 == (hd.krylov_precision == LLG_KRYLOV_FP32 ? 1 : 0)) ? hd.have_setup : 0;
  c->gamma_setup = hd.gamma_setup;
  c->nfe_demag = hd.nfe_demag;
  b->ycor_zero = false;
  return 0;
}

// ── batch graph support (batch.cpp) ─────────────────────────────────────
// An instance joins a batch graph once its host-driven start is done (the
// initial step size and first step run on the host) and its settings are
// covered by the device-resident form.
int integrator_batch_prepare(llg_ctx* c, DevInteg** d_out, DState* hs_out) {
  Integrator* b = c->integ;
  if (!b) { llg_set_error("batch graph: llg_batch_integrator_init first"); return LLG_ERR_STATE; }
  if (!b->started) {
    llg_set_error("batch graph: advance the batch once with llg_batch_integrate (host start-up) first");
    return LLG_ERR_STATE;
  }
  const bool dr = b->device_resident;
  b->device_resident = 1;
  const bool ok_dev = b->device_applies();
  b->device_resident = dr;
  if (!ok_dev) {
    llg_set_error("batch graph: an instance uses a setting the device-resident step graph does not cover "
                  "(modified Gram-Schmidt, learned preconditioner, harvesting, replay/recording, a source "
                  "term, the demag-derivative Jacobian or an FP32 Krylov basis)");
    return LLG_ERR_NOTSUP;
  }
  if (!b->dev) {
    const int rc = devint_create(c, &b->dev);
    if (rc) return rc;
  }
  devint_mark_batched(b->dev);
  b->materialise();
  b->export_state(*hs_out);
  *d_out = b->dev;
  return 0;
}

// the device copy of the state, current (after the graph was built)
int integrator_batch_sync(llg_ctx* c) {
  Integrator* b = c->integ;
  if (b->dev_current) return 0;
  b->materialise();
  DState hs;
  b->export_state(hs);
  const int rc = devint_upload(b->dev, hs, c);
  if (rc) return rc;
  b->dev_current = true;
  return 0;
}

int integrator_batch_finish(llg_ctx* c, const DState& hs, double* tret) {
  Integrator* b = c->integ;
  b->y_ready = false;
  b->import_state(hs);
  *tret = hs.tret;
  return hs.status;
}
