// integrator_dev.cu — the device-resident form of the BDF/Newton/SPGMR
// integrator (llg_solver_opts.device_resident = 1).
//
// The host-driven integrator (integrator.cu) makes every decision of a CVODE
// step on the CPU: it reads back a norm or a set of Gram–Schmidt dots,
// decides, and launches the next kernel — six to eight round trips per BDF
// step, each leaving the GPU idle for the read-back and the next launch.
// Here the same decisions run on the GPU:
//
//   * DState (dev_integ.h) holds the integrator's scalar state in device
//     memory;
//   * k_ctl runs one segment of the scalar logic (one thread) between vector
//     kernels — the same formulas as integrator.cu, in the same order;
//   * the loops and branches of a step (step loop, retry loop, Newton
//     iterations, GMRES iterations, reorthogonalisation, failure recovery)
//     are CUDA graph conditional nodes (WHILE / IF) whose conditions k_ctl
//     sets with cudaGraphSetConditional;
//   * kernels whose coefficients change from step to step read them from
//     DState (the vector kernels below, and DevArgs in the physics / fused
//     kernels); kernels whose arguments are fixed are the host path's own.
//
// One llg_integrate call = one small parameter kernel + one graph launch +
// one read-back of DState.  The host path still performs the first call
// (start-up: initial step size, first step) and is used where the device
// form does not apply (harvesting training pairs for the learned
// preconditioner).  Every handle of a conditional node is set by a control
// kernel in that node's own graph or in a body nested inside it.
#include <float.h>
#include <math.h>
#include <string.h>

#include <functional>
#include <vector>

#include "llg_internal.h"
#include "launch.h"
#include "cvode_consts.h"
#include "dev_reduce.cuh"

namespace {

constexpr int NSTREAM = 8;   // capture streams, one per nesting depth

// ───────────────────────── scalar logic (device) ─────────────────────────

__device__ double d_powr(double b, double e) { return (b <= 0.0) ? 0.0 : pow(b, e); }
__device__ double d_powi(double b, int e) {
  double p = 1.0;
  for (int i = 1; i <= (e < 0 ? -e : e); i++) p *= b;
  return e < 0 ? 1.0 / p : p;
}
__device__ double wrms_of(const DState& s, double v) { return sqrt(v / (double)s.neq); }
__device__ void setc(DState& s, int h, int v) { cudaGraphSetConditional(s.hnd[h], v ? 1u : 0u); }

__device__ void set_bdf(DState& s) {
  double alpha0, alpha0_hat, xi_inv, xistar_inv, hsum;
  const int q = s.q;
  s.l[0] = s.l[1] = xi_inv = xistar_inv = 1.0;
  for (int i = 2; i <= q; i++) s.l[i] = 0.0;
  alpha0 = alpha0_hat = -1.0;
  hsum = s.h;
  if (q > 1) {
    for (int j = 2; j < q; j++) {
      hsum += s.tau[j - 1];
      xi_inv = s.h / hsum;
      alpha0 -= 1.0 / j;
      for (int i = j; i >= 1; i--) s.l[i] += s.l[i - 1] * xi_inv;
    }
    alpha0 -= 1.0 / q;
    xistar_inv = -s.l[1] - alpha0;
    hsum += s.tau[q - 1];
    xi_inv = s.h / hsum;
    alpha0_hat = -s.l[1] - xi_inv;
    for (int i = q; i >= 1; i--) s.l[i] += s.l[i - 1] * xistar_inv;
  }
  const double A1 = 1.0 - alpha0_hat + alpha0;
  const double A2 = 1.0 + q * A1;
  s.tq[2] = fabs(A1 / (alpha0 * A2));
  s.tq[5] = fabs(A2 * xistar_inv / (s.l[q] * xi_inv));
  if (s.qwait == 1) {
    if (q > 1) {
      const double C = xistar_inv / s.l[q];
      const double A3 = alpha0 + 1.0 / q;
      const double A4 = alpha0_hat + xi_inv;
      const double Cpinv = (1.0 - A4 + A3) / A3;
      s.tq[1] = fabs(C * Cpinv);
    } else {
      s.tq[1] = 1.0;
    }
    hsum += s.tau[q];
    xi_inv = s.h / hsum;
    const double A5 = alpha0 - (1.0 / (q + 1));
    const double A6 = alpha0_hat - xi_inv;
    const double Cppinv = (1.0 - A6 + A5) / A2;
    s.tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
  }
  s.tq[4] = CORTES / s.tq[2];
}

__device__ void cv_set(DState& s) {
  set_bdf(s);
  s.rl1 = 1.0 / s.l[1];
  s.gamma = s.h * s.rl1;
  if (s.nst == 0) s.gammap = s.gamma;
  s.gamrat = (s.nst > 0) ? s.gamma / s.gammap : 1.0;
}

__device__ int qr_fact(DState& s, int n) {
  const int n1 = n - 1;
  int code = 0;
  for (int k = 0; k < n1; k++) {
    const int i = 2 * k;
    const double t1 = s.Hes[k][n1], t2 = s.Hes[k + 1][n1];
    const double cc = s.givens[i], sn = s.givens[i + 1];
    s.Hes[k][n1] = cc * t1 - sn * t2;
    s.Hes[k + 1][n1] = sn * t1 + cc * t2;
  }
  const double t1 = s.Hes[n1][n1], t2 = s.Hes[n][n1];
  double cc, sn;
  if (t2 == 0.0) { cc = 1.0; sn = 0.0; }
  else if (fabs(t2) >= fabs(t1)) { const double t3 = t1 / t2; sn = -1.0 / sqrt(1.0 + t3 * t3); cc = -sn * t3; }
  else { const double t3 = t2 / t1; cc = 1.0 / sqrt(1.0 + t3 * t3); sn = -cc * t3; }
  s.givens[2 * n1] = cc;
  s.givens[2 * n1 + 1] = sn;
  if ((s.Hes[n1][n1] = cc * t1 - sn * t2) == 0.0) code = n;
  return code;
}

__device__ int qr_sol(DState& s, int n, double* bb) {
  int code = 0;
  for (int k = 0; k < n; k++) {
    const double cc = s.givens[2 * k], sn = s.givens[2 * k + 1];
    const double t1 = bb[k], t2 = bb[k + 1];
    bb[k] = cc * t1 - sn * t2;
    bb[k + 1] = sn * t1 + cc * t2;
  }
  for (int k = n - 1; k >= 0; k--) {
    if (s.Hes[k][k] == 0.0) { code = k + 1; break; }
    bb[k] /= s.Hes[k][k];
    for (int i = 0; i < k; i++) bb[i] -= bb[k] * s.Hes[i][k];
  }
  return code;
}

// zn[j] *= eta^j (j = 1..q) at the next predict
__device__ void rescale(DState& s) {
  double factor = s.eta;
  if (s.rescale_pending) {
    for (int j = 1; j <= s.q; j++) { s.pf[j] *= factor; factor *= s.eta; }
  } else {
    for (int j = 1; j <= s.q; j++) { s.pf[j] = factor; factor *= s.eta; }
  }
  s.rescale_pending = 1;
  s.h = s.hscale * s.eta;
  s.next_h = s.h;
  s.hscale = s.h;
  s.nscon = 0;
}

__device__ void increase_bdf(DState& s) {
  double alpha0, alpha1, prod, xi, xiold, hsum, A1;
  for (int i = 0; i <= s.qmax; i++) s.l[i] = 0.0;
  s.l[2] = alpha1 = prod = xiold = 1.0;
  alpha0 = -1.0;
  hsum = s.hscale;
  if (s.q > 1) {
    for (int j = 1; j < s.q; j++) {
      hsum += s.tau[j + 1];
      xi = hsum / s.hscale;
      prod *= xi;
      alpha0 -= 1.0 / (j + 1);
      alpha1 += 1.0 / xi;
      for (int i = j + 2; i >= 2; i--) s.l[i] = s.l[i] * xiold + s.l[i - 1];
      xiold = xi;
    }
  }
  A1 = (-alpha0 - alpha1) / prod;
  s.ord_type = 1;
  s.ord_q = s.q;
  s.ord_A1 = A1;
  for (int j = 0; j <= DS_QMAXL + 1; j++) s.ord_l[j] = s.l[j];
}

__device__ void decrease_bdf(DState& s) {
  double hsum, xi;
  for (int i = 0; i <= s.qmax; i++) s.l[i] = 0.0;
  s.l[2] = 1.0;
  hsum = 0.0;
  for (int j = 1; j <= s.q - 2; j++) {
    hsum += s.tau[j];
    xi = hsum / s.hscale;
    for (int i = j + 2; i >= 2; i--) s.l[i] = s.l[i] * xi + s.l[i - 1];
  }
  s.ord_type = 2;
  s.ord_q = s.q;
  for (int j = 0; j <= DS_QMAXL + 1; j++) s.ord_l[j] = s.l[j];
}

// returns 1 when an order-change kernel must run
__device__ int adjust_order(DState& s, int dq) {
  if (s.q == 2 && dq != 1) return 0;
  if (dq == 1) { increase_bdf(s); return 1; }
  if (dq == -1) { decrease_bdf(s); return 1; }
  return 0;
}

__device__ void set_eta(DState& s) {
  if (s.eta < THRESH) {
    s.eta = 1.0;
    s.hprime = s.h;
  } else {
    s.eta = (s.eta < s.etamax) ? s.eta : s.etamax;
    const double d = fabs(s.h) * s.hmax_inv * s.eta;
    s.eta /= (d > 1.0 ? d : 1.0);
    s.hprime = s.h * s.eta;
    if (s.qprime < s.q) s.nscon = 0;
  }
}

// returns 1 when acor must be copied into zn[qmax]
__device__ int choose_eta(DState& s) {
  double etam = s.etaqm1 > s.etaq ? s.etaqm1 : s.etaq;
  etam = etam > s.etaqp1 ? etam : s.etaqp1;
  if (etam < THRESH) { s.eta = 1.0; s.qprime = s.q; return 0; }
  if (etam == s.etaq) { s.eta = s.etaq; s.qprime = s.q; }
  else if (etam == s.etaqm1) { s.eta = s.etaqm1; s.qprime = s.q - 1; }
  else { s.eta = s.etaqp1; s.qprime = s.q + 1; return 1; }
  return 0;
}

__device__ int nls_ctest(DState& s, double s0, double s1, double tol, int m) {
  const double dn = wrms_of(s, s0);
  if (m > 0) {
    const double r = dn / s.delp;
    s.crate = (CRDOWN * s.crate > r) ? CRDOWN * s.crate : r;
  }
  const double dcon = dn * (s.crate < 1.0 ? s.crate : 1.0) / tol;
  if (dcon <= 1.0) {
    s.acnrm = (m == 0) ? dn : wrms_of(s, s1);
    return 0;
  }
  if ((m >= 1) && (dn > RDIV * s.delp)) return NLS_CONV_RECVR;
  s.delp = dn;
  return NLS_CONTINUE;
}

// end of one Newton pass (integrator.cu newton(): retry once with a fresh
// preconditioner setup when a recoverable failure used a stale one)
__device__ void newton_end(DState& s) {
  if (s.retval > 0 && !s.jcur_nls) {
    s.call_setup = 1;
    s.jbad = 1;
    s.ycor_zero = 1;
    s.da.ycor_zero = 1;
    s.newton_first = 1;
    setc(s, H_NEWTON, 1);
  } else {
    setc(s, H_NEWTON, 0);
  }
}

// Krylov iteration bookkeeping at the start of iteration s.li
__device__ void iter_begin(DState& s) {
  s.nl++;
  s.krydim = s.li + 1;
  s.njv++;
  s.nps++;
  s.da.arn_in = s.V[s.li];
  s.da.arn_out = s.V[s.li + 1];
}

// end of one Arnoldi iteration with h_{l+1,l} = nrm
__device__ void iter_end(DState& s, double nrm) {
  const int l = s.li;
  s.Hes[l + 1][l] = nrm;
  if (qr_fact(s, s.krydim) != 0) {
    s.nli += s.nl;
    s.gm_fail = 1;
    setc(s, H_GMITER, 0);
    return;
  }
  s.rot *= s.givens[2 * l + 1];
  s.rho = fabs(s.rot * s.rnorm);
  if (s.rho <= s.dtol) {
    s.converged = 1;
    setc(s, H_GMITER, 0);
    return;
  }
  s.sc = 1.0 / s.Hes[l + 1][l];
  s.li = l + 1;
  if (s.li >= s.maxl) { setc(s, H_GMITER, 0); return; }
  iter_begin(s);
  setc(s, H_GMITER, 1);
}

__device__ void count_resid(DState& s) {
  s.kcount[KID_NORM]++;
  if (s.has_demag) {
    s.kcount[KID_DEMAG_ROWS_FWD]++;
    s.kcount[KID_DEMAG_COLS]++;
    s.kcount[KID_DEMAG_ROWS_INV]++;
    s.nfe_demag++;
  }
  s.kcount[KID_RHS]++;
}

// The reorthogonalisation test of classical Gram-Schmidt: the predicated
// second-pass kernels and the control op evaluate the same expression on the
// same stored values, so they agree.
__device__ __forceinline__ bool reorth_needed(const DState* s) {
  const int k = s->li + 1;
  return GS_FACTOR * sqrt(s->scal[SLOT_A]) < sqrt(s->scal[SLOT_DOTS + k]);
}

// Control ops, in graph order.  One WHILE(H_LOOP) iteration is one attempt
// at a step; one WHILE(H_NEWTON) iteration is one Newton iteration (residual,
// optional preconditioner setup, SPGMR solve, update, convergence test); one
// WHILE(H_GMITER) iteration is one Arnoldi iteration.  Every other branch of
// the host integrator is a kernel that reads its own run flag from DState and
// returns at once when it is not set (a skipped kernel costs a launch; an IF
// node costs several) except the failure path, which sits behind one IF.
enum CtlOp {
  OP_CALL_BEGIN = 0, OP_ATTEMPT, OP_RESID_DONE, OP_GM_BEGIN, OP_GS_END, OP_GM_END, OP_CTEST, OP_NLS_END,
  OP_FAIL_BEGIN, OP_PREP_END, OP_CALL_END, OP_COUNT
};

// Every control op counts against a per-call bound.  Past it (a state the
// step logic cannot reach: mxstep, MXNCF, MXNEF, NLS_MAXCOR and maxl bound
// every loop), the call ends with LLG_ERR_TIMEOUT: each op then clears the
// conditions it owns and every run flag, so every WHILE node of the graph
// exits within one pass.
__device__ void trip_clear(DState& s, int op) {
  s.run_predict = s.ord_run = s.small = s.lcdiv = 0;
  s.f_acor0 = s.f_restore = s.f_decr = s.f_q1f = s.f_sam = s.f_cpy1 = s.f_w2 = s.f_cpy2 = s.f_dky = 0;
  s.da.run_setup = s.da.run_ewt = s.da.run_update = 0;
  switch (op) {
    case OP_CALL_BEGIN: case OP_PREP_END: setc(s, H_LOOP, 0); break;
    case OP_ATTEMPT: case OP_CTEST: setc(s, H_NEWTON, 0); break;
    case OP_GM_BEGIN: case OP_GS_END: setc(s, H_GMITER, 0); break;
    case OP_NLS_END: setc(s, H_FAIL, 0); break;
    case OP_FAIL_BEGIN: setc(s, H_Q1F, 0); break;
    case OP_CALL_END: s.f_copyy = 1; break;
    default: break;
  }
}

static_assert(sizeof(DState) % 8 == 0, "DState is staged in 8-byte words");

__device__ void ctl_exec(DState& s, int op);

// One warp stages DState in shared memory (coalesced, independent loads),
// lane 0 runs the scalar logic there, the warp writes it back: the logic's
// long dependent chains then hit shared memory instead of L2.
__global__ void __launch_bounds__(32) k_ctl(DState* sp, int op) {
  __shared__ DState S;
  constexpr int NW = (int)(sizeof(DState) / 8);
  long long* dst = reinterpret_cast<long long*>(&S);
  const long long* src = reinterpret_cast<const long long*>(sp);
  for (int i = threadIdx.x; i < NW; i += 32) dst[i] = src[i];
  __syncwarp();
  if (threadIdx.x == 0) ctl_exec(S, op);
  __syncwarp();
  long long* back = reinterpret_cast<long long*>(sp);
  for (int i = threadIdx.x; i < NW; i += 32) back[i] = dst[i];
}

__device__ void ctl_exec(DState& s, int op) {
  s.kcount[KID_OTHER]++;
  if (s.trace && s.trace_n < s.trace_cap) {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    s.trace[s.trace_n++] = (t << 5) | (unsigned long long)op;
  }
  if (!s.tripped && ++s.guard_count > s.guard_max) {
    s.tripped = 1;
    s.status = LLG_ERR_TIMEOUT;
    s.tret = s.tn;
  }
  if (s.tripped) {
    trip_clear(s, op);
    return;
  }
  double* sc = s.scal;
  switch (op) {
    case OP_CALL_BEGIN: {
      s.status = 0;
      s.nstloc = 0;
      s.f_copyy = 0;
      s.f_dky = 0;
      s.dky = 0;
      s.new_step = 1;
      s.da.run_ewt = 1;
      int loop = 1;
      if ((s.tn - s.tout) * s.h >= 0.0) { s.dky = 1; s.tret = s.tout; loop = 0; s.da.run_ewt = 0; }
      setc(s, H_LOOP, loop);
      break;
    }
    case OP_ATTEMPT: {   // top of an attempt: step checks and order change (new step), predict
      s.ord_run = 0;
      if (s.new_step) {
        s.kcount[KID_REDUCE]++;   // ewt + ||zn0||
        s.next_h = s.h;
        s.next_q = s.q;
        const double bad = sc[SLOT_A], ssum = sc[SLOT_A + 1];
        int stop = 0;
        if (bad != 0.0) { s.status = LLG_CV_ILL_INPUT; stop = 1; }
        const double nrm = wrms_of(s, ssum);
        if (!stop && (s.mxstep > 0) && (s.nstloc >= s.mxstep)) { s.status = LLG_CV_TOO_MUCH_WORK; stop = 1; }
        if (!stop && !isfinite(nrm)) { s.status = LLG_CV_BAD_STATE; stop = 1; }
        if (!stop && UROUND * nrm > 1.0) { s.status = LLG_CV_TOO_MUCH_ACC; stop = 1; }
        if (stop) {
          s.f_copyy = 1;
          s.tret = s.tn;
          s.run_predict = 0;
          setc(s, H_NEWTON, 0);
          break;
        }
        // cv_step start
        s.saved_t = s.tn;
        s.ncf = s.nef = 0;
        s.nflag = FIRST_CALL;
        s.dsm = 0.0;
        if ((s.nst > 0) && (s.hprime != s.h)) {   // adjust_params
          if (s.qprime != s.q) {
            s.ord_run = adjust_order(s, s.qprime - s.q);
            s.q = s.qprime;
            s.L = s.q + 1;
            s.qwait = s.L;
          }
          rescale(s);
        }
        if (s.ord_run) s.kcount[KID_ELEMWISE]++;
      }
      // predict (the kernel follows) and cv_set / cv_nls set-up
      s.run_predict = 1;
      s.kcount[KID_ELEMWISE]++;
      s.tn += s.h;
      cv_set(s);
      const int nflag = s.nflag;
      s.convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL)) ? CV_NO_FAILURES : CV_FAIL_OTHER;
      s.call_setup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL) || (s.nst == 0) ||
                     (s.nst >= s.nstlp + MSBP) || (fabs(s.gamrat - 1.0) > DGMAX);
      s.ycor_zero = 1;
      s.jbad = 0;
      s.retval = 0;
      s.newton_first = 1;
      s.da.ycor_zero = 1;
      s.da.rl1 = s.rl1;
      s.da.gamma = s.gamma;
      setc(s, H_NEWTON, 1);
      break;
    }
    case OP_RESID_DONE: {   // after the residual of a Newton iteration
      s.rescale_pending = 0;   // the predict of this attempt applied it
      s.nfe++;
      count_resid(s);
      s.da.run_setup = 0;
      if (s.newton_first) {
        if (s.call_setup) {   // nls_lsetup (the psetup kernel follows)
          if (s.jbad) s.convfail = CV_FAIL_BAD_J;
          s.kcount[KID_PSETUP]++;
          s.npe++;
          s.nstlj = s.nst;
          s.jcur = 1;
          s.nsetups++;
          s.jcur_nls = s.jcur;
          s.gamrat = 1.0;
          s.gammap = s.gamma;
          s.crate = 1.0;
          s.nstlp = s.nst;
          s.da.gamma_setup = s.gamma;
          s.have_setup = 1;
          s.da.run_setup = 1;
        }
        s.m = 0;
        s.newton_first = 0;
      }
      break;
    }
    case OP_GM_BEGIN: {
      s.kcount[KID_PSOLVE]++;
      s.nni++;
      s.ls_curiter = s.m;
      const double deltar = LS_EPLIN * s.tq[4];
      s.dtol = deltar * sqrt((double)s.neq);
      s.nli0_pol = s.nli;
      s.nps++;
      const double ss = sc[SLOT_A];
      s.beta = sqrt(ss);
      s.rnorm = s.rho = s.beta;
      s.nl = 0;
      s.krydim = 0;
      s.converged = 0;
      s.gm_fail = 0;
      s.lcdiv = 0;
      s.li = 0;
      if (s.rnorm <= s.dtol) {
        s.small = 1;
        s.lres = LS_SUCCESS;
        s.kcount[KID_ELEMWISE]++;
        setc(s, H_GMITER, 0);
        break;
      }
      s.small = 0;
      for (int i = 0; i <= s.maxl; i++)
        for (int j = 0; j < s.maxl; j++) s.Hes[i][j] = 0.0;
      s.rot = 1.0;
      s.sc = 1.0 / s.rnorm;
      iter_begin(s);
      setc(s, H_GMITER, 1);
      break;
    }
    case OP_GS_END: {   // classical Gram-Schmidt of V[k], k = li + 1 (and its second pass)
      s.kcount[KID_ELEMWISE]++;   // scale V[li]
      s.kcount[KID_ARNOLDI]++;
      s.kcount[KID_REDUCE] += 2;  // dots + update
      const int k = s.li + 1;
      const double* dots = sc + SLOT_DOTS;
      s.vk_norm = sqrt(dots[k]);
      for (int i = 0; i < k; i++) s.Hes[i][k - 1] = dots[i];
      double nrm = sqrt(sc[SLOT_A]);
      if (reorth_needed(&s)) {
        s.kcount[KID_REDUCE] += 2;
        const double* d2 = sc + SLOT_DOTS2;
        for (int i = 0; i < k; i++) s.Hes[i][k - 1] += d2[i];
        nrm = sqrt(sc[SLOT_A2]);
      }
      iter_end(s, nrm);
      break;
    }
    case OP_GM_END: {
      if (!s.small && !s.gm_fail) {
        s.nli += s.nl;
        s.yg[0] = s.rnorm;
        for (int i = 1; i <= s.krydim; i++) s.yg[i] = 0.0;
        if (qr_sol(s, s.krydim, s.yg) != 0) {
          s.lres = LS_QRSOL_FAIL;
        } else if (s.converged || s.rho < s.beta) {
          s.lcdiv = 1;
          s.kcount[KID_ELEMWISE]++;
          s.lres = s.converged ? LS_SUCCESS : LS_RES_REDUCED;
        } else {
          s.lres = LS_CONV_FAIL;
        }
      } else if (s.gm_fail) {
        s.lres = LS_CONV_FAIL;
      }
      if (s.lres != LS_SUCCESS) s.nlcf++;
      int r;
      if (s.lres == LS_SUCCESS) r = 0;
      else if (s.lres == LS_RES_REDUCED) r = (s.ls_curiter == 0) ? 0 : 1;
      else r = 1;
      s.retval = r;
      s.da.run_update = (r == 0);
      if (r == 0) s.kcount[KID_REDUCE]++;   // update + norms
      break;
    }
    case OP_CTEST: {   // Newton convergence test; decides the next Newton iteration
      if (!s.da.run_update) {   // the linear solve failed
        newton_end(s);
        break;
      }
      s.ycor_zero = 0;
      s.da.ycor_zero = 0;
      const int r = nls_ctest(s, sc[SLOT_A], sc[SLOT_A + 1], s.tq[4], s.m);
      if (r == 0) {
        s.jcur_nls = 0;
        s.retval = 0;
        setc(s, H_NEWTON, 0);
        break;
      }
      if (r != NLS_CONTINUE) {
        s.retval = r;
        newton_end(s);
        break;
      }
      s.m++;
      if (s.m >= NLS_MAXCOR) {
        s.retval = NLS_CONV_RECVR;
        newton_end(s);
        break;
      }
      setc(s, H_NEWTON, 1);   // next iteration: residual at the updated correction
      break;
    }
    case OP_NLS_END: {
      s.f_acor0 = s.f_restore = s.f_decr = s.f_q1f = s.f_sam = s.f_cpy1 = s.f_w2 = 0;
      s.attempt_again = 0;
      s.need_wrms2 = 0;
      if (s.status != 0) {   // stopped before the attempt
        setc(s, H_FAIL, 0);
        break;
      }
      const int flag = s.retval;
      int fail = 0, ok = 0;
      if (flag != 0) {
        if (s.ycor_zero) { s.f_acor0 = 1; s.ycor_zero = 0; s.kcount[KID_ELEMWISE]++; }
      } else {
        s.jcur = 0;
      }
      s.nflag = flag;
      if (flag != 0) {   // handle_nflag
        s.ncfn++;
        s.f_restore = 1;
        s.res_q = s.q;
        s.tn = s.saved_t;
        s.ncf++;
        s.etamax = 1.0;
        if ((fabs(s.h) <= s.hmin * ONEPSM) || (s.ncf == MXNCF)) {
          s.status = LLG_CV_CONV_FAILURE;
          fail = 1;
        } else {
          s.eta = (ETACF > s.hmin / fabs(s.h)) ? ETACF : s.hmin / fabs(s.h);
          s.nflag = PREV_CONV_FAIL;
          rescale(s);
          s.attempt_again = 1;
        }
      } else {   // error test
        const double dsm = s.acnrm * s.tq[2];
        s.dsm = dsm;
        if (dsm <= 1.0) {
          ok = 1;
        } else {
          s.nef++;
          s.netf++;
          s.nflag = PREV_ERR_FAIL;
          s.f_restore = 1;
          s.res_q = s.q;
          s.tn = s.saved_t;
          if ((fabs(s.h) <= s.hmin * ONEPSM) || (s.nef == MXNEF)) {
            s.status = LLG_CV_ERR_FAILURE;
            fail = 1;
          } else {
            s.etamax = 1.0;
            s.attempt_again = 1;
            if (s.nef <= MXNEF1) {
              double e = 1.0 / (d_powr(BIAS2 * dsm, 1.0 / s.L) + ADDON);
              const double lo = s.hmin / fabs(s.h);
              e = (e > lo) ? e : lo;
              e = (e > ETAMIN) ? e : ETAMIN;
              if (s.nef >= SMALL_NEF) e = (e < ETAMXF) ? e : ETAMXF;
              s.eta = e;
              rescale(s);
            } else if (s.q > 1) {
              s.eta = (ETAMIN > s.hmin / fabs(s.h)) ? ETAMIN : s.hmin / fabs(s.h);
              s.f_decr = adjust_order(s, -1);
              s.L = s.q;
              s.q--;
              s.qwait = s.L;
              rescale(s);
            } else {
              s.eta = (ETAMIN > s.hmin / fabs(s.h)) ? ETAMIN : s.hmin / fabs(s.h);
              s.h *= s.eta;
              s.next_h = s.h;
              s.hscale = s.h;
              s.qwait = LONG_WAIT;
              s.nscon = 0;
              s.nfe++;
              s.f_q1f = 1;
              count_resid(s);
              s.kcount[KID_ELEMWISE]++;
            }
          }
        }
      }
      if (s.f_restore) s.kcount[KID_ELEMWISE]++;
      if (s.f_decr) s.kcount[KID_ELEMWISE]++;
      if (fail) {
        s.f_copyy = 1;
        s.tret = s.tn;
      } else if (ok) {
        // complete_step (the kernel follows)
        s.nst++;
        s.nscon++;
        s.hu = s.h;
        s.qu = s.q;
        for (int i = s.q; i >= 2; i--) s.tau[i] = s.tau[i - 1];
        if ((s.q == 1) && (s.nst > 1)) s.tau[2] = s.tau[1];
        s.tau[1] = s.h;
        s.f_sam = 1;
        s.kcount[KID_ELEMWISE]++;
        s.qwait--;
        if ((s.qwait == 1) && (s.q != s.qmax)) {
          s.f_cpy1 = 1;
          s.kcount[KID_ELEMWISE]++;
          s.saved_tq5 = s.tq[5];
          s.indx_acor = s.qmax;
        }
        // prepare_next, up to the norms it needs
        if (s.etamax == 1.0) {
          s.qwait = s.qwait > 2 ? s.qwait : 2;
          s.qprime = s.q;
          s.hprime = s.h;
          s.eta = 1.0;
        } else {
          s.etaq = 1.0 / (d_powr(BIAS2 * s.dsm, 1.0 / s.L) + ADDON);
          if (s.qwait != 0) {
            s.eta = s.etaq;
            s.qprime = s.q;
            set_eta(s);
          } else {
            s.qwait = 2;
            s.need_wrms2 = 1;
            s.cquot = (s.saved_tq5 != 0.0) ? (s.tq[5] / s.saved_tq5) * d_powi(s.h / s.tau[2], s.L) : 0.0;
            s.f_w2 = 1;
            s.kcount[KID_REDUCE]++;
          }
        }
      }
      setc(s, H_FAIL, s.f_acor0 || s.f_restore || s.f_decr || s.f_q1f);
      break;
    }
    case OP_FAIL_BEGIN: {
      setc(s, H_Q1F, s.f_q1f);
      break;
    }
    case OP_PREP_END: {
      s.f_cpy2 = 0;
      s.da.run_ewt = 0;
      if (s.status != 0) {
        setc(s, H_LOOP, 0);
        break;
      }
      if (s.attempt_again) {   // retry this step
        s.new_step = 0;
        setc(s, H_LOOP, 1);
        break;
      }
      if (s.need_wrms2) {
        s.etaqm1 = 0.0;
        if (s.q > 1) {
          const double ddn = wrms_of(s, sc[SLOT_A]) * s.tq[1];
          s.etaqm1 = 1.0 / (d_powr(BIAS1 * ddn, 1.0 / s.q) + ADDON);
        }
        s.etaqp1 = 0.0;
        if (s.q != s.qmax && s.saved_tq5 != 0.0) {
          const double dup = wrms_of(s, sc[SLOT_A + 1]) * s.tq[3];
          s.etaqp1 = 1.0 / (d_powr(BIAS3 * dup, 1.0 / (s.L + 1)) + ADDON);
        }
        s.f_cpy2 = choose_eta(s);
        if (s.f_cpy2) s.kcount[KID_ELEMWISE]++;
        set_eta(s);
      }
      s.etamax = (s.nst <= SMALL_NST) ? ETAMX2 : ETAMX3;
      s.nstloc++;
      s.new_step = 1;
      if ((s.tn - s.tout) * s.h >= 0.0) {
        s.tret = s.tout;
        s.dky = 1;
        s.next_q = s.qprime;
        s.next_h = s.hprime;
        setc(s, H_LOOP, 0);
      } else {
        s.da.run_ewt = 1;
        setc(s, H_LOOP, 1);
      }
      break;
    }
    case OP_CALL_END: {
      s.f_dky = 0;
      if (s.dky && s.status == 0) {
        // get_dky(tout)
        double tfuzz = FUZZ_FACTOR * UROUND * (fabs(s.tn) + fabs(s.hu));
        if (s.hu < 0.0) tfuzz = -tfuzz;
        const double tp = s.tn - s.hu - tfuzz;
        const double tn1 = s.tn + tfuzz;
        if ((s.tout - tp) * (s.tout - tn1) > 0.0) {
          s.status = LLG_CV_ILL_INPUT;
        } else {
          const double sv = (s.tout - s.tn) / s.h;
          int nv = 0;
          for (int j = s.q; j >= 0; j--) {
            double cc = 1.0;
            for (int i = 0; i < j; i++) cc *= sv;
            s.dky_c[nv++] = cc;
          }
          s.dky_nv = nv;
          s.f_dky = 1;
          s.kcount[KID_ELEMWISE]++;
        }
      }
      if (s.f_copyy) s.kcount[KID_ELEMWISE]++;
      break;
    }
    default:
      break;
  }
}

__global__ void k_call_args(DState* s, double tout, double* yout, long long limit) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    s->tout = tout;
    s->yout = yout;
    s->guard_count = 0;
    s->trace_n = 0;
    s->guard_max = limit > 0 ? limit : 200LL * ((s->mxstep > 0 ? s->mxstep : 500) + 10) * (s->maxl + 4);
    s->tripped = 0;
    for (int k = 0; k < 16; k++) s->kcount[k] = 0;
  }
}

// ───────────────────── vector kernels with device coefficients ─────────────
// Each applies, element by element, the same arithmetic as the host path's
// kernel for that update (k_vector.cu / k_fused.cu), with the coefficients,
// the vector count and the vector choice read from DState, and returns at
// once when its run flag is clear.

template <int Q>
__device__ __forceinline__ void nordsieck_at(double* const* zp, const double* f, int pend, int sign, long long i) {
  double v[Q + 1];
#pragma unroll
  for (int j = 0; j <= Q; j++) v[j] = zp[j][i];
  if (pend) {
#pragma unroll
    for (int j = 1; j <= Q; j++) v[j] = f[j] * v[j];
  }
#pragma unroll
  for (int k = 1; k <= Q; k++)
#pragma unroll
    for (int j = Q; j >= k; j--) v[j - 1] = (sign > 0) ? v[j - 1] + v[j] : v[j - 1] - v[j];
#pragma unroll
  for (int j = 0; j < Q; j++) zp[j][i] = v[j];
  if (pend) zp[Q][i] = v[Q];
}

// predict (sign +1, applying a pending rescale first) or restore (sign -1)
__global__ void k_d_nordsieck(DState* s, int sign, long long n) {
  if (!(sign > 0 ? s->run_predict : s->f_restore)) return;
  const int q = (sign > 0) ? s->q : s->res_q;
  const int pend = (sign > 0) ? s->rescale_pending : 0;
  double f[DS_QMAXL + 1];
  double* zp[DS_QMAXL + 1];
  for (int j = 0; j <= DS_QMAXL; j++) { f[j] = s->pf[j]; zp[j] = s->zn[j]; }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    switch (q) {
      case 1: nordsieck_at<1>(zp, f, pend, sign, i); break;
      case 2: nordsieck_at<2>(zp, f, pend, sign, i); break;
      case 3: nordsieck_at<3>(zp, f, pend, sign, i); break;
      case 4: nordsieck_at<4>(zp, f, pend, sign, i); break;
      default: nordsieck_at<5>(zp, f, pend, sign, i); break;
    }
  }
}

// order change (which 0: at a step start, 1: after error-test failures):
// increase (zn[q+1] = A1 zn[indx_acor]; zn[j] += l_j zn[q+1]) or decrease
// (zn[j] += -l_j zn[q]), q the order before the change
__global__ void k_d_order(DState* s, int which, long long n) {
  if (!(which == 0 ? s->ord_run : s->f_decr)) return;
  const int type = s->ord_type, q = s->ord_q;
  double* zp[DS_QMAXL + 1];
  for (int j = 0; j <= DS_QMAXL; j++) zp[j] = s->zn[j];
  double lj[DS_QMAXL + 2];
  for (int j = 0; j <= DS_QMAXL + 1; j++) lj[j] = s->ord_l[j];
  const double A1 = s->ord_A1;
  const double* src = s->zn[s->indx_acor];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (type == 1) {
      const double t = A1 * src[i];
      zp[q + 1][i] = t;
      for (int j = 2; j <= q; j++) zp[j][i] = lj[j] * t + 1.0 * zp[j][i];
    } else {
      const double zq = zp[q][i];
      for (int j = 2; j < q; j++) zp[j][i] = (-lj[j]) * zq + 1.0 * zp[j][i];
    }
  }
}

// V[li] = sc V[li]
__global__ void k_d_scale_v(DState* s, long long n) {
  const double a = s->sc;
  double* z = s->V[s->li];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = a * z[i];
}

// dots of V[k] (k = li + 1) with V[0..nv-1]; pass 0: nv = k + 1 into SLOT_DOTS
// (classical GS), pass 1: nv = k into SLOT_DOTS2, only when reorthogonalising
__global__ void __launch_bounds__(RT) k_d_dots(DState* s, int pass, long long n, double* partials,
                                              unsigned int* counter) {
  if (pass == 1 && !reorth_needed(s)) return;
  __shared__ double sm[(DS_MAXLL + 1) * (RT / 32)];
  const int k = s->li + 1;
  const int nv = (pass == 0) ? k + 1 : k;
  const double* x = s->V[k];
  const double* Y[DS_MAXLL + 1];
#pragma unroll
  for (int j = 0; j <= DS_MAXLL; j++) Y[j] = (j < nv) ? s->V[j] : nullptr;
  double acc[DS_MAXLL + 1];
#pragma unroll
  for (int j = 0; j <= DS_MAXLL; j++) acc[j] = 0.0;
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double xi = x[i];
#pragma unroll
    for (int j = 0; j <= DS_MAXLL; j++)
      if (j < nv) acc[j] += xi * Y[j][i];
  }
  // block sums of the first nv accumulators (the tree of block_sum<K>)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j <= DS_MAXLL; j++) {
    if (j < nv) {
      const double v = warp_sum(acc[j]);
      if (lane == 0) sm[j * (RT / 32) + wid] = v;
    }
  }
  __syncthreads();
  if (wid == 0) {
#pragma unroll
    for (int j = 0; j <= DS_MAXLL; j++) {
      if (j < nv) {
        const double v = (lane < RT / 32) ? sm[j * (RT / 32) + lane] : 0.0;
        acc[j] = warp_sum(v);
      }
    }
  }
  __shared__ bool last;
  double* out = s->scal + (pass == 0 ? SLOT_DOTS : SLOT_DOTS2);
  const int nb = gridDim.x;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j <= DS_MAXLL; j++)
      if (j < nv) partials[j * nb + blockIdx.x] = acc[j];
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int j = 0; j < nv; j++) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += RT) v += ((volatile double*)partials)[j * nb + b];
    const double w = warp_sum(v);
    __syncthreads();
    if (lane == 0) sm[wid] = w;
    __syncthreads();
    if (wid == 0) {
      double u = (lane < RT / 32) ? sm[lane] : 0.0;
      u = warp_sum(u);
      if (lane == 0) out[j] = u;
    }
  }
  if (threadIdx.x == 0) *counter = 0u;
}

// V[k] = 1 V[k] + sum_{i<k} (-dots_i) V[i], and sum V[k]^2 (pass 0: dots of
// SLOT_DOTS, norm to SLOT_A; pass 1: SLOT_DOTS2 to SLOT_A2, when reorthogonalising)
__global__ void __launch_bounds__(RT) k_d_gs_update(DState* s, int pass, long long n, double* partials,
                                                   unsigned int* counter) {
  if (pass == 1 && !reorth_needed(s)) return;
  __shared__ double sm[RT / 32];
  const int k = s->li + 1;
  const int nv = k;
  const double* dots = s->scal + (pass == 0 ? SLOT_DOTS : SLOT_DOTS2);
  double cf[DS_MAXLL];
  const double* X[DS_MAXLL];
#pragma unroll
  for (int j = 0; j < DS_MAXLL; j++) {
    cf[j] = (j < nv) ? -dots[j] : 0.0;
    X[j] = (j < nv) ? s->V[j] : nullptr;
  }
  double* z = s->V[k];
  double acc[1] = {0.0};
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    double v = 1.0 * z[i];
#pragma unroll
    for (int j = 0; j < DS_MAXLL; j++)
      if (j < nv) v = cf[j] * X[j][i] + v;
    z[i] = v;
    acc[0] += v * v;
  }
  block_sum<1>(acc, sm);
  finalize<1>(partials, gridDim.x, counter, s->scal + (pass == 0 ? SLOT_A : SLOT_A2), 0, 1.0, acc);
}

// del = (sum_k yg_k V[k]) / ewt, k < krydim
__global__ void k_d_lincomb_div(DState* s, long long n) {
  if (!s->lcdiv) return;
  const int nv = s->krydim;
  double cf[DS_MAXLL];
  const double* X[DS_MAXLL];
#pragma unroll
  for (int j = 0; j < DS_MAXLL; j++) {
    cf[j] = (j < nv) ? s->yg[j] : 0.0;
    X[j] = (j < nv) ? s->V[j] : nullptr;
  }
  const double* w = s->ewt;
  double* z = s->delta;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = cf[0] * X[0][i];
#pragma unroll
    for (int j = 1; j < DS_MAXLL; j++)
      if (j < nv) v = cf[j] * X[j][i] + v;
    z[i] = v / w[i];
  }
}

// zn[j] = l_j acor + zn[j], j = 0..q
__global__ void k_d_complete(DState* s, long long n) {
  if (!s->f_sam) return;
  const int nv = s->q + 1;
  double a[DS_QMAXL + 1];
  double* Z[DS_QMAXL + 1];
#pragma unroll
  for (int j = 0; j <= DS_QMAXL; j++) { a[j] = s->l[j]; Z[j] = s->zn[j]; }
  const double* x = s->acor;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double xi = x[i];
#pragma unroll
    for (int j = 0; j <= DS_QMAXL; j++)
      if (j < nv) Z[j][i] = a[j] * xi + Z[j][i];
  }
}

// zn[qmax] = acor (which 0: in complete_step, 1: when the next order is q + 1)
__global__ void k_d_save_acor(DState* s, int which, long long n) {
  if (!(which == 0 ? s->f_cpy1 : s->f_cpy2)) return;
  const double* x = s->acor;
  double* z = s->zn[s->qmax];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = x[i];
}

// sums (zn[q] w)^2 and ((-cquot zn[qmax] + acor) w)^2
__global__ void __launch_bounds__(RT) k_d_wrms2(DState* s, long long n, double* partials, unsigned int* counter) {
  if (!s->f_w2) return;
  __shared__ double sm[2 * (RT / 32)];
  const double* x1 = s->zn[s->q];
  const double a = -s->cquot;
  const double* x2 = s->zn[s->qmax];
  const double b = 1.0;
  const double* x3 = s->acor;
  const double* w = s->ewt;
  double acc[2] = {0.0, 0.0};
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    const double wi = w[i];
    const double p = x1[i] * wi;
    const double v = a * x2[i] + b * x3[i];
    const double q = v * wi;
    acc[0] += p * p;
    acc[1] += q * q;
  }
  block_sum<2>(acc, sm);
  finalize<2>(partials, gridDim.x, counter, s->scal + SLOT_A, 0, 1.0, acc);
}

// yout = sum_k c_k zn[q - k] (get_dky), or yout = zn[0] (a call that stopped)
__global__ void k_d_output(DState* s, long long n) {
  double* z = s->yout;
  if (s->f_copyy) {
    const double* x = s->zn[0];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      z[i] = x[i];
    return;
  }
  if (!s->f_dky) return;
  const int nv = s->dky_nv;
  const int q = s->q;
  double cf[DS_QMAXL + 1];
  const double* X[DS_QMAXL + 1];
#pragma unroll
  for (int j = 0; j <= DS_QMAXL; j++) {
    cf[j] = (j < nv) ? s->dky_c[j] : 0.0;
    X[j] = (j < nv) ? s->zn[q - j] : nullptr;
  }
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = cf[0] * X[0][i];
#pragma unroll
    for (int j = 1; j <= DS_QMAXL; j++)
      if (j < nv) v = cf[j] * X[j][i] + v;
    z[i] = v;
  }
}

// zn[1] = h tempv (order-1 error-test recovery)
__global__ void k_d_scale_h(DState* s, long long n) {
  const double a = s->h;
  const double* x = s->tempv;
  double* z = s->zn[1];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = a * x[i];
}

// which 0: del = 0 (the residual is already below the tolerance); 1: acor = 0
__global__ void k_d_zero(DState* s, int which, long long n) {
  if (!(which == 0 ? s->small : s->f_acor0)) return;
  double* z = (which == 0) ? s->delta : s->acor;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    z[i] = 0.0;
}

}  // namespace

// ───────────────────────────── graph builder ─────────────────────────────


struct DevInteg {
  DState* d_s = nullptr;        // device state
  DState* h_s = nullptr;        // pinned mirror (read-back)
  cudaGraphExec_t exec = nullptr;
  cudaStream_t cap[NSTREAM] = {};
  cudaGraphConditionalHandle hnd[H_COUNT] = {};
  int depth = 0;
  long long neq = 0;
  bool batched = false;         // its step loop lives in a batch graph (no graph of its own)
};

namespace {

struct Builder {
  llg_ctx* c;
  DevInteg* d;
  const DState& hs;   // host copy: buffer pointers and fixed settings
  int rc = 0;
  Builder(llg_ctx* c_, DevInteg* d_, const DState& hs_) : c(c_), d(d_), hs(hs_) {}
  void ok(int r) {
    if (r && !rc) rc = r;
  }
  bool cu(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
      if (!rc) {
        llg_set_error(std::string("device-resident graph: ") + what + ": " + cudaGetErrorString(e));
        rc = LLG_ERR_CUDA;
      }
      return false;
    }
    return true;
  }
  cudaStream_t st() const { return d->cap[d->depth]; }
  int ew() const {
    long long g = (d->neq + 255) / 256;
    const long long cap = (long long)c->num_sms * 8;
    return (int)(g > cap ? cap : (g < 1 ? 1 : g));
  }
  int rb() const { return red_blocks(d->neq); }
  DState* S() const { return d->d_s; }
  const DevArgs* DA() const { return &d->d_s->da; }
  void launched(const char* what) { cu(cudaPeekAtLastError(), what); }
  void ctl(int op) {
    k_ctl<<<1, 32, 0, st()>>>(S(), op);
    launched("control kernel");
  }
  // conditional node in the graph being captured on st(); fill(i) captures body i
  void cond(int hid, cudaGraphConditionalNodeType type, unsigned nbody, const std::function<void(int)>& fill) {
    if (rc) return;
    cudaStream_t s = st();
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    if (!cu(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd), "capture info")) return;
    cudaGraphConditionalHandle h;
    if (!cu(cudaGraphConditionalHandleCreate(&h, g, 0, 0), "conditional handle")) return;
    d->hnd[hid] = h;
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = nbody;
    cudaGraphNode_t node;
    if (!cu(cudaGraphAddNode(&node, g, deps, nd, &p), "conditional node")) return;
    if (!cu(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies), "capture deps"))
      return;
    cudaGraph_t bodies[2] = {p.conditional.phGraph_out[0], nbody > 1 ? p.conditional.phGraph_out[1] : nullptr};
    for (unsigned i = 0; i < nbody && !rc; i++) {
      if (d->depth + 1 >= NSTREAM) {
        llg_set_error("device-resident graph: conditional nesting too deep");
        rc = LLG_ERR_STATE;
        return;
      }
      d->depth++;
      cudaStream_t bs = st();
      if (!cu(cudaStreamBeginCaptureToGraph(bs, bodies[i], nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
              "body capture")) {
        d->depth--;
        return;
      }
      cudaStream_t saved = c->stream;
      c->stream = bs;
      fill((int)i);
      c->stream = saved;
      cudaGraph_t outg = nullptr;
      const cudaError_t e = cudaStreamEndCapture(bs, &outg);
      d->depth--;
      cu(e, "body end capture");
    }
  }
  void IF(int hid, const std::function<void()>& body) {
    cond(hid, cudaGraphCondTypeIf, 1, [&](int) { body(); });
  }
  void WHILE(int hid, const std::function<void()>& body) {
    cond(hid, cudaGraphCondTypeWhile, 1, [&](int) { body(); });
  }

  void emit() {
    const long long n = d->neq;
    DState* s = S();
    double* red = c->d_red;
    unsigned int* cnt = c->d_counter;
    const int EW = ew(), RB = rb();
    ctl(OP_CALL_BEGIN);
    WHILE(H_LOOP, [&] {   // one attempt at a step
      ok(fused_ewt_wrms(c, hs.rtol, hs.atol, hs.zn[0], hs.ewt, SLOT_A, DA()));
      ctl(OP_ATTEMPT);
      k_d_order<<<EW, 256, 0, st()>>>(s, 0, n);
      launched("order change");
      k_d_nordsieck<<<EW, 256, 0, st()>>>(s, +1, n);
      launched("predict");
      WHILE(H_NEWTON, [&] {   // one Newton iteration
        ok(fused_lin_normalize(c, hs.zn[0], hs.acor, hs.y, DA()));
        ok(fused_field(c, hs.y));
        ok(fused_resid(c, hs.y, hs.zn[1], hs.acor, 0.0, 0.0, hs.delta, DA()));
        ctl(OP_RESID_DONE);
        ok(launch_psetup(c, hs.y, 0.0, DA()));
        ok(fused_psolve_scale_dot(c, hs.delta, hs.ewt, hs.V[0], SLOT_A, DA()));
        ctl(OP_GM_BEGIN);
        k_d_zero<<<EW, 256, 0, st()>>>(s, 0, n);
        launched("zero");
        WHILE(H_GMITER, [&] {   // one Arnoldi iteration
          k_d_scale_v<<<EW, 256, 0, st()>>>(s, n);
          launched("scale");
          ok(launch_arnoldi_op(c, nullptr, hs.ewt, nullptr, hs.y, 0.0, 1, DA()));
          for (int pass = 0; pass < 2; pass++) {
            k_d_dots<<<RB, RT, 0, st()>>>(s, pass, n, red, cnt);
            launched("dots");
            k_d_gs_update<<<RB, RT, 0, st()>>>(s, pass, n, red, cnt);
            launched("gram-schmidt update");
          }
          ctl(OP_GS_END);
        });
        ctl(OP_GM_END);
        k_d_lincomb_div<<<EW, 256, 0, st()>>>(s, n);
        launched("correction");
        ok(fused_update_wrms2(c, false, hs.acor, hs.delta, hs.ewt, SLOT_A, DA()));
        ctl(OP_CTEST);
      });
      ctl(OP_NLS_END);
      IF(H_FAIL, [&] {
        ctl(OP_FAIL_BEGIN);
        k_d_zero<<<EW, 256, 0, st()>>>(s, 1, n);
        launched("zero");
        k_d_nordsieck<<<EW, 256, 0, st()>>>(s, -1, n);
        launched("restore");
        k_d_order<<<EW, 256, 0, st()>>>(s, 1, n);
        launched("order change");
        IF(H_Q1F, [&] {
          ok(rhs_full(c, 0.0, hs.zn[0], hs.tempv));
          k_d_scale_h<<<EW, 256, 0, st()>>>(s, n);
          launched("scale");
        });
      });
      k_d_complete<<<EW, 256, 0, st()>>>(s, n);
      launched("complete step");
      k_d_save_acor<<<EW, 256, 0, st()>>>(s, 0, n);
      launched("save acor");
      k_d_wrms2<<<RB, RT, 0, st()>>>(s, n, red, cnt);
      launched("norms");
      ctl(OP_PREP_END);
      k_d_save_acor<<<EW, 256, 0, st()>>>(s, 1, n);
      launched("save acor");
    });
    ctl(OP_CALL_END);
    k_d_output<<<EW, 256, 0, st()>>>(s, n);
    launched("output");
  }
};

// Capture one instance's step loop into graph g as a new independent branch
// (no dependencies on what g already holds).
int capture_into(DevInteg* d, llg_ctx* c, const DState& hs, cudaGraph_t g) {
  // the capture runs the host wrappers once; keep what they record on the host
  const double gs_saved = c->gamma_setup;
  const int hv_saved = c->have_setup;
  const long long nd_saved = c->nfe_demag;
  cudaStream_t saved = c->stream;
  d->depth = 0;
  cudaError_t e = cudaStreamBeginCaptureToGraph(d->cap[0], g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    llg_set_error(std::string("device-resident graph: begin capture: ") + cudaGetErrorString(e));
    return LLG_ERR_CUDA;
  }
  c->stream = d->cap[0];
  c->capturing = 1;
  g_count_off = 1;
  const int pdl_saved = g_no_pdl;
  g_no_pdl = 1;
  Builder b(c, d, hs);
  b.emit();
  g_no_pdl = pdl_saved;
  g_count_off = 0;
  c->capturing = 0;
  c->stream = saved;
  c->gamma_setup = gs_saved;
  c->have_setup = hv_saved;
  c->nfe_demag = nd_saved;
  cudaGraph_t outg = nullptr;
  e = cudaStreamEndCapture(d->cap[0], &outg);
  if (b.rc) return b.rc;
  if (e != cudaSuccess) {
    llg_set_error(std::string("device-resident graph: end capture: ") + cudaGetErrorString(e));
    return LLG_ERR_CUDA;
  }
  return 0;
}

int build_graph(DevInteg* d, llg_ctx* c, const DState& hs) {
  cudaGraph_t g = nullptr;
  LLG_CUDA_TRY(cudaGraphCreate(&g, 0));
  const int rc = capture_into(d, c, hs, g);
  if (rc) { cudaGraphDestroy(g); return rc; }
  cudaError_t e = cudaGraphInstantiate(&d->exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    d->exec = nullptr;
    llg_set_error(std::string("device-resident graph: instantiate: ") + cudaGetErrorString(e));
    return LLG_ERR_CUDA;
  }
  return 0;
}

}  // namespace

int devint_create(llg_ctx* c, DevInteg** out) {
  DevInteg* d = new DevInteg();
  d->neq = c->neq;
  int rc = 0;
  if (cudaMalloc(&d->d_s, sizeof(DState)) != cudaSuccess ||
      cudaMallocHost(&d->h_s, sizeof(DState)) != cudaSuccess) {
    llg_set_error("device-resident integrator: allocation failed");
    rc = LLG_ERR_CUDA;
  }
  for (int i = 0; i < NSTREAM && !rc; i++)
    if (cudaStreamCreateWithFlags(&d->cap[i], cudaStreamNonBlocking) != cudaSuccess) {
      llg_set_error("device-resident integrator: stream creation failed");
      rc = LLG_ERR_CUDA;
    }
  if (rc) { devint_destroy(d); return rc; }
  *out = d;
  return 0;
}

void devint_destroy(DevInteg* d) {
  if (!d) return;
  if (d->exec) cudaGraphExecDestroy(d->exec);
  for (auto& s : d->cap)
    if (s) cudaStreamDestroy(s);
  cudaFree(d->d_s);
  if (d->h_s) cudaFreeHost(d->h_s);
  delete d;
}

int devint_upload(DevInteg* d, const DState& hs_in, llg_ctx* c) {
  if (!d->exec && !d->batched) {
    const int rc = build_graph(d, c, hs_in);
    if (rc) return rc;
  }
  *d->h_s = hs_in;
  for (int k = 0; k < H_COUNT; k++) d->h_s->hnd[k] = d->hnd[k];
  d->h_s->scal = c->d_scal;
  d->h_s->rescale_pending = 0;
  for (int j = 0; j <= DS_QMAXL + 1; j++) d->h_s->pf[j] = 1.0;
  d->h_s->da.gamma_setup = c->gamma_setup;
  d->h_s->have_setup = c->have_setup;
  d->h_s->has_demag = c->demag != nullptr;
  d->h_s->nfe_demag = c->nfe_demag;
  LLG_CUDA_TRY(cudaMemcpyAsync(d->d_s, d->h_s, sizeof(DState), cudaMemcpyHostToDevice, c->stream));
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return 0;
}

int devint_run(DevInteg* d, llg_ctx* c, double tout, double* yout, DState& hs) {
  k_call_args<<<1, 1, 0, c->stream>>>(d->d_s, tout, yout, c->ctl_limit);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  LLG_CUDA_TRY(cudaGraphLaunch(d->exec, c->stream));
  LLG_CUDA_TRY(cudaMemcpyAsync(d->h_s, d->d_s, sizeof(DState), cudaMemcpyDeviceToHost, c->stream));
  LLG_CUDA_TRY(cudaMemcpyAsync(c->h_scal + SLOT_TCERR, c->d_scal + SLOT_TCERR, sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream));
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  hs = *d->h_s;
  g_kcount[KID_OTHER].fetch_add(1, std::memory_order_relaxed);   // k_call_args
  for (int k = 0; k < KID_COUNT && k < 16; k++) g_kcount[k].fetch_add(hs.kcount[k], std::memory_order_relaxed);
  c->gamma_setup = hs.da.gamma_setup;
  c->have_setup = hs.have_setup;
  c->nfe_demag = hs.nfe_demag;
  return 0;
}

// ── batches: the step loops of many instances in ONE graph ───────────────
// Conditional nodes cannot live in child graphs, so each instance's WHILE /
// IF structure is captured directly into the shared graph as an independent
// branch; one cudaGraphLaunch then advances every instance to its tout, the
// branches running concurrently on the device with no host work between
// steps.  Each instance keeps its own DState, conditional handles, buffers
// and capture streams.
int devint_mark_batched(DevInteg* d) {
  d->batched = true;
  return 0;
}

int devint_build_batch(llg_ctx* const* cs, DevInteg* const* ds, const DState* const* hss, int n,
                       cudaGraphExec_t* exec) {
  cudaGraph_t g = nullptr;
  LLG_CUDA_TRY(cudaGraphCreate(&g, 0));
  for (int i = 0; i < n; i++) {
    const int rc = capture_into(ds[i], cs[i], *hss[i], g);
    if (rc) { cudaGraphDestroy(g); return rc; }
  }
  const cudaError_t e = cudaGraphInstantiate(exec, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    *exec = nullptr;
    llg_set_error(std::string("batch graph: instantiate: ") + cudaGetErrorString(e));
    return LLG_ERR_CUDA;
  }
  return 0;
}

// per call: set tout / yout of one instance on stream s (before the launch)
int devint_batch_args(DevInteg* d, llg_ctx* c, double tout, double* yout, cudaStream_t s) {
  k_call_args<<<1, 1, 0, s>>>(d->d_s, tout, yout, c->ctl_limit);
  LLG_CUDA_TRY(cudaPeekAtLastError());
  return 0;
}

// per call: bring one instance's state home on stream s (after the launch)
int devint_batch_fetch(DevInteg* d, llg_ctx* c, cudaStream_t s) {
  LLG_CUDA_TRY(cudaMemcpyAsync(d->h_s, d->d_s, sizeof(DState), cudaMemcpyDeviceToHost, s));
  LLG_CUDA_TRY(cudaMemcpyAsync(c->h_scal + SLOT_TCERR, c->d_scal + SLOT_TCERR, sizeof(double), cudaMemcpyDeviceToHost,
                               s));
  return 0;
}

// after the stream synchronised: the instance's final state (as devint_run)
int devint_batch_collect(DevInteg* d, llg_ctx* c, DState& hs) {
  hs = *d->h_s;
  g_kcount[KID_OTHER].fetch_add(1, std::memory_order_relaxed);   // k_call_args
  for (int k = 0; k < KID_COUNT && k < 16; k++) g_kcount[k].fetch_add(hs.kcount[k], std::memory_order_relaxed);
  c->gamma_setup = hs.da.gamma_setup;
  c->have_setup = hs.have_setup;
  c->nfe_demag = hs.nfe_demag;
  return 0;
}

// profiling aid: record (op, time) of each control op into a device buffer
int devint_trace(DevInteg* d, llg_ctx* c, unsigned long long* dbuf, int cap) {
  DState hs;
  LLG_CUDA_TRY(cudaMemcpyAsync(&hs, d->d_s, sizeof(DState), cudaMemcpyDeviceToHost, c->stream));
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  hs.trace = dbuf;
  hs.trace_cap = cap;
  hs.trace_n = 0;
  LLG_CUDA_TRY(cudaMemcpyAsync(d->d_s, &hs, sizeof(DState), cudaMemcpyHostToDevice, c->stream));
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return 0;
}
int devint_trace_count(DevInteg* d) { return d->h_s ? d->h_s->trace_n : 0; }
