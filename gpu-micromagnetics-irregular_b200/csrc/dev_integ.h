// dev_integ.h — state of the device-resident integrator (llg_solver_opts.
// device_resident = 1).
//
// The BDF/Newton/SPGMR step control of integrator.cu runs on the GPU: its
// scalar state lives in one DState in device memory, single-thread control
// kernels (integrator_dev.cu, k_ctl) execute the scalar logic between the
// vector kernels, and the branches and loops of a CVODE step are CUDA graph
// conditional nodes (WHILE / IF) whose conditions those control kernels set.
// One llg_integrate call is one graph launch plus one read-back of the step
// counters; nothing waits on the host between BDF steps.
//
// DevArgs is the part of DState that the physics and fused kernels read
// when they are launched inside that graph (a null DevArgs pointer means
// "use the by-value arguments", the host-driven path).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

struct DevArgs {
  double rl1, gamma, gamma_setup;
  int ycor_zero;          // 1: the Newton correction is the zero vector
  int run_setup;          // run flags of kernels shared with the host path:
  int run_ewt;            //   psetup, ewt + ||zn0||, Newton update + norms
  int run_update;         //   (0: the kernel returns at once)
  const double* arn_in;   // Arnoldi operator input V[l]
  double* arn_out;        // Arnoldi operator output V[l+1]
};

// Scalars shared with the host integrator (same names, same meaning); the
// lists drive the copies between the two (integrator.cu).
#define LLG_DS_DOUBLES(X)                                                                                     \
  X(rtol) X(atol) X(tn) X(h) X(hscale) X(hprime) X(next_h) X(eta) X(etamax) X(hu) X(hmin) X(hmax_inv) X(etaq)  \
  X(etaqm1) X(etaqp1) X(gamma) X(gammap) X(gamrat) X(rl1) X(crate) X(delp) X(acnrm) X(saved_tq5) X(kappa)
#define LLG_DS_INTS(X)                                                                                      \
  X(qmax) X(maxl) X(classical_gs) X(mxstep) X(q) X(qprime) X(next_q) X(qwait) X(L) X(qu) X(indx_acor)        \
  X(jcur_nls) X(jcur) X(convfail) X(started) X(ls_curiter)
#define LLG_DS_LLS(X)                                                                                       \
  X(neq) X(nst) X(nfe) X(nsetups) X(nni) X(ncfn) X(netf) X(nli) X(nlcf) X(njv) X(nps) X(npe) X(nstlp)        \
  X(nstlj) X(nscon) X(pol_solves) X(nsl) X(nil) X(nsb) X(nib)
#define LLG_DS_ARRAYS(X) X(l) X(tq) X(tau)

constexpr int DS_QMAXL = 5;
constexpr int DS_MAXLL = 16;

// conditional-node handles, one per conditional node of the step graph:
// the attempt loop, the Newton loop, the Arnoldi loop, the failure path and,
// inside it, the order-1 restart
enum DsHandle { H_LOOP = 0, H_NEWTON, H_GMITER, H_FAIL, H_Q1F, H_COUNT };

// reduction result slots (doubles) in the context's scalar buffer
constexpr int SLOT_A2 = 2;       // norm of the second Gram-Schmidt pass
constexpr int SLOT_DOTS2 = 44;   // dots of the second Gram-Schmidt pass (16)

struct DState {
  DevArgs da;
#define LLG_DS_DECL_D(f) double f;
#define LLG_DS_DECL_I(f) int f;
#define LLG_DS_DECL_LL(f) long long f;
  LLG_DS_DOUBLES(LLG_DS_DECL_D)
  LLG_DS_INTS(LLG_DS_DECL_I)
  LLG_DS_LLS(LLG_DS_DECL_LL)
#undef LLG_DS_DECL_D
#undef LLG_DS_DECL_I
#undef LLG_DS_DECL_LL
  double l[DS_QMAXL + 2], tq[6], tau[DS_QMAXL + 2];

  // SPGMR of the current linear solve
  double Hes[DS_MAXLL + 1][DS_MAXLL], givens[2 * DS_MAXLL], yg[DS_MAXLL + 1];
  double rnorm, rho, rot, beta, dtol, sc, vk_norm;
  int nl, krydim, converged, li, small, gm_fail, lres, lcdiv, reorth;

  // step control
  double tout, tret, saved_t, dsm, cquot;
  int status, nstloc, ncf, nef, nflag, call_setup, jbad, m, retval, dky, need_wrms2, ycor_zero;
  int new_step, newton_first, attempt_again, run_predict, ord_run;
  // run flags of the predicated kernels
  int f_acor0, f_restore, f_decr, f_q1f, f_sam, f_cpy1, f_w2, f_cpy2, f_copyy, f_dky;
  int rescale_pending, ord_type, ord_q, res_q;
  long long nli0_pol;
  long long guard_count, guard_max;   // control ops this call / bound
  int tripped, guard_pad;
  double pf[DS_QMAXL + 2];        // pending rescale factors eta^j
  double ord_l[DS_QMAXL + 2];     // order-change coefficients
  double ord_A1;
  double dky_c[DS_QMAXL + 2];
  int dky_nv;
  long long nfe_demag;
  int has_demag, have_setup;

  // learned preconditioner (block-Jacobi probe / cost policy, as on the host)
  int learned_on, learned_now, probe, policy, fell_back, learned_pad;
  double pol_it_learned, pol_it_bj, pol_kappa;

  // launch tallies of this graph, per kernel family (added to the host counters)
  long long kcount[16];

  // device buffers
  double* zn[DS_QMAXL + 1];
  double* V[DS_MAXLL + 1];
  double *ewt, *acor, *y, *tempv, *delta, *yout, *zb;
  double* scal;
  // optional trace: (op, globaltimer ns) of every control op of the call
  unsigned long long* trace;
  int trace_cap, trace_n;

  cudaGraphConditionalHandle hnd[H_COUNT];
};

struct llg_ctx;
struct DevInteg;   // graph + device state of one integrator (integrator_dev.cu)
int devint_create(llg_ctx* c, DevInteg** out);
void devint_destroy(DevInteg* d);
// host state -> device (before the first device call, or after host steps)
int devint_upload(DevInteg* d, const DState& hs, llg_ctx* c);
// one llg_integrate call on the device; the final state comes back in hs
int devint_run(DevInteg* d, llg_ctx* c, double tout, double* yout, DState& hs);
// batches (batch.cpp): one graph holding every instance's step loop as an
// independent branch; per call, set each instance's arguments, launch once,
// fetch each state, synchronise, collect
int devint_mark_batched(DevInteg* d);
int devint_build_batch(llg_ctx* const* cs, DevInteg* const* ds, const DState* const* hss, int n,
                       cudaGraphExec_t* exec);
int devint_batch_args(DevInteg* d, llg_ctx* c, double tout, double* yout, cudaStream_t s);
int devint_batch_fetch(DevInteg* d, llg_ctx* c, cudaStream_t s);
int devint_batch_collect(DevInteg* d, llg_ctx* c, DState& hs);
