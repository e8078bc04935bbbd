// llg_internal.h — shared declarations of libllg.so (B200 / sm_100a).
//
// HBM layout of one problem instance (ncell = ng*ny, FP64 unless noted):
//   y, ydot, Jv, z, Krylov vectors   3*ncell   SoA [mx|my|mz]
//   act                               ncell     uint8, 1 active / 0 hole (EXEC_YMSK)
//   active_ids / inactive_ids         int32 lists (EXEC_COMPACT)
//   w                                 ncell     window (polycrystal only)
//   msk3 / nsk3                       3*ncell   per-cell axes (polycrystal only)
//   hd                                3*ncell   demag field of the last RHS
//   pm, ph                            3*ncell   m and h frozen at the last psetup;
//                                               psolve rebuilds each 3x3 block from
//                                               them (48 B/cell instead of 72 B of P^-1)
//   spec                              3*Hx*ny   complex row spectra, column-major
//                                               (x-frequency outer, y inner)
//   tensor spectra                    Hx*Py     xx, yy, zz real + xy complex, scaled
//                                               by strength/(Px*Py)
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#include "../../include/llg.h"
#include "dev_integ.h"

#define LLG_CUDA_TRY(expr)                                                   \
  do {                                                                       \
    cudaError_t _e = (expr);                                                 \
    if (_e != cudaSuccess) {                                                 \
      llg_set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));     \
      return LLG_ERR_CUDA;                                                   \
    }                                                                        \
  } while (0)

void llg_set_error(const std::string& msg);

// Launch accounting (host counters, one per kernel family), read by
// llg_kernel_counts; every launch site bumps exactly one counter.
enum LlgKernel {
  KID_RHS = 0, KID_JTV, KID_ARNOLDI, KID_PSETUP, KID_PSOLVE, KID_NORM,
  KID_DEMAG_ROWS_FWD, KID_DEMAG_COLS, KID_DEMAG_ROWS_INV, KID_REDUCE, KID_ELEMWISE,
  KID_LEARNED, KID_OTHER, KID_COUNT
};
extern std::atomic<long long> g_kcount[KID_COUNT];
// nonzero while a CUDA graph is being captured on this thread: the capture
// launches nothing (the graph's own launches are tallied on the device)
extern thread_local int g_count_off;
#define LLG_COUNT(k) (g_count_off ? 0LL : g_kcount[(k)].fetch_add(1, std::memory_order_relaxed))
struct llg_ctx;
// event before (pre = true) / after a launch of family kid, when it is timed
void ktimer_mark(llg_ctx* c, int kid, bool pre);

// Physics + geometry view passed by value to every per-cell kernel.
// scalar result slots (doubles) in d_scal / h_scal
constexpr int NSCAL = 512;
constexpr int SLOT_TCERR = 6;   // the tensor-core demag stage's timeout flag (int in the slot's low word)

struct DevProblem {
  int ng, ny;
  int ncell;
  int bc;          // LLG_BC_*
  int aniso;       // LLG_ANISO_*
  int windowed;    // 0/1
  int jv_full;     // 1: Jv field includes hd + happ
  double che, chk, cha, chb, alpha, chg;
  double msk[3], nsk[3], happ[3];
  double n0[3];    // strength-scaled N(0) diagonal
  int src_on, src_col, pml_cells, pad0;
  double src_h;          // soft-source field of the current evaluation (set per RHS call)
  double pml_alpha_max;
  const double* jv_hv;   // LLG_JV_FULL_DEMAG: demag field of the Jv input (set per launch), else null
  const uint8_t* act;    // nullptr: all active
  const double* w;       // windowed
  const double* msk3;    // windowed
  const double* nsk3;    // windowed
};

struct DemagPlan;   // k_demag.cu
struct DemagTc;     // k_demag_tc.cu
struct Integrator;  // integrator.cu
struct Learned;     // k_learned.cu

// A read-back carried by the reduction that produces its last value: warp 0
// of that kernel's last block copies scal[lo, hi) into the mapped mailbox and
// then writes the sequence word, in place of a separate publish launch after
// it (seq 0: nothing to publish).
struct Pub {
  const double* scal;
  double* mail;
  int lo, hi;
  unsigned long long seq;
};

struct llg_ctx {
  llg_params p{};
  DevProblem dp{};
  int ncell = 0;
  long long neq = 0;
  cudaStream_t stream = nullptr;
  int device = 0;
  int num_sms = 148;
  int arn_grid[2] = {0, 0};   // persistent Arnoldi operator: CTAs (without / with the demag field staged)
  int arn_grid_f[2] = {0, 0}; // the same for an FP32 Krylov basis
  int arn_tuned[2] = {0, 0}, arn_tuned_f[2] = {0, 0};   // grid autotuned (first host-path launch)

  // geometry
  uint8_t* d_act = nullptr;
  int32_t* d_active_ids = nullptr;
  int32_t* d_inactive_ids = nullptr;
  int n_active = 0, n_inactive = 0;
  double* d_w = nullptr;
  double* d_msk3 = nullptr;
  double* d_nsk3 = nullptr;

  // fields
  double* d_hd = nullptr;    // demag field of the last RHS (3N)
  double* d_pm = nullptr;    // m at the last psetup (3N)
  double* d_ph = nullptr;    // h at the last psetup (3N)
  double* d_pinv = nullptr;  // (I - gamma_setup J)^-1 per cell at the last psetup, 9 planes (9N)
  double* d_hv = nullptr;    // LLG_JV_FULL_DEMAG: demag field of the Jv input (3N)
  double* d_vt = nullptr;    // LLG_JV_FULL_DEMAG: the Arnoldi operator's scaled input (3N)
  double gamma_setup = 0.0;
  int have_setup = 0;
  int pinv_f32 = 0;          // d_pinv holds FP32 values (the FP32-basis Krylov solver's operator)

  // reductions
  double* d_red = nullptr;      // partial sums scratch (17 x 1024 doubles)
  double* d_scal = nullptr;     // scalar results (device)
  unsigned int* d_counter = nullptr;
  double* h_scal = nullptr;     // pinned host mirror
  // read-back mailbox: mapped pinned host memory that a one-warp kernel fills
  // with d_scal[lo, hi) and then a sequence number (the host spins on it)
  double* h_mail = nullptr;     // NSCAL values + the sequence word (host view)
  double* d_mail = nullptr;     // the same memory, device view
  unsigned long long mail_seq = 0;
  Pub pub_armed{};              // requested, not yet given to a launch
  Pub pub_carried{};            // given to the last launch that took one
  int red_blocks_max = 0;

  DemagPlan* demag = nullptr;
  Integrator* integ = nullptr;
  Learned* learned = nullptr;
  long long nfe_demag = 0;
  int capturing = 0;   // 1 while the device-resident step graph is captured
  // live timing of selected kernel families (llg_kernel_timer_*): one event
  // pair around each launch of a family whose bit is set in timer_mask
  unsigned timer_mask = 0;
  std::vector<cudaEvent_t>* timer_ev = nullptr;   // [KID_COUNT] lists, pre-created
  int timer_cap = 0;
  int timer_n[16] = {};
  int timer_stride = 1;        // time every timer_stride-th launch of a family
  long long timer_seen[16] = {};
  // test hooks: the inject_rhs_after-th and later RHS evaluations of the
  // integrator fail on the host (< 0: off); bound on the device-resident
  // integrator's control ops per call (0: its default)
  long long inject_rhs_after = -1, inject_rhs_seen = 0;
  long long ctl_limit = 0;
};

// ── physics kernels (k_physics.cu) ─────────────────────────────────────
int launch_normalize(llg_ctx* c, double* y);
int launch_rhs(llg_ctx* c, const double* y, const double* hd, double* ydot);
int launch_jtv(llg_ctx* c, const double* v, double* Jv, const double* y);
int launch_psetup(llg_ctx* c, const double* y, double gamma, const DevArgs* da = nullptr);
int launch_psolve(llg_ctx* c, const double* r, double* z, const DevArgs* da = nullptr);
// fused Arnoldi operator:  out = s1 ⊙ P^-1 ( vt − γ J vt ),  vt = in / s2
// (scale_out 0: out = P^-1 (...) without the s1 factor)
// (da non-null: in, out, gamma and the setup gamma come from the device-resident
// integrator's DevArgs at run time; the pointer arguments are ignored)
int arnoldi_setup(llg_ctx* c);   // shared-memory opt-in and grid of the persistent Arnoldi operator
// (in_a: the input's KScale scale; null: the input is used as stored)
int launch_arnoldi_op(llg_ctx* c, const double* in, const double* ewt, double* out,
                      const double* y, double gamma, int scale_out = 1, const DevArgs* da = nullptr,
                      const double* in_a = nullptr);
// the same operator on an FP32 Krylov basis (host-driven integrator only)
int launch_arnoldi_op_f(llg_ctx* c, const float* in, const double* ewt, float* out, const double* y, double gamma,
                        const double* in_a);
int rhs_full(llg_ctx* c, double t, double* y, double* ydot);
// value of the soft source at t into c->dp.src_h (the field the next RHS,
// residual and setup launches add at the source column)
void set_source_time(llg_ctx* c, double t);

// ── demag (k_demag.cu) ─────────────────────────────────────────────────
int demag_create(llg_ctx* c);
void demag_destroy(DemagPlan* d);
int demag_apply(llg_ctx* c, const double* y, double* h);
int demag_apply_w(llg_ctx* c, const double* y, const double* w, double* h);
int demag_self(llg_ctx* c, double out3[3]);
int demag_stage(llg_ctx* c, int stage, const double* y, double* h);
int demag_dims(llg_ctx* c, int out[4]);
int demag_tensor_host(llg_ctx* c, int comp, int dx, int dy, double* out);
// tensor-core (tcgen05, FP16 hi+lo split, FP32 accumulation) column stage of the
// mixed chain; *out stays null when the column shape is not supported
int demag_tc_create(llg_ctx* c, int px, int py, int hx, int ny, const float* txx, const float* tyy,
                    const float* tzz, const float2* txy, DemagTc** out);
void demag_tc_destroy(DemagTc* t);
int demag_tc_cols(llg_ctx* c, DemagTc* t, float2* Sf);
int demag_tc_failed(llg_ctx* c, DemagTc* t);
// LLG_ERR_TIMEOUT if a bounded tensor-core wait of the demag chain ran out
// (reads the flag back and waits)
int demag_check(llg_ctx* c);
// the same, from the copy of the flag that the integrator's last read-back
// brought home (no wait; integrate calls use it)
int demag_check_last(llg_ctx* c);

// ── learned preconditioner (k_learned.cu) ──────────────────────────────
bool learned_active(llg_ctx* c);                 // LLG_PREC_LEARNED with weights, no fallback
double* learned_zbuf(llg_ctx* c);                // 3N scratch for the block-Jacobi stage
int learned_apply(llg_ctx* c, const double* ewt, double* out, int slot /* <0: no norm */);
void learned_fall_back(llg_ctx* c, int reason /* 1 failed solve, 2 cost */);
void learned_policy_record(llg_ctx* c, double it_learned, double it_bj, double kappa);
bool learned_policy_on(llg_ctx* c);
bool learned_harvest_wanted(llg_ctx* c);
int learned_harvest(llg_ctx* c, const double* u, const double* x, const double* ewt, double gamma);

// ── vector ops (k_vector.cu) ───────────────────────────────────────────
int reductions_init(llg_ctx* c);
void reductions_free(llg_ctx* c);
// Krylov basis vectors that the read-back-light SPGMR keeps unnormalised in
// memory: vector i is read as a_i * V_i, with a_i the device scalar *a[i] (1
// when a[i] is null).  The kernel that forms a vector's norm also writes its
// scale (gs_scale_of: 1 / ||v||, or 1 when classical Gram-Schmidt's norm test
// asks for a second pass, after which the host normalises the vector
// itself).  Each consumer forms a_i * V_i before using it, the product a
// normalising pass would have stored, so the results are those of
// normalising in place.
constexpr int KS_MAX = 17;
struct KScale {
  const double* a[KS_MAX];
};
#ifdef __CUDACC__
__device__ __forceinline__ double kscale_of(const double* a) { return a ? *a : 1.0; }
// scale of a vector with sum of squares ss; vk (optional): its sum of squares
// before the Gram-Schmidt update (1000 ||v|| < ||v before||: a second pass is due)
__device__ __forceinline__ double gs_scale_of(double ss, const double* vk) {
  if (vk && 1000.0 * sqrt(ss) < sqrt(*vk)) return 1.0;
  return 1.0 / sqrt(ss);
}
#endif

// device-side: results land in c->d_scal[slot..]; host copy via fetch_scalars
// (ks: scales of the Y vectors; null: none)
int vdot_multi_dev(llg_ctx* c, int nvec, const double* x, const double* const* Y, int slot,
                   const KScale* ks = nullptr);
int vwrms_dev(llg_ctx* c, const double* x, const double* w, int slot);
int vwrms_diff_dev(llg_ctx* c, double a, const double* x, double b, const double* y,
                   const double* w, int slot);
int fetch_scalars(llg_ctx* c, int slot, int n, double* out);
// copy d_scal[lo, hi) to c->h_scal[lo, hi) and wait (one read-back)
int fetch_range(llg_ctx* c, int lo, int hi);
// request the read-back of d_scal[lo, hi) from the next reduction launched
// through a helper that carries one (vgs_update_dev[_f], fused_update_wrms2,
// fused_lincomb_update[_f]); a fetch_range of the same range right after it
// then only waits.  take_publish: the launch helpers' side.
void arm_publish(llg_ctx* c, int lo, int hi);
Pub take_publish(llg_ctx* c);
// device-coefficient forms used by the read-back-light SPGMR
// (aout: also write the updated vector's KScale scale there, gs_scale_of with
// the vector's pre-update sum of squares at d_scal[slot_dots + k])
int vgs_update_dev(llg_ctx* c, int k, double* const* V, int slot_dots, int slot_ss, const KScale* ks = nullptr,
                   int slot_aout = -1);
// FP32 Krylov basis (LLG_KRYLOV_FP32): the basis is stored as float, every
// product and sum is formed in FP64
int vdot_multi_dev_f(llg_ctx* c, int nvec, const float* x, const float* const* Y, int slot,
                     const KScale* ks = nullptr);
int vgs_update_dev_f(llg_ctx* c, int k, float* const* V, int slot_dots, int slot_ss, const KScale* ks = nullptr,
                     int slot_aout = -1);
int vscale_f(llg_ctx* c, double a, const float* x, float* z);
int fused_psolve_scale_dot_f(llg_ctx* c, const double* r, const double* ewt, float* v0, int slot, int slot_aout);
int fused_lincomb_norm_f(llg_ctx* c, int nv, const double* coef, const float* const* X, float* z, int slot,
                         const KScale* ks = nullptr);
int fused_lincomb_div_f(llg_ctx* c, int nv, const double* coef, const float* const* X, const double* w, double* z,
                        const KScale* ks = nullptr);
int fused_lincomb_update_f(llg_ctx* c, int nv, const double* coef, const float* const* X, const double* w,
                           double* del, bool ycor_zero, double* ycor, int slot, const KScale* ks = nullptr);
double vmaxnorm_host(llg_ctx* c, const double* x);
int vlin(llg_ctx* c, double a, const double* x, double b, const double* y, double* z);
int vscale(llg_ctx* c, double a, const double* x, double* z);
int vconst(llg_ctx* c, double a, double* z);
int vprod(llg_ctx* c, const double* x, const double* y, double* z);
int vdiv(llg_ctx* c, const double* x, const double* y, double* z);
int vlincomb(llg_ctx* c, int nvec, const double* coef, const double* const* X, double* z);
int vscale_add_multi(llg_ctx* c, int nvec, const double* a, const double* x,
                     double* const* Y, double* const* Z);
int vnordsieck_shift(llg_ctx* c, int q, double* const* zn, int sign);
int vscale_columns(llg_ctx* c, int q, double eta, double* const* zn);
int vscale_columns_f(llg_ctx* c, int q, const double* f, double* const* zn);   // zn[j] *= f[j], j = 1..q
int vset_ewt(llg_ctx* c, double rtol, double atol, const double* y, double* ewt, int slot);
int vhin_bound(llg_ctx* c, double rtol, double atol, const double* y0, const double* f0,
               double* tmp);

// fused integrator passes (k_fused.cu); reductions leave raw sums in d_scal[slot..]
int fused_ewt_wrms(llg_ctx* c, double rtol, double atol, const double* y, double* ewt, int slot,
                   const DevArgs* da = nullptr);
// (da non-null: rl1, gamma, the setup gamma and whether ycor is zero come from
// the device-resident integrator's DevArgs at run time)
int fused_lin_normalize(llg_ctx* c, const double* zn0, const double* ycor /* null: zero */, double* y,
                        const DevArgs* da = nullptr);
int fused_field(llg_ctx* c, const double* y);
int fused_resid(llg_ctx* c, const double* y, const double* zn1, const double* ycor /* null: zero */, double rl1,
                double gamma, double* negres, const DevArgs* da = nullptr);
// (slot_aout >= 0: also write V0's KScale scale 1 / ||V0|| to d_scal[slot_aout])
int fused_psolve_scale_dot(llg_ctx* c, const double* r, const double* ewt, double* v0, int slot,
                           const DevArgs* da = nullptr, int slot_aout = -1);
int fused_lincomb_norm(llg_ctx* c, int nv, const double* coef, const double* const* X, double* z, int slot,
                       const KScale* ks = nullptr);
int fused_lincomb_div(llg_ctx* c, int nv, const double* coef, const double* const* X, const double* w, double* z,
                      const KScale* ks = nullptr);
int fused_update_wrms2(llg_ctx* c, bool ycor_zero, double* ycor, const double* del, const double* w, int slot,
                       const DevArgs* da = nullptr);
int fused_wrms2(llg_ctx* c, const double* x1, double a, const double* x2, double b, const double* x3,
                const double* w, int slot);

// start of a BDF attempt: (do_ewt) weights + checks, (pend) zn[j] *= f[j], the
// Nordsieck predictor and y = normalise(zn0)  [k_fused.cu]
// (lazy_l non-null: the previous step's completion zn[j] += lazy_l[j] acor,
// j = 0..q, and zsave (non-null) = acor, applied first in the same pass)
int fused_predict(llg_ctx* c, int q, double* const* zn, const double* f, bool pend, bool do_ewt, double rtol,
                  double atol, double* ewt, double* y, int slot, const double* lazy_l = nullptr,
                  const double* acor = nullptr, double* zsave = nullptr);
// complete_step (+ zn[qmax] = acor when save) and, when norms, the order-
// selection sums of the updated vectors
// (store false: only the norms of the completed values, nothing written)
int fused_complete(llg_ctx* c, int q, int qmax, const double* l, const double* acor, double* const* zn, bool save,
                   bool norms, double cquot, const double* w, int slot, bool store = true);
// GMRES correction (stored only when del is non-null) + Newton update + both norms
int fused_lincomb_update(llg_ctx* c, int nv, const double* coef, const double* const* X, const double* w,
                         double* del, bool ycor_zero, double* ycor, int slot, const KScale* ks = nullptr);

