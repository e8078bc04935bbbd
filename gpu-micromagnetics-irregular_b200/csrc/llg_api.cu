// llg_api.cu — the extern "C" entry points of libllg.so (include/llg.h).
//
// One llg_ctx owns every device buffer of one problem instance; the
// reference's byte-mirrored UserData structs (configs/sim_config.h:467-499)
// collapse into it.  Host → device traffic happens only in the geometry
// setters (once) and through the caller's own buffers.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <string>
#include <vector>

#include "llg_internal.h"
#include "launch.h"

static thread_local std::string g_last_error;
void llg_set_error(const std::string& msg) { g_last_error = msg; }
std::atomic<long long> g_kcount[KID_COUNT];
thread_local int g_count_off = 0;
// programmatic dependent launch is switched on only inside the host
// integrator's step loop on the legacy default stream (PdlScope)
thread_local int g_no_pdl = 1;
thread_local int g_pdl_break = 0;
int integrator_time_kernel(llg_ctx* c, int kid, int iters, double* avg_ms);

int integrator_create(llg_ctx* c, double t0, const double* y0, const llg_solver_opts* o);
void integrator_destroy(Integrator* b);
int integrator_run(llg_ctx* c, double tout, double* yout, double* tret);
int integrator_stats(llg_ctx* c, llg_stats* st);
int integrator_trace(llg_ctx* c, unsigned long long* buf, int cap);
int integrator_trace_count(llg_ctx* c);
int integrator_record_steps(llg_ctx* c, int cap);
int integrator_recorded_steps(llg_ctx* c, double* h, int32_t* q, int cap);
int integrator_replay_steps(llg_ctx* c, const double* h, const int32_t* q, int n);
int integrator_replay_status(llg_ctx* c, int32_t* position, int64_t* forced);
int integrator_checkpoint_size(llg_ctx* c, uint64_t* bytes);
int integrator_checkpoint_save(llg_ctx* c, void* buf, uint64_t cap, uint64_t* written);
int integrator_checkpoint_load(llg_ctx* c, const void* buf, uint64_t n);
void learned_destroy(Learned* l);

void set_source_time(llg_ctx* c, double t) {
  if (c->dp.src_on) c->dp.src_h = llg_source_value(&c->p, t);
}

static void sync_dp(llg_ctx* c) {
  DevProblem& d = c->dp;
  const llg_params& p = c->p;
  d.ng = p.ng;
  d.ny = p.ny;
  d.ncell = c->ncell;
  d.bc = p.bc;
  d.aniso = p.aniso_kind;
  d.windowed = p.windowed;
  d.jv_full = (p.jv_mode == LLG_JV_FULL_FIELD || p.jv_mode == LLG_JV_FULL_DEMAG);
  d.jv_hv = nullptr;
  d.che = p.che; d.chk = p.chk; d.cha = p.cha; d.chb = p.chb; d.alpha = p.alpha; d.chg = p.chg;
  for (int a = 0; a < 3; a++) { d.msk[a] = p.msk[a]; d.nsk[a] = p.nsk[a]; d.happ[a] = p.happ[a]; }
  double n0[3] = {0, 0, 0};
  if (c->demag) demag_self(c, n0);
  for (int a = 0; a < 3; a++) d.n0[a] = n0[a];
  d.src_on = (p.src_amp != 0.0 && p.src_col >= 0 && p.src_col < p.ng) ? 1 : 0;
  d.src_col = d.src_on ? p.src_col : -1;
  d.pml_cells = p.pml_cells > 0 ? p.pml_cells : 0;
  d.pml_alpha_max = p.pml_alpha_max;
  d.act = c->d_act;
  d.w = c->d_w;
  d.msk3 = c->d_msk3;
  d.nsk3 = c->d_nsk3;
}

static int validate(const llg_params* p) {
  if (!p) { llg_set_error("null params"); return LLG_ERR_ARG; }
  if (p->ng <= 0 || p->ny <= 0) { llg_set_error("ng, ny must be positive"); return LLG_ERR_ARG; }
  if ((long long)p->ng * p->ny * 3 > (1LL << 31) - 1) { llg_set_error("grid too large for 32-bit indexing"); return LLG_ERR_ARG; }
  if (p->exec_model != LLG_EXEC_YMSK && p->exec_model != LLG_EXEC_COMPACT) { llg_set_error("bad exec_model"); return LLG_ERR_ARG; }
  if (p->bc != LLG_BC_PERIODIC && p->bc != LLG_BC_FREE) { llg_set_error("bad bc"); return LLG_ERR_ARG; }
  if (p->norm_kind < LLG_NORM_NONE || p->norm_kind > LLG_NORM_REG) { llg_set_error("bad norm_kind"); return LLG_ERR_ARG; }
  if (p->norm_kind == LLG_NORM_REG && !(p->norm_eps > 0.0)) { llg_set_error("norm_eps must be > 0"); return LLG_ERR_ARG; }
  if (p->aniso_kind != LLG_ANISO_LINEAR && p->aniso_kind != LLG_ANISO_CUBIC) { llg_set_error("bad aniso_kind"); return LLG_ERR_ARG; }
  if (p->demag_mode < LLG_DEMAG_OFF || p->demag_mode > LLG_DEMAG_OPEN) { llg_set_error("bad demag_mode"); return LLG_ERR_ARG; }
  if (p->demag_mode != LLG_DEMAG_OFF && !(p->demag_thick > 0.0)) { llg_set_error("demag_thick must be > 0"); return LLG_ERR_ARG; }
  if (p->demag_precision != LLG_DEMAG_FP64 && p->demag_precision != LLG_DEMAG_MIXED) { llg_set_error("bad demag_precision"); return LLG_ERR_ARG; }
  if (p->windowed && p->exec_model != LLG_EXEC_YMSK) { llg_set_error("windowed runs use the full-grid execution model"); return LLG_ERR_ARG; }
  if (p->jv_mode < LLG_JV_REFERENCE || p->jv_mode > LLG_JV_FULL_DEMAG) { llg_set_error("bad jv_mode"); return LLG_ERR_ARG; }
  if (p->pml_cells < 0 || 2LL * p->pml_cells > p->ng) { llg_set_error("pml_cells must be 0..ng/2"); return LLG_ERR_ARG; }
  const double vals[] = {p->che, p->chk, p->cha, p->chb, p->alpha, p->chg, p->demag_strength,
                         p->src_amp, p->src_omega, p->src_ramp, p->pml_alpha_max};
  for (double v : vals)
    if (!isfinite(v)) { llg_set_error("non-finite physics constant"); return LLG_ERR_ARG; }
  return 0;
}

void ktimer_mark(llg_ctx* c, int kid, bool pre) {
  if (!(c->timer_mask & (1u << kid)) || !c->timer_ev || c->capturing) return;
  int& k = c->timer_n[kid];
  // a pair per sampled launch (every timer_stride-th); a launch without room
  // for both events is not timed
  if (pre && (c->timer_seen[kid]++ % c->timer_stride) != 0) return;
  if (pre ? (k + 2 > c->timer_cap) : ((k & 1) == 0)) return;
  cudaEventRecord(c->timer_ev[kid][k], c->stream);
  pdl_break();   // the launch after an event record follows it in full
  k++;
}

static void timer_free(llg_ctx* c) {
  if (!c->timer_ev) return;
  for (int f = 0; f < KID_COUNT; f++)
    for (auto e : c->timer_ev[f]) cudaEventDestroy(e);
  delete[] c->timer_ev;
  c->timer_ev = nullptr;
  c->timer_mask = 0;
}

extern "C" {

const char* llg_last_error(void) { return g_last_error.c_str(); }

int llg_default_params(llg_params* p) {
  if (!p) return LLG_ERR_ARG;
  memset(p, 0, sizeof(*p));
  p->ng = 128; p->ny = 64;
  p->exec_model = LLG_EXEC_YMSK;
  p->bc = LLG_BC_FREE;
  p->norm_kind = LLG_NORM_NONE;
  p->norm_eps = 1e-3;
  p->aniso_kind = LLG_ANISO_LINEAR;
  p->demag_mode = LLG_DEMAG_OFF;
  p->demag_precision = LLG_DEMAG_FP64;
  p->jv_mode = LLG_JV_REFERENCE;
  p->precond_kind = LLG_PREC_BLOCK_JACOBI;
  p->che = 1.0; p->chk = 0.1; p->cha = 0.0; p->chb = 0.0; p->alpha = 0.02; p->chg = 1.0;
  p->msk[0] = 1.0; p->nsk[0] = 1.0;
  p->happ[2] = 0.05;
  p->demag_strength = 0.0;
  p->demag_thick = 1.0;
  return 0;
}

// smoothstep ramp of the source amplitude (src/slit/2d_slit.cu:236-240)
double llg_source_value(const llg_params* p, double t) {
  if (!p || p->src_amp == 0.0 || p->src_col < 0 || p->src_col >= p->ng) return 0.0;
  double ramp = 1.0;
  if (p->src_ramp > 0.0 && t < p->src_ramp) {
    const double x = t / p->src_ramp;
    ramp = x * x * (3.0 - 2.0 * x);
  }
  return p->src_amp * ramp * sin(p->src_omega * t);
}

int llg_default_solver_opts(llg_solver_opts* o) {
  if (!o) return LLG_ERR_ARG;
  memset(o, 0, sizeof(*o));
  o->rtol = 1e-4; o->atol = 1e-6; o->maxl = 5; o->maxord = 5; o->gs_type = LLG_GS_AUTO; o->mxstep = 500;
  return 0;
}

int llg_create(const llg_params* p, llg_ctx** out) {
  if (!out) return LLG_ERR_ARG;
  *out = nullptr;
  int rc = validate(p);
  if (rc) return rc;
  int dev_count = 0;
  if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
    llg_set_error("no CUDA device: libllg.so has no CPU path");
    return LLG_ERR_CUDA;
  }
  llg_ctx* c = new llg_ctx();
  c->p = *p;
  c->ncell = p->ng * p->ny;
  c->neq = 3LL * c->ncell;
  cudaGetDevice(&c->device);
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
  const size_t v3 = sizeof(double) * 3 * (size_t)c->ncell;
  auto fail = [&](int r) { llg_destroy(c); return r; };
  if (cudaMalloc(&c->d_hd, v3) != cudaSuccess || cudaMalloc(&c->d_pm, v3) != cudaSuccess ||
      cudaMalloc(&c->d_ph, v3) != cudaSuccess || cudaMalloc(&c->d_pinv, 3 * v3) != cudaSuccess) {
    llg_set_error("cudaMalloc of field buffers failed");
    return fail(LLG_ERR_NOMEM);
  }
  cudaMemset(c->d_hd, 0, v3);
  if ((rc = reductions_init(c))) return fail(rc);
  if (p->demag_mode != LLG_DEMAG_OFF && p->demag_strength > 0.0) {
    if ((rc = demag_create(c))) return fail(rc);
    if (p->jv_mode == LLG_JV_FULL_DEMAG &&
        (cudaMalloc(&c->d_hv, v3) != cudaSuccess || cudaMalloc(&c->d_vt, v3) != cudaSuccess)) {
      llg_set_error("cudaMalloc of the Jv demag buffers failed");
      return fail(LLG_ERR_NOMEM);
    }
  }
  sync_dp(c);
  if ((rc = arnoldi_setup(c))) return fail(rc);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    llg_set_error(std::string("llg_create: ") + cudaGetErrorString(cudaGetLastError()));
    return fail(LLG_ERR_CUDA);
  }
  *out = c;
  return 0;
}

void llg_destroy(llg_ctx* c) {
  if (!c) return;
  if (c->stream) cudaStreamSynchronize(c->stream);
  timer_free(c);
  integrator_destroy(c->integ);
  learned_destroy(c->learned);
  demag_destroy(c->demag);
  reductions_free(c);
  cudaFree(c->d_act);
  cudaFree(c->d_active_ids);
  cudaFree(c->d_inactive_ids);
  cudaFree(c->d_w);
  cudaFree(c->d_msk3);
  cudaFree(c->d_nsk3);
  cudaFree(c->d_hd);
  cudaFree(c->d_pm);
  cudaFree(c->d_ph);
  cudaFree(c->d_pinv);
  cudaFree(c->d_hv);
  cudaFree(c->d_vt);
  delete c;
}

int llg_set_stream(llg_ctx* c, void* s) {
  if (!c) return LLG_ERR_ARG;
  c->stream = (cudaStream_t)s;
  return 0;
}

int llg_set_mask(llg_ctx* c, const double* h_ymsk3) {
  if (!c || !h_ymsk3) { llg_set_error("llg_set_mask: null argument"); return LLG_ERR_ARG; }
  const int n = c->ncell;
  std::vector<uint8_t> act(n);
  for (int k = 0; k < n; k++) {
    const double a = h_ymsk3[k], b = h_ymsk3[n + k], d = h_ymsk3[2 * n + k];
    if (!((a == 0.0 || a == 1.0) && a == b && a == d)) {
      llg_set_error("ymsk must be 0/1 and equal across the three components (cell " + std::to_string(k) + ")");
      return LLG_ERR_ARG;
    }
    act[k] = (a == 1.0) ? 1 : 0;
  }
  if (!c->d_act) LLG_CUDA_TRY(cudaMalloc(&c->d_act, n));
  LLG_CUDA_TRY(cudaMemcpy(c->d_act, act.data(), n, cudaMemcpyHostToDevice));
  sync_dp(c);
  return 0;
}

int llg_set_active_ids(llg_ctx* c, const int32_t* h_active, int32_t n_active, const int32_t* h_inactive,
                       int32_t n_inactive) {
  if (!c || n_active < 0 || n_inactive < 0 || (n_active && !h_active) || (n_inactive && !h_inactive)) {
    llg_set_error("llg_set_active_ids: bad argument");
    return LLG_ERR_ARG;
  }
  const int n = c->ncell;
  if (n_active + n_inactive != n) { llg_set_error("active + inactive must cover every cell once"); return LLG_ERR_ARG; }
  std::vector<uint8_t> seen(n, 0), act(n, 0);
  for (int k = 0; k < n_active; k++) {
    const int id = h_active[k];
    if (id < 0 || id >= n || seen[id]) { llg_set_error("active id out of range or repeated"); return LLG_ERR_ARG; }
    seen[id] = 1;
    act[id] = 1;
  }
  for (int k = 0; k < n_inactive; k++) {
    const int id = h_inactive[k];
    if (id < 0 || id >= n || seen[id]) { llg_set_error("inactive id out of range or repeated"); return LLG_ERR_ARG; }
    seen[id] = 1;
  }
  cudaFree(c->d_active_ids);
  cudaFree(c->d_inactive_ids);
  c->d_active_ids = c->d_inactive_ids = nullptr;
  if (n_active) {
    LLG_CUDA_TRY(cudaMalloc(&c->d_active_ids, sizeof(int32_t) * n_active));
    LLG_CUDA_TRY(cudaMemcpy(c->d_active_ids, h_active, sizeof(int32_t) * n_active, cudaMemcpyHostToDevice));
  }
  if (n_inactive) {
    LLG_CUDA_TRY(cudaMalloc(&c->d_inactive_ids, sizeof(int32_t) * n_inactive));
    LLG_CUDA_TRY(cudaMemcpy(c->d_inactive_ids, h_inactive, sizeof(int32_t) * n_inactive, cudaMemcpyHostToDevice));
  }
  c->n_active = n_active;
  c->n_inactive = n_inactive;
  if (!c->d_act) LLG_CUDA_TRY(cudaMalloc(&c->d_act, n));
  LLG_CUDA_TRY(cudaMemcpy(c->d_act, act.data(), n, cudaMemcpyHostToDevice));
  sync_dp(c);
  return 0;
}

int llg_set_window(llg_ctx* c, const double* h_w, const double* h_msk3, const double* h_nsk3) {
  if (!c || !h_w || !h_msk3 || !h_nsk3) { llg_set_error("llg_set_window: null argument"); return LLG_ERR_ARG; }
  if (!c->p.windowed) { llg_set_error("llg_set_window needs params.windowed = 1"); return LLG_ERR_ARG; }
  const size_t n = (size_t)c->ncell;
  for (size_t k = 0; k < n; k++)
    if (!(h_w[k] >= 0.0 && h_w[k] <= 1.0)) { llg_set_error("window values must lie in [0, 1]"); return LLG_ERR_ARG; }
  if (!c->d_w) LLG_CUDA_TRY(cudaMalloc(&c->d_w, sizeof(double) * n));
  if (!c->d_msk3) LLG_CUDA_TRY(cudaMalloc(&c->d_msk3, sizeof(double) * 3 * n));
  if (!c->d_nsk3) LLG_CUDA_TRY(cudaMalloc(&c->d_nsk3, sizeof(double) * 3 * n));
  LLG_CUDA_TRY(cudaMemcpy(c->d_w, h_w, sizeof(double) * n, cudaMemcpyHostToDevice));
  LLG_CUDA_TRY(cudaMemcpy(c->d_msk3, h_msk3, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
  LLG_CUDA_TRY(cudaMemcpy(c->d_nsk3, h_nsk3, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
  sync_dp(c);
  return 0;
}

static int ready(llg_ctx* c) {
  if (!c) return LLG_ERR_ARG;
  if (c->p.windowed && !c->d_w) { llg_set_error("windowed problem without llg_set_window"); return LLG_ERR_STATE; }
  if (c->p.exec_model == LLG_EXEC_COMPACT && c->n_active + c->n_inactive != c->ncell) {
    llg_set_error("compact problem without llg_set_active_ids");
    return LLG_ERR_STATE;
  }
  return 0;
}

int llg_rhs(llg_ctx* c, double t, double* d_y, double* d_ydot) {
  int rc = ready(c);
  if (rc) return rc;
  if (!d_y || !d_ydot) return LLG_ERR_ARG;
  rc = rhs_full(c, t, d_y, d_ydot);
  return rc ? LLG_ERR_LAUNCH : 0;
}

int llg_jtv(llg_ctx* c, const double* d_v, double* d_Jv, double t, const double* d_y, const double* d_fy) {
  (void)d_fy;
  int rc = ready(c);
  if (rc) return rc;
  if (!d_v || !d_Jv || !d_y) return LLG_ERR_ARG;
  set_source_time(c, t);
  return launch_jtv(c, d_v, d_Jv, d_y) ? LLG_ERR_LAUNCH : 0;
}

int llg_psetup(llg_ctx* c, double t, const double* d_y, const double* d_fy, int jok, int* jcur, double gamma) {
  (void)d_fy; (void)jok;
  int rc = ready(c);
  if (rc) return rc;
  if (!d_y) return LLG_ERR_ARG;
  if (jcur) *jcur = 1;
  set_source_time(c, t);
  return launch_psetup(c, d_y, gamma) ? LLG_ERR_LAUNCH : 0;
}

int llg_psolve(llg_ctx* c, double t, const double* d_y, const double* d_fy, const double* d_r, double* d_z,
               double gamma, double delta, int lr) {
  (void)t; (void)d_y; (void)d_fy; (void)gamma; (void)delta; (void)lr;
  int rc = ready(c);
  if (rc) return rc;
  if (!d_r || !d_z) return LLG_ERR_ARG;
  rc = launch_psolve(c, d_r, d_z);
  if (rc == LLG_ERR_STATE) return rc;
  return rc ? LLG_ERR_LAUNCH : 0;
}

int llg_normalize(llg_ctx* c, double* d_y) {
  if (!c || !d_y) return LLG_ERR_ARG;
  return launch_normalize(c, d_y) ? LLG_ERR_LAUNCH : 0;
}

int llg_demag_apply(llg_ctx* c, const double* d_y, double* d_h) {
  int rc = ready(c);
  if (rc) return rc;
  if (!d_y || !d_h) return LLG_ERR_ARG;
  if (demag_apply(c, d_y, d_h)) return LLG_ERR_LAUNCH;
  return demag_check(c);
}

int llg_demag_self_coupling(llg_ctx* c, double out3[3]) {
  if (!c || !out3) return LLG_ERR_ARG;
  return demag_self(c, out3);
}

int llg_demag_tensor_host(llg_ctx* c, int comp, int dx, int dy, double* out) {
  if (!c || !out) return LLG_ERR_ARG;
  return demag_tensor_host(c, comp, dx, dy, out);
}

const double* llg_hdemag_device(llg_ctx* c) { return c ? c->d_hd : nullptr; }

int llg_dot_multi(llg_ctx* c, int nvec, const double* d_x, const double* const* d_Y, double* h_out) {
  if (!c || !d_x || !d_Y || !h_out || nvec < 1 || nvec > 16) return LLG_ERR_ARG;
  int rc = vdot_multi_dev(c, nvec, d_x, d_Y, 8);
  if (rc) return rc;
  return fetch_scalars(c, 8, nvec, h_out);
}

int llg_linear_combination(llg_ctx* c, int nvec, const double* coef, const double* const* d_X, double* d_z) {
  if (!c || !coef || !d_X || !d_z || nvec < 1 || nvec > 16) return LLG_ERR_ARG;
  return vlincomb(c, nvec, coef, d_X, d_z);
}

int llg_wrms_norm(llg_ctx* c, const double* d_x, const double* d_w, double* h_out) {
  if (!c || !d_x || !d_w || !h_out) return LLG_ERR_ARG;
  int rc = vwrms_dev(c, d_x, d_w, 0);
  if (rc) return rc;
  return fetch_scalars(c, 0, 1, h_out);
}

int llg_integrator_init(llg_ctx* c, double t0, const double* d_y0, const llg_solver_opts* opts) {
  int rc = ready(c);
  if (rc) return rc;
  if (!d_y0 || !opts) return LLG_ERR_ARG;
  if (!(opts->rtol >= 0.0) || !(opts->atol >= 0.0) || (opts->rtol == 0.0 && opts->atol == 0.0)) {
    llg_set_error("tolerances must be >= 0 and not both zero");
    return LLG_CV_ILL_INPUT;
  }
  if (opts->maxord < 0 || opts->maxord > 5) { llg_set_error("maxord must be 1..5"); return LLG_CV_ILL_INPUT; }
  return integrator_create(c, t0, d_y0, opts);
}

int llg_integrate(llg_ctx* c, double tout, double* d_yout, double* tret) {
  if (!c || !d_yout || !tret) return LLG_ERR_ARG;
  const int rc = integrator_run(c, tout, d_yout, tret);
  // the flag as of the call's last read-back (the BDF step's first linear
  // solve reads it home with its other scalars); llg_get_stats checks it again
  const int dc = demag_check_last(c);
  return dc ? dc : rc;
}

int llg_get_stats(llg_ctx* c, llg_stats* st) {
  if (!c || !st) return LLG_ERR_ARG;
  const int rc = integrator_stats(c, st);
  if (rc) return rc;
  return demag_check(c);
}

int llg_integrator_record_steps(llg_ctx* c, int32_t cap) {
  if (!c) return LLG_ERR_ARG;
  return integrator_record_steps(c, cap);
}

int llg_integrator_recorded_steps(llg_ctx* c, double* h, int32_t* q, int32_t cap) {
  if (!c || cap < 0) return LLG_ERR_ARG;
  return integrator_recorded_steps(c, h, q, cap);
}

int llg_integrator_replay_steps(llg_ctx* c, const double* h, const int32_t* q, int32_t n) {
  if (!c) return LLG_ERR_ARG;
  return integrator_replay_steps(c, h, q, n);
}

int llg_integrator_replay_status(llg_ctx* c, int32_t* position, int64_t* forced_accepts) {
  if (!c) return LLG_ERR_ARG;
  return integrator_replay_status(c, position, forced_accepts);
}

int llg_inject_rhs_failure(llg_ctx* c, int64_t after) {
  if (!c) return LLG_ERR_ARG;
  c->inject_rhs_after = after < 0 ? -1 : after;
  c->inject_rhs_seen = 0;
  return 0;
}

int llg_set_control_op_limit(llg_ctx* c, int64_t limit) {
  if (!c || limit < 0) return LLG_ERR_ARG;
  c->ctl_limit = limit;
  return 0;
}

int llg_checkpoint_size(llg_ctx* c, uint64_t* bytes) {
  if (!c || !bytes) return LLG_ERR_ARG;
  return integrator_checkpoint_size(c, bytes);
}

int llg_checkpoint_save(llg_ctx* c, void* h_buf, uint64_t cap, uint64_t* written) {
  if (!c) return LLG_ERR_ARG;
  return integrator_checkpoint_save(c, h_buf, cap, written);
}

int llg_checkpoint_load(llg_ctx* c, const void* h_buf, uint64_t n) {
  int rc = ready(c);
  if (rc) return rc;
  return integrator_checkpoint_load(c, h_buf, n);
}

int llg_checkpoint_write_file(llg_ctx* c, const char* path) {
  if (!c || !path) return LLG_ERR_ARG;
  uint64_t n = 0;
  int rc = integrator_checkpoint_size(c, &n);
  if (rc) return rc;
  std::vector<unsigned char> buf(n);
  uint64_t w = 0;
  rc = integrator_checkpoint_save(c, buf.data(), n, &w);
  if (rc) return rc;
  FILE* f = fopen(path, "wb");
  if (!f) { llg_set_error(std::string("checkpoint: cannot open ") + path); return LLG_ERR_ARG; }
  const size_t put = fwrite(buf.data(), 1, w, f);
  const int cl = fclose(f);
  if (put != w || cl != 0) { llg_set_error(std::string("checkpoint: short write to ") + path); return LLG_ERR_ARG; }
  return 0;
}

int llg_checkpoint_read_file(llg_ctx* c, const char* path) {
  if (!c || !path) return LLG_ERR_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) { llg_set_error(std::string("checkpoint: cannot open ") + path); return LLG_ERR_ARG; }
  std::vector<unsigned char> buf;
  unsigned char chunk[1 << 16];
  size_t got;
  while ((got = fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
  fclose(f);
  return integrator_checkpoint_load(c, buf.data(), buf.size());
}

int llg_kernel_timer_start(llg_ctx* c, uint32_t family_mask, int32_t max_launches, int32_t stride) {
  if (!c || max_launches <= 0 || stride <= 0) return LLG_ERR_ARG;
  timer_free(c);
  c->timer_ev = new std::vector<cudaEvent_t>[KID_COUNT];
  c->timer_cap = 2 * max_launches;
  c->timer_stride = stride;
  for (int f = 0; f < KID_COUNT; f++) {
    c->timer_n[f] = 0;
    c->timer_seen[f] = 0;
    if (!(family_mask & (1u << f))) continue;
    c->timer_ev[f].resize(c->timer_cap);
    for (auto& e : c->timer_ev[f])
      if (cudaEventCreate(&e) != cudaSuccess) { timer_free(c); llg_set_error("kernel timer: event creation"); return LLG_ERR_CUDA; }
  }
  c->timer_mask = family_mask;
  return 0;
}

int llg_kernel_timer_stop(llg_ctx* c, double* total_ms, int64_t* launches, int32_t n) {
  if (!c || !total_ms || !launches || n <= 0) return LLG_ERR_ARG;
  if (!c->timer_ev) { llg_set_error("kernel timer not started"); return LLG_ERR_STATE; }
  LLG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  for (int f = 0; f < n; f++) { total_ms[f] = 0.0; launches[f] = 0; }
  for (int f = 0; f < KID_COUNT && f < n; f++) {
    for (int k = 0; k + 1 < c->timer_n[f]; k += 2) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, c->timer_ev[f][k], c->timer_ev[f][k + 1]) == cudaSuccess) {
        total_ms[f] += ms;
        launches[f]++;
      }
    }
  }
  timer_free(c);
  return 0;
}

int llg_kernel_counts(int64_t* out, int n) {
  if (!out || n <= 0) return LLG_ERR_ARG;
  const int m = n < KID_COUNT ? n : KID_COUNT;
  for (int k = 0; k < m; k++) out[k] = g_kcount[k].load();
  return KID_COUNT;
}

void llg_reset_kernel_counts(void) {
  for (int k = 0; k < KID_COUNT; k++) g_kcount[k].store(0);
}

int llg_trace_control(llg_ctx* c, uint64_t* d_buf, int32_t cap) {
  if (!c || cap < 0) return LLG_ERR_ARG;
  return integrator_trace(c, reinterpret_cast<unsigned long long*>(d_buf), cap);
}

int llg_trace_count(llg_ctx* c) {
  if (!c) return LLG_ERR_ARG;
  return integrator_trace_count(c);
}

int llg_time_kernel(llg_ctx* c, int kernel_id, int iters, double* avg_ms) {
  if (!c || !avg_ms || iters <= 0 || kernel_id < 0 || kernel_id >= KID_COUNT) return LLG_ERR_ARG;
  return integrator_time_kernel(c, kernel_id, iters, avg_ms);
}

}  // extern "C"
