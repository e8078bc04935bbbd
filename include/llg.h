/*
 * llg.h — C ABI of the B200-native 2-D Landau–Lifshitz–Gilbert hot path.
 *
 * Everything here is plain C: pointers, sizes and POD structs, no CUDA or
 * torch types.  Vectors are FP64 SoA [mx | my | mz], each block `ncell`
 * long, cell = j*ng + i (row-major, x fastest), exactly the N_Vector layout
 * of the reference (src/irregular/2d_fft/2d_i2/2d_fft.cu:233-235).
 *
 * Entry points and the reference interface each one replaces:
 *
 *   llg_rhs        ← f(t, y, ydot, user_data)            2d_i2/2d_fft.cu:366-411
 *                                                        (compact 2d_i6/2d_i6.cu:352-396,
 *                                                         polycrystal 2d_i3/2d_fft.cu:656-726,
 *                                                         linear+DMI 2d_i1/2d_fft.cu:380-435)
 *   llg_jtv        ← JtvProduct(v, Jv, t, y, fy, ud, tmp) 2d_i2/jtv.h:26-27, jtv.cu:131-149
 *   llg_psetup     ← PrecondSetup(t,y,fy,jok,jcur,γ,ud)   2d_i2/precond.h:31-34, precond.cu:323-357
 *   llg_psolve     ← PrecondSolve(t,y,fy,r,z,γ,δ,lr,ud)   2d_i2/precond.h:35-38, precond.cu:360-384
 *   llg_demag_apply← Demag_Apply(d, y, h)                 2d_i2/demag_fft.h:33
 *   llg_dot_multi  ← FusedNVec_DotProdMulti (nvdotprodmulti slot)
 *                                                        2d_i2/deferred_nvector.cu:146-180
 *   llg_integrator_* / llg_integrate
 *                  ← CVodeCreate(CV_BDF)/CVodeInit/CVodeSVtolerances/
 *                    SUNLinSol_SPGMR/CVode(…, CV_NORMAL)  2d_i2/2d_fft.cu:648-724
 *
 * Status convention (CVODE callback convention, 2d_i2/2d_fft.cu:404-410):
 *   0 success, <0 unrecoverable, >0 recoverable.
 */
#ifndef LLG_H
#define LLG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ── status codes ─────────────────────────────────────────────────────── */
#define LLG_SUCCESS          0
#define LLG_RECOVERABLE      1     /* callback: recoverable failure          */
#define LLG_ERR_LAUNCH      (-1)   /* callback: CUDA launch failed (ref. -1) */
#define LLG_ERR_ARG       (-100)   /* bad argument / inconsistent config     */
#define LLG_ERR_CUDA      (-101)   /* CUDA runtime error                     */
#define LLG_ERR_NOMEM     (-102)   /* allocation failed                      */
#define LLG_ERR_STATE     (-103)   /* call out of order (e.g. no integrator) */
#define LLG_ERR_TIMEOUT   (-104)   /* bounded device wait ran out            */
#define LLG_ERR_NOTSUP    (-105)   /* size/feature not supported             */

/* integrator return codes (same values as CVODE's CV_* flags) */
#define LLG_CV_SUCCESS          0
#define LLG_CV_TOO_MUCH_WORK  (-1)
#define LLG_CV_TOO_MUCH_ACC   (-2)
#define LLG_CV_ERR_FAILURE    (-3)
#define LLG_CV_CONV_FAILURE   (-4)
#define LLG_CV_LSETUP_FAIL    (-6)
#define LLG_CV_LSOLVE_FAIL    (-7)
#define LLG_CV_RHSFUNC_FAIL   (-8)
#define LLG_CV_ILL_INPUT     (-22)
#define LLG_CV_TOO_CLOSE     (-27)
#define LLG_CV_BAD_STATE     (-40)  /* non-finite state detected (no CVODE twin) */

/* ── knob enums (values follow configs/sim_config.h) ──────────────────── */
#define LLG_EXEC_YMSK        0     /* sim_config.h EXEC_YMSK    */
#define LLG_EXEC_COMPACT     1     /* sim_config.h EXEC_COMPACT */

#define LLG_BC_PERIODIC      0     /* wrap in x and y (every reference kernel) */
#define LLG_BC_FREE          1     /* out-of-grid neighbour reads 0            */

#define LLG_NORM_NONE        0     /* i4/i5/i6: no normalisation inside f       */
#define LLG_NORM_EXACT       1     /* i1: m/|m| when |m| > 1e-30                */
#define LLG_NORM_REG         2     /* i2/i3: m/(|m| + eps)                      */

#define LLG_ANISO_LINEAR     0     /* sim_config.h ANISO_LINEAR: h += msk (chk (m·msk) + cha) */
#define LLG_ANISO_CUBIC      1     /* sim_config.h ANISO_CUBIC:  h_a += msk_a chk m_a (m_a^2 - 1) */

#define LLG_DEMAG_OFF        0
#define LLG_DEMAG_PERIODIC   1     /* reference: circular convolution on ng x ny */
#define LLG_DEMAG_OPEN       2     /* zero-padded 2ng x 2ny (open boundaries)    */

#define LLG_DEMAG_FP64       0     /* plain FP64 transform chain                 */
#define LLG_DEMAG_MIXED      1     /* reduced-precision transform chain          */

#define LLG_JV_REFERENCE     0     /* Jv field without demag/Zeeman (2d_i2/jtv.cu:87-97) */
#define LLG_JV_FULL_FIELD    1     /* Jv field includes h_demag and h_app          */
#define LLG_JV_FULL_DEMAG    2     /* full field and the demag derivative N ⊛ (w v),
                                      which the reference omits (2d_i2/jtv.h:9-13):
                                      one more demag evaluation per Jv / Arnoldi step */

#define LLG_GS_AUTO          0     /* classical if neq < 500000 (2d_i2/2d_fft.cu:674) */
#define LLG_GS_CLASSICAL     1
#define LLG_GS_MODIFIED      2

#define LLG_PREC_BLOCK_JACOBI 0
#define LLG_PREC_LEARNED      1    /* learned stencil correction on top of block-Jacobi */

/* ── problem parameters (one source of truth for f, Jv, P) ───────────── */
typedef struct llg_params {
  int32_t ng, ny;          /* cells in x and y (the reference's ng = NX_VAL/3)   */
  int32_t exec_model;      /* LLG_EXEC_*                                          */
  int32_t bc;              /* LLG_BC_*                                            */
  int32_t norm_kind;       /* LLG_NORM_*                                          */
  int32_t aniso_kind;      /* LLG_ANISO_*                                         */
  int32_t demag_mode;      /* LLG_DEMAG_*                                         */
  int32_t demag_precision; /* LLG_DEMAG_FP64 | LLG_DEMAG_MIXED                    */
  int32_t windowed;        /* 1: per-cell window w + per-cell msk/nsk (polycrystal) */
  int32_t jv_mode;         /* LLG_JV_*                                            */
  int32_t precond_kind;    /* LLG_PREC_*                                          */
  int32_t reserved0;
  double  norm_eps;        /* LLG_NORM_REG epsilon (reference 1e-3)               */
  double  che;             /* exchange coupling                                   */
  double  chk;             /* anisotropy constant                                 */
  double  cha;             /* linear-anisotropy offset                            */
  double  chb;             /* DMI strength                                        */
  double  alpha;           /* Gilbert damping                                     */
  double  chg;             /* gyromagnetic prefactor                              */
  double  msk[3];          /* easy axis (uniform; per-cell when windowed)         */
  double  nsk[3];          /* DMI direction (uniform; per-cell when windowed)     */
  double  happ[3];         /* uniform applied field                               */
  double  demag_strength;  /* DEMAG_STRENGTH                                      */
  double  demag_thick;     /* DEMAG_THICK                                         */
  /* spin-wave soft source and absorbing edge layers (src/slit/2d_slit.cu:
   * 80-135, 236-240, 297-340): h_x += src_amp · ramp(t) · sin(src_omega t) on
   * column src_col (ramp: smoothstep over src_ramp, 1 after it), active when
   * src_amp != 0 and 0 <= src_col < ng; in the pml_cells columns next to each
   * x edge the damping of the RHS rises as alpha + (pml_alpha_max - alpha)
   * s^3, s = 1 at the edge and 0 inside (off when pml_cells = 0).  Jv and the
   * block-Jacobi preconditioner use the uniform alpha, as the reference's
   * slit Jacobian does (src/slit/jtv.cu:48).                               */
  int32_t src_col;         /* source column (SRC_X_FRAC · ng + 0.5)              */
  int32_t pml_cells;       /* PML_CELLS                                           */
  double  src_amp;         /* H_DRIVE                                             */
  double  src_omega;       /* 2π DRIVE_FREQ                                       */
  double  src_ramp;        /* RAMP_TIME                                           */
  double  pml_alpha_max;   /* PML_ALPHA_MAX                                       */
} llg_params;

/* ── integrator options ───────────────────────────────────────────────── */
typedef struct llg_solver_opts {
  double  rtol;            /* RTOL_VAL                                            */
  double  atol;            /* ATOL_VAL (scalar; SV tolerances with one value)     */
  int32_t maxl;            /* KRYLOV_DIM (<=0 → 5, the SPGMR default)             */
  int32_t maxord;          /* MAX_BDF_ORDER (1..5)                                */
  int32_t gs_type;         /* LLG_GS_*                                            */
  int32_t mxstep;          /* max internal steps per llg_integrate call (500)     */
  int32_t device_resident; /* 1: whole step loop on the device (CUDA graph)       */
  int32_t krylov_precision;/* LLG_KRYLOV_FP64 (0) | LLG_KRYLOV_FP32 (1)           */
} llg_solver_opts;
/* Storage of the SPGMR Krylov basis.  FP32 halves the basis traffic of the
 * Arnoldi operator, the Gram-Schmidt dots and update and the final
 * correction; every product, dot and sum is still formed in FP64, and the
 * state, the norms and the Newton update stay FP64.  Host-driven integrator
 * with classical Gram-Schmidt only (LLG_ERR_NOTSUP otherwise; the
 * device-resident form is not used with it).  With LLG_PREC_LEARNED the
 * basis stays FP64 while the network runs; once it is off for good (no
 * weights, or the cost policy or a failed solve dropped it) the next step
 * starts a fresh block-Jacobi setup and continues on the FP32 basis.  No
 * reference counterpart (SUNDIALS keeps the basis in the state's precision). */
#define LLG_KRYLOV_FP64       0
#define LLG_KRYLOV_FP32       1

/* counters, same meaning as PrintFinalStats (2d_i2/2d_fft.cu:414-435) */
typedef struct llg_stats {
  int64_t nst, nfe, nsetups, nni, ncfn, netf, nli, nlcf, njvevals, npsolves, npe;
  int64_t nfe_demag;       /* RHS calls that ran the demag chain                  */
  int32_t qlast, qcur;
  double  hlast, hcur, tcur;
} llg_stats;

typedef struct llg_ctx llg_ctx;

/* ── lifecycle ────────────────────────────────────────────────────────── */
/* Fill p with the physics of the reference's 128x64 free-edge film (A=1, k=0.1 along +x, …). */
int  llg_default_params(llg_params* p);
int  llg_default_solver_opts(llg_solver_opts* o);
int  llg_create(const llg_params* p, llg_ctx** out);
void llg_destroy(llg_ctx* ctx);
/* All work of ctx is issued on this stream (a cudaStream_t; NULL = legacy default). */
int  llg_set_stream(llg_ctx* ctx, void* cuda_stream);
const char* llg_last_error(void);

/* ── geometry upload (host arrays, copied once) ──────────────────────── */
/* EXEC_YMSK: reference SoA mask ymsk[3*ncell], entries 0 or 1, equal across
 * the three components (2d_i2/2d_fft.cu:538-566).                          */
int  llg_set_mask(llg_ctx* ctx, const double* h_ymsk3);
/* EXEC_COMPACT: active / inactive cell lists (2d_i6/2d_i6.cu:462-533).    */
int  llg_set_active_ids(llg_ctx* ctx, const int32_t* h_active, int32_t n_active,
                        const int32_t* h_inactive, int32_t n_inactive);
/* windowed (polycrystal): w[ncell], msk[3*ncell], nsk[3*ncell]
 * (2d_i3/2d_fft.cu:317-387).                                               */
int  llg_set_window(llg_ctx* ctx, const double* h_w, const double* h_msk3,
                    const double* h_nsk3);

/* ── operator callbacks (device pointers, SoA, length 3*ncell) ───────── */
/* f: normalise y in place (norm_kind), demag → h_demag, RHS → ydot.        */
int  llg_rhs(llg_ctx* ctx, double t, double* d_y, double* d_ydot);
/* Jv = J(y)·v, analytic (exchange + anisotropy + DMI; demag excluded).     */
int  llg_jtv(llg_ctx* ctx, const double* d_v, double* d_Jv, double t,
             const double* d_y, const double* d_fy);
/* Build the 3×3 block-Jacobi inverse (I − γJ)^-1 at y using the demag field
 * of the last llg_rhs call; always rebuilds and sets *jcur = 1.            */
int  llg_psetup(llg_ctx* ctx, double t, const double* d_y, const double* d_fy,
                int jok, int* jcur, double gamma);
/* z = P^-1 r, masked.                                                        */
int  llg_psolve(llg_ctx* ctx, double t, const double* d_y, const double* d_fy,
                const double* d_r, double* d_z, double gamma, double delta, int lr);
/* In-place normalisation kernel alone (the first stage of llg_rhs).        */
int  llg_normalize(llg_ctx* ctx, double* d_y);
/* Demag field h = strength · N ⊛ (w·m), overwriting d_h (3*ncell).          */
int  llg_demag_apply(llg_ctx* ctx, const double* d_y, double* d_h);
/* N(0)·strength diagonal (Demag_GetSelfCoupling, 2d_i2/demag_fft.cu:365-377). */
int  llg_demag_self_coupling(llg_ctx* ctx, double out3[3]);
/* Unscaled Newell tensor component c (0..8 = xx,xy,xz,yx,yy,yz,zx,zy,zz) at
 * displacement (dx, dy) on the demag grid, host copy (for checks).          */
int  llg_demag_tensor_host(llg_ctx* ctx, int comp, int dx, int dy, double* out);
/* Device pointer of the demag field written by the last llg_rhs call.      */
const double* llg_hdemag_device(llg_ctx* ctx);

/* ── fused vector ops (deterministic: fixed reduction order, no atomics) ── */
/* out[k] = x · Y[k], k < nvec ≤ 16, one launch; h_out is host memory.       */
int  llg_dot_multi(llg_ctx* ctx, int nvec, const double* d_x,
                   const double* const* d_Y, double* h_out);
/* z = Σ_k c[k] X[k], nvec ≤ 16, one pass.                                   */
int  llg_linear_combination(llg_ctx* ctx, int nvec, const double* c,
                            const double* const* d_X, double* d_z);
/* sqrt(mean((x·w)^2)), host result.                                          */
int  llg_wrms_norm(llg_ctx* ctx, const double* d_x, const double* d_w, double* h_out);

/* d_out[k] = x · Y[k] (k < nvec), d_out a caller-owned device buffer of nvec
 * doubles, on cuda_stream (NULL = legacy default).  No counterpart in the
 * reference: this is the llg_dot_multi reduction for callers that cannot
 * let a library allocate device memory when they need it — an application
 * whose device memory belongs to another allocator (a framework pool that
 * has reserved the GPU), or a solver loop that allows no allocation after
 * set-up because cudaMalloc/cudaFree may synchronise the device.  It needs
 * no llg_ctx and calls no cudaMalloc/cudaFree: its scratch is a fixed
 * file-scope device array of LLG_NOALLOC_MAX_VECS x LLG_NOALLOC_MAX_BLOCKS
 * doubles (~128 KiB) that every GPU loading the library keeps until exit.
 * nvec > LLG_NOALLOC_MAX_VECS is rejected (LLG_ERR_ARG).  The first call on
 * a device looks up the array's device address (cudaGetSymbolAddress) in
 * the CUDA runtime's primary context of that device and caches it: use the
 * entry point from that context only; later calls on the device make no
 * such runtime call.  Calls share the array: calls that overlap on
 * the GPU race.  Same result, bit for bit, as llg_dot_multi for the same
 * vectors (same block partition, per-thread order and reduction tree).      */
#define LLG_NOALLOC_MAX_VECS   16
#define LLG_NOALLOC_MAX_BLOCKS 1024
int  llg_dot_multi_noalloc(int nvec, const double* d_x, const double* const* d_Y, int64_t n,
                           double* d_out, void* cuda_stream);

/* ── integrator: BDF (orders 1..5, Nordsieck) + Newton + SPGMR ───────── */
int  llg_integrator_init(llg_ctx* ctx, double t0, const double* d_y0,
                         const llg_solver_opts* opts);
/* Advance to tout (CV_NORMAL: may step past tout, returns y(tout) by
 * interpolation).  d_yout: device, 3*ncell.  LLG_ERR_TIMEOUT when a bounded
 * tensor-core wait of the mixed demag chain ran out, as of the call's last
 * scalar read-back; llg_get_stats reads that flag again and waits for it.  */
int  llg_integrate(llg_ctx* ctx, double tout, double* d_yout, double* tret);
int  llg_get_stats(llg_ctx* ctx, llg_stats* st);

/* ── step-sequence record / replay (no counterpart in the reference) ──── *
 * Two forms of one problem (FP64 and mixed-precision demag, block-Jacobi and
 * learned preconditioner) that choose their own steps differ by the step
 * selection as much as by their arithmetic.  Recording keeps the (h, q) of
 * every accepted step of a run (up to cap; cap <= 0 stops); replaying makes
 * a fresh run (set after llg_integrator_init, before its first
 * llg_integrate) take exactly that sequence: step n uses order q_n and size
 * h_n, the local error test is evaluated but does not reject (the steps it
 * would have rejected are counted), the Newton iteration may take up to 10
 * iterations without CVODE's divergence test (the step size cannot shrink),
 * and a Newton failure retries the same step with a fresh preconditioner
 * setup, at most twice, then returns LLG_CV_CONV_FAILURE.  A run that needs more steps than were recorded
 * returns LLG_ERR_STATE.  Host-driven integrator only (the device-resident
 * form is bypassed while recording or replaying).                          */
int  llg_integrator_record_steps(llg_ctx* ctx, int32_t cap);
/* copies min(n, cap) recorded steps; returns n, the number recorded        */
int  llg_integrator_recorded_steps(llg_ctx* ctx, double* h, int32_t* q, int32_t cap);
int  llg_integrator_replay_steps(llg_ctx* ctx, const double* h, const int32_t* q, int32_t n);
/* steps taken so far and error-test rejections overridden by the replay    */
int  llg_integrator_replay_status(llg_ctx* ctx, int32_t* position, int64_t* forced_accepts);

/* ── failure injection and bounds for tests (no counterpart in the
 * reference) ──────────────────────────────────────────────────────────── *
 * llg_inject_rhs_failure: from the after-th RHS evaluation of ctx's
 * integrator on (counted from this call; after < 0 switches it off), each
 * evaluation fails on the host without launching anything, as a reference
 * callback returning -1 after a launch error (2d_i2/2d_fft.cu:404-410); the
 * integrator then returns LLG_CV_RHSFUNC_FAIL, as CVODE does.
 * llg_set_control_op_limit: bound on the control operations of one
 * llg_integrate call of the device-resident integrator (0: the default
 * 200·(mxstep + 10)·(maxl + 4)); past it every loop of the step graph
 * exits and the call returns LLG_ERR_TIMEOUT.                              */
int  llg_inject_rhs_failure(llg_ctx* ctx, int64_t after);
int  llg_set_control_op_limit(llg_ctx* ctx, int64_t limit);

/* ── checkpoint / restart (no counterpart in the reference, whose runs are
 * one CVode loop from t0) ──────────────────────────────────────────────── *
 * A checkpoint is the integrator's complete state between two
 * llg_integrate calls: CVODE's scalars (t, h, order, step-size history,
 * counters, order-selection state) and its device vectors (the Nordsieck
 * history zn[0..qmax], the last correction, the demag field of the last RHS
 * and, after a preconditioner setup, the frozen block-Jacobi state).  A
 * context with the same llg_params and geometry that loads it continues
 * bit for bit as the saved run would have.  The blob starts with
 * llg_ckpt_info and carries a checksum; load rejects other grids,
 * other physics parameters, other builds' layouts and corrupt buffers.
 * A learned-preconditioner context is not checkpointed (LLG_ERR_NOTSUP;
 * save its weights with llg_learned_get_weights).                         */
typedef struct llg_ckpt_info {
  char     magic[8];             /* "LLGCKPT1"                               */
  uint32_t version, header_bytes, scalar_bytes, krylov_precision;
  int32_t  ng, ny;
  int64_t  neq;
  int32_t  qmax, maxl, classical_gs, mxstep, device_resident, have_setup;
  double   rtol, atol, gamma_setup, tn;
  int64_t  nst, nfe_demag;
  uint64_t payload_bytes, checksum;
  llg_params params;
} llg_ckpt_info;
int  llg_checkpoint_size(llg_ctx* ctx, uint64_t* bytes);
/* host buffer of at least llg_checkpoint_size bytes                        */
int  llg_checkpoint_save(llg_ctx* ctx, void* h_buf, uint64_t cap, uint64_t* written);
/* replaces the context's integrator (llg_integrator_init not needed)       */
int  llg_checkpoint_load(llg_ctx* ctx, const void* h_buf, uint64_t n);
/* header + checksum validation without a GPU; info may be NULL             */
int  llg_checkpoint_inspect(const void* h_buf, uint64_t n, llg_ckpt_info* info);
int  llg_checkpoint_write_file(llg_ctx* ctx, const char* path);
int  llg_checkpoint_read_file(llg_ctx* ctx, const char* path);

/* ── learned preconditioner (no counterpart in the reference) ──────────── *
 * z = (P_BJ^-1 r + gamma * Net(P_BJ^-1 r; m)) on active cells, Net a 3-layer
 * 3x3 convolution 9 -> 16 -> 16 -> 3 channels without bias or activation
 * (linear in r), inputs [u, m x u, m x (m x u)], BF16 weights at inference,
 * FP32 accumulation.  Used by the integrator when params.precond_kind ==
 * LLG_PREC_LEARNED and weights are set; a failed GMRES solve switches the
 * context back to block-Jacobi for good (llg_learned_status).  Weights:
 * 4032 floats, [W1 (16,9,3,3) | W2 (16,16,3,3) | W3 (3,16,3,3)] row-major.  */
#define LLG_LEARNED_NWEIGHTS 4032
typedef struct llg_train_opts {
  int32_t iters;           /* Adam iterations                                     */
  int32_t batch;           /* patches per iteration                               */
  int32_t patch;           /* patch side (cells); 3-cell border excluded from loss */
  int32_t seed;            /* patch sampling / initial weights                     */
  double  lr;              /* Adam learning rate                                   */
  double  init_scale;      /* initial weight scale (fresh weights only)            */
} llg_train_opts;
/* Record (P_BJ^-1 r, x, ewt, m, gamma) of every `stride`-th converged
 * block-Jacobi SPGMR solve of the integrator, up to max_samples.           */
int  llg_learned_harvest(llg_ctx* ctx, int32_t max_samples, int32_t stride);
int  llg_learned_num_samples(llg_ctx* ctx);
/* Train on the harvested samples with the library's forward/backward/Adam
 * kernels; loss = mean over patches of sum (ewt (z - x))^2 / sum (ewt x)^2.  */
int  llg_learned_train(llg_ctx* ctx, const llg_train_opts* o, double* loss_first, double* loss_last);
int  llg_learned_set_weights(llg_ctx* ctx, const float* h_w, int32_t n);
int  llg_learned_get_weights(llg_ctx* ctx, float* h_w, int32_t n);
int  llg_learned_status(llg_ctx* ctx, int32_t* active, int32_t* fell_back, int64_t* napply);
/* The integrator's cost judgement (every 8th solve of a learned context runs
 * block-Jacobi as a probe): mean GMRES iterations per solve with the learned
 * and with the block-Jacobi preconditioner, and kappa = time of one learned
 * application / one fused Arnoldi operator step; -1 before the first
 * judgement.  fell_back in llg_learned_status: 0 none, 1 a learned solve
 * failed, 2 the learned path did not pay for its cost.                     */
int  llg_learned_policy(llg_ctx* ctx, double* it_learned, double* it_bj, double* kappa);
/* 1 (default): the cost-aware probing above; 0: learned on every solve.    */
int  llg_learned_set_policy(llg_ctx* ctx, int32_t cost_aware);
/* Inference path: 1 (default) one fused tensor-core kernel (tcgen05, BF16
 * operands and activations, FP32 accumulation); 0 layer-by-layer FP32
 * kernels with the same BF16-rounded weights (reference path).             */
int  llg_learned_set_fused(llg_ctx* ctx, int32_t fused);
/* d_out = ewt (z + gamma Net(z; m)) on active cells for device z, m, ewt;
 * *norm2 = sum d_out^2 (may be NULL).                                      */
int  llg_learned_apply(llg_ctx* ctx, const double* d_z, const double* d_m, const double* d_ewt, double gamma,
                       double* d_out, double* norm2);
/* Loss, weight gradient and output z of the training kernels on host FP32
 * patches [nb][3][P][P] (mask [nb][P][P], gamma [nb]); h_z may be NULL.     */
int  llg_learned_loss_grad(const float* h_w, int32_t nb, int32_t P, const float* h_u, const float* h_m,
                           const float* h_mask, const float* h_ewt, const float* h_x, const float* h_gamma,
                           double* loss, float* h_grad, float* h_z);

/* ── batches of independent instances (no counterpart in the reference) ─ *
 * One context per instance, each on its own CUDA stream; llg_batch_integrate
 * advances every instance to tout concurrently from `nthreads` host threads
 * (<= 0: one per instance), largest instances first.  Instances are set up
 * through llg_batch_ctx (set_mask / set_active_ids / set_window / learned
 * weights) before llg_batch_integrator_init.  rcs[i] receives each
 * instance's llg_integrate code (may be NULL).                            */
typedef struct llg_batch llg_batch;
int      llg_batch_create(int32_t n, const llg_params* params, llg_batch** out);
int      llg_batch_size(const llg_batch* b);
llg_ctx* llg_batch_ctx(llg_batch* b, int32_t i);
int      llg_batch_integrator_init(llg_batch* b, double t0, const double* const* d_y0, const llg_solver_opts* o);
int      llg_batch_integrate(llg_batch* b, double tout, double* const* d_yout, int32_t nthreads, int32_t* rcs);
void     llg_batch_destroy(llg_batch* b);
/* The same step for every instance as ONE CUDA graph launch: each
 * instance's device-resident step loop (BDF attempts, Newton and Arnoldi
 * iterations as graph WHILE / IF nodes set by control kernels) is an
 * independent branch of a single graph, built on the first call.  Every
 * instance must have advanced once with llg_batch_integrate (the host-side
 * start-up: initial step size and first step) and use settings the
 * device-resident form covers (classical Gram-Schmidt, block-Jacobi, no
 * source term, no recording/replay; LLG_ERR_NOTSUP otherwise).  Either
 * entry point may be used after the other.                                */
int      llg_batch_integrate_graph(llg_batch* b, double tout, double* const* d_yout, int32_t* rcs);
/* Split n independent instances across nparts GPUs (host function, no
 * counterpart in the reference, which runs one geometry per process):
 * longest-processing-time bin packing on the given cost estimates —
 * instances by decreasing cost, each to the least-loaded part so far (ties
 * to the lower index), deterministic, within 4/3 of the optimal makespan.
 * part_of[i] receives instance i's part; load (optional, nparts values) the
 * summed cost per part.  No collective is involved: every rank computes the
 * same split from the same seeded instance list.                          */
int      llg_partition_lpt(int32_t n, const double* cost, int32_t nparts, int32_t* part_of, double* load);

/* ── instrumentation ──────────────────────────────────────────────────── */
/* Kernel families, in this order: RHS, JTV, ARNOLDI (fused Krylov operator),
 * PSETUP, PSOLVE, NORM, DEMAG_ROWS_FWD, DEMAG_COLS, DEMAG_ROWS_INV, REDUCE,
 * ELEMWISE, LEARNED, OTHER.  Counts are process-wide launch counts.        */
#define LLG_KERNEL_FAMILIES 13
int  llg_kernel_counts(int64_t* out, int n);
void llg_reset_kernel_counts(void);
/* Average device time of one launch of family kernel_id (CUDA events on the
 * context's stream), measured on the live integrator buffers.              */
int  llg_time_kernel(llg_ctx* ctx, int kernel_id, int iters, double* avg_ms);
/* Live kernel timing (no reference counterpart): an event pair on the
 * context's stream around every stride-th launch (the 1st, (stride+1)-th,
 * ...) of every family whose bit (1 << family) is set in family_mask, up to
 * max_launches timed launches per family — the fused Arnoldi operator and
 * the three demag stages are instrumented.  A timed launch waits for its
 * predecessor in full (no programmatic dependent launch across an event).
 * _stop waits, then writes per family (arrays of n) the summed device time
 * and the launches timed.                                                 */
int  llg_kernel_timer_start(llg_ctx* ctx, uint32_t family_mask, int32_t max_launches, int32_t stride);
int  llg_kernel_timer_stop(llg_ctx* ctx, double* total_ms, int64_t* launches, int32_t n);
/* Device-resident integrator only (no reference counterpart): record, for
 * the following llg_integrate calls, one 64-bit word per control step —
 * (globaltimer ns << 5) | step id — into the device buffer d_buf (cap
 * words, cleared at each call).  d_buf = NULL stops recording.  Returns the
 * number of words the last call wrote through llg_trace_count.            */
int  llg_trace_control(llg_ctx* ctx, uint64_t* d_buf, int32_t cap);
int  llg_trace_count(llg_ctx* ctx);
/* Known-answer check of the tensor-core path the mixed demag chain uses
 * (no counterpart in the reference): one 128x64x64 FP16 GEMM into tensor
 * memory against a host FP64 product; *max_rel_err = max |D - ref| /
 * sum |a b|.  flags bit 0: A operand MN-major (else K-major); bit 1: A
 * values in the FP16 subnormal range (shows whether the MMA keeps them).   */
int  llg_selftest_tcgen05(int flags, double* max_rel_err);

/* ── geometry / initial-condition builders (host) ────────────────────── */
#define LLG_GEOM_BULK         0   /* sim_config.h GEOMETRY_BULK          */
#define LLG_GEOM_HOLE_SQUARE  1   /* GEOMETRY_HOLE_SQUARE (2d_i2)          */
#define LLG_GEOM_RING         2   /* GEOMETRY_RING: outer rect − inner rect */
#define LLG_GEOM_POLYCRYSTAL  3   /* GEOMETRY_POLYCRYSTAL (2d_i3)          */
#define LLG_GEOM_CUSTOM       4   /* caller builds the arrays              */
#define LLG_GEOM_ELLIPSE      5   /* GEOMETRY_ELLIPSE (2d_i6)              */
#define LLG_GEOM_ANNULUS      6   /* circular ring r_in..r_out (no reference twin) */
#define LLG_GEOM_SLIT         7   /* screen column with a slit (src/slit/2d_slit.cu:482-560) */

#define LLG_IC_UNIFORM        0   /* IC_UNIFORM                            */
#define LLG_IC_HEAD_ON_STRIPES 1  /* IC_HEAD_ON_STRIPES (2d_i1)            */
#define LLG_IC_TWO_DOMAIN     2   /* IC_TWO_DOMAIN (2d_i4)                 */
#define LLG_IC_GRAIN_BUMPS    3   /* IC_GRAIN_BUMPS (2d_i3)                */
#define LLG_IC_CUSTOM         4
#define LLG_IC_TWO_DOMAIN_X   5   /* +x left half, −x right half (no reference twin) */
#define LLG_IC_VORTEX         6   /* (−y, x, 0.1)/norm about the centre (no reference twin) */
#define LLG_IC_NEEL           7   /* Néel-like circular texture (src/2d_fft/2d_fft.cu:533-580) */

typedef struct llg_geom_spec {
  int32_t ng, ny;
  int32_t geometry_kind;          /* LLG_GEOM_*                              */
  int32_t ic_kind;                /* LLG_IC_*                                */
  /* square hole */
  double  hole_center_x_frac, hole_center_y_frac, hole_radius_frac_y;
  /* rectangular ring */
  double  outer_w_frac, outer_h_frac, inner_w_frac_of_outer, inner_h_frac_of_outer;
  /* ellipse */
  double  active_rx_frac, active_ry_frac;
  /* annulus (radii as fractions of min(ng, ny)) */
  double  annulus_r_in_frac, annulus_r_out_frac;
  /* polycrystal */
  int32_t num_grains;
  uint32_t hole_seed;
  double  dead_grain_frac, mask_eps_cells, grain_z_bias;
  /* initial condition */
  double  init_m[3];
  uint32_t init_random_seed;
  int32_t reserved0;
  double  init_random_eps;        /* stripes: my, mz amplitude (2d_i1)       */
  double  stripe_left_frac, stripe_right_frac;
  double  two_domain_split_frac, two_domain_tail_my;
  double  ic_core_mz;
  double  ic_jitter_eps;          /* U(±eps) on every component, then |m|=1  */
  /* Néel texture: mz from core to outer across a tanh wall of width
   * width_frac · radius (>= 1 cell) at radius r_frac_y · ny about
   * (cx_frac (ng-1), cy_frac (ny-1)); in-plane part radial             */
  double  texture_core_mz, texture_outer_mz, texture_width_frac, texture_eps;
  double  circle_cx_frac, circle_cy_frac, circle_r_frac_y;
  /* slit: screen at column (int)(screen_x_frac ng + 0.5), inactive except
   * the slit_w = (int)(slit_w_frac ny + 0.5) rows from ny/2 - slit_w/2     */
  double  screen_x_frac, slit_w_frac;
} llg_geom_spec;

int llg_default_geom_spec(llg_geom_spec* g);
/* The soft source's field at time t for parameters p (0 when inactive).    */
double llg_source_value(const llg_params* p, double t);
/* Fills the arrays that are non-NULL:
 *   active[ncell] (1 active / 0 hole), w[ncell], msk3[3*ncell], nsk3[3*ncell],
 *   grain_id[ncell], y0[3*ncell].  Returns the number of active cells (≥0)
 *   or a negative LLG_ERR_*.  Uses the C library srand/rand in the
 *   reference's call order.                                                 */
int llg_build_geometry(const llg_geom_spec* g, uint8_t* active, double* w,
                       double* msk3, double* nsk3, int32_t* grain_id, double* y0);

/* ── text outputs (the reference's formats) ──────────────────────────── *
 * Magnetisation frames as the reference writes them (WriteFrame,
 * 2d_i2/2d_fft.cu:437-455; final state 2d_i2/2d_fft.cu:735-757): a
 * "%f NX NY" header (NX = 3*ng, the reference's doubles per row), one
 * "mx my mz" line per cell in row-major order, "%f" lines and a closing
 * empty line for trajectory frames, "%e" lines for the final state.
 * append != 0 adds the frame to the file (trajectories hold many frames).  */
#define LLG_FRAME_TRAJECTORY  0
#define LLG_FRAME_FINAL       1
int llg_write_frame(const char* path, int32_t append, double t, int32_t ng, int32_t ny,
                    const double* h_m3, int32_t style);
/* The same from a device vector of ctx's grid (copied on ctx's stream).     */
int llg_write_frame_device(llg_ctx* ctx, const char* path, int32_t append, double t,
                           const double* d_m3, int32_t style);
/* ShouldWriteFrame (2d_i2/2d_fft.cu:457-463): 1 when output iout is due.   */
int llg_should_write_frame(int64_t iout, double t, double early_until, int32_t early_every,
                           int32_t late_every);
/* write_aux_files (2d_i3/2d_fft.cu:390-408): dir/mask.txt from the window w
 * and dir/grain_id.txt, each skipped when its array is NULL.                */
int llg_write_aux_files(const char* dir, int32_t ng, int32_t ny, const double* h_w,
                        const int32_t* h_grain_id);

/* The same active flags, window, per-cell axes and grain ids as
 * llg_build_geometry, built on the device into device buffers (each may be
 * NULL) on cuda_stream (NULL = legacy default); returns the number of
 * active cells.  No counterpart in the reference, whose host builders scan
 * every grain image per cell for the Voronoi partition
 * (2d_i3/2d_fft.cu:300-315) and every hole cell per cell for the window
 * (2d_i3/2d_fft.cu:346-371): here one thread per cell finds its grain with
 * the host's rounding, and the window's hole distances come from an exact
 * two-pass distance transform.  Grain ids and flags are identical to the
 * host builder's; the window agrees to the last bits of tanh.  Initial
 * states stay with llg_build_geometry (they follow the C library's rand()
 * sequence).                                                              */
int llg_build_geometry_device(const llg_geom_spec* g, uint8_t* d_active, double* d_w, double* d_msk3,
                              double* d_nsk3, int32_t* d_grain_id, void* cuda_stream);

/* KEY=VALUE parser using the sim_config.h / params.mk knob names
 * (configs/sim_config.h); lines or whitespace separated; '#' comments.     */
int llg_parse_config(const char* text, llg_params* p, llg_geom_spec* g,
                     llg_solver_opts* o);

#ifdef __cplusplus
}
#endif
#endif /* LLG_H */
