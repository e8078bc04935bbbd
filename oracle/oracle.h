/*
 * oracle.h — CPU FP64 restatement of the reference's 2-D LLG hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the
 * smoke check in __graft_entry__.py and the cpu_baseline / reference arm
 * of bench.py call it to produce the expected answer or the CPU timing.
 * Nothing in the product (libllg.so) links, loads or calls it.
 *
 * Every function names the reference file:line it restates.  Paths are
 * relative to the reference repository root (Angelawoo572/
 * gpu-micromagnetics-irregular).  SUNDIALS (CVODE, SPGMR, Newton) is not
 * part of the reference tree; or_bdf.c restates its published algorithm
 * with the call settings of src/irregular/2d_fft/2d_i2/2d_fft.cu:648-681.
 *
 * Parity pins: the Newell self-coupling N(0) printed by every reference log
 * (src/irregular/2d_fft/2d_i1/scaling_logs/fft_*.txt:8-9) and the reference's
 * own demag_fft.cu built from its sources (oracle/Makefile, target ref).
 */
#ifndef LLG_ORACLE_H
#define LLG_ORACLE_H

#include <stdint.h>
#include "../include/llg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_ctx or_ctx;

or_ctx* or_create(const llg_params* p);
void    or_destroy(or_ctx* c);
/* geometry (copied): active flags (NULL = all active), window + per-cell axes */
int     or_set_active(or_ctx* c, const uint8_t* active);
int     or_set_window(or_ctx* c, const double* w, const double* msk3, const double* nsk3);
int     or_set_threads(int n);

/* operators (host arrays, SoA 3*ncell) */
void    or_normalize(or_ctx* c, double* y);
int     or_rhs(or_ctx* c, double t, double* y, double* ydot);
int     or_jtv(or_ctx* c, const double* v, double* Jv, const double* y);
int     or_psetup(or_ctx* c, const double* y, double gamma);
int     or_psolve(or_ctx* c, const double* r, double* z);
const double* or_hdemag(or_ctx* c);
const double* or_pinv(or_ctx* c);

/* demag */
int     or_demag_apply(or_ctx* c, const double* y, double* h);      /* via FFT    */
int     or_demag_direct(or_ctx* c, const double* y, double* h);     /* O(N^2) sum */
int     or_demag_self(or_ctx* c, double out3[3]);
double  or_demag_tensor(or_ctx* c, int comp, int dx, int dy);       /* unscaled   */
void    or_newell_point(double thick, double sx, double sy, double out9[9]);
void    or_newell_avg(double thick, int dx, int dy, double out9[9]);

/* FFT (complex, interleaved re/im), unnormalised; sign = -1 forward */
int     or_fft(int n, double* data, int sign);

/* integrator */
int     or_integrator_init(or_ctx* c, double t0, const double* y0,
                           const llg_solver_opts* o);
int     or_integrate(or_ctx* c, double tout, double* yout, double* tret);
int     or_get_stats(or_ctx* c, llg_stats* st);

/* geometry / IC builders (same contract as llg_build_geometry) */
int     or_build_geometry(const llg_geom_spec* g, uint8_t* active, double* w,
                          double* msk3, double* nsk3, int32_t* grain_id, double* y0);

/* deterministic reductions used by the integrator */
double  or_wrms(const double* x, const double* w, long n);
double  or_dot(const double* x, const double* y, long n);

#ifdef __cplusplus
}
#endif
#endif
