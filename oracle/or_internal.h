/*
 * or_internal.h — shared state of the CPU oracle (test infrastructure only).
 */
#ifndef LLG_OR_INTERNAL_H
#define LLG_OR_INTERNAL_H

#include "oracle.h"

typedef struct or_demag {
  int px, py;             /* transform grid (ng x ny periodic, 2ng x 2ny open) */
  double strength, thick;
  double* t[9];           /* unscaled tensor, wrapped placement, px*py each    */
  double* that[9];        /* complex spectra, interleaved, px*py each          */
  double n0[3];           /* unscaled N(0) diagonal                            */
} or_demag;

typedef struct or_bdf or_bdf;

struct or_ctx {
  llg_params p;
  long ncell, neq;
  uint8_t* active;        /* NULL = all active                                 */
  double* w;              /* windowed only                                     */
  double* msk3;
  double* nsk3;
  double* hd;             /* demag field of the last or_rhs call (3*ncell)     */
  double* pinv;           /* 9*ncell block-Jacobi inverses                     */
  double src_h;           /* soft-source field of the last or_rhs call's t      */
  or_demag* dm;
  or_bdf* bdf;
};

or_demag* or_demag_create(const llg_params* p);
void      or_demag_free(or_demag* d);
int       or_demag_run(const or_ctx* c, const double* y, double* h);

#endif
