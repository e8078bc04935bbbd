// reference_api.cu — the reference's own module entry points, implemented on
// top of libllg.so so existing callers link unchanged.
//
//   Demag_Init / Demag_Apply / Demag_Destroy / Demag_GetSelfCoupling
//        src/irregular/2d_fft/2d_i2/demag_fft.h:29-42
//   Demag_ApplyWindowed / Demag_SetStream
//        src/irregular/2d_fft/2d_i3/demag_fft.h:36-43
//   Precond_Create / Precond_Destroy
//        src/irregular/2d_fft/2d_i2/precond.h:28-29
//
// Semantics follow the reference: Demag_Init(nx, ny, thick, strength) takes
// the cell grid (nx = ng cells) with periodic (un-padded) boundaries; the
// output is overwritten, scaled by strength; GetSelfCoupling returns
// N(0)·strength.  Demag_InitOpen is the zero-padded (open-boundary) twin.
#include <stdio.h>
#include <string.h>

#include "llg_internal.h"

struct DemagData {
  llg_ctx* ctx;
};

struct PrecondData {
  int ng, ny, ncell;
};

static DemagData* demag_init_mode(int nx, int ny, double thick, double strength, int mode) {
  llg_params p;
  llg_default_params(&p);
  p.ng = nx;
  p.ny = ny;
  p.bc = LLG_BC_PERIODIC;
  p.demag_mode = mode;
  p.demag_thick = thick;
  p.demag_strength = strength;
  llg_ctx* c = nullptr;
  if (llg_create(&p, &c) != 0) {
    fprintf(stderr, "[Demag B200] init failed: %s\n", llg_last_error());
    return nullptr;
  }
  DemagData* d = new DemagData();
  d->ctx = c;
  return d;
}

extern "C" {

DemagData* Demag_Init(int nx, int ny, double thick, double demag_strength) {
  return demag_init_mode(nx, ny, thick, demag_strength, LLG_DEMAG_PERIODIC);
}

DemagData* Demag_InitOpen(int nx, int ny, double thick, double demag_strength) {
  return demag_init_mode(nx, ny, thick, demag_strength, LLG_DEMAG_OPEN);
}

void Demag_Apply(DemagData* d, const double* y_dev, double* h_out_dev) {
  if (!d) return;
  demag_apply_w(d->ctx, y_dev, nullptr, h_out_dev);
}

void Demag_ApplyWindowed(DemagData* d, const double* y_dev, const double* w_dev, double* h_out_dev) {
  if (!d) return;
  demag_apply_w(d->ctx, y_dev, w_dev, h_out_dev);
}

void Demag_SetStream(DemagData* d, struct CUstream_st* stream) {
  if (!d) return;
  d->ctx->stream = (cudaStream_t)stream;
}

void Demag_GetSelfCoupling(DemagData* d, double* nxx0, double* nyy0, double* nzz0) {
  double v[3] = {0.0, 0.0, 0.0};
  if (d) demag_self(d->ctx, v);
  if (nxx0) *nxx0 = v[0];
  if (nyy0) *nyy0 = v[1];
  if (nzz0) *nzz0 = v[2];
}

void Demag_Destroy(DemagData* d) {
  if (!d) return;
  llg_destroy(d->ctx);
  delete d;
}

PrecondData* Precond_Create(int ng, int ny, int ncell) {
  if (ng <= 0 || ny <= 0 || ncell != ng * ny) return nullptr;
  PrecondData* pd = new PrecondData();
  pd->ng = ng;
  pd->ny = ny;
  pd->ncell = ncell;
  return pd;
}

void Precond_Destroy(PrecondData* pd) { delete pd; }

}  // extern "C"
