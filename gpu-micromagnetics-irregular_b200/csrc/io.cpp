// io.cpp — the reference's text outputs: magnetisation frames and the
// polycrystal's auxiliary mask / grain-id files.
//
// Formats (what the reference's plotting scripts read):
//   frame   "%f %d %d\n" (t, NX, NY) then one "%f %f %f\n" (mx, my, mz) line
//           per cell, row-major (cell = j*ng + i), then an empty line
//           (WriteFrame, src/irregular/2d_fft/2d_i2/2d_fft.cu:437-455); the
//           final-state file uses "%e %e %e\n" lines and no empty line
//           (2d_i2/2d_fft.cu:735-757).  NX is the reference's x extent in
//           doubles per row, 3*ng (GROUPSIZE 3).
//   cadence ShouldWriteFrame (2d_i2/2d_fft.cu:457-463): output iout is
//           written when iout % EARLY_SAVE_EVERY == 0 while t <=
//           EARLY_SAVE_UNTIL, else when iout % LATE_SAVE_EVERY == 0.
//   aux     mask.txt: "%d %d\n" (ng, ny) then one "%f\n" per cell of the
//           window w; grain_id.txt: the same header then one "%d\n" per cell
//           (write_aux_files, 2d_i3/2d_fft.cu:390-408).
//
// Frames are formatted into one buffer per call and written with a single
// fwrite; the number formatting is the C library's, as in the reference.
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "llg_internal.h"

namespace {

int put_all(const char* path, const char* mode, const std::string& s) {
  FILE* f = fopen(path, mode);
  if (!f) {
    llg_set_error(std::string("cannot open ") + path);
    return LLG_ERR_ARG;
  }
  const size_t w = fwrite(s.data(), 1, s.size(), f);
  const int cl = fclose(f);
  if (w != s.size() || cl != 0) {
    llg_set_error(std::string("short write to ") + path);
    return LLG_ERR_ARG;
  }
  return 0;
}

void append_fmt(std::string& s, const char* fmt, double a, double b, double c) {
  char line[128];
  const int n = snprintf(line, sizeof(line), fmt, a, b, c);
  s.append(line, (size_t)n);
}

}  // namespace

extern "C" {

int llg_should_write_frame(int64_t iout, double t, double early_until, int32_t early_every, int32_t late_every) {
  if (early_every <= 0 || late_every <= 0) {
    llg_set_error("frame cadence must be positive");
    return LLG_ERR_ARG;
  }
  return (t <= early_until) ? (iout % early_every == 0) : (iout % late_every == 0);
}

int llg_write_frame(const char* path, int32_t append, double t, int32_t ng, int32_t ny, const double* h_m3,
                    int32_t style) {
  if (!path || !h_m3 || ng <= 0 || ny <= 0 || (style != LLG_FRAME_TRAJECTORY && style != LLG_FRAME_FINAL)) {
    llg_set_error("llg_write_frame: bad argument");
    return LLG_ERR_ARG;
  }
  const size_t n = (size_t)ng * (size_t)ny;
  std::string s;
  s.reserve(n * 40 + 64);
  char head[96];
  const int hn = snprintf(head, sizeof(head), "%f %d %d\n", t, 3 * ng, ny);
  s.append(head, (size_t)hn);
  const char* fmt = (style == LLG_FRAME_FINAL) ? "%e %e %e\n" : "%f %f %f\n";
  for (size_t cell = 0; cell < n; cell++) append_fmt(s, fmt, h_m3[cell], h_m3[n + cell], h_m3[2 * n + cell]);
  if (style == LLG_FRAME_TRAJECTORY) s.push_back('\n');
  return put_all(path, append ? "ab" : "wb", s);
}

int llg_write_frame_device(llg_ctx* ctx, const char* path, int32_t append, double t, const double* d_m3,
                           int32_t style) {
  if (!ctx || !d_m3) {
    llg_set_error("llg_write_frame_device: bad argument");
    return LLG_ERR_ARG;
  }
  std::vector<double> h((size_t)3 * ctx->ncell);
  LLG_CUDA_TRY(cudaMemcpyAsync(h.data(), d_m3, h.size() * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  LLG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return llg_write_frame(path, append, t, ctx->p.ng, ctx->p.ny, h.data(), style);
}

int llg_write_aux_files(const char* dir, int32_t ng, int32_t ny, const double* h_w, const int32_t* h_grain_id) {
  if (!dir || ng <= 0 || ny <= 0) {
    llg_set_error("llg_write_aux_files: bad argument");
    return LLG_ERR_ARG;
  }
  const size_t n = (size_t)ng * (size_t)ny;
  char head[64];
  const int hn = snprintf(head, sizeof(head), "%d %d\n", ng, ny);
  const std::string base = std::string(dir) + "/";
  if (h_w) {
    std::string s(head, (size_t)hn);
    s.reserve(n * 10 + 32);
    char line[64];
    for (size_t k = 0; k < n; k++) s.append(line, (size_t)snprintf(line, sizeof(line), "%f\n", h_w[k]));
    const int rc = put_all((base + "mask.txt").c_str(), "wb", s);
    if (rc) return rc;
  }
  if (h_grain_id) {
    std::string s(head, (size_t)hn);
    s.reserve(n * 4 + 32);
    char line[32];
    for (size_t k = 0; k < n; k++) s.append(line, (size_t)snprintf(line, sizeof(line), "%d\n", h_grain_id[k]));
    const int rc = put_all((base + "grain_id.txt").c_str(), "wb", s);
    if (rc) return rc;
  }
  return 0;
}

}  // extern "C"
