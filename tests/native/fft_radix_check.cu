// fft_radix_check.cu — host-side check of the in-register DFTs of the
// shared-memory FFT core (csrc/dev_fft.cuh): every fixed radix, both
// directions, FP64 and FP32, against a direct DFT in long double.  The
// butterflies are __host__ __device__, so this runs on the CPU; it prints one
// line per case and exits non-zero if any error is above its bound.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include "dev_fft.cuh"

template <typename R, int RAD, int SIGN>
static int check(double bound) {
  cx_t<R> v[RAD];
  long double xr[RAD], xi[RAD];
  unsigned s = 12345u + 977u * RAD + (SIGN > 0 ? 7u : 0u);
  for (int r = 0; r < RAD; r++) {
    s = s * 1664525u + 1013904223u;
    const double a = (double)(s >> 8) / 16777216.0 - 0.5;
    s = s * 1664525u + 1013904223u;
    const double b = (double)(s >> 8) / 16777216.0 - 0.5;
    v[r] = mk<R>((R)a, (R)b);
    xr[r] = (long double)v[r].x;
    xi[r] = (long double)v[r].y;
  }
  dft_fixed<R, RAD, SIGN>(v);
  const long double pi = 3.14159265358979323846264338327950288L;
  double err = 0.0, scale = 0.0;
  for (int q = 0; q < RAD; q++) {
    long double yr = 0.0L, yi = 0.0L;
    for (int r = 0; r < RAD; r++) {
      const long double ang = (long double)SIGN * 2.0L * pi * (long double)((r * q) % RAD) / (long double)RAD;
      const long double c = cosl(ang), sn = sinl(ang);
      yr += xr[r] * c - xi[r] * sn;
      yi += xr[r] * sn + xi[r] * c;
    }
    err = fmax(err, fmax(fabs((double)(yr - (long double)v[q].x)), fabs((double)(yi - (long double)v[q].y))));
    scale = fmax(scale, fmax(fabs((double)yr), fabs((double)yi)));
  }
  const double rel = err / scale;
  const int bad = !(rel <= bound);
  printf("%s radix %2d sign %+d: rel err %.3e (bound %.1e)%s\n", sizeof(R) == 8 ? "f64" : "f32", RAD, SIGN, rel,
         bound, bad ? "  FAIL" : "");
  return bad;
}

template <typename R>
static int all(double bound) {
  int bad = 0;
  bad += check<R, 2, -1>(bound) + check<R, 2, 1>(bound);
  bad += check<R, 3, -1>(bound) + check<R, 3, 1>(bound);
  bad += check<R, 4, -1>(bound) + check<R, 4, 1>(bound);
  bad += check<R, 5, -1>(bound) + check<R, 5, 1>(bound);
  bad += check<R, 6, -1>(bound) + check<R, 6, 1>(bound);
  bad += check<R, 8, -1>(bound) + check<R, 8, 1>(bound);
  bad += check<R, 12, -1>(bound) + check<R, 12, 1>(bound);
  bad += check<R, 16, -1>(bound) + check<R, 16, 1>(bound);
  return bad;
}

int main() {
  const int bad = all<double>(1e-15) + all<float>(1e-6);
  return bad ? 1 : 0;
}
