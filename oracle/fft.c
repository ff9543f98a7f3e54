/*
 * FP64 radix-2 Stockham FFT, direct DFT, Blackman-Harris window and the
 * windowed half-plane 2D spectrum: the oracle's restatement of
 * motility-ddm/src/fft.js. TEST INFRASTRUCTURE ONLY (see oracle.h).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

/* Twiddle table exp(-2*pi*i*m/n), m < n/2, interleaved (fft.js:18-29). The
 * angle is formed as ((-2*pi)*m)/n, the reference's evaluation order. */
static void make_twiddles(double *t, int n) {
  for (int m = 0; m < n / 2; m++) {
    const double a = (-2.0 * M_PI * m) / n;
    t[2 * m] = cos(a);
    t[2 * m + 1] = sin(a);
  }
}

static int is_pow2(int n) { return n >= 1 && (n & (n - 1)) == 0; }

/* Autosort Stockham, natural order, unnormalised both ways (fft.js:59-93).
 * Pass Ns reads src[j], src[j+n/2], twiddles the second by
 * exp(-+2*pi*i*(j%Ns)/(2Ns)) and writes dst[(j/Ns)*2Ns + j%Ns] and +Ns. */
void or_fft(double *data, int n, int inverse) {
  if (!is_pow2(n)) abort(); /* the reference throws (fft.js:35-39) */
  if (n == 1) return;
  /* per-thread twiddle and scratch cache per length (fft.js:10-50) */
  static __thread double *cache_tw[31], *cache_a[31], *cache_b[31];
  const int lg = __builtin_ctz((unsigned)n);
  if (!cache_tw[lg]) {
    cache_tw[lg] = (double *)malloc(sizeof(double) * n);
    cache_a[lg] = (double *)malloc(sizeof(double) * 2 * n);
    cache_b[lg] = (double *)malloc(sizeof(double) * 2 * n);
    make_twiddles(cache_tw[lg], n);
  }
  double *tw = cache_tw[lg], *a = cache_a[lg], *b = cache_b[lg];
  const int half = n >> 1;
  const double sgn = inverse ? -1.0 : 1.0;
  memcpy(a, data, sizeof(double) * 2 * n);
  double *src = a, *dst = b;
  for (int Ns = 1; Ns < n; Ns <<= 1) {
    const int step = half / Ns;
    for (int j = 0; j < half; j++) {
      const int k = j % Ns;
      const double wr = tw[2 * k * step];
      const double wi = sgn * tw[2 * k * step + 1];
      const int i0 = 2 * j, i1 = 2 * (j + half);
      const double xr = src[i1] * wr - src[i1 + 1] * wi;
      const double xi = src[i1] * wi + src[i1 + 1] * wr;
      const int o = 2 * ((j - k) * 2 + k);
      const int o2 = o + 2 * Ns;
      dst[o] = src[i0] + xr;
      dst[o + 1] = src[i0 + 1] + xi;
      dst[o2] = src[i0] - xr;
      dst[o2 + 1] = src[i0 + 1] - xi;
    }
    double *t = src;
    src = dst;
    dst = t;
  }
  memcpy(data, src, sizeof(double) * 2 * n);
}

/* Direct O(n^2) DFT (fft.js:101-119). */
void or_dft(const double *in, double *out, int n, int inverse) {
  const double sgn = inverse ? 1.0 : -1.0;
  for (int k = 0; k < n; k++) {
    double sr = 0, si = 0;
    for (int t = 0; t < n; t++) {
      const double a = (sgn * 2 * M_PI * (double)(((long long)k * t) % n)) / n;
      const double c = cos(a), s = sin(a);
      sr += in[2 * t] * c - in[2 * t + 1] * s;
      si += in[2 * t] * s + in[2 * t + 1] * c;
    }
    out[2 * k] = sr;
    out[2 * k + 1] = si;
  }
}

/* Periodic 4-term Blackman-Harris (fft.js:126-133). */
void or_blackman_harris(double *w, int n) {
  for (int i = 0; i < n; i++) {
    const double x = (2 * M_PI * i) / n;
    w[i] = 0.35875 - 0.48829 * cos(x) + 0.14128 * cos(2 * x) -
           0.01168 * cos(3 * x);
  }
}

/* Mean-subtracted, separably windowed half-plane 2D spectrum scaled by 1/N
 * (fft.js:149-183). out[2*(ky*NH + kx) + {re,im}], kx in [0, N/2]. */
/* Extension (the reference has no spatial mask): with smask != NULL the mean
 * is taken over the pixels where smask != 0, and those pixels alone enter the
 * transform, ((I - mean) * w(x) * w(y) * S(x, y)). smask == NULL is the
 * reference's spectrum2dHalf exactly. */
void or_spectrum2d_half_masked(const double *img, int N, const double *win,
                               const uint8_t *smask, double *out) {
  const int NH = (N >> 1) + 1;
  double mean = 0, cnt = 0;
  if (smask) {
    for (int i = 0; i < N * N; i++)
      if (smask[i]) mean += img[i], cnt += 1;
    mean = cnt > 0 ? mean / cnt : 0;
  } else {
    for (int i = 0; i < N * N; i++) mean += img[i];
    mean /= (double)N * N;
  }
  double *row = (double *)malloc(sizeof(double) * 2 * N);
  double *rows = (double *)malloc(sizeof(double) * 2 * N * NH);
  for (int y = 0; y < N; y++) {
    const double wy = win[y];
    for (int x = 0; x < N; x++) {
      row[2 * x] = (smask && !smask[y * N + x]) ? 0 : (img[y * N + x] - mean) * win[x] * wy;
      row[2 * x + 1] = 0;
    }
    or_fft(row, N, 0);
    for (int kx = 0; kx < NH; kx++) {
      rows[2 * (y * NH + kx)] = row[2 * kx];
      rows[2 * (y * NH + kx) + 1] = row[2 * kx + 1];
    }
  }
  double *col = row;
  const double s = 1.0 / N;
  for (int kx = 0; kx < NH; kx++) {
    for (int y = 0; y < N; y++) {
      col[2 * y] = rows[2 * (y * NH + kx)];
      col[2 * y + 1] = rows[2 * (y * NH + kx) + 1];
    }
    or_fft(col, N, 0);
    for (int ky = 0; ky < N; ky++) {
      out[2 * (ky * NH + kx)] = col[2 * ky] * s;
      out[2 * (ky * NH + kx) + 1] = col[2 * ky + 1] * s;
    }
  }
  free(row);
  free(rows);
}

void or_spectrum2d_half(const double *img, int N, const double *win,
                        double *out) {
  or_spectrum2d_half_masked(img, N, win, NULL, out);
}
