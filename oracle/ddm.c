/*
 * FP64 DDM analysis: radial bin table, history ring, masked Wiener-Khinchin
 * temporal analysis, radial reduction and temporal metadata. The oracle's
 * restatement of motility-ddm/src/ddm_ref.js. TEST INFRASTRUCTURE ONLY.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define DRIFT_STRIDE 8 /* ddm_ref.js:28 */

static double js_round(double x) { /* Math.round: ties toward +infinity */
  const double r = floor(x);
  return (x - r >= 0.5) ? r + 1.0 : r;
}

/* |W(d)|^2 of the Blackman-Harris window on d = -4..4 (step), normalised to
 * sum 1 (ddm_ref.js:40-55). Returns the number of offsets. */
int or_window_leakage(int N, double step, double *d, double *p) {
  double *w = (double *)malloc(sizeof(double) * N);
  or_blackman_harris(w, N);
  int cnt = 0;
  for (double x = -4; x <= 4 + 1e-9; x += step) {
    double re = 0, im = 0;
    for (int n = 0; n < N; n++) {
      const double a = (-2 * M_PI * x * n) / N;
      re += w[n] * cos(a);
      im += w[n] * sin(a);
    }
    d[cnt] = x;
    p[cnt] = re * re + im * im;
    cnt++;
  }
  double s = 0;
  for (int i = 0; i < cnt; i++) s += p[i];
  for (int i = 0; i < cnt; i++) p[i] = p[i] / s;
  free(w);
  return cnt;
}

/* Signed wavevector of half-plane mode m (ddm_ref.js:63-69). */
void or_mode_k(int m, int N, int *kx, int *ky) {
  const int NH = (N >> 1) + 1;
  *kx = m % NH;
  const int kyi = (m - *kx) / NH;
  *ky = kyi < N / 2 ? kyi : kyi - N;
}

/* Bin of mode m or -1 (ddm_ref.js:89-96). sqrt(kx^2+ky^2) is exact-input
 * correctly rounded, which gives the same bins as the reference's Math.hypot
 * at every geometry used here (checked by the tests). */
static int mode_bin(int m, int N, int NB, double kmin, double width) {
  int kx, ky;
  or_mode_k(m, N, &kx, &ky);
  if (kx == 0 && ky <= 0) return -1;
  if (kx == N / 2 || ky == -N / 2) return -1; /* Nyquist lines */
  const double kr = sqrt((double)kx * kx + (double)ky * ky);
  const double b = floor((kr - kmin) / width);
  if (b >= 0 && b < NB) return (int)b;
  return -1;
}

int or_make_bins_count(int N, int NB, double kmin, double kmax) {
  const int NH = (N >> 1) + 1;
  const double width = (kmax - kmin) / NB;
  int total = 0;
  for (int m = 0; m < N * NH; m++)
    if (mode_bin(m, N, NB, kmin, width) >= 0) total++;
  return total;
}

/* Radial bin table with effective-|k| quantile nodes (ddm_ref.js:84-170). */
void or_make_bins(int N, int NB, double kmin, double kmax, int K,
                  uint32_t *binOffsets, int32_t *binModes, double *kCenter,
                  uint32_t *nModes, double *kNodes) {
  const int NH = (N >> 1) + 1;
  const int M = N * NH;
  const double width = (kmax - kmin) / NB;
  int *bin = (int *)malloc(sizeof(int) * M);
  for (int b = 0; b <= NB; b++) binOffsets[b] = 0;
  for (int m = 0; m < M; m++) {
    bin[m] = mode_bin(m, N, NB, kmin, width);
    if (bin[m] >= 0) binOffsets[bin[m] + 1]++;
  }
  for (int b = 0; b < NB; b++) binOffsets[b + 1] += binOffsets[b];
  uint32_t *fill = (uint32_t *)calloc(NB, sizeof(uint32_t));
  for (int m = 0; m < M; m++) { /* modes in increasing order per bin */
    if (bin[m] < 0) continue;
    const uint32_t o = 4 * (binOffsets[bin[m]] + fill[bin[m]]++);
    int kx, ky;
    or_mode_k(m, N, &kx, &ky);
    binModes[o] = m;
    binModes[o + 1] = kx;
    binModes[o + 2] = ky;
    binModes[o + 3] = 0;
  }
  double ld[64], lp[64];
  const int nl = or_window_leakage(N, 0.5, ld, lp);
  const double h0 = fmax(0.0, kmin - 6), hres = 0.01;
  const int hlen = (int)ceil((kmax + 6 - h0) / hres) + 1;
  double *hist = (double *)malloc(sizeof(double) * hlen);
  double *hk = (double *)malloc(sizeof(double) * hlen);
  for (int b = 0; b < NB; b++) {
    const uint32_t i0 = binOffsets[b], i1 = binOffsets[b + 1];
    double sk = 0;
    for (uint32_t i = i0; i < i1; i++) {
      const double kx = binModes[4 * i + 1], ky = binModes[4 * i + 2];
      sk += sqrt(kx * kx + ky * ky);
    }
    nModes[b] = i1 - i0;
    kCenter[b] = nModes[b] ? sk / nModes[b] : kmin + (b + 0.5) * width;
    memset(hist, 0, sizeof(double) * hlen);
    memset(hk, 0, sizeof(double) * hlen);
    for (uint32_t i = i0; i < i1; i++) {
      const double kx = binModes[4 * i + 1], ky = binModes[4 * i + 2];
      for (int a = 0; a < nl; a++) {
        const double ax = kx + ld[a];
        for (int c = 0; c < nl; c++) {
          const double ay = ky + ld[c];
          const double k = sqrt(ax * ax + ay * ay);
          const double wt = lp[a] * lp[c];
          double cc = js_round((k - h0) / hres);
          if (cc < 0) cc = 0;
          if (cc > hlen - 1) cc = hlen - 1;
          hist[(int)cc] += wt;
          hk[(int)cc] += wt * k;
        }
      }
    }
    double wsum = 0;
    for (int c = 0; c < hlen; c++) wsum += hist[c];
    if (!(wsum > 0)) {
      for (int n = 0; n < K; n++) kNodes[b * K + n] = kCenter[b];
      continue;
    }
    /* node n = weighted mean |k| of the n-th equal-weight quantile slice */
    double acc = 0, sw = 0, swk = 0;
    int n = 0;
    for (int c = 0; c < hlen && n < K; c++) {
      double rem = hist[c];
      const double kc = hist[c] > 0 ? hk[c] / hist[c] : 0;
      while (rem > 0 && n < K) {
        const double target = ((double)(n + 1) / K) * wsum;
        const double take = fmin(rem, target - acc);
        sw += take;
        swk += take * kc;
        acc += take;
        rem -= take;
        if (acc >= ((double)(n + 1) / K) * wsum * (1 - 1e-12)) {
          kNodes[b * K + n] = sw > 0 ? swk / sw : kc;
          n++;
          sw = 0;
          swk = 0;
        }
      }
    }
    for (; n < K; n++) kNodes[b * K + n] = kmax;
  }
  free(bin);
  free(fill);
  free(hist);
  free(hk);
}

/* Transform luma frames into ring slots (ddm_ref.js:196-206); smask: the
 * spatial-mask extension of or_spectrum2d_half_masked (NULL = none). */
void or_history_ingest_masked(double *hist, int N, int T, const double *luma,
                              const uint8_t *smask, const int *slots, int nframes) {
  const int NH = (N >> 1) + 1, M = N * NH;
  double *win = (double *)malloc(sizeof(double) * N);
  or_blackman_harris(win, N);
#pragma omp parallel for schedule(dynamic)
  for (int f = 0; f < nframes; f++) {
    double *spec = (double *)malloc(sizeof(double) * 2 * M);
    or_spectrum2d_half_masked(luma + (size_t)f * N * N, N, win, smask, spec);
    const int slot = slots[f];
    for (int m = 0; m < M; m++) {
      const size_t o = ((size_t)m * T + slot) * 2;
      hist[o] = spec[2 * m];
      hist[o + 1] = spec[2 * m + 1];
    }
    free(spec);
  }
  free(win);
}

void or_history_ingest(double *hist, int N, int T, const double *luma,
                       const int *slots, int nframes) {
  or_history_ingest_masked(hist, N, T, luma, NULL, slots, nframes);
}

/* Masked Wiener-Khinchin structure function of one mode (ddm_ref.js:229-288).
 * z = m + i*p packs the mask and the power so A and N(tau) come from one FFT;
 * G = IFFT(|FFT(y)|^2). n = TPAD (the reference fixes n = 2T). */
double or_temporal_mode(const double *hist, int mode, int T, int TPAD,
                        const uint32_t *order, const double *mask, int L,
                        double *outD, double *outC) {
  const int n = TPAD;
  double *z = (double *)calloc(2 * n, sizeof(double));
  double *y = (double *)calloc(2 * n, sizeof(double));
  double *S = (double *)malloc(sizeof(double) * 2 * n);
  const size_t base = (size_t)mode * T * 2;
  for (int j = 0; j < T; j++) {
    if (!mask[j]) continue;
    const uint32_t s = order[j];
    const double xr = hist[base + 2 * s], xi = hist[base + 2 * s + 1];
    z[2 * j] = 1;
    z[2 * j + 1] = xr * xr + xi * xi;
    y[2 * j] = xr;
    y[2 * j + 1] = xi;
  }
  or_fft(z, n, 0);
  for (int k = 0; k < n; k++) {
    const int kk = (n - k) % n;
    const double zr = z[2 * k], zi = z[2 * k + 1];
    const double cr = z[2 * kk], ci = -z[2 * kk + 1]; /* conj(Z[-k]) */
    const double Mr = 0.5 * (zr + cr), Mi = 0.5 * (zi + ci);
    const double dr = zr - cr, di = zi - ci;
    const double Pr = 0.5 * di, Pi = -0.5 * dr; /* (Z_k - conj Z_-k)/(2i) */
    S[2 * k] = Mr * Pr + Mi * Pi; /* conj(M) P + i |M|^2 */
    S[2 * k + 1] = Mr * Pi - Mi * Pr + (Mr * Mr + Mi * Mi);
  }
  or_fft(S, n, 1);
  or_fft(y, n, 0);
  for (int k = 0; k < n; k++) {
    const double yr = y[2 * k], yi = y[2 * k + 1];
    y[2 * k] = yr * yr + yi * yi;
    y[2 * k + 1] = 0;
  }
  or_fft(y, n, 1);
  const double inv = 1.0 / n;
  const double den = S[1] * inv > 1e-300 ? S[1] * inv : 1e-300;
  const double P = S[0] * inv / den;
  for (int tau = 0; tau < L; tau++) {
    const double A = S[2 * tau] * inv;
    const double B = S[2 * ((n - tau) % n)] * inv;
    const double Np = js_round(S[2 * tau + 1] * inv);
    if (Np > 0) {
      const double Gr = y[2 * tau] * inv, Gi = y[2 * tau + 1] * inv;
      outD[tau] = (A + B - 2 * Gr) / Np;
      outC[2 * tau] = Gr / Np;
      outC[2 * tau + 1] = Gi / Np;
    } else {
      outD[tau] = 0;
      outC[2 * tau] = 0;
      outC[2 * tau + 1] = 0;
    }
  }
  const double res = S[1] * inv > 0.5 ? P : 0;
  free(z);
  free(y);
  free(S);
  return res;
}

/* Direct O(T*L) masked estimators (ddm_ref.js:306-333). */
double or_temporal_mode_direct(const double *hist, int mode, int T,
                               const uint32_t *order, const double *mask,
                               int L, double *outD, double *outC) {
  const size_t base = (size_t)mode * T * 2;
  double *xr = (double *)calloc(T, sizeof(double));
  double *xi = (double *)calloc(T, sizeof(double));
  double pSum = 0, nSum = 0;
  for (int j = 0; j < T; j++) {
    if (!mask[j]) continue;
    xr[j] = hist[base + 2 * order[j]];
    xi[j] = hist[base + 2 * order[j] + 1];
    pSum += xr[j] * xr[j] + xi[j] * xi[j];
    nSum++;
  }
  for (int tau = 0; tau < L; tau++) {
    double d = 0, gr = 0, gi = 0, cnt = 0;
    for (int t = 0; t + tau < T; t++) {
      if (!mask[t] || !mask[t + tau]) continue;
      const double dr = xr[t + tau] - xr[t], di = xi[t + tau] - xi[t];
      d += dr * dr + di * di;
      gr += xr[t] * xr[t + tau] + xi[t] * xi[t + tau];
      gi += xr[t] * xi[t + tau] - xi[t] * xr[t + tau];
      cnt++;
    }
    outD[tau] = cnt ? d / cnt : 0;
    outC[2 * tau] = cnt ? gr / cnt : 0;
    outC[2 * tau + 1] = cnt ? gi / cnt : 0;
  }
  free(xr);
  free(xi);
  return nSum ? pSum / nSum : 0;
}

/* Add one mode to the radial sums of bin b (ddm_ref.js:360-382). */
static void accumulate_mode(int L, int b, int kx, int ky, const double *D,
                            const double *C, double P, double *rD, double *rP,
                            double *rDrift) {
  rP[b] += P;
  for (int tau = 0; tau < L; tau++) rD[b * L + tau] += D[tau];
  for (int tau = 0; tau < L - 1; tau++) {
    const double ar = C[2 * tau], ai = C[2 * tau + 1];
    const double br = C[2 * tau + 2], bi = C[2 * tau + 3];
    const double zr = br * ar + bi * ai; /* C(tau+1) conj C(tau) */
    const double zi = bi * ar - br * ai;
    const double w = hypot(zr, zi);
    const double phi = atan2(zi, zr);
    double *o = rDrift + (size_t)(b * L + tau) * DRIFT_STRIDE;
    o[0] += w;
    o[1] += w * kx * kx;
    o[2] += w * kx * ky;
    o[3] += w * ky * ky;
    o[4] += w * kx * phi;
    o[5] += w * ky * phi;
    o[6] += w * phi * phi;
    o[7] += w > 0 ? 1 : 0;
  }
}

static void finalize_radial(int NB, int L, const uint32_t *nModes, double *D,
                            double *P) { /* ddm_ref.js:404-412 */
  for (int b = 0; b < NB; b++) {
    const uint32_t n = nModes[b];
    if (!n) continue;
    P[b] /= n;
    for (int tau = 0; tau < L; tau++) D[b * L + tau] /= n;
  }
}

/* ddm_ref.js:425-437. Bins are independent, so they run in parallel while
 * each bin's sums keep the reference's mode order. */
void or_analyze_radial(const double *hist, int N, int T, int TPAD,
                       const uint32_t *order, const double *mask, int NB,
                       const uint32_t *binOffsets, const int32_t *binModes,
                       const uint32_t *nModes, int L, double *D, double *P,
                       double *drift, int threads) {
  (void)N;
  memset(D, 0, sizeof(double) * NB * L);
  memset(P, 0, sizeof(double) * NB);
  memset(drift, 0, sizeof(double) * NB * L * DRIFT_STRIDE);
#pragma omp parallel for schedule(dynamic) num_threads(threads > 0 ? threads : 1)
  for (int b = 0; b < NB; b++) {
    double *d = (double *)malloc(sizeof(double) * L);
    double *c = (double *)malloc(sizeof(double) * 2 * L);
    for (uint32_t i = binOffsets[b]; i < binOffsets[b + 1]; i++) {
      const int m = binModes[4 * i];
      const double p = or_temporal_mode(hist, m, T, TPAD, order, mask, L, d, c);
      accumulate_mode(L, b, binModes[4 * i + 1], binModes[4 * i + 2], d, c, p,
                      D, P, drift);
    }
    free(d);
    free(c);
  }
  finalize_radial(NB, L, nModes, D, P);
}

/* ddm_ref.js:450-463 over an explicit list of modes. */
void or_analyze_modes(const double *hist, int T, int TPAD,
                      const uint32_t *order, const double *mask, int L,
                      const int32_t *modes, int nmodes, double *D, double *C,
                      double *P, int threads) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
  for (int i = 0; i < nmodes; i++)
    P[i] = or_temporal_mode(hist, modes[i], T, TPAD, order, mask, L,
                            D + (size_t)i * L, C + (size_t)i * 2 * L);
}

/* ddm_ref.js:474-487 */
void or_radial_from_full(const double *fullD, const double *fullC,
                         const double *fullP, int NB,
                         const uint32_t *binOffsets, const int32_t *binModes,
                         const uint32_t *nModes, int L, double *D, double *P,
                         double *drift) {
  memset(D, 0, sizeof(double) * NB * L);
  memset(P, 0, sizeof(double) * NB);
  memset(drift, 0, sizeof(double) * NB * L * DRIFT_STRIDE);
  for (int b = 0; b < NB; b++) {
    for (uint32_t i = binOffsets[b]; i < binOffsets[b + 1]; i++) {
      const size_t m = (size_t)binModes[4 * i];
      accumulate_mode(L, b, binModes[4 * i + 1], binModes[4 * i + 2],
                      fullD + m * L, fullC + m * 2 * L, fullP[m], D, P, drift);
    }
  }
  finalize_radial(NB, L, nModes, D, P);
}

/* ddm_ref.js:538-560: exact pair counts N(tau) and the FP64 spectrum of the
 * zero-padded mask. */
void or_temporal_meta(const uint32_t *order, const double *mask, int T,
                      int TPAD, int L, double *npairs, double *mspec) {
  (void)order;
  memset(mspec, 0, sizeof(double) * 2 * TPAD);
  for (int j = 0; j < T; j++) mspec[2 * j] = mask[j] ? 1 : 0;
  for (int tau = 0; tau < L; tau++) {
    int c = 0;
    for (int t = 0; t + tau < T; t++)
      if (mask[t] && mask[t + tau]) c++;
    npairs[tau] = c;
  }
  or_fft(mspec, TPAD, 0);
}
