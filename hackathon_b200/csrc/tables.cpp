#include "tables.h"

#include <algorithm>
#include <cmath>

namespace ddm {

// Decimation in time by the smallest prime factor p of n (p = 2 or 3, else
// a direct DFT): p transforms of n/p points, combined with FP64 twiddles.
// For lengths that are not powers of two (384, 768).
static void mixed_fft(std::vector<cd>& a, bool inverse) {
  const size_t n = a.size();
  if (n <= 1) return;
  const size_t p = n % 2 == 0 ? 2 : n % 3 == 0 ? 3 : n;
  const double sgn = inverse ? 1.0 : -1.0;
  if (p == n) {
    std::vector<cd> out(n);
    for (size_t k = 0; k < n; k++) {
      cd s(0, 0);
      for (size_t j = 0; j < n; j++) {
        const double ang = sgn * 2.0 * M_PI * (double)((j * k) % n) / (double)n;
        s += a[j] * cd(std::cos(ang), std::sin(ang));
      }
      out[k] = s;
    }
    a.swap(out);
    return;
  }
  const size_t m = n / p;
  std::vector<std::vector<cd>> sub(p, std::vector<cd>(m));
  for (size_t r = 0; r < p; r++)
    for (size_t k = 0; k < m; k++) sub[r][k] = a[k * p + r];
  for (size_t r = 0; r < p; r++) mixed_fft(sub[r], inverse);
  for (size_t k = 0; k < n; k++) {
    cd s(0, 0);
    for (size_t r = 0; r < p; r++) {
      const double ang = sgn * 2.0 * M_PI * (double)((r * k) % n) / (double)n;
      s += sub[r][k % m] * cd(std::cos(ang), std::sin(ang));
    }
    a[k] = s;
  }
}

void host_fft(std::vector<cd>& a, bool inverse) {
  const size_t n = a.size();
  if (n & (n - 1)) {  // not a power of two
    mixed_fft(a, inverse);
    return;
  }
  for (size_t i = 1, j = 0; i < n; i++) {  // bit reversal
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  const double sgn = inverse ? 1.0 : -1.0;
  for (size_t len = 2; len <= n; len <<= 1) {
    const size_t h = len / 2;
    for (size_t k = 0; k < h; k++) {
      const double ang = sgn * 2.0 * M_PI * (double)k / (double)len;
      const cd w(std::cos(ang), std::sin(ang));
      for (size_t i = 0; i < n; i += len) {
        const cd u = a[i + k], v = a[i + k + h] * w;
        a[i + k] = u + v;
        a[i + k + h] = u - v;
      }
    }
  }
}

std::vector<double> blackman_harris(int n) {
  std::vector<double> w(n);
  for (int i = 0; i < n; i++) {
    const double x = 2.0 * M_PI * i / n;
    w[i] = 0.35875 - 0.48829 * std::cos(x) + 0.14128 * std::cos(2 * x) - 0.01168 * std::cos(3 * x);
  }
  return w;
}

std::vector<float> twiddle_table(int n, int P) {
  // stage blocks w[(m-1)*Ns + k] = exp(-2 pi i m k / (Ns R)) (fft_block.cuh),
  // radix P while n/Ns >= P, then the remainder; sizes with a factor 3 take
  // the mixed-radix plan of fft_p (radix 8 while n/Ns is a multiple of 8,
  // then 6, 4, 3, 2)
  std::vector<float> t;
  const bool mixed = n % 3 == 0;
  for (int ns = 1; ns < n;) {
    const int q = n / ns;
    const int r = mixed ? (q % 8 == 0 ? 8 : q % 6 == 0 ? 6 : q % 4 == 0 ? 4 : q % 3 == 0 ? 3 : 2)
                        : (q >= P ? P : q);
    if (ns > 1)
      for (int m = 1; m < r; m++)
        for (int k = 0; k < ns; k++) {
          const double a = -2.0 * M_PI * (double)(m * k) / (double)(ns * r);
          t.push_back((float)std::cos(a));
          t.push_back((float)std::sin(a));
        }
    ns *= r;
  }
  if (t.empty()) t.assign(2, 0.f);
  return t;
}

// |W(d)|^2 of the window at fractional bin offsets d = -4..4 step 0.5,
// normalised to sum 1 (ddm_ref.js:40-55).
static void window_leakage(int N, std::vector<double>& d, std::vector<double>& p) {
  const std::vector<double> w = blackman_harris(N);
  d.clear();
  p.clear();
  for (double x = -4; x <= 4 + 1e-9; x += 0.5) {
    double re = 0, im = 0;
    for (int n = 0; n < N; n++) {
      const double a = (-2 * M_PI * x * n) / N;
      re += w[n] * std::cos(a);
      im += w[n] * std::sin(a);
    }
    d.push_back(x);
    p.push_back(re * re + im * im);
  }
  double s = 0;
  for (double v : p) s += v;
  for (double& v : p) v /= s;
}

BinTable make_bins(int N, int NB, double kmin, double kmax, int K) {
  BinTable b;
  b.N = N;
  b.NB = NB;
  b.K = K;
  b.kmin = kmin;
  b.kmax = kmax;
  const int NH = N / 2 + 1;
  const double width = (kmax - kmin) / NB;
  std::vector<std::vector<int>> lists(NB);
  for (int m = 0; m < N * NH; m++) {
    const int kx = m % NH, kyi = m / NH;
    const int ky = kyi < N / 2 ? kyi : kyi - N;
    if (kx == 0 && ky <= 0) continue;            // conjugates of ky > 0
    if (kx == N / 2 || ky == -N / 2) continue;   // Nyquist lines
    // sqrt of the exact integer sum: correctly rounded, the same bin as the
    // reference's Math.hypot at every supported geometry
    const double kr = std::sqrt((double)kx * kx + (double)ky * ky);
    const double bb = std::floor((kr - kmin) / width);
    if (bb >= 0 && bb < NB) lists[(int)bb].push_back(m);
  }
  b.offsets.assign(NB + 1, 0);
  for (int i = 0; i < NB; i++) b.offsets[i + 1] = b.offsets[i] + (uint32_t)lists[i].size();
  b.modes.assign(4 * (size_t)b.offsets[NB], 0);
  b.kCenter.assign(NB, 0);
  b.nModes.assign(NB, 0);
  b.kNodes.assign((size_t)NB * K, 0);
  std::vector<double> ld, lp;
  window_leakage(N, ld, lp);
  const double h0 = std::max(0.0, kmin - 6), hres = 0.01;
  const int hlen = (int)std::ceil((kmax + 6 - h0) / hres) + 1;
  std::vector<double> hist(hlen), hk(hlen);
  for (int bin = 0; bin < NB; bin++) {
    double sk = 0;
    for (size_t i = 0; i < lists[bin].size(); i++) {
      const int m = lists[bin][i];
      const int kx = m % NH, kyi = m / NH;
      const int ky = kyi < N / 2 ? kyi : kyi - N;
      const size_t o = 4 * ((size_t)b.offsets[bin] + i);
      b.modes[o] = m;
      b.modes[o + 1] = kx;
      b.modes[o + 2] = ky;
      sk += std::sqrt((double)kx * kx + (double)ky * ky);
    }
    const size_t n = lists[bin].size();
    b.nModes[bin] = (uint32_t)n;
    b.kCenter[bin] = n ? sk / n : kmin + (bin + 0.5) * width;
    // leakage-smeared |k| histogram (resolution 0.01), then K equal-weight
    // quantile slices, node = weighted mean |k| of each slice
    std::fill(hist.begin(), hist.end(), 0.0);
    std::fill(hk.begin(), hk.end(), 0.0);
    for (size_t i = 0; i < n; i++) {
      const size_t o = 4 * ((size_t)b.offsets[bin] + i);
      const double kx = b.modes[o + 1], ky = b.modes[o + 2];
      for (size_t a = 0; a < ld.size(); a++) {
        const double ax = kx + ld[a];
        for (size_t c = 0; c < ld.size(); c++) {
          const double ay = ky + ld[c];
          const double k = std::sqrt(ax * ax + ay * ay);
          const double wt = lp[a] * lp[c];
          const double f = (k - h0) / hres;
          double r = std::floor(f);
          if (f - r >= 0.5) r += 1;  // round half up
          const int cell = (int)std::min<double>(hlen - 1, std::max(0.0, r));
          hist[cell] += wt;
          hk[cell] += wt * k;
        }
      }
    }
    double wsum = 0;
    for (double v : hist) wsum += v;
    if (!(wsum > 0)) {
      for (int q = 0; q < K; q++) b.kNodes[(size_t)bin * K + q] = b.kCenter[bin];
      continue;
    }
    double acc = 0, sw = 0, swk = 0;
    int q = 0;
    for (int c = 0; c < hlen && q < K; c++) {
      double rem = hist[c];
      const double kc = hist[c] > 0 ? hk[c] / hist[c] : 0;
      while (rem > 0 && q < K) {
        const double take = std::min(rem, ((double)(q + 1) / K) * wsum - acc);
        sw += take;
        swk += take * kc;
        acc += take;
        rem -= take;
        if (acc >= ((double)(q + 1) / K) * wsum * (1 - 1e-12)) {
          b.kNodes[(size_t)bin * K + q] = sw > 0 ? swk / sw : kc;
          q++;
          sw = 0;
          swk = 0;
        }
      }
    }
    for (; q < K; q++) b.kNodes[(size_t)bin * K + q] = kmax;
  }
  return b;
}

void temporal_meta(const float* mask, int T, int TPAD, int L, std::vector<float>& npairs,
                   std::vector<float>& mspec) {
  std::vector<uint8_t> m(T);
  for (int j = 0; j < T; j++) m[j] = mask[j] != 0.f;
  npairs.assign(L, 0.f);
  for (int tau = 0; tau < L; tau++) {
    int c = 0;
    for (int t = 0; t + tau < T; t++) c += m[t] & m[t + tau];
    npairs[tau] = (float)c;
  }
  std::vector<cd> z(TPAD, cd(0, 0));
  for (int j = 0; j < T; j++) z[j] = cd(m[j], 0);
  host_fft(z, false);
  mspec.resize(2 * (size_t)TPAD);
  for (int k = 0; k < TPAD; k++) {
    mspec[2 * k] = (float)z[k].real();
    mspec[2 * k + 1] = (float)z[k].imag();
  }
}

}  // namespace ddm
