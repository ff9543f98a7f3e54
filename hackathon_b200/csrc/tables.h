// Host-side FP64 tables the kernels consume: window, twiddles, window
// spectrum, radial bin table and per-analysis temporal metadata. All are
// computed in FP64 and rounded once to FP32 where the device reads FP32, as
// the reference does (ddm-engine.ts:193-197, ddm_ref.js:538-574).
#pragma once

#include <complex>
#include <cstdint>
#include <vector>

namespace ddm {

using cd = std::complex<double>;

// In-place FP64 FFT of a power-of-two length (forward: exp(-2 pi i k t/n)).
void host_fft(std::vector<cd>& a, bool inverse);

// 4-term periodic Blackman-Harris window (fft.js:126-133).
std::vector<double> blackman_harris(int n);

// Per-stage twiddle blocks of the n-point device FFT (layout in
// fft_block.cuh), FP64 rounded to FP32, re/im interleaved.
std::vector<float> twiddle_table(int n, int P = 8);

struct BinTable {
  int N = 0, NB = 0, K = 0;
  double kmin = 0, kmax = 0;
  std::vector<uint32_t> offsets;  // NB + 1
  std::vector<int32_t> modes;     // 4 per entry: mode, kx, ky, 0
  std::vector<double> kCenter;    // NB
  std::vector<uint32_t> nModes;   // NB
  std::vector<double> kNodes;     // NB * K
};

// Radial bin table with effective-|k| quantile nodes (ddm_ref.js:84-170).
BinTable make_bins(int N, int NB, double kmin, double kmax, int K);

// Exact valid-pair counts N(tau), tau < L, and the FFT of the zero-padded
// mask (length TPAD) (ddm_ref.js:538-560, generalised to T/TPAD/L).
void temporal_meta(const float* mask, int T, int TPAD, int L, std::vector<float>& npairs,
                   std::vector<float>& mspec);

}  // namespace ddm
