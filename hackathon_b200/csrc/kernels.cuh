// Kernel parameter blocks and launchers shared by the engine.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "isf.cuh"

namespace ddm {

constexpr int KB = 2;       // kx columns per block of the row-spectrum scratch
constexpr int DRIFT = 8;    // drift fields per (bin, lag) (ddm_ref.js:28)
constexpr int PFIELDS = 9;  // D + 8 drift sums per lag in a partial record
constexpr int MAX_CHUNK = 256;  // frames per spatial launch (slots travel as a kernel parameter)

struct RowParams {
  const void* frames;      // [nframes][N][N] u8 / u16 / f32 (16-byte aligned)
  long long frame_stride;  // elements between frames
  int nframes;
  const float* win;        // w(x), FP32 (from the FP64 window)
  const float* wys;        // w(y) * scale
  const uint8_t* smask;    // spatial mask [N][N] or nullptr (extension)
  const float2* tw;        // per-stage twiddle blocks of the N-point FFT
  float2* rows;            // [nframes][NHB][KB][N]
  float* framec;           // [nframes] frame reference level c_f (raw units, out)
  double* framesum;        // [nframes] masked pixel sums (zeroed before launch)
  int* err;                // error word (bounded waits that timed out), or nullptr
  int framec_ready;        // 1: framec already holds these frames' c_f (launch_cref ran for the call)
};

struct ColParams {
  const float2* rows;      // [nframes][NHB][KB][N]
  const float* framec;     // [nframes] c_f
  const double* framesum;  // [nframes]
  const double* inv_total; // [1] 1 / (valid pixels of the frame)
  const float2* w2d;       // [NH][N] 2D spectrum of w(x) w(y) m(x,y) (kx-major), or nullptr
  const float2* wc4;       // [4] window spectrum W(k), k = 0..3 (separable case)
  int slots[MAX_CHUNK];    // ring slot of each frame of the chunk
  const float2* tw;        // per-stage twiddle blocks of the N-point FFT
  float2* hist;            // [modes][T]
  double* means;           // [nframes] frame mean luma (out)
  float scale;
  int nframes, T, NH, NHB;
  int* err;                // error word (bounded waits that timed out), or nullptr
  // history band (0 = the whole half-plane): column blocks kb0 .. kb0 + nkb - 1
  // (KB columns each) and hist_w columns per history row, so mode (ky, kx)
  // of the band is stored at ((ky * hist_w) + kx - kb0 * KB) * T + slot
  int kb0, nkb, hist_w;
};

// One video of a batched temporal launch (units carry the video index in .w).
struct VideoDesc {
  const float2* hist;      // [modes][T]
  const uint32_t* order;   // [T]
  const float* mask;       // [T]
  const float* npairs;     // [L]
  const float2* mspec;     // [TPAD of the launch]
  const int4* items;       // bin-sorted (mode, kx, ky, bin)
  double* partials;        // [nunits][PFIELDS][L] + P at [nunits*PFIELDS*L + u]
  int T, L, unit0, nunits; // unit0: first global unit of this video
};

struct TemporalParams {
  const float2* hist;      // [modes][T]
  const uint32_t* order;   // [T]
  const float* mask;       // [T] 0/1
  const float* npairs;     // [L] exact valid-pair counts N(tau)
  const float2* mspec;     // [TPAD] FFT of the zero-padded mask
  const float2* tw;        // per-stage twiddle blocks, radix-8 plan of TPAD
  const float2* tw16;      // per-stage twiddle blocks, radix-16 plan of TPAD
  const int4* items;       // (mode, kx, ky, bin); nullptr: item i is mode i
  const int4* units;       // (first item, count, bin, 0)
  int nunits;
  int* unit_counter;
  double* partials;        // [nunits][PFIELDS][L] + P at [nunits*PFIELDS*L + u]
  float* outD;             // [modes][L] (full outputs) or nullptr
  float2* outC;            // [modes][L]
  float* outP;             // [modes]
  int* err;                // error word (bounded waits that timed out)
  int T, L;                // single video; batched: the largest T and L
  const VideoDesc* videos; // nullptr: one video (the fields above); else units[u].w indexes it
  int variant;             // 0: one-group radix-8 kernel; 1: two-group radix-16 (TPAD 1024..4096);
                           // 2: blocked kernel (TPAD 8192, L <= 128, fused radial path)
  int sparse;              // 1: single video whose mask has <= SPARSE_ZMAX zeros: A+B from
                           // prefix sums (temporal_sparse_kernel); 0: by transforms
};

constexpr int SPARSE_ZMAX = 64;  // masked time indices the sparse temporal kernel takes
constexpr int SPARSE_ZMAX_BIG = 256;  // ... and its TPAD 8192 variant (zero-list capacity)

struct ReduceParams {
  int accumulate;          // 1: add into D, P, drift (a band of a banded analysis after the first)
  const double* partials;
  const int* bin_units;    // [NB+1] unit range of each bin
  const uint32_t* nmodes;  // [NB]
  int nunits, NB, L;
  double* D;               // [NB][L]
  double* P;               // [NB]
  double* drift;           // [NB][L][8]
};

struct RadialFullParams {
  const float* D;          // [modes][L]
  const float2* C;         // [modes][L]
  const float* P;          // [modes]
  const int4* items;       // bin-sorted (mode, kx, ky, 0)
  const int4* units;       // the fused path's units (first item, count, bin, 0)
  int nunits, L;
  double* partials;        // [nunits][PFIELDS][L], then [nunits] P sums (reduce_kernel's input)
};

enum { LM_PLAIN = 0, LM_SEEDED = 1, LM_SEEDED_FALLBACK = 2, LM_BROWNIAN = 3, LM_SEEDED_COST = 4 };

struct LmParams {
  int nfit, nt_max, K;
  const int* nt;           // [nfit] lags used by each fit (<= nt_max, <= 128)
  const float* d;          // [nfit][nt_max] D(q_b, tau_j)
  const float* tau;        // [nfit][nt_max] lag times
  const float* qn;         // [nfit][K] effective-|k| nodes as q
  const float* w;          // [nfit] weight (1 / max d, motility_fit.js:391)
  const float* bounds;     // [nfit][6] vmin vmax Zmin Zmax Dmin Dmax
  const float* start;      // [nfit][4] alpha vbar Z D (LM_SEEDED)
  double* theta;           // [nfit][6] out: A B alpha ln vbar ln Z ln D
  double* cost;            // [nfit] out
  int* iters;              // [nfit] out (or nullptr)
  int* evals;              // [nfit] out (or nullptr)
  int* status;             // [nfit] out (or nullptr): bit 0 converged, bit 1 fell back to mode 0
  int* counter;            // work counter, 0 at launch (warps fetch fits)
  int mode, max_iter, nrefine;
  double tol;
  int geometry2d;          // swimmer kernel: 0 3D closed form, 1 2D table
  const float* vmag;       // [nfit] drift speed |V| of the J0 factor, or nullptr (none)
  Isf2dTable tab;          // the 2D table (geometry2d = 1)
};

// launchers (return cudaGetLastError())
cudaError_t launch_rows(int N, int dtype, const RowParams& p, cudaStream_t s);
cudaError_t launch_cols(int N, const ColParams& p, cudaStream_t s);
// the frames' reference levels c_f of nframes device frames (cref_kernel),
// for a whole ingest call at once
cudaError_t launch_cref(int N, int dtype, const void* frames, long long frame_stride, int nframes, float* framec,
                        cudaStream_t s);
// frames handled by one column-kernel CTA (one per FFT group); ingest chunks
// are multiples of it
int frames_per_col_cta(int N);
// Largest radix of the spatial transforms' plan for N (the twiddle table's layout).
int spatial_twiddle_radix(int N);
cudaError_t launch_temporal(int TPAD, int L, bool full, const TemporalParams& p, int grid,
                            cudaStream_t s);
int temporal_max_grid(int TPAD, int T, int L, bool full, int variant = 0, bool sparse = false);
// whether the two-group radix-16 variant exists for this TPAD (fused path)
bool temporal_has_variant16(int TPAD);
// TPAD sizes the sparse-mask temporal kernel serves
bool temporal_sparse_ok(int TPAD);
// most masked time indices the sparse path takes for this geometry (0: none)
int temporal_sparse_limit(int TPAD, int T, int L, bool full);
// which temporal kernel launch_temporal runs for these settings (DDM_TK_*)
int temporal_kernel_id(int TPAD, bool full, int variant, bool sparse);
// The blocked kernel (variant 2) serves this analysis: TPAD 8192, L <= 128, fused path.
bool temporal_blocked_ok(int TPAD, int T, int L, bool full);
cudaError_t launch_reduce(const ReduceParams& p, cudaStream_t s);
cudaError_t launch_radial_full(const RadialFullParams& p, cudaStream_t s);
cudaError_t launch_lm(const LmParams& p, cudaStream_t s);

}  // namespace ddm
