// The engine behind the C ABI (include/ddm_b200.h): device buffers, host
// tables, ingest chunking with copy/compute overlap, temporal + radial
// launches and readback. Mirrors the lifetime and call rules of the
// reference's WebGPU engine (motility-ddm/src/ddm-engine.ts).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/ddm_b200.h"
#include "kernels.cuh"
#include "tables.h"

using namespace ddm;

namespace {

constexpr int MAX_PENDING = 2;  // ddm-engine.ts:46
constexpr int NSTAGE = 2;       // host->device staging buffers (double buffer)

thread_local std::string g_create_error;

}  // namespace

struct ddm_engine {
  ddm_geometry g{};
  int NH = 0, NHB = 0, modes = 0, chunk = 0, chunk_cap = 0, unit_size = 0, variant = 0;
  bool sparse_enabled = true;  // the sparse-mask temporal kernel for masks with few zeros
  bool blocked_enabled = true;  // the blocked temporal kernel (TPAD 8192, L <= 128)
  int last_tk = -1;             // DDM_TK_* of the last temporal launch
  std::vector<float> meta_mask, meta_npairs, meta_mspec;  // temporal_meta of the last mask
  int device = 0;
  std::string err;
  int64_t launches = 0, throttled = 0;

  cudaStream_t own_stream = nullptr, stream = nullptr, copy_stream = nullptr;
  cudaEvent_t ready_ev[NSTAGE]{}, free_ev[NSTAGE]{}, meta_ev = nullptr;
  std::vector<cudaEvent_t> inflight;  // completion events of recent ingests
  // live analyses run on their own stream, concurrently with later ingests
  cudaStream_t ana_stream = nullptr;
  cudaEvent_t ana_ev = nullptr, ingest_ev = nullptr;
  bool ana_busy = false;          // a live analysis may still be running
  bool radial_from_live = false;  // the radial record is a live analysis' snapshot

  // geometry tables
  BinTable bins;
  float2 *d_hist = nullptr;            // [modes][T]
  float2 *d_rows = nullptr;            // [chunk][NHB][KB][N]
  float *d_rowc = nullptr;             // [rowc_cap] frame reference levels c_f
  size_t rowc_cap = 0;                 // c_f slots: a chunk's, or a whole device ingest's up to this
  double *d_framesum = nullptr;        // [chunk] pixel sums
  double *d_means = nullptr;           // [chunk]
  float *d_win = nullptr, *d_wys = nullptr;
  double *d_ninv = nullptr, *d_invtot = nullptr;
  float2 *d_tw_s = nullptr, *d_tw_t = nullptr, *d_tw_t16 = nullptr;
  float2 *d_wcorr4 = nullptr, *d_wcorr_full = nullptr;  // W(k), k < 4; FFT2(w m) [NH][N]
  uint8_t *d_smask = nullptr;
  void *d_stage[NSTAGE]{};             // device staging for host frames
  size_t stage_bytes = 0;
  double scale_last = 1.0;
  bool wys_ready = false;              // d_wys holds w(y) * scale_last
  int last_mean_index = -1;
  bool have_frames = false;

  // temporal
  uint32_t *d_order = nullptr;
  float *d_mask = nullptr, *d_npairs = nullptr;
  float2 *d_mspec = nullptr;
  char *h_meta = nullptr;              // pinned staging for order/mask/npairs/mspec
  size_t meta_bytes = 0;
  int4 *d_items = nullptr;             // bin-sorted (mode, kx, ky, bin)
  int4 *d_units = nullptr;             // fused-path units
  std::vector<int4> h_units;           // host copy (batched launches concatenate them)
  int nunits = 0;
  int *d_bin_units = nullptr;          // [NB+1]
  uint32_t *d_offsets = nullptr, *d_nmodes = nullptr;
  int4 *d_units_full = nullptr;
  int nunits_full = 0;
  int *d_counter = nullptr;
  int *d_err = nullptr;                // device error word (bounded waits)
  double *d_partials = nullptr;
  double *d_radD = nullptr, *d_radP = nullptr, *d_radDrift = nullptr;
  float *d_fullD = nullptr, *d_fullP = nullptr;
  float2 *d_fullC = nullptr;
  bool full_valid = false, radial_valid = false;

  // banded analysis (ddm_create_banded): the history holds band_w spectrum
  // columns of every row at a time; each band has its own work units
  struct Band {
    int kb0 = 0, nkb = 0, nunits = 0;
    int4 *d_items = nullptr, *d_units = nullptr;
    int *d_bin_units = nullptr;
  };
  int band_w = 0;            // columns per history row; 0 = the whole half-plane (NH)
  std::vector<Band> bands;
  int cur_kb0 = 0, cur_nkb = 0;  // the band the spatial pass writes (0, 0: all)
  bool in_banded = false;        // inside ddm_analyze_banded
};

static int fail(ddm_engine *h, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  return code;
}

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess)                                                           \
      return fail(h, DDM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
  } while (0)

#define CKL(call)                                                                    \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    h->launches++;                                                                   \
    if (e_ != cudaSuccess)                                                           \
      return fail(h, DDM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));  \
  } while (0)

template <typename T>
static int dalloc(ddm_engine *h, T **p, size_t count) {
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void **)p, sizeof(T) * count);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(h, DDM_ERR_NOMEM, "cudaMalloc of %zu bytes failed: %s", sizeof(T) * count,
                cudaGetErrorString(e));
  }
  return DDM_OK;
}

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static void release(ddm_engine *h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->own_stream) cudaStreamSynchronize(h->own_stream);
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  if (h->ana_stream) cudaStreamSynchronize(h->ana_stream);
  void *dev[] = {h->d_hist, h->d_rows, h->d_rowc, h->d_framesum, h->d_means, h->d_win, h->d_wys, h->d_ninv,
                 h->d_invtot, h->d_tw_s, h->d_tw_t, h->d_tw_t16, h->d_wcorr4, h->d_wcorr_full, h->d_smask,
                 h->d_order, h->d_mask, h->d_npairs,
                 h->d_mspec, h->d_items, h->d_units, h->d_bin_units, h->d_offsets, h->d_nmodes,
                 h->d_units_full, h->d_counter, h->d_err, h->d_partials, h->d_radD, h->d_radP,
                 h->d_radDrift, h->d_fullD, h->d_fullP, h->d_fullC};
  for (void *p : dev)
    if (p) cudaFree(p);
  for (void *p : h->d_stage)
    if (p) cudaFree(p);
  for (auto &b : h->bands)
    for (void *p : {(void *)b.d_items, (void *)b.d_units, (void *)b.d_bin_units})
      if (p) cudaFree(p);
  if (h->h_meta) cudaFreeHost(h->h_meta);
  for (int i = 0; i < NSTAGE; i++) {
    if (h->ready_ev[i]) cudaEventDestroy(h->ready_ev[i]);
    if (h->free_ev[i]) cudaEventDestroy(h->free_ev[i]);
  }
  for (cudaEvent_t e : h->inflight) cudaEventDestroy(e);
  if (h->meta_ev) cudaEventDestroy(h->meta_ev);
  if (h->ana_ev) cudaEventDestroy(h->ana_ev);
  if (h->ingest_ev) cudaEventDestroy(h->ingest_ev);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->ana_stream) cudaStreamDestroy(h->ana_stream);
  delete h;
}

// Work units of the fused temporal path: runs of up to U modes inside one
// bin, bins in order. U = 0: about three units per persistent CTA.
static int build_units(ddm_engine *h, int U = 0) {
  const int NB = h->g.NB;
  const int total = (int)h->bins.offsets[NB];
  if (U <= 0) {
    const int grid = std::max(1, temporal_max_grid(h->g.TPAD, h->g.T, h->g.L, false, h->variant));
    U = total / (3 * grid);
    U = std::max(16, std::min(256, U + (U & 1)));
  }
  h->unit_size = U;
  for (void *p : {(void *)h->d_items, (void *)h->d_units, (void *)h->d_bin_units, (void *)h->d_offsets,
                  (void *)h->d_nmodes, (void *)h->d_units_full, (void *)h->d_counter, (void *)h->d_err,
                  (void *)h->d_partials})
    if (p) cudaFree(p);
  h->d_items = nullptr;
  h->d_units = nullptr;
  h->d_bin_units = nullptr;
  h->d_offsets = h->d_nmodes = nullptr;
  h->d_units_full = nullptr;
  h->d_counter = h->d_err = nullptr;
  h->d_partials = nullptr;
  std::vector<int4> units;
  std::vector<int> bin_units(NB + 1, 0);
  for (int b = 0; b < NB; b++) {
    bin_units[b] = (int)units.size();
    const int i0 = (int)h->bins.offsets[b], i1 = (int)h->bins.offsets[b + 1];
    for (int i = i0; i < i1; i += U) units.push_back(make_int4(i, std::min(U, i1 - i), b, 0));
  }
  bin_units[NB] = (int)units.size();
  h->nunits = (int)units.size();
  h->h_units = units;
  std::vector<int4> items(std::max(total, 1));
  for (int i = 0; i < total; i++) {
    const int32_t *m = &h->bins.modes[4 * (size_t)i];
    items[i] = make_int4(m[0], m[1], m[2], 0);
  }
  for (int b = 0; b < NB; b++)
    for (uint32_t i = h->bins.offsets[b]; i < h->bins.offsets[b + 1]; i++) items[i].w = b;
  // full path: all modes in runs of 64
  std::vector<int4> uf;
  for (int m = 0; m < h->modes; m += 64) uf.push_back(make_int4(m, std::min(64, h->modes - m), -1, 0));
  h->nunits_full = (int)uf.size();
  int rc;
  if ((rc = dalloc(h, &h->d_items, items.size())) || (rc = dalloc(h, &h->d_units, units.size())) ||
      (rc = dalloc(h, &h->d_bin_units, NB + 1)) || (rc = dalloc(h, &h->d_offsets, NB + 1)) ||
      (rc = dalloc(h, &h->d_nmodes, NB)) || (rc = dalloc(h, &h->d_units_full, uf.size())) ||
      (rc = dalloc(h, &h->d_counter, 1)) || (rc = dalloc(h, &h->d_err, 1)) ||
      (rc = dalloc(h, &h->d_partials, (size_t)h->nunits * PFIELDS * h->g.L + h->nunits)))
    return rc;
  CK(cudaMemset(h->d_err, 0, sizeof(int)));
  CK(cudaMemcpy(h->d_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice));
  if (!units.empty())
    CK(cudaMemcpy(h->d_units, units.data(), sizeof(int4) * units.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_bin_units, bin_units.data(), sizeof(int) * (NB + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_offsets, h->bins.offsets.data(), sizeof(uint32_t) * (NB + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_nmodes, h->bins.nModes.data(), sizeof(uint32_t) * NB, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_units_full, uf.data(), sizeof(int4) * uf.size(), cudaMemcpyHostToDevice));
  return DDM_OK;
}

// Work units of each band of a banded engine: the binned modes whose column
// kx lies in the band, renumbered to the band's history rows (mode (ky, kx)
// -> ky * band_w + kx - kb0 * KB), in runs of up to unit_size modes inside
// one bin, bins in order -- the fused path's units restricted to the band.
static int build_band_units(ddm_engine *h) {
  const int NB = h->g.NB, NH = h->NH, W = h->band_w, U = h->unit_size;
  for (auto &b : h->bands) {
    for (void *p : {(void *)b.d_items, (void *)b.d_units, (void *)b.d_bin_units})
      if (p) cudaFree(p);
    b.d_items = b.d_units = nullptr;
    b.d_bin_units = nullptr;
    const int kx0 = b.kb0 * KB, kx1 = std::min(NH, (b.kb0 + b.nkb) * KB);
    std::vector<int4> items, units;
    std::vector<int> bin_units(NB + 1, 0);
    for (int bin = 0; bin < NB; bin++) {
      const int i0 = (int)items.size();
      for (uint32_t i = h->bins.offsets[bin]; i < h->bins.offsets[bin + 1]; i++) {
        const int32_t *m = &h->bins.modes[4 * (size_t)i];
        const int kx = m[0] % NH, row = m[0] / NH;
        if (kx < kx0 || kx >= kx1) continue;
        items.push_back(make_int4(row * W + kx - kx0, m[1], m[2], bin));
      }
      const int i1 = (int)items.size();
      bin_units[bin] = (int)units.size();
      for (int i = i0; i < i1; i += U) units.push_back(make_int4(i, std::min(U, i1 - i), bin, 0));
    }
    bin_units[NB] = (int)units.size();
    b.nunits = (int)units.size();
    int rc;
    if ((rc = dalloc(h, &b.d_items, std::max<size_t>(items.size(), 1))) ||
        (rc = dalloc(h, &b.d_units, std::max<size_t>(units.size(), 1))) || (rc = dalloc(h, &b.d_bin_units, NB + 1)))
      return rc;
    if (!items.empty()) CK(cudaMemcpy(b.d_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice));
    if (!units.empty()) CK(cudaMemcpy(b.d_units, units.data(), sizeof(int4) * units.size(), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(b.d_bin_units, bin_units.data(), sizeof(int) * (NB + 1), cudaMemcpyHostToDevice));
  }
  return DDM_OK;
}

// Uploads the spatial weighting: window, w(y)*scale is per call (scale), row
// normalisers and the window-spectrum correction for the current mask.
static int upload_mask_tables(ddm_engine *h, const uint8_t *mask) {
  const int N = h->g.N, NH = h->NH;
  const std::vector<double> w = blackman_harris(N);
  std::vector<double> ninv(N);
  double total = 0;
  for (int y = 0; y < N; y++) {
    double c = 0;
    for (int x = 0; x < N; x++) c += mask ? (mask[(size_t)y * N + x] ? 1 : 0) : 1;
    ninv[y] = c > 0 ? 1.0 / c : 0.0;
    total += c;
  }
  const double invtot = total > 0 ? 1.0 / total : 0.0;
  CK(cudaMemcpy(h->d_ninv, ninv.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(h->d_invtot, &invtot, sizeof(double), cudaMemcpyHostToDevice));
  if (!mask) {
    if (h->d_smask) {
      cudaFree(h->d_smask);
      h->d_smask = nullptr;
    }
    if (h->d_wcorr_full) {
      cudaFree(h->d_wcorr_full);
      h->d_wcorr_full = nullptr;
    }
    return DDM_OK;
  }
  int rc;
  if (!h->d_smask && (rc = dalloc(h, &h->d_smask, (size_t)N * N))) return rc;
  if (!h->d_wcorr_full && (rc = dalloc(h, &h->d_wcorr_full, (size_t)N * NH))) return rc;
  std::vector<uint8_t> m01((size_t)N * N);
  for (size_t i = 0; i < m01.size(); i++) m01[i] = mask[i] ? 1 : 0;
  CK(cudaMemcpy(h->d_smask, m01.data(), m01.size(), cudaMemcpyHostToDevice));
  // 2D spectrum of the masked window, W2(ky, kx) = FFT2(w(x) w(y) m(x, y)),
  // FP64, stored kx-major as FP32 (the mean correction's table)
  std::vector<std::vector<cd>> rs(N, std::vector<cd>(N));
  for (int y = 0; y < N; y++) {
    for (int x = 0; x < N; x++) rs[y][x] = cd(w[x] * w[y] * m01[(size_t)y * N + x], 0);
    host_fft(rs[y], false);
  }
  std::vector<float> wc(2 * (size_t)N * NH);
  std::vector<cd> col(N);
  for (int kx = 0; kx < NH; kx++) {
    for (int y = 0; y < N; y++) col[y] = rs[y][kx];
    host_fft(col, false);
    for (int ky = 0; ky < N; ky++) {
      wc[2 * ((size_t)kx * N + ky)] = (float)col[ky].real();
      wc[2 * ((size_t)kx * N + ky) + 1] = (float)col[ky].imag();
    }
  }
  CK(cudaMemcpy(h->d_wcorr_full, wc.data(), sizeof(float) * wc.size(), cudaMemcpyHostToDevice));
  return DDM_OK;
}

// Message slot shared by the calls that have no engine (ddm_create,
// ddm_spectra_noalloc in noalloc.cu).
std::string &ddm_detached_error() { return g_create_error; }

extern "C" const char *ddm_create_error(void) { return g_create_error.c_str(); }

static int create_impl(const ddm_geometry *geometry, uint64_t band_budget, ddm_engine **out) {
  g_create_error.clear();
  if (!geometry || !out) {
    g_create_error = "ddm_create: null argument";
    return DDM_ERR_ARG;
  }
  *out = nullptr;
  ddm_geometry g = *geometry;
  if (g.TPAD == 0) {  // smallest supported power of two >= 2T
    g.TPAD = 128;
    while (g.TPAD < 2 * g.T) g.TPAD <<= 1;
  }
  char msg[256] = {0};
  if (!((is_pow2(g.N) && g.N >= 64 && g.N <= 2048) || g.N == 384 || g.N == 768))
    snprintf(msg, sizeof msg, "N = %d: must be a power of two in [64, 2048], or 384 or 768", g.N);
  else if (g.T < 2 || !is_pow2(g.TPAD) || g.TPAD < 128 || g.TPAD > 8192 || 2 * g.T > g.TPAD)
    snprintf(msg, sizeof msg, "T = %d, TPAD = %d: need TPAD a power of two in [128, 8192] and TPAD >= 2T",
             g.T, g.TPAD);
  else if (g.T & 1)
    snprintf(msg, sizeof msg, "T = %d: must be even (time series are staged in 16-byte units)", g.T);
  else if (g.L < 2 || g.L > g.T)
    snprintf(msg, sizeof msg, "L = %d: need 2 <= L <= T", g.L);
  else if (g.NB < 1 || !(g.kmax > g.kmin) || g.kmin < 0)
    snprintf(msg, sizeof msg, "bins: need NB >= 1 and 0 <= kmin < kmax");
  else if (g.knodes < 1 || g.knodes > 16)
    snprintf(msg, sizeof msg, "knodes = %d: need 1..16", g.knodes);
  if (msg[0]) {
    g_create_error = msg;
    return DDM_ERR_ARG;
  }
  int dev = 0, ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    g_create_error = "no CUDA device";
    return DDM_ERR_NODEV;
  }
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  if (prop.major != 10) {
    snprintf(msg, sizeof msg, "device %d is sm_%d%d; this library is built for sm_100a", dev,
             prop.major, prop.minor);
    g_create_error = msg;
    return DDM_ERR_NODEV;
  }

  ddm_engine *h = new ddm_engine();
  h->g = g;
  h->device = dev;
  h->NH = g.N / 2 + 1;
  h->NHB = (h->NH + KB - 1) / KB;
  h->modes = g.N * h->NH;
  {
    const size_t per = (size_t)h->NHB * g.N * KB * sizeof(float2);
    // default chunk: ~128 MB of row spectra (at 512^2 x 1024 the autotuner's
    // choice is larger still: fewer launches and persistent-grid tails
    // outweigh the scratch no longer fitting L2)
    const size_t target = 128u << 20;
    const int fg = frames_per_col_cta(g.N);
    size_t c = std::max<size_t>(1, target / per);
    c = std::min<size_t>(MAX_CHUNK, std::max<size_t>(c, fg));
    h->chunk = (int)(c / fg * fg);  // whole column-kernel frame groups
    // buffers hold up to chunk_cap frames, so the autotuner may pick larger
    // chunks (at N >= 1024 one frame's scratch is 4 MB or more and a chunk
    // of four, the column kernel's tile, is already 17 MB)
    const size_t cap_bytes = g.N >= 1024 ? (size_t(1) << 30) : (256u << 20);
    h->chunk_cap = std::max(h->chunk, std::min<int>(MAX_CHUNK, (int)std::max<size_t>(fg, cap_bytes / per)) / fg * fg);
  }
  h->bins = make_bins(g.N, g.NB, g.kmin, g.kmax, g.knodes);
  if (band_budget) {
    // columns of history that fit the budget, in whole column blocks
    const uint64_t per_col = (uint64_t)g.N * g.T * sizeof(float2);
    const uint64_t cols = band_budget / per_col;
    if (cols < (uint64_t)KB) {
      snprintf(msg, sizeof msg, "history budget %llu B holds fewer than %d spectrum columns (%llu B each)",
               (unsigned long long)band_budget, KB, (unsigned long long)per_col);
      g_create_error = msg;
      delete h;
      return DDM_ERR_ARG;
    }
    const int bkb = (int)std::min<uint64_t>((uint64_t)h->NHB, cols / KB);
    h->band_w = bkb * KB;
    for (int kb0 = 0; kb0 < h->NHB; kb0 += bkb) {
      ddm_engine::Band b;
      b.kb0 = kb0;
      b.nkb = std::min(bkb, h->NHB - kb0);
      h->bands.push_back(b);
    }
  }
  const size_t hist_modes = (size_t)g.N * (h->band_w ? h->band_w : h->NH);
  int rc = DDM_OK;
  auto bail = [&](int code) {
    g_create_error = h->err;
    release(h);
    return code;
  };
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&h->ana_stream, cudaStreamNonBlocking) != cudaSuccess) {
    h->err = "stream creation failed";
    return bail(DDM_ERR_CUDA);
  }
  h->stream = h->own_stream;
  for (int i = 0; i < NSTAGE; i++) {
    cudaEventCreateWithFlags(&h->ready_ev[i], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&h->free_ev[i], cudaEventDisableTiming);
  }
  cudaEventCreateWithFlags(&h->meta_ev, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&h->ana_ev, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&h->ingest_ev, cudaEventDisableTiming);
  const int N = g.N;
  h->stage_bytes = (size_t)h->chunk_cap * N * N * sizeof(float);
  h->rowc_cap = std::max<size_t>((size_t)h->chunk_cap * N, (size_t)g.T);
  if ((rc = dalloc(h, &h->d_hist, hist_modes * g.T)) ||
      (rc = dalloc(h, &h->d_rows, (size_t)h->chunk_cap * h->NHB * N * KB)) ||
      (rc = dalloc(h, &h->d_rowc, h->rowc_cap)) ||
      (rc = dalloc(h, &h->d_framesum, (size_t)h->chunk_cap)) ||
      (rc = dalloc(h, &h->d_means, (size_t)h->chunk_cap)) || (rc = dalloc(h, &h->d_win, N)) ||
      (rc = dalloc(h, &h->d_wys, N)) || (rc = dalloc(h, &h->d_ninv, N)) ||
      (rc = dalloc(h, &h->d_invtot, 1)) || (rc = dalloc(h, &h->d_tw_s, N)) ||
      (rc = dalloc(h, &h->d_tw_t, g.TPAD)) || (rc = dalloc(h, &h->d_tw_t16, g.TPAD)) ||
      (rc = dalloc(h, &h->d_wcorr4, 4)) ||
      (rc = dalloc(h, &h->d_order, g.T)) || (rc = dalloc(h, &h->d_mask, g.T)) ||
      (rc = dalloc(h, &h->d_npairs, g.L)) || (rc = dalloc(h, &h->d_mspec, g.TPAD)) ||
      (rc = dalloc(h, &h->d_radD, (size_t)g.NB * g.L)) || (rc = dalloc(h, &h->d_radP, g.NB)) ||
      (rc = dalloc(h, &h->d_radDrift, (size_t)g.NB * g.L * DRIFT)))
    return bail(rc);
  h->meta_bytes = sizeof(uint32_t) * g.T + sizeof(float) * g.T + sizeof(float) * g.L +
                  sizeof(float2) * g.TPAD;
  if (cudaHostAlloc((void **)&h->h_meta, h->meta_bytes, cudaHostAllocDefault) != cudaSuccess) {
    h->err = "pinned host allocation failed";
    return bail(DDM_ERR_NOMEM);
  }
  // tables
  const std::vector<double> w = blackman_harris(N);
  std::vector<float> wf(N);
  for (int i = 0; i < N; i++) wf[i] = (float)w[i];
  std::vector<float> tws = twiddle_table(N, spatial_twiddle_radix(N)), twt = twiddle_table(g.TPAD), twt16 = twiddle_table(g.TPAD, 16);
  // DFT of the window at kx = 0..3 (zero beyond for the 4-term window)
  float wc4[8];
  for (int kx = 0; kx < 4; kx++) {
    double re = 0, im = 0;
    for (int x = 0; x < N; x++) {
      const double a = -2.0 * M_PI * kx * x / N;
      re += w[x] * std::cos(a);
      im += w[x] * std::sin(a);
    }
    wc4[2 * kx] = (float)re;
    wc4[2 * kx + 1] = (float)im;
  }
  if (cudaMemcpy(h->d_win, wf.data(), sizeof(float) * N, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->d_tw_s, tws.data(), sizeof(float) * tws.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->d_tw_t, twt.data(), sizeof(float) * twt.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->d_tw_t16, twt16.data(), sizeof(float) * twt16.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(h->d_wcorr4, wc4, sizeof wc4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(h->d_hist, 0, sizeof(float2) * hist_modes * g.T) != cudaSuccess) {
    h->err = "table upload failed";
    return bail(DDM_ERR_CUDA);
  }
  if ((rc = upload_mask_tables(h, nullptr)) || (rc = build_units(h))) return bail(rc);
  if (h->band_w && (rc = build_band_units(h))) return bail(rc);
  *out = h;
  return DDM_OK;
}

extern "C" int ddm_create(const ddm_geometry *geometry, ddm_engine **out) {
  return create_impl(geometry, 0, out);
}

extern "C" int ddm_create_banded(const ddm_geometry *geometry, uint64_t history_budget_bytes, ddm_engine **out) {
  if (history_budget_bytes == 0) {
    g_create_error = "ddm_create_banded: the history budget must be > 0";
    return DDM_ERR_ARG;
  }
  return create_impl(geometry, history_budget_bytes, out);
}

extern "C" int ddm_get_bands(const ddm_engine *h, int32_t *nbands, int32_t *band_cols) {
  if (!h) return DDM_ERR_ARG;
  if (nbands) *nbands = h->band_w ? (int32_t)h->bands.size() : 1;
  if (band_cols) *band_cols = h->band_w ? h->band_w : h->NH;
  return DDM_OK;
}

extern "C" void ddm_destroy(ddm_engine *h) { release(h); }

extern "C" const char *ddm_last_error(const ddm_engine *h) { return h ? h->err.c_str() : ""; }

extern "C" int ddm_get_geometry(const ddm_engine *h, ddm_geometry *out) {
  if (!h || !out) return DDM_ERR_ARG;
  *out = h->g;
  return DDM_OK;
}

extern "C" int ddm_bins_count(const ddm_engine *h) {
  return h ? (int)h->bins.offsets[h->g.NB] : -1;
}

extern "C" int ddm_get_bins(const ddm_engine *h, uint32_t *binOffsets, int32_t *binModes,
                            double *kCenter, uint32_t *nModes, double *kNodes) {
  if (!h) return DDM_ERR_ARG;
  const BinTable &b = h->bins;
  if (binOffsets) memcpy(binOffsets, b.offsets.data(), sizeof(uint32_t) * b.offsets.size());
  if (binModes) memcpy(binModes, b.modes.data(), sizeof(int32_t) * b.modes.size());
  if (kCenter) memcpy(kCenter, b.kCenter.data(), sizeof(double) * b.kCenter.size());
  if (nModes) memcpy(nModes, b.nModes.data(), sizeof(uint32_t) * b.nModes.size());
  if (kNodes) memcpy(kNodes, b.kNodes.data(), sizeof(double) * b.kNodes.size());
  return DDM_OK;
}

extern "C" int ddm_set_stream(ddm_engine *h, void *stream) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  cudaStreamSynchronize(h->stream);
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return DDM_OK;
}

extern "C" int64_t ddm_kernel_launches(const ddm_engine *h) { return h ? h->launches : 0; }

// Rows + columns for one chunk of frames already in device memory.
// framec: the chunk's c_f already computed for the whole call (device frames),
// or nullptr: cref_kernel runs with the rows kernel for this chunk
static int launch_chunk(ddm_engine *h, const void *dframes, int dtype, int n, const int32_t *slots,
                        float scale, float *framec = nullptr) {
  const int N = h->g.N;
  // w(y) * scale for this call's scale
  RowParams rp{};
  rp.frames = dframes;
  rp.frame_stride = (long long)N * N;
  rp.nframes = n;
  rp.win = h->d_win;
  rp.wys = h->d_wys;
  rp.smask = h->d_smask;
  rp.tw = h->d_tw_s;
  rp.rows = h->d_rows;
  rp.framec = framec ? framec : h->d_rowc;
  rp.framec_ready = framec != nullptr;
  rp.framesum = h->d_framesum;
  rp.err = h->d_err;
  CK(cudaMemsetAsync(h->d_framesum, 0, sizeof(double) * n, h->stream));
  CKL(launch_rows(N, dtype, rp, h->stream));
  if (n > 0 && !framec) h->launches++;  // launch_rows also ran cref_kernel (the frames' reference levels)
  ColParams cp{};
  cp.rows = h->d_rows;
  cp.framec = rp.framec;
  cp.framesum = h->d_framesum;
  cp.inv_total = h->d_invtot;
  cp.w2d = h->d_smask ? h->d_wcorr_full : nullptr;
  cp.wc4 = h->d_wcorr4;
  for (int i = 0; i < n; i++) cp.slots[i] = slots[i] % h->g.T;
  cp.tw = h->d_tw_s;
  cp.hist = h->d_hist;
  cp.means = h->d_means;
  cp.scale = scale;
  cp.nframes = n;
  cp.T = h->g.T;
  cp.NH = h->NH;
  cp.NHB = h->NHB;
  cp.err = h->d_err;
  cp.kb0 = h->cur_kb0;
  cp.nkb = h->cur_nkb;
  cp.hist_w = h->band_w;
  CKL(launch_cols(N, cp, h->stream));
  h->last_mean_index = n - 1;
  h->have_frames = true;
  return DDM_OK;
}

static int set_scale(ddm_engine *h, float scale) {
  if (!(scale > 0) || !std::isfinite(scale)) return fail(h, DDM_ERR_ARG, "scale must be finite and > 0");
  if ((double)scale == h->scale_last && h->wys_ready) return DDM_OK;
  const int N = h->g.N;
  const std::vector<double> w = blackman_harris(N);
  std::vector<float> wys(N);
  for (int y = 0; y < N; y++) wys[y] = (float)(w[y] * (double)scale);
  // ordered on the engine stream behind earlier chunks that read d_wys
  CK(cudaStreamSynchronize(h->stream));
  CK(cudaMemcpy(h->d_wys, wys.data(), sizeof(float) * N, cudaMemcpyHostToDevice));
  h->scale_last = scale;
  h->wys_ready = true;
  return DDM_OK;
}

static int check_frames_args(ddm_engine *h, const void *frames, int dtype, int n, const int32_t *slots) {
  if (!frames && n > 0) return fail(h, DDM_ERR_ARG, "frames is NULL");
  if (dtype < 0 || dtype > 2) return fail(h, DDM_ERR_ARG, "dtype %d: expected 0 (u8), 1 (u16), 2 (f32)", dtype);
  if (n < 0) return fail(h, DDM_ERR_ARG, "n = %d < 0", n);
  if (n > 0 && !slots) return fail(h, DDM_ERR_ARG, "slots is NULL");
  for (int i = 0; i < n; i++)
    if (slots[i] < 0) return fail(h, DDM_ERR_ARG, "slot %d < 0", slots[i]);
  return DDM_OK;
}

static void note_inflight(ddm_engine *h) {
  cudaEvent_t e;
  if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) {
    cudaEventRecord(e, h->stream);
    h->inflight.push_back(e);
  }
}

static int dtype_size(int dtype) { return dtype == 0 ? 1 : dtype == 1 ? 2 : 4; }

static int ingest_impl(ddm_engine *h, const void *frames, int dtype, int n, const int32_t *slots,
                       float scale, bool device, bool wait_copies = true) {
  cudaSetDevice(h->device);
  if (h->band_w && !h->in_banded)
    return fail(h, DDM_ERR_STATE, "a banded engine analyses a video with ddm_analyze_banded");
  int rc = check_frames_args(h, frames, dtype, n, slots);
  if (rc) return rc;
  if (device && ((uintptr_t)frames & 15))
    return fail(h, DDM_ERR_ARG, "device frames must be 16-byte aligned (they are staged by bulk copies)");
  if ((rc = set_scale(h, scale))) return rc;
  const int N = h->g.N;
  const size_t fbytes = (size_t)N * N * dtype_size(dtype);
  // the host-frame staging buffers exist from the first host ingest on
  // (engines fed from device memory never hold them)
  if (!device && n > 0)
    for (void *&p : h->d_stage)
      if (!p && (rc = dalloc(h, (char **)&p, h->stage_bytes))) return rc;
  // device frames: every frame's reference level in one launch ahead of the
  // chunks (host frames arrive chunk by chunk: per chunk with the rows kernel)
  const bool cref_all = device && n > 0 && (size_t)n <= h->rowc_cap;
  if (cref_all) CKL(launch_cref(N, dtype, frames, (long long)N * N, n, h->d_rowc, h->stream));
  for (int c0 = 0, ci = 0; c0 < n; c0 += h->chunk, ci++) {
    const int m = std::min(h->chunk, n - c0);
    const void *src;
    if (device) {
      src = (const char *)frames + (size_t)c0 * fbytes;
    } else {
      // staging buffer s is free once the chunk that last used it has run
      const int s = ci % NSTAGE;
      CK(cudaStreamWaitEvent(h->copy_stream, h->free_ev[s], 0));
      CK(cudaMemcpyAsync(h->d_stage[s], (const char *)frames + (size_t)c0 * fbytes, m * fbytes,
                         cudaMemcpyHostToDevice, h->copy_stream));
      CK(cudaEventRecord(h->ready_ev[s], h->copy_stream));
      CK(cudaStreamWaitEvent(h->stream, h->ready_ev[s], 0));
      src = h->d_stage[s];
    }
    if ((rc = launch_chunk(h, src, dtype, m, slots + c0, scale, cref_all ? h->d_rowc + c0 : nullptr))) return rc;
    if (!device) CK(cudaEventRecord(h->free_ev[ci % NSTAGE], h->stream));
  }
  // the caller's host buffer is free once the copies have run (the async
  // entry point leaves that wait to ddm_ingest_wait)
  if (wait_copies) CK(cudaStreamSynchronize(h->copy_stream));
  note_inflight(h);
  if (!h->radial_from_live) h->radial_valid = false;  // a live snapshot stays readable
  return DDM_OK;
}

extern "C" int ddm_ingest_frames(ddm_engine *h, const void *frames, int32_t dtype, int32_t n,
                                 const int32_t *slots, float scale) {
  if (!h) return DDM_ERR_ARG;
  return ingest_impl(h, frames, dtype, n, slots, scale, false);
}

extern "C" int ddm_ingest_frames_device(ddm_engine *h, const void *frames, int32_t dtype, int32_t n,
                                        const int32_t *slots, float scale) {
  if (!h) return DDM_ERR_ARG;
  return ingest_impl(h, frames, dtype, n, slots, scale, true);
}

extern "C" int ddm_ingest_frames_async(ddm_engine *h, const void *frames, int32_t dtype, int32_t n,
                                       const int32_t *slots, float scale) {
  if (!h) return DDM_ERR_ARG;
  return ingest_impl(h, frames, dtype, n, slots, scale, false, false);
}

extern "C" int ddm_ingest_wait(ddm_engine *h) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  CK(cudaStreamSynchronize(h->copy_stream));
  return DDM_OK;
}

static int prune_inflight(ddm_engine *h) {
  std::vector<cudaEvent_t> keep;
  for (cudaEvent_t e : h->inflight) {
    if (cudaEventQuery(e) == cudaSuccess)
      cudaEventDestroy(e);
    else
      keep.push_back(e);
  }
  cudaGetLastError();  // cudaErrorNotReady is not an error here
  h->inflight.swap(keep);
  return (int)h->inflight.size();
}

extern "C" int ddm_pending(ddm_engine *h) { return h ? prune_inflight(h) : 0; }

extern "C" int ddm_wait_for_capacity(ddm_engine *h) {
  if (!h) return DDM_ERR_ARG;
  while (prune_inflight(h) > MAX_PENDING) CK(cudaEventSynchronize(h->inflight.front()));
  return DDM_OK;
}

extern "C" int64_t ddm_throttled(const ddm_engine *h) { return h ? h->throttled : 0; }

extern "C" int ddm_ingest_luma(ddm_engine *h, const float *luma, int32_t slot, int32_t *accepted) {
  if (!h) return DDM_ERR_ARG;
  if (accepted) *accepted = 0;
  if (!luma) return fail(h, DDM_ERR_ARG, "ingestLuma expects %d values", h->g.N * h->g.N);
  if (prune_inflight(h) > MAX_PENDING) {
    h->throttled++;
    return DDM_OK;
  }
  const int32_t s = slot;
  int rc = ingest_impl(h, luma, DDM_F32, 1, &s, 1.0f, false);
  if (rc == DDM_OK && accepted) *accepted = 1;
  return rc;
}

extern "C" int ddm_set_spatial_mask(ddm_engine *h, const uint8_t *mask) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  CK(cudaStreamSynchronize(h->stream));
  return upload_mask_tables(h, mask);
}

static int temporal_impl(ddm_engine *h, const uint32_t *order, const float *mask, int full, cudaStream_t st,
                         const ddm_engine::Band *band = nullptr) {
  cudaSetDevice(h->device);
  if (h->band_w && !band)
    return fail(h, DDM_ERR_STATE, "a banded engine analyses a video with ddm_analyze_banded");
  const int T = h->g.T, L = h->g.L, TPAD = h->g.TPAD;
  if (!order || !mask) return fail(h, DDM_ERR_ARG, "computeTemporal: order/mask must have length %d", T);
  for (int j = 0; j < T; j++)
    if (order[j] >= (uint32_t)T) return fail(h, DDM_ERR_ARG, "order[%d] = %u is not a slot < %d", j, order[j], T);
  // N(tau) and the mask spectrum depend on the mask alone: reused while the
  // mask is the previous analysis' (a stream of videos with the same drops)
  if (h->meta_mask.size() != (size_t)T || memcmp(h->meta_mask.data(), mask, sizeof(float) * T) != 0) {
    temporal_meta(mask, T, TPAD, L, h->meta_npairs, h->meta_mspec);
    h->meta_mask.assign(mask, mask + T);
  }
  const std::vector<float> &npairs = h->meta_npairs, &mspec = h->meta_mspec;
  // the pinned staging may still be read by the previous analysis' copies
  CK(cudaEventSynchronize(h->meta_ev));
  char *p = h->h_meta;
  uint32_t *ho = (uint32_t *)p;
  float *hm = (float *)(ho + T);
  float *hn = hm + T;
  float *hs = hn + L;
  memcpy(ho, order, sizeof(uint32_t) * T);
  for (int j = 0; j < T; j++) hm[j] = mask[j] != 0.f ? 1.f : 0.f;
  memcpy(hn, npairs.data(), sizeof(float) * L);
  memcpy(hs, mspec.data(), sizeof(float) * 2 * TPAD);
  CK(cudaMemcpyAsync(h->d_order, ho, sizeof(uint32_t) * T, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->d_mask, hm, sizeof(float) * T, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->d_npairs, hn, sizeof(float) * L, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(h->d_mspec, hs, sizeof(float2) * TPAD, cudaMemcpyHostToDevice, st));
  CK(cudaEventRecord(h->meta_ev, st));

  TemporalParams tp{};
  tp.hist = h->d_hist;
  tp.order = h->d_order;
  tp.mask = h->d_mask;
  tp.npairs = h->d_npairs;
  tp.mspec = h->d_mspec;
  tp.tw = h->d_tw_t;
  tp.tw16 = h->d_tw_t16;
  tp.variant = h->variant;
  {  // a 0/1 mask with few zeros: A + B from prefix sums (temporal_sparse_kernel)
    int nz = 0;
    bool binary = true;
    for (int j = 0; j < T; j++) {
      nz += mask[j] == 0.f;
      binary = binary && (mask[j] == 0.f || mask[j] == 1.f);
    }
    tp.sparse = h->sparse_enabled && binary && nz <= temporal_sparse_limit(TPAD, T, L, full) ? 1 : 0;
  }
  if (h->blocked_enabled && temporal_blocked_ok(TPAD, T, L, full)) {  // short lags on a long series
    tp.variant = 2;
    tp.sparse = 0;
  }
  h->last_tk = temporal_kernel_id(TPAD, full, tp.variant, tp.sparse != 0);
  tp.unit_counter = h->d_counter;
  tp.err = h->d_err;
  tp.T = T;
  tp.L = L;
  int rc;
  if (full) {
    if (!h->d_fullD) {
      if ((rc = dalloc(h, &h->d_fullD, (size_t)h->modes * L)) ||
          (rc = dalloc(h, &h->d_fullC, (size_t)h->modes * L)) || (rc = dalloc(h, &h->d_fullP, h->modes)))
        return rc;
    }
    tp.items = nullptr;
    tp.units = h->d_units_full;
    tp.nunits = h->nunits_full;
    tp.outD = h->d_fullD;
    tp.outC = h->d_fullC;
    tp.outP = h->d_fullP;
    const int grid = std::min(temporal_max_grid(TPAD, T, L, true, 0, tp.sparse != 0), h->nunits_full);
    CK(cudaMemsetAsync(h->d_counter, 0, sizeof(int), st));
    CKL(launch_temporal(TPAD, L, true, tp, std::max(grid, 1), st));
    // the radial record from the full outputs: unit partial records, then
    // the fused path's reduction over each bin's units in order
    RadialFullParams fp{};
    fp.D = h->d_fullD;
    fp.C = h->d_fullC;
    fp.P = h->d_fullP;
    fp.items = h->d_items;
    fp.units = h->d_units;
    fp.nunits = h->nunits;
    fp.L = L;
    fp.partials = h->d_partials;
    CKL(launch_radial_full(fp, st));
    ReduceParams rp{};
    rp.partials = h->d_partials;
    rp.bin_units = h->d_bin_units;
    rp.nmodes = h->d_nmodes;
    rp.nunits = h->nunits;
    rp.NB = h->g.NB;
    rp.L = L;
    rp.D = h->d_radD;
    rp.P = h->d_radP;
    rp.drift = h->d_radDrift;
    CKL(launch_reduce(rp, st));
    h->full_valid = true;
  } else {
    // the engine's work units, or those of one band of a banded analysis
    const int nunits = band ? band->nunits : h->nunits;
    tp.items = band ? band->d_items : h->d_items;
    tp.units = band ? band->d_units : h->d_units;
    tp.nunits = nunits;
    tp.partials = h->d_partials;
    const int grid = std::min(temporal_max_grid(TPAD, T, L, false, tp.variant, tp.sparse != 0), nunits);
    CK(cudaMemsetAsync(h->d_counter, 0, sizeof(int), st));
    if (nunits > 0) CKL(launch_temporal(TPAD, L, false, tp, std::max(grid, 1), st));
    ReduceParams rp{};
    rp.accumulate = band && band != &h->bands[0];
    rp.partials = h->d_partials;
    rp.bin_units = band ? band->d_bin_units : h->d_bin_units;
    rp.nmodes = h->d_nmodes;
    rp.nunits = nunits;
    rp.NB = h->g.NB;
    rp.L = L;
    rp.D = h->d_radD;
    rp.P = h->d_radP;
    rp.drift = h->d_radDrift;
    CKL(launch_reduce(rp, st));
    h->full_valid = false;
  }
  h->radial_valid = true;
  return DDM_OK;
}

// After a synchronisation: surfaces a device-side error word (a bounded wait
// in a kernel that gave up) as an error status, and clears it.
static int check_device_error(ddm_engine *h) {
  int e = 0;
  CK(cudaMemcpy(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    CK(cudaMemset(h->d_err, 0, sizeof(int)));
    h->radial_valid = h->full_valid = false;
    return fail(h, DDM_ERR_CUDA, "%s (code %d)",
                e == 4 ? "the sparse-mask temporal kernel met more masked time indices than it holds"
                       : "a staged copy did not complete in time (1 temporal, 2 row, 3 column kernel)",
                e);
  }
  return DDM_OK;
}

// Waits for a live analysis still in flight (it shares the temporal buffers
// and the record the reads return) and surfaces its device error word.
static int join_analysis(ddm_engine *h) {
  if (!h->ana_busy) return DDM_OK;
  CK(cudaEventSynchronize(h->ana_ev));
  h->ana_busy = false;
  return check_device_error(h);
}

extern "C" int ddm_compute_temporal_async(ddm_engine *h, const uint32_t *order, const float *mask,
                                          int32_t full) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  int rc = join_analysis(h);
  if (rc) return rc;
  h->radial_from_live = false;
  return temporal_impl(h, order, mask, full, h->stream);
}

extern "C" int ddm_compute_temporal(ddm_engine *h, const uint32_t *order, const float *mask,
                                    int32_t full) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  int rc = join_analysis(h);
  if (rc) return rc;
  h->radial_from_live = false;
  if ((rc = temporal_impl(h, order, mask, full, h->stream))) return rc;
  CK(cudaStreamSynchronize(h->stream));
  return check_device_error(h);
}

// Live analysis (the dashboard's analysis tick, main.ts:366-398, with
// computeTemporal running while frames keep arriving, ddm-engine.ts:331-365):
// the snapshot holds every frame queued on the ingest stream so far; the
// analysis runs on its own stream and later ingests proceed concurrently.
// Slots those ingests overwrite must be masked out of `mask` by the caller
// (FrameClock.snapshot's guard). One live analysis at a time, as the
// reference's temporalBusy.
extern "C" int ddm_compute_temporal_live(ddm_engine *h, const uint32_t *order, const float *mask,
                                         int32_t full) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->ana_busy) {
    const cudaError_t q = cudaEventQuery(h->ana_ev);
    if (q == cudaErrorNotReady) {
      cudaGetLastError();
      return fail(h, DDM_ERR_STATE, "computeTemporal is already running");
    }
    int rc = join_analysis(h);
    if (rc) return rc;
  }
  CK(cudaEventRecord(h->ingest_ev, h->stream));
  CK(cudaStreamWaitEvent(h->ana_stream, h->ingest_ev, 0));
  int rc = temporal_impl(h, order, mask, full, h->ana_stream);
  if (rc) return rc;
  CK(cudaEventRecord(h->ana_ev, h->ana_stream));
  h->ana_busy = true;
  h->radial_from_live = true;
  return DDM_OK;
}

extern "C" int ddm_analysis_poll(ddm_engine *h, int32_t *done) {
  if (!h || !done) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  *done = 1;
  if (!h->ana_busy) return DDM_OK;
  const cudaError_t q = cudaEventQuery(h->ana_ev);
  if (q == cudaErrorNotReady) {
    cudaGetLastError();
    *done = 0;
    return DDM_OK;
  }
  return join_analysis(h);
}

extern "C" int ddm_wait_analysis(ddm_engine *h) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  return join_analysis(h);
}

extern "C" int ddm_read_radial(ddm_engine *h, double *D, double *P, double *drift) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  int rc = join_analysis(h);
  if (rc) return rc;
  if (!h->radial_valid) return fail(h, DDM_ERR_STATE, "readRadial: no computeTemporal since the last ingest");
  const size_t NB = h->g.NB, L = h->g.L;
  // a live snapshot's record is read on the analysis stream: no waiting for
  // the ingests queued after it
  cudaStream_t st = h->radial_from_live ? h->ana_stream : h->stream;
  if (D) CK(cudaMemcpyAsync(D, h->d_radD, sizeof(double) * NB * L, cudaMemcpyDeviceToHost, st));
  if (P) CK(cudaMemcpyAsync(P, h->d_radP, sizeof(double) * NB, cudaMemcpyDeviceToHost, st));
  if (drift) CK(cudaMemcpyAsync(drift, h->d_radDrift, sizeof(double) * NB * L * DRIFT, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return check_device_error(h);
}

extern "C" int ddm_read_history(ddm_engine *h, float *out) {
  if (!h || !out) return DDM_ERR_ARG;
  if (h->band_w) return fail(h, DDM_ERR_STATE, "readHistory: a banded engine holds one band of the history at a time");
  cudaSetDevice(h->device);
  CK(cudaMemcpyAsync(out, h->d_hist, sizeof(float2) * (size_t)h->modes * h->g.T, cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DDM_OK;
}

extern "C" int ddm_read_temporal_full(ddm_engine *h, float *D, float *C, float *P) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  int rc = join_analysis(h);
  if (rc) return rc;
  if (!h->full_valid)
    return fail(h, DDM_ERR_STATE, "readTemporalFull: the last computeTemporal did not keep full outputs");
  const size_t M = h->modes, L = h->g.L;
  cudaStream_t st = h->radial_from_live ? h->ana_stream : h->stream;
  if (D) CK(cudaMemcpyAsync(D, h->d_fullD, sizeof(float) * M * L, cudaMemcpyDeviceToHost, st));
  if (C) CK(cudaMemcpyAsync(C, h->d_fullC, sizeof(float2) * M * L, cudaMemcpyDeviceToHost, st));
  if (P) CK(cudaMemcpyAsync(P, h->d_fullP, sizeof(float) * M, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return check_device_error(h);
}

extern "C" int ddm_read_mean(ddm_engine *h, double *mean) {
  if (!h || !mean) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  if (h->last_mean_index < 0) return fail(h, DDM_ERR_STATE, "readMean: no frame ingested yet");
  CK(cudaMemcpyAsync(mean, h->d_means + h->last_mean_index, sizeof(double), cudaMemcpyDeviceToHost,
                     h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return DDM_OK;
}

extern "C" int ddm_idle(ddm_engine *h) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->device);
  CK(cudaStreamSynchronize(h->copy_stream));
  CK(cudaStreamSynchronize(h->stream));
  prune_inflight(h);
  int rc = join_analysis(h);
  if (rc) return rc;
  return check_device_error(h);
}

// ================================================================== batches
//
// Many videos (engines of any geometry on one device) analysed together:
// every engine's spatial chunks are queued on the batch stream without host
// synchronisation, and the temporal analysis of ALL videos is one persistent
// launch over the concatenated units of every engine (units carry their
// video index; per-video descriptors hold the history, order, mask, N(tau),
// mask spectrum and partials). The launch uses the largest TPAD of the
// batch: zero padding beyond T + L - 1 leaves every lag < L exact, so each
// video's radial record equals its own engine's. Each video's unit partials
// are then reduced by its engine's reduce kernel. The whole step can be
// captured once into a CUDA graph and replayed.

struct ddm_batch {
  std::vector<ddm_engine *> e;
  int device = 0;
  int TPAD = 0, Tmax = 0, Lmax = 0, nunits = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  VideoDesc *d_videos = nullptr;
  int4 *d_units = nullptr;
  float2 *d_tw = nullptr, *d_tw16 = nullptr;
  float2 *d_mspec = nullptr;           // [n][TPAD]
  float *d_npairs = nullptr;           // [n][Lmax]
  uint32_t *d_order = nullptr;         // [n][Tmax]
  float *d_mask = nullptr;             // [n][Tmax]
  char *h_meta = nullptr;              // pinned: order, mask, npairs, mspec of every video
  size_t meta_bytes = 0;
  int *d_counter = nullptr, *d_err = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::string err;
};

static int bfail(ddm_batch *b, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (b)
    b->err = buf;
  else
    g_create_error = buf;
  return code;
}

#define BCK(x)                                                                                \
  do {                                                                                        \
    cudaError_t e_ = (x);                                                                     \
    if (e_ != cudaSuccess) return bfail(b, DDM_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

static void batch_release(ddm_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (void *p : {(void *)b->d_videos, (void *)b->d_units, (void *)b->d_tw, (void *)b->d_tw16, (void *)b->d_mspec,
                  (void *)b->d_npairs, (void *)b->d_order, (void *)b->d_mask, (void *)b->d_counter,
                  (void *)b->d_err})
    if (p) cudaFree(p);
  if (b->h_meta) cudaFreeHost(b->h_meta);
  if (b->own) cudaStreamDestroy(b->own);
}

extern "C" const char *ddm_batch_last_error(const ddm_batch *b) { return b ? b->err.c_str() : g_create_error.c_str(); }

extern "C" int ddm_batch_create(ddm_engine *const *engines, int32_t n, ddm_batch **out) {
  g_create_error.clear();
  if (!out || !engines || n < 1) return bfail(nullptr, DDM_ERR_ARG, "ddm_batch_create: need n >= 1 engines");
  *out = nullptr;
  for (int i = 0; i < n; i++) {
    if (!engines[i]) return bfail(nullptr, DDM_ERR_ARG, "ddm_batch_create: engine %d is NULL", i);
    if (engines[i]->band_w) return bfail(nullptr, DDM_ERR_ARG, "ddm_batch_create: engine %d is banded", i);
  }
  ddm_batch *b = new ddm_batch();
  b->e.assign(engines, engines + n);
  b->device = engines[0]->device;
  for (auto *h : b->e) {
    if (h->device != b->device) {
      delete b;
      return bfail(nullptr, DDM_ERR_ARG, "ddm_batch_create: engines on different devices");
    }
    b->TPAD = std::max(b->TPAD, h->g.TPAD);
    b->Tmax = std::max(b->Tmax, h->g.T);
    b->Lmax = std::max(b->Lmax, h->g.L);
  }
  cudaSetDevice(b->device);
  std::vector<VideoDesc> vids(n);
  std::vector<int4> units;
  for (int i = 0; i < n; i++) {
    ddm_engine *h = b->e[i];
    VideoDesc &v = vids[i];
    v.hist = h->d_hist;
    v.items = h->d_items;
    v.partials = h->d_partials;
    v.T = h->g.T;
    v.L = h->g.L;
    v.unit0 = (int)units.size();
    v.nunits = h->nunits;
    for (int4 u : h->h_units) units.push_back(make_int4(u.x, u.y, u.z, i));
  }
  b->nunits = (int)units.size();
  b->meta_bytes = (size_t)n * (sizeof(uint32_t) * b->Tmax + sizeof(float) * b->Tmax + sizeof(float) * b->Lmax +
                               sizeof(float2) * b->TPAD);
  const std::vector<float> tw = twiddle_table(b->TPAD), tw16 = twiddle_table(b->TPAD, 16);
  bool ok = cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking) == cudaSuccess;
  b->stream = b->own;
  auto al = [&](void **p, size_t bytes) { ok = ok && cudaMalloc(p, bytes ? bytes : 1) == cudaSuccess; };
  al((void **)&b->d_videos, sizeof(VideoDesc) * n);
  al((void **)&b->d_units, sizeof(int4) * units.size());
  al((void **)&b->d_tw, sizeof(float) * tw.size());
  al((void **)&b->d_tw16, sizeof(float) * tw16.size());
  al((void **)&b->d_mspec, sizeof(float2) * n * (size_t)b->TPAD);
  al((void **)&b->d_npairs, sizeof(float) * n * (size_t)b->Lmax);
  al((void **)&b->d_order, sizeof(uint32_t) * n * (size_t)b->Tmax);
  al((void **)&b->d_mask, sizeof(float) * n * (size_t)b->Tmax);
  al((void **)&b->d_counter, sizeof(int));
  al((void **)&b->d_err, sizeof(int));
  ok = ok && cudaHostAlloc((void **)&b->h_meta, b->meta_bytes, cudaHostAllocDefault) == cudaSuccess;
  if (ok) {
    for (int i = 0; i < n; i++) {
      vids[i].order = b->d_order + (size_t)i * b->Tmax;
      vids[i].mask = b->d_mask + (size_t)i * b->Tmax;
      vids[i].npairs = b->d_npairs + (size_t)i * b->Lmax;
      vids[i].mspec = b->d_mspec + (size_t)i * b->TPAD;
    }
    ok = cudaMemcpy(b->d_videos, vids.data(), sizeof(VideoDesc) * n, cudaMemcpyHostToDevice) == cudaSuccess &&
         (units.empty() ||
          cudaMemcpy(b->d_units, units.data(), sizeof(int4) * units.size(), cudaMemcpyHostToDevice) == cudaSuccess) &&
         cudaMemcpy(b->d_tw, tw.data(), sizeof(float) * tw.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(b->d_tw16, tw16.data(), sizeof(float) * tw16.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(b->d_err, 0, sizeof(int)) == cudaSuccess;
  }
  if (!ok) {
    batch_release(b);
    delete b;
    return bfail(nullptr, DDM_ERR_NOMEM, "ddm_batch_create: device allocation or upload failed");
  }
  *out = b;
  return DDM_OK;
}

extern "C" void ddm_batch_destroy(ddm_batch *b) {
  if (!b) return;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  batch_release(b);
  delete b;
}

extern "C" int ddm_batch_set_stream(ddm_batch *b, void *stream) {
  if (!b) return DDM_ERR_ARG;
  b->stream = stream ? (cudaStream_t)stream : b->own;
  return DDM_OK;
}

// Spatial stage of every video from DEVICE frames, queued on the batch
// stream with no host synchronisation (capturable). frames[i]: n[i] frames of
// engine i's N*N pixels of dtypes[i] (16-byte aligned), slots[i][n[i]], scale
// per video. A scale differing from the engine's last one is uploaded first
// (a host synchronisation: set scales before capturing).
extern "C" int ddm_batch_ingest(ddm_batch *b, const void *const *frames, const int32_t *dtypes,
                                const int32_t *n, const int32_t *const *slots, const float *scales) {
  if (!b || !frames || !dtypes || !n || !slots || !scales) return bfail(b, DDM_ERR_ARG, "null argument");
  cudaSetDevice(b->device);
  for (size_t i = 0; i < b->e.size(); i++) {
    ddm_engine *h = b->e[i];
    if (n[i] == 0) continue;
    int rc = check_frames_args(h, frames[i], dtypes[i], n[i], slots[i]);
    if (rc) return bfail(b, rc, "video %zu: %s", i, h->err.c_str());
    if ((uintptr_t)frames[i] & 15) return bfail(b, DDM_ERR_ARG, "video %zu: frames must be 16-byte aligned", i);
    if ((rc = set_scale(h, scales[i]))) return bfail(b, rc, "video %zu: %s", i, h->err.c_str());
    cudaStream_t keep = h->stream;
    h->stream = b->stream;
    const size_t fbytes = (size_t)h->g.N * h->g.N * dtype_size(dtypes[i]);
    // the video's frame reference levels in one launch (as ingest_impl)
    const bool cref_all = n[i] > 0 && (size_t)n[i] <= h->rowc_cap;
    if (cref_all) {
      const cudaError_t e = launch_cref(h->g.N, dtypes[i], frames[i], (long long)h->g.N * h->g.N, n[i], h->d_rowc,
                                        h->stream);
      h->launches++;
      if (e != cudaSuccess) rc = fail(h, DDM_ERR_CUDA, "launch_cref failed: %s", cudaGetErrorString(e));
    }
    for (int c0 = 0; c0 < n[i] && !rc; c0 += h->chunk) {
      const int m = std::min(h->chunk, n[i] - c0);
      rc = launch_chunk(h, (const char *)frames[i] + (size_t)c0 * fbytes, dtypes[i], m, slots[i] + c0, scales[i],
                        cref_all ? h->d_rowc + c0 : nullptr);
    }
    h->stream = keep;
    if (rc) return bfail(b, rc, "video %zu: %s", i, h->err.c_str());
    h->radial_valid = false;
  }
  return DDM_OK;
}

extern "C" int ddm_batch_enqueue_temporal(ddm_batch *b);

// Temporal analysis of every video in ONE launch; orders[i], masks[i] of
// length T_i. Queued on the batch stream (no host synchronisation; the meta
// tables are computed on the host and copied from pinned memory in order).
extern "C" int ddm_batch_compute_temporal(ddm_batch *b, const uint32_t *const *orders, const float *const *masks) {
  if (!b || !orders || !masks) return bfail(b, DDM_ERR_ARG, "null argument");
  cudaSetDevice(b->device);
  const int nv = (int)b->e.size();
  uint32_t *ho = (uint32_t *)b->h_meta;
  float *hm = (float *)(ho + (size_t)nv * b->Tmax);
  float *hn = hm + (size_t)nv * b->Tmax;
  float *hs = hn + (size_t)nv * b->Lmax;
  // the pinned tables may still be read by the previous call's copies
  BCK(cudaStreamSynchronize(b->stream));
  for (int i = 0; i < nv; i++) {
    ddm_engine *h = b->e[i];
    const int T = h->g.T, L = h->g.L;
    if (!orders[i] || !masks[i]) return bfail(b, DDM_ERR_ARG, "video %d: order/mask is NULL", i);
    for (int j = 0; j < T; j++)
      if (orders[i][j] >= (uint32_t)T) return bfail(b, DDM_ERR_ARG, "video %d: order[%d] >= T", i, j);
    std::vector<float> npairs, mspec;
    temporal_meta(masks[i], T, b->TPAD, L, npairs, mspec);
    memcpy(ho + (size_t)i * b->Tmax, orders[i], sizeof(uint32_t) * T);
    for (int j = 0; j < T; j++) hm[(size_t)i * b->Tmax + j] = masks[i][j] != 0.f ? 1.f : 0.f;
    memcpy(hn + (size_t)i * b->Lmax, npairs.data(), sizeof(float) * L);
    memcpy(hs + (size_t)i * 2 * b->TPAD, mspec.data(), sizeof(float) * 2 * b->TPAD);
  }
  return ddm_batch_enqueue_temporal(b);
}

// The device part of ddm_batch_compute_temporal, from the pinned tables as
// they are when it runs (a graph replay re-reads them).
extern "C" int ddm_batch_enqueue_temporal(ddm_batch *b) {
  if (!b) return DDM_ERR_ARG;
  const int nv = (int)b->e.size();
  // pinned layout: order [n][Tmax], mask [n][Tmax], npairs [n][Lmax], mspec [n][TPAD]
  const char *hp = b->h_meta;
  BCK(cudaMemcpyAsync(b->d_order, hp, sizeof(uint32_t) * nv * (size_t)b->Tmax, cudaMemcpyHostToDevice, b->stream));
  BCK(cudaMemcpyAsync(b->d_mask, hp + sizeof(uint32_t) * nv * (size_t)b->Tmax, sizeof(float) * nv * (size_t)b->Tmax,
                      cudaMemcpyHostToDevice, b->stream));
  hp += (sizeof(uint32_t) + sizeof(float)) * nv * (size_t)b->Tmax;
  BCK(cudaMemcpyAsync(b->d_npairs, hp, sizeof(float) * nv * (size_t)b->Lmax, cudaMemcpyHostToDevice, b->stream));
  hp += sizeof(float) * nv * (size_t)b->Lmax;
  BCK(cudaMemcpyAsync(b->d_mspec, hp, sizeof(float2) * nv * (size_t)b->TPAD, cudaMemcpyHostToDevice, b->stream));
  TemporalParams tp{};
  tp.tw = b->d_tw;
  tp.tw16 = b->d_tw16;
  tp.variant = b->e[0]->variant;
  {  // every video's (binarised) mask within the sparse path's zero limit: the sparse-mask kernel
    const float *hm = (const float *)(b->h_meta + sizeof(uint32_t) * nv * (size_t)b->Tmax);
    const int limit = temporal_sparse_limit(b->TPAD, b->Tmax, b->Lmax, false);
    bool sparse = b->e[0]->sparse_enabled && limit > 0;
    for (int i = 0; sparse && i < nv; i++) {
      int nz = 0;
      for (int j = 0; j < b->e[i]->g.T; j++) nz += hm[(size_t)i * b->Tmax + j] == 0.f;
      sparse = nz <= limit;
    }
    tp.sparse = sparse ? 1 : 0;
  }
  tp.units = b->d_units;
  tp.nunits = b->nunits;
  tp.unit_counter = b->d_counter;
  tp.err = b->d_err;
  tp.T = b->Tmax;
  tp.L = b->Lmax;
  tp.videos = b->d_videos;
  BCK(cudaMemsetAsync(b->d_counter, 0, sizeof(int), b->stream));
  if (b->nunits > 0) {
    const int grid =
        std::min(temporal_max_grid(b->TPAD, b->Tmax, b->Lmax, false, tp.variant, tp.sparse != 0), b->nunits);
    BCK(launch_temporal(b->TPAD, b->Lmax, false, tp, std::max(grid, 1), b->stream));
  }
  const int tk = temporal_kernel_id(b->TPAD, false, tp.variant, tp.sparse != 0);
  for (ddm_engine *h : b->e) {
    h->last_tk = tk;
    ReduceParams rp{};
    rp.partials = h->d_partials;
    rp.bin_units = h->d_bin_units;
    rp.nmodes = h->d_nmodes;
    rp.nunits = h->nunits;
    rp.NB = h->g.NB;
    rp.L = h->g.L;
    rp.D = h->d_radD;
    rp.P = h->d_radP;
    rp.drift = h->d_radDrift;
    BCK(launch_reduce(rp, b->stream));
    h->radial_valid = true;
    h->full_valid = false;
  }
  return DDM_OK;
}

// Waits for the batch stream and surfaces device-side error words.
extern "C" int ddm_batch_sync(ddm_batch *b) {
  if (!b) return DDM_ERR_ARG;
  cudaSetDevice(b->device);
  BCK(cudaStreamSynchronize(b->stream));
  int e = 0;
  BCK(cudaMemcpy(&e, b->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  for (ddm_engine *h : b->e) {
    int he = 0;
    BCK(cudaMemcpy(&he, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (he) cudaMemset(h->d_err, 0, sizeof(int));
    e |= he;
  }
  if (e) {
    cudaMemset(b->d_err, 0, sizeof(int));
    return bfail(b, DDM_ERR_CUDA, "%s (code %d)",
                 e == 4 ? "a mask changed since the launch was recorded has more masked time indices than the "
                          "sparse-mask kernel holds"
                        : "a staged copy did not complete in time",
                 e);
  }
  return DDM_OK;
}

// Captures one full step -- ddm_batch_ingest of the given device frames and
// the temporal launch -- into a CUDA graph (replaces any earlier one). The
// meta tables are read from the pinned buffer at replay time: call
// ddm_batch_compute_temporal once before capturing (it fills them), and
// again with new orders/masks to refresh them before a replay.
extern "C" int ddm_batch_capture(ddm_batch *b, const void *const *frames, const int32_t *dtypes,
                                 const int32_t *n, const int32_t *const *slots, const float *scales) {
  if (!b) return DDM_ERR_ARG;
  cudaSetDevice(b->device);
  // scales must be in place before capture (their upload synchronises)
  for (size_t i = 0; i < b->e.size(); i++) {
    int rc = set_scale(b->e[i], scales[i]);
    if (rc) return bfail(b, rc, "video %zu: %s", i, b->e[i]->err.c_str());
  }
  BCK(cudaStreamSynchronize(b->stream));
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
  int rc = ddm_batch_ingest(b, frames, dtypes, n, slots, scales);
  if (!rc) rc = ddm_batch_enqueue_temporal(b);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return bfail(b, DDM_ERR_CUDA, "stream capture: %s", cudaGetErrorString(e));
  b->graph = g;
  BCK(cudaGraphInstantiate(&b->exec, g, 0));
  return DDM_OK;
}

extern "C" int ddm_batch_launch_graph(ddm_batch *b) {
  if (!b || !b->exec) return bfail(b, DDM_ERR_STATE, "no captured graph");
  cudaSetDevice(b->device);
  BCK(cudaGraphLaunch(b->exec, b->stream));
  for (ddm_engine *h : b->e) {
    h->radial_valid = true;
    h->full_valid = false;
  }
  return DDM_OK;
}

// ================================================================ autotuner
//
// Times the engine's own kernels on this device for its geometry and keeps
// the fastest choices:
//   spatial chunk  frames per row/column launch pair (multiples of the
//                  column kernel's frame group, up to the buffers' capacity):
//                  larger chunks amortise launches and waves, smaller ones
//                  keep the row-spectrum scratch resident in L2;
//   temporal unit  modes per work unit of the persistent temporal kernel:
//                  smaller units balance uneven bins, larger ones write fewer
//                  partial records.
// Each candidate is timed with CUDA events on the engine stream (median of 3
// after a warm-up) over a synthetic u16 video in a temporary device buffer.
// The runs overwrite the history ring: tune right after ddm_create, before
// ingesting, and before building batches over the engine.
extern "C" int ddm_autotune(ddm_engine *h, char *report, int32_t report_len) {
  if (!h) return DDM_ERR_ARG;
  if (h->band_w) return fail(h, DDM_ERR_STATE, "autotune: not available on a banded engine (use ddm_set_tuning)");
  cudaSetDevice(h->device);
  if (int rc0 = join_analysis(h)) return rc0;
  h->radial_from_live = false;
  const int N = h->g.N, T = h->g.T;
  const int fg = frames_per_col_cta(N);
  const int nfr = std::min(T, std::max(4 * h->chunk_cap, 64) / fg * fg);
  void *frames = nullptr;
  int rc = DDM_OK;
  CK(cudaMalloc(&frames, (size_t)nfr * N * N * 2));
  CK(cudaMemset(frames, 0x5A, (size_t)nfr * N * N * 2));  // any pixels: FFT time is data-independent
  std::vector<int32_t> slots(nfr);
  for (int i = 0; i < nfr; i++) slots[i] = i;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto med3 = [](float a, float b, float c) { return std::max(std::min(a, b), std::min(std::max(a, b), c)); };
  std::string rep = "{\"spatial_chunk\": {";
  // ---- spatial chunk
  int best_chunk = h->chunk;
  float best_t = 1e30f;
  const int keep_chunk = h->chunk;
  for (int c = fg; c <= h->chunk_cap; c += (c < 8 * fg ? fg : 2 * fg)) {
    h->chunk = c;
    float t[3];
    for (int r = -1; r < 3; r++) {
      cudaEventRecord(e0, h->stream);
      if ((rc = ingest_impl(h, frames, 1, nfr, slots.data(), 1.0f / 65535, true))) {
        h->chunk = keep_chunk;
        cudaFree(frames);
        return rc;
      }
      cudaEventRecord(e1, h->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        h->chunk = keep_chunk;
        cudaFree(frames);
        return fail(h, DDM_ERR_CUDA, "autotune: %s", cudaGetErrorString(cudaGetLastError()));
      }
      if (r >= 0) cudaEventElapsedTime(&t[r], e0, e1);
    }
    const float us = 1e3f * med3(t[0], t[1], t[2]) / nfr;
    char b[64];
    snprintf(b, sizeof b, "%s\"%d\": %.4f", c == fg ? "" : ", ", c, us);
    rep += b;
    if (us < best_t) best_t = us, best_chunk = c;
  }
  h->chunk = best_chunk;
  {
    char b[96];
    snprintf(b, sizeof b, "}, \"best_chunk\": %d, \"us_per_frame\": %.4f, \"temporal_unit\": {", best_chunk, best_t);
    rep += b;
  }
  // ---- temporal unit size
  std::vector<uint32_t> order(T);
  std::vector<float> mask(T, 1.f);
  for (int i = 0; i < T; i++) order[i] = i;
  int best_u = h->unit_size, best_var = h->variant;
  float best_tu = 1e30f;
  bool first = true;
  // the transform kernels (masks with many zeros) pick the variant and, when
  // the sparse path is off, the unit; an all-ones mask then times the
  // sparse-mask kernel, whose best unit wins when it is on (the common case:
  // a recording with few dropped frames)
  const bool sparse_was = h->sparse_enabled;
  const bool sparse_on = sparse_was && temporal_sparse_limit(h->g.TPAD, T, h->g.L, false) > 0;
  h->sparse_enabled = false;
  const int nvar = temporal_has_variant16(h->g.TPAD) ? 2 : 1;
  const int ncand = 6 * nvar + (sparse_on ? 6 : 0);
  int best_su = 0;
  float best_ts = 1e30f;
  for (int cand = 0; cand < ncand && !rc; cand++) {
    const bool sp = cand >= 6 * nvar;
    const int U = 8 << (cand % 6), var = sp ? best_var : cand / 6;
    if (sp && cand == 6 * nvar) {
      h->sparse_enabled = true;
      rep += "}, \"sparse_unit\": {";
      first = true;
    }
    h->variant = var;
    if ((rc = build_units(h, U))) break;
    float t[3];
    for (int r = -1; r < 3; r++) {
      cudaEventRecord(e0, h->stream);
      if ((rc = temporal_impl(h, order.data(), mask.data(), 0, h->stream))) break;
      cudaEventRecord(e1, h->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        rc = fail(h, DDM_ERR_CUDA, "autotune: %s", cudaGetErrorString(cudaGetLastError()));
        break;
      }
      if (r >= 0) cudaEventElapsedTime(&t[r], e0, e1);
    }
    if (rc) break;
    const float ms = med3(t[0], t[1], t[2]);
    char b[64];
    snprintf(b, sizeof b, "%s\"%s%d\": %.4f", first ? "" : ", ", !sp && var ? "r16:" : "", U, ms);
    rep += b;
    first = false;
    if (sp) {
      if (ms < best_ts) best_ts = ms, best_su = U;
    } else if (ms < best_tu) {
      best_tu = ms, best_u = U, best_var = var;
    }
  }
  h->sparse_enabled = sparse_was;
  h->variant = best_var;
  if (best_su > 0) best_u = best_su, best_tu = best_ts;
  if (!rc) rc = build_units(h, best_u);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(frames);
  h->have_frames = false;
  h->radial_valid = h->full_valid = false;
  if (rc) return rc;
  {
    char b[96];
    snprintf(b, sizeof b, "}, \"best_unit\": %d, \"best_variant\": %d, \"temporal_ms\": %.4f}", best_u,
             best_var, best_tu);
    rep += b;
  }
  if (report && report_len > 0) {
    strncpy(report, rep.c_str(), report_len - 1);
    report[report_len - 1] = 0;
  }
  return check_device_error(h);
}

extern "C" int ddm_set_sparse(ddm_engine *h, int32_t enable) {
  if (!h) return DDM_ERR_ARG;
  h->sparse_enabled = enable != 0;
  return DDM_OK;
}

extern "C" int ddm_set_blocked(ddm_engine *h, int32_t enable) {
  if (!h) return DDM_ERR_ARG;
  h->blocked_enabled = enable != 0;
  return DDM_OK;
}

extern "C" int ddm_last_temporal_kernel(const ddm_engine *h) { return h ? h->last_tk : DDM_ERR_ARG; }

extern "C" int ddm_get_tuning(const ddm_engine *h, int32_t *chunk, int32_t *unit_size, int32_t *variant) {
  if (!h) return DDM_ERR_ARG;
  if (chunk) *chunk = h->chunk;
  if (unit_size) *unit_size = h->unit_size;
  if (variant) *variant = h->variant;
  return DDM_OK;
}

// Applies a tuning found earlier (e.g. a cached ddm_autotune result) without
// timing: chunk a multiple of the column kernel's frame group within the
// buffers' capacity, unit_size >= 1 (0 keeps the current value).
extern "C" int ddm_set_tuning(ddm_engine *h, int32_t chunk, int32_t unit_size, int32_t variant) {
  if (!h) return DDM_ERR_ARG;
  if (variant < -1 || variant > 1 || (variant == 1 && !temporal_has_variant16(h->g.TPAD)))
    return fail(h, DDM_ERR_ARG, "variant %d: 0 (radix-8), 1 (radix-16, TPAD 1024..4096) or -1 (keep)", variant);
  cudaSetDevice(h->device);
  const int fg = frames_per_col_cta(h->g.N);
  if (chunk) {
    if (chunk < fg || chunk > h->chunk_cap || chunk % fg)
      return fail(h, DDM_ERR_ARG, "chunk %d: need a multiple of %d in [%d, %d]", chunk, fg, fg, h->chunk_cap);
  }
  if (unit_size < 0) return fail(h, DDM_ERR_ARG, "unit_size must be >= 0");
  CK(cudaStreamSynchronize(h->stream));
  if (chunk) h->chunk = chunk;
  if (variant >= 0 && variant != h->variant) {
    h->variant = variant;
    h->radial_valid = h->full_valid = false;
  }
  if (unit_size && unit_size != h->unit_size) {
    int rc = build_units(h, unit_size);
    if (!rc && h->band_w) rc = build_band_units(h);
    if (rc) return rc;
    h->radial_valid = h->full_valid = false;
  }
  return DDM_OK;
}

// The analysis of a video on a banded engine: for each band of spectrum
// columns, the spatial pass of every frame (host frames stream through the
// pinned staging again: the frame stack is not held on the device) writing
// only that band's history, then the band's temporal pass, whose radial sums
// are added to the record band after band.
extern "C" int ddm_analyze_banded(ddm_engine *h, const void *frames, int32_t dtype, int32_t n, const int32_t *slots,
                                  float scale, const uint32_t *order, const float *mask, int32_t on_device) {
  if (!h) return DDM_ERR_ARG;
  if (!h->band_w) return fail(h, DDM_ERR_STATE, "ddm_analyze_banded: the engine was not created banded");
  cudaSetDevice(h->device);
  int rc = check_frames_args(h, frames, dtype, n, slots);
  if (rc) return rc;
  if (!order || !mask) return fail(h, DDM_ERR_ARG, "ddm_analyze_banded: order/mask must have length %d", h->g.T);
  h->radial_valid = false;
  h->in_banded = true;
  for (const auto &b : h->bands) {
    h->cur_kb0 = b.kb0;
    h->cur_nkb = b.nkb;
    if ((rc = ingest_impl(h, frames, dtype, n, slots, scale, on_device != 0)) ||
        (rc = temporal_impl(h, order, mask, 0, h->stream, &b)))
      break;
  }
  h->in_banded = false;
  h->cur_kb0 = h->cur_nkb = 0;
  if (rc) return rc;
  CK(cudaStreamSynchronize(h->stream));
  if ((rc = check_device_error(h))) return rc;
  h->radial_valid = true;
  return DDM_OK;
}
