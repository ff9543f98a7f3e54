// ddm_spectra_noalloc: the spatial stage (windowed half-plane 2D FFT of each
// frame into a mode-major history ring) for callers that cannot allocate
// device memory.
//
// Who needs it: code that runs where cudaMalloc is off limits -- an embedding
// host that owns every device allocation and hands its plugins only the
// buffers it planned (an acquisition or streaming framework with a fixed
// memory budget), or a real-time capture loop that must never enter the
// allocator, whose cudaMalloc/cudaFree can block on device-wide
// synchronisation. Such a caller still provides the frames and the output
// ring; everything else this path needs lives in fixed, file-scope device
// arrays of this library.
//
// Scratch: the row spectra between the row and column passes live in
// g_rows_scratch, a static __device__ array of NOALLOC_SCRATCH_BYTES (8 MiB);
// together with the small tables below every GPU that loads this library
// holds about 8.6 MiB until the process exits. Frames are processed in
// chunks that fit the scratch; ROIs with N > 512 do not fit and are
// rejected. Nothing needs clearing: each call writes every scratch element
// before reading it, except the per-frame pixel sums, which it zeroes.
//
// Calls share the arrays: two calls whose work overlaps on the GPU (different
// streams, or different host threads on the same device) race on the
// scratch and the tables. Serialise them.
//
// Set-up: the first call on a device, with that device current, looks up the
// device addresses of the arrays (cudaGetSymbolAddress) and fills the tables;
// make that first call before any stream capture. A later call with another N
// or scale refills the tables, ordered on the caller's stream.
//
// Errors on the device: the row and column kernels wait for their staged
// copies with bounded waits. A wait that gives up leaves part of the ring
// unwritten and records a code in g_err, a file-scope device word that each
// call zeroes on its stream before its kernels run. The call itself returns
// once the work is queued; ddm_spectra_noalloc_status(stream) waits for the
// stream, reads the word (a copy from the symbol, no allocation) and turns
// a recorded code into DDM_ERR_CUDA.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ddm_b200.h"
#include "kernels.cuh"
#include "tables.h"

using namespace ddm;

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 8u << 20;
constexpr int NOALLOC_MAX_N = 512;

static __device__ __align__(256) float2 g_rows_scratch[NOALLOC_SCRATCH_BYTES / sizeof(float2)];
static __device__ __align__(256) float g_rowc[MAX_CHUNK * NOALLOC_MAX_N];
static __device__ __align__(256) double g_framesum[MAX_CHUNK];
static __device__ __align__(256) double g_means[MAX_CHUNK];
static __device__ __align__(256) float g_win[NOALLOC_MAX_N];
static __device__ __align__(256) float g_wys[NOALLOC_MAX_N];
static __device__ __align__(256) float2 g_tw[NOALLOC_MAX_N];
static __device__ __align__(256) float2 g_wcorr4[4];
static __device__ __align__(256) double g_invtot[1];
static __device__ __align__(256) int g_err[1];  // 0, or the code of a bounded wait that gave up

struct DeviceState {
  bool ready = false;
  float2* rows = nullptr;
  float* rowc = nullptr;
  double* framesum = nullptr;
  double* means = nullptr;
  float* win = nullptr;
  float* wys = nullptr;
  float2* tw = nullptr;
  float2* wcorr4 = nullptr;
  double* invtot = nullptr;
  int* err = nullptr;
  int N = 0;
  float scale = 0.f;
};

std::mutex g_mu;
std::vector<DeviceState> g_state;

int lookup(const void* symbol, void** out) {
  return cudaGetSymbolAddress(out, symbol) == cudaSuccess ? DDM_OK : DDM_ERR_CUDA;
}

}  // namespace

extern std::string& ddm_detached_error();  // message slot of calls without an engine (engine.cu)

static int nf_fail(int code, const char* msg) {
  ddm_detached_error() = msg;
  return code;
}

extern "C" int ddm_spectra_noalloc(const void* frames, int32_t dtype, int32_t n, int32_t N, int32_t T,
                                   const int32_t* slots, float scale, void* hist, void* stream) {
  if (N < 64 || N > NOALLOC_MAX_N || (N & (N - 1)))
    return nf_fail(N > NOALLOC_MAX_N ? DDM_ERR_TOO_LARGE : DDM_ERR_ARG,
                   "ddm_spectra_noalloc: N must be a power of two in [64, 512] (the fixed 8 MiB scratch)");
  if (dtype < 0 || dtype > 2) return nf_fail(DDM_ERR_ARG, "ddm_spectra_noalloc: dtype must be 0, 1 or 2");
  if (n < 0 || T < 1) return nf_fail(DDM_ERR_ARG, "ddm_spectra_noalloc: need n >= 0 and T >= 1");
  if (n > 0 && (!frames || !slots || !hist)) return nf_fail(DDM_ERR_ARG, "ddm_spectra_noalloc: null pointer");
  if (!(scale > 0) || !std::isfinite(scale)) return nf_fail(DDM_ERR_ARG, "ddm_spectra_noalloc: scale must be > 0");
  if ((uintptr_t)frames & 15) return nf_fail(DDM_ERR_ARG, "ddm_spectra_noalloc: frames must be 16-byte aligned");
  for (int i = 0; i < n; i++)
    if (slots[i] < 0) return nf_fail(DDM_ERR_ARG, "ddm_spectra_noalloc: slots must be >= 0");
  if (n == 0) return DDM_OK;
  const int NH = N / 2 + 1, NHB = (NH + KB - 1) / KB;
  const size_t per_frame = (size_t)NHB * N * KB * sizeof(float2);
  const int fg = frames_per_col_cta(N);
  const int chunk = (int)std::min<size_t>(MAX_CHUNK, NOALLOC_SCRATCH_BYTES / per_frame) / fg * fg;
  if (chunk < 1) return nf_fail(DDM_ERR_TOO_LARGE, "ddm_spectra_noalloc: frame does not fit the scratch");
  cudaStream_t s = (cudaStream_t)stream;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nf_fail(DDM_ERR_NODEV, "ddm_spectra_noalloc: no device");
  DeviceState st;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if ((int)g_state.size() <= dev) g_state.resize(dev + 1);
    DeviceState& d = g_state[dev];
    if (!d.ready) {  // once per device, with that device current
      if (lookup(g_rows_scratch, (void**)&d.rows) || lookup(g_rowc, (void**)&d.rowc) ||
          lookup(g_framesum, (void**)&d.framesum) || lookup(g_means, (void**)&d.means) ||
          lookup(g_win, (void**)&d.win) || lookup(g_wys, (void**)&d.wys) || lookup(g_tw, (void**)&d.tw) ||
          lookup(g_wcorr4, (void**)&d.wcorr4) || lookup(g_invtot, (void**)&d.invtot) ||
          lookup(g_err, (void**)&d.err))
        return nf_fail(DDM_ERR_CUDA, "ddm_spectra_noalloc: cudaGetSymbolAddress failed");
      d.ready = true;
    }
    if (d.N != N || d.scale != scale) {  // tables for this geometry and scale
      const std::vector<double> w = blackman_harris(N);
      std::vector<float> wf(N), wys(N);
      for (int i = 0; i < N; i++) {
        wf[i] = (float)w[i];
        wys[i] = (float)(w[i] * (double)scale);
      }
      const std::vector<float> tw = twiddle_table(N);
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
      const double invtot = 1.0 / ((double)N * N);
      if (cudaMemcpyToSymbolAsync(g_win, wf.data(), sizeof(float) * N, 0, cudaMemcpyHostToDevice, s) ||
          cudaMemcpyToSymbolAsync(g_wys, wys.data(), sizeof(float) * N, 0, cudaMemcpyHostToDevice, s) ||
          cudaMemcpyToSymbolAsync(g_tw, tw.data(), sizeof(float) * tw.size(), 0, cudaMemcpyHostToDevice, s) ||
          cudaMemcpyToSymbolAsync(g_wcorr4, wc4, sizeof wc4, 0, cudaMemcpyHostToDevice, s) ||
          cudaMemcpyToSymbolAsync(g_invtot, &invtot, sizeof invtot, 0, cudaMemcpyHostToDevice, s) ||
          cudaStreamSynchronize(s))  // the host vectors above go out of scope
        return nf_fail(DDM_ERR_CUDA, "ddm_spectra_noalloc: table upload failed");
      d.N = N;
      d.scale = scale;
    }
    st = d;
  }
  const size_t fbytes = (size_t)N * N * (dtype == 0 ? 1 : dtype == 1 ? 2 : 4);
  if (cudaMemsetAsync(st.err, 0, sizeof(int), s) != cudaSuccess)
    return nf_fail(DDM_ERR_CUDA, "ddm_spectra_noalloc: cudaMemsetAsync failed");
  for (int c0 = 0; c0 < n; c0 += chunk) {
    const int m = std::min(chunk, n - c0);
    if (cudaMemsetAsync(st.framesum, 0, sizeof(double) * m, s) != cudaSuccess)
      return nf_fail(DDM_ERR_CUDA, "ddm_spectra_noalloc: cudaMemsetAsync failed");
    RowParams rp{};
    rp.frames = (const char*)frames + (size_t)c0 * fbytes;
    rp.frame_stride = (long long)N * N;
    rp.nframes = m;
    rp.win = st.win;
    rp.wys = st.wys;
    rp.smask = nullptr;
    rp.tw = st.tw;
    rp.rows = st.rows;
    rp.framec = st.rowc;
    rp.framesum = st.framesum;
    rp.err = st.err;
    if (launch_rows(N, dtype, rp, s) != cudaSuccess)
      return nf_fail(DDM_ERR_CUDA, "ddm_spectra_noalloc: row kernel launch failed");
    ColParams cp{};
    cp.rows = st.rows;
    cp.framec = st.rowc;
    cp.framesum = st.framesum;
    cp.inv_total = st.invtot;
    cp.w2d = nullptr;
    cp.wc4 = st.wcorr4;
    for (int i = 0; i < m; i++) cp.slots[i] = slots[c0 + i] % T;
    cp.tw = st.tw;
    cp.hist = (float2*)hist;
    cp.means = st.means;
    cp.scale = scale;
    cp.nframes = m;
    cp.T = T;
    cp.NH = NH;
    cp.NHB = NHB;
    cp.err = st.err;
    if (launch_cols(N, cp, s) != cudaSuccess)
      return nf_fail(DDM_ERR_CUDA, "ddm_spectra_noalloc: column kernel launch failed");
  }
  return DDM_OK;
}

extern "C" int ddm_spectra_noalloc_status(void* stream) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nf_fail(DDM_ERR_NODEV, "ddm_spectra_noalloc_status: no device");
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if ((int)g_state.size() <= dev || !g_state[dev].ready) return DDM_OK;  // no call on this device yet
  }
  if (cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
    return nf_fail(DDM_ERR_CUDA, "ddm_spectra_noalloc_status: stream synchronisation failed");
  int e = 0;
  if (cudaMemcpyFromSymbol(&e, g_err, sizeof(int)) != cudaSuccess)
    return nf_fail(DDM_ERR_CUDA, "ddm_spectra_noalloc_status: reading the error word failed");
  if (e) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_err, &zero, sizeof(int));
    return nf_fail(DDM_ERR_CUDA, e == 2 ? "ddm_spectra_noalloc: a staged row copy did not complete in time (code 2)"
                                        : "ddm_spectra_noalloc: a staged column copy did not complete in time (code 3)");
  }
  return DDM_OK;
}
