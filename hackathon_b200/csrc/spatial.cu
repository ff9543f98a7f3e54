// Per-frame windowed half-plane 2D FFT into the mode-major history ring.
//
// Reference semantics (motility-ddm/src/fft.js:149-183, ddm.wgsl:134-192,
// ddm_ref.js:196-206): subtract the frame mean, multiply by w(x) w(y), 2D FFT,
// keep kx = 0..N/2, scale by 1/N, store mode m = ky*NH + kx at
// hist[m*T + slot].
//
// B200 formulation, two kernels per chunk of frames:
//  rows_kernel  reads raw u8/u16/f32 pixels (convert and luma scale fused
//               into the load) and transforms two rows per complex FFT
//               (real-input packing) after subtracting a per-row reference
//               level c_y (the mean of four pixels of the row, exact in FP32
//               for integer frames). It writes the row spectra to an
//               L2-resident scratch in a [frame][kx/2][y][2] blocked layout
//               (full 32 B sectors), c_y, and one FP64 atomic per CTA into
//               the frame's pixel sum.
//  cols_kernel  restores the exact frame mean by linearity:
//                 FFT_x((I - mu) w) = FFT_x((I - c_y) w) + (c_y - mu) W(kx),
//               W the window's DFT (non-zero only at kx <= 3 for the 4-term
//               Blackman-Harris; a per-row table when a spatial ROI mask is
//               set), computed in FP64. One FFT group per frame reads its
//               column pair straight into registers (one float4 per row),
//               runs the column FFTs, scales by 1/N, and the CTA stores the
//               FG frames of a mode together: FG consecutive ring slots form
//               one 32 B sector.
// Subtracting c_y keeps the FP32 row transform free of the large DC term
// (the cancellation the reference avoids with its (hi, lo) mean,
// ddm.wgsl:129-150); the correction term is the small (c_y - mu) and is
// formed in FP64.
#include <cstdint>
#include <type_traits>

#include "fft_block.cuh"
#include "kernels.cuh"

namespace ddm {

template <typename Tin>
__device__ __forceinline__ float ld_pix(const Tin* p) {
  return (float)__ldg(p);
}

// Pixels of one row pair (8 per thread per row, FFT input pattern) and the
// rows' reference levels, loaded one iteration ahead of their use.
template <int N, typename Tin>
struct RowInput {
  float a0[8], a1[8];
  float c0, c1;
  __device__ __forceinline__ void load(const RowParams& p, long long pair, int t) {
    constexpr int NT = N / 8;
    const bool valid = pair < (long long)p.nframes * (N / 2);
    const int f = valid ? (int)(pair / (N / 2)) : 0;
    const int y0 = valid ? 2 * (int)(pair % (N / 2)) : 0;
    const Tin* r0 = (const Tin*)p.frames + (size_t)f * p.frame_stride + (size_t)y0 * N;
    const Tin* r1 = r0 + N;
    c0 = c1 = 0.f;
    if (valid) {
      // per-row reference level: mean of four pixels (broadcast loads)
      c0 = 0.25f * ((ld_pix(r0) + ld_pix(r0 + N / 4)) + (ld_pix(r0 + N / 2) + ld_pix(r0 + 3 * N / 4)));
      c1 = 0.25f * ((ld_pix(r1) + ld_pix(r1 + N / 4)) + (ld_pix(r1 + N / 2) + ld_pix(r1 + 3 * N / 4)));
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      a0[q] = valid ? ld_pix(r0 + t + q * NT) : 0.f;
      a1[q] = valid ? ld_pix(r1 + t + q * NT) : 0.f;
    }
  }
};

// Persistent: each CTA walks batches of G row pairs (one frame per batch),
// prefetching the next batch's pixels while it transforms the current one.
template <int N, typename Tin>
__global__ void __launch_bounds__(256) rows_kernel(RowParams p) {
  constexpr int NT = N / 8;
  constexpr int G = 256 / NT >= 1 ? 256 / NT : 1;
  constexpr int PN = padded(N);
  constexpr int NHB = (N / 2 + 1 + KB - 1) / KB;
  constexpr int WARPS = (G * NT + 31) / 32;
  constexpr int SYNC = sync_kind(N, G);
  extern __shared__ float2 sm[];
  __shared__ double red[WARPS];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  float2* buf0 = sm + (size_t)g * 2 * PN;
  float2* buf1 = buf0 + PN;
  float2* s_tw = sm + (size_t)G * 2 * PN;
  for (int i = threadIdx.x; i < tw_size(N); i += blockDim.x) s_tw[i] = p.tw[i];
  const long long npairs = (long long)p.nframes * (N / 2);
  const long long nbatch = (npairs + G - 1) / G;
  // pixel sums: exact integers for u8/u16 (warp totals < 2^31), FP64 for f32
  constexpr bool INT = !std::is_floating_point<Tin>::value;
  using acc_t = typename std::conditional<INT, int, double>::type;
  RowInput<N, Tin> cur, nxt;
  long long b = blockIdx.x;
  cur.load(p, b * G + g, t);
  __syncthreads();
  for (; b < nbatch; b += gridDim.x) {
    if (b + gridDim.x < nbatch) nxt.load(p, (b + gridDim.x) * G + g, t);
    const long long pair = b * G + g;
    const bool valid = pair < npairs;
    const int f = (int)((b * G) / (N / 2));  // all G pairs of a batch share the frame
    const int y0 = valid ? 2 * (int)(pair % (N / 2)) : 0;
    const uint8_t* m0p = p.smask ? p.smask + (size_t)y0 * N : nullptr;
    const float wy0 = p.wys[y0], wy1 = p.wys[y0 + 1];
    float2 v[8];
    acc_t s = 0;
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int x = t + q * NT;
      float m0 = 1.f, m1 = 1.f;
      if (m0p) {
        m0 = (float)m0p[x];
        m1 = (float)m0p[N + x];
      }
      const float a0 = cur.a0[q] * m0, a1 = cur.a1[q] * m1;
      if constexpr (INT)
        s += (int)a0 + (int)a1;
      else
        s += (double)a0 + (double)a1;
      const float wx = __ldg(&p.win[x]);
      v[q] = make_float2((cur.a0[q] - cur.c0) * (wx * m0 * wy0), (cur.a1[q] - cur.c1) * (wx * m1 * wy1));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = (double)s;
    const float2* Z = fft<N, false, true, SYNC>(v, t, buf0, buf1, s_tw, 1 + g);
    __syncthreads();  // red[] complete; every group done with its buffers' reads below
    if (threadIdx.x == 0) {
      double tot = 0.0;
#pragma unroll
      for (int w = 0; w < WARPS; w++) tot += red[w];
      atomicAdd(&p.framesum[f], tot);
    }
    if (valid) {
      float2* out = p.rows + (size_t)f * NHB * N * KB;
      for (int kx = t; kx <= N / 2; kx += NT) {
        const float2 zk = Z[pad(kx)];
        const float2 zn = Z[pad((N - kx) & (N - 1))];
        const float2 R0 = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
        const float2 R1 = make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
        float2* o = out + ((size_t)(kx / KB) * N + y0) * KB + (kx % KB);
        o[0] = R0;
        o[KB] = R1;
      }
      if (t == 0) {
        p.rowc[(size_t)f * N + y0] = cur.c0;
        p.rowc[(size_t)f * N + y0 + 1] = cur.c1;
      }
    }
    cur = nxt;
    __syncthreads();  // buffers and red[] are reused by the next batch
  }
}

// Inputs of one column-pair tile for this thread's group: both columns at the
// group's 8 rows (one float4 per row) and the correction coefficients.
template <int N>
struct ColInput {
  float4 col[8];
  float dy[8];
  __device__ __forceinline__ void load(const ColParams& p, int kb, int f, bool fvalid, int t) {
    constexpr int NT = N / 8;
    const double mu = fvalid ? p.framesum[f] * p.inv_total[0] : 0.0;
    const float4* src = (const float4*)(p.rows + ((size_t)f * p.NHB + kb) * N * KB);
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int y = t + q * NT;
      col[q] = fvalid ? __ldg(&src[y]) : make_float4(0.f, 0.f, 0.f, 0.f);
      dy[q] = fvalid ? (float)(((double)p.rowc[(size_t)f * N + y] - mu) * (double)p.wys[y]) : 0.f;
    }
  }
};

// Persistent: each CTA walks tiles (column pair kb, group of G frames) and
// prefetches the next tile's inputs while it transforms the current one.
template <int N>
__global__ void __launch_bounds__(256, 2) cols_kernel(ColParams p) {
  constexpr int NT = N / 8;
  constexpr int G = 256 / NT >= 1 ? 256 / NT : 1;  // frames per tile, one per group
  constexpr int PN = padded(N);
  constexpr int SYNC = sync_kind(N, G);
  extern __shared__ float2 sm[];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  float2* buf0 = sm + (size_t)g * 2 * PN;
  float2* buf1 = buf0 + PN;
  float2* s_tw = sm + (size_t)G * 2 * PN;
  for (int i = threadIdx.x; i < tw_size(N); i += blockDim.x) s_tw[i] = p.tw[i];
  const int nfg = (p.nframes + G - 1) / G;
  const int ntiles = p.NHB * nfg;
  const float invN = 1.f / N;
  const int sf = threadIdx.x % G;  // frame of the tile this thread stores
  ColInput<N> cur, nxt;
  int tile = blockIdx.x;
  {
    const int kb = tile % p.NHB, f0 = (tile / p.NHB) * G;
    cur.load(p, kb, f0 + g, tile < ntiles && f0 + g < p.nframes, t);
  }
  __syncthreads();
  for (; tile < ntiles; tile += gridDim.x) {
    const int kb = tile % p.NHB;
    const int f0 = (tile / p.NHB) * G;
    const int nf = min(G, p.nframes - f0);
    {
      const int tn = tile + gridDim.x;
      const int kbn = tn % p.NHB, f0n = (tn / p.NHB) * G;
      if (tn < ntiles) nxt.load(p, kbn, f0n + g, f0n + g < p.nframes, t);
    }
    if (kb == 0 && t == 0 && g < nf) p.means[f0 + g] = p.framesum[f0 + g] * p.inv_total[0] * (double)p.scale;
    const int slot = sf < nf ? p.slots[f0 + sf] : 0;
#pragma unroll 1
    for (int c = 0; c < KB; c++) {
      const int kx = kb * KB + c;
      if (kx >= p.NH) break;  // uniform over the CTA
      float2 v[8];
      const bool sep = !p.wcorr_full && kx < 4;
      const float2 wc = sep ? p.wcorr[kx] : make_float2(0.f, 0.f);
#pragma unroll
      for (int q = 0; q < 8; q++) {
        float2 a = c == 0 ? make_float2(cur.col[q].x, cur.col[q].y) : make_float2(cur.col[q].z, cur.col[q].w);
        float2 w = wc;
        if (p.wcorr_full) w = p.wcorr[(size_t)(t + q * NT) * p.NH + kx];
        if (sep || p.wcorr_full) {
          a.x = fmaf(cur.dy[q], w.x, a.x);
          a.y = fmaf(cur.dy[q], w.y, a.y);
        }
        v[q] = a;
      }
      const float2* Y = fft<N, false, true, SYNC>(v, t, buf0, buf1, s_tw, 1 + g);
      __syncthreads();  // every group's column is in shared memory
      // Y of group g sits at the same offset in every group's buffer pair; the
      // CTA writes frame sf = tid % G of each mode: G consecutive ring slots
      if (sf < nf) {
        const int yoff = (int)(Y - (sm + (size_t)g * 2 * PN));
        const float2* ys = sm + (size_t)sf * 2 * PN + yoff;
        float2* hs = p.hist + (size_t)kx * p.T + slot;
        const size_t mstride = (size_t)p.NH * p.T;
        for (int ky = threadIdx.x / G; ky < N; ky += 256 / G) {
          const float2 y = ys[pad(ky)];
          hs[(size_t)ky * mstride] = make_float2(y.x * invN, y.y * invN);
        }
      }
      __syncthreads();
    }
    cur = nxt;
  }
}

// ------------------------------------------------------------------ launchers

template <int N>
static constexpr int groups() {
  return 256 / (N / 8) >= 1 ? 256 / (N / 8) : 1;
}

template <int N>
static size_t fft_smem() {
  return ((size_t)groups<N>() * 2 * padded(N) + tw_size(N)) * sizeof(float2);
}

template <typename K>
static int persistent_grid(K k, int threads, size_t smem, long long work) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, threads, smem);
  const long long g = (long long)sms * (per > 0 ? per : 1);
  return (int)(work < g ? (work > 0 ? work : 1) : g);
}

template <int N, typename Tin>
static cudaError_t rows_n(const RowParams& p, cudaStream_t s) {
  constexpr int G = groups<N>();
  const long long npairs = (long long)p.nframes * (N / 2);
  auto k = rows_kernel<N, Tin>;
  const size_t sm = fft_smem<N>();
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const int grid = persistent_grid(k, G * (N / 8), sm, (npairs + G - 1) / G);
  k<<<grid, G * (N / 8), sm, s>>>(p);
  return cudaGetLastError();
}

template <int N>
static cudaError_t rows_dt(int dtype, const RowParams& p, cudaStream_t s) {
  switch (dtype) {
    case 0: return rows_n<N, uint8_t>(p, s);
    case 1: return rows_n<N, uint16_t>(p, s);
    case 2: return rows_n<N, float>(p, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_rows(int N, int dtype, const RowParams& p, cudaStream_t s) {
  switch (N) {
    case 64: return rows_dt<64>(dtype, p, s);
    case 128: return rows_dt<128>(dtype, p, s);
    case 256: return rows_dt<256>(dtype, p, s);
    case 512: return rows_dt<512>(dtype, p, s);
    case 1024: return rows_dt<1024>(dtype, p, s);
    case 2048: return rows_dt<2048>(dtype, p, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int N>
static cudaError_t cols_n(const ColParams& p, cudaStream_t s) {
  constexpr int G = groups<N>();
  auto k = cols_kernel<N>;
  const size_t sm = fft_smem<N>();
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  const int grid = persistent_grid(k, G * (N / 8), sm, (long long)p.NHB * ((p.nframes + G - 1) / G));
  k<<<grid, G * (N / 8), sm, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_cols(int N, const ColParams& p, cudaStream_t s) {
  switch (N) {
    case 64: return cols_n<64>(p, s);
    case 128: return cols_n<128>(p, s);
    case 256: return cols_n<256>(p, s);
    case 512: return cols_n<512>(p, s);
    case 1024: return cols_n<1024>(p, s);
    case 2048: return cols_n<2048>(p, s);
    default: return cudaErrorInvalidValue;
  }
}

int frames_per_col_cta(int N) { return N >= 2048 ? 1 : 256 / (N / 8); }

}  // namespace ddm
