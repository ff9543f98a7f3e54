// Per-frame windowed half-plane 2D FFT into the mode-major history ring.
//
// Reference semantics (motility-ddm/src/fft.js:149-183, ddm.wgsl:134-192,
// ddm_ref.js:196-206): subtract the frame mean, multiply by w(x) w(y), 2D FFT,
// keep kx = 0..N/2, scale by 1/N, store mode m = ky*NH + kx at
// hist[m*T + slot].
//
// B200 formulation, two kernels per chunk of frames:
//  rows_kernel  stages batches of raw u8/u16/f32 rows (and the spatial mask's
//               rows) into shared memory with bulk copies, converts, subtracts
//               a frame reference level c_f (mean of a fixed 16 x 16 grid of
//               the frame's pixels, reduced in a fixed order so that every
//               CTA gets the same value; exact for integer frames), multiplies by
//               w(x) w(y) scale m(x,y), and transforms two rows per complex
//               FFT (real-input packing). It writes the row spectra to an
//               L2-resident scratch in a [frame][kx/2][2][y] blocked layout,
//               c_f, and one FP64 atomic per CTA into the frame's pixel sum.
//  cols_kernel  stages a tile (column pair, G frames) of row spectra with bulk
//               copies, runs the column FFTs and restores the exact frame mean
//               by linearity on the way out:
//                 FFT2((I - mu) w m) = FFT2((I - c_f) w m) + (c_f - mu) FFT2(w m),
//               FFT2(w m) a host FP64 table (non-zero only at kx <= 3 and
//               |ky| <= 3 for the separable 4-term Blackman-Harris window
//               without a mask), the coefficient c_f - mu in FP64. The CTA
//               stores the G frames of a mode together: G consecutive ring
//               slots form one 32 B sector.
// Subtracting c_f keeps the FP32 transforms free of the large DC term (the
// cancellation the reference avoids with its (hi, lo) mean,
// ddm.wgsl:129-150); the correction term is the small (c_f - mu).
#include <cstdint>
#include <map>
#include <mutex>
#include <type_traits>
#include <utility>

#include "async_copy.cuh"
#include "fft_block.cuh"
#include "kernels.cuh"

namespace ddm {

template <typename Tin>
__device__ __forceinline__ float ld_pix(const Tin* p) {
  return (float)__ldg(p);
}

// The 2048-point rows and columns take the radix-16 plan (16 points per
// thread, 2048 = 16 x 16 x 8: three passes through shared memory instead of
// the radix-8 plan's four, two FFT groups of 128 threads per CTA, one
// in-place buffer per group).
#ifndef SPATIAL_R16
#define SPATIAL_R16 1
#endif
__host__ __device__ constexpr bool r16(int N) { return SPATIAL_R16 && N == 2048; }

// Points per thread of an N-point transform: 8 (radix-8 plan) for powers of
// two, 16 for the radix-16 plan, 24 (mixed radix, fft_p) for the sizes with a
// factor 3 (384, 768).
__host__ __device__ constexpr int pts(int N) { return r16(N) ? 16 : N % 3 == 0 ? 24 : 8; }

// Shared-memory index of point k of a transform's natural-order result.
template <int N>
__device__ __forceinline__ int padk(int k) {
  if constexpr (r16(N))
    return pad16(k);
  else
    return pad(k);
}

template <int N>
__host__ __device__ constexpr int row_groups() {
  return 256 / (N / pts(N)) >= 1 ? 256 / (N / pts(N)) : 1;
}

// twiddle table length and barrier scope of the plan of N
template <int N>
__host__ __device__ constexpr int tw_count() {
  return r16(N) ? tw_size16(N) : pts(N) == 8 ? tw_size(N) : tw_size_p(N);
}
template <int N>
__host__ __device__ constexpr int sync_of() {
  return sync_kind(8 * N / pts(N), row_groups<N>());  // groups of N/pts(N) threads
}

// Twiddles of the power-of-two row and column transforms by products of W^1
// (see SPARSE_TW_REC in temporal.cu). Measured at 512^2 x 1024: spatial stage
// 1.377 -> 1.355 ms per video, spectra within 2.3e-7 of a bin's scale of the
// table form.
#ifndef SPATIAL_TW_REC
#define SPATIAL_TW_REC 1
#endif

// The column / row transform of this size.
template <int N, bool INV, int SYNC>
__device__ __forceinline__ float2* fft_n(float2 (&v)[pts(N)], int t, float2* buf0, float2* buf1,
                                         const float2* __restrict__ tw, int bar_id) {
  if constexpr (r16(N)) {
    fft16<N, INV>(v, t, buf0, tw, bar_id);  // in place in the group's one buffer
    return buf0;
  } else if constexpr (pts(N) == 8) {
    return fft<N, INV, true, SYNC, SPATIAL_TW_REC>(v, t, buf0, buf1, tw, bar_id);
  } else {
    return fft_p<N, pts(N), INV, SYNC>(v, t, buf0, buf1, tw, bar_id);
  }
}
constexpr int ROW_STAGES = 2;  // depth of the row-batch staging ring

// float2 between the buffer pairs of consecutive FFT groups: two buffers
// plus a skew, so accesses that read the same index from several groups at
// once (the column kernel's stores, the row kernel's output loop) hit
// different banks. 4 float2 from N = 512 on, 2 below (where a warp spans
// groups inside the transforms); chosen by simulating every shared-memory
// access pattern of both kernels. Even, so the bulk-copy destinations after
// the groups stay 16-byte aligned.
template <int N>
__host__ __device__ constexpr int GSTRIDE() {
  return r16(N) ? N + 4 : 2 * padded(N) + (N >= 512 ? 4 : 2);  // the radix-16 plan: one buffer
}

// The pixels whose mean is a frame's reference level c_f: a 16 x 16 grid at
// the centres of N/16 x N/16 cells, pixel i of the 256 read by thread i. The
// closer c_f is to the frame mean, the smaller the offset the FP32
// transforms carry and the correction term (c_f - mu) FFT2(w m) has to
// cancel (the error of that cancellation grows with N).
constexpr int CREF = 256;
template <int N>
__device__ __forceinline__ int cref_offset(int i) {
  return ((2 * (i >> 4) + 1) * (N / 32)) * N + (2 * (i & 15) + 1) * (N / 32);
}

// Frame reference levels c_f of a chunk, one CTA per frame: the mean of the
// CREF grid pixels, warp sums added in a fixed order (the rows kernel reads
// the result for every batch of the frame).
template <int N, typename Tin>
__global__ void __launch_bounds__(CREF) cref_kernel(const Tin* __restrict__ frames, long long frame_stride,
                                                    float* __restrict__ framec) {
  constexpr bool INT = !std::is_floating_point<Tin>::value;
  using acc_t = typename std::conditional<INT, int, double>::type;
  __shared__ acc_t cred[CREF / 32];
  const long long f = blockIdx.x;
  acc_t c = (acc_t)__ldg(frames + f * frame_stride + cref_offset<N>(threadIdx.x));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) cred[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    acc_t sum = 0;
#pragma unroll
    for (int w = 0; w < CREF / 32; w++) sum += cred[w];
    framec[f] = (float)((double)sum * (1.0 / CREF));
  }
}

// Persistent: each CTA walks batches of G row pairs (2G consecutive rows of
// one frame; G divides N/2, so a batch never straddles frames). A batch (and
// the mask's matching rows) is staged into shared memory by bulk copies (TMA,
// cp.async.bulk) issued ROW_STAGES batches ahead into a ring, so raw pixels
// never sit in registers waiting and the copy engine, not the warps, moves
// them.
// CTAs per SM the radix-16 rows kernel's registers are bounded for: two (128
// registers, 12 B spilled) against one (158 registers). Measured at 2048^2
// with a pixel mask, spatial stage per frame: radix-8 plan 32.0 us, radix-16
// with one CTA per SM 30.0 us, with two 28.4 us; the history within 1.4e-6 of
// its RMS of the radix-8 plan's.
#ifndef ROWS16_MIN_BLOCKS
#define ROWS16_MIN_BLOCKS 2
#endif
template <int N>
__host__ __device__ constexpr int rows_min_blocks() {
  return r16(N) ? ROWS16_MIN_BLOCKS : 1;
}
template <int N, typename Tin>
__global__ void __launch_bounds__(256, rows_min_blocks<N>()) rows_kernel(RowParams p) {
  constexpr int P = pts(N);
  constexpr int NT = N / P;
  constexpr int G = row_groups<N>();
  constexpr int PN = padded(N);
  constexpr int NHB = (N / 2 + 1 + KB - 1) / KB;
  constexpr int WARPS = (G * NT + 31) / 32;
  constexpr int SYNC = sync_of<N>();
  constexpr int BPF = N / (2 * G);  // batches per frame
  constexpr uint32_t BATCH_ELEMS = 2u * G * N;
  constexpr uint32_t BATCH_BYTES = BATCH_ELEMS * sizeof(Tin);
  static_assert(BATCH_BYTES % 16 == 0 && BATCH_ELEMS % 16 == 0, "bulk copies move multiples of 16 bytes");
  extern __shared__ __align__(16) float2 sm[];
  __shared__ double red[WARPS];
  __shared__ __align__(8) uint64_t bar[ROW_STAGES];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  float2* buf0 = sm + (size_t)g * GSTRIDE<N>();
  float2* buf1 = buf0 + PN;
  float2* s_tw = sm + (size_t)G * GSTRIDE<N>();
  float* s_wy = (float*)(s_tw + tw_count<N>());                     // [N] w(y) scale
  Tin* ring = (Tin*)(s_wy + N);                                   // [ROW_STAGES][2G][N]
  uint8_t* mring = (uint8_t*)(ring + ROW_STAGES * BATCH_ELEMS);  // [ROW_STAGES][2G][N]
  for (int i = threadIdx.x; i < tw_count<N>(); i += blockDim.x) s_tw[i] = p.tw[i];
  for (int i = threadIdx.x; i < N; i += blockDim.x) s_wy[i] = p.wys[i];
  const long long nbatch = (long long)p.nframes * BPF;
  const Tin* frames = (const Tin*)p.frames;
  const bool masked = p.smask != nullptr;
  auto issue = [&](long long b, int st) {
    const long long f = b / BPF, r = b % BPF;
    mbar_arrive_expect_tx(&bar[st], BATCH_BYTES + (masked ? BATCH_ELEMS : 0u));
    bulk_g2s(ring + st * BATCH_ELEMS, frames + f * p.frame_stride + r * (long long)BATCH_ELEMS, BATCH_BYTES,
             &bar[st]);
    if (masked) bulk_g2s(mring + st * BATCH_ELEMS, p.smask + r * BATCH_ELEMS, BATCH_ELEMS, &bar[st]);
  };
  if (threadIdx.x == 0) {
    for (int s = 0; s < ROW_STAGES; s++) mbar_init(&bar[s], 1);
    fence_barrier_init();
    for (int s = 0; s < ROW_STAGES; s++) {
      const long long b = blockIdx.x + (long long)s * gridDim.x;
      if (b < nbatch) issue(b, s);
    }
  }
  float wxs[P];  // w(x) at this thread's columns, fixed for the whole kernel
#pragma unroll
  for (int q = 0; q < P; q++) wxs[q] = __ldg(&p.win[t + q * NT]);
  // pixel sums: exact integers for u8/u16 (warp totals < 2^31), FP64 for f32
  constexpr bool INT = !std::is_floating_point<Tin>::value;
  using acc_t = typename std::conditional<INT, int, double>::type;
  __syncthreads();  // barriers initialised, twiddles and w(y) in shared memory
  int it = 0;
  for (long long b = blockIdx.x; b < nbatch; b += gridDim.x, it++) {
    const int st = it % ROW_STAGES;
    const int f = (int)(b / BPF);
    const int r = (int)(b % BPF);
    const float cf = p.framec[f];  // cref_kernel, earlier on this stream
    if (!mbar_wait(&bar[st], (uint32_t)(it / ROW_STAGES) & 1u, p.err, 2)) {
      // give up: let this CTA's other copies in flight land (bounded), then stop
      if (threadIdx.x == 0)
        for (int k = 1; k < ROW_STAGES; k++)
          if (b + (long long)k * gridDim.x < nbatch)
            mbar_wait(&bar[(it + k) % ROW_STAGES], (uint32_t)((it + k) / ROW_STAGES) & 1u, nullptr, 0);
      return;
    }
    const int y0 = r * 2 * G + 2 * g;  // this group's row pair
    const Tin* r0 = ring + st * BATCH_ELEMS + 2 * g * N;
    const Tin* r1 = r0 + N;
    const uint8_t* m0p = mring + st * BATCH_ELEMS + 2 * g * N;
    const float wy0 = s_wy[y0], wy1 = s_wy[y0 + 1];
    float2 v[P];
    acc_t s = 0;
#pragma unroll
    for (int q = 0; q < P; q++) {
      const int x = t + q * NT;
      const float m0 = masked ? (float)m0p[x] : 1.f;
      const float m1 = masked ? (float)m0p[N + x] : 1.f;
      const float a0 = (float)r0[x] * m0, a1 = (float)r1[x] * m1;
      if constexpr (INT)
        s += (int)a0 + (int)a1;
      else
        s += (double)a0 + (double)a1;
      const float wx = wxs[q];
      v[q] = make_float2((a0 - cf * m0) * (wx * wy0), (a1 - cf * m1) * (wx * wy1));
    }
    fence_proxy_async_smem();  // this thread's reads of the stage before the next bulk write
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = (double)s;
    const float2* Z = fft_n<N, false, SYNC>(v, t, buf0, buf1, s_tw, 1 + g);
    __syncthreads();  // red[] and every group's row spectra complete; stage st is free
    if (threadIdx.x == 0) {
      const long long bn = b + (long long)ROW_STAGES * gridDim.x;
      if (bn < nbatch) issue(bn, st);
      double tot = 0.0;
#pragma unroll
      for (int w = 0; w < WARPS; w++) tot += red[w];
      atomicAdd(&p.framesum[f], tot);
    }
    // Row spectra out by the CTA as a whole: item (kx pair kb, row rr of the
    // batch) writes both kx of the pair, and consecutive items are
    // consecutive rows, so a warp writes whole sectors of the
    // [frame][kx/2][2][y] scratch (each column contiguous in y, as the column
    // kernel reads it). Row rr of the batch is the
    // real-input half (rr even: real part, odd: imaginary part) of group
    // rr/2's packed transform, split by Hermitian symmetry.
    {
      const int zoff = (int)(Z - (sm + (size_t)g * GSTRIDE<N>()));  // same in every group
      const int yb = r * 2 * G;
      float2* out = p.rows + (size_t)f * NHB * N * KB;
      for (int item = threadIdx.x; item < NHB * 2 * G; item += blockDim.x) {
        const int rr = item % (2 * G), kb = item / (2 * G);
        const float2* Zg = sm + (size_t)(rr >> 1) * GSTRIDE<N>() + zoff;
        float2 R[KB];
#pragma unroll
        for (int c = 0; c < KB; c++) {
          const int kx = kb * KB + c;
          const float2 zk = Zg[padk<N>(kx < N ? kx : 0)];
          const float2 zn = Zg[padk<N>((N - kx) % N)];
          R[c] = (rr & 1) ? make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x))
                          : make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
          if (kx > N / 2) R[c] = make_float2(0.f, 0.f);  // past the half plane
        }
#pragma unroll
        for (int c = 0; c < KB; c++) out[((size_t)kb * KB + c) * N + yb + rr] = R[c];
      }
    }
    __syncthreads();  // buffers and red[] are reused by the next batch
  }
}

// Persistent: each CTA walks tiles (column pair kb, group of G frames). The
// tile's G row-spectrum blocks ([KB][y] float2, contiguous per frame) are
// staged into shared memory by bulk copies; the next tile's copies are
// issued as soon as every thread has read the current one, so they overlap
// the second column's transform and the history stores. Group g transforms
// frame f0 + g; the CTA then writes frame sf = tid % G of each mode, so G
// consecutive ring slots of a mode leave together (one 32 B sector at G = 4),
// adding the mean correction (c_f - mu) FFT2(w m)(ky, kx) on the way.
// Paired stores: a full tile whose frames go to slot pairs (2s, 2s + 1) --
// the usual case, consecutive frames into consecutive slots -- stores two
// frames of a mode with one 16-byte store. Measured at 512^2 x 1024: spatial
// stage 1.477 -> 1.369 ms per video, the history bit for bit the same.
#ifndef COLS_PAIRED
#define COLS_PAIRED 1
#endif
// CTAs per SM the power-of-two column kernels' registers are bounded for
// (the mixed-radix 384 and 768 would spill under a bound of 3). Measured at
// 512^2 x 1024: unbounded (126 registers, 2 CTAs per SM) 1.383 ms per video,
// bounded to 3 CTAs (80 registers, no spills) 1.393 ms.
#ifndef COLS_MIN_BLOCKS
#define COLS_MIN_BLOCKS 1
#endif
template <int N>
__host__ __device__ constexpr int cols_min_blocks() {
  return pts(N) == 8 ? COLS_MIN_BLOCKS : 1;
}
template <int N>
__global__ void __launch_bounds__(256, cols_min_blocks<N>()) cols_kernel(ColParams p) {
  constexpr int P = pts(N);
  constexpr int NT = N / P;
  constexpr int G = row_groups<N>();  // frames per tile, one per group
  constexpr int PN = padded(N);
  constexpr int SYNC = sync_of<N>();
  constexpr uint32_t FRAME_ELEMS = N * KB;  // float2 of one frame's block
  constexpr uint32_t FRAME_BYTES = FRAME_ELEMS * sizeof(float2);
  extern __shared__ __align__(16) float2 sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ float s_dc[G];  // (c_f - mu) scale / N per frame of the tile
  __shared__ float2 s_wc4[4];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  float2* buf0 = sm + (size_t)g * GSTRIDE<N>();
  float2* buf1 = buf0 + PN;
  float2* s_tw = sm + (size_t)G * GSTRIDE<N>();
  float2* stage = s_tw + tw_count<N>();  // [G][KB][N]
  for (int i = threadIdx.x; i < tw_count<N>(); i += blockDim.x) s_tw[i] = p.tw[i];
  if (threadIdx.x < 4) s_wc4[threadIdx.x] = p.wc4[threadIdx.x];
  const int nfg = (p.nframes + G - 1) / G;
  const int NKB = p.nkb > 0 ? p.nkb : p.NHB, kb0 = p.kb0;  // the column blocks of the history band
  const int W = p.hist_w > 0 ? p.hist_w : p.NH;            // columns per history row
  const int ntiles = NKB * nfg;
  const float invN = 1.f / N;
  const int sf = threadIdx.x % G;  // frame of the tile this thread stores
  const double inv_total = p.inv_total[0];
  auto issue = [&](int tile) {
    const int kb = kb0 + tile % NKB, f0 = (tile / NKB) * G;
    const int nf = min(G, p.nframes - f0);
    mbar_arrive_expect_tx(&bar, nf * FRAME_BYTES);
    for (int i = 0; i < nf; i++)
      bulk_g2s(stage + i * FRAME_ELEMS, p.rows + ((size_t)(f0 + i) * p.NHB + kb) * FRAME_ELEMS, FRAME_BYTES,
               &bar);
  };
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_barrier_init();
    if (blockIdx.x < ntiles) issue(blockIdx.x);
  }
  __syncthreads();
  uint32_t phase = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int kb = kb0 + tile % NKB;
    const int f0 = (tile / NKB) * G;
    const int nf = min(G, p.nframes - f0);
    if (threadIdx.x < nf) {
      const int f = f0 + threadIdx.x;
      const double mu = p.framesum[f] * inv_total;
      s_dc[threadIdx.x] = (float)(((double)p.framec[f] - mu) * (double)p.scale / N);
      if (kb == kb0) p.means[f] = mu * (double)p.scale;
    }
    if (!mbar_wait(&bar, phase, p.err, 3)) return;  // nothing else is in flight
    phase ^= 1u;
    const int slot = sf < nf ? p.slots[f0 + sf] : 0;
    const bool fvalid = g < nf;
    // a full tile whose frames go to slot pairs (2s, 2s + 1): each thread
    // stores two frames of a mode with one 16-byte store
    bool paired = COLS_PAIRED && (G % 2 == 0) && nf == G;
    if (paired)
      for (int j = 0; j < G / 2; j++) {
        const int s0 = p.slots[f0 + 2 * j];
        paired = paired && !(s0 & 1) && p.slots[f0 + 2 * j + 1] == s0 + 1;
      }
    const float2* blk = stage + g * FRAME_ELEMS;
#pragma unroll 1
    for (int c = 0; c < KB; c++) {
      const int kx = kb * KB + c;
      if (kx >= p.NH) break;  // uniform over the CTA
      float2 v[P];
#pragma unroll
      for (int q = 0; q < P; q++) v[q] = fvalid ? blk[c * N + t + q * NT] : make_float2(0.f, 0.f);
      if (c == KB - 1 || kx + 1 >= p.NH) {
        // every thread has read the stage: the next tile's copies may land
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0 && tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x);
      }
      // this thread's 8 output modes of the correction table, loaded now so
      // the column transform hides their latency
      constexpr int KYS = 256 / G;  // ky stride of the store loop
      constexpr int GP = G >= 2 ? G / 2 : 1;  // frame pairs of a tile
      constexpr int KYS2 = 2 * KYS;  // ky stride of the paired store loop
      float2 wreg[N / KYS];
      if (p.w2d) {
        if (paired) {
#pragma unroll
          for (int i = 0; i < N / KYS2; i++)
            wreg[i] = __ldg(&p.w2d[(size_t)kx * N + threadIdx.x / GP + i * KYS2]);
        } else {
#pragma unroll
          for (int i = 0; i < N / KYS; i++) wreg[i] = __ldg(&p.w2d[(size_t)kx * N + threadIdx.x / G + i * KYS]);
        }
      }
      const float2* Y = fft_n<N, false, SYNC>(v, t, buf0, buf1, s_tw, 1 + g);
      __syncthreads();  // every group's column (and s_dc) is in shared memory
      // Y of group g sits at the same offset in every group's buffer pair; the
      // CTA writes frame sf = tid % G of each mode: G consecutive ring slots
      if (paired) {
        const int pj = threadIdx.x % GP;
        const int yoff = (int)(Y - (sm + (size_t)g * GSTRIDE<N>()));
        const float2* ys0 = sm + (size_t)(2 * pj) * GSTRIDE<N>() + yoff;
        const float2* ys1 = ys0 + GSTRIDE<N>();
        float4* hs = reinterpret_cast<float4*>(p.hist + (size_t)(kx - kb0 * KB) * p.T + p.slots[f0 + 2 * pj]);
        const size_t mstride = (size_t)W * p.T / 2;  // float4 units (T even)
        const float dc0 = s_dc[2 * pj], dc1 = s_dc[2 * pj + 1];
        const float2 wkx = kx < 4 ? s_wc4[kx] : make_float2(0.f, 0.f);
#pragma unroll
        for (int i = 0; i < N / KYS2; i++) {
          const int ky = threadIdx.x / GP + i * KYS2;
          const float2 y0 = ys0[pad(ky)], y1 = ys1[pad(ky)];
          float2 w = make_float2(0.f, 0.f);
          if (p.w2d) {
            w = wreg[i];
          } else if (kx < 4 && (ky < 4 || ky > N - 4)) {
            const float2 wk = ky < 4 ? s_wc4[ky] : make_float2(s_wc4[N - ky].x, -s_wc4[N - ky].y);
            w = cmul(wkx, wk);
          }
          hs[(size_t)ky * mstride] = make_float4(fmaf(dc0, w.x, y0.x * invN), fmaf(dc0, w.y, y0.y * invN),
                                                 fmaf(dc1, w.x, y1.x * invN), fmaf(dc1, w.y, y1.y * invN));
        }
      } else if (sf < nf) {
        const int yoff = (int)(Y - (sm + (size_t)g * GSTRIDE<N>()));
        const float2* ys = sm + (size_t)sf * GSTRIDE<N>() + yoff;
        float2* hs = p.hist + (size_t)(kx - kb0 * KB) * p.T + slot;
        const size_t mstride = (size_t)W * p.T;
        const float dc = s_dc[sf];
        const float2 wkx = kx < 4 ? s_wc4[kx] : make_float2(0.f, 0.f);
#pragma unroll
        for (int i = 0; i < N / KYS; i++) {
          const int ky = threadIdx.x / G + i * KYS;
          const float2 y = ys[pad(ky)];
          float2 w = make_float2(0.f, 0.f);
          if (p.w2d) {
            w = wreg[i];
          } else if (kx < 4 && (ky < 4 || ky > N - 4)) {
            // separable window: W(kx) W(ky), W(N - k) = conj W(k)
            const float2 wk = ky < 4 ? s_wc4[ky] : make_float2(s_wc4[N - ky].x, -s_wc4[N - ky].y);
            w = cmul(wkx, wk);
          }
          hs[(size_t)ky * mstride] = make_float2(fmaf(dc, w.x, y.x * invN), fmaf(dc, w.y, y.y * invN));
        }
      }
      __syncthreads();
    }
  }
}

// Column pass for N >= 1024, where fewer than four FFT groups of N/8 threads
// fit a CTA. A tile is (column pair kb, four frames): the frames' row-spectrum
// blocks stream through a two-deep ring of bulk copies (one block per group
// at a time, G frames per ring entry), each group transforms both columns of
// its frame into the tile's output slabs R[c][frame] (the transform's last
// ping-pong buffer), and the CTA then stores four consecutive ring slots of a
// mode together -- one full 32 B sector. With one frame per tile every
// history store covered a quarter sector and the memory controller had to
// read-modify-write it (about 4x the algorithmic DRAM traffic at N = 2048).
constexpr int WIDE_F = 4;  // frames per tile of the wide column kernel

template <int N>
__global__ void __launch_bounds__(256, 1) cols_wide_kernel(ColParams p) {
  constexpr int NT = N / 8;
  constexpr int G = row_groups<N>();  // 1 (N = 2048) or 2 (N = 1024)
  constexpr int F = WIDE_F;
  constexpr int SYNC = sync_kind(N, G);
  constexpr uint32_t FRAME_ELEMS = N * KB;
  constexpr uint32_t FRAME_BYTES = FRAME_ELEMS * sizeof(float2);
  constexpr uint32_t ITEM_ELEMS = G * FRAME_ELEMS;
  static_assert(F % G == 0, "groups divide the tile's frames");
  static_assert((fft_stages(N) & 1) == 0, "the transform must end in its second buffer (the output slab)");
  extern __shared__ __align__(16) float2 sm[];
  float2* ring = sm;                   // [2][G][KB][N] staged blocks
  float2* R = ring + 2 * ITEM_ELEMS;   // [KB][F][N] column transforms of the tile
  float2* scr = R + KB * F * N;        // [G][N] first ping-pong buffer of each group
  float2* s_tw = scr + G * N;
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ float s_dc[F];
  __shared__ float2 s_wc4[4];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  for (int i = threadIdx.x; i < tw_size(N); i += blockDim.x) s_tw[i] = p.tw[i];
  if (threadIdx.x < 4) s_wc4[threadIdx.x] = p.wc4[threadIdx.x];
  const int nfg = (p.nframes + F - 1) / F;
  const int NKB = p.nkb > 0 ? p.nkb : p.NHB, kb0 = p.kb0;  // the column blocks of the history band
  const int W = p.hist_w > 0 ? p.hist_w : p.NH;            // columns per history row
  const int ntiles = NKB * nfg;
  const float invN = 1.f / N;
  const double inv_total = p.inv_total[0];
  // item (tile, j): frames f0 + j*G .. f0 + j*G + G - 1 of the tile (those < nframes)
  auto items_of = [&](int tile) {
    const int f0 = (tile / NKB) * F;
    return (min(F, p.nframes - f0) + G - 1) / G;
  };
  auto issue = [&](int tile, int j, int s) {
    const int kb = kb0 + tile % NKB, f0 = (tile / NKB) * F + j * G;
    const int nf = min(G, p.nframes - f0);
    mbar_arrive_expect_tx(&bar[s], nf * FRAME_BYTES);
    for (int i = 0; i < nf; i++)
      bulk_g2s(ring + s * ITEM_ELEMS + i * FRAME_ELEMS,
               p.rows + ((size_t)(f0 + i) * p.NHB + kb) * FRAME_ELEMS, FRAME_BYTES, &bar[s]);
  };
  // the item after (tile, j) in this CTA's sequence
  auto advance = [&](int& tile, int& j) {
    if (++j >= items_of(tile)) {
      j = 0;
      tile += gridDim.x;
    }
  };
  // thread 0 keeps the issue cursor two items ahead of the consumer
  int it_tile = blockIdx.x, it_j = 0;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
    for (int s = 0; s < 2 && it_tile < ntiles; s++) {
      issue(it_tile, it_j, s);
      advance(it_tile, it_j);
    }
  }
  __syncthreads();
  int e = 0;  // items consumed by this CTA
  constexpr int SPT = 256 / F;  // ky stride of the store loop
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int kb = kb0 + tile % NKB;
    const int f0 = (tile / NKB) * F;
    const int nf = min(F, p.nframes - f0);
    if (threadIdx.x < nf) {
      const int f = f0 + threadIdx.x;
      const double mu = p.framesum[f] * inv_total;
      s_dc[threadIdx.x] = (float)(((double)p.framec[f] - mu) * (double)p.scale / N);
      if (kb == kb0) p.means[f] = mu * (double)p.scale;
    }
    if (p.w2d && threadIdx.x == 0) {
      // the correction rows of this tile's columns, read by the store loop
      // after the transforms: into L2 now (one bulk prefetch), so those reads
      // do not wait on DRAM
      const int ncol = min(KB, p.NH - kb * KB);
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p.w2d + (size_t)kb * KB * N),
                   "r"((uint32_t)(ncol * N * sizeof(float2)))
                   : "memory");
    }
    const int nit = (nf + G - 1) / G;
    for (int j = 0; j < nit; j++, e++) {
      const int s = e & 1;
      if (!mbar_wait(&bar[s], (uint32_t)(e >> 1) & 1u, p.err, 3)) {
        // give up: let the other copy in flight land (bounded), then stop
        mbar_wait(&bar[s ^ 1], (uint32_t)((e + 1) >> 1) & 1u, nullptr, 0);
        return;
      }
      const int fi = j * G + g;  // this group's frame within the tile
      const bool fvalid = fi < nf;
      const float2* blk = ring + s * ITEM_ELEMS + g * FRAME_ELEMS;
#pragma unroll 1
      for (int c = 0; c < KB; c++) {
        float2 v[8];
#pragma unroll
        for (int q = 0; q < 8; q++) v[q] = fvalid ? blk[c * N + t + q * NT] : make_float2(0.f, 0.f);
        if (c == KB - 1) {
          // every thread has read ring entry s: its next copy may land
          fence_proxy_async_smem();
          __syncthreads();
          if (threadIdx.x == 0 && it_tile < ntiles) {
            issue(it_tile, it_j, s);
            advance(it_tile, it_j);
          }
        }
        fft<N, false, true, SYNC, SPATIAL_TW_REC>(v, t, scr + g * N, R + (size_t)(c * F + fi) * N, s_tw, 1 + g);
      }
    }
    __syncthreads();  // R and s_dc complete
    // store: thread -> (frame sf, ky); lanes 4k..4k+3 write one mode's four slots
    const int sf = threadIdx.x % F;
    if (sf < nf) {
      const int slot = p.slots[f0 + sf];
      const float dc = s_dc[sf];
      const size_t mstride = (size_t)W * p.T;
#pragma unroll 1
      for (int c = 0; c < KB; c++) {
        const int kx = kb * KB + c;
        if (kx >= p.NH) break;
        const float2* ys = R + (size_t)(c * F + sf) * N;
        float2* hs = p.hist + (size_t)(kx - kb0 * KB) * p.T + slot;
        const float2 wkx = kx < 4 ? s_wc4[kx] : make_float2(0.f, 0.f);
        if (p.w2d) {
          // correction table loads run one batch of WB ahead of the stores
          constexpr int WB = 8, NI = N / SPT;
          static_assert(NI % WB == 0, "store batches");
          const float2* wcol = p.w2d + (size_t)kx * N + threadIdx.x / F;
          float2 wcur[WB], wnxt[WB];
#pragma unroll
          for (int j = 0; j < WB; j++) wcur[j] = __ldg(&wcol[j * SPT]);
#pragma unroll 1
          for (int i0 = 0; i0 < NI; i0 += WB) {
            if (i0 + WB < NI)
#pragma unroll
              for (int j = 0; j < WB; j++) wnxt[j] = __ldg(&wcol[(i0 + WB + j) * SPT]);
#pragma unroll
            for (int j = 0; j < WB; j++) {
              const int ky = threadIdx.x / F + (i0 + j) * SPT;
              const float2 y = ys[pad(ky)];
              const float2 w = wcur[j];
              hs[(size_t)ky * mstride] = make_float2(fmaf(dc, w.x, y.x * invN), fmaf(dc, w.y, y.y * invN));
            }
#pragma unroll
            for (int j = 0; j < WB; j++) wcur[j] = wnxt[j];
          }
        } else {
#pragma unroll 8
          for (int i = 0; i < N / SPT; i++) {
            const int ky = threadIdx.x / F + i * SPT;
            const float2 y = ys[pad(ky)];
            float2 w = make_float2(0.f, 0.f);
            if (kx < 4 && (ky < 4 || ky > N - 4)) {
              const float2 wk = ky < 4 ? s_wc4[ky] : make_float2(s_wc4[N - ky].x, -s_wc4[N - ky].y);
              w = cmul(wkx, wk);
            }
            hs[(size_t)ky * mstride] = make_float2(fmaf(dc, w.x, y.x * invN), fmaf(dc, w.y, y.y * invN));
          }
        }
      }
    }
    __syncthreads();  // R and s_dc are rewritten by the next tile
  }
}

// Column pass for the radix-16 plan (N = 2048): the same tiles (column pair
// kb, WIDE_F frames) and stores as cols_wide_kernel, with two FFT groups of
// N/16 threads. An item is one frame's [KB][N] block, staged by one bulk copy
// into a two-deep ring; group g transforms column g of the pair in place in
// its output slab R[g][frame], so the CTA runs both columns of a frame at once
// (one group idles on a lone last column, kx = N/2).
template <int N>
__global__ void __launch_bounds__(256, 1) cols_wide16_kernel(ColParams p) {
  constexpr int NT = N / 16;
  constexpr int F = WIDE_F;
  constexpr uint32_t FRAME_ELEMS = N * KB;
  constexpr uint32_t FRAME_BYTES = FRAME_ELEMS * sizeof(float2);
  static_assert(2 * NT == 256 && KB == 2, "one group per column of the pair");
  extern __shared__ __align__(16) float2 sm[];
  float2* ring = sm;                  // [2][KB][N] staged blocks, one frame each
  float2* R = ring + 2 * FRAME_ELEMS;  // [KB][F][N] column transforms of the tile
  float2* s_tw = R + KB * F * N;
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ float s_dc[F];
  __shared__ float2 s_wc4[4];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  for (int i = threadIdx.x; i < tw_size16(N); i += blockDim.x) s_tw[i] = p.tw[i];
  if (threadIdx.x < 4) s_wc4[threadIdx.x] = p.wc4[threadIdx.x];
  const int nfg = (p.nframes + F - 1) / F;
  const int NKB = p.nkb > 0 ? p.nkb : p.NHB, kb0 = p.kb0;  // the column blocks of the history band
  const int W = p.hist_w > 0 ? p.hist_w : p.NH;            // columns per history row
  const int ntiles = NKB * nfg;
  const float invN = 1.f / N;
  const double inv_total = p.inv_total[0];
  auto items_of = [&](int tile) { return min(F, p.nframes - (tile / NKB) * F); };
  auto issue = [&](int tile, int j, int s) {
    const int kb = kb0 + tile % NKB, f = (tile / NKB) * F + j;
    mbar_arrive_expect_tx(&bar[s], FRAME_BYTES);
    bulk_g2s(ring + s * FRAME_ELEMS, p.rows + ((size_t)f * p.NHB + kb) * FRAME_ELEMS, FRAME_BYTES, &bar[s]);
  };
  auto advance = [&](int& tile, int& j) {
    if (++j >= items_of(tile)) {
      j = 0;
      tile += gridDim.x;
    }
  };
  // thread 0 keeps the issue cursor two items ahead of the consumer
  int it_tile = blockIdx.x, it_j = 0;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
    for (int s = 0; s < 2 && it_tile < ntiles; s++) {
      issue(it_tile, it_j, s);
      advance(it_tile, it_j);
    }
  }
  __syncthreads();
  int e = 0;  // items consumed by this CTA
  constexpr int SPT = 256 / F;  // ky stride of the store loop
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int kb = kb0 + tile % NKB;
    const int f0 = (tile / NKB) * F;
    const int nf = min(F, p.nframes - f0);
    const bool col_ok = kb * KB + g < p.NH;  // the last block holds one column
    if (threadIdx.x < nf) {
      const int f = f0 + threadIdx.x;
      const double mu = p.framesum[f] * inv_total;
      s_dc[threadIdx.x] = (float)(((double)p.framec[f] - mu) * (double)p.scale / N);
      if (kb == kb0) p.means[f] = mu * (double)p.scale;
    }
    if (p.w2d && threadIdx.x == 0) {
      // the correction rows of this tile's columns into L2 ahead of the stores
      const int ncol = min(KB, p.NH - kb * KB);
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p.w2d + (size_t)kb * KB * N),
                   "r"((uint32_t)(ncol * N * sizeof(float2)))
                   : "memory");
    }
    for (int fi = 0; fi < nf; fi++, e++) {
      const int s = e & 1;
      if (!mbar_wait(&bar[s], (uint32_t)(e >> 1) & 1u, p.err, 3)) {
        // give up: let the other copy in flight land (bounded), then stop
        mbar_wait(&bar[s ^ 1], (uint32_t)((e + 1) >> 1) & 1u, nullptr, 0);
        return;
      }
      float2 v[16];
      const float2* col = ring + s * FRAME_ELEMS + g * N;
#pragma unroll
      for (int q = 0; q < 16; q++) v[q] = col_ok ? col[t + q * NT] : make_float2(0.f, 0.f);
      // every thread has read ring entry s: its next copy may land
      fence_proxy_async_smem();
      __syncthreads();
      if (threadIdx.x == 0 && it_tile < ntiles) {
        issue(it_tile, it_j, s);
        advance(it_tile, it_j);
      }
      fft16<N, false>(v, t, R + (size_t)(g * F + fi) * N, s_tw, 1 + g);
    }
    __syncthreads();  // R and s_dc complete
    // store: thread -> (frame sf, ky); lanes 4k..4k+3 write one mode's four slots
    const int sf = threadIdx.x % F;
    if (sf < nf) {
      const int slot = p.slots[f0 + sf];
      const float dc = s_dc[sf];
      const size_t mstride = (size_t)W * p.T;
#pragma unroll 1
      for (int c = 0; c < KB; c++) {
        const int kx = kb * KB + c;
        if (kx >= p.NH) break;
        const float2* ys = R + (size_t)(c * F + sf) * N;
        float2* hs = p.hist + (size_t)(kx - kb0 * KB) * p.T + slot;
        const float2 wkx = kx < 4 ? s_wc4[kx] : make_float2(0.f, 0.f);
        if (p.w2d) {
          // correction table loads run one batch of WB ahead of the stores
          constexpr int WB = 8, NI = N / SPT;
          static_assert(NI % WB == 0, "store batches");
          const float2* wcol = p.w2d + (size_t)kx * N + threadIdx.x / F;
          float2 wcur[WB], wnxt[WB];
#pragma unroll
          for (int j = 0; j < WB; j++) wcur[j] = __ldg(&wcol[j * SPT]);
#pragma unroll 1
          for (int i0 = 0; i0 < NI; i0 += WB) {
            if (i0 + WB < NI)
#pragma unroll
              for (int j = 0; j < WB; j++) wnxt[j] = __ldg(&wcol[(i0 + WB + j) * SPT]);
#pragma unroll
            for (int j = 0; j < WB; j++) {
              const int ky = threadIdx.x / F + (i0 + j) * SPT;
              const float2 y = ys[pad16(ky)];
              const float2 w = wcur[j];
              hs[(size_t)ky * mstride] = make_float2(fmaf(dc, w.x, y.x * invN), fmaf(dc, w.y, y.y * invN));
            }
#pragma unroll
            for (int j = 0; j < WB; j++) wcur[j] = wnxt[j];
          }
        } else {
#pragma unroll 8
          for (int i = 0; i < N / SPT; i++) {
            const int ky = threadIdx.x / F + i * SPT;
            const float2 y = ys[pad16(ky)];
            float2 w = make_float2(0.f, 0.f);
            if (kx < 4 && (ky < 4 || ky > N - 4)) {
              const float2 wk = ky < 4 ? s_wc4[ky] : make_float2(s_wc4[N - ky].x, -s_wc4[N - ky].y);
              w = cmul(wkx, wk);
            }
            hs[(size_t)ky * mstride] = make_float2(fmaf(dc, w.x, y.x * invN), fmaf(dc, w.y, y.y * invN));
          }
        }
      }
    }
    __syncthreads();  // R and s_dc are rewritten by the next tile
  }
}

// ------------------------------------------------------------------ launchers

template <int N>
static constexpr int groups() {
  return row_groups<N>();
}

template <int N>
static size_t fft_smem() {
  return ((size_t)groups<N>() * GSTRIDE<N>() + tw_count<N>()) * sizeof(float2);
}

// One wave of persistent CTAs. The occupancy query and the shared-memory
// opt-in are made once per kernel and device (they cost more host time than
// the launch itself).
template <typename K>
static int persistent_grid(K k, int threads, size_t smem, long long work) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> waves;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_pair((const void*)k, dev);
  int g = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    auto it = waves.find(key);
    if (it != waves.end()) g = it->second;
  }
  if (g <= 0) {
    int sms = 0, per = 0;
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, threads, smem);
    g = sms * (per > 0 ? per : 1);
    std::lock_guard<std::mutex> lk(mu);
    waves[key] = g;
  }
  return (int)(work < g ? (work > 0 ? work : 1) : g);
}

template <int N, typename Tin>
static cudaError_t rows_n(const RowParams& p, cudaStream_t s) {
  constexpr int G = groups<N>();
  const long long npairs = (long long)p.nframes * (N / 2);
  auto k = rows_kernel<N, Tin>;
  const size_t sm = fft_smem<N>() + N * sizeof(float) + (size_t)ROW_STAGES * 2 * G * N * (sizeof(Tin) + 1);
  const int grid = persistent_grid(k, G * (N / pts(N)), sm, (npairs + G - 1) / G);
  if (p.nframes > 0 && !p.framec_ready)
    cref_kernel<N, Tin><<<p.nframes, CREF, 0, s>>>((const Tin*)p.frames, p.frame_stride, p.framec);
  k<<<grid, G * (N / pts(N)), sm, s>>>(p);
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

template <int N>
static cudaError_t cref_n(int dtype, const void* frames, long long stride, int n, float* framec, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  switch (dtype) {
    case 0: cref_kernel<N, uint8_t><<<n, CREF, 0, s>>>((const uint8_t*)frames, stride, framec); break;
    case 1: cref_kernel<N, uint16_t><<<n, CREF, 0, s>>>((const uint16_t*)frames, stride, framec); break;
    case 2: cref_kernel<N, float><<<n, CREF, 0, s>>>((const float*)frames, stride, framec); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_cref(int N, int dtype, const void* frames, long long stride, int n, float* framec,
                        cudaStream_t s) {
  switch (N) {
    case 64: return cref_n<64>(dtype, frames, stride, n, framec, s);
    case 128: return cref_n<128>(dtype, frames, stride, n, framec, s);
    case 256: return cref_n<256>(dtype, frames, stride, n, framec, s);
    case 384: return cref_n<384>(dtype, frames, stride, n, framec, s);
    case 512: return cref_n<512>(dtype, frames, stride, n, framec, s);
    case 768: return cref_n<768>(dtype, frames, stride, n, framec, s);
    case 1024: return cref_n<1024>(dtype, frames, stride, n, framec, s);
    case 2048: return cref_n<2048>(dtype, frames, stride, n, framec, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_rows(int N, int dtype, const RowParams& p, cudaStream_t s) {
  switch (N) {
    case 64: return rows_dt<64>(dtype, p, s);
    case 128: return rows_dt<128>(dtype, p, s);
    case 256: return rows_dt<256>(dtype, p, s);
    case 384: return rows_dt<384>(dtype, p, s);
    case 512: return rows_dt<512>(dtype, p, s);
    case 768: return rows_dt<768>(dtype, p, s);
    case 1024: return rows_dt<1024>(dtype, p, s);
    case 2048: return rows_dt<2048>(dtype, p, s);
    default: return cudaErrorInvalidValue;
  }
}

// the wide column kernel (four frames per tile) where fewer than four FFT
// groups fit a CTA
__host__ __device__ constexpr bool use_wide_cols(int N) { return N >= 1024; }

template <int N>
static size_t cols_wide_smem() {
  if constexpr (r16(N)) {  // ring of two one-frame blocks, the tile's slabs, radix-16 twiddles
    return ((size_t)2 * N * KB + (size_t)KB * WIDE_F * N + tw_size16(N)) * sizeof(float2);
  } else {
    constexpr int G = groups<N>();
    return ((size_t)2 * G * N * KB + (size_t)KB * WIDE_F * N + (size_t)G * N + tw_size(N)) * sizeof(float2);
  }
}

template <int N>
static cudaError_t cols_n(const ColParams& p, cudaStream_t s) {
  constexpr int G = groups<N>();
  const long long wide_tiles = (long long)(p.nkb > 0 ? p.nkb : p.NHB) * ((p.nframes + WIDE_F - 1) / WIDE_F);
  if constexpr (r16(N)) {
    auto k = cols_wide16_kernel<N>;
    const size_t sm = cols_wide_smem<N>();
    const int grid = persistent_grid(k, 256, sm, wide_tiles);
    k<<<grid, 256, sm, s>>>(p);
    return cudaGetLastError();
  } else if constexpr (use_wide_cols(N)) {
    auto k = cols_wide_kernel<N>;
    const size_t sm = cols_wide_smem<N>();
    const int grid = persistent_grid(k, G * (N / 8), sm, wide_tiles);
    k<<<grid, G * (N / pts(N)), sm, s>>>(p);
    return cudaGetLastError();
  } else {
    auto k = cols_kernel<N>;
    const size_t sm = fft_smem<N>() + (size_t)G * N * KB * sizeof(float2);
    const int grid = persistent_grid(k, G * (N / pts(N)), sm, (long long)(p.nkb > 0 ? p.nkb : p.NHB) * ((p.nframes + G - 1) / G));
    k<<<grid, G * (N / pts(N)), sm, s>>>(p);
    return cudaGetLastError();
  }
}

int spatial_twiddle_radix(int N) { return N == 2048 && r16(2048) ? 16 : 8; }

cudaError_t launch_cols(int N, const ColParams& p, cudaStream_t s) {
  switch (N) {
    case 64: return cols_n<64>(p, s);
    case 128: return cols_n<128>(p, s);
    case 256: return cols_n<256>(p, s);
    case 384: return cols_n<384>(p, s);
    case 512: return cols_n<512>(p, s);
    case 768: return cols_n<768>(p, s);
    case 1024: return cols_n<1024>(p, s);
    case 2048: return cols_n<2048>(p, s);
    default: return cudaErrorInvalidValue;
  }
}

int frames_per_col_cta(int N) { return use_wide_cols(N) ? WIDE_F : 256 / (N / pts(N)); }

}  // namespace ddm
