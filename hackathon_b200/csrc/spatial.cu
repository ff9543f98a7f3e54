// Per-frame windowed half-plane 2D FFT into the mode-major history ring.
//
// Reference semantics (motility-ddm/src/fft.js:149-183, ddm.wgsl:134-192,
// ddm_ref.js:196-206): subtract the frame mean, multiply by w(x) w(y), 2D FFT,
// keep kx = 0..N/2, scale by 1/N, store mode m = ky*NH + kx at
// hist[m*T + slot].
//
// B200 formulation, two kernels per group of frames:
//  rows_kernel  reads raw u8/u16/f32 pixels (the int->FP32 convert and the
//               luma scale are fused into the load), subtracts each ROW's own
//               mean (exact: FP64 row sums of the raw integers), windows, and
//               transforms two rows per complex FFT (real-input packing). It
//               writes the row spectra to an L2-resident scratch in a
//               [frame][kx/2][y][2] blocked layout (full 32 B sectors) plus
//               the FP64 row sums.
//  cols_kernel  recovers the FRAME mean from the row sums and restores it
//               exactly by linearity: (I - mu) = (I - c_y) + (c_y - mu), so
//               the row spectrum gains (c_y - mu) * scale * w(y) * W(kx), where
//               W is the window's DFT (non-zero only for kx <= 3 of the
//               4-term Blackman-Harris). It then runs the column FFTs, scales
//               by 1/N and stores FG consecutive frames of a mode together,
//               so ring slots s..s+3 of one mode form one 32 B sector.
// Centering each row on its own mean keeps the FP32 row transform free of the
// large DC term (the cancellation the reference avoids with its (hi, lo) mean,
// ddm.wgsl:129-150); the correction term is small and computed in FP64.
#include <cstdint>

#include "fft_block.cuh"
#include "kernels.cuh"

namespace ddm {

template <typename Tin>
__device__ __forceinline__ float ld_pix(const Tin* p) {
  return (float)__ldg(p);
}

// Sum of a double over the NT threads of an FFT group (NT a power of two).
// Groups of >= 32 threads combine warp sums through `red` (per group).
template <int NT>
__device__ __forceinline__ double group_sum(double v, double* red, int t) {
  constexpr int W = NT < 32 ? NT : 32;
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o, W);
  if constexpr (NT > 32) {
    if ((t & 31) == 0) red[t >> 5] = v;
    __syncthreads();
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < NT / 32; w++) s += red[w];
    __syncthreads();
    return s;
  } else {
    return v;
  }
}

template <int N, typename Tin>
__global__ void __launch_bounds__(256) rows_kernel(RowParams p) {
  constexpr int NT = N / 8;
  constexpr int G = 256 / NT >= 1 ? 256 / NT : 1;
  constexpr int PN = padded(N);
  constexpr int NHB = (N / 2 + 1 + KB - 1) / KB;
  extern __shared__ float2 sm[];
  __shared__ double red[G][2][NT > 32 ? NT / 32 : 1];
  const int g = threadIdx.x / NT, t = threadIdx.x % NT;
  float2* buf0 = sm + (size_t)g * 2 * PN;
  float2* buf1 = buf0 + PN;
  const long long pair = (long long)blockIdx.x * G + g;
  const long long npairs = (long long)p.nframes * (N / 2);
  const bool valid = pair < npairs;
  const int f = valid ? (int)(pair / (N / 2)) : 0;
  const int y0 = valid ? 2 * (int)(pair % (N / 2)) : 0;
  const Tin* img = (const Tin*)p.frames + (size_t)f * p.frame_stride;
  const Tin* r0 = img + (size_t)y0 * N;
  const Tin* r1 = r0 + N;

  float a0[8], a1[8];
  double s0 = 0.0, s1 = 0.0;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int x = t + q * NT;
    a0[q] = valid ? ld_pix(r0 + x) : 0.f;
    a1[q] = valid ? ld_pix(r1 + x) : 0.f;
    if (p.smask) {
      a0[q] *= (float)p.smask[(size_t)y0 * N + x];
      a1[q] *= (float)p.smask[(size_t)(y0 + 1) * N + x];
    }
    s0 += (double)a0[q];
    s1 += (double)a1[q];
  }
  s0 = group_sum<NT>(s0, &red[g][0][0], t);
  s1 = group_sum<NT>(s1, &red[g][1][0], t);
  // row means as an unevaluated (hi, lo) FP32 pair
  const double c0 = s0 * p.ninv[y0], c1 = s1 * p.ninv[y0 + 1];
  const float c0h = (float)c0, c0l = (float)(c0 - (double)c0h);
  const float c1h = (float)c1, c1l = (float)(c1 - (double)c1h);
  const float wy0 = p.wys[y0], wy1 = p.wys[y0 + 1];
  float2 v[8];
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int x = t + q * NT;
    const float wx = __ldg(&p.win[x]);
    float m0 = 1.f, m1 = 1.f;
    if (p.smask) {
      m0 = (float)p.smask[(size_t)y0 * N + x];
      m1 = (float)p.smask[(size_t)(y0 + 1) * N + x];
    }
    v[q] = make_float2(((a0[q] - c0h) - c0l) * wx * m0 * wy0, ((a1[q] - c1h) - c1l) * wx * m1 * wy1);
  }
  const float2* Z = fft<N, false>(v, t, buf0, buf1, p.tw);
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
      p.rowsum[(size_t)f * N + y0] = s0;
      p.rowsum[(size_t)f * N + y0 + 1] = s1;
    }
  }
}

template <int N, int FG>
__global__ void __launch_bounds__(256) cols_kernel(ColParams p) {
  constexpr int NT = N / 8;
  constexpr int G = 256 / NT >= 1 ? 256 / NT : 1;
  constexpr int PN = padded(N);
  constexpr int ITEMS = KB * FG;
  extern __shared__ float2 sm[];
  float2* tile = sm;                        // [FG][N][KB]
  float2* outt = tile + FG * N * KB;        // [KB][N][FG]
  float2* fbuf = outt + KB * N * FG;        // G groups x 2 x PN
  float* dy = (float*)(fbuf + (size_t)G * 2 * PN);  // [FG][N]
  __shared__ double s_mu[FG];
  __shared__ double s_red[256 / 32];

  const int kb = blockIdx.x;
  const int f0 = blockIdx.y * FG;
  const int nf = min(FG, p.nframes - f0);
  const int tid = threadIdx.x;

  // frame means from the FP64 row sums
  for (int f = 0; f < nf; f++) {
    double s = 0.0;
    for (int y = tid; y < N; y += blockDim.x) s += p.rowsum[(size_t)(f0 + f) * N + y];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((tid & 31) == 0) s_red[tid >> 5] = s;
    __syncthreads();
    if (tid == 0) {
      double tot = 0.0;
      for (int w = 0; w < (int)(blockDim.x / 32); w++) tot += s_red[w];
      s_mu[f] = tot * p.inv_total[0];
      if (kb == 0) p.means[f0 + f] = s_mu[f] * (double)p.scale;
    }
    __syncthreads();
  }
  // correction coefficients dy = (c_y - mu) * scale * w(y), and the tile load
  for (int i = tid; i < FG * N; i += blockDim.x) {
    const int f = i / N, y = i % N;
    float d = 0.f;
    if (f < nf) {
      const double c = p.rowsum[(size_t)(f0 + f) * N + y] * p.ninv[y];
      d = (float)((c - s_mu[f]) * (double)p.wys[y]);
    }
    dy[i] = d;
  }
  {
    const float4* src = (const float4*)p.rows;
    float4* dst = (float4*)tile;
    const int per = N * KB / 2;  // float4 per frame block
    for (int i = tid; i < FG * per; i += blockDim.x) {
      const int f = i / per, j = i % per;
      float4 val = make_float4(0.f, 0.f, 0.f, 0.f);
      if (f < nf) val = __ldg(&src[((size_t)(f0 + f) * p.NHB + kb) * per + j]);
      dst[i] = val;
    }
  }
  __syncthreads();

  const int g = tid / NT, t = tid % NT;
  float2* b0 = fbuf + (size_t)g * 2 * PN;
  float2* b1 = b0 + PN;
  const float invN = 1.f / N;
  for (int it0 = 0; it0 < ITEMS; it0 += G) {
    const int it = it0 + g;
    const int c = it % KB, f = (it / KB) % FG;
    const int kx = kb * KB + c;
    float2 v[8];
    float2 wc = make_float2(0.f, 0.f);
    const bool corr = !p.wcorr_full && kx < 4;
    if (corr) wc = p.wcorr[kx];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int y = t + q * NT;
      float2 a = tile[((size_t)f * N + y) * KB + c];
      const float d = dy[f * N + y];
      if (p.wcorr_full) {
        const float2 w = kx < p.NH ? p.wcorr[(size_t)y * p.NH + kx] : make_float2(0.f, 0.f);
        a.x = fmaf(d, w.x, a.x);
        a.y = fmaf(d, w.y, a.y);
      } else if (corr) {
        a.x = fmaf(d, wc.x, a.x);
        a.y = fmaf(d, wc.y, a.y);
      }
      v[q] = a;
    }
    const float2* Y = fft<N, false>(v, t, b0, b1, p.tw);
    if (it < ITEMS) {
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int ky = t + q * NT;
        const float2 y = Y[pad(ky)];
        outt[((size_t)c * N + ky) * FG + f] = make_float2(y.x * invN, y.y * invN);
      }
    }
    __syncthreads();
  }

  // transposed store: FG consecutive slots of one mode together
  for (int i = tid; i < KB * N * FG; i += blockDim.x) {
    const int f = i % FG;
    const int ky = (i / FG) % N;
    const int c = i / (FG * N);
    const int kx = kb * KB + c;
    if (f < nf && kx < p.NH) {
      const size_t mode = (size_t)ky * p.NH + kx;
      p.hist[mode * p.T + p.slots[f0 + f]] = outt[i];
    }
  }
}

// ------------------------------------------------------------------ launchers

template <int N>
static size_t rows_smem() {
  constexpr int NT = N / 8;
  constexpr int G = 256 / NT >= 1 ? 256 / NT : 1;
  return (size_t)G * 2 * padded(N) * sizeof(float2);
}

template <int N>
static size_t cols_smem() {
  constexpr int NT = N / 8;
  constexpr int G = 256 / NT >= 1 ? 256 / NT : 1;
  constexpr int FG = col_frames(N);
  return (size_t)(2 * FG * N * KB + G * 2 * padded(N)) * sizeof(float2) +
         (size_t)FG * N * sizeof(float);
}

template <int N, typename Tin>
static cudaError_t rows_n(const RowParams& p, cudaStream_t s) {
  constexpr int NT = N / 8;
  constexpr int G = 256 / NT >= 1 ? 256 / NT : 1;
  const long long npairs = (long long)p.nframes * (N / 2);
  const int grid = (int)((npairs + G - 1) / G);
  auto k = rows_kernel<N, Tin>;
  const size_t sm = rows_smem<N>();
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k<<<grid, G * NT, sm, s>>>(p);
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
  constexpr int NT = N / 8;
  constexpr int G = 256 / NT >= 1 ? 256 / NT : 1;
  constexpr int FG = col_frames(N);
  dim3 grid(p.NHB, (p.nframes + FG - 1) / FG);
  auto k = cols_kernel<N, FG>;
  const size_t sm = cols_smem<N>();
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k<<<grid, G * NT, sm, s>>>(p);
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

}  // namespace ddm
