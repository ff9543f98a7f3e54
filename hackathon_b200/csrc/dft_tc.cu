// Batched zero-padded 2048-point DFT on the fifth-generation tensor cores: a
// measured reference point for the temporal stage's transforms (its forward
// transform: a series of T = 1024 samples, zero-padded to TPAD = 2048). Not on
// the analysis path: as a pass of its own its spectra cross HBM, while the
// fused CUDA-core kernel of temporal.cu keeps them on chip and runs its 1.5
// transforms per mode, the masked Wiener-Khinchin arithmetic and the radial
// epilogue in about the time this kernel takes for one transform per mode
// (the bench's roofline.library_fft_reference.tensor_core_forward). Software
// pipeline per CTA: step A's products overlap the previous group's spectrum
// leaving, step C's the next group's operand arriving.
//
// Four-step factorisation 2048 = 64 x 32 with the samples t = 32 n1 + n2
// (n1 < 32 hold data, n2 < 32) and the bins k = k1 + 64 k2:
//   X[k] = sum_n2 W32^{n2 k2} W2048^{n2 k1} sum_n1 x[32 n1 + n2] W64^{n1 k1}
// as two tcgen05 products per group of four series, complex numbers as
// (re, im) pairs along K and N:
//   step A  rows (series, n2)  x  K (n1, re/im) = 64  ->  N (k1, re/im) = 128
//           one 128 x 128 product per group;
//   step B  the accumulators back through tcgen05.ld, the twiddle
//           W2048^{n2 k1} (first power from a table, the next by products),
//           and the transpose into rows (series, k1) x K (n2, re/im);
//   step C  two 128 x 64 products (rows (series, k1), N (k2, re/im)).
// BF16 operands with a three-term split (hi hi + hi lo + lo hi, FP32
// accumulation in tensor memory): ~2e-5 of the series' RMS spectrum.
// Operands are K-major without swizzle (core matrices of 8 rows x 16 B); the
// transposed operand of step C has a padded K stride (LBO 144 B) so that the
// 32 lanes' 4-byte stores of one row fall in 32 different banks.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ddm_b200.h"
#include "async_copy.cuh"
#include "umma.cuh"

namespace ddm {
namespace dfttc {

constexpr int NPT = 2048, NS = 1024;           // transform length, samples per series
constexpr int B1_BYTES = 128 * 64 * 2;         // B of step A: [N 128][K 64] BF16
constexpr int B2_BYTES = 64 * 64 * 2;          // B of step C: [N 64][K 64]
constexpr int A1_BYTES = 128 * 64 * 2;         // A of step A: [128][64], LBO 128, SBO 1024
constexpr int A2_LBO = 144, A2_SBO = 8 * A2_LBO;
constexpr int A2_TILE = 16 * A2_SBO;           // A of step C: two [128][64] tiles, padded
constexpr int OFF_B1H = 0, OFF_B1L = OFF_B1H + B1_BYTES, OFF_B2H = OFF_B1L + B1_BYTES;
constexpr int OFF_B2L = OFF_B2H + B2_BYTES, CONST_BYTES = OFF_B2L + B2_BYTES;
constexpr int OFF_A1H = CONST_BYTES, OFF_A1L = OFF_A1H + A1_BYTES;
constexpr int OFF_A2H = OFF_A1L + A1_BYTES, OFF_A2L = OFF_A2H + 2 * A2_TILE;
constexpr int OFF_TW = OFF_A2L + 2 * A2_TILE;  // float2 W2048^j
constexpr int SMEM = OFF_TW + NPT * 8;

// byte offset of element (row r, k) in a K-major no-swizzle tile with K = 64
__host__ __device__ constexpr int off64(int r, int k) {
  return (r >> 3) * 1024 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2;
}
__device__ __forceinline__ int offA2(int r, int k) {
  return (r >> 3) * A2_SBO + (k >> 3) * A2_LBO + (r & 7) * 16 + (k & 7) * 2;
}

__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

__global__ void __launch_bounds__(256, 1) dft2048_kernel(const float2* __restrict__ x, long long ld, int n,
                                                         const uint4* __restrict__ consts,
                                                         const float2* __restrict__ tw, float2* __restrict__ X,
                                                         int* err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < CONST_BYTES / 16; i += 256) reinterpret_cast<uint4*>(sm)[i] = consts[i];
  float2* stw = reinterpret_cast<float2*>(sm + OFF_TW);
  for (int i = tid; i < NPT; i += 256) stw[i] = tw[i];
  if (warp == 0) {
    umma::tmem_alloc(&tslot, 256);
    umma::tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  umma::fence_before_sync();
  __syncthreads();
  umma::fence_after_sync();
  const uint32_t tmem = tslot;
  const int ngroups = (n + 3) / 4;
  uint32_t ph0 = 0, ph1 = 0;
  bool ok = true;
  // A of step A: thread -> row (series, n2), half of the n1 range
  auto build_a1 = [&](int grp) {
    const int r = tid >> 1, h = tid & 1, s = r >> 5, n2 = r & 31;
    const int m = grp * 4 + s;
    const float2* xs = x + (size_t)(m < n ? m : 0) * ld;
#pragma unroll
    for (int cm = 0; cm < 4; cm++) {
      uint32_t hi[4], lo[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int n1 = 16 * h + 4 * cm + j;
        const float2 v = m < n ? __ldg(&xs[32 * n1 + n2]) : make_float2(0.f, 0.f);
        split2(v.x, v.y, hi[j], lo[j]);
      }
      const int k = 2 * (16 * h + 4 * cm);
      *reinterpret_cast<uint4*>(sm + OFF_A1H + off64(r, k)) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
      *reinterpret_cast<uint4*>(sm + OFF_A1L + off64(r, k)) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    }
    fence_proxy_async_smem();
  };
  // the spectrum of a group from tensor-memory columns 128..255: tile t lane
  // (series % 2) * 64 + k1, columns (k2, re/im), halves per warp pair
  auto output = [&](int grp) {
    const int rr = (warp & 3) * 32 + lane, c0 = (warp >> 2) * 32;
#pragma unroll
    for (int t = 0; t < 2; t++) {
      float v[32];
      umma::ld32(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(128 + 64 * t + c0), v);
      const int m = grp * 4 + 2 * t + (rr >> 6), k1 = rr & 63;
      if (m < n) {
        float2* xo = X + (size_t)m * NPT;
#pragma unroll
        for (int i = 0; i < 16; i++) xo[k1 + 64 * (c0 / 2 + i)] = make_float2(v[2 * i], v[2 * i + 1]);
      }
    }
  };
  // Software pipeline per group: products of step A || the previous group's
  // spectrum leaving; products of step C || the next group's operand of
  // step A arriving.
  int prev = -1;
  if ((int)blockIdx.x < ngroups) build_a1(blockIdx.x);
  __syncthreads();
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    if (tid == 0) {
      umma::fence_after_sync();
      constexpr uint32_t ID = umma::idesc_bf16_f32(128, 128);
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const uint64_t ah = umma::desc_kmajor(sm + OFF_A1H + j * 256, 128, 1024);
        const uint64_t al = umma::desc_kmajor(sm + OFF_A1L + j * 256, 128, 1024);
        const uint64_t bh = umma::desc_kmajor(sm + OFF_B1H + j * 256, 128, 1024);
        const uint64_t bl = umma::desc_kmajor(sm + OFF_B1L + j * 256, 128, 1024);
        umma::mma_bf16(tmem, ah, bh, ID, j > 0);
        umma::mma_bf16(tmem, ah, bl, ID, true);
        umma::mma_bf16(tmem, al, bh, ID, true);
      }
      umma::commit(&bar[0]);
    }
    if (prev >= 0) output(prev);
    if (!mbar_wait(&bar[0], ph0, err, 1)) ok = false;
    ph0 ^= 1u;
    ok = __syncthreads_and(ok);
    if (!ok) break;
    umma::fence_after_sync();
    // step B: lane row (warp % 4) * 32 + lane, half of the columns per warp pair
    {
      const int r = (warp & 3) * 32 + lane, s = r >> 5, n2 = r & 31;
      const int c0 = (warp >> 2) * 64;
#pragma unroll
      for (int q = 0; q < 2; q++) {
        float v[32];
        umma::ld32(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(c0 + 32 * q), v);
        const int kb = (c0 + 32 * q) / 2;
        float2 w = stw[(n2 * kb) & (NPT - 1)];
        const float2 s1 = stw[n2];
#pragma unroll
        for (int i = 0; i < 16; i++) {
          if (i) w = make_float2(fmaf(w.x, s1.x, -w.y * s1.y), fmaf(w.x, s1.y, w.y * s1.x));
          const float yr = fmaf(v[2 * i], w.x, -v[2 * i + 1] * w.y);
          const float yi = fmaf(v[2 * i], w.y, v[2 * i + 1] * w.x);
          uint32_t hi, lo;
          split2(yr, yi, hi, lo);
          const int r2 = s * 64 + kb + i;
          const int o = (r2 >> 7) * A2_TILE + offA2(r2 & 127, 2 * n2);
          *reinterpret_cast<uint32_t*>(sm + OFF_A2H + o) = hi;
          *reinterpret_cast<uint32_t*>(sm + OFF_A2L + o) = lo;
        }
      }
    }
    fence_proxy_async_smem();
    umma::fence_before_sync();
    __syncthreads();  // A2 written; the previous spectrum read out of tensor memory
    if (tid == 0) {
      umma::fence_after_sync();
      constexpr uint32_t ID = umma::idesc_bf16_f32(128, 64);
#pragma unroll
      for (int t = 0; t < 2; t++) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const uint64_t ah = umma::desc_kmajor(sm + OFF_A2H + t * A2_TILE + j * 2 * A2_LBO, A2_LBO, A2_SBO);
          const uint64_t al = umma::desc_kmajor(sm + OFF_A2L + t * A2_TILE + j * 2 * A2_LBO, A2_LBO, A2_SBO);
          const uint64_t bh = umma::desc_kmajor(sm + OFF_B2H + j * 256, 128, 1024);
          const uint64_t bl = umma::desc_kmajor(sm + OFF_B2L + j * 256, 128, 1024);
          const uint32_t d = tmem + 128 + 64 * t;
          umma::mma_bf16(d, ah, bh, ID, j > 0);
          umma::mma_bf16(d, ah, bl, ID, true);
          umma::mma_bf16(d, al, bh, ID, true);
        }
      }
      umma::commit(&bar[1]);
    }
    // step A's operand is free (its products completed): the next group's
    const int nxt = grp + (int)gridDim.x;
    if (nxt < ngroups) build_a1(nxt);
    if (!mbar_wait(&bar[1], ph1, err, 2)) ok = false;
    ph1 ^= 1u;
    ok = __syncthreads_and(ok);  // also: the next operand of step A is complete
    if (!ok) break;
    umma::fence_after_sync();
    prev = grp;
  }
  if (ok && prev >= 0) output(prev);
  if (!ok) {
    // a wait gave up: let the products in flight finish (bounded) before freeing tensor memory
    mbar_wait(&bar[0], ph0 ^ 1u, nullptr, 0);
    mbar_wait(&bar[1], ph1 ^ 1u, nullptr, 0);
  }
  umma::fence_after_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, 256);
}

// BF16 round to nearest even (finite inputs)
uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
}
float bf16_value(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// The DFT matrices of steps A and C as B operands ([N][K] K-major, hi and lo
// parts), in FP64 from the angles, then split.
std::vector<uint16_t> build_consts() {
  std::vector<uint16_t> c(CONST_BYTES / 2, 0);
  auto put = [&](int off_hi, int off_lo, int row, int k, double v) {
    const uint16_t h = bf16_bits((float)v);
    const uint16_t l = bf16_bits((float)(v - (double)bf16_value(h)));
    c[(off_hi + off64(row, k)) / 2] = h;
    c[(off_lo + off64(row, k)) / 2] = l;
  };
  // (yr, yi) = (xr wr - xi wi, xr wi + xi wr): rows n = 2 kout + d, K = 2 nin + c
  auto block = [&](int off_hi, int off_lo, int nin, int nout, int len) {
    for (int a = 0; a < nin; a++)
      for (int b = 0; b < nout; b++) {
        const double ang = -2.0 * M_PI * (double)((a * b) % len) / len;
        const double wr = std::cos(ang), wi = std::sin(ang);
        put(off_hi, off_lo, 2 * b, 2 * a, wr);
        put(off_hi, off_lo, 2 * b, 2 * a + 1, -wi);
        put(off_hi, off_lo, 2 * b + 1, 2 * a, wi);
        put(off_hi, off_lo, 2 * b + 1, 2 * a + 1, wr);
      }
  };
  block(OFF_B1H, OFF_B1L, 32, 64, 64);  // W64^{n1 k1}
  block(OFF_B2H, OFF_B2L, 32, 32, 32);  // W32^{n2 k2}
  return c;
}

struct DevTables {
  uint4* consts = nullptr;
  float2* tw = nullptr;
  int* err = nullptr;
  int sms = 0;
};

cudaError_t tables(DevTables* out) {
  static std::mutex mu;
  static std::map<int, DevTables> cache;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  DevTables t;
  const std::vector<uint16_t> c = build_consts();
  std::vector<float2> w(NPT);
  for (int j = 0; j < NPT; j++) {
    const double ang = -2.0 * M_PI * j / NPT;
    w[j] = make_float2((float)std::cos(ang), (float)std::sin(ang));
  }
  e = cudaMalloc((void**)&t.consts, CONST_BYTES);
  if (e == cudaSuccess) e = cudaMalloc((void**)&t.tw, NPT * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc((void**)&t.err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(t.consts, c.data(), CONST_BYTES, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(t.tw, w.data(), NPT * sizeof(float2), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(t.err, 0, sizeof(int));
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&t.sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(dft2048_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
  if (e != cudaSuccess) {
    cudaFree(t.consts);
    cudaFree(t.tw);
    cudaFree(t.err);
    return e;
  }
  cache[dev] = t;
  *out = t;
  return cudaSuccess;
}

}  // namespace dfttc
}  // namespace ddm

extern std::string& ddm_detached_error();  // message slot of calls without an engine (engine.cu)

extern "C" int ddm_dft2048_tc(const void* x, int64_t ld, int32_t n, void* X, void* stream) {
  ddm_detached_error().clear();
  if (n < 0 || ld < ddm::dfttc::NS) {
    ddm_detached_error() = "ddm_dft2048_tc: need n >= 0 and ld >= 1024";
    return DDM_ERR_ARG;
  }
  if (n == 0) return DDM_OK;
  if (!x || !X || ((uintptr_t)x & 7) || ((uintptr_t)X & 7)) {
    ddm_detached_error() = "ddm_dft2048_tc: null or misaligned array";
    return DDM_ERR_ARG;
  }
  ddm::dfttc::DevTables t;
  cudaError_t e = ddm::dfttc::tables(&t);
  if (e != cudaSuccess) {
    ddm_detached_error() = std::string("ddm_dft2048_tc: ") + cudaGetErrorString(e);
    return DDM_ERR_CUDA;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int groups = (n + 3) / 4;
  const int grid = groups < t.sms ? groups : t.sms;
  ddm::dfttc::dft2048_kernel<<<grid, 256, ddm::dfttc::SMEM, s>>>(
      (const float2*)x, (long long)ld, n, t.consts, t.tw, (float2*)X, t.err);
  e = cudaGetLastError();
  int werr = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(&werr, t.err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    ddm_detached_error() = std::string("ddm_dft2048_tc: ") + cudaGetErrorString(e);
    return DDM_ERR_CUDA;
  }
  if (werr) {
    cudaMemset(t.err, 0, sizeof(int));
    ddm_detached_error() = "ddm_dft2048_tc: a bounded wait for the tensor cores gave up";
    return DDM_ERR_CUDA;
  }
  return DDM_OK;
}
