// BF16 tensor-core MLP (training and inference) for the motility surrogate:
// a normalised ISF curve (64 log-spaced lags) and ln q in, the motility
// parameters out; 65 -> 256 -> 256 -> 256 -> 256 -> 5, GELU between layers.
// No counterpart in the reference (a learned seed for the fit, required by
// the batched-LM design); its prediction only ever seeds the batched LM
// (ddm_fit_lm mode 1), and the LM from the reference's start strategy stays
// the fallback and the reference its error is measured against.
//
// Every matrix product is one tcgen05 kernel (gemm_kernel): 128 x N output
// tiles, BF16 operands staged K-major in shared memory (64-wide K chunks,
// double-buffered with cp.async), FP32 accumulators in tensor memory, one
// thread issuing the MMAs and committing them to an mbarrier, and an
// epilogue that reads the accumulators back with tcgen05.ld and applies the
// layer's operation in registers:
//   forward hidden   z = acc + b, h = GELU(z): h (BF16, row-major and
//                    transposed for the weight-gradient product), z (FP32)
//   forward output   o = acc + b (FP32)
//   backward data    dz = acc * GELU'(z): dz (BF16, both layouts) and the
//                    column sums (bias gradient)
//   weight gradient  split-K partial sums added into FP32 dW
// Adam keeps FP32 master weights and writes the BF16 copies (W and W^T)
// each step. Layer widths are padded for the MMA shapes: input 65 -> 80,
// output 5 -> 16 (padding rows/columns are zero and stay zero).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/ddm_b200.h"
#include "async_copy.cuh"
#include "umma.cuh"

namespace ddm {
namespace mlp {

using bf16 = __nv_bfloat16;

constexpr int NIN = 65, KIN = 80;   // input features, padded
constexpr int HID = 256;            // hidden width
constexpr int NOUT = 5, NOP = 16;   // outputs, padded
constexpr int NL = 5;               // layers
constexpr int IN_P[NL] = {KIN, HID, HID, HID, HID};
constexpr int OUT_P[NL] = {HID, HID, HID, HID, NOP};
constexpr int IN_R[NL] = {NIN, HID, HID, HID, HID};
constexpr int OUT_R[NL] = {HID, HID, HID, HID, NOUT};
constexpr int KC = 64;              // K per shared-memory stage

enum Epi { EPI_STORE_F32 = 0, EPI_ATOMIC_F32 = 1, EPI_BIAS_F32 = 2, EPI_BIAS_GELU = 3, EPI_GELU_BWD = 4 };

struct GemmParams {
  int M, K;             // output rows, reduction length (multiple of 16)
  const bf16* A;        // [M][lda], K contiguous
  const bf16* B;        // [N][ldb], K contiguous
  int lda, ldb;
  int nreal;            // output columns written (<= N)
  int ksplit;           // K per CTA along grid.y (multiple of KC)
  int epi;
  const float* bias;    // [N]
  float* outf;          // FP32 out [M][ldo]
  int ldo;
  bf16* outh;           // BF16 out [M][ldh]
  int ldh;
  bf16* outt;           // BF16 transposed out [N][ldt]
  int ldt;
  float* zsave;         // FP32 pre-activation [M][ldo]: written (forward), read (backward)
  float* colsum;        // [N] column sums of dz (bias gradient), or nullptr
  int* err;
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

template <int N>
__host__ __device__ constexpr uint32_t tmem_cols() {
  return N <= 32 ? 32 : N <= 64 ? 64 : N <= 128 ? 128 : 256;
}

// Shared-memory stage: A chunk [128 rows][KC] then B chunk [N rows][KC],
// each as core matrices (8 rows x 16 B) at ((row/8) * (KC/8) + k/8) * 128 B:
// LBO (K step) = 128 B, SBO (8-row step) = KC/8 * 128 B = 1024 B.
template <int N>
struct Stage {
  static constexpr int A_BYTES = 128 * KC * 2;
  static constexpr int B_BYTES = N * KC * 2;
  static constexpr int BYTES = A_BYTES + B_BYTES;
};

__device__ __forceinline__ void load_rows(uint8_t* dst, const bf16* src, int ld, int rows, int row0, int nrows,
                                          int k0, int K, int tid) {
  // copy i: core matrix (rg, kg), row-in-group r8; consecutive i fill
  // consecutive 16 B of shared memory
  const int total = rows * (KC / 8);
  for (int i = tid; i < total; i += 128) {
    const int r8 = i & 7, kg = (i >> 3) % (KC / 8), rg = (i >> 3) / (KC / 8);
    const int r = rg * 8 + r8, k = k0 + kg * 8;
    const bool ok = (row0 + r) < nrows && k < K;
    const bf16* s = ok ? src + (size_t)(row0 + r) * ld + k : src;
    umma::cp_async16(dst + (size_t)i * 16, s, ok ? 16u : 0u);
  }
}

template <int N>
__global__ void __launch_bounds__(128, 1) gemm_kernel(GemmParams p) {
  constexpr uint32_t TCOLS = tmem_cols<N>();
  constexpr uint32_t IDESC = umma::idesc_bf16_f32(128, N);
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) {
    umma::tmem_alloc(&tslot, TCOLS);
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
  const uint32_t taddr = tslot;
  const int m0 = blockIdx.x * 128;
  const int k0 = blockIdx.y * p.ksplit;
  const int k1 = min(p.K, k0 + p.ksplit);
  const int nc = (k1 - k0 + KC - 1) / KC;
  auto stage_ptr = [&](int s) { return smem + (size_t)s * Stage<N>::BYTES; };
  auto load = [&](int c, int s) {
    uint8_t* st = stage_ptr(s);
    load_rows(st, p.A, p.lda, 128, m0, p.M, k0 + c * KC, k1, tid);
    load_rows(st + Stage<N>::A_BYTES, p.B, p.ldb, N, 0, N, k0 + c * KC, k1, tid);
  };
  bool ok = true;
  if (nc > 0) {
    load(0, 0);
    umma::cp_async_wait_all();
    fence_proxy_async_smem();
    __syncthreads();
    for (int c = 0; c < nc && ok; c++) {
      const int s = c & 1;
      if (c + 1 < nc) {
        // stage s^1 was last read by the MMAs of chunk c - 1
        if (c >= 1 && !mbar_wait(&bar[s ^ 1], (uint32_t)((c - 1) >> 1) & 1u, p.err, 10)) ok = false;
        if (ok) load(c + 1, s ^ 1);
      }
      if (ok && tid == 0) {
        umma::fence_after_sync();
        const uint8_t* st = stage_ptr(s);
        // K steps of 16 (a ragged tail is zero-filled by the copies)
        const int ksteps = (min(KC, k1 - (k0 + c * KC)) + 15) / 16;
        for (int j = 0; j < ksteps; j++) {
          const uint64_t ad = umma::desc_kmajor(st + j * 256, 128, (KC / 8) * 128);
          const uint64_t bd = umma::desc_kmajor(st + Stage<N>::A_BYTES + j * 256, 128, (KC / 8) * 128);
          umma::mma_bf16(taddr, ad, bd, IDESC, c > 0 || j > 0);
        }
        umma::commit(&bar[s]);
      }
      umma::cp_async_wait_all();
      fence_proxy_async_smem();
      ok = __syncthreads_and(ok);  // one verdict for the whole CTA
    }
    // accumulators complete once the last chunk's commit arrives
    const int cl = nc - 1;
    if (ok && !mbar_wait(&bar[cl & 1], (uint32_t)(cl >> 1) & 1u, p.err, 11)) ok = false;
    ok = __syncthreads_and(ok);  // tcgen05.ld below is warp-collective
    if (!ok) {
      // a wait gave up: let the MMAs in flight finish (bounded) before freeing TMEM
      mbar_wait(&bar[cl & 1], (uint32_t)(cl >> 1) & 1u, nullptr, 0);
    }
  }
  umma::fence_after_sync();
  const int m = m0 + warp * 32 + lane;
  const bool mv = m < p.M;
  if (ok && nc > 0) {
#pragma unroll 1
    for (int n0 = 0; n0 < N; n0 += 16) {
      float v[16];
      ld16(taddr + ((uint32_t)(warp * 32) << 16) + (uint32_t)n0, v);
      if (p.epi == EPI_STORE_F32 || p.epi == EPI_ATOMIC_F32 || p.epi == EPI_BIAS_F32) {
        if (mv)
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const int n = n0 + i;
            if (n >= p.nreal) continue;
            float* o = p.outf + (size_t)m * p.ldo + n;
            if (p.epi == EPI_ATOMIC_F32)
              atomicAdd(o, v[i]);
            else
              *o = v[i] + (p.epi == EPI_BIAS_F32 ? p.bias[n] : 0.f);
          }
      } else {
        float outv[16];
        if (p.epi == EPI_BIAS_GELU) {
#pragma unroll
          for (int i = 0; i < 16; i++) {
            const float z = v[i] + p.bias[n0 + i];
            outv[i] = gelu(z);
            v[i] = z;
          }
          if (mv && p.zsave) {
            float4* zs = (float4*)(p.zsave + (size_t)m * p.ldo + n0);
#pragma unroll
            for (int i = 0; i < 4; i++) zs[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
          }
        } else {  // EPI_GELU_BWD
          float z[16];
          if (mv) {
            const float4* zs = (const float4*)(p.zsave + (size_t)m * p.ldo + n0);
#pragma unroll
            for (int i = 0; i < 4; i++) {
              const float4 q = zs[i];
              z[4 * i] = q.x;
              z[4 * i + 1] = q.y;
              z[4 * i + 2] = q.z;
              z[4 * i + 3] = q.w;
            }
          }
#pragma unroll
          for (int i = 0; i < 16; i++) outv[i] = mv ? v[i] * gelu_grad(z[i]) : 0.f;
        }
        // BF16 copies: row-major (two 16 B stores) and transposed (lanes write
        // consecutive rows: 64 B per column per warp)
        bf16 hb[16];
#pragma unroll
        for (int i = 0; i < 16; i++) hb[i] = __float2bfloat16_rn(outv[i]);
        if (mv && p.outh) {
          uint4* dst = (uint4*)(p.outh + (size_t)m * p.ldh + n0);
          dst[0] = *(const uint4*)&hb[0];
          dst[1] = *(const uint4*)&hb[8];
        }
        if (mv && p.outt)
#pragma unroll
          for (int i = 0; i < 16; i++) p.outt[(size_t)(n0 + i) * p.ldt + m] = hb[i];
        if (p.colsum) {
#pragma unroll
          for (int i = 0; i < 16; i++) {
            float sv = outv[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) sv += __shfl_xor_sync(0xffffffffu, sv, o);
            if (lane == 0) atomicAdd(&p.colsum[n0 + i], sv);
          }
        }
      }
    }
  }
  umma::fence_before_sync();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(taddr, TCOLS);
}

template <int N>
static cudaError_t gemm_n(const GemmParams& p, int splits, cudaStream_t s) {
  const size_t sm = 2 * (size_t)Stage<N>::BYTES;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(gemm_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  dim3 grid((p.M + 127) / 128, splits);
  gemm_kernel<N><<<grid, 128, sm, s>>>(p);
  return cudaGetLastError();
}

// C[M][N] (epilogue) = A[M][K] B[N][K]^T; splits > 1 divides K over grid.y.
static cudaError_t gemm(int N, GemmParams p, int splits, cudaStream_t s) {
  if (splits < 1) splits = 1;
  p.ksplit = ((p.K + splits - 1) / splits + KC - 1) / KC * KC;
  splits = (p.K + p.ksplit - 1) / p.ksplit;
  switch (N) {
    case 16: return gemm_n<16>(p, splits, s);
    case 80: return gemm_n<80>(p, splits, s);
    case 256: return gemm_n<256>(p, splits, s);
    default: return cudaErrorInvalidValue;
  }
}

// ------------------------------------------------------------ elementwise

// features [n][65] FP32 -> BF16 [n][80] (zero padding) and its transpose [80][n]
__global__ void cast_input_kernel(const float* __restrict__ x, int n, bf16* __restrict__ xh,
                                  bf16* __restrict__ xt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * KIN) return;
  const int r = i / KIN, c = i % KIN;
  const bf16 v = __float2bfloat16_rn(c < NIN ? x[(size_t)r * NIN + c] : 0.f);
  xh[i] = v;
  if (xt) xt[(size_t)c * n + r] = v;
}

// MSE over the 5 outputs: loss = sum (o - y)^2 / (n * 5); dO = 2 (o - y) / (n * 5)
// (BF16, both layouts, zero in the padding columns); bias gradient of the
// output layer = column sums of dO.
__global__ void loss_kernel(const float* __restrict__ o, const float* __restrict__ y, int n, bf16* __restrict__ dO,
                            bf16* __restrict__ dOT, float* __restrict__ db, float* __restrict__ loss) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  float g[NOUT];
#pragma unroll
  for (int j = 0; j < NOUT; j++) g[j] = 0.f;
  if (r < n) {
    const float sc = 2.f / ((float)n * NOUT);
#pragma unroll
    for (int j = 0; j < NOP; j++) {
      float d = 0.f;
      if (j < NOUT) {
        d = o[(size_t)r * NOP + j] - y[(size_t)r * NOUT + j];
        l += d * d;
        g[j] = sc * d;
      }
      const bf16 b = __float2bfloat16_rn(j < NOUT ? sc * d : 0.f);
      dO[(size_t)r * NOP + j] = b;
      dOT[(size_t)j * n + r] = b;
    }
  }
#pragma unroll
  for (int o2 = 16; o2 > 0; o2 >>= 1) {
    l += __shfl_xor_sync(0xffffffffu, l, o2);
#pragma unroll
    for (int j = 0; j < NOUT; j++) g[j] += __shfl_xor_sync(0xffffffffu, g[j], o2);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(loss, l / ((float)n * NOUT));
#pragma unroll
    for (int j = 0; j < NOUT; j++) atomicAdd(&db[j], g[j]);
  }
}

// Adam on FP32 masters (real extent only; padding stays zero), then the BF16
// copies W [out][in] and W^T [in][out].
__global__ void adam_kernel(float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                            const float* __restrict__ g, int rows, int cols, int ldw, int rreal, int creal,
                            float lr, float b1, float b2, float eps, float c1, float c2, bf16* __restrict__ wh,
                            bf16* __restrict__ wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int r = i / cols, c = i % cols;
  const size_t k = (size_t)r * ldw + c;
  if (r < rreal && c < creal) {
    const float gi = g[k];
    const float mi = b1 * m[k] + (1.f - b1) * gi;
    const float vi = b2 * v[k] + (1.f - b2) * gi * gi;
    m[k] = mi;
    v[k] = vi;
    w[k] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
  if (wh) {
    const bf16 b = __float2bfloat16_rn(w[k]);
    wh[k] = b;
    wt[(size_t)c * rows + r] = b;
  }
}

__global__ void bf16_copies_kernel(const float* __restrict__ w, int rows, int cols, bf16* __restrict__ wh,
                                   bf16* __restrict__ wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows * cols) return;
  const int r = i / cols, c = i % cols;
  const bf16 b = __float2bfloat16_rn(w[i]);
  wh[i] = b;
  wt[(size_t)c * rows + r] = b;
}

}  // namespace mlp
}  // namespace ddm

// ------------------------------------------------------------------ engine

using namespace ddm::mlp;

struct ddm_mlp {
  int dev = 0;
  int bmax = 0;
  cudaStream_t stream = nullptr;
  int* d_err = nullptr;
  float *W[NL] = {}, *b[NL] = {};              // FP32 masters [out_p][in_p], [out_p]
  float *mW[NL] = {}, *vW[NL] = {}, *mb[NL] = {}, *vb[NL] = {};
  float *dW[NL] = {}, *db[NL] = {};
  bf16 *Wh[NL] = {}, *WhT[NL] = {};            // BF16 [out_p][in_p], [in_p][out_p]
  bf16 *xh = nullptr, *xt = nullptr;           // [B][80], [80][B]
  bf16 *Hh[4] = {}, *Ht[4] = {};               // [B][256], [256][B]
  float* Z[4] = {};                            // [B][256]
  float* out = nullptr;                        // [B][16]
  bf16 *dA = nullptr, *dAt = nullptr, *dB = nullptr, *dBt = nullptr;  // dz ping-pong [B][256], [256][B]
  bf16 *dO = nullptr, *dOt = nullptr;          // [B][16], [16][B]
  float* loss = nullptr;
  int step = 0;
  std::string err;
};

namespace {

thread_local std::string g_mlp_err;

int mlp_fail(ddm_mlp* h, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (h)
    h->err = buf;
  else
    g_mlp_err = buf;
  return code;
}

#define MCK(x)                                                                   \
  do {                                                                           \
    cudaError_t e_ = (x);                                                        \
    if (e_ != cudaSuccess) return mlp_fail(h, DDM_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
cudaError_t zalloc(T** p, size_t n) {
  cudaError_t e = cudaMalloc((void**)p, sizeof(T) * (n ? n : 1));
  if (e == cudaSuccess) e = cudaMemset(*p, 0, sizeof(T) * (n ? n : 1));
  return e;
}

void release(ddm_mlp* h) {
  auto f = [](void* p) {
    if (p) cudaFree(p);
  };
  for (int l = 0; l < NL; l++) {
    f(h->W[l]); f(h->b[l]); f(h->mW[l]); f(h->vW[l]); f(h->mb[l]); f(h->vb[l]);
    f(h->dW[l]); f(h->db[l]); f(h->Wh[l]); f(h->WhT[l]);
  }
  for (int i = 0; i < 4; i++) {
    f(h->Hh[i]); f(h->Ht[i]); f(h->Z[i]);
  }
  f(h->xh); f(h->xt); f(h->out); f(h->dA); f(h->dAt); f(h->dB); f(h->dBt); f(h->dO); f(h->dOt);
  f(h->loss); f(h->d_err);
}

int refresh_bf16(ddm_mlp* h) {
  for (int l = 0; l < NL; l++) {
    const int n = OUT_P[l] * IN_P[l];
    bf16_copies_kernel<<<(n + 255) / 256, 256, 0, h->stream>>>(h->W[l], OUT_P[l], IN_P[l], h->Wh[l], h->WhT[l]);
  }
  MCK(cudaGetLastError());
  return DDM_OK;
}

GemmParams base(ddm_mlp* h) {
  GemmParams p{};
  p.err = h->d_err;
  return p;
}

// Forward over n rows of h->xh; keep = store H^T and Z for the backward pass.
int forward(ddm_mlp* h, int n, bool keep) {
  const bf16* A = h->xh;
  int lda = KIN;
  for (int l = 0; l < NL; l++) {
    GemmParams p = base(h);
    p.M = n;
    p.K = IN_P[l];
    p.A = A;
    p.lda = lda;
    p.B = h->Wh[l];
    p.ldb = IN_P[l];
    p.nreal = OUT_P[l];
    p.bias = h->b[l];
    if (l < NL - 1) {
      p.epi = EPI_BIAS_GELU;
      p.outh = h->Hh[l];
      p.ldh = HID;
      p.outt = keep ? h->Ht[l] : nullptr;
      p.ldt = n;
      p.zsave = keep ? h->Z[l] : nullptr;
      p.ldo = HID;
      MCK(gemm(HID, p, 1, h->stream));
      A = h->Hh[l];
      lda = HID;
    } else {
      p.epi = EPI_BIAS_F32;
      p.outf = h->out;
      p.ldo = NOP;
      p.nreal = NOP;
      MCK(gemm(NOP, p, 1, h->stream));
    }
  }
  return DDM_OK;
}

// Backward from dO (set by loss_kernel) into dW, db.
int backward(ddm_mlp* h, int n) {
  for (int l = 0; l < NL; l++) {
    MCK(cudaMemsetAsync(h->dW[l], 0, sizeof(float) * OUT_P[l] * IN_P[l], h->stream));
    if (l < NL - 1) MCK(cudaMemsetAsync(h->db[l], 0, sizeof(float) * OUT_P[l], h->stream));
  }
  const bf16* dz = h->dO;    // [n][out_p]
  const bf16* dzt = h->dOt;  // [out_p][n]
  const int splits = n >= 2048 ? n / 512 : 1;
  for (int l = NL - 1; l >= 0; l--) {
    // dW_l [out_p][in_p] = dz^T [out_p][n] . X_l^T [in_p][n]^T
    {
      GemmParams p = base(h);
      p.M = OUT_P[l];
      p.K = n;
      p.A = dzt;
      p.lda = n;
      p.B = l == 0 ? h->xt : h->Ht[l - 1];
      p.ldb = n;
      p.nreal = IN_P[l];
      p.epi = EPI_ATOMIC_F32;
      p.outf = h->dW[l];
      p.ldo = IN_P[l];
      MCK(gemm(IN_P[l], p, splits, h->stream));
    }
    if (l == 0) break;
    // dz_{l-1} [n][256] = (dz [n][out_p] . W_l [out_p][256]) * GELU'(Z_{l-1})
    {
      bf16* oh = (l & 1) ? h->dA : h->dB;
      bf16* ot = (l & 1) ? h->dAt : h->dBt;
      GemmParams p = base(h);
      p.M = n;
      p.K = OUT_P[l];
      p.A = dz;
      p.lda = OUT_P[l];
      p.B = h->WhT[l];
      p.ldb = OUT_P[l];
      p.nreal = HID;
      p.epi = EPI_GELU_BWD;
      p.zsave = h->Z[l - 1];
      p.ldo = HID;
      p.outh = oh;
      p.ldh = HID;
      p.outt = ot;
      p.ldt = n;
      p.colsum = h->db[l - 1];
      MCK(gemm(HID, p, 1, h->stream));
      dz = oh;
      dzt = ot;
    }
  }
  return DDM_OK;
}

int check_rows(ddm_mlp* h, int n) {
  if (n < 1 || n > h->bmax || (n & 7))
    return mlp_fail(h, DDM_ERR_ARG, "rows = %d: need 1 <= rows <= %d and rows a multiple of 8", n, h->bmax);
  return DDM_OK;
}

int device_error(ddm_mlp* h) {
  int e = 0;
  MCK(cudaMemcpy(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (e) {
    cudaMemset(h->d_err, 0, sizeof(int));
    return mlp_fail(h, DDM_ERR_CUDA, "tensor-core GEMM: an mbarrier wait gave up (code %d)", e);
  }
  return DDM_OK;
}

}  // namespace

extern "C" const char* ddm_mlp_last_error(const ddm_mlp* h) { return h ? h->err.c_str() : g_mlp_err.c_str(); }

extern "C" int ddm_mlp_create(int32_t batch_max, uint64_t seed, ddm_mlp** out) {
  g_mlp_err.clear();
  if (!out) return mlp_fail(nullptr, DDM_ERR_ARG, "ddm_mlp_create: out is NULL");
  *out = nullptr;
  if (batch_max < 8 || batch_max > (1 << 20) || (batch_max & 7))
    return mlp_fail(nullptr, DDM_ERR_ARG, "batch_max = %d: need a multiple of 8 in [8, 2^20]", batch_max);
  int dev = 0, ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return mlp_fail(nullptr, DDM_ERR_NODEV, "no CUDA device");
  cudaGetDevice(&dev);
  cudaDeviceProp prop;
  cudaGetDeviceProperties(&prop, dev);
  if (prop.major != 10) return mlp_fail(nullptr, DDM_ERR_NODEV, "device is sm_%d%d, need sm_100", prop.major, prop.minor);
  ddm_mlp* h = new ddm_mlp();
  h->dev = dev;
  h->bmax = batch_max;
  const size_t B = batch_max;
  h->stream = nullptr;  // set-up work on the legacy default stream; calls name their stream
  bool ok = zalloc(&h->d_err, 1) == cudaSuccess && zalloc(&h->loss, 1) == cudaSuccess;
  for (int l = 0; l < NL && ok; l++) {
    const size_t nw = (size_t)OUT_P[l] * IN_P[l];
    ok = zalloc(&h->W[l], nw) == cudaSuccess && zalloc(&h->b[l], OUT_P[l]) == cudaSuccess &&
         zalloc(&h->mW[l], nw) == cudaSuccess && zalloc(&h->vW[l], nw) == cudaSuccess &&
         zalloc(&h->mb[l], OUT_P[l]) == cudaSuccess && zalloc(&h->vb[l], OUT_P[l]) == cudaSuccess &&
         zalloc(&h->dW[l], nw) == cudaSuccess && zalloc(&h->db[l], OUT_P[l]) == cudaSuccess &&
         zalloc(&h->Wh[l], nw) == cudaSuccess && zalloc(&h->WhT[l], nw) == cudaSuccess;
  }
  for (int i = 0; i < 4 && ok; i++)
    ok = zalloc(&h->Hh[i], B * HID) == cudaSuccess && zalloc(&h->Ht[i], B * HID) == cudaSuccess &&
         zalloc(&h->Z[i], B * HID) == cudaSuccess;
  ok = ok && zalloc(&h->xh, B * KIN) == cudaSuccess && zalloc(&h->xt, B * KIN) == cudaSuccess &&
       zalloc(&h->out, B * NOP) == cudaSuccess && zalloc(&h->dA, B * HID) == cudaSuccess &&
       zalloc(&h->dAt, B * HID) == cudaSuccess && zalloc(&h->dB, B * HID) == cudaSuccess &&
       zalloc(&h->dBt, B * HID) == cudaSuccess && zalloc(&h->dO, B * NOP) == cudaSuccess &&
       zalloc(&h->dOt, B * NOP) == cudaSuccess;
  if (!ok) {
    release(h);
    delete h;
    return mlp_fail(nullptr, DDM_ERR_NOMEM, "ddm_mlp_create: device allocation failed");
  }
  // He-style uniform initialisation of the real extent, zero bias
  std::mt19937_64 rng(seed);
  for (int l = 0; l < NL; l++) {
    std::vector<float> w((size_t)OUT_P[l] * IN_P[l], 0.f);
    const float a = std::sqrt(6.f / IN_R[l]) * (l == NL - 1 ? 0.5f : 1.f);
    std::uniform_real_distribution<float> u(-a, a);
    for (int o = 0; o < OUT_R[l]; o++)
      for (int i = 0; i < IN_R[l]; i++) w[(size_t)o * IN_P[l] + i] = u(rng);
    if (cudaMemcpy(h->W[l], w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
      release(h);
      delete h;
      return mlp_fail(nullptr, DDM_ERR_CUDA, "ddm_mlp_create: weight upload failed");
    }
  }
  if (refresh_bf16(h) || cudaStreamSynchronize(h->stream) != cudaSuccess) {
    const std::string m = h->err;
    release(h);
    delete h;
    return mlp_fail(nullptr, DDM_ERR_CUDA, "ddm_mlp_create: %s", m.c_str());
  }
  *out = h;
  return DDM_OK;
}

extern "C" void ddm_mlp_destroy(ddm_mlp* h) {
  if (!h) return;
  cudaSetDevice(h->dev);
  cudaDeviceSynchronize();
  release(h);
  delete h;
}

extern "C" int32_t ddm_mlp_param_count(void) {
  int n = 0;
  for (int l = 0; l < NL; l++) n += OUT_R[l] * IN_R[l] + OUT_R[l];
  return n;
}

// Flat layout, per layer: W [out][in] (real extent, row-major), then b [out].
static int copy_params(ddm_mlp* h, float* const* src_dev, float* const* bsrc_dev, float* host, bool to_host) {
  size_t off = 0;
  for (int l = 0; l < NL; l++) {
    for (int o = 0; o < OUT_R[l]; o++) {
      float* d = src_dev[l] + (size_t)o * IN_P[l];
      if (to_host)
        MCK(cudaMemcpy(host + off, d, sizeof(float) * IN_R[l], cudaMemcpyDeviceToHost));
      else
        MCK(cudaMemcpy(d, host + off, sizeof(float) * IN_R[l], cudaMemcpyHostToDevice));
      off += IN_R[l];
    }
    if (to_host)
      MCK(cudaMemcpy(host + off, bsrc_dev[l], sizeof(float) * OUT_R[l], cudaMemcpyDeviceToHost));
    else
      MCK(cudaMemcpy(bsrc_dev[l], host + off, sizeof(float) * OUT_R[l], cudaMemcpyHostToDevice));
    off += OUT_R[l];
  }
  return DDM_OK;
}

extern "C" int ddm_mlp_get_params(ddm_mlp* h, float* params) {
  if (!h || !params) return mlp_fail(h, DDM_ERR_ARG, "null argument");
  cudaSetDevice(h->dev);
  MCK(cudaDeviceSynchronize());
  return copy_params(h, h->W, h->b, params, true);
}

extern "C" int ddm_mlp_set_params(ddm_mlp* h, const float* params) {
  if (!h || !params) return mlp_fail(h, DDM_ERR_ARG, "null argument");
  cudaSetDevice(h->dev);
  MCK(cudaDeviceSynchronize());
  h->stream = nullptr;
  int rc = copy_params(h, h->W, h->b, const_cast<float*>(params), false);
  if (rc) return rc;
  for (int l = 0; l < NL; l++) {
    MCK(cudaMemset(h->mW[l], 0, sizeof(float) * OUT_P[l] * IN_P[l]));
    MCK(cudaMemset(h->vW[l], 0, sizeof(float) * OUT_P[l] * IN_P[l]));
    MCK(cudaMemset(h->mb[l], 0, sizeof(float) * OUT_P[l]));
    MCK(cudaMemset(h->vb[l], 0, sizeof(float) * OUT_P[l]));
  }
  h->step = 0;
  if ((rc = refresh_bf16(h))) return rc;
  MCK(cudaStreamSynchronize(h->stream));
  return DDM_OK;
}

extern "C" int ddm_mlp_forward(ddm_mlp* h, const float* x, int32_t n, float* out, void* stream) {
  if (!h || !x || !out) return mlp_fail(h, DDM_ERR_ARG, "null argument");
  int rc = check_rows(h, n);
  if (rc) return rc;
  cudaSetDevice(h->dev);
  h->stream = (cudaStream_t)stream;
  cast_input_kernel<<<(n * KIN + 255) / 256, 256, 0, h->stream>>>(x, n, h->xh, nullptr);
  rc = forward(h, n, false);
  if (!rc) {
    // [n][16] -> [n][5]
    cudaError_t e = cudaMemcpy2DAsync(out, sizeof(float) * NOUT, h->out, sizeof(float) * NOP, sizeof(float) * NOUT,
                                      n, cudaMemcpyDeviceToDevice, h->stream);
    if (e != cudaSuccess) rc = mlp_fail(h, DDM_ERR_CUDA, "output copy: %s", cudaGetErrorString(e));
  }
  return rc;
}

// One pass of forward + backward on n rows; gradients left in dW/db.
static int grads(ddm_mlp* h, const float* x, const float* y, int n) {
  cast_input_kernel<<<(n * KIN + 255) / 256, 256, 0, h->stream>>>(x, n, h->xh, h->xt);
  int rc = forward(h, n, true);
  if (rc) return rc;
  MCK(cudaMemsetAsync(h->loss, 0, sizeof(float), h->stream));
  MCK(cudaMemsetAsync(h->db[NL - 1], 0, sizeof(float) * NOP, h->stream));
  loss_kernel<<<(n + 255) / 256, 256, 0, h->stream>>>(h->out, y, n, h->dO, h->dOt, h->db[NL - 1], h->loss);
  MCK(cudaGetLastError());
  return backward(h, n);
}

extern "C" int ddm_mlp_gradients(ddm_mlp* h, const float* x, const float* y, int32_t n, float* grads_host,
                                 float* loss_host, void* stream) {
  if (!h || !x || !y || !grads_host) return mlp_fail(h, DDM_ERR_ARG, "null argument");
  int rc = check_rows(h, n);
  if (rc) return rc;
  cudaSetDevice(h->dev);
  h->stream = (cudaStream_t)stream;
  if ((rc = grads(h, x, y, n))) return rc;
  MCK(cudaStreamSynchronize(h->stream));
  if ((rc = device_error(h))) return rc;
  if (loss_host) MCK(cudaMemcpy(loss_host, h->loss, sizeof(float), cudaMemcpyDeviceToHost));
  return copy_params(h, h->dW, h->db, grads_host, true);
}

extern "C" int ddm_mlp_train_step(ddm_mlp* h, const float* x, const float* y, int32_t n, float lr,
                                  float* loss_host, void* stream) {
  if (!h || !x || !y) return mlp_fail(h, DDM_ERR_ARG, "null argument");
  int rc = check_rows(h, n);
  if (rc) return rc;
  if (!(lr > 0)) return mlp_fail(h, DDM_ERR_ARG, "lr must be > 0");
  cudaSetDevice(h->dev);
  h->stream = (cudaStream_t)stream;
  if ((rc = grads(h, x, y, n))) return rc;
  h->step++;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - std::pow(b1, (float)h->step), c2 = 1.f - std::pow(b2, (float)h->step);
  for (int l = 0; l < NL; l++) {
    const int nw = OUT_P[l] * IN_P[l];
    adam_kernel<<<(nw + 255) / 256, 256, 0, h->stream>>>(h->W[l], h->mW[l], h->vW[l], h->dW[l], OUT_P[l], IN_P[l],
                                                         IN_P[l], OUT_R[l], IN_R[l], lr, b1, b2, eps, c1, c2,
                                                         h->Wh[l], h->WhT[l]);
    adam_kernel<<<(OUT_P[l] + 255) / 256, 256, 0, h->stream>>>(h->b[l], h->mb[l], h->vb[l], h->db[l], OUT_P[l], 1,
                                                               1, OUT_R[l], 1, lr, b1, b2, eps, c1, c2, nullptr,
                                                               nullptr);
  }
  MCK(cudaGetLastError());
  if (loss_host) {
    MCK(cudaMemcpyAsync(loss_host, h->loss, sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    MCK(cudaStreamSynchronize(h->stream));
    return device_error(h);
  }
  return DDM_OK;
}

extern "C" int ddm_mlp_sync(ddm_mlp* h, void* stream) {
  if (!h) return DDM_ERR_ARG;
  cudaSetDevice(h->dev);
  MCK(cudaStreamSynchronize((cudaStream_t)stream));
  return device_error(h);
}
