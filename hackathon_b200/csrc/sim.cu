// Seeded synthetic DDM movies on the GPU: the reference's simulator
// (motility-ddm/test/sim.mjs:14-186) with the same random streams, so a seed
// gives the reference's movie.
//
// The reference draws everything from one mulberry32 stream (sim.mjs:14-23):
// draw j after seed a0 is a hash of a0 + j * 0x6d2b79f5, so any draw can be
// computed directly. After the particles are set up (a few hundred
// sequential draws, made on the host in the reference's order), the movie
// only consumes normals (sim.mjs:26-44, Marsaglia's polar method with a
// cached spare): per frame N*N noise normals in pixel order, then two step
// normals per mobile particle. A polar attempt is a pair of consecutive
// draws, accepted when 0 < x^2 + y^2 < 1, and gives two normals. So for a
// chunk of frames the GPU evaluates every attempt at once, a prefix count over
// the acceptances places each accepted pair in the normal stream, and frame t
// reads its normals at fixed offsets. The spare and the stream position carry
// over between chunks exactly as in the reference.
//
// Rendering (sim.mjs:135-167): a frame starts at the background and each
// particle adds amp exp(-dx^2 / 2 s^2) exp(-dy^2 / 2 s^2) on its
// (2R+2)^2 window (R = ceil(4 s)), periodic, particles in order. Each CTA
// owns a 16 x 16 tile: it walks the particles in order, keeps those whose
// window reaches the tile (order-preserving compaction), and each thread adds
// their terms to its pixel in that order, so every pixel sums exactly the
// reference's terms in the reference's order. The file is compiled without
// FMA contraction (the reference's JavaScript arithmetic rounds every
// product and sum); exp and log are CUDA's (within an ulp or so of the
// host's), so a pixel can differ by one grey level only where its value sits
// on a rounding boundary.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "ddm_b200.h"

namespace {

constexpr uint32_t MB_STEP = 0x6d2b79f5u;
constexpr int TILE = 16;

__host__ __device__ inline double mb_hash(uint32_t a) {
  uint32_t t = a;
  t = (t ^ (t >> 15)) * (t | 1u);
  t ^= t + (t ^ (t >> 7)) * (t | 61u);
  return (double)(t ^ (t >> 14)) / 4294967296.0;
}

// The reference's generator on the host (sim.mjs:14-61).
struct HostRng {
  uint32_t a;
  bool has_spare = false;
  double spare = 0;
  explicit HostRng(uint32_t seed) : a(seed) {}
  double uniform() {
    a += MB_STEP;
    return mb_hash(a);
  }
  double normal() {
    if (has_spare) {
      has_spare = false;
      return spare;
    }
    double x, y, r;
    do {
      x = 2 * uniform() - 1;
      y = 2 * uniform() - 1;
      r = x * x + y * y;
    } while (r >= 1 || r == 0);
    const double f = std::sqrt((-2 * std::log(r)) / r);
    spare = y * f;
    has_spare = true;
    return x * f;
  }
  double gamma(double k, double theta) {
    if (k < 1) return gamma(k + 1, theta) * std::pow(uniform(), 1 / k);
    const double d = k - 1.0 / 3;
    const double c = 1 / std::sqrt(9 * d);
    for (;;) {
      double x, v;
      do {
        x = normal();
        v = 1 + c * x;
      } while (v <= 0);
      v = v * v * v;
      const double uu = uniform();
      if (uu < 1 - 0.0331 * std::pow(x, 4)) return d * v * theta;
      if (std::log(uu) < 0.5 * x * x + d * (1 - v + std::log(v))) return d * v * theta;
    }
  }
};

// attempt i of a chunk uses draws 2i+1 and 2i+2 after the chunk's state a0
__device__ inline bool attempt(uint32_t a0, long long i, double& x, double& y, double& r) {
  x = 2 * mb_hash(a0 + (uint32_t)(2 * i + 1) * MB_STEP) - 1;
  y = 2 * mb_hash(a0 + (uint32_t)(2 * i + 2) * MB_STEP) - 1;
  r = x * x + y * y;
  return r < 1 && r != 0;
}

__global__ void attempt_flags(uint32_t a0, long long A, int* flag) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A; i += (long long)gridDim.x * blockDim.x) {
    double x, y, r;
    flag[i] = attempt(a0, i, x, y, r) ? 1 : 0;
  }
}

// accepted attempt of rank q -> normals base + 2q (x f) and base + 2q + 1 (y f)
__global__ void write_normals(uint32_t a0, long long A, const int* flag, const int* rank, long long need,
                              double* normals, long long base, int* acc_idx) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < A; i += (long long)gridDim.x * blockDim.x) {
    if (!flag[i]) continue;
    const long long q = rank[i];
    if (q >= need) continue;
    double x, y, r;
    attempt(a0, i, x, y, r);
    const double f = sqrt((-2 * log(r)) / r);
    normals[base + 2 * q] = x * f;
    normals[base + 2 * q + 1] = y * f;
    acc_idx[q] = (int)i;
  }
}

// per particle: window origin and the separable profiles (sim.mjs:141-148)
__global__ void blob_profiles(const double* px_um, const double* py_um, int np, double dxUm, int R, int S,
                              double sig, double amp, int* x0, int* y0, double* gx, double* gy) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= np) return;
  const double px = px_um[k] / dxUm, py = py_um[k] / dxUm;
  const int bx = (int)floor(px) - R, by = (int)floor(py) - R;
  x0[k] = bx;
  y0[k] = by;
  for (int i = 0; i < S; i++) {
    const double ddx = (double)(bx + i) - px, ddy = (double)(by + i) - py;
    gx[(size_t)k * S + i] = exp((-ddx * ddx) / (2 * sig * sig));
    gy[(size_t)k * S + i] = amp * exp((-ddy * ddy) / (2 * sig * sig));
  }
}

// Math.round: ties toward +infinity
__device__ inline double js_round(double v) {
  const double f = floor(v);
  return (v - f >= 0.5) ? f + 1.0 : f;
}

__device__ inline int wrap(int v, int N) { return ((v % N) + N) % N; }

// One CTA per 16 x 16 tile of one frame.
__global__ void __launch_bounds__(256) render_tiles(int N, int np, int S, const int* x0, const int* y0,
                                                    const double* gx, const double* gy, double bg, double noise,
                                                    const double* normals, uint8_t* frame) {
  __shared__ int s_list[256];
  __shared__ int s_wcount[8];
  const int tx = blockIdx.x * TILE, ty = blockIdx.y * TILE;
  const int X = tx + (threadIdx.x % TILE), Y = ty + (threadIdx.x / TILE);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double img = bg;
  for (int c0 = 0; c0 < np; c0 += 256) {
    const int k = c0 + threadIdx.x;
    bool hit = false;
    if (k < np) {
      // the tile's columns sit at window offsets dx .. dx+15 (mod N)
      const int dx = wrap(tx - x0[k], N), dy = wrap(ty - y0[k], N);
      hit = (dx < S || dx + TILE - 1 >= N) && (dy < S || dy + TILE - 1 >= N);
    }
    const unsigned b = __ballot_sync(0xffffffffu, hit);
    if (lane == 0) s_wcount[w] = __popc(b);
    __syncthreads();
    int off = 0, m = 0;
    for (int i = 0; i < 8; i++) {
      off += i < w ? s_wcount[i] : 0;
      m += s_wcount[i];
    }
    if (hit) s_list[off + __popc(b & ((1u << lane) - 1u))] = k;
    __syncthreads();
    for (int e = 0; e < m; e++) {  // this chunk's particles that reach the tile, in order
      const int q = s_list[e];
      const int i = wrap(X - x0[q], N), j = wrap(Y - y0[q], N);
      if (i < S && j < S) img = img + gx[(size_t)q * S + i] * gy[(size_t)q * S + j];
    }
    __syncthreads();
  }
  const double v = js_round((img + noise * normals[(size_t)Y * N + X]) * 255);
  frame[(size_t)Y * N + X] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
}

// sim.mjs:169-175: mobile particles (indices < nmob) take normals 2k, 2k+1
__global__ void move_particles(double* x, double* y, const double* vx, const double* vy, int nmob, double Vx,
                               double Vy, double dt, double step, double Lf, const double* normals) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nmob) return;
  const double a = x[k] + ((vx[k] + Vx) * dt + step * normals[2 * k]);
  const double b = y[k] + ((vy[k] + Vy) * dt + step * normals[2 * k + 1]);
  x[k] = fmod(fmod(a, Lf) + Lf, Lf);
  y[k] = fmod(fmod(b, Lf) + Lf, Lf);
}

thread_local std::string g_sim_error;

int sim_fail(int code, const std::string& msg) {
  g_sim_error = msg;
  return code;
}

struct DevBufs {
  std::vector<void*> ptrs;
  ~DevBufs() {
    cudaDeviceSynchronize();  // an error return may leave kernels queued on these buffers
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  bool alloc(T** p, size_t n) {
    *p = nullptr;
    if (cudaMalloc((void**)p, sizeof(T) * (n ? n : 1)) != cudaSuccess) return false;
    ptrs.push_back(*p);
    return true;
  }
};

}  // namespace

#define SCK(x)                                                                                             \
  do {                                                                                                     \
    cudaError_t e_ = (x);                                                                                  \
    if (e_ != cudaSuccess) return sim_fail(DDM_ERR_CUDA, std::string("simulate: ") + cudaGetErrorString(e_)); \
  } while (0)

extern "C" const char* ddm_simulate_error(void) { return g_sim_error.c_str(); }

extern "C" int ddm_simulate(const ddm_sim_params* p, uint8_t* frames, int32_t frames_on_device, uint8_t* valid,
                            double* truth, void* stream_) {
  if (!p || !frames || !valid) return sim_fail(DDM_ERR_ARG, "simulate: NULL argument");
  const int N = p->N, T = p->T;
  if (N < TILE || N % TILE || N > 8192 || T < 1)
    return sim_fail(DDM_ERR_ARG, "simulate: N must be a multiple of 16 in [16, 8192], T >= 1");
  if (p->nSwim < 0 || p->nPassive < 0 || p->nFixed < 0 || !(p->fps > 0) || !(p->dxUm > 0) ||
      !(p->blobSigmaPx > 0) || p->dropExact < 0 || p->dropExact > T - 1 || (p->nSwim > 0 && !(p->swimSigma > 0)))
    return sim_fail(DDM_ERR_ARG, "simulate: invalid particle counts or parameters");
  const int R = (int)std::ceil(4 * p->blobSigmaPx), S = 2 * R + 2;
  if (S >= N) return sim_fail(DDM_ERR_ARG, "simulate: the blob window does not fit the frame");
  cudaStream_t st = (cudaStream_t)stream_;
  const double dt = 1 / p->fps, dxUm = p->dxUm, Lf = N * dxUm;
  double Vx = 0, Vy = 0;
  if (p->hasDrift) {
    Vx = p->driftSpeed * std::cos((p->driftAngleDeg * M_PI) / 180);
    Vy = p->driftSpeed * std::sin((p->driftAngleDeg * M_PI) / 180);
  }
  // particles, in the reference's order and draws (sim.mjs:106-131)
  HostRng rng(p->seed);
  const int np = p->nSwim + p->nPassive + p->nFixed, nmob = p->nSwim + p->nPassive;
  std::vector<double> hx(np), hy(np), hvx(np, 0.0), hvy(np, 0.0);
  double speedSum = 0;
  int c = 0;
  if (p->nSwim > 0) {
    const double Z = std::pow(p->swimVbar / p->swimSigma, 2) - 1;
    for (int i = 0; i < p->nSwim; i++, c++) {
      const double v = rng.gamma(Z + 1, p->swimVbar / (Z + 1));
      speedSum += v;
      const double phi = 2 * M_PI * rng.uniform();
      double s = 1;
      if (!p->swim2d) {
        const double cz = 2 * rng.uniform() - 1;
        s = std::sqrt(1 - cz * cz);
      }
      hx[c] = rng.uniform() * Lf;
      hy[c] = rng.uniform() * Lf;
      hvx[c] = v * s * std::cos(phi);
      hvy[c] = v * s * std::sin(phi);
    }
  }
  for (int i = 0; i < p->nPassive + p->nFixed; i++, c++) {
    hx[c] = rng.uniform() * Lf;
    hy[c] = rng.uniform() * Lf;
  }
  const double step = std::sqrt(2 * p->Dum2s * dt);

  // normals per frame and frames per chunk (<= 32 Mi normals at a time)
  const long long per = (long long)N * N + 2LL * nmob;
  const int F = (int)std::max<long long>(1, std::min<long long>(T, (32LL << 20) / per));
  const long long Acap = (long long)std::ceil((F * per / 2.0 + 2) / 0.78) + 4096;
  DevBufs db;
  double *d_x, *d_y, *d_vx, *d_vy, *d_gx, *d_gy, *d_norm;
  int *d_x0, *d_y0, *d_flag, *d_rank, *d_acc;
  uint8_t* d_frames = frames;
  if (!db.alloc(&d_x, np) || !db.alloc(&d_y, np) || !db.alloc(&d_vx, np) || !db.alloc(&d_vy, np) ||
      !db.alloc(&d_gx, (size_t)np * S) || !db.alloc(&d_gy, (size_t)np * S) || !db.alloc(&d_x0, np) ||
      !db.alloc(&d_y0, np) || !db.alloc(&d_norm, (size_t)F * per + 2) || !db.alloc(&d_flag, Acap) ||
      !db.alloc(&d_rank, Acap) || !db.alloc(&d_acc, Acap))  // accepted attempts <= attempts
    return sim_fail(DDM_ERR_NOMEM, "simulate: device allocation failed");
  if (!frames_on_device && !db.alloc(&d_frames, (size_t)F * N * N))
    return sim_fail(DDM_ERR_NOMEM, "simulate: device allocation failed");
  size_t tmp_bytes = 0;
  SCK(cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, d_flag, d_rank, (int)Acap, st));
  char* d_tmp = nullptr;
  if (!db.alloc(&d_tmp, tmp_bytes)) return sim_fail(DDM_ERR_NOMEM, "simulate: device allocation failed");
  if (np > 0) {
    SCK(cudaMemcpyAsync(d_x, hx.data(), sizeof(double) * np, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_y, hy.data(), sizeof(double) * np, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_vx, hvx.data(), sizeof(double) * np, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(d_vy, hvy.data(), sizeof(double) * np, cudaMemcpyHostToDevice, st));
  }

  uint32_t a = rng.a;
  bool has_spare = rng.has_spare;
  double spare = rng.spare;
  const int gridA = 148 * 8;
  const dim3 tiles(N / TILE, N / TILE);
  for (int t0 = 0; t0 < T; t0 += F) {
    const int Fc = std::min(F, T - t0);
    const long long Mc = (long long)Fc * per;
    const long long m = Mc - (has_spare ? 1 : 0);  // normals taken from attempts
    const long long need = (m + 1) / 2;           // accepted attempts needed
    long long A = std::min(Acap, (long long)std::ceil(need / 0.78) + 4096);
    for (;;) {
      attempt_flags<<<gridA, 256, 0, st>>>(a, A, d_flag);
      SCK(cudaGetLastError());
      SCK(cub::DeviceScan::ExclusiveSum(d_tmp, tmp_bytes, d_flag, d_rank, (int)A, st));
      int last[2];
      SCK(cudaMemcpyAsync(&last[0], d_rank + A - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
      SCK(cudaMemcpyAsync(&last[1], d_flag + A - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
      SCK(cudaStreamSynchronize(st));
      if (last[0] + last[1] >= need) break;
      if (A >= Acap) return sim_fail(DDM_ERR_CUDA, "simulate: too few accepted attempts");
      A = std::min(Acap, A + A / 4 + 4096);
    }
    const long long base = has_spare ? 1 : 0;
    if (has_spare) SCK(cudaMemcpyAsync(d_norm, &spare, sizeof(double), cudaMemcpyHostToDevice, st));
    write_normals<<<gridA, 256, 0, st>>>(a, A, d_flag, d_rank, need, d_norm, base, d_acc);
    SCK(cudaGetLastError());
    int ilast = 0;
    double sp = 0;
    SCK(cudaMemcpyAsync(&ilast, d_acc + need - 1, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (m & 1)
      SCK(cudaMemcpyAsync(&sp, d_norm + base + 2 * (need - 1) + 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    for (int f = 0; f < Fc; f++) {
      const double* nf = d_norm + (size_t)f * per;
      uint8_t* out = d_frames + (size_t)(frames_on_device ? t0 + f : f) * N * N;
      if (np > 0) {
        blob_profiles<<<(np + 127) / 128, 128, 0, st>>>(d_x, d_y, np, dxUm, R, S, p->blobSigmaPx, p->amp, d_x0,
                                                          d_y0, d_gx, d_gy);
        SCK(cudaGetLastError());
      }
      render_tiles<<<tiles, 256, 0, st>>>(N, np, S, d_x0, d_y0, d_gx, d_gy, p->background, p->noise, nf, out);
      SCK(cudaGetLastError());
      if (nmob > 0) {
        move_particles<<<(nmob + 127) / 128, 128, 0, st>>>(d_x, d_y, d_vx, d_vy, nmob, Vx, Vy, dt, step, Lf,
                                                             nf + (size_t)N * N);
        SCK(cudaGetLastError());
      }
    }
    if (!frames_on_device)
      SCK(cudaMemcpyAsync(frames + (size_t)t0 * N * N, d_frames, (size_t)Fc * N * N, cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    a += (uint32_t)(2 * ((long long)ilast + 1)) * MB_STEP;
    has_spare = (m & 1) != 0;
    spare = sp;
  }

  // drop masks (sim.mjs:177-187)
  for (int t = 0; t < T; t++) valid[t] = 1;
  HostRng drng(p->seed * 7919u + 13u);
  if (p->dropExact) {
    std::vector<int> idx(T - 1);
    for (int i = 0; i < T - 1; i++) idx[i] = i + 1;
    for (int i = T - 2; i > 0; i--) {
      const int j = (int)std::floor(drng.uniform() * (i + 1));
      std::swap(idx[i], idx[j]);
    }
    for (int i = 0; i < p->dropExact; i++) valid[idx[i]] = 0;
  } else if (p->dropFrac > 0) {
    for (int t = 1; t < T; t++)
      if (drng.uniform() < p->dropFrac) valid[t] = 0;
  }
  if (truth) {
    truth[0] = p->nSwim > 0 ? speedSum / p->nSwim : 0;
    truth[1] = Vx;
    truth[2] = Vy;
    truth[3] = p->Dum2s;
  }
  return DDM_OK;
}
