// Masked Wiener-Khinchin temporal analysis and the radial reduction.
//
// Reference semantics (motility-ddm/src/ddm_ref.js:229-288, ddm.wgsl:202-259):
// for each Fourier mode, x(t) = hist[mode][order[t]] * mask[t], t < T, zero
// padded to TPAD, p = |x|^2, and
//   A(tau) + B(tau) = IFFT(2 Re(conj(M) P)),   G(tau) = IFFT(|Y|^2),
//   D(tau) = (A + B - 2 Re G) / N(tau),  C(tau) = G / N(tau),  P = sum p / N(0)
// with M = FFT(mask) and N(tau) the exact valid-pair counts (host, FP64).
//
// B200 formulation: one CTA of TPAD/8 threads processes modes in pairs (a, b)
// with five register-resident FFTs per pair instead of the reference's four
// per mode:
//   Z  = FFT(p_a + i p_b)                 -> P_a, P_b by Hermitian split
//   Y  = FFT(x_a);  W_a = IFFT(|Y|^2 + i 2 Re(conj(M) P_a))
//   Y  = FFT(x_b);  W_b = IFFT(|Y|^2 + i 2 Re(conj(M) P_b))
// |Y|^2 and 2 Re(conj(M) P) are both real, so W = n (G + i E) splits into
//   G(tau) = (W(tau) + conj W(-tau)) / 2n,  E(tau) = Im(W(tau) - conj W(-tau)) / 2n
// where E = A + B. That is 2.5 transforms per mode instead of 4.
//
// Two epilogues:
//  * fused radial (default): modes are visited in bin order in "units" (a run
//    of modes of one bin); each thread owns lags and accumulates the bin's D
//    and the eight phase-drift sums of (tau, tau+1) (ddm_ref.js:360-382) in
//    FP64 registers, writing one partial record per unit. reduce_kernel sums
//    the units of each bin in a fixed order (deterministic) and divides by the
//    bin's mode count (ddm_ref.js:404-412).
//  * full outputs: per-mode D[mode][tau], C[mode][tau], P[mode] as the
//    reference's GPU pass writes them (ddm.wgsl:243-258); radial_full_kernel
//    then reduces them like the reference's `radial` pass (ddm.wgsl:265-322)
//    but with FP64 sums.
// Work is handed out through an atomic unit counter (no waiting on other
// CTAs), so a persistent grid of one wave load-balances uneven bins.
#include <cstdint>

#include "async_copy.cuh"
#include "ddm_b200.h"
#include "fft_block.cuh"
#include "kernels.cuh"

namespace ddm {

__device__ __forceinline__ int4 load_item(const int4* items, int i) {
  return items ? items[i] : make_int4(i, 0, 0, 0);
}

template <int NP>
struct TemporalCommon {
  static constexpr int NT = NP / 8;
  static constexpr int PN = padded(NP);
};

// Gathers x(t) = row[order[t]] * mask[t] from the staged time series into the
// FFT input pattern. T <= TPAD/2, so only q < 4 can hold samples; q >= 4 are
// the zero padding and stay compile-time zeros (the first FFT stage folds
// them away).
template <int NP>
__device__ __forceinline__ void gather(float2 (&x)[8], const float2* __restrict__ row,
                                       const uint32_t (&ord)[4], const float (&msk)[4]) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    float2 v = row[ord[q]];
    x[q] = make_float2(v.x * msk[q], v.y * msk[q]);
  }
#pragma unroll
  for (int q = 4; q < 8; q++) x[q] = make_float2(0.f, 0.f);
}

// Spectrum V(k) = |Y(k)|^2 + i 2 Re(conj(M_k) P(k)) of one mode (P from the
// packed Z buffer; `second` selects the imaginary half of the pack), left in
// registers in the FFT input pattern.
template <int NP>
__device__ __forceinline__ void spectrum_v(float2 (&v)[8], int t, const float2* __restrict__ Y,
                                           const float2* __restrict__ Z,
                                           const float2* __restrict__ mspec, bool second) {
  constexpr int NT = NP / 8;
#pragma unroll
  for (int q = 0; q < 8; q++) {
    const int k = t + q * NT;
    const float2 y = Y[pad(k)];
    const float2 zk = Z[pad(k)];
    const float2 zn = Z[pad((NP - k) & (NP - 1))];
    const float2 M = __ldg(&mspec[k]);
    const float Px = second ? 0.5f * (zk.y + zn.y) : 0.5f * (zk.x + zn.x);
    const float Py = second ? -0.5f * (zk.x - zn.x) : 0.5f * (zk.y - zn.y);
    const float S = fmaf(y.x, y.x, y.y * y.y);
    const float R = 2.f * fmaf(M.x, Px, M.y * Py);
    v[q] = make_float2(S, R);
  }
}

// Occupancy hint: cap registers at 128 per thread (2+ CTAs of 256 threads).
template <int NP>
struct TemporalBounds {
  static constexpr int NT = NP / 8;
  static constexpr int MIN_BLOCKS = NT >= 512 ? 1 : 512 / NT;
};

// The video a unit belongs to (batched launches) or the single video.
__device__ __forceinline__ VideoDesc video_of(const TemporalParams& p, int vi) {
  if (p.videos) return p.videos[vi];
  VideoDesc v;
  v.hist = p.hist;
  v.order = p.order;
  v.mask = p.mask;
  v.npairs = p.npairs;
  v.mspec = p.mspec;
  v.items = p.items;
  v.partials = p.partials;
  v.T = p.T;
  v.L = p.L;
  v.unit0 = 0;
  v.nunits = p.nunits;
  return v;
}

// Thread 0: stage the time series of pair k of `unit` into staging buffer
// `stage` (rows Tstride apart).
__device__ __forceinline__ void issue_pair(const TemporalParams& p, int unit, int k, float2* stage, int Tstride,
                                           uint64_t* bar) {
  const int4 U = p.units[unit];
  const VideoDesc v = video_of(p, p.videos ? U.w : 0);
  const bool hasb = k + 1 < U.y;
  const int ma = load_item(v.items, U.x + k).x;
  const uint32_t bytes = (uint32_t)v.T * sizeof(float2);
  mbar_arrive_expect_tx(bar, hasb ? 2 * bytes : bytes);
  bulk_g2s(stage, v.hist + (size_t)ma * v.T, bytes, bar);
  if (hasb) {
    const int mb = load_item(v.items, U.x + k + 1).x;
    bulk_g2s(stage + Tstride, v.hist + (size_t)mb * v.T, bytes, bar);
  }
}

template <int NP, int LPT, bool FULL>
__global__ void __launch_bounds__(NP / 8, TemporalBounds<NP>::MIN_BLOCKS)
    temporal_kernel(TemporalParams p) {
  constexpr int NT = NP / 8;
  constexpr int PN = padded(NP);
  constexpr bool ODD = fft_stages(NP) & 1;
  extern __shared__ __align__(16) float2 sm[];
  float2* bufZ = sm;
  float2* bufA = sm + PN;
  float2* bufB = sm + 2 * PN;
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ int s_next;
  const int t = threadIdx.x;
  const int TS = p.T;                 // staging stride: the (largest) T
  float2* stage = sm + 3 * PN;        // [2 buffers][2 rows][TS]
  float2* s_tw = stage + 4 * TS;      // per-stage twiddle blocks
  float* s_np = (float*)(s_tw + tw_size(NP));  // N(tau), tau < L
  const float invn = 0.5f / NP;
  for (int i = t; i < tw_size(NP); i += NT) s_tw[i] = p.tw[i];

  // per-video state, (re)loaded when a unit of another video comes up
  VideoDesc vd;
  int cur_v = -1, L = 0;
  float np0 = 0.f;
  uint32_t ord[4];
  float msk[4];
  auto load_video = [&](int vi) {
    vd = video_of(p, vi);
    cur_v = vi;
    L = vd.L;
    np0 = vd.npairs[0];
    for (int i = t; i < L; i += NT) s_np[i] = vd.npairs[i];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = t + q * NT;
      ord[q] = i < vd.T ? __ldg(&vd.order[i]) : 0u;
      msk[q] = i < vd.T ? __ldg(&vd.mask[i]) : 0.f;
    }
  };
  if (t == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    fence_barrier_init();
    s_next = atomicAdd(p.unit_counter, 1);
  }
  __syncthreads();
  int u = s_next;
  __syncthreads();
  if (t == 0) {
    s_next = atomicAdd(p.unit_counter, 1);
    if (u < p.nunits) issue_pair(p, u, 0, stage, TS, &mbar[0]);
  }
  __syncthreads();
  int unext = s_next;
  int k = 0, buf = 0;
  uint32_t phase = 0;  // bit b: parity to wait for on mbar[b]
  double acc[LPT][PFIELDS];
  double accP = 0.0;
#pragma unroll
  for (int r = 0; r < LPT; r++)
#pragma unroll
    for (int c = 0; c < PFIELDS; c++) acc[r][c] = 0.0;

  while (u < p.nunits) {
    const int4 U = p.units[u];
    const int vi = p.videos ? U.w : 0;
    if (vi != cur_v) {  // uniform over the CTA (every thread holds the same u)
      __syncthreads();  // s_np is no longer read
      load_video(vi);
      __syncthreads();
    }
    // prefetch the next pair (this unit's, or the next unit's first) into the
    // other staging buffer; its last readers finished before the loop-end sync
    int nu = u, nk = k + 2;
    if (nk >= U.y) {
      nu = unext;
      nk = 0;
    }
    const bool prefetched = nu < p.nunits;
    if (t == 0 && prefetched) issue_pair(p, nu, nk, stage + (buf ^ 1) * 2 * TS, TS, &mbar[buf ^ 1]);
    if (!mbar_wait(&mbar[buf], (phase >> buf) & 1u, p.err, 1)) {
      // give up: let the copy in flight land (bounded), then stop
      if (prefetched) mbar_wait(&mbar[buf ^ 1], (phase >> (buf ^ 1)) & 1u, p.err, 1);
      return;
    }
    phase ^= 1u << buf;
    const float2* rowa = stage + buf * 2 * TS;
    const float2* rowb = rowa + TS;
    const bool hasb = k + 1 < U.y;
    const int4 ea = load_item(vd.items, U.x + k);
    const int4 eb = hasb ? load_item(vd.items, U.x + k + 1) : ea;
    float2 v[8];
    {
      float2 w[8];
      gather<NP>(v, rowa, ord, msk);
      if (hasb)
        gather<NP>(w, rowb, ord, msk);
      else
#pragma unroll
        for (int q = 0; q < 8; q++) w[q] = make_float2(0.f, 0.f);
#pragma unroll
      for (int q = 0; q < 8; q++)
        v[q] = make_float2(fmaf(v[q].x, v[q].x, v[q].y * v[q].y), fmaf(w[q].x, w[q].x, w[q].y * w[q].y));
    }
    if (ODD)
      fft<NP, false, true>(v, t, bufZ, bufA, s_tw);
    else
      fft<NP, false, true>(v, t, bufA, bufZ, s_tw);
    const float2 zsum = bufZ[0];  // (sum p_a, sum p_b)

#pragma unroll 1
    for (int s = 0; s < 2; s++) {
      if (s == 1 && !hasb) break;
      const int4 e = s ? eb : ea;
      gather<NP>(v, s ? rowb : rowa, ord, msk);
      const float2* Y = fft<NP, false, true>(v, t, bufA, bufB, s_tw);
      spectrum_v<NP>(v, t, Y, bufZ, vd.mspec, s == 1);
      __syncthreads();
      const float2* W = fft<NP, true, true>(v, t, bufA, bufB, s_tw);
      const float ps = s ? zsum.y : zsum.x;
      const float P = np0 > 0.5f ? ps / np0 : 0.f;
      if (FULL) {
        const size_t mode = (size_t)e.x;
        for (int tau = t; tau < L; tau += NT) {
          const float np = s_np[tau];
          const float inv = np > 0.5f ? 1.f / np : 0.f;
          const float2 w0 = W[pad(tau)];
          const float2 w1 = W[pad((NP - tau) & (NP - 1))];
          const float gx = (w0.x + w1.x) * invn, gy = (w0.y - w1.y) * invn;
          const float ee = (w0.y + w1.y) * invn;
          p.outD[mode * L + tau] = (ee - 2.f * gx) * inv;
          p.outC[mode * L + tau] = make_float2(gx * inv, gy * inv);
        }
        if (t == 0) p.outP[mode] = P;
      } else {
        // D and the drift sums of the lag pair (tau, tau+1) at owned lags
        const double kx = e.y, ky = e.z;
#pragma unroll
        for (int r = 0; r < LPT; r++) {
          const int tau = t + r * NT;
          if (tau < L) {
            const float n0 = s_np[tau];
            const float inp = n0 > 0.5f ? 1.f / n0 : 0.f;
            const float2 w0 = W[pad(tau)];
            const float2 w1 = W[pad((NP - tau) & (NP - 1))];
            const float gx = (w0.x + w1.x) * invn, gy = (w0.y - w1.y) * invn;
            const float ee = (w0.y + w1.y) * invn;
            acc[r][0] += (double)((ee - 2.f * gx) * inp);
            if (tau + 1 < L) {
              const float n1 = s_np[tau + 1];
              const float inp1 = n1 > 0.5f ? 1.f / n1 : 0.f;
              const float2 u0 = W[pad(tau + 1)];
              const float2 u1 = W[pad((NP - tau - 1) & (NP - 1))];
              const float cx = gx * inp, cy = gy * inp;
              const float c1x = (u0.x + u1.x) * invn * inp1;
              const float c1y = (u0.y - u1.y) * invn * inp1;
              const float zr = fmaf(c1x, cx, c1y * cy);  // C(tau+1) conj C(tau)
              const float zi = fmaf(c1y, cx, -c1x * cy);
              const float w = sqrtf(fmaf(zr, zr, zi * zi));
              if (w > 0.f) {
                const double wd = w, ph = atan2f(zi, zr);
                acc[r][1] += wd;
                acc[r][2] += wd * kx * kx;
                acc[r][3] += wd * kx * ky;
                acc[r][4] += wd * ky * ky;
                acc[r][5] += wd * kx * ph;
                acc[r][6] += wd * ky * ph;
                acc[r][7] += wd * ph * ph;
                acc[r][8] += 1.0;
              }
            }
          }
        }
        accP += (double)P;
      }
      __syncthreads();
    }
    if (k + 2 >= U.y) {
      if (!FULL) {
        // one partial record per unit: [u][field][tau], P after all records
        // (u local to the unit's video)
        const int ul = u - vd.unit0;
#pragma unroll
        for (int r = 0; r < LPT; r++) {
          const int tau = t + r * NT;
          if (tau < L)
#pragma unroll
            for (int c = 0; c < PFIELDS; c++) {
              vd.partials[((size_t)ul * PFIELDS + c) * L + tau] = acc[r][c];
              acc[r][c] = 0.0;
            }
        }
        if (t == 0) vd.partials[(size_t)vd.nunits * PFIELDS * L + ul] = accP;
        accP = 0.0;
      }
      u = unext;
      k = 0;
      if (t == 0) s_next = atomicAdd(p.unit_counter, 1);
    } else {
      k += 2;
    }
    buf ^= 1;
    fence_proxy_async_smem();  // this CTA's reads of the staged rows before the next TMA write
    __syncthreads();
    unext = s_next;
  }
}

// ---------------------------------------------------------------------------
// Two-group variant for TPAD 1024..4096 (fused radial epilogue only): the CTA
// is two groups of TPAD/16 threads, each running 16-point-per-thread radix-16
// transforms (three exchange passes at 2048 instead of four, one buffer per
// group). Per mode pair (a, b) the five transforms run in three steps:
//   1: group 0  Z = FFT(p_a + i p_b)        group 1  Y_b = FFT(x_b)
//   2: group 0  Y_a = FFT(x_a)              group 1  W_b = IFFT(V_b)
//   3: group 0  W_a = IFFT(V_a)
// then all threads run the epilogue of both modes (same lags per thread as
// the one-group kernel, so the FP64 accumulators stay in registers).
template <int NP>
__device__ __forceinline__ void gather16(float2 (&x)[16], const float2* __restrict__ row, const int (&om)[8]) {
#pragma unroll
  for (int q = 0; q < 8; q++) x[q] = om[q] >= 0 ? row[om[q]] : make_float2(0.f, 0.f);
#pragma unroll
  for (int q = 8; q < 16; q++) x[q] = make_float2(0.f, 0.f);
}

template <int NP>
__device__ __forceinline__ void spectrum16(float2 (&v)[16], int t, const float2* __restrict__ Y,
                                           const float2* __restrict__ Z, const float2* __restrict__ mspec,
                                           bool second) {
  constexpr int NTG = NP / 16;
#pragma unroll
  for (int q = 0; q < 16; q++) {
    const int k = t + q * NTG;
    const float2 y = Y[pad16(k)];
    const float2 zk = Z[pad16(k)];
    const float2 zn = Z[pad16((NP - k) & (NP - 1))];
    const float2 M = __ldg(&mspec[k]);
    const float Px = second ? 0.5f * (zk.y + zn.y) : 0.5f * (zk.x + zn.x);
    const float Py = second ? -0.5f * (zk.x - zn.x) : 0.5f * (zk.y - zn.y);
    const float S = fmaf(y.x, y.x, y.y * y.y);
    const float R = 2.f * fmaf(M.x, Px, M.y * Py);
    v[q] = make_float2(S, R);
  }
}

template <int NP, int LPT>
__global__ void __launch_bounds__(NP / 8, TemporalBounds<NP>::MIN_BLOCKS) temporal16_kernel(TemporalParams p) {
  constexpr int NTG = NP / 16;  // threads per group
  constexpr int NTH = 2 * NTG;  // threads per CTA
  extern __shared__ __align__(16) float2 sm[];
  float2* bufG0 = sm;
  float2* bufG1 = sm + NP;
  float2* bufZ = sm + 2 * NP;
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ int s_next;
  const int t = threadIdx.x;
  const int g = t / NTG, tl = t % NTG;
  const int TS = p.T;                 // staging stride: the (largest) T
  float2* stage = sm + 3 * NP;        // [2 buffers][2 rows][TS]
  float2* s_tw = stage + 4 * TS;      // per-stage twiddle blocks (radix-16 plan)
  float* s_np = (float*)(s_tw + tw_size16(NP));
  const float invn = 0.5f / NP;
  for (int i = t; i < tw_size16(NP); i += NTH) s_tw[i] = p.tw16[i];

  // per-video state (few registers: the FFTs need them): the slot of each
  // of this thread's samples, -1 where the mask drops it or beyond T
  const int4* v_items = nullptr;
  const float2* v_mspec = nullptr;
  double* v_partials = nullptr;
  int cur_v = -1, L = 0, v_unit0 = 0, v_nunits = 0;
  float np0 = 0.f;
  int om[8];
  auto load_video = [&](int vi) {
    const VideoDesc vd = video_of(p, vi);
    cur_v = vi;
    L = vd.L;
    v_items = vd.items;
    v_mspec = vd.mspec;
    v_partials = vd.partials;
    v_unit0 = vd.unit0;
    v_nunits = vd.nunits;
    np0 = vd.npairs[0];
    for (int i = t; i < L; i += NTH) s_np[i] = vd.npairs[i];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int i = tl + q * NTG;
      om[q] = (i < vd.T && __ldg(&vd.mask[i]) != 0.f) ? (int)__ldg(&vd.order[i]) : -1;
    }
  };
  if (t == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    fence_barrier_init();
    s_next = atomicAdd(p.unit_counter, 1);
  }
  __syncthreads();
  int u = s_next;
  __syncthreads();
  if (t == 0) {
    s_next = atomicAdd(p.unit_counter, 1);
    if (u < p.nunits) issue_pair(p, u, 0, stage, TS, &mbar[0]);
  }
  __syncthreads();
  int unext = s_next;
  int k = 0, buf = 0;
  uint32_t phase = 0;
  double acc[LPT][PFIELDS];
  double accP = 0.0;
#pragma unroll
  for (int r = 0; r < LPT; r++)
#pragma unroll
    for (int c = 0; c < PFIELDS; c++) acc[r][c] = 0.0;

  while (u < p.nunits) {
    const int4 U = p.units[u];
    const int vi = p.videos ? U.w : 0;
    if (vi != cur_v) {
      __syncthreads();
      load_video(vi);
      __syncthreads();
    }
    int nu = u, nk = k + 2;
    if (nk >= U.y) {
      nu = unext;
      nk = 0;
    }
    const bool prefetched = nu < p.nunits;
    if (t == 0 && prefetched) issue_pair(p, nu, nk, stage + (buf ^ 1) * 2 * TS, TS, &mbar[buf ^ 1]);
    if (!mbar_wait(&mbar[buf], (phase >> buf) & 1u, p.err, 1)) {
      if (prefetched) mbar_wait(&mbar[buf ^ 1], (phase >> (buf ^ 1)) & 1u, p.err, 1);
      return;
    }
    phase ^= 1u << buf;
    const float2* rowa = stage + buf * 2 * TS;
    const float2* rowb = rowa + TS;
    const bool hasb = k + 1 < U.y;
    const int4 ea = load_item(v_items, U.x + k);
    const int4 eb = hasb ? load_item(v_items, U.x + k + 1) : ea;
    float2 v[16];
    // step 1
    if (g == 0) {
      // p_a + i p_b at this thread's samples (T <= TPAD/2: q >= 8 is padding)
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const bool on = om[q] >= 0;
        const float2 xa = on ? rowa[om[q]] : make_float2(0.f, 0.f);
        const float2 xb = on && hasb ? rowb[om[q]] : make_float2(0.f, 0.f);
        v[q] = make_float2(fmaf(xa.x, xa.x, xa.y * xa.y), fmaf(xb.x, xb.x, xb.y * xb.y));
      }
#pragma unroll
      for (int q = 8; q < 16; q++) v[q] = make_float2(0.f, 0.f);
      fft16<NP, false>(v, tl, bufZ, s_tw, 1);
    } else if (hasb) {
      gather16<NP>(v, rowb, om);
      fft16<NP, false>(v, tl, bufG1, s_tw, 2);
    }
    __syncthreads();  // Z and Y_b complete
    const float2 zsum = bufZ[0];  // (sum p_a, sum p_b)
    // step 2
    if (g == 0) {
      gather16<NP>(v, rowa, om);
      fft16<NP, false>(v, tl, bufG0, s_tw, 1);
    } else if (hasb) {
      spectrum16<NP>(v, tl, bufG1, bufZ, v_mspec, true);
      fft16<NP, true>(v, tl, bufG1, s_tw, 2);
    }
    // step 3 (group 0 only: its own barriers order Y_a)
    if (g == 0) {
      spectrum16<NP>(v, tl, bufG0, bufZ, v_mspec, false);
      fft16<NP, true>(v, tl, bufG0, s_tw, 1);
    }
    __syncthreads();  // W_a, W_b complete
#pragma unroll 1
    for (int s = 0; s < 2; s++) {
      if (s == 1 && !hasb) break;
      const int4 e = s ? eb : ea;
      const float2* W = s ? bufG1 : bufG0;
      const float ps = s ? zsum.y : zsum.x;
      const float P = np0 > 0.5f ? ps / np0 : 0.f;
      const double kx = e.y, ky = e.z;
#pragma unroll
      for (int r = 0; r < LPT; r++) {
        const int tau = t + r * NTH;
        if (tau < L) {
          const float n0 = s_np[tau];
          const float inp = n0 > 0.5f ? 1.f / n0 : 0.f;
          const float2 w0 = W[pad16(tau)];
          const float2 w1 = W[pad16((NP - tau) & (NP - 1))];
          const float gx = (w0.x + w1.x) * invn, gy = (w0.y - w1.y) * invn;
          const float ee = (w0.y + w1.y) * invn;
          acc[r][0] += (double)((ee - 2.f * gx) * inp);
          if (tau + 1 < L) {
            const float n1 = s_np[tau + 1];
            const float inp1 = n1 > 0.5f ? 1.f / n1 : 0.f;
            const float2 u0 = W[pad16(tau + 1)];
            const float2 u1 = W[pad16((NP - tau - 1) & (NP - 1))];
            const float cx = gx * inp, cy = gy * inp;
            const float c1x = (u0.x + u1.x) * invn * inp1;
            const float c1y = (u0.y - u1.y) * invn * inp1;
            const float zr = fmaf(c1x, cx, c1y * cy);  // C(tau+1) conj C(tau)
            const float zi = fmaf(c1y, cx, -c1x * cy);
            const float wgt = sqrtf(fmaf(zr, zr, zi * zi));
            if (wgt > 0.f) {
              const double wd = wgt, ph = atan2f(zi, zr);
              acc[r][1] += wd;
              acc[r][2] += wd * kx * kx;
              acc[r][3] += wd * kx * ky;
              acc[r][4] += wd * ky * ky;
              acc[r][5] += wd * kx * ph;
              acc[r][6] += wd * ky * ph;
              acc[r][7] += wd * ph * ph;
              acc[r][8] += 1.0;
            }
          }
        }
      }
      accP += (double)P;
    }
    if (k + 2 >= U.y) {
      const int ul = u - v_unit0;
#pragma unroll
      for (int r = 0; r < LPT; r++) {
        const int tau = t + r * NTH;
        if (tau < L)
#pragma unroll
          for (int c = 0; c < PFIELDS; c++) {
            v_partials[((size_t)ul * PFIELDS + c) * L + tau] = acc[r][c];
            acc[r][c] = 0.0;
          }
      }
      if (t == 0) v_partials[(size_t)v_nunits * PFIELDS * L + ul] = accP;
      accP = 0.0;
      u = unext;
      k = 0;
      if (t == 0) s_next = atomicAdd(p.unit_counter, 1);
    } else {
      k += 2;
    }
    buf ^= 1;
    fence_proxy_async_smem();  // this CTA's reads of the staged rows before the next TMA write
    __syncthreads();           // also: the epilogue is done with bufG0/G1 before the next pair
    unext = s_next;
  }
}

// ---------------------------------------------------------------------------
// One-group radix-16 kernel for TPAD 8192, where the staged kernels above do
// not fit shared memory (three exchange buffers of 64 KB plus 128 KB of
// staged rows). NP/16 = 512 threads, 16 points per thread, in-place
// exchange buffers: F for the transforms of one mode, Z for the packed p
// spectrum of the pair (2 x 64 KB), and one staging buffer for the pair's two
// time series (bulk copy, 2 x T x 8 B <= 64 KB): the next pair's copy is
// issued as soon as the last gather of this pair is done, so it lands while
// this pair's remaining transforms and epilogue run. Twiddles come from the
// FP64-derived radix-16 table through L1. Per pair (a, b), as above:
//   Z = FFT(p_a + i p_b);  for s in (a, b): Y = FFT(x_s), W = IFFT(V_s)
// with V_s = |Y|^2 + i 2 Re(conj(M) P_s), then the fused radial epilogue or
// the full per-mode outputs.
template <int NP, int LPT, bool FULL>
__global__ void __launch_bounds__(NP / 16, 1) temporal_big_kernel(TemporalParams p) {
  constexpr int NTH = NP / 16;
  extern __shared__ __align__(16) float2 sm[];
  float2* bufF = sm;
  float2* bufZ = sm + NP;
  const int TS = p.T;             // staging stride: the (largest) T
  float2* stage = sm + 2 * NP;    // [2 rows][TS]
  float* s_np = (float*)(stage + 2 * TS);
  __shared__ __align__(8) uint64_t mbar;
  __shared__ int s_next;
  const int t = threadIdx.x;
  const float invn = 0.5f / NP;
  const float2* __restrict__ tw = p.tw16;

  const int4* v_items = nullptr;
  const float2* v_mspec = nullptr;
  double* v_partials = nullptr;
  int cur_v = -1, L = 0, v_unit0 = 0, v_nunits = 0;
  float np0 = 0.f;
  int om[8];  // slot of each of this thread's samples, -1 where masked or beyond T
  auto load_video = [&](int vi) {
    const VideoDesc vd = video_of(p, vi);
    cur_v = vi;
    L = vd.L;
    v_items = vd.items;
    v_mspec = vd.mspec;
    v_partials = vd.partials;
    v_unit0 = vd.unit0;
    v_nunits = vd.nunits;
    np0 = vd.npairs[0];
    for (int i = t; i < L; i += NTH) s_np[i] = vd.npairs[i];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int i = t + q * NTH;
      om[q] = (i < vd.T && __ldg(&vd.mask[i]) != 0.f) ? (int)__ldg(&vd.order[i]) : -1;
    }
  };
  if (t == 0) {
    mbar_init(&mbar, 1);
    fence_barrier_init();
    s_next = atomicAdd(p.unit_counter, 1);
  }
  __syncthreads();
  int u = s_next;
  __syncthreads();
  if (t == 0) {
    s_next = atomicAdd(p.unit_counter, 1);
    if (u < p.nunits) issue_pair(p, u, 0, stage, TS, &mbar);
  }
  __syncthreads();
  int unext = s_next;
  uint32_t phase = 0;
  int k = 0;
  double acc[LPT][PFIELDS];
  double accP = 0.0;
#pragma unroll
  for (int r = 0; r < LPT; r++)
#pragma unroll
    for (int c = 0; c < PFIELDS; c++) acc[r][c] = 0.0;

  while (u < p.nunits) {
    const int4 U = p.units[u];
    const int vi = p.videos ? U.w : 0;
    if (vi != cur_v) {
      __syncthreads();  // s_np is no longer read
      load_video(vi);
      __syncthreads();
    }
    if (!mbar_wait(&mbar, phase, p.err, 1)) return;  // nothing else is in flight
    phase ^= 1u;
    const bool hasb = k + 1 < U.y;
    const int4 ea = load_item(v_items, U.x + k);
    const int4 eb = hasb ? load_item(v_items, U.x + k + 1) : ea;
    const float2* rowa = stage;
    const float2* rowb = stage + TS;
    float2 v[16];
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const bool on = om[q] >= 0;
      const float2 xa = on ? rowa[om[q]] : make_float2(0.f, 0.f);
      const float2 xb = on && hasb ? rowb[om[q]] : make_float2(0.f, 0.f);
      v[q] = make_float2(fmaf(xa.x, xa.x, xa.y * xa.y), fmaf(xb.x, xb.x, xb.y * xb.y));
    }
#pragma unroll
    for (int q = 8; q < 16; q++) v[q] = make_float2(0.f, 0.f);
    fft16<NP, false>(v, t, bufZ, tw, 0);  // ends with a barrier after its last store
    const float2 zsum = bufZ[0];          // (sum p_a, sum p_b)

#pragma unroll 1
    for (int s = 0; s < 2; s++) {
      if (s == 1 && !hasb) break;
      const int4 e = s ? eb : ea;
      const float2* row = s ? rowb : rowa;
#pragma unroll
      for (int q = 0; q < 8; q++) v[q] = om[q] >= 0 ? row[om[q]] : make_float2(0.f, 0.f);
#pragma unroll
      for (int q = 8; q < 16; q++) v[q] = make_float2(0.f, 0.f);
      if (s == 1 || !hasb) {
        // the pair's last gather: every thread is done with the staged rows,
        // so the next pair's copy may land there while this one finishes
        fence_proxy_async_smem();
        __syncthreads();
        int nu = u, nk = k + 2;
        if (nk >= U.y) {
          nu = unext;
          nk = 0;
        }
        if (t == 0 && nu < p.nunits) issue_pair(p, nu, nk, stage, TS, &mbar);
      }
      // the first store of each transform waits for the whole CTA, so the
      // previous readers of F (epilogue, spectrum) are done by then
      fft16<NP, false>(v, t, bufF, tw, 0);
      spectrum16<NP>(v, t, bufF, bufZ, v_mspec, s == 1);
      fft16<NP, true>(v, t, bufF, tw, 0);
      const float2* W = bufF;
      const float ps = s ? zsum.y : zsum.x;
      const float P = np0 > 0.5f ? ps / np0 : 0.f;
      if (FULL) {
        const size_t mode = (size_t)e.x;
        for (int tau = t; tau < L; tau += NTH) {
          const float np = s_np[tau];
          const float inv = np > 0.5f ? 1.f / np : 0.f;
          const float2 w0 = W[pad16(tau)];
          const float2 w1 = W[pad16((NP - tau) & (NP - 1))];
          const float gx = (w0.x + w1.x) * invn, gy = (w0.y - w1.y) * invn;
          const float ee = (w0.y + w1.y) * invn;
          p.outD[mode * L + tau] = (ee - 2.f * gx) * inv;
          p.outC[mode * L + tau] = make_float2(gx * inv, gy * inv);
        }
        if (t == 0) p.outP[mode] = P;
      } else {
        const double kx = e.y, ky = e.z;
#pragma unroll
        for (int r = 0; r < LPT; r++) {
          const int tau = t + r * NTH;
          if (tau < L) {
            const float n0 = s_np[tau];
            const float inp = n0 > 0.5f ? 1.f / n0 : 0.f;
            const float2 w0 = W[pad16(tau)];
            const float2 w1 = W[pad16((NP - tau) & (NP - 1))];
            const float gx = (w0.x + w1.x) * invn, gy = (w0.y - w1.y) * invn;
            const float ee = (w0.y + w1.y) * invn;
            acc[r][0] += (double)((ee - 2.f * gx) * inp);
            if (tau + 1 < L) {
              const float n1 = s_np[tau + 1];
              const float inp1 = n1 > 0.5f ? 1.f / n1 : 0.f;
              const float2 u0 = W[pad16(tau + 1)];
              const float2 u1 = W[pad16((NP - tau - 1) & (NP - 1))];
              const float cx = gx * inp, cy = gy * inp;
              const float c1x = (u0.x + u1.x) * invn * inp1;
              const float c1y = (u0.y - u1.y) * invn * inp1;
              const float zr = fmaf(c1x, cx, c1y * cy);  // C(tau+1) conj C(tau)
              const float zi = fmaf(c1y, cx, -c1x * cy);
              const float wgt = sqrtf(fmaf(zr, zr, zi * zi));
              if (wgt > 0.f) {
                const double wd = wgt, ph = atan2f(zi, zr);
                acc[r][1] += wd;
                acc[r][2] += wd * kx * kx;
                acc[r][3] += wd * kx * ky;
                acc[r][4] += wd * ky * ky;
                acc[r][5] += wd * kx * ph;
                acc[r][6] += wd * ky * ph;
                acc[r][7] += wd * ph * ph;
                acc[r][8] += 1.0;
              }
            }
          }
        }
        accP += (double)P;
      }
    }
    if (k + 2 >= U.y) {
      if (!FULL) {
        const int ul = u - v_unit0;
#pragma unroll
        for (int r = 0; r < LPT; r++) {
          const int tau = t + r * NTH;
          if (tau < L)
#pragma unroll
            for (int c = 0; c < PFIELDS; c++) {
              v_partials[((size_t)ul * PFIELDS + c) * L + tau] = acc[r][c];
              acc[r][c] = 0.0;
            }
        }
        if (t == 0) v_partials[(size_t)v_nunits * PFIELDS * L + ul] = accP;
        accP = 0.0;
      }
      u = unext;
      k = 0;
      if (t == 0) s_next = atomicAdd(p.unit_counter, 1);
    } else {
      k += 2;
    }
    __syncthreads();  // the epilogue is done with F; s_next is complete
    unext = s_next;
  }
}

// ---------------------------------------------------------------------------
// Sparse-mask variant (videos whose binary masks drop at most SPARSE_ZMAX
// time indices each, as recordings with a few missing frames): A + B comes
// from the time domain instead of a transform. With p(t) = m(t)|x(t)|^2 (zero
// at the masked t, and zero outside [0, T)) and S(n) = sum_{t<n} p(t),
//   A(tau) = sum_t m(t+tau) p(t) = S(T - tau) - sum_{d in Z} p(d - tau)
//   B(tau) = sum_t m(t) p(t+tau) = S(T) - S(tau) - sum_{d in Z} p(d + tau)
// over the masked set Z -- exact, and cheaper than FFT(p) and the inverse
// transform of conj(M) P while |Z| is small. The two modes of a pair then
// share ONE inverse transform, of |Y_a|^2 + i |Y_b|^2 (both real, so
// W = n (G_a + i G_b) splits by W(tau) +- conj W(-tau)): three transforms per
// pair instead of five, 1.5 per mode. Same staging, unit scheduling and
// epilogues as temporal_kernel; in batched launches a CTA reloads the video's
// tables (zero list, 1/N(tau), order and mask) when its unit changes video.
// Layout: p of the pair interleaved (p_a, p_b) in a zero-padded shared row
// (PADL zeros either side, PADL >= every lag a thread touches), so each
// correction term is one unconditional 8-byte load serving both modes and
// summed in FP32 (at most 2 SPARSE_ZMAX terms); S in FP64, scanned per pair
// into the exchange buffer the inverse transform leaves free (2 T doubles
// <= TPAD float2 as T <= TPAD / 2).
__host__ __device__ constexpr int sparse_padl(int NP, int L, int LPT) {
  return ((L > LPT * (NP / 8) ? L : LPT * (NP / 8)) + 1) & ~1;  // even: pz stays 16-byte aligned
}
// Slot of S(j + 1) in the scan buffer: a permutation inside aligned groups of
// four, so the scan's stores (thread t: j = 4t + e) hit eight distinct 16-byte
// bank groups per quarter-warp while consecutive-j reads stay conflict-free.
__device__ __forceinline__ int sparse_sidx(int j) { return j ^ ((j >> 3) & 3); }

// Twiddles of the sparse kernel's transforms: W^1 from the FP64-derived table,
// the higher powers of a radix-8 stage as products (one shared load instead
// of seven). Measured at 512^2 x 1024: 1.100 -> 1.059 ms per video; radial D
// moves by 1.8e-7 of each bin's scale.
#ifndef SPARSE_TW_REC
#define SPARSE_TW_REC 1
#endif
template <int NP, int LPT, bool FULL>
__global__ void __launch_bounds__(NP / 8, TemporalBounds<NP>::MIN_BLOCKS)
    temporal_sparse_kernel(TemporalParams p) {
  constexpr int NT = NP / 8;
  constexpr int PN = padded(NP);
  constexpr int WARPS = NT / 32;
  static_assert(NT % 32 == 0 && WARPS >= 1, "whole warps (TPAD >= 256)");
  extern __shared__ __align__(16) float2 sm[];
  float2* bufA = sm;
  float2* bufB = sm + PN;
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ int s_next, s_nz;
  __shared__ int s_zero[SPARSE_ZMAX];
  __shared__ double s_wt[2][WARPS];
  const int t = threadIdx.x;
  const int TS = p.T;                              // staging stride: the (largest) T
  const int PADL = sparse_padl(NP, p.L, LPT);      // p.L: the (largest) L
  float2* stage = sm + 2 * PN;                     // [2 buffers][2 rows][TS]
  float2* s_tw = stage + 4 * TS;                   // per-stage twiddle blocks
  float2* s_pp = s_tw + tw_size(NP);               // [PADL + TS + PADL] (p_a, p_b)
  float* s_inp = (float*)(s_pp + TS + 2 * PADL);   // 1 / N(tau) (0 where N = 0), tau < L
  float2* pz = s_pp + PADL;                        // pz[j] = p at time index j
  const float invn = 0.5f / NP;
  for (int i = t; i < tw_size(NP); i += NT) s_tw[i] = p.tw[i];

  // per-video state: tables in shared memory, the slot and mask of this
  // thread's samples, the masked time indices
  const int4* v_items = nullptr;
  double* v_partials = nullptr;
  int cur_v = -1, L = 0, T = 0, v_unit0 = 0, v_nunits = 0, nz = 0;
  float np0 = 0.f;
  uint32_t ord[4];
  float msk[4];
  auto load_video = [&](int vi) {  // between two CTA barriers
    const VideoDesc vd = video_of(p, vi);
    cur_v = vi;
    L = vd.L;
    T = vd.T;
    v_items = vd.items;
    v_partials = vd.partials;
    v_unit0 = vd.unit0;
    v_nunits = vd.nunits;
    np0 = vd.npairs[0];
    for (int i = t; i < TS + 2 * PADL; i += NT) s_pp[i] = make_float2(0.f, 0.f);
    for (int i = t; i < L; i += NT) {
      const float n = vd.npairs[i];
      s_inp[i] = n > 0.5f ? 1.f / n : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int i = t + q * NT;
      ord[q] = i < T ? __ldg(&vd.order[i]) : 0u;
      msk[q] = i < T ? __ldg(&vd.mask[i]) : 0.f;
    }
    if (t < 32) {  // the masked time indices, ascending (one warp, ballots)
      int n = 0;
      for (int j0 = 0; j0 < T; j0 += 32) {
        const bool z = j0 + t < T && __ldg(&vd.mask[j0 + t]) == 0.f;
        const unsigned b = __ballot_sync(0xffffffffu, z);
        if (z) {
          const int at = n + __popc(b & ((1u << t) - 1u));
          if (at < SPARSE_ZMAX) s_zero[at] = j0 + t;
        }
        n += __popc(b);
      }
      if (t == 0) {
        // the host picks this kernel for masks within SPARSE_ZMAX zeros; a
        // replayed launch whose tables changed since is reported, not run
        if (n > SPARSE_ZMAX) atomicExch(p.err, 4);
        s_nz = n > SPARSE_ZMAX ? -1 : n;
      }
    }
  };
  if (t == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    fence_barrier_init();
    s_next = atomicAdd(p.unit_counter, 1);
  }
  __syncthreads();
  int u = s_next;
  __syncthreads();
  if (t == 0) {
    s_next = atomicAdd(p.unit_counter, 1);
    if (u < p.nunits) issue_pair(p, u, 0, stage, TS, &mbar[0]);
  }
  __syncthreads();
  int unext = s_next;
  int k = 0, buf = 0;
  uint32_t phase = 0;
  double acc[LPT][PFIELDS];
  double accP = 0.0;
#pragma unroll
  for (int r = 0; r < LPT; r++)
#pragma unroll
    for (int c = 0; c < PFIELDS; c++) acc[r][c] = 0.0;

  while (u < p.nunits) {
    const int4 U = p.units[u];
    const int vi = p.videos ? U.w : 0;
    if (vi != cur_v) {
      __syncthreads();  // the previous video's shared tables are no longer read
      load_video(vi);
      __syncthreads();
      nz = s_nz;
      if (nz < 0) {  // more masked indices than the kernel holds: stop (reported)
        if (t == 0) mbar_wait(&mbar[buf], (phase >> buf) & 1u, nullptr, 0);  // the copy in flight
        return;
      }
    }
    int nu = u, nk = k + 2;
    if (nk >= U.y) {
      nu = unext;
      nk = 0;
    }
    const bool prefetched = nu < p.nunits;
    if (t == 0 && prefetched) issue_pair(p, nu, nk, stage + (buf ^ 1) * 2 * TS, TS, &mbar[buf ^ 1]);
    if (!mbar_wait(&mbar[buf], (phase >> buf) & 1u, p.err, 1)) {
      if (prefetched) mbar_wait(&mbar[buf ^ 1], (phase >> (buf ^ 1)) & 1u, p.err, 1);
      return;
    }
    phase ^= 1u << buf;
    const float2* rowa = stage + buf * 2 * TS;
    const float2* rowb = rowa + TS;
    const bool hasb = k + 1 < U.y;
    const int4 ea = load_item(v_items, U.x + k);
    const int4 eb = hasb ? load_item(v_items, U.x + k + 1) : ea;
    float2 v[8];
    float pa[4], sa[8];
    // mode a: p_a(t) and Y_a = FFT(x_a); |Y_a|^2 kept in registers
    gather<NP>(v, rowa, ord, msk);
#pragma unroll
    for (int q = 0; q < 4; q++) pa[q] = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
    {
      const float2* Y = fft<NP, false, true, SYNC_CTA, SPARSE_TW_REC>(v, t, bufA, bufB, s_tw);
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const float2 y = Y[pad(t + q * NT)];
        sa[q] = fmaf(y.x, y.x, y.y * y.y);
      }
    }
    __syncthreads();  // Y_a read before the next transform writes the buffers
    // mode b (zeros for the odd last mode of a unit)
    if (hasb)
      gather<NP>(v, rowb, ord, msk);
    else
#pragma unroll
      for (int q = 0; q < 8; q++) v[q] = make_float2(0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int j = t + q * NT;
      if (j < T) pz[j] = make_float2(pa[q], fmaf(v[q].x, v[q].x, v[q].y * v[q].y));
    }
    {
      const float2* Y = fft<NP, false, true, SYNC_CTA, SPARSE_TW_REC>(v, t, bufA, bufB, s_tw);
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const float2 y = Y[pad(t + q * NT)];
        v[q] = make_float2(sa[q], fmaf(y.x, y.x, y.y * y.y));
      }
    }
    __syncthreads();
    const float2* W = fft<NP, true, true, SYNC_CTA, SPARSE_TW_REC>(v, t, bufA, bufB, s_tw);
    // S(j + 1) of both modes at Sd[sparse_sidx(j)] (slots < T rounded up to
    // 4 <= TPAD / 2): thread t sums time indices 4t..4t+3, warps scan, warp
    // totals combine through shared memory
    double2* Sd = reinterpret_cast<double2*>(W == bufA ? bufB : bufA);
    {
      double2 loc[4];
      double ra = 0.0, rb = 0.0;
      // four consecutive (p_a, p_b) as two 16-byte loads (T even: a pair is
      // either inside [0, T) or wholly beyond it)
      float4 q2[2];
#pragma unroll
      for (int h = 0; h < 2; h++)
        q2[h] = 4 * t + 2 * h < T ? reinterpret_cast<const float4*>(pz)[2 * t + h] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const float4 q = q2[e >> 1];
        ra += (double)((e & 1) ? q.z : q.x);
        rb += (double)((e & 1) ? q.w : q.y);
        loc[e] = make_double2(ra, rb);
      }
      double ta = ra, tb = rb;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double ya = __shfl_up_sync(0xffffffffu, ta, o);
        const double yb = __shfl_up_sync(0xffffffffu, tb, o);
        if ((t & 31) >= o) {
          ta += ya;
          tb += yb;
        }
      }
      if ((t & 31) == 31) {
        s_wt[0][t >> 5] = ta;
        s_wt[1][t >> 5] = tb;
      }
      __syncthreads();
      double ba = ta - ra, bb = tb - rb;  // inclusive scan minus this thread's own sums
      for (int w = 0; w < (t >> 5); w++) {
        ba += s_wt[0][w];
        bb += s_wt[1][w];
      }
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int j = 4 * t + e;
        if (j < T) Sd[sparse_sidx(j)] = make_double2(ba + loc[e].x, bb + loc[e].y);
      }
      __syncthreads();
    }
    const double2 ST = Sd[sparse_sidx(T - 1)];
    // E(tau) = A + B of both modes
    auto base_of = [&](int tau) {
      const double2 s1 = tau > 0 ? Sd[sparse_sidx(tau - 1)] : make_double2(0.0, 0.0);
      const double2 s2 = T - tau > 0 ? Sd[sparse_sidx(T - tau - 1)] : make_double2(0.0, 0.0);
      return make_double2(ST.x - s1.x + s2.x, ST.y - s1.y + s2.y);
    };
    // G of mode s from the shared transform: W = n (G_a + i G_b)
    auto G_of = [&](int s, int tau, float& gx, float& gy) {
      const float2 w0 = W[pad(tau)];
      const float2 w1 = W[pad((NP - tau) & (NP - 1))];
      if (s == 0) {
        gx = (w0.x + w1.x) * invn;
        gy = (w0.y - w1.y) * invn;
      } else {
        gx = (w0.y + w1.y) * invn;
        gy = (w1.x - w0.x) * invn;
      }
    };
    if (FULL) {
      for (int tau = t; tau < L; tau += NT) {
        float2 cr = make_float2(0.f, 0.f);
        for (int z = 0; z < nz; z++) {
          const int d = s_zero[z];
          const float2 lo = pz[d - tau], hi = pz[d + tau];
          cr.x += lo.x + hi.x;
          cr.y += lo.y + hi.y;
        }
        const double2 E0 = base_of(tau);
        const float inv = s_inp[tau];
#pragma unroll
        for (int s = 0; s < 2; s++) {
          if (s == 1 && !hasb) break;
          const size_t mode = (size_t)(s ? eb : ea).x;
          const double E = s ? E0.y - (double)cr.y : E0.x - (double)cr.x;
          float gx, gy;
          G_of(s, tau, gx, gy);
          p.outD[mode * L + tau] = (float)((E - 2.0 * gx) * inv);
          p.outC[mode * L + tau] = make_float2(gx * inv, gy * inv);
        }
      }
      if (t == 0) {
        p.outP[(size_t)ea.x] = np0 > 0.5f ? (float)(ST.x / np0) : 0.f;
        if (hasb) p.outP[(size_t)eb.x] = np0 > 0.5f ? (float)(ST.y / np0) : 0.f;
      }
    } else {
      float2 cr[LPT];
#pragma unroll
      for (int r = 0; r < LPT; r++) cr[r] = make_float2(0.f, 0.f);
      for (int z = 0; z < nz; z++) {
        const int d = s_zero[z];
        const float2* lo = pz + (d - t);  // lo[-r NT] = p(d - tau)
        const float2* hi = pz + (d + t);  // hi[r NT] = p(d + tau)
#pragma unroll
        for (int r = 0; r < LPT; r++) {
          const float2 a = lo[-r * NT], b = hi[r * NT];
          cr[r].x += a.x + b.x;
          cr[r].y += a.y + b.y;
        }
      }
      double2 E[LPT];
#pragma unroll
      for (int r = 0; r < LPT; r++) {
        const int tau = t + r * NT;
        const double2 E0 = base_of(tau < L ? tau : 0);
        E[r] = make_double2(E0.x - (double)cr[r].x, E0.y - (double)cr[r].y);
      }
      // lag-major: W(tau), W(-tau) (and at tau + 1) are read once for both
      // modes of the pair; per lag the modes still add in the order a, b
#pragma unroll
      for (int r = 0; r < LPT; r++) {
        const int tau = t + r * NT;
        if (tau < L) {
          const float inp = s_inp[tau];
          const bool next = tau + 1 < L;
          const float inp1 = next ? s_inp[tau + 1] : 0.f;
          const float2 w0 = W[pad(tau)], w1 = W[pad((NP - tau) & (NP - 1))];
          const float2 u0 = next ? W[pad(tau + 1)] : make_float2(0.f, 0.f);
          const float2 u1 = next ? W[pad((NP - tau - 1) & (NP - 1))] : make_float2(0.f, 0.f);
#pragma unroll 1
          for (int s = 0; s < 2; s++) {
            if (s == 1 && !hasb) break;
            const int4 e = s ? eb : ea;
            const double kx = e.y, ky = e.z;
            // G of mode s from the shared transform: W = n (G_a + i G_b)
            const float gx = (s ? w0.y + w1.y : w0.x + w1.x) * invn;
            const float gy = (s ? w1.x - w0.x : w0.y - w1.y) * invn;
            acc[r][0] += ((s ? E[r].y : E[r].x) - 2.0 * gx) * (double)inp;
            if (next) {
              const float g1x = (s ? u0.y + u1.y : u0.x + u1.x) * invn;
              const float g1y = (s ? u1.x - u0.x : u0.y - u1.y) * invn;
              const float cx = gx * inp, cy = gy * inp;
              const float c1x = g1x * inp1, c1y = g1y * inp1;
              const float zr = fmaf(c1x, cx, c1y * cy);  // C(tau+1) conj C(tau)
              const float zi = fmaf(c1y, cx, -c1x * cy);
              const float w = sqrtf(fmaf(zr, zr, zi * zi));
              if (w > 0.f) {
                const double wd = w, ph = atan2f(zi, zr);
                acc[r][1] += wd;
                acc[r][2] += wd * kx * kx;
                acc[r][3] += wd * kx * ky;
                acc[r][4] += wd * ky * ky;
                acc[r][5] += wd * kx * ph;
                acc[r][6] += wd * ky * ph;
                acc[r][7] += wd * ph * ph;
                acc[r][8] += 1.0;
              }
            }
          }
        }
      }
      accP += np0 > 0.5f ? (double)(float)(ST.x / np0) : 0.0;
      if (hasb) accP += np0 > 0.5f ? (double)(float)(ST.y / np0) : 0.0;
    }
    if (k + 2 >= U.y) {
      if (!FULL) {
        const int ul = u - v_unit0;
#pragma unroll
        for (int r = 0; r < LPT; r++) {
          const int tau = t + r * NT;
          if (tau < L)
#pragma unroll
            for (int c = 0; c < PFIELDS; c++) {
              v_partials[((size_t)ul * PFIELDS + c) * L + tau] = acc[r][c];
              acc[r][c] = 0.0;
            }
        }
        if (t == 0) v_partials[(size_t)v_nunits * PFIELDS * L + ul] = accP;
        accP = 0.0;
      }
      u = unext;
      k = 0;
      if (t == 0) s_next = atomicAdd(p.unit_counter, 1);
    } else {
      k += 2;
    }
    buf ^= 1;
    fence_proxy_async_smem();  // this CTA's reads of the staged rows before the next TMA write
    __syncthreads();           // also: the epilogue is done with W, Sd and pz before the next pair
    unext = s_next;
  }
}

// ---------------------------------------------------------------------------
// Sparse-mask variant of temporal_big_kernel (TPAD 8192; same A + B from
// prefix sums and shared inverse transform as temporal_sparse_kernel). One
// group of TPAD/16 = 512 threads, 16 points per thread, in-place radix-16
// transforms in ONE 64 KB buffer:
//   Y_a = FFT(x_a) (|Y_a|^2 kept in registers); Y_b = FFT(x_b);
//   W = IFFT(|Y_a|^2 + i |Y_b|^2)
// -- three transforms per pair instead of five. The whole scan S does not
// fit beside the 64 KB staged pair, so only the values the lags use are
// kept: S(n) for n <= L (head) and n >= T - L (tail). Up to
// SPARSE_ZMAX_BIG masked indices (the host also bounds zeros x lags per
// thread, the corrections' cost).
__host__ __device__ constexpr int sparse_padl_big(int NP, int L, int LPT) {
  return ((L > LPT * (NP / 16) ? L : LPT * (NP / 16)) + 1) & ~1;
}

template <int NP, int LPT, bool FULL>
__global__ void __launch_bounds__(NP / 16, 1) temporal_sparse_big_kernel(TemporalParams p) {
  constexpr int NTH = NP / 16;
  constexpr int WARPS = NTH / 32;
  extern __shared__ __align__(16) float2 sm[];
  float2* bufF = sm;
  __shared__ __align__(8) uint64_t mbar;
  __shared__ int s_next, s_nz;
  __shared__ int s_zero[SPARSE_ZMAX_BIG];
  __shared__ double s_wt[2][WARPS];
  const int t = threadIdx.x;
  const float invn = 0.5f / NP;
  const float2* __restrict__ tw = p.tw16;
  const int TS = p.T;                              // staging stride: the (largest) T
  const int LM = p.L;                              // the (largest) L
  const int PADL = sparse_padl_big(NP, LM, LPT);
  float2* stage = sm + NP;                         // [2 rows][TS]
  float2* s_pp = stage + 2 * TS;                   // [PADL + TS + PADL] (p_a, p_b)
  float2* pz = s_pp + PADL;
  double2* Sh = reinterpret_cast<double2*>(s_pp + TS + 2 * PADL);  // S(n), n <= L
  double2* St = Sh + (LM + 1);                                     // S(T - L + m), m <= L
  float* s_inp = reinterpret_cast<float*>(St + (LM + 1));          // 1 / N(tau)

  const int4* v_items = nullptr;
  double* v_partials = nullptr;
  int cur_v = -1, L = 0, T = 0, v_unit0 = 0, v_nunits = 0, nz = 0;
  float np0 = 0.f;
  int om[8];  // slot of each of this thread's samples, -1 where masked or beyond T
  auto load_video = [&](int vi) {  // between two CTA barriers
    const VideoDesc vd = video_of(p, vi);
    cur_v = vi;
    L = vd.L;
    T = vd.T;
    v_items = vd.items;
    v_partials = vd.partials;
    v_unit0 = vd.unit0;
    v_nunits = vd.nunits;
    np0 = vd.npairs[0];
    for (int i = t; i < TS + 2 * PADL; i += NTH) s_pp[i] = make_float2(0.f, 0.f);
    for (int i = t; i < L; i += NTH) {
      const float n = vd.npairs[i];
      s_inp[i] = n > 0.5f ? 1.f / n : 0.f;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      const int i = t + q * NTH;
      om[q] = (i < T && __ldg(&vd.mask[i]) != 0.f) ? (int)__ldg(&vd.order[i]) : -1;
    }
    if (t < 32) {  // the masked time indices, ascending (one warp, ballots)
      int n = 0;
      for (int j0 = 0; j0 < T; j0 += 32) {
        const bool z = j0 + t < T && __ldg(&vd.mask[j0 + t]) == 0.f;
        const unsigned b = __ballot_sync(0xffffffffu, z);
        if (z) {
          const int at = n + __popc(b & ((1u << t) - 1u));
          if (at < SPARSE_ZMAX_BIG) s_zero[at] = j0 + t;
        }
        n += __popc(b);
      }
      if (t == 0) {
        if (n > SPARSE_ZMAX_BIG) atomicExch(p.err, 4);  // see temporal_sparse_kernel
        s_nz = n > SPARSE_ZMAX_BIG ? -1 : n;
      }
    }
  };
  if (t == 0) {
    mbar_init(&mbar, 1);
    fence_barrier_init();
    s_next = atomicAdd(p.unit_counter, 1);
  }
  __syncthreads();
  int u = s_next;
  __syncthreads();
  if (t == 0) {
    s_next = atomicAdd(p.unit_counter, 1);
    if (u < p.nunits) issue_pair(p, u, 0, stage, TS, &mbar);
  }
  __syncthreads();
  int unext = s_next;
  uint32_t phase = 0;
  int k = 0;
  double acc[LPT][PFIELDS];
  double accP = 0.0;
#pragma unroll
  for (int r = 0; r < LPT; r++)
#pragma unroll
    for (int c = 0; c < PFIELDS; c++) acc[r][c] = 0.0;

  while (u < p.nunits) {
    const int4 U = p.units[u];
    const int vi = p.videos ? U.w : 0;
    if (vi != cur_v) {
      __syncthreads();
      load_video(vi);
      __syncthreads();
      nz = s_nz;
      if (nz < 0) {  // more masked indices than the kernel holds: stop (reported)
        if (t == 0) mbar_wait(&mbar, phase, nullptr, 0);  // the copy in flight
        return;
      }
    }
    if (!mbar_wait(&mbar, phase, p.err, 1)) return;  // nothing else is in flight
    phase ^= 1u;
    const bool hasb = k + 1 < U.y;
    const int4 ea = load_item(v_items, U.x + k);
    const int4 eb = hasb ? load_item(v_items, U.x + k + 1) : ea;
    const float2* rowa = stage;
    const float2* rowb = stage + TS;
    float2 v[16];
    float sa[16];
    float* pzf = reinterpret_cast<float*>(pz);  // p_a at 2j, p_b at 2j + 1
    // mode a: p_a straight to shared memory (registers are short here) and
    // Y_a; |Y_a|^2 kept in registers
#pragma unroll
    for (int q = 0; q < 8; q++) {
      v[q] = om[q] >= 0 ? rowa[om[q]] : make_float2(0.f, 0.f);
      const int j = t + q * NTH;
      if (j < T) pzf[2 * j] = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
    }
#pragma unroll
    for (int q = 8; q < 16; q++) v[q] = make_float2(0.f, 0.f);
    fft16<NP, false>(v, t, bufF, tw, 0);  // ends with a barrier after its last store
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const float2 y = bufF[pad16(t + q * NTH)];
      sa[q] = fmaf(y.x, y.x, y.y * y.y);
    }
    // mode b: the pair's last gather, then the stage takes the next pair
#pragma unroll
    for (int q = 0; q < 8; q++) {
      v[q] = hasb && om[q] >= 0 ? rowb[om[q]] : make_float2(0.f, 0.f);
      const int j = t + q * NTH;
      if (j < T) pzf[2 * j + 1] = fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
    }
#pragma unroll
    for (int q = 8; q < 16; q++) v[q] = make_float2(0.f, 0.f);
    fence_proxy_async_smem();
    __syncthreads();
    {
      int nu = u, nk = k + 2;
      if (nk >= U.y) {
        nu = unext;
        nk = 0;
      }
      if (t == 0 && nu < p.nunits) issue_pair(p, nu, nk, stage, TS, &mbar);
    }
    // the first store of each transform waits for the group: the reads of
    // the buffer before it are done by then
    fft16<NP, false>(v, t, bufF, tw, 0);
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const float2 y = bufF[pad16(t + q * NTH)];
      v[q] = make_float2(sa[q], fmaf(y.x, y.x, y.y * y.y));
    }
    fft16<NP, true>(v, t, bufF, tw, 0);
    const float2* W = bufF;
    // S(n) of both modes at the head (n <= L) and tail (n >= T - L): thread
    // t sums time indices 8t..8t+7, warps scan, warp totals combine
    {
      // pass 1: this thread's sums; pass 2 (threads whose indices reach the
      // head or the tail) re-reads its 8 values to write the S(n) kept
      double ra = 0.0, rb = 0.0;
#pragma unroll
      for (int h = 0; h < 4; h++) {
        const float4 q = 8 * t + 2 * h < T ? reinterpret_cast<const float4*>(pz)[4 * t + h]
                                           : make_float4(0.f, 0.f, 0.f, 0.f);
        ra += (double)q.x;
        rb += (double)q.y;
        ra += (double)q.z;
        rb += (double)q.w;
      }
      double ta = ra, tb = rb;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double ya = __shfl_up_sync(0xffffffffu, ta, o);
        const double yb = __shfl_up_sync(0xffffffffu, tb, o);
        if ((t & 31) >= o) {
          ta += ya;
          tb += yb;
        }
      }
      if ((t & 31) == 31) {
        s_wt[0][t >> 5] = ta;
        s_wt[1][t >> 5] = tb;
      }
      __syncthreads();
      if (8 * t + 1 <= L || 8 * t + 8 >= T - L) {
        double ba = ta - ra, bb = tb - rb;  // exclusive prefix of this thread's indices
        for (int w = 0; w < (t >> 5); w++) {
          ba += s_wt[0][w];
          bb += s_wt[1][w];
        }
#pragma unroll
        for (int e = 0; e < 8; e++) {
          const int j = 8 * t + e;  // S(j + 1) = S(j) + p(j)
          if (j < T) {
            const float2 pv = pz[j];
            ba += (double)pv.x;
            bb += (double)pv.y;
            const int n = j + 1;
            const double2 sv = make_double2(ba, bb);
            if (n <= L) Sh[n] = sv;
            if (n >= T - L) St[n - (T - L)] = sv;
          }
        }
      }
      if (t == 0) {
        Sh[0] = make_double2(0.0, 0.0);
        if (T == L) St[0] = make_double2(0.0, 0.0);
      }
      __syncthreads();
    }
    const double2 ST = St[L];
    auto base_of = [&](int tau) {  // S(T) - S(tau) + S(T - tau), tau < L
      const double2 s1 = Sh[tau], s2 = St[L - tau];
      return make_double2(ST.x - s1.x + s2.x, ST.y - s1.y + s2.y);
    };
    auto G_of = [&](int s, int tau, float& gx, float& gy) {
      const float2 w0 = W[pad16(tau)];
      const float2 w1 = W[pad16((NP - tau) & (NP - 1))];
      if (s == 0) {
        gx = (w0.x + w1.x) * invn;
        gy = (w0.y - w1.y) * invn;
      } else {
        gx = (w0.y + w1.y) * invn;
        gy = (w1.x - w0.x) * invn;
      }
    };
    if (FULL) {
      for (int tau = t; tau < L; tau += NTH) {
        float2 cr = make_float2(0.f, 0.f);
#pragma unroll 4
        for (int z = 0; z < nz; z++) {
          const int d = s_zero[z];
          const float2 lo = pz[d - tau], hi = pz[d + tau];
          cr.x += lo.x + hi.x;
          cr.y += lo.y + hi.y;
        }
        const double2 E0 = base_of(tau);
        const float inv = s_inp[tau];
#pragma unroll
        for (int s = 0; s < 2; s++) {
          if (s == 1 && !hasb) break;
          const size_t mode = (size_t)(s ? eb : ea).x;
          const double E = s ? E0.y - (double)cr.y : E0.x - (double)cr.x;
          float gx, gy;
          G_of(s, tau, gx, gy);
          p.outD[mode * L + tau] = (float)((E - 2.0 * gx) * inv);
          p.outC[mode * L + tau] = make_float2(gx * inv, gy * inv);
        }
      }
      if (t == 0) {
        p.outP[(size_t)ea.x] = np0 > 0.5f ? (float)(ST.x / np0) : 0.f;
        if (hasb) p.outP[(size_t)eb.x] = np0 > 0.5f ? (float)(ST.y / np0) : 0.f;
      }
    } else {
      double2 E[LPT];
#pragma unroll
      for (int r = 0; r < LPT; r++) E[r] = make_double2(0.0, 0.0);
      if (t < L) {  // threads without a lag skip the corrections
        float2 cr[LPT];
#pragma unroll
        for (int r = 0; r < LPT; r++) cr[r] = make_float2(0.f, 0.f);
#pragma unroll 2
        for (int z = 0; z < nz; z++) {
          const int d = s_zero[z];
          const float2* lo = pz + (d - t);
          const float2* hi = pz + (d + t);
#pragma unroll
          for (int r = 0; r < LPT; r++) {
            const float2 a = lo[-r * NTH], b = hi[r * NTH];
            cr[r].x += a.x + b.x;
            cr[r].y += a.y + b.y;
          }
        }
#pragma unroll
        for (int r = 0; r < LPT; r++) {
          const int tau = t + r * NTH;
          const double2 E0 = base_of(tau < L ? tau : 0);
          E[r] = make_double2(E0.x - (double)cr[r].x, E0.y - (double)cr[r].y);
        }
      }
#pragma unroll 1
      for (int s = 0; s < 2; s++) {
        if (s == 1 && !hasb) break;
        const int4 e = s ? eb : ea;
        const double kx = e.y, ky = e.z;
#pragma unroll
        for (int r = 0; r < LPT; r++) {
          const int tau = t + r * NTH;
          if (tau < L) {
            const float inp = s_inp[tau];
            float gx, gy;
            G_of(s, tau, gx, gy);
            acc[r][0] += ((s ? E[r].y : E[r].x) - 2.0 * gx) * (double)inp;
            if (tau + 1 < L) {
              const float inp1 = s_inp[tau + 1];
              float g1x, g1y;
              G_of(s, tau + 1, g1x, g1y);
              const float cx = gx * inp, cy = gy * inp;
              const float c1x = g1x * inp1, c1y = g1y * inp1;
              const float zr = fmaf(c1x, cx, c1y * cy);  // C(tau+1) conj C(tau)
              const float zi = fmaf(c1y, cx, -c1x * cy);
              const float w = sqrtf(fmaf(zr, zr, zi * zi));
              if (w > 0.f) {
                const double wd = w, ph = atan2f(zi, zr);
                acc[r][1] += wd;
                acc[r][2] += wd * kx * kx;
                acc[r][3] += wd * kx * ky;
                acc[r][4] += wd * ky * ky;
                acc[r][5] += wd * kx * ph;
                acc[r][6] += wd * ky * ph;
                acc[r][7] += wd * ph * ph;
                acc[r][8] += 1.0;
              }
            }
          }
        }
        accP += np0 > 0.5f ? (double)(float)((s ? ST.y : ST.x) / np0) : 0.0;
      }
    }
    if (k + 2 >= U.y) {
      if (!FULL) {
        const int ul = u - v_unit0;
#pragma unroll
        for (int r = 0; r < LPT; r++) {
          const int tau = t + r * NTH;
          if (tau < L)
#pragma unroll
            for (int c = 0; c < PFIELDS; c++) {
              v_partials[((size_t)ul * PFIELDS + c) * L + tau] = acc[r][c];
              acc[r][c] = 0.0;
            }
        }
        if (t == 0) v_partials[(size_t)v_nunits * PFIELDS * L + ul] = accP;
        accP = 0.0;
      }
      u = unext;
      k = 0;
      if (t == 0) s_next = atomicAdd(p.unit_counter, 1);
    } else {
      k += 2;
    }
    __syncthreads();  // the epilogue is done with W, S and pz; s_next is complete
    unext = s_next;
  }
}

// Sums the unit partials of each bin in unit order (deterministic), divides
// D and P by the bin's mode count (ddm_ref.js:404-412) and writes the
// reference's Radial layout: D[b*L+tau], P[b], drift[(b*L+tau)*8+c] (or adds
// to it: the bands of a banded analysis after the first, in band order).
// Grid (lag blocks, bins), one thread per (bin, lag): the unit loop is
// unrolled so several units' loads are in flight (the sums still add in
// unit order).
__global__ void reduce_kernel(ReduceParams p) {
  const int b = blockIdx.y;
  const int L = p.L;
  const int tau = blockIdx.x * blockDim.x + threadIdx.x;
  const int u0 = p.bin_units[b], u1 = p.bin_units[b + 1];
  const double n = (double)p.nmodes[b];
  const double inv = n > 0 ? 1.0 / n : 0.0;
  if (tau < L) {
    double s[PFIELDS];
#pragma unroll
    for (int c = 0; c < PFIELDS; c++) s[c] = 0.0;
    const double* __restrict__ src = p.partials + tau;
#pragma unroll 4
    for (int u = u0; u < u1; u++)
#pragma unroll
      for (int c = 0; c < PFIELDS; c++) s[c] += __ldg(&src[((size_t)u * PFIELDS + c) * L]);
    double* dD = &p.D[(size_t)b * L + tau];
    *dD = p.accumulate ? *dD + s[0] * inv : s[0] * inv;
#pragma unroll
    for (int c = 0; c < DRIFT; c++) {
      double* d = &p.drift[((size_t)b * L + tau) * DRIFT + c];
      *d = p.accumulate ? *d + s[c + 1] : s[c + 1];
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double s = 0.0;
    for (int u = u0; u < u1; u++) s += p.partials[(size_t)p.nunits * PFIELDS * L + u];
    p.P[b] = p.accumulate ? p.P[b] + s * inv : s * inv;
  }
}

// Radial sums of full per-mode outputs (ddm.wgsl:265-322 with FP64 sums), in
// the fused path's work units: block (lag block, unit u) sums the unit's modes
// (a run of at most U modes of one bin, in table order) at its lags and
// writes the unit's partial record; reduce_kernel then adds the units of each
// bin in unit order -- the same reduction as the fused epilogue's, with a
// unit's loads all issued before its sums.
__device__ __forceinline__ void radial_full_add(double (&s)[PFIELDS], float D, float2 a, float2 c1, bool next,
                                                int4 e) {
  s[0] += (double)D;
  if (next) {
    const float zr = fmaf(c1.x, a.x, c1.y * a.y);
    const float zi = fmaf(c1.y, a.x, -c1.x * a.y);
    const float w = sqrtf(fmaf(zr, zr, zi * zi));
    if (w > 0.f) {
      const double wd = w, ph = atan2f(zi, zr), kx = e.y, ky = e.z;
      s[1] += wd;
      s[2] += wd * kx * kx;
      s[3] += wd * kx * ky;
      s[4] += wd * ky * ky;
      s[5] += wd * kx * ph;
      s[6] += wd * ky * ph;
      s[7] += wd * ph * ph;
      s[8] += 1.0;
    }
  }
}

__global__ void radial_full_kernel(RadialFullParams p) {
  const int u = blockIdx.y;
  const int L = p.L;
  const int tau = blockIdx.x * blockDim.x + threadIdx.x;
  const int4 U = p.units[u];
  if (tau < L) {
    double s[PFIELDS];
#pragma unroll
    for (int c = 0; c < PFIELDS; c++) s[c] = 0.0;
    const bool next = tau + 1 < L;
    constexpr int AH = 8;
    for (int k0 = 0; k0 < U.y; k0 += AH) {
      int4 e[AH];
      float D[AH];
      float2 a[AH], c1[AH];
#pragma unroll
      for (int k = 0; k < AH; k++) {
        e[k] = k0 + k < U.y ? __ldg(&p.items[U.x + k0 + k]) : make_int4(0, 0, 0, 0);
        const size_t m = (size_t)e[k].x;
        const bool in = k0 + k < U.y;
        D[k] = in ? __ldg(&p.D[m * L + tau]) : 0.f;
        a[k] = in ? __ldg(&p.C[m * L + tau]) : make_float2(0.f, 0.f);
        c1[k] = in && next ? __ldg(&p.C[m * L + tau + 1]) : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int k = 0; k < AH; k++)
        if (k0 + k < U.y) radial_full_add(s, D[k], a[k], c1[k], next, e[k]);
    }
#pragma unroll
    for (int c = 0; c < PFIELDS; c++) p.partials[((size_t)u * PFIELDS + c) * L + tau] = s[c];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < U.y; k++) s += (double)p.P[p.items[U.x + k].x];
    p.partials[(size_t)p.nunits * PFIELDS * L + u] = s;
  }
}

// ---------------------------------------------------------------------------
// Blocked masked Wiener-Khinchin for short lag ranges (L <= 128) on long
// series (TPAD 8192): only lags tau < L are needed, so the series is cut into
// blocks of BL = 128 samples and every correlation is assembled from
// 256-point transforms, one warp per mode, instead of three 8192-point
// transforms per pair. With x~ = m x (masked series), p = m |x|^2, block
// spectra X_b = FFT_256(x~_b zero-padded), P_b, M_b likewise (M: the mask), and
// s_k = (-1)^k (the shift of block b + 1 by BL inside a 2 BL transform):
//   G(tau)     = sum_t x~*(t) x~(t + tau)
//              = IFFT[ sum_b conj(X_b) (X_b + s_k X_{b+1}) ](tau)
//   A+B(tau)   = sum_t p(t) m(t + tau) + m(t) p(t + tau)
//              = IFFT[ sum_b conj(P_b) (M_b + s_k M_{b+1})
//                            + conj(M_b) (P_b + s_k P_{b+1}) ](tau)
// exact for tau < BL (the window of block b covers blocks b and b + 1). Per
// mode: one 256-point transform per block of x~, one per pair of blocks of p
// (two real blocks in one complex transform), two inverse transforms; the
// mask spectra M_b are computed once per CTA and video. D, C and P as the
// other kernels (ddm_ref.js:275-285); the radial epilogue runs over the
// CTA's threads (lag, quarter of the warps), FP64 sums in a fixed order.
constexpr int BLK_L = 128, BLK_F = 256;
#ifndef BLK_WARPS_N
#define BLK_WARPS_N 8
#endif
constexpr int BLK_WARPS = BLK_WARPS_N;  // modes in flight per CTA, one per warp
__host__ __device__ constexpr int blk_count(int T) { return (T + BLK_L - 1) / BLK_L; }
static size_t temporal_blocked_smem(int T) {
  return sizeof(float2) * ((size_t)(blk_count(T) + 1) * BLK_F    // mask block spectra (and a zero block)
                           + (size_t)BLK_WARPS * 2 * BLK_F        // per-warp transform buffers
                           + tw_size(BLK_F)) +                    // 256-point twiddles
         sizeof(float4) * (size_t)BLK_WARPS * BLK_L +               // per-warp (A+B, G) by lag
         sizeof(double) * (size_t)(BLK_WARPS * 32 / BLK_L) * PFIELDS * BLK_L +  // partial sums to combine
         sizeof(float) * (BLK_L + BLK_WARPS);                       // 1/N(tau), P per warp
}

__global__ void __launch_bounds__(32 * BLK_WARPS, 1) temporal_blocked_kernel(TemporalParams p) {
  constexpr int NTH = 32 * BLK_WARPS;
  constexpr int QG = NTH / BLK_L;  // thread groups per lag in the epilogue
  constexpr int WPG = BLK_WARPS / QG;  // warps (modes) per group
  extern __shared__ __align__(16) float2 sm[];
  __shared__ int s_next;
  const int TS = p.T;  // the (largest) T: sizes the mask-spectrum table
  float2* s_M = sm;                                        // [(nblk + 1)][BLK_F]
  float2* s_buf = s_M + (size_t)(blk_count(TS) + 1) * BLK_F; // [warp][2][BLK_F]
  float2* s_tw = s_buf + BLK_WARPS * 2 * BLK_F;
  float4* s_E = reinterpret_cast<float4*>(s_tw + tw_size(BLK_F));  // [warp][BLK_L] (ab, g.x, g.y, -)
  double* s_acc = reinterpret_cast<double*>(s_E + BLK_WARPS * BLK_L);  // [QG][PFIELDS][BLK_L]
  float* s_inp = reinterpret_cast<float*>(s_acc + QG * PFIELDS * BLK_L);
  float* s_P = s_inp + BLK_L;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  float2* b0 = s_buf + warp * 2 * BLK_F;
  float2* b1 = b0 + BLK_F;
  // 256-point twiddle blocks (radix 8, 8, 4), the table layout of fft_block.cuh
  for (int i = tid; i < tw_size(BLK_F); i += NTH) {
    const int ns = i < 7 * 8 ? 8 : 64, r = ns == 8 ? 8 : 4;
    const int j = ns == 8 ? i : i - 7 * 8;
    const int m = j / ns + 1, k = j % ns;
    float s, c;
    sincospif(-2.0f * (float)(m * k) / (float)(ns * r), &s, &c);
    s_tw[i] = make_float2(c, s);
  }
  const float sk = (lane & 1) ? -1.f : 1.f;  // (-1)^k, k = lane + 32 q
  const float inv_f = 1.f / BLK_F;

  int cur_v = -1, L = 0, T = 0, nblk = 0, v_unit0 = 0, v_nunits = 0;
  const float2* v_hist = nullptr;
  const uint32_t* v_order = nullptr;
  const float* v_mask = nullptr;
  const int4* v_items = nullptr;
  double* v_partials = nullptr;
  float np0 = 0.f;
  auto load_video = [&](int vi) {  // between two CTA barriers
    const VideoDesc vd = video_of(p, vi);
    cur_v = vi;
    L = vd.L;
    T = vd.T;
    nblk = blk_count(T);
    v_hist = vd.hist;
    v_order = vd.order;
    v_mask = vd.mask;
    v_items = vd.items;
    v_partials = vd.partials;
    v_unit0 = vd.unit0;
    v_nunits = vd.nunits;
    np0 = vd.npairs[0];
    for (int i = tid; i < BLK_L; i += NTH) {
      const float n = i < L ? vd.npairs[i] : 0.f;
      s_inp[i] = n > 0.5f ? 1.f / n : 0.f;
    }
    // mask block spectra M_b, one warp per block; block nblk (past T) is zero
    for (int b = warp; b <= nblk; b += BLK_WARPS) {
      float2 v[8];
#pragma unroll
      for (int q = 0; q < 8; q++) {
        const int t = b * BLK_L + lane + 32 * q;
        v[q] = make_float2(q < 4 && t < T ? __ldg(&v_mask[t]) : 0.f, 0.f);
      }
      const float2* Y = fft<BLK_F, false, true, SYNC_WARP>(v, lane, b0, b1, s_tw);
#pragma unroll
      for (int q = 0; q < 8; q++) s_M[(size_t)b * BLK_F + lane + 32 * q] = Y[pad(lane + 32 * q)];
      __syncwarp();  // Y read before the next transform writes the buffers
    }
  };
  // one block's masked samples and p = m |x|^2 at this lane's offsets lane + 32 q
  // a block's raw samples and mask at this lane's offsets lane + 32 q (loads
  // only: consumed a block pair later, so they are in flight meanwhile;
  // measured on 15,676 modes x 4096 frames: 1.064 -> 1.040 ms)
  auto fetch = [&](const float2* row, int b, float2 (&v)[4], float (&m)[4]) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const int t = b * BLK_L + lane + 32 * q;
      const bool in = b < nblk && t < T;
      m[q] = in ? __ldg(&v_mask[t]) : 0.f;
      v[q] = in ? __ldg(&row[__ldg(&v_order[t])]) : make_float2(0.f, 0.f);
    }
  };
  // masked samples x~ = m x and p = m |x|^2 of fetched samples
  auto prep = [&](const float2 (&v)[4], const float (&m)[4], float2 (&x)[4], float (&pw)[4], double& psum) {
#pragma unroll
    for (int q = 0; q < 4; q++) {
      pw[q] = m[q] * fmaf(v[q].x, v[q].x, v[q].y * v[q].y);
      x[q] = make_float2(m[q] * v[q].x, m[q] * v[q].y);
      psum += (double)pw[q];
    }
  };

  if (tid == 0) s_next = atomicAdd(p.unit_counter, 1);
  __syncthreads();
  int u = s_next;
  const int etau = tid % BLK_L, egrp = tid / BLK_L;  // epilogue: this thread's lag and warp group
  double acc[PFIELDS];
#pragma unroll
  for (int c = 0; c < PFIELDS; c++) acc[c] = 0.0;
  double accP = 0.0;  // thread 0
  while (u < p.nunits) {
    const int4 U = p.units[u];
    const int vi = p.videos ? U.w : 0;
    if (vi != cur_v) {
      __syncthreads();  // the previous video's tables are no longer read
      load_video(vi);
      __syncthreads();
    }
    for (int r0 = 0; r0 < U.y; r0 += BLK_WARPS) {  // rounds of one mode per warp
      const int k = r0 + warp;
      if (k < U.y) {
        const int4 e = load_item(v_items, U.x + k);
        const float2* row = v_hist + (size_t)e.x * T;
        float2 aG[8], aAB[8], pX[8], pP[8];
#pragma unroll
        for (int q = 0; q < 8; q++) aG[q] = aAB[q] = pX[q] = pP[q] = make_float2(0.f, 0.f);
        double psum = 0.0;
        // G: a block's spectrum X_n completes block n - 1's term
        auto g_step = [&](const float2* Y) {
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const float2 xn = Y[pad(lane + 32 * q)];
            const float2 w = make_float2(fmaf(sk, xn.x, pX[q].x), fmaf(sk, xn.y, pX[q].y));
            aG[q].x += pX[q].x * w.x + pX[q].y * w.y;  // conj(X_{n-1}) (X_{n-1} + s_k X_n)
            aG[q].y += pX[q].x * w.y - pX[q].y * w.x;
            pX[q] = xn;
          }
          __syncwarp();
        };
        // A + B: block b's spectrum P_b completes block b - 1's term
        auto ab_step = [&](int bn, const float2 (&pn)[8]) {
#pragma unroll
          for (int q = 0; q < 8; q++) {
            if (bn > 0) {
              const float2 m0 = s_M[(size_t)(bn - 1) * BLK_F + lane + 32 * q];
              const float2 m1 = s_M[(size_t)bn * BLK_F + lane + 32 * q];
              const float2 pb = pP[q];
              const float re0 = pb.x * m0.x + pb.y * m0.y;        // Re conj(P_b) M_b
              const float r1 = pb.x * m1.x + pb.y * m1.y, i1 = pb.x * m1.y - pb.y * m1.x;  // conj(P_b) M_{b+1}
              const float r2 = m0.x * pn[q].x + m0.y * pn[q].y, i2 = m0.x * pn[q].y - m0.y * pn[q].x;  // conj(M_b) P_{b+1}
              aAB[q].x += 2.f * re0 + sk * (r1 + r2);
              aAB[q].y += sk * (i1 + i2);
            }
            pP[q] = pn[q];
          }
        };
        float2 ra[4], rb[4];  // raw samples of the current block pair
        float ma[4], mb[4];
        fetch(row, 0, ra, ma);
        fetch(row, 1, rb, mb);
        for (int b = 0; b < nblk; b += 2) {
          float2 na[4], nb[4];  // the next pair's loads, in flight during this pair's transforms
          float nma[4], nmb[4];
          fetch(row, b + 2, na, nma);
          fetch(row, b + 3, nb, nmb);
          float2 xv[4];
          float p0[4], p1[4];
          float2 v[8];
          prep(ra, ma, xv, p0, psum);
#pragma unroll
          for (int q = 0; q < 8; q++) v[q] = q < 4 ? xv[q] : make_float2(0.f, 0.f);
          g_step(fft<BLK_F, false, true, SYNC_WARP>(v, lane, b0, b1, s_tw));
          const bool two = b + 1 < nblk;
          prep(rb, mb, xv, p1, psum);  // zeros past the last block
          if (two) {
#pragma unroll
            for (int q = 0; q < 8; q++) v[q] = q < 4 ? xv[q] : make_float2(0.f, 0.f);
            g_step(fft<BLK_F, false, true, SYNC_WARP>(v, lane, b0, b1, s_tw));
          }
#pragma unroll
          for (int q = 0; q < 4; q++) {
            ra[q] = na[q];
            rb[q] = nb[q];
            ma[q] = nma[q];
            mb[q] = nmb[q];
          }
          // P_b and P_{b+1} from one transform of p_b + i p_{b+1}
#pragma unroll
          for (int q = 0; q < 8; q++) v[q] = q < 4 ? make_float2(p0[q], p1[q]) : make_float2(0.f, 0.f);
          const float2* Z = fft<BLK_F, false, true, SYNC_WARP>(v, lane, b0, b1, s_tw);
          float2 pa[8], pb[8];
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const int kk = lane + 32 * q;
            const float2 zk = Z[pad(kk)], zn = Z[pad((BLK_F - kk) & (BLK_F - 1))];
            pa[q] = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
            pb[q] = make_float2(0.5f * (zk.y + zn.y), 0.5f * (zn.x - zk.x));
          }
          __syncwarp();
          ab_step(b, pa);
          if (two) ab_step(b + 1, pb);
        }
        // the last block's terms: X_nblk = P_nblk = 0, M_nblk = 0 (the zero block)
#pragma unroll
        for (int q = 0; q < 8; q++) {
          aG[q].x += pX[q].x * pX[q].x + pX[q].y * pX[q].y;
          const float2 m0 = s_M[(size_t)(nblk - 1) * BLK_F + lane + 32 * q];
          const float2 m1 = s_M[(size_t)nblk * BLK_F + lane + 32 * q];
          const float2 pbq = pP[q];
          aAB[q].x += 2.f * (pbq.x * m0.x + pbq.y * m0.y) + sk * (pbq.x * m1.x + pbq.y * m1.y);
          aAB[q].y += sk * (pbq.x * m1.y - pbq.y * m1.x);
        }
        // G(tau) and (A + B)(tau), tau = lane + 32 q < BLK_L
        float4* E = s_E + warp * BLK_L;
        {
          const float2* Y = fft<BLK_F, true, true, SYNC_WARP>(aG, lane, b0, b1, s_tw);
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const float2 g = Y[pad(lane + 32 * q)];
            E[lane + 32 * q] = make_float4(0.f, g.x * inv_f, g.y * inv_f, 0.f);
          }
          __syncwarp();
          const float2* W = fft<BLK_F, true, true, SYNC_WARP>(aAB, lane, b0, b1, s_tw);
#pragma unroll
          for (int q = 0; q < 4; q++) E[lane + 32 * q].x = W[pad(lane + 32 * q)].x * inv_f;
          __syncwarp();
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) psum += __shfl_xor_sync(0xffffffffu, psum, o);
        if (lane == 0) s_P[warp] = np0 > 0.5f ? (float)(psum / np0) : 0.f;
      }
      __syncthreads();  // the round's (A + B, G) complete
      // radial epilogue: thread (lag etau, group egrp) adds the modes of warps
      // egrp * WPG .. egrp * WPG + WPG - 1 of this round, in warp order
      if (etau < L) {
        const float inp = s_inp[etau];
        const bool next = etau + 1 < L;
        const float inp1 = next ? s_inp[etau + 1] : 0.f;
        for (int w = egrp * WPG; w < egrp * WPG + WPG && r0 + w < U.y; w++) {
          const int4 e = load_item(v_items, U.x + r0 + w);
          const double kx = e.y, ky = e.z;
          const float4 E0 = s_E[w * BLK_L + etau];
          acc[0] += (double)((E0.x - 2.f * E0.y) * inp);
          if (next) {
            const float4 E1 = s_E[w * BLK_L + etau + 1];
            const float cx = E0.y * inp, cy = E0.z * inp;
            const float c1x = E1.y * inp1, c1y = E1.z * inp1;
            const float zr = fmaf(c1x, cx, c1y * cy);  // C(tau+1) conj C(tau)
            const float zi = fmaf(c1y, cx, -c1x * cy);
            const float wgt = sqrtf(fmaf(zr, zr, zi * zi));
            if (wgt > 0.f) {
              const double wd = wgt, ph = atan2f(zi, zr);
              acc[1] += wd;
              acc[2] += wd * kx * kx;
              acc[3] += wd * kx * ky;
              acc[4] += wd * ky * ky;
              acc[5] += wd * kx * ph;
              acc[6] += wd * ky * ph;
              acc[7] += wd * ph * ph;
              acc[8] += 1.0;
            }
          }
        }
      }
      if (tid == 0)
        for (int w = 0; w < BLK_WARPS && r0 + w < U.y; w++) accP += (double)s_P[w];
      __syncthreads();  // s_E and s_P are rewritten by the next round
    }
    // the unit's partial record: the warp groups' sums added in group order
    const int ul = u - v_unit0;
    if (egrp > 0 && etau < L)
#pragma unroll
      for (int c = 0; c < PFIELDS; c++) s_acc[((egrp - 1) * PFIELDS + c) * BLK_L + etau] = acc[c];
    __syncthreads();
    if (egrp == 0 && etau < L)
#pragma unroll
      for (int c = 0; c < PFIELDS; c++) {
        double t = acc[c];
        for (int g = 1; g < QG; g++) t += s_acc[((g - 1) * PFIELDS + c) * BLK_L + etau];
        v_partials[((size_t)ul * PFIELDS + c) * L + etau] = t;
      }
#pragma unroll
    for (int c = 0; c < PFIELDS; c++) acc[c] = 0.0;
    if (tid == 0) {
      v_partials[(size_t)v_nunits * PFIELDS * L + ul] = accP;
      accP = 0.0;
      s_next = atomicAdd(p.unit_counter, 1);
    }
    __syncthreads();  // s_acc read; the next unit index published
    u = s_next;
  }
}

// ------------------------------------------------------------------ launchers

template <int NP>
static size_t temporal_smem(int T, int L) {
  return sizeof(float2) * (3 * (size_t)padded(NP) + 4 * (size_t)T + tw_size(NP)) + sizeof(float) * (size_t)L;
}

static int lpt_of(int TPAD, int L) {
  const int NT = TPAD / 8;
  const int r = (L + NT - 1) / NT;
  return r <= 1 ? 1 : r <= 2 ? 2 : 4;
}

// The two-group radix-16 kernel exists for the fused radial path at TPAD
// 1024..4096 and is chosen by TemporalParams::variant (the autotuner times
// both); the one-group kernel serves the rest and the full per-mode outputs.
__host__ __device__ constexpr bool use16(int NP, bool full) { return !full && NP >= 1024 && NP <= 4096; }

template <int NP>
static size_t temporal16_smem(int T, int L) {
  return sizeof(float2) * (3 * (size_t)NP + 4 * (size_t)T + tw_size16(NP)) + sizeof(float) * (size_t)L;
}

// TPAD 8192 runs the one-group radix-16 kernel with in-place buffers, for
// both epilogues: the staged kernels need more shared memory than a CTA has.
__host__ __device__ constexpr bool use_big(int NP) { return NP >= 8192; }

template <int NP>
static size_t temporal_big_smem(int T, int L) {
  return sizeof(float2) * (2 * (size_t)NP + 2 * (size_t)T) + sizeof(float) * (size_t)L;
}

template <int NP>
static size_t temporal_sparse_big_smem(int T, int L, int LPT) {
  return sizeof(float2) * ((size_t)NP + 3 * (size_t)T + 2 * (size_t)sparse_padl_big(NP, L, LPT)) +
         sizeof(double2) * 2 * ((size_t)L + 1) + sizeof(float) * (size_t)L;
}

// lags per thread of the big kernel (NP/16 threads)
static int lpt_big(int TPAD, int L) {
  const int NTH = TPAD / 16;
  const int r = (L + NTH - 1) / NTH;
  return r <= 1 ? 1 : r <= 2 ? 2 : r <= 4 ? 4 : 8;
}

// the sparse-mask kernel: whole warps per transform group and room for its
// buffers (TPAD 256..4096)
__host__ __device__ constexpr bool sparse_ok(int NP) { return NP >= 256 && NP <= 4096; }

template <int NP>
static size_t temporal_sparse_smem(int T, int L, int LPT) {
  return sizeof(float2) * (2 * (size_t)padded(NP) + 5 * (size_t)T + tw_size(NP) + 2 * (size_t)sparse_padl(NP, L, LPT)) +
         sizeof(float) * (size_t)L;
}

template <int NP, int LPT, bool FULL>
static cudaError_t launch_k(const TemporalParams& p, int grid, cudaStream_t s) {
  if constexpr (use_big(NP)) {
    if constexpr (!FULL) {
      if (p.variant == 2) {
        const size_t sm = temporal_blocked_smem(p.T);
        cudaFuncSetAttribute(temporal_blocked_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        temporal_blocked_kernel<<<grid, 32 * BLK_WARPS, sm, s>>>(p);
        return cudaGetLastError();
      }
    }
    if (p.sparse) {
      auto k = temporal_sparse_big_kernel<NP, LPT, FULL>;
      const size_t sm = temporal_sparse_big_smem<NP>(p.T, p.L, LPT);
      cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      k<<<grid, NP / 16, sm, s>>>(p);
      return cudaGetLastError();
    }
    auto k = temporal_big_kernel<NP, LPT, FULL>;
    const size_t sm = temporal_big_smem<NP>(p.T, p.L);
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<grid, NP / 16, sm, s>>>(p);
    return cudaGetLastError();
  } else {
    if constexpr (sparse_ok(NP)) {
      if (p.sparse) {
        auto k = temporal_sparse_kernel<NP, LPT, FULL>;
        const size_t sm = temporal_sparse_smem<NP>(p.T, p.L, LPT);
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k<<<grid, NP / 8, sm, s>>>(p);
        return cudaGetLastError();
      }
    }
    if constexpr (use16(NP, FULL)) {
      if (p.variant == 1) {
        auto k = temporal16_kernel<NP, LPT>;
        const size_t sm = temporal16_smem<NP>(p.T, p.L);
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        k<<<grid, NP / 8, sm, s>>>(p);
        return cudaGetLastError();
      }
    }
    auto k = temporal_kernel<NP, LPT, FULL>;
    const size_t sm = temporal_smem<NP>(p.T, p.L);
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k<<<grid, NP / 8, sm, s>>>(p);
    return cudaGetLastError();
  }
}

template <typename K>
static int occupancy_grid(K k, int threads, size_t smem) {
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, threads, smem);
  return sms * (per > 0 ? per : 1);
}

template <int NP, int LPT, bool FULL>
static int grid_of(int T, int L, int variant, bool sparse) {
  if constexpr (use_big(NP)) {
    if (variant == 2 && !FULL) return occupancy_grid(temporal_blocked_kernel, 32 * BLK_WARPS, temporal_blocked_smem(T));
    if (sparse)
      return occupancy_grid(temporal_sparse_big_kernel<NP, LPT, FULL>, NP / 16,
                            temporal_sparse_big_smem<NP>(T, L, LPT));
    return occupancy_grid(temporal_big_kernel<NP, LPT, FULL>, NP / 16, temporal_big_smem<NP>(T, L));
  } else {
    if constexpr (sparse_ok(NP))
      if (sparse)
        return occupancy_grid(temporal_sparse_kernel<NP, LPT, FULL>, NP / 8, temporal_sparse_smem<NP>(T, L, LPT));
    if constexpr (use16(NP, FULL))
      if (variant == 1) return occupancy_grid(temporal16_kernel<NP, LPT>, NP / 8, temporal16_smem<NP>(T, L));
    return occupancy_grid(temporal_kernel<NP, LPT, FULL>, NP / 8, temporal_smem<NP>(T, L));
  }
}

template <int NP>
static cudaError_t dispatch_np(int T, int L, bool full, const TemporalParams* p, int grid,
                               cudaStream_t s, int* grid_out, int variant, bool sparse) {
  if (full) {
    if (grid_out) *grid_out = grid_of<NP, 1, true>(T, L, variant, sparse);
    return p ? launch_k<NP, 1, true>(*p, grid, s) : cudaSuccess;
  }
  if constexpr (use_big(NP)) {
    switch (lpt_big(NP, L)) {
      case 1:
        if (grid_out) *grid_out = grid_of<NP, 1, false>(T, L, variant, sparse);
        return p ? launch_k<NP, 1, false>(*p, grid, s) : cudaSuccess;
      case 2:
        if (grid_out) *grid_out = grid_of<NP, 2, false>(T, L, variant, sparse);
        return p ? launch_k<NP, 2, false>(*p, grid, s) : cudaSuccess;
      case 4:
        if (grid_out) *grid_out = grid_of<NP, 4, false>(T, L, variant, sparse);
        return p ? launch_k<NP, 4, false>(*p, grid, s) : cudaSuccess;
      default:
        if (grid_out) *grid_out = grid_of<NP, 8, false>(T, L, variant, sparse);
        return p ? launch_k<NP, 8, false>(*p, grid, s) : cudaSuccess;
    }
  }
  switch (lpt_of(NP, L)) {
    case 1:
      if (grid_out) *grid_out = grid_of<NP, 1, false>(T, L, variant, sparse);
      return p ? launch_k<NP, 1, false>(*p, grid, s) : cudaSuccess;
    case 2:
      if (grid_out) *grid_out = grid_of<NP, 2, false>(T, L, variant, sparse);
      return p ? launch_k<NP, 2, false>(*p, grid, s) : cudaSuccess;
    default:
      if (grid_out) *grid_out = grid_of<NP, 4, false>(T, L, variant, sparse);
      return p ? launch_k<NP, 4, false>(*p, grid, s) : cudaSuccess;
  }
}

static cudaError_t dispatch(int TPAD, int T, int L, bool full, const TemporalParams* p, int grid,
                            cudaStream_t s, int* grid_out, int variant, bool sparse) {
  switch (TPAD) {
    case 128: return dispatch_np<128>(T, L, full, p, grid, s, grid_out, variant, sparse);
    case 256: return dispatch_np<256>(T, L, full, p, grid, s, grid_out, variant, sparse);
    case 512: return dispatch_np<512>(T, L, full, p, grid, s, grid_out, variant, sparse);
    case 1024: return dispatch_np<1024>(T, L, full, p, grid, s, grid_out, variant, sparse);
    case 2048: return dispatch_np<2048>(T, L, full, p, grid, s, grid_out, variant, sparse);
    case 4096: return dispatch_np<4096>(T, L, full, p, grid, s, grid_out, variant, sparse);
    case 8192: return dispatch_np<8192>(T, L, full, p, grid, s, grid_out, variant, sparse);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_temporal(int TPAD, int L, bool full, const TemporalParams& p, int grid,
                            cudaStream_t s) {
  return dispatch(TPAD, p.T, L, full, &p, grid, s, nullptr, p.variant, p.sparse != 0);
}

int temporal_max_grid(int TPAD, int T, int L, bool full, int variant, bool sparse) {
  int g = 0;
  dispatch(TPAD, T, L, full, nullptr, 0, nullptr, &g, variant, sparse);
  return g;
}

bool temporal_has_variant16(int TPAD) { return use16(TPAD, false); }

bool temporal_sparse_ok(int TPAD) { return sparse_ok(TPAD) || use_big(TPAD); }

int temporal_sparse_limit(int TPAD, int T, int L, bool full) {
  if (sparse_ok(TPAD)) return SPARSE_ZMAX;
  if (TPAD != 8192) return 0;
  // the corrections cost zeros x lags per thread: bound their product
  const int lpt = full ? 1 : lpt_big(TPAD, L);
  if (temporal_sparse_big_smem<8192>(T, L, lpt) > 225 * 1024) return 0;  // with the static tables
  return SPARSE_ZMAX_BIG / lpt;
}

bool temporal_blocked_ok(int TPAD, int T, int L, bool full) {
  return TPAD == 8192 && !full && L <= BLK_L && temporal_blocked_smem(T) <= 227 * 1024;
}

int temporal_kernel_id(int TPAD, bool full, int variant, bool sparse) {
  if (use_big(TPAD) && !full && variant == 2) return DDM_TK_BLOCKED;
  if (use_big(TPAD)) return sparse ? DDM_TK_SPARSE_BIG : DDM_TK_BIG;
  if (sparse && sparse_ok(TPAD)) return DDM_TK_SPARSE;
  if (use16(TPAD, full) && variant == 1) return DDM_TK_RADIX16;
  return DDM_TK_RADIX8;
}

cudaError_t launch_reduce(const ReduceParams& p, cudaStream_t s) {
  const int threads = p.L >= 128 ? 128 : ((p.L + 31) / 32) * 32;
  reduce_kernel<<<dim3((p.L + threads - 1) / threads, p.NB), threads, 0, s>>>(p);
  return cudaGetLastError();
}

cudaError_t launch_radial_full(const RadialFullParams& p, cudaStream_t s) {
  if (p.nunits <= 0) return cudaSuccess;
  const int threads = p.L >= 128 ? 128 : ((p.L + 31) / 32) * 32;
  radial_full_kernel<<<dim3((p.L + threads - 1) / threads, p.nunits), threads, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace ddm
