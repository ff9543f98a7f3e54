// Batched Levenberg-Marquardt fit of the motility model, one warp per q-bin.
//
// Model (the reference's model column, motility_fit.js:417-432, per bin):
//   y(tau) = A c(tau) + B,
//   c(tau) = 1 - <exp(-D q^2 tau) J0(q |V| tau) (1 - alpha + alpha g(q vbar tau; Z))>_nodes
// with g the Schulz-averaged swimmer ISF -- 3D (isf3d, motility_fit.js:140-144)
// or 2D (isf2d, :152-159, read from the device table of isf2d.cu; the
// reference's swimmerKernel, :227-229) -- averaged over the bin's
// effective-|k| nodes, and J0(q |V| tau) the radial average of a known
// uniform drift |V| per fit (0: no factor). Parameters
//   theta = (A, B, alpha, ln vbar, ln Z, ln D),  A, B >= 0, alpha in [0, 1],
// ln vbar, ln Z, ln D clamped to the reference's bounds (bounds(),
// motility_fit.js:480-491). The reference fits (alpha, vbar, Z, D) globally by
// VarPro + Nelder-Mead (motility_fit.js:577-611); it has no LM. This kernel
// solves the per-bin problem; the FP64 LM of oracle/lm.c is its checker.
//
// Per iteration each lane evaluates the model and the analytic Jacobian at its
// lags (FP32, the ISF derivatives in closed form), accumulates J^T J, J^T r
// and the cost in FP64, the warp reduces them, and every lane solves
// (J^T J + lambda diag J^T J) delta = -J^T r by FP64 Cholesky (same values on
// every lane, so control flow stays warp-uniform). Marquardt's rule: accept a
// step that lowers the cost (lambda /= 3) else reject it (lambda *= 4); stop
// after two consecutive accepted steps with relative decrease < tol, when
// lambda > 1e12, or at max_iter -- the iteration of oracle/lm.c.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/ddm_b200.h"
#include "isf.cuh"
#include "kernels.cuh"

namespace ddm {

constexpr int LM_NP = 6;
constexpr int LM_MAX_LAGS = 128;   // 4 per lane
constexpr int LM_MAX_NODES = 8;
constexpr int LM_WARPS = 8;        // fits per 256-thread CTA
// CTAs per SM the register budget is sized for: 1 (no cap). The model and
// normal-equation routines (varpro, varpro_brownian64, lm_normal, lm_solve)
// are not inlined: inlined at every call site they overflowed the
// instruction cache (ncu: "no instruction" was the top stall). Measured on
// B200 over 1e5 analytic curves (q-fits/s, plain / seeded from the truth):
// inlined, 3 CTAs (80 registers) 132K / 1.13M; not inlined, 1 CTA 144K /
// 1.31M, 2 CTAs 104K / 1.04M, 3 CTAs 99K / 1.35M.
#ifndef LM_MIN_BLOCKS
#define LM_MIN_BLOCKS 1
#endif

// Precision-generic math for the model: FP32 for the bulk of the
// iterations, FP64 for the final refinement.
__device__ __forceinline__ float m_exp(float x) { return expf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }

template <bool G2D>
struct LmProblemT {
  static constexpr bool g2d_kernel = G2D;
  int nt, K;
  float V;             // drift speed |V| of the J0 factor (0: none)
  Isf2dTable tab;
  float w;
  float qn[LM_MAX_NODES];
  float d[4], tau[4];  // this lane's lags j = lane + 32 r
  double lo[LM_NP], hi[LM_NP];
};

__device__ __forceinline__ float m_j0(float y) { return j0f(y); }
__device__ __forceinline__ double m_j0(double y) { return j0(y); }

// The swimmer kernel of the fit's geometry: g, x dg/dx, Z dg/dZ.
template <typename R, class PR>
__device__ __forceinline__ void swim_isf(const PR& P, R x, R Z, R& g, R& gx, R& gz) {
  if constexpr (PR::g2d_kernel) {
    double a, b, c;
    isf2d_d(P.tab, (double)x, (double)Z, a, b, c);
    g = (R)a;
    gx = (R)b;
    gz = (R)c;
  } else {
    isf3d_d<R>(x, Z, g, gx, gz);
  }
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;  // the xor butterfly leaves the same bits on every lane
}

// Model column c(tau) at this lane's lags (FP32), 0 beyond nt.
template <class PR>
__device__ __forceinline__ void model_c(const PR& P, int lane, float al, float v, float Z, float D,
                                        float (&c)[4]) {
  const float iK = 1.f / P.K;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int j = lane + 32 * r;
    c[r] = 0.f;
    if (j >= P.nt) continue;
    const float t = P.tau[r];
    float sE = 0.f;
    for (int n = 0; n < P.K; n++) {
      const float q = P.qn[n];
      float E = expf(-D * q * q * t);
      if (P.V > 0.f) E *= m_j0(q * P.V * t);
      if (al > 0.f) {
        float g, gx, gz;
        swim_isf<float>(P, q * v * t, Z, g, gx, gz);
        sE += E * (1.f - al + al * g);
      } else {
        sE += E;
      }
    }
    c[r] = 1.f - sE * iK;
  }
}

// VarPro amplitudes at fixed nonlinear parameters: the 2-column NNLS of the
// reference's evalModel (motility_fit.js:450-474) by nnls3's support
// enumeration (:243-263) over {A}, {B}, {A, B}. Returns the weighted cost.
template <typename CT, class PR>
__device__ __forceinline__ double varpro_c(const PR& P, int lane, const CT (&c)[4], double& A, double& B) {
  double g11 = 0, g12 = 0, h1 = 0, h2 = 0, dd = 0;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    if (lane + 32 * r >= P.nt) continue;
    const double cc = c[r], d = P.d[r];
    g11 += cc * cc;
    g12 += cc;
    h1 += cc * d;
    h2 += d;
    dd += d * d;
  }
  g11 = warp_sum(g11);
  g12 = warp_sum(g12);
  h1 = warp_sum(h1);
  h2 = warp_sum(h2);
  dd = warp_sum(dd);
  const double n = P.nt;
  double best = dd, bA = 0, bB = 0;
  if (g11 > 1e-300) {
    const double a = h1 / g11, rs = dd - a * h1;
    if (a >= 0 && rs < best) best = rs, bA = a, bB = 0;
  }
  {
    const double b = h2 / n, rs = dd - b * h2;
    if (b >= 0 && rs < best) best = rs, bA = 0, bB = b;
  }
  {
    const double det = g11 * n - g12 * g12, sc = fmax(g11, n);
    if (fabs(det) > 1e-11 * sc * sc) {
      const double a = (h1 * n - g12 * h2) / det, b = (g11 * h2 - g12 * h1) / det;
      const double rs = dd - a * h1 - b * h2;
      if (a >= 0 && b >= 0 && rs < best) best = rs, bA = a, bB = b;
    }
  }
  A = bA;
  B = bB;
  return fmax(best, 0.0) * (double)P.w * (double)P.w;
}

template <class PR>
__device__ __noinline__ double varpro(const PR& P, int lane, double al, double lv, double lZ,
                                         double lD, double& A, double& B) {
  float c[4];
  model_c(P, lane, (float)al, (float)exp(lv), (float)exp(lZ), (float)exp(lD), c);
  return varpro_c(P, lane, c, A, B);
}

// The Brownian column c(tau) = 1 - <exp(-D q_n^2 tau)> in FP64, for the
// Brownian-only fit: its golden section walks a valley that can be flat to
// FP32 rounding (noise-dominated or barely decaying bins).
template <class PR>
__device__ __noinline__ double varpro_brownian64(const PR& P, int lane, double lD, double& A,
                                                    double& B) {
  const double D = exp(lD), iK = 1.0 / P.K;
  double c[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    c[r] = 0.0;
    if (lane + 32 * r >= P.nt) continue;
    const double t = P.tau[r];
    double sE = 0.0;
    for (int n = 0; n < P.K; n++) {
      const double q = P.qn[n];
      sE += P.V > 0.f ? exp(-D * q * q * t) * j0(q * (double)P.V * t) : exp(-D * q * q * t);
    }
    c[r] = 1.0 - sE * iK;
  }
  return varpro_c(P, lane, c, A, B);
}

// Normal equations, spread over the warp. The 28 sums (J^T J lower triangle,
// J^T r, cost) are laid out in 32 slots -- slot tri(i, j) = i (i + 1) / 2 + j
// for J^T J (i >= j), 21 + i for J^T r, 27 for the cost -- and reduced with a
// reduce-scatter (recursive halving over the xor partners 16, 8, 4, 2, 1:
// 31 shuffles): lane l ends holding the total of slot l. Nothing else of the
// normal equations lives in every lane, which keeps the kernel's registers
// low enough for several CTAs per SM; the Cholesky factorisation below works
// on these lane-held entries through shuffles.
constexpr int LM_SLOT_G = 21, LM_SLOT_COST = 27;
__device__ __forceinline__ constexpr int tri(int i, int j) { return i * (i + 1) / 2 + j; }

__device__ __forceinline__ double reduce_scatter32(double (&v)[32], int lane) {
  double h16[16], h8[8], h4[4], h2[2];
#pragma unroll
  for (int i = 0; i < 16; i++) {
    const bool up = lane & 16;
    h16[i] = (up ? v[i + 16] : v[i]) + __shfl_xor_sync(0xffffffffu, up ? v[i] : v[i + 16], 16);
  }
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const bool up = lane & 8;
    h8[i] = (up ? h16[i + 8] : h16[i]) + __shfl_xor_sync(0xffffffffu, up ? h16[i] : h16[i + 8], 8);
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const bool up = lane & 4;
    h4[i] = (up ? h8[i + 4] : h8[i]) + __shfl_xor_sync(0xffffffffu, up ? h8[i] : h8[i + 4], 4);
  }
#pragma unroll
  for (int i = 0; i < 2; i++) {
    const bool up = lane & 2;
    h2[i] = (up ? h4[i + 2] : h4[i]) + __shfl_xor_sync(0xffffffffu, up ? h4[i] : h4[i + 2], 2);
  }
  const bool up = lane & 1;
  return (up ? h2[1] : h2[0]) + __shfl_xor_sync(0xffffffffu, up ? h2[0] : h2[1], 1);
}

// The normal equations at theta; returns this lane's slot total. The model
// and Jacobian are evaluated in R; the sums are FP64.
template <typename R, class PR>
__device__ __noinline__ double lm_normal(const PR& P, const double (&th)[LM_NP], int lane) {
  const R A = (R)th[0], B = (R)th[1], al = (R)th[2];
  const R v = (R)exp(th[3]), Z = (R)exp(th[4]), D = (R)exp(th[5]);
  double acc[32];
#pragma unroll
  for (int i = 0; i < 32; i++) acc[i] = 0.0;
  const R iK = R(1) / R(P.K);
  const R w = (R)P.w;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int j = lane + 32 * r;
    if (j >= P.nt) break;
    const R t = (R)P.tau[r];
    R sE = 0, sEg = 0, sdD = 0, sgx = 0, sgz = 0;
    for (int n = 0; n < P.K; n++) {
      const R q = (R)P.qn[n];
      R E = m_exp(-D * q * q * t);
      if (P.V > 0.f) E *= m_j0(q * (R)P.V * t);
      R g, gx, gz;
      swim_isf<R>(P, q * v * t, Z, g, gx, gz);
      const R mix = R(1) - al + al * g;
      sE += E * mix;
      sEg += E * (g - R(1));
      sdD += E * D * q * q * t * mix;
      sgx += E * al * gx;
      sgz += E * al * gz;
    }
    const R c = R(1) - sE * iK;
    const double rr = (double)w * ((double)A * (double)c + (double)B - (double)P.d[r]);
    double J[LM_NP];
    J[0] = (double)(w * c);
    J[1] = (double)w;
    J[2] = (double)(-w * A * sEg * iK);
    J[3] = (double)(-w * A * sgx * iK);
    J[4] = (double)(-w * A * sgz * iK);
    J[5] = (double)(w * A * sdD * iK);
    acc[LM_SLOT_COST] += rr * rr;
#pragma unroll
    for (int a = 0; a < LM_NP; a++) {
      acc[LM_SLOT_G + a] += J[a] * rr;
#pragma unroll
      for (int b = 0; b <= a; b++) acc[tri(a, b)] += J[a] * J[b];
    }
  }
  return reduce_scatter32(acc, lane);
}

__device__ __forceinline__ double lm_cost(double hv) { return __shfl_sync(0xffffffffu, hv, LM_SLOT_COST); }

// (H + lambda diag H) delta = -g by Cholesky on the lane-held entries: lane
// tri(i, j) (< 21) owns entry (i, j) of the lower triangle, (li, lj) its
// position; pivots, column entries and the triangular solves travel by
// shuffles, and every lane ends with the same delta. False if not positive
// definite (the same on every lane).
__device__ __noinline__ bool lm_solve(double hv, double lambda, int lane, int li, int lj,
                                         double (&delta)[LM_NP]) {
  const bool in = lane < LM_SLOT_G;
  double a = hv;
  if (in && li == lj) a += lambda * (a > 0 ? a : 1e-30);
#pragma unroll
  for (int k = 0; k < LM_NP; k++) {
    const double dkk = __shfl_sync(0xffffffffu, a, tri(k, k));
    if (!(dkk > 0)) return false;
    const double lkk = sqrt(dkk);
    if (in && lj == k) a = li == k ? lkk : a / lkk;
    const double lik = __shfl_sync(0xffffffffu, a, in && li > k ? tri(li, k) : lane);
    const double ljk = __shfl_sync(0xffffffffu, a, in && lj > k ? tri(lj, k) : lane);
    if (in && lj > k) a -= lik * ljk;
  }
  double y[LM_NP];
#pragma unroll
  for (int i = 0; i < LM_NP; i++) {
    double s = -__shfl_sync(0xffffffffu, hv, LM_SLOT_G + i);
#pragma unroll
    for (int q = 0; q < i; q++) s -= __shfl_sync(0xffffffffu, a, tri(i, q)) * y[q];
    y[i] = s / __shfl_sync(0xffffffffu, a, tri(i, i));
  }
#pragma unroll
  for (int i = LM_NP - 1; i >= 0; i--) {
    double s = y[i];
#pragma unroll
    for (int q = i + 1; q < LM_NP; q++) s -= __shfl_sync(0xffffffffu, a, tri(q, i)) * delta[q];
    delta[i] = s / __shfl_sync(0xffffffffu, a, tri(i, i));
  }
  return true;
}

// Marquardt iterations with the model in R from th (projected, amplitudes
// set), continuing from lambda; returns the iterations taken.
// max_reject > 0 ends the phase after that many consecutive rejected steps
// (used by the FP32 phase, whose cost cannot resolve the last decreases).
template <typename R, class PR>
__device__ int lm_phase(const PR& P, int lane, double (&th)[LM_NP], double& cost, double& lambda,
                        int max_iter, double tol, bool& converged, int max_reject = 0) {
  int li = 0;
  while (tri(li + 1, 0) <= lane) li++;
  const int lj = lane - tri(li, 0);
  double hv = lm_normal<R>(P, th, lane);
  cost = lm_cost(hv);
  int small = 0, it = 0, rejected = 0;
  converged = false;
  for (it = 0; it < max_iter; it++) {
    double delta[LM_NP];
    if (!lm_solve(hv, lambda, lane, li, lj, delta)) {
      lambda *= 4;
      if (lambda > 1e12 || (max_reject && ++rejected >= max_reject)) {
        converged = lambda > 1e12;  // no step lowers the cost: a numerical minimum
        break;
      }
      continue;
    }
    double th2[LM_NP];
#pragma unroll
    for (int a = 0; a < LM_NP; a++) th2[a] = fmin(P.hi[a], fmax(P.lo[a], th[a] + delta[a]));
    const double hv2 = lm_normal<R>(P, th2, lane);
    const double c2 = lm_cost(hv2);
    if (c2 < cost) {
      const double rel = (cost - c2) / (cost > 0 ? cost : 1e-300);
#pragma unroll
      for (int a = 0; a < LM_NP; a++) th[a] = th2[a];
      hv = hv2;
      cost = c2;
      lambda = fmax(lambda / 3, 1e-12);
      rejected = 0;
      small = rel < tol ? small + 1 : 0;
      if (small >= 2) {
        it++;
        converged = true;
        break;
      }
    } else {
      lambda *= 4;
      if (lambda > 1e12 || (max_reject && ++rejected >= max_reject)) {
        converged = lambda > 1e12;  // no step lowers the cost: a numerical minimum
        break;
      }
    }
  }
  return it;
}

// Marquardt's method (the iteration of oracle/lm.c): FP32 model until the
// FP32 cost stops resolving progress, then FP64 model iterations from there
// (the FP32 cost carries ~1e-7 relative noise, which would otherwise stop
// the walk early along flat valleys). Returns the iterations taken;
// `converged` = the FP64 phase stopped at a minimum (the relative-decrease
// test, or no step lowering the cost any more) rather than at the cap.
template <class PR>
__device__ int lm_run(const PR& P, int lane, double (&th)[LM_NP], double& cost, int max_iter,
                      double tol, bool& converged) {
  double lambda = 1e-3;
  bool c32;
  // FP32 phase: ends when two accepted steps gain < 1e-6 (the FP32 cost's
  // resolution) or after 4 rejected steps in a row
  const int it32 = lm_phase<float>(P, lane, th, cost, lambda, max_iter, fmax(tol, 1e-6), c32, 4);
  // FP64 phase with the caller's tolerance; restart the damping
  lambda = 1e-3;
  const int it64 =
      lm_phase<double>(P, lane, th, cost, lambda, max_iter - it32 > 8 ? max_iter - it32 : 8, tol, converged);
  return it32 + it64;
}

// The Brownian fit of one bin (fitBrownian, motility_fit.js:500-536, per
// bin): the model at alpha = 0, c(tau) = 1 - <exp(-D q_n^2 tau)> over the
// q-nodes, VarPro amplitudes; a 49-point scan of ln D over its bounds, then
// golden section (at most 60 steps, to 1e-6 in ln D). Returns ln D;
// `settled` when the bracket closed.
template <bool F64, class PR>
__device__ double brownian_search(const PR& P, int lane, int& evals, bool& settled) {
  double A, B;
  auto cost_at = [&](double x) {
    return F64 ? varpro_brownian64(P, lane, x, A, B) : varpro(P, lane, 0.0, P.lo[3], 0.0, x, A, B);
  };
  const double lo = P.lo[5], hi = P.hi[5];
  int bi = 0;
  double bf = 1e308;
  for (int i = 0; i <= 48; i++) {
    const double x = lo + ((hi - lo) * i) / 48;
    const double v = cost_at(x);
    if (v < bf) bf = v, bi = i;
  }
  evals += 49;
  double a = lo + ((hi - lo) * (bi > 0 ? bi - 1 : 0)) / 48;
  double b = lo + ((hi - lo) * (bi < 48 ? bi + 1 : 48)) / 48;
  const double gr = (sqrt(5.0) - 1) / 2;
  double c = b - gr * (b - a), dd = a + gr * (b - a);
  double fc = cost_at(c);
  double fd = cost_at(dd);
  evals += 2;
  for (int it = 0; it < 60 && b - a > 1e-6; it++) {
    if (fc < fd) {
      b = dd;
      dd = c;
      fd = fc;
      c = b - gr * (b - a);
      fc = cost_at(c);
    } else {
      a = c;
      c = dd;
      fc = fd;
      dd = a + gr * (b - a);
      fd = cost_at(dd);
    }
    evals++;
  }
  settled = b - a <= 1e-6;
  return fc < fd ? c : dd;
}

// The reference's start strategy (fitBrownian, motility_fit.js:500-536;
// fitSwimmer :577-611) per bin, LM from the best `nrefine` of 64 starts
// (oracle/lm.c or_lm_fit_plain). Accumulates iterations and evaluations.
template <class PR>
__device__ void plain_fit(const PR& P, int lane, int nrefine, int max_iter, double tol,
                          double (&th)[LM_NP], double& cost, int& iters, int& evals, bool& converged) {
  double A, B;
  bool settled;
  const double lD0 = brownian_search<false>(P, lane, evals, settled);
  // 64 starts: lane l holds starts 2l and 2l+1 (index = 4 iv + 2 iz + ia)
  const double lZs0 = fmin(P.hi[4], fmax(P.lo[4], log(1.5)));
  const double lZs1 = fmin(P.hi[4], fmax(P.lo[4], log(8.0)));
  double sc[2];
  for (int s = 0; s < 64; s++) {
    const int iv = s >> 2, iz = (s >> 1) & 1, ia = s & 1;
    const double lv = P.lo[3] + ((P.hi[3] - P.lo[3]) * (iv + 0.5)) / 16;
    const double f = varpro(P, lane, ia ? 0.8 : 0.3, lv, iz ? lZs1 : lZs0, lD0, A, B);
    if ((s >> 1) == lane) sc[s & 1] = f;
  }
  evals += 64;
  double best = 1e308;
  double bth[LM_NP] = {0, 0, 0, 0, 0, 0};
  bool bconv = false;
  for (int k = 0; k < nrefine && k < 64; k++) {
    // k-th smallest cost, lowest index on ties (a stable sort's order)
    double m = sc[0] <= sc[1] ? sc[0] : sc[1];
    int mi = sc[0] <= sc[1] ? 2 * lane : 2 * lane + 1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double m2 = __shfl_xor_sync(0xffffffffu, m, o);
      const int i2 = __shfl_xor_sync(0xffffffffu, mi, o);
      if (m2 < m || (m2 == m && i2 < mi)) m = m2, mi = i2;
    }
    if ((mi >> 1) == lane) sc[mi & 1] = 1e308;  // taken
    const int iv = mi >> 2, iz = (mi >> 1) & 1, ia = mi & 1;
    double t2[LM_NP];
    t2[2] = ia ? 0.8 : 0.3;
    t2[3] = P.lo[3] + ((P.hi[3] - P.lo[3]) * (iv + 0.5)) / 16;
    t2[4] = iz ? lZs1 : lZs0;
    t2[5] = lD0;
    varpro(P, lane, t2[2], t2[3], t2[4], t2[5], t2[0], t2[1]);
    double cst;
    bool cv;
    const int it = lm_run(P, lane, t2, cst, max_iter, tol, cv);
    iters += it;
    evals += 2 + it;
    if (cst < best) {
      best = cst;
      bconv = cv;
#pragma unroll
      for (int q = 0; q < LM_NP; q++) bth[q] = t2[q];
    }
  }
#pragma unroll
  for (int q = 0; q < LM_NP; q++) th[q] = bth[q];
  cost = best;
  converged = bconv;
}

template <bool G2D>
__device__ __noinline__ void lm_one(const LmParams& p, int fit, int lane) {
  LmProblemT<G2D> P;
  P.nt = min(p.nt[fit], min(p.nt_max, LM_MAX_LAGS));
  P.K = min(p.K, LM_MAX_NODES);
  P.V = p.vmag ? p.vmag[fit] : 0.f;
  P.tab = p.tab;
  P.w = p.w[fit];
#pragma unroll
  for (int n = 0; n < LM_MAX_NODES; n++) P.qn[n] = n < P.K ? p.qn[(size_t)fit * p.K + n] : 0.f;
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int j = lane + 32 * r;
    const bool in = j < P.nt;
    P.d[r] = in ? p.d[(size_t)fit * p.nt_max + j] : 0.f;
    P.tau[r] = in ? p.tau[(size_t)fit * p.nt_max + j] : 0.f;
  }
  const float* bd = p.bounds + (size_t)fit * 6;
  P.lo[0] = 0.0;
  P.hi[0] = 1e300;
  P.lo[1] = 0.0;
  P.hi[1] = 1e300;
  P.lo[2] = 0.0;
  P.hi[2] = 1.0;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    P.lo[3 + a] = log((double)bd[2 * a]);
    P.hi[3 + a] = log((double)bd[2 * a + 1]);
  }
  double th[LM_NP], cost = 0;
  int iters = 0, evals = 0, status = 0;
  bool conv = false;
  if (p.mode == LM_SEEDED || p.mode == LM_SEEDED_FALLBACK || p.mode == LM_SEEDED_COST) {
    const float* s = p.start + (size_t)fit * 4;
    th[2] = (double)s[0];
    th[3] = log((double)s[1]);
    th[4] = log((double)s[2]);
    th[5] = log((double)s[3]);
#pragma unroll
    for (int a = 2; a < LM_NP; a++) th[a] = fmin(P.hi[a], fmax(P.lo[a], th[a]));
    varpro(P, lane, th[2], th[3], th[4], th[5], th[0], th[1]);
    iters = lm_run(P, lane, th, cost, p.max_iter, p.tol, conv);
    evals = 2 + iters;
    bool bad = !conv;
    if (p.mode == LM_SEEDED_FALLBACK && !bad) {
      // The Brownian null (alpha = 0) is nested in the model, so no optimum
      // costs more than the best Brownian fit: a seeded fit above a coarse
      // 17-point Brownian scan (itself an upper bound of the Brownian
      // optimum) sits in a wrong basin.
      double A, B, bmin = 1e308;
      for (int i = 0; i <= 16; i++) {
        const double x = P.lo[5] + ((P.hi[5] - P.lo[5]) * i) / 16;
        bmin = fmin(bmin, varpro(P, lane, 0.0, P.lo[3], 0.0, x, A, B));
      }
      evals += 17;
      bad = cost > bmin;
    }
    if (p.mode == LM_SEEDED_COST) {
      // cost alone decides: the bin's Brownian optimum (fitBrownian's scan
      // and golden section, FP64 model) bounds the optimum from above; a
      // seeded fit above it sits in a wrong basin, whether or not its LM
      // converged. A fit at or below it is kept even when the LM stopped at
      // max_iter (a long valley it was still walking down).
      bool settled;
      int be = 0;
      const double lD = brownian_search<true>(P, lane, be, settled);
      double A, B;
      const double bopt = varpro_brownian64(P, lane, lD, A, B);
      evals += be + 1;
      bad = cost > bopt * (1.0 + 1e-9);
    }
    if ((p.mode == LM_SEEDED_FALLBACK || p.mode == LM_SEEDED_COST) && bad) {
      // the seed did not lead to a converged fit: the reference's start
      // strategy decides, and the lower cost wins
      double t2[LM_NP], c2;
      bool cv2;
      plain_fit(P, lane, p.nrefine, p.max_iter, p.tol, t2, c2, iters, evals, cv2);
      status |= 2;
      if (c2 < cost) {
        cost = c2;
        conv = cv2;
#pragma unroll
        for (int q = 0; q < LM_NP; q++) th[q] = t2[q];
      }
    }
  } else if (p.mode == LM_BROWNIAN) {
    // the Brownian model alone: theta = (A, B, 0, ln vbar_lo, ln Z_lo, ln D)
    th[5] = brownian_search<true>(P, lane, evals, conv);
    th[2] = 0.0;
    th[3] = P.lo[3];
    th[4] = P.lo[4];
    cost = varpro_brownian64(P, lane, th[5], th[0], th[1]);
    evals++;
  } else {
    plain_fit(P, lane, p.nrefine, p.max_iter, p.tol, th, cost, iters, evals, conv);
  }
  status |= conv ? 1 : 0;
#pragma unroll
  for (int a = 0; a < LM_NP; a++)
    if (lane == a) p.theta[(size_t)fit * LM_NP + a] = th[a];
  if (lane == 0) {
    p.cost[fit] = cost;
    if (p.iters) p.iters[fit] = iters;
    if (p.evals) p.evals[fit] = evals;
    if (p.status) p.status[fit] = status;
  }
}

// Persistent: each warp takes the next fit from an atomic counter until all
// are done, so fits of very different cost (a fallback, a slow valley) do
// not hold a CTA's other warps.
template <bool G2D>
__global__ void __launch_bounds__(32 * LM_WARPS, LM_MIN_BLOCKS) lm_kernel(LmParams p) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    int fit = 0;
    if (lane == 0) fit = atomicAdd(p.counter, 1);
    fit = __shfl_sync(0xffffffffu, fit, 0);
    if (fit >= p.nfit) return;  // whole warp
    lm_one<G2D>(p, fit, lane);
  }
}

// p.counter: a device int set to 0 before the launch (stream-ordered).
cudaError_t launch_lm(const LmParams& p, cudaStream_t s) {
  if (p.nfit <= 0) return cudaSuccess;
  int dev = 0, sms = 0, per = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  auto k = p.geometry2d ? lm_kernel<true> : lm_kernel<false>;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, 32 * LM_WARPS, 0);
  const int need = (p.nfit + LM_WARPS - 1) / LM_WARPS;
  const int wave = sms * (per > 0 ? per : 1);
  k<<<need < wave ? need : wave, 32 * LM_WARPS, 0, s>>>(p);
  return cudaGetLastError();
}

}  // namespace ddm

// ------------------------------------------------------------------ C ABI
#include <cstdarg>
#include <cstdio>
#include <string>

extern std::string& ddm_detached_error();  // message slot of calls without an engine (engine.cu)

namespace {

int lm_fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  ddm_detached_error() = buf;
  return code;
}

template <typename T>
cudaError_t stage_in(T** dst, const T* src, size_t n, cudaStream_t s) {
  cudaError_t e = cudaMallocAsync((void**)dst, sizeof(T) * (n ? n : 1), s);
  if (e != cudaSuccess || !src) return e;
  return cudaMemcpyAsync(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice, s);
}

}  // namespace

extern "C" int ddm_fit_lm_model(int32_t nfit, int32_t nt_max, int32_t K, const int32_t* nt, const float* d,
                                const float* tau, const float* qn, const float* w, const float* bounds,
                                const float* start, int32_t mode, int32_t max_iter, double tol, int32_t nrefine,
                                int32_t geometry2d, const float* vmag, double* theta, double* cost, int32_t* iters,
                                int32_t* evals, int32_t* status, int32_t on_device, void* stream) {
  ddm_detached_error().clear();
  if (nfit < 0 || nt_max < 1 || nt_max > ddm::LM_MAX_LAGS || K < 1 || K > ddm::LM_MAX_NODES)
    return lm_fail(DDM_ERR_ARG, "ddm_fit_lm: need nfit >= 0, 1 <= nt_max <= %d, 1 <= K <= %d",
                   ddm::LM_MAX_LAGS, ddm::LM_MAX_NODES);
  if (mode < ddm::LM_PLAIN || mode > ddm::LM_SEEDED_COST)
    return lm_fail(DDM_ERR_ARG,
                   "ddm_fit_lm: mode must be 0 (reference starts), 1 (seeded), 2 (seeded, fallback), 3 (Brownian) "
                   "or 4 (seeded, fallback by cost)");
  if (max_iter < 1 || nrefine < 1 || nrefine > 64 || !(tol >= 0))
    return lm_fail(DDM_ERR_ARG, "ddm_fit_lm: need max_iter >= 1, 1 <= nrefine <= 64, tol >= 0");
  if (geometry2d != 0 && geometry2d != 1) return lm_fail(DDM_ERR_ARG, "ddm_fit_lm: geometry2d must be 0 or 1");
  if (nfit == 0) return DDM_OK;
  const bool seeded = mode == ddm::LM_SEEDED || mode == ddm::LM_SEEDED_FALLBACK || mode == ddm::LM_SEEDED_COST;
  if (!nt || !d || !tau || !qn || !w || !bounds || !theta || !cost || (seeded && !start))
    return lm_fail(DDM_ERR_ARG, "ddm_fit_lm: null array");
  cudaStream_t s = (cudaStream_t)stream;
  ddm::LmParams p{};
  p.nfit = nfit;
  p.nt_max = nt_max;
  p.K = K;
  p.mode = mode;
  p.max_iter = max_iter;
  p.nrefine = nrefine;
  p.tol = tol;
  p.geometry2d = geometry2d;
  if (geometry2d) {
    const cudaError_t te = ddm::isf2d_table(&p.tab);
    if (te != cudaSuccess) return lm_fail(DDM_ERR_CUDA, "ddm_fit_lm: 2D table: %s", cudaGetErrorString(te));
  }
  if (on_device) {
    p.vmag = vmag;
    p.nt = nt; p.d = d; p.tau = tau; p.qn = qn; p.w = w; p.bounds = bounds; p.start = start;
    p.theta = theta; p.cost = cost; p.iters = iters; p.evals = evals; p.status = status;
    int* ctr = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&ctr, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctr, 0, sizeof(int), s);
    p.counter = ctr;
    if (e == cudaSuccess) e = ddm::launch_lm(p, s);
    if (ctr) cudaFreeAsync(ctr, s);
    if (e != cudaSuccess) return lm_fail(DDM_ERR_CUDA, "ddm_fit_lm: %s", cudaGetErrorString(e));
    return DDM_OK;
  }
  const size_t nf = (size_t)nfit, nd = nf * nt_max;
  int *dnt = nullptr, *dit = nullptr, *dev = nullptr, *dst = nullptr;
  float *dd = nullptr, *dtau = nullptr, *dqn = nullptr, *dw = nullptr, *db = nullptr, *ds = nullptr, *dv = nullptr;
  double *dth = nullptr, *dc = nullptr;
  cudaError_t e = cudaSuccess;
  auto step = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
  step(stage_in(&dnt, nt, nf, s));
  step(stage_in(&dd, d, nd, s));
  step(stage_in(&dtau, tau, nd, s));
  step(stage_in(&dqn, qn, nf * K, s));
  step(stage_in(&dw, w, nf, s));
  step(stage_in(&db, bounds, nf * 6, s));
  if (seeded) step(stage_in(&ds, start, nf * 4, s));
  if (vmag) step(stage_in(&dv, vmag, nf, s));
  step(stage_in<double>(&dth, nullptr, nf * 6, s));
  step(stage_in<double>(&dc, nullptr, nf, s));
  step(stage_in<int>(&dit, nullptr, nf, s));
  step(stage_in<int>(&dev, nullptr, nf, s));
  step(stage_in<int>(&dst, nullptr, nf, s));
  int* ctr = nullptr;
  step(stage_in<int>(&ctr, nullptr, 1, s));
  step(cudaMemsetAsync(ctr, 0, sizeof(int), s));
  if (e == cudaSuccess) {
    p.nt = dnt; p.d = dd; p.tau = dtau; p.qn = dqn; p.w = dw; p.bounds = db; p.start = ds; p.vmag = dv;
    p.theta = dth; p.cost = dc; p.iters = dit; p.evals = dev; p.status = dst; p.counter = ctr;
    step(ddm::launch_lm(p, s));
    step(cudaMemcpyAsync(theta, dth, sizeof(double) * nf * 6, cudaMemcpyDeviceToHost, s));
    step(cudaMemcpyAsync(cost, dc, sizeof(double) * nf, cudaMemcpyDeviceToHost, s));
    if (iters) step(cudaMemcpyAsync(iters, dit, sizeof(int) * nf, cudaMemcpyDeviceToHost, s));
    if (evals) step(cudaMemcpyAsync(evals, dev, sizeof(int) * nf, cudaMemcpyDeviceToHost, s));
    if (status) step(cudaMemcpyAsync(status, dst, sizeof(int) * nf, cudaMemcpyDeviceToHost, s));
  }
  for (void* ptr : {(void*)dnt, (void*)dd, (void*)dtau, (void*)dqn, (void*)dw, (void*)db, (void*)ds, (void*)dv,
                    (void*)dth, (void*)dc, (void*)dit, (void*)dev, (void*)dst, (void*)ctr})
    if (ptr) cudaFreeAsync(ptr, s);
  step(cudaStreamSynchronize(s));
  if (e != cudaSuccess) return lm_fail(DDM_ERR_CUDA, "ddm_fit_lm: %s", cudaGetErrorString(e));
  return DDM_OK;
}

extern "C" int ddm_fit_lm(int32_t nfit, int32_t nt_max, int32_t K, const int32_t* nt, const float* d,
                          const float* tau, const float* qn, const float* w, const float* bounds,
                          const float* start, int32_t mode, int32_t max_iter, double tol,
                          int32_t nrefine, double* theta, double* cost, int32_t* iters, int32_t* evals,
                          int32_t* status, int32_t on_device, void* stream) {
  return ddm_fit_lm_model(nfit, nt_max, K, nt, d, tau, qn, w, bounds, start, mode, max_iter, tol, nrefine, 0,
                          nullptr, theta, cost, iters, evals, status, on_device, stream);
}

// ------------------------------------------------------------------ model curves

namespace ddm {

// counter-based standard normal (splitmix64 hash -> Box-Muller)
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
__device__ __forceinline__ float normal01(uint64_t seed, uint64_t i, uint64_t j) {
  const uint64_t h = mix64(seed ^ mix64(i * 0x100000001B3ull + j));
  const float u1 = ((float)(h >> 40) + 0.5f) * (1.f / 16777216.f);
  const float u2 = ((float)((h >> 16) & 0xFFFFFFull) + 0.5f) * (1.f / 16777216.f);
  return sqrtf(-2.f * logf(u1)) * cospif(2.f * u2);
}

// c(tau) of one curve (FP32), the model column of lm_normal
__device__ __forceinline__ float model_at(const float* qn, int K, float al, float v, float Z, float D, float t) {
  float sE = 0.f;
  for (int n = 0; n < K; n++) {
    const float q = qn[n];
    const float E = expf(-D * q * q * t);
    float g = 1.f, gx, gz;
    if (al > 0.f) isf3d_d<float>(q * v * t, Z, g, gx, gz);
    sE += E * (1.f - al + al * g);
  }
  return 1.f - sE / K;
}

__global__ void curves_kernel(int n, int K, const float* __restrict__ qn, const float* __restrict__ th, int nt,
                              const float* __restrict__ tau, float noise, uint64_t seed, float* __restrict__ y) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * nt) return;
  const int i = (int)(idx / nt), j = (int)(idx % nt);
  const float* t6 = th + (size_t)i * 6;
  const float c = model_at(qn + (size_t)i * K, K, t6[2], t6[3], t6[4], t6[5], tau[j]);
  float v = t6[0] * c + t6[1];
  if (noise > 0.f) v *= 1.f + noise * normal01(seed, (uint64_t)i, (uint64_t)j);
  y[idx] = v;
}

// first lag where c reaches 1 - 1/e: a 256-point log scan over [1e-3, 1e7]
// brackets it, 40 bisection steps refine it; 1e7 if never reached
__global__ void tau_e_kernel(int n, int K, const float* __restrict__ qn, const float* __restrict__ th,
                             float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float* t6 = th + (size_t)i * 6;
  const float* q = qn + (size_t)i * K;
  const float target = 1.f - 0.36787944117144233f;
  const float l0 = logf(1e-3f), l1 = logf(1e7f);
  float lo = l0, hi = l1;
  bool found = false;
  float prev = l0;
  for (int s = 1; s <= 256 && !found; s++) {
    const float x = l0 + (l1 - l0) * s / 256.f;
    if (model_at(q, K, t6[2], t6[3], t6[4], t6[5], expf(x)) >= target) {
      lo = prev;
      hi = x;
      found = true;
    }
    prev = x;
  }
  if (!found) {
    out[i] = 1e7f;
    return;
  }
  for (int it = 0; it < 40; it++) {
    const float mid = 0.5f * (lo + hi);
    if (model_at(q, K, t6[2], t6[3], t6[4], t6[5], expf(mid)) >= target)
      hi = mid;
    else
      lo = mid;
  }
  out[i] = expf(0.5f * (lo + hi));
}

}  // namespace ddm

extern "C" int ddm_model_curves(int32_t n, int32_t K, const float* qn, const float* theta, int32_t nt,
                                const float* tau, float noise, uint64_t seed, float* y, float* tau_e,
                                void* stream) {
  ddm_detached_error().clear();
  if (n < 0 || K < 1 || K > ddm::LM_MAX_NODES || nt < 0 || !(noise >= 0))
    return lm_fail(DDM_ERR_ARG, "ddm_model_curves: need n >= 0, 1 <= K <= %d, nt >= 0, noise >= 0",
                   ddm::LM_MAX_NODES);
  if (n == 0) return DDM_OK;
  if (!qn || !theta || (nt > 0 && (!tau || !y))) return lm_fail(DDM_ERR_ARG, "ddm_model_curves: null array");
  cudaStream_t s = (cudaStream_t)stream;
  const long long tot = (long long)n * nt;
  if (tot > 0) ddm::curves_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(n, K, qn, theta, nt, tau, noise, seed, y);
  if (tau_e) ddm::tau_e_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, K, qn, theta, tau_e);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return lm_fail(DDM_ERR_CUDA, "ddm_model_curves: %s", cudaGetErrorString(e));
  return DDM_OK;
}
