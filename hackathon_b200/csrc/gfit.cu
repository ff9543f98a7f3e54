// Global VarPro fits of the motility model on the device.
//
// The reference fits ONE parameter set shared by all q-bins -- alpha, vbar, Z,
// D (and a drift speed |V|) -- with the per-bin amplitudes A_b, B_b >= 0
// solved exactly inside every objective evaluation (variable projection;
// evalModel, motility_fit.js:450-474):
//   cost(phi) = sum_b w_b^2 min_{A,B >= 0} sum_j (A c_b(tau_j; phi) + B - d_bj)^2,
//   c_b(tau) = 1 - <exp(-D q^2 tau) J0(q |V| tau) (1 - alpha + alpha g(q vbar tau; Z))>_nodes
// (modelColumn, :417-432). It searches phi with a scan plus golden section
// (Brownian), a grid plus Nelder-Mead (Brownian + drift) and 64 starts plus
// Nelder-Mead from the best three (swimmer), on one CPU thread.
//
// Here every objective evaluation is one pass of a thread-block cluster over
// all bins: warps own bins, lanes own lags (FP64), the two-column NNLS is
// solved per bin from warp-reduced Gram sums, and the per-bin terms are summed
// across the cluster through distributed shared memory, in a fixed order, so
// every thread of the cluster holds the same totals and takes the same
// decisions. Scans and start sets are independent jobs (one cluster each, in
// parallel); the search from a start is a bounded Levenberg-Marquardt
// iteration on the VarPro objective:
//  - gradient: exact (the amplitudes are optimal, so only the explicit
//    dependence through c_b counts): g_k = sum_b w_b^2 A_b <dc_b/dphi_k, r_b>;
//  - curvature: Kaufman's approximation of the projected Jacobian,
//    J_b = w_b (I - P_b) A_b dc_b/dphi, P_b the projector on the active
//    amplitude columns ({c_b, 1}, or {c_b} when B_b = 0);
//  - box constraints: parameters at a bound whose gradient points outward,
//    and directions without curvature, are held for the step; the step is
//    clipped to the box; Marquardt's damping (x1/3 on success, x4 on failure).
// The evaluation is FP64 throughout, as the reference's.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdint>

#include "gfit.cuh"
#include "isf.cuh"

namespace cg = cooperative_groups;

namespace ddm {

namespace {

constexpr int GF_THREADS = 256;
constexpr int GF_WARPS = GF_THREADS / 32;
constexpr int GF_MAX_CLUSTER = 16;  // CTAs per job at most (a non-portable cluster size)
constexpr int GF_NV = 1 + 4 + 10;  // cost, gradient, upper triangle of the 4x4 curvature

template <int M>
struct Free;
template <>
struct Free<GF_BROWN> {
  static constexpr int n = 1;
  __device__ static constexpr int at(int) { return GP_LD; }
};
template <>
struct Free<GF_DRIFT> {
  static constexpr int n = 2;
  __device__ static constexpr int at(int k) { return k == 0 ? GP_LD : GP_V; }
};
template <>
struct Free<GF_SWIM> {
  static constexpr int n = 4;
  __device__ static constexpr int at(int k) { return k; }  // ln vbar, ln Z, ln D, alpha
};

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;  // the xor butterfly leaves the same bits on every lane
}

struct Phys {
  double v, Z, D, al, V;
};

__device__ __forceinline__ Phys phys(const double (&ph)[GP_N]) {
  return Phys{exp(ph[GP_LV]), exp(ph[GP_LZ]), exp(ph[GP_LD]), ph[GP_AL], ph[GP_V]};
}

// Model column c(tau) of one bin and its derivatives along the moving parameters.
template <int M>
__device__ __forceinline__ void column(const GfitProblem& P, const Isf2dTable& tab, const double* qn, double t,
                                       const Phys& p, double& c, double (&e)[Free<M>::n]) {
  const double iK = 1.0 / P.K;
  double sE = 0, sD = 0, sA = 0, sX = 0, sZ = 0, sV = 0;
  for (int n = 0; n < P.K; n++) {
    const double q = qn[n];
    const double Ed = exp(-p.D * q * q * t);
    double J = 1.0, Jv = 0.0;
    if (M == GF_DRIFT || p.V > 0) {  // J0(q |V| tau), the radial average of a uniform drift
      const double y = q * p.V * t;
      J = j0(y);
      if (M == GF_DRIFT) Jv = -j1(y) * q * t;
    }
    const double E = Ed * J;
    double mix = 1.0;
    if (M == GF_SWIM) {
      double g, gx, gz;
      if (P.geometry2d)
        isf2d_d(tab, q * p.v * t, p.Z, g, gx, gz);
      else
        isf3d_d<double>(q * p.v * t, p.Z, g, gx, gz);
      mix = 1.0 - p.al + p.al * g;
      sA += E * (g - 1.0);
      sX += E * p.al * gx;
      sZ += E * p.al * gz;
    }
    sE += E * mix;
    sD += p.D * q * q * t * E * mix;
    if (M == GF_DRIFT) sV += Ed * Jv * mix;
  }
  c = 1.0 - sE * iK;
  if (M == GF_SWIM) {
    e[0] = -sX * iK;  // d c / d ln vbar
    e[1] = -sZ * iK;  // d c / d ln Z
    e[2] = sD * iK;   // d c / d ln D
    e[3] = -sA * iK;  // d c / d alpha
  } else {
    e[0] = sD * iK;
    if (M == GF_DRIFT) e[Free<M>::n - 1] = -sV * iK;  // d c / d |V|
  }
}

// Two-column NNLS from the Gram sums by support enumeration ({A}, {B},
// {A, B}; the first strictly lower RSS wins), as nnls3 with an empty third
// column (motility_fit.js:243-263, 466): Gaussian elimination with partial
// pivoting and the 1e-11 singularity test of solveSmall (:270-291).
__device__ __forceinline__ double nnls2(double g11, double g12, double n, double h1, double h2, double dd,
                                        double& A, double& B, bool& sa, bool& sb) {
  double best = dd;
  A = B = 0.0;
  sa = sb = false;
  if (fabs(g11) >= 1e-11 * fmax(fabs(g11), 1e-300) && g11 != 0.0) {
    const double a = h1 / g11;
    const double rs = dd - a * h1;
    if (a >= 0 && rs < best) best = rs, A = a, B = 0, sa = true, sb = false;
  }
  if (n > 0) {
    const double b = h2 / n;
    const double rs = dd - b * h2;
    if (b >= 0 && rs < best) best = rs, A = 0, B = b, sa = false, sb = true;
  }
  {
    const double sc = fmax(fmax(fabs(g11), fabs(n)), 1e-300);
    // rows (g11, g12 | h1), (g12, n | h2); pivot on the larger first entry
    const bool sw = fabs(g12) > fabs(g11);
    const double p0 = sw ? g12 : g11, p1 = sw ? n : g12, pb = sw ? h2 : h1;
    const double o0 = sw ? g11 : g12, o1 = sw ? g12 : n, ob = sw ? h1 : h2;
    if (fabs(p0) >= 1e-11 * sc) {
      const double f = o0 / p0;
      const double r1 = o1 - f * p1, rb = ob - f * pb;
      if (fabs(r1) >= 1e-11 * sc) {
        const double x1 = rb / r1, x0 = (pb - p1 * x1) / p0;
        const double rs = dd - x0 * h1 - x1 * h2;
        if (x0 >= 0 && x1 >= 0 && rs < best) best = rs, A = x0, B = x1, sa = true, sb = true;
      }
    }
  }
  return fmax(best, 0.0);
}

struct Shared {
  double part[GF_WARPS][GF_NV];
  double cta[2][GF_NV];  // this CTA's totals, double-buffered across evaluations
  double tot[GF_NV];     // cluster totals
};

// Sums GF_NV values held (identically) by the lanes of every warp over the
// CTA, then over the cluster in rank order; every thread returns the totals.
template <int NV>
__device__ __forceinline__ void cluster_total(Shared& sh, cg::cluster_group& cl, int& parity, const double* v,
                                              double* out) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
#pragma unroll
    for (int i = 0; i < NV; i++) sh.part[warp][i] = v[i];
  __syncthreads();
  if (threadIdx.x < NV) {
    double s = 0;
    for (int w = 0; w < GF_WARPS; w++) s += sh.part[w][threadIdx.x];
    sh.cta[parity][threadIdx.x] = s;
  }
  cl.sync();
  if (threadIdx.x < NV) {
    double s = 0;
    for (unsigned r = 0; r < cl.num_blocks(); r++) s += cl.map_shared_rank(&sh.cta[parity][0], r)[threadIdx.x];
    sh.tot[threadIdx.x] = s;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < NV; i++) out[i] = sh.tot[i];
  parity ^= 1;
  // sh.tot and sh.part are rewritten only after the next cluster barrier
}

template <int M>
struct Eval {
  static constexpr int NF = Free<M>::n;
  static constexpr int NS = NF * (NF + 1) / 2;
  static constexpr int NV = 1 + NF + NS;
};

// One evaluation of the objective (and, with JAC, its gradient and curvature)
// at ph. Bins are dealt to the cluster's warps round-robin.
template <int M, bool JAC>
__device__ __noinline__ void evaluate(const GfitProblem& P, const Isf2dTable& tab, const double (&ph)[GP_N], const double (&tau)[4],
                         Shared& sh, cg::cluster_group& cl, int& parity, double* tot) {
  constexpr int NF = Eval<M>::NF, NS = Eval<M>::NS, NV = Eval<M>::NV;
  const int lane = threadIdx.x & 31;
  const int gw = cl.block_rank() * GF_WARPS + (threadIdx.x >> 5), nw = cl.num_blocks() * GF_WARPS;
  const Phys p = phys(ph);
  double acc[NV];
#pragma unroll
  for (int i = 0; i < NV; i++) acc[i] = 0.0;
  for (int b = gw; b < P.nb; b += nw) {
    const double* qn = P.qn + (size_t)b * P.K;
    const double* d = P.d + (size_t)b * P.nt;
    double Scc = 0, Sc = 0, Sdc = 0, Sd = 0, Sdd = 0;
    double Sec[NF], Se[NF], Sed[NF], See[NS];
#pragma unroll
    for (int k = 0; k < NF; k++) Sec[k] = Se[k] = Sed[k] = 0;
#pragma unroll
    for (int k = 0; k < NS; k++) See[k] = 0;
#pragma unroll
    for (int r = 0; r < 4; r++) {
      const int j = lane + 32 * r;
      if (j >= P.nt) break;
      const double dj = d[j];
      double c, e[NF];
      column<M>(P, tab, qn, tau[r], p, c, e);
      Scc += c * c;
      Sc += c;
      Sdc += dj * c;
      Sd += dj;
      Sdd += dj * dj;
      if (JAC) {
        int s = 0;
#pragma unroll
        for (int k = 0; k < NF; k++) {
          Sec[k] += e[k] * c;
          Se[k] += e[k];
          Sed[k] += e[k] * dj;
#pragma unroll
          for (int l = k; l < NF; l++) See[s++] += e[k] * e[l];
        }
      }
    }
    Scc = wsum(Scc);
    Sc = wsum(Sc);
    Sdc = wsum(Sdc);
    Sd = wsum(Sd);
    Sdd = wsum(Sdd);
    double A, B;
    bool sa, sb;
    const double n = P.nt;
    const double rss = nnls2(Scc, Sc, n, Sdc, Sd, Sdd, A, B, sa, sb);
    const double w2 = P.w[b] * P.w[b];
    acc[0] += rss * w2;
    if (JAC && sa && A > 0) {
#pragma unroll
      for (int k = 0; k < NF; k++) {
        Sec[k] = wsum(Sec[k]);
        Se[k] = wsum(Se[k]);
        Sed[k] = wsum(Sed[k]);
      }
#pragma unroll
      for (int k = 0; k < NS; k++) See[k] = wsum(See[k]);
#pragma unroll
      for (int k = 0; k < NF; k++) acc[1 + k] += w2 * A * (A * Sec[k] + B * Se[k] - Sed[k]);
      const double det = Scc * n - Sc * Sc;
      const bool both = sb && det > 1e-300;
      int s = 0;
#pragma unroll
      for (int k = 0; k < NF; k++) {
#pragma unroll
        for (int l = k; l < NF; l++) {
          double proj;
          if (both)  // u^T G^-1 u' with u = (<c, e_k>, <1, e_k>), G = [[Scc, Sc], [Sc, n]]
            proj = (Sec[k] * (n * Sec[l] - Sc * Se[l]) + Se[k] * (Scc * Se[l] - Sc * Sec[l])) / det;
          else
            proj = Scc > 0 ? Sec[k] * Sec[l] / Scc : 0.0;
          acc[1 + NF + s] += w2 * A * A * (See[s] - proj);
          s++;
        }
      }
    }
  }
  cluster_total<NV>(sh, cl, parity, acc, tot);
}

// (H + lambda diag H) delta = -g on the free set by Cholesky; false if not
// positive definite.
template <int NF>
__device__ __forceinline__ bool solve_free(const double* H, const double* g, const int* fi, int nf, double lambda,
                                           double* delta) {
  double Mx[4][4], Lm[4][4], y[4];
  auto hidx = [](int a, int b) {  // upper-triangle index of (a, b), a <= b
    int k = 0;
    for (int i = 0; i < a; i++) k += NF - i;
    return k + (b - a);
  };
  for (int a = 0; a < nf; a++)
    for (int b = 0; b < nf; b++) {
      const int i = fi[a] < fi[b] ? fi[a] : fi[b], j = fi[a] < fi[b] ? fi[b] : fi[a];
      Mx[a][b] = H[hidx(i, j)];
    }
  for (int a = 0; a < nf; a++) Mx[a][a] *= 1.0 + lambda;
  for (int i = 0; i < nf; i++) {
    for (int j = 0; j <= i; j++) {
      double s = Mx[i][j];
      for (int q = 0; q < j; q++) s -= Lm[i][q] * Lm[j][q];
      if (i == j) {
        if (!(s > 0)) return false;
        Lm[i][i] = sqrt(s);
      } else {
        Lm[i][j] = s / Lm[j][j];
      }
    }
  }
  for (int i = 0; i < nf; i++) {
    double s = -g[fi[i]];
    for (int q = 0; q < i; q++) s -= Lm[i][q] * y[q];
    y[i] = s / Lm[i][i];
  }
  for (int i = nf - 1; i >= 0; i--) {
    double s = y[i];
    for (int q = i + 1; q < nf; q++) s -= Lm[q][i] * delta[q];
    delta[i] = s / Lm[i][i];
  }
  return true;
}

// The objective at a point of the moving parameters, clamped to the job's box
// first (the reference clamps inside its objective: unpack, :581-587, :547-553).
template <int M>
__device__ __forceinline__ double cost_at(const GfitProblem& P, const Isf2dTable& tab, const GfitJob& J,
                                          const double* u, const double (&tau)[4], Shared& sh, cg::cluster_group& cl,
                                          int& parity) {
  double ph[GP_N], t[Eval<M>::NV];
#pragma unroll
  for (int i = 0; i < GP_N; i++) ph[i] = J.phi[i];
#pragma unroll
  for (int k = 0; k < Free<M>::n; k++) {
    const int q = Free<M>::at(k);
    ph[q] = fmin(J.hi[q], fmax(J.lo[q], u[k]));
  }
  evaluate<M, false>(P, tab, ph, tau, sh, cl, parity, t);
  return t[0];
}

// The reference's Nelder-Mead (nelderMead, motility_fit.js:302-350) on the
// device objective: the same initial simplex, the stable ordering of the
// vertices, reflection (-1), expansion (-2), outside/inside contraction
// (-1/2, +1/2), shrink (1/2) and the relative spread test. Every thread of the
// cluster holds the same simplex. Vertex arithmetic is rounded operation by
// operation (no fused multiply-add), as the reference's JavaScript.
template <int M>
__device__ void nelder_mead(const GfitProblem& P, const Isf2dTable& tab, const GfitJob& J, int max_iter,
                            const double (&tau)[4], Shared& sh, cg::cluster_group& cl, int& parity, double* xbest,
                            double& fbest, int& iters, int& evals, bool& conv) {
  constexpr int n = Free<M>::n;
  double S[n + 1][n], F[n + 1];
#pragma unroll
  for (int i = 0; i <= n; i++)
#pragma unroll
    for (int j = 0; j < n; j++) S[i][j] = J.phi[Free<M>::at(j)];
#pragma unroll
  for (int i = 0; i < n; i++) S[i + 1][i] = __dadd_rn(S[i + 1][i], J.step[i]);
  for (int i = 0; i <= n; i++) F[i] = cost_at<M>(P, tab, J, S[i], tau, sh, cl, parity);
  evals = n + 1;
  conv = false;
  int it = 0;
  for (; it < max_iter; it++) {
    // stable sort by cost (insertion sort: equal costs keep their order)
    for (int i = 1; i <= n; i++) {
      const double fk = F[i];
      double xk[n];
#pragma unroll
      for (int j = 0; j < n; j++) xk[j] = S[i][j];
      int k = i - 1;
      while (k >= 0 && F[k] > fk) {
        F[k + 1] = F[k];
#pragma unroll
        for (int j = 0; j < n; j++) S[k + 1][j] = S[k][j];
        k--;
      }
      F[k + 1] = fk;
#pragma unroll
      for (int j = 0; j < n; j++) S[k + 1][j] = xk[j];
    }
    if (fabs(F[n] - F[0]) <= J.tol * (fabs(F[0]) + 1e-30)) {
      conv = true;
      break;
    }
    double c[n];
#pragma unroll
    for (int j = 0; j < n; j++) {
      c[j] = 0.0;
      for (int i = 0; i < n; i++) c[j] = __dadd_rn(c[j], __ddiv_rn(S[i][j], (double)n));
    }
    auto pt = [&](double t, double* x) {
#pragma unroll
      for (int j = 0; j < n; j++) x[j] = __dadd_rn(c[j], __dmul_rn(t, __dsub_rn(S[n][j], c[j])));
    };
    double xr[n], xe[n], xc[n];
    pt(-1.0, xr);
    const double fr = cost_at<M>(P, tab, J, xr, tau, sh, cl, parity);
    evals++;
    if (fr < F[0]) {
      pt(-2.0, xe);
      const double fe = cost_at<M>(P, tab, J, xe, tau, sh, cl, parity);
      evals++;
      const bool ex = fe < fr;
#pragma unroll
      for (int j = 0; j < n; j++) S[n][j] = ex ? xe[j] : xr[j];
      F[n] = ex ? fe : fr;
    } else if (fr < F[n - 1]) {
#pragma unroll
      for (int j = 0; j < n; j++) S[n][j] = xr[j];
      F[n] = fr;
    } else {
      const bool outside = fr < F[n];
      pt(outside ? -0.5 : 0.5, xc);
      const double fc = cost_at<M>(P, tab, J, xc, tau, sh, cl, parity);
      evals++;
      if (fc < (outside ? fr : F[n])) {
#pragma unroll
        for (int j = 0; j < n; j++) S[n][j] = xc[j];
        F[n] = fc;
      } else {
        for (int i = 1; i <= n; i++) {
#pragma unroll
          for (int j = 0; j < n; j++) S[i][j] = __dadd_rn(S[0][j], __dmul_rn(0.5, __dsub_rn(S[i][j], S[0][j])));
          F[i] = cost_at<M>(P, tab, J, S[i], tau, sh, cl, parity);
          evals++;
        }
      }
    }
  }
  int ib = 0;
  for (int i = 1; i <= n; i++)
    if (F[i] < F[ib]) ib = i;
#pragma unroll
  for (int j = 0; j < n; j++) xbest[j] = S[ib][j];
  fbest = F[ib];
  iters = it;
}

// fitBrownian's golden section of ln D on the bracket [lo, hi] (:514-533): at
// most 60 steps, until the bracket is narrower than 1e-6.
__device__ void golden(const GfitProblem& P, const Isf2dTable& tab, const GfitJob& J, const double (&tau)[4],
                       Shared& sh, cg::cluster_group& cl, int& parity, double& x, double& fx, int& iters, bool& conv) {
  double a = J.lo[GP_LD], b = J.hi[GP_LD];
  const double gr = (sqrt(5.0) - 1) / 2;
  double c = __dsub_rn(b, __dmul_rn(gr, __dsub_rn(b, a)));
  double d = __dadd_rn(a, __dmul_rn(gr, __dsub_rn(b, a)));
  double u = c;
  double fc = cost_at<GF_BROWN>(P, tab, J, &u, tau, sh, cl, parity);
  u = d;
  double fd = cost_at<GF_BROWN>(P, tab, J, &u, tau, sh, cl, parity);
  int it = 0;
  for (; it < 60 && b - a > 1e-6; it++) {
    if (fc < fd) {
      b = d;
      d = c;
      fd = fc;
      c = __dsub_rn(b, __dmul_rn(gr, __dsub_rn(b, a)));
      u = c;
      fc = cost_at<GF_BROWN>(P, tab, J, &u, tau, sh, cl, parity);
    } else {
      a = c;
      c = d;
      fc = fd;
      d = __dadd_rn(a, __dmul_rn(gr, __dsub_rn(b, a)));
      u = d;
      fd = cost_at<GF_BROWN>(P, tab, J, &u, tau, sh, cl, parity);
    }
  }
  conv = !(b - a > 1e-6);
  x = fc < fd ? c : d;
  fx = fc < fd ? fc : fd;
  iters = it;
}

template <int M>
__global__ void __launch_bounds__(GF_THREADS) gfit_kernel(GfitLaunch a) {
  constexpr int NF = Eval<M>::NF, NV = Eval<M>::NV;
  __shared__ Shared sh;
  cg::cluster_group cl = cg::this_cluster();
  const int job = blockIdx.x / cl.num_blocks();
  if (job >= a.njobs) return;  // whole clusters (the grid is a multiple of the cluster)
  const GfitJob J = a.jobs[job];
  const GfitProblem P = a.probs[J.prob];
  const int lane = threadIdx.x & 31;
  double tau[4];
#pragma unroll
  for (int r = 0; r < 4; r++) {
    const int j = lane + 32 * r;
    tau[r] = j < P.nt ? P.tau[j] : 0.0;
  }
  double ph[GP_N];
#pragma unroll
  for (int i = 0; i < GP_N; i++) ph[i] = J.phi[i];
  int parity = 0;
  double tot[NV];
  GfitResult R{};
  if (J.kind == GJ_EVAL) {
    evaluate<M, false>(P, a.tab, ph, tau, sh, cl, parity, tot);
    R.cost = tot[0];
  } else if (J.kind == GJ_NM) {
    double x[NF], f;
    bool conv;
    nelder_mead<M>(P, a.tab, J, J.max_iter > 0 ? J.max_iter : a.max_iter, tau, sh, cl, parity, x, f, R.iters,
                   R.evals, conv);
#pragma unroll
    for (int k = 0; k < NF; k++) {  // the clamped point, unpack(best.x)
      const int q = Free<M>::at(k);
      ph[q] = fmin(J.hi[q], fmax(J.lo[q], x[k]));
    }
    R.cost = f;
    R.status = conv ? 1 : 0;
  } else if (J.kind == GJ_GOLDEN) {
    double x, f;
    bool conv;
    golden(P, a.tab, J, tau, sh, cl, parity, x, f, R.iters, conv);
    ph[GP_LD] = x;
    R.cost = f;
    R.status = conv ? 1 : 0;
  } else if (J.kind == GJ_LM) {
#pragma unroll
    for (int k = 0; k < NF; k++) {
      const int q = Free<M>::at(k);
      ph[q] = fmin(J.hi[q], fmax(J.lo[q], ph[q]));
    }
    evaluate<M, true>(P, a.tab, ph, tau, sh, cl, parity, tot);
    double cost = tot[0], lambda = 1e-3;
    int small = 0, it = 0;
    bool conv = false;
    for (it = 0; it < a.max_iter; it++) {
      const double* g = tot + 1;
      const double* H = tot + 1 + NF;
      // free set: not pressed against a bound, with curvature
      int fi[4], nf = 0;
      double hmax = 0;
      {
        int s = 0;
        for (int k = 0; k < NF; k++) {
          hmax = fmax(hmax, H[s]);
          s += NF - k;
        }
      }
      {
        int s = 0;
        for (int k = 0; k < NF; k++) {
          const int q = Free<M>::at(k);
          const bool lo = ph[q] <= J.lo[q] && g[k] > 0, hi = ph[q] >= J.hi[q] && g[k] < 0;
          if (!lo && !hi && H[s] > 1e-14 * hmax) fi[nf++] = k;
          s += NF - k;
        }
      }
      if (nf == 0) {
        conv = true;
        break;
      }
      double delta[4];
      if (!solve_free<NF>(H, g, fi, nf, lambda, delta)) {
        lambda *= 4;
        if (lambda > 1e10) {
          conv = true;
          break;
        }
        continue;
      }
      double p2[GP_N];
      bool moved = false;
#pragma unroll
      for (int i = 0; i < GP_N; i++) p2[i] = ph[i];
      for (int a2 = 0; a2 < nf; a2++) {
        const int q = Free<M>::at(fi[a2]);
        p2[q] = fmin(J.hi[q], fmax(J.lo[q], ph[q] + delta[a2]));
        moved |= p2[q] != ph[q];
      }
      if (!moved) {
        conv = true;
        break;
      }
      double t2[NV];
      evaluate<M, true>(P, a.tab, p2, tau, sh, cl, parity, t2);
      if (t2[0] < cost) {
        const double rel = (cost - t2[0]) / fmax(cost, 1e-300);
#pragma unroll
        for (int i = 0; i < GP_N; i++) ph[i] = p2[i];
#pragma unroll
        for (int i = 0; i < NV; i++) tot[i] = t2[i];
        cost = t2[0];
        lambda = fmax(lambda / 3, 1e-12);
        small = rel < a.tol ? small + 1 : 0;
        if (small >= 2) {
          it++;
          conv = true;
          break;
        }
      } else {
        lambda *= 4;
        if (lambda > 1e10) {
          conv = true;
          break;
        }
      }
    }
    R.cost = cost;
    R.iters = it;
    R.status = conv ? 1 : 0;
  } else {  // GJ_FINAL
    // amplitudes and lag-1 residual products; one pass like evaluate<M, false>
    const int gw = cl.block_rank() * GF_WARPS + (threadIdx.x >> 5), nw = cl.num_blocks() * GF_WARPS;
    const Phys p = phys(ph);
    double acc[3] = {0, 0, 0};
    for (int b = gw; b < P.nb; b += nw) {
      const double* qn = P.qn + (size_t)b * P.K;
      const double* d = P.d + (size_t)b * P.nt;
      double c[4] = {0, 0, 0, 0};
      double Scc = 0, Sc = 0, Sdc = 0, Sd = 0, Sdd = 0;
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int j = lane + 32 * r;
        if (j >= P.nt) break;
        double e[NF];
        column<M>(P, a.tab, qn, tau[r], p, c[r], e);
        const double dj = d[j];
        Scc += c[r] * c[r];
        Sc += c[r];
        Sdc += dj * c[r];
        Sd += dj;
        Sdd += dj * dj;
      }
      double A, B;
      bool sa, sb;
      const double rss = nnls2(wsum(Scc), wsum(Sc), (double)P.nt, wsum(Sdc), wsum(Sd), wsum(Sdd), A, B, sa, sb);
      const double w = P.w[b];
      acc[0] += rss * w * w;
      // residuals (d - A c - B) w at consecutive lags: lag j-1 sits on the lane before
      double num = 0, den = 0, last = 0;
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int j = lane + 32 * r;
        const double rr = j < P.nt ? (d[j] - (A * c[r] + B)) * w : 0.0;
        double prev = __shfl_up_sync(0xffffffffu, rr, 1);
        const double wrap = __shfl_sync(0xffffffffu, last, 31);  // lag 32 r - 1
        if (lane == 0) prev = wrap;
        if (j < P.nt) {
          den += rr * rr;
          if (j > 0) num += prev * rr;
        }
        last = rr;
      }
      acc[1] += wsum(num);
      acc[2] += wsum(den);
      if (lane == 0 && P.amps) {
        P.amps[2 * b] = A;
        P.amps[2 * b + 1] = B;
      }
    }
    cluster_total<3>(sh, cl, parity, acc, tot);
    R.cost = tot[0];
    R.num = tot[1];
    R.den = tot[2];
    // drift-lag mask of the swimmer fit: |g(q_b vbar tau dt; Z)| < 0.2
    if (M == GF_SWIM && P.dmask) {
      const long long total = (long long)P.nb * P.Lr;
      const long long stride = (long long)cl.num_blocks() * blockDim.x;
      for (long long i = (long long)cl.block_rank() * blockDim.x + threadIdx.x; i < total; i += stride) {
        const int b = (int)(i / P.Lr), t = (int)(i % P.Lr);
        uint8_t m = 0;
        if (t >= 1 && t <= P.Lr - 2) {
          double g, gx, gz;
          const double x = P.qc[b] * p.v * t * P.dt;
          if (P.geometry2d)
            isf2d_d(a.tab, x, p.Z, g, gx, gz);
          else
            isf3d_d<double>(x, p.Z, g, gx, gz);
          m = fabs(g) < 0.2 ? 1 : 0;
        }
        P.dmask[i] = m;
      }
    }
  }
  if (cl.block_rank() == 0 && threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < GP_N; i++) R.phi[i] = ph[i];
    a.res[job] = R;
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// CTAs per job: about two bins per warp (each warp walks its bins in turn,
// so fewer bins per warp shortens every objective evaluation, the search's
// serial step), a power of two from 2 to 16, but no more than leaves every
// job of the launch a cluster at once (a batch of records runs many jobs:
// smaller clusters, more of them in flight), and no more than the device can
// co-schedule as one cluster.
template <int M>
int cluster_size(const GfitLaunch& a) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  int want = 2;
  while (want < GF_MAX_CLUSTER && want * GF_WARPS * 2 < a.max_bins && 2 * want * a.njobs <= sms) want *= 2;
  auto k = gfit_kernel<M>;
  if (want > 8) cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  for (; want > 2; want /= 2) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)want);
    cfg.blockDim = dim3(GF_THREADS);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = want;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k, &cfg) == cudaSuccess && n >= 1) break;
    cudaGetLastError();
  }
  return want;
}

template <int M>
cudaError_t launch_model(const GfitLaunch& a, cudaStream_t s) {
  const int cl = cluster_size<M>(a);
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(a.njobs * cl));
  cfg.blockDim = dim3(GF_THREADS);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, gfit_kernel<M>, a);
}

}  // namespace

// All jobs of one launch share a model (the job's .model is checked by the
// host before the launch).
cudaError_t launch_gfit_model(int model, const GfitLaunch& a, cudaStream_t s) {
  if (a.njobs <= 0) return cudaSuccess;
  switch (model) {
    case GF_BROWN: return launch_model<GF_BROWN>(a, s);
    case GF_DRIFT: return launch_model<GF_DRIFT>(a, s);
    case GF_SWIM: return launch_model<GF_SWIM>(a, s);
  }
  return cudaErrorInvalidValue;
}

}  // namespace ddm
