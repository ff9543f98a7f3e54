/*
 * FP64 per-bin Levenberg-Marquardt oracle for the motility model.
 * TEST INFRASTRUCTURE ONLY: the checker for the GPU batched LM.
 *
 * The reference fits its model globally by VarPro + Nelder-Mead
 * (motility-ddm/src/motility_fit.js:577-611); it has no LM. This file states
 * the per-bin problem the GPU solves, in FP64, with the reference's model
 * column (modelColumn, motility_fit.js:417-432: the 3D Schulz ISF averaged
 * over the bin's effective-|k| nodes) and the reference's parameter bounds
 * (bounds(), motility_fit.js:480-491):
 *
 *   y(tau) = A c(tau) + B,  c = 1 - <exp(-D q^2 tau) (1 - alpha + alpha g(q vbar tau; Z))>_nodes
 *   theta = (A, B, alpha, ln vbar, ln Z, ln D), A, B >= 0, alpha in [0, 1],
 *   ln vbar, ln Z, ln D clamped to the bounds,
 *   cost = sum_j (w (y(tau_j) - d_j))^2.
 *
 * Marquardt's method with diagonal scaling: solve (H + lambda diag H) delta =
 * -g, project onto the bounds, accept if the cost drops (lambda /= 3) else
 * reject (lambda *= 4); stop after two consecutive accepted steps whose
 * relative cost decrease is below tol, or when lambda exceeds 1e12, or at
 * max_iter. The GPU kernel implements the same iteration (model in FP32,
 * normal equations in FP64).
 */
#include <math.h>
#include <string.h>

#include "oracle.h"

#define NP 6

/* g(x; Z) = <sin(q v tau)/(q v tau)>_Schulz (motility_fit.js:140-144) and
 * its log-derivatives x dg/dx, Z dg/dZ. */
static void isf3d_d(double x, double Z, double *g, double *gx, double *gz) {
  const double L = x / (Z + 1);
  if (L < 1e-4) {
    *g = 1 - (x * x * (Z + 2)) / (6 * (Z + 1));
    *gx = -2 * x * x * (Z + 2) / (6 * (Z + 1));
    *gz = x * x * Z / (6 * (Z + 1) * (Z + 1));
    return;
  }
  const double a = atan(L), u = 1 + L * L, lu = log1p(L * L);
  const double U = exp(0.5 * Z * lu);
  const double s = sin(Z * a), c = cos(Z * a);
  const double G = s / (Z * L * U);
  const double LgL = c / (u * U) - G * (1 + Z * L * L / u); /* L dg/dL at fixed Z */
  *g = G;
  *gx = LgL;
  *gz = a * c / (L * U) - G - 0.5 * Z * G * lu - (Z / (Z + 1)) * LgL;
}

typedef struct {
  int nt, K;
  const double *d, *tau, *qn;
  double w;
  double lo[NP], hi[NP];
} lm_prob;

/* residuals r[j] and (if J) Jacobian rows J[j*6 + p]; returns the cost */
static double model(const lm_prob *P, const double *th, double *r, double *J) {
  const double A = th[0], B = th[1], al = th[2];
  const double v = exp(th[3]), Z = exp(th[4]), D = exp(th[5]);
  double cost = 0;
  for (int j = 0; j < P->nt; j++) {
    const double t = P->tau[j];
    double sE = 0, sEg = 0, sdD = 0, sgx = 0, sgz = 0;
    for (int n = 0; n < P->K; n++) {
      const double q = P->qn[n];
      const double E = exp(-D * q * q * t);
      double g, gx, gz;
      isf3d_d(q * v * t, Z, &g, &gx, &gz);
      sE += E * (1 - al + al * g);
      sEg += E * (g - 1);
      sdD += E * D * q * q * t * (1 - al + al * g);
      sgx += E * al * gx;
      sgz += E * al * gz;
    }
    const double iK = 1.0 / P->K;
    const double c = 1 - sE * iK;
    const double y = A * c + B;
    const double rr = P->w * (y - P->d[j]);
    r[j] = rr;
    cost += rr * rr;
    if (J) {
      double *Jj = J + j * NP;
      Jj[0] = P->w * c;
      Jj[1] = P->w;
      Jj[2] = -P->w * A * sEg * iK;
      Jj[3] = -P->w * A * sgx * iK;
      Jj[4] = -P->w * A * sgz * iK;
      Jj[5] = P->w * A * sdD * iK;
    }
  }
  return cost;
}

static void project(const lm_prob *P, double *th) {
  for (int p = 0; p < NP; p++) th[p] = fmin(P->hi[p], fmax(P->lo[p], th[p]));
}

/* Cholesky solve of the 6x6 SPD system M x = b; 0 if not positive definite */
static int chol6(double M[NP][NP], const double *b, double *x) {
  double Lm[NP][NP];
  memset(Lm, 0, sizeof Lm);
  for (int i = 0; i < NP; i++) {
    for (int j = 0; j <= i; j++) {
      double s = M[i][j];
      for (int k = 0; k < j; k++) s -= Lm[i][k] * Lm[j][k];
      if (i == j) {
        if (!(s > 0)) return 0;
        Lm[i][i] = sqrt(s);
      } else {
        Lm[i][j] = s / Lm[j][j];
      }
    }
  }
  double y[NP];
  for (int i = 0; i < NP; i++) {
    double s = b[i];
    for (int k = 0; k < i; k++) s -= Lm[i][k] * y[k];
    y[i] = s / Lm[i][i];
  }
  for (int i = NP - 1; i >= 0; i--) {
    double s = y[i];
    for (int k = i + 1; k < NP; k++) s -= Lm[k][i] * x[k];
    x[i] = s / Lm[i][i];
  }
  return 1;
}

/* One bin. bounds6 = (vmin, vmax, Zmin, Zmax, Dmin, Dmax). Returns iterations;
 * theta (6) in/out, *cost_out. */
int or_lm_fit(int nt, int K, const double *d, const double *tau, const double *qn, double w,
              const double *bounds6, double *theta, int max_iter, double tol, double *cost_out) {
  lm_prob P = {nt, K, d, tau, qn, w, {0}, {0}};
  P.lo[0] = 0;
  P.hi[0] = INFINITY;
  P.lo[1] = 0;
  P.hi[1] = INFINITY;
  P.lo[2] = 0;
  P.hi[2] = 1;
  P.lo[3] = log(bounds6[0]);
  P.hi[3] = log(bounds6[1]);
  P.lo[4] = log(bounds6[2]);
  P.hi[4] = log(bounds6[3]);
  P.lo[5] = log(bounds6[4]);
  P.hi[5] = log(bounds6[5]);
  double r[512], J[512 * NP], rt[512], Jt[512 * NP];
  if (nt > 512) return -1;
  project(&P, theta);
  double cost = model(&P, theta, r, J);
  double lambda = 1e-3;
  int small = 0, it = 0;
  double H[NP][NP], g[NP];
  int need_normal = 1;
  for (it = 0; it < max_iter; it++) {
    if (need_normal) {
      for (int a = 0; a < NP; a++) {
        g[a] = 0;
        for (int b = 0; b < NP; b++) H[a][b] = 0;
      }
      for (int j = 0; j < nt; j++)
        for (int a = 0; a < NP; a++) {
          g[a] += J[j * NP + a] * r[j];
          for (int b = 0; b < NP; b++) H[a][b] += J[j * NP + a] * J[j * NP + b];
        }
      need_normal = 0;
    }
    double M[NP][NP], mg[NP], delta[NP];
    for (int a = 0; a < NP; a++) {
      for (int b = 0; b < NP; b++) M[a][b] = H[a][b];
      M[a][a] += lambda * (H[a][a] > 0 ? H[a][a] : 1e-30);
      mg[a] = -g[a];
    }
    if (!chol6(M, mg, delta)) {
      lambda *= 4;
      if (lambda > 1e12) break;
      continue;
    }
    double th2[NP];
    for (int p = 0; p < NP; p++) th2[p] = theta[p] + delta[p];
    project(&P, th2);
    const double c2 = model(&P, th2, rt, Jt);
    if (c2 < cost) {
      const double rel = (cost - c2) / (cost > 0 ? cost : 1e-300);
      memcpy(theta, th2, sizeof th2);
      memcpy(r, rt, sizeof(double) * nt);
      memcpy(J, Jt, sizeof(double) * nt * NP);
      cost = c2;
      need_normal = 1;
      lambda /= 3;
      if (lambda < 1e-12) lambda = 1e-12;
      small = rel < tol ? small + 1 : 0;
      if (small >= 2) {
        it++;
        break;
      }
    } else {
      lambda *= 4;
      if (lambda > 1e12) break;
    }
  }
  *cost_out = cost;
  return it;
}

/* Model curve y(tau) for given theta (used to synthesise test curves). */
void or_lm_model(int nt, int K, const double *tau, const double *qn, const double *theta,
                 double *y) {
  double zero[512];
  memset(zero, 0, sizeof zero);
  lm_prob P = {nt, K, zero, tau, qn, 1.0, {0}, {0}};
  double r[512];
  model(&P, theta, r, NULL);
  for (int j = 0; j < nt; j++) y[j] = r[j];
}

/* ------------------------------------------------------------------ starts */

/* VarPro amplitudes at fixed (alpha, vbar, Z, D): the 2-column NNLS of
 * evalModel (motility_fit.js:450-474) by nnls3's support enumeration
 * (:243-263) over {A}, {B}, {A, B}; returns the weighted cost and A, B. */
static double varpro(const lm_prob *P, double al, double lv, double lZ, double lD, double *A,
                     double *B) {
  double th[NP] = {1, 0, al, lv, lZ, lD}, r[512];
  /* model() with A = 1, B = 0 and d = 0 gives w*c in r */
  lm_prob Q = *P;
  double zero[512];
  memset(zero, 0, sizeof(double) * P->nt);
  Q.d = zero;
  Q.w = 1.0;
  model(&Q, th, r, NULL);
  double g11 = 0, g12 = 0, h1 = 0, h2 = 0, dd = 0;
  for (int j = 0; j < P->nt; j++) {
    const double c = r[j], d = P->d[j];
    g11 += c * c;
    g12 += c;
    h1 += c * d;
    h2 += d;
    dd += d * d;
  }
  const double n = P->nt;
  double best = dd, bA = 0, bB = 0;
  /* {A} */
  if (g11 > 1e-300) {
    const double a = h1 / g11;
    const double rs = dd - a * h1;
    if (a >= 0 && rs < best) best = rs, bA = a, bB = 0;
  }
  /* {B} */
  {
    const double b = h2 / n;
    const double rs = dd - b * h2;
    if (b >= 0 && rs < best) best = rs, bA = 0, bB = b;
  }
  /* {A, B} */
  {
    const double det = g11 * n - g12 * g12;
    const double sc = fmax(g11, n);
    if (fabs(det) > 1e-11 * sc * sc) {
      const double a = (h1 * n - g12 * h2) / det, b = (g11 * h2 - g12 * h1) / det;
      const double rs = dd - a * h1 - b * h2;
      if (a >= 0 && b >= 0 && rs < best) best = rs, bA = a, bB = b;
    }
  }
  *A = bA;
  *B = bB;
  return fmax(best, 0.0) * P->w * P->w;
}

static void init_prob(lm_prob *P, int nt, int K, const double *d, const double *tau,
                      const double *qn, double w, const double *bounds6) {
  P->nt = nt;
  P->K = K;
  P->d = d;
  P->tau = tau;
  P->qn = qn;
  P->w = w;
  P->lo[0] = 0;
  P->hi[0] = INFINITY;
  P->lo[1] = 0;
  P->hi[1] = INFINITY;
  P->lo[2] = 0;
  P->hi[2] = 1;
  P->lo[3] = log(bounds6[0]);
  P->hi[3] = log(bounds6[1]);
  P->lo[4] = log(bounds6[2]);
  P->hi[4] = log(bounds6[3]);
  P->lo[5] = log(bounds6[4]);
  P->hi[5] = log(bounds6[5]);
}

/* LM from one start (alpha, vbar, Z, D), amplitudes from VarPro. */
int or_lm_fit_start(int nt, int K, const double *d, const double *tau, const double *qn, double w,
                    const double *bounds6, const double *start4, int max_iter, double tol,
                    double *theta, double *cost_out) {
  lm_prob P;
  init_prob(&P, nt, K, d, tau, qn, w, bounds6);
  double th[NP] = {0, 0, start4[0], log(start4[1]), log(start4[2]), log(start4[3])};
  project(&P, th);
  varpro(&P, th[2], th[3], th[4], th[5], &th[0], &th[1]);
  memcpy(theta, th, sizeof th);
  return or_lm_fit(nt, K, d, tau, qn, w, bounds6, theta, max_iter, tol, cost_out);
}

/* The reference's start strategy, per bin (fitBrownian :500-536 then
 * fitSwimmer :577-611 with LM in place of Nelder-Mead):
 *  1. Brownian null (alpha = 0): 49-point scan of ln D over [Dmin, Dmax],
 *     golden section on the bracketing interval (<= 60 steps, width 1e-6);
 *  2. 64 starts at that D: 16 ln vbar at the centres of equal cells of
 *     [vmin, vmax], Z in {1.5, 8}, alpha in {0.3, 0.8}, ranked by the VarPro
 *     cost (stable order on ties);
 *  3. LM from the best `nrefine` starts; the lowest cost wins (first on ties).
 * Returns total LM iterations; *evals counts model evaluations. */
/* fitBrownian's search (motility_fit.js:500-536) for one bin: 49-point scan
 * of ln D, then golden section (<= 60 steps, to 1e-6). Returns ln D. */
static double brownian_search(const lm_prob *Pp, int *ne_out) {
  const lm_prob P = *Pp;
  double A, B;
  int ne = 0;
  const double lo = P.lo[5], hi = P.hi[5];
  const int n = 48;
  int bi = 0;
  double bf = INFINITY, xs[49];
  for (int i = 0; i <= n; i++) {
    xs[i] = lo + ((hi - lo) * i) / n;
    const double v = varpro(&P, 0, P.lo[3], 0, xs[i], &A, &B);
    ne++;
    if (v < bf) bf = v, bi = i;
  }
  double a = xs[bi > 0 ? bi - 1 : 0], b = xs[bi < n ? bi + 1 : n];
  const double gr = (sqrt(5.0) - 1) / 2;
  double c = b - gr * (b - a), dd = a + gr * (b - a);
  double fc = varpro(&P, 0, P.lo[3], 0, c, &A, &B), fd = varpro(&P, 0, P.lo[3], 0, dd, &A, &B);
  ne += 2;
  for (int it = 0; it < 60 && b - a > 1e-6; it++) {
    if (fc < fd) {
      b = dd;
      dd = c;
      fd = fc;
      c = b - gr * (b - a);
      fc = varpro(&P, 0, P.lo[3], 0, c, &A, &B);
    } else {
      a = c;
      c = dd;
      fc = fd;
      dd = a + gr * (b - a);
      fd = varpro(&P, 0, P.lo[3], 0, dd, &A, &B);
    }
    ne++;
  }
  *ne_out += ne;
  return fc < fd ? c : dd;
}

/* The Brownian model alone per bin (alpha = 0): theta = (A, B, 0, ln vbar_lo,
 * ln Z_lo, ln D), cost = VarPro weighted RSS at that D. */
double or_lm_fit_brownian(int nt, int K, const double *d, const double *tau, const double *qn, double w,
                          const double *bounds6, double *theta) {
  lm_prob P;
  init_prob(&P, nt, K, d, tau, qn, w, bounds6);
  int ne = 0;
  const double lD = brownian_search(&P, &ne);
  double A, B;
  const double cost = varpro(&P, 0, P.lo[3], 0, lD, &A, &B);
  theta[0] = A;
  theta[1] = B;
  theta[2] = 0;
  theta[3] = P.lo[3];
  theta[4] = P.lo[4];
  theta[5] = lD;
  return cost;
}

int or_lm_fit_plain(int nt, int K, const double *d, const double *tau, const double *qn, double w,
                    const double *bounds6, int max_iter, double tol, int nrefine, double *theta,
                    double *cost_out, int *evals) {
  lm_prob P;
  init_prob(&P, nt, K, d, tau, qn, w, bounds6);
  double A, B;
  int ne = 0;
  const double lD0 = brownian_search(&P, &ne);
  /* 64 starts */
  double su[64][3], sf[64];
  int ord[64], ns = 0;
  const double lZs[2] = {log(1.5), log(8.0)}, als[2] = {0.3, 0.8};
  for (int i = 0; i < 16; i++) {
    const double lv = P.lo[3] + ((P.hi[3] - P.lo[3]) * (i + 0.5)) / 16;
    for (int z = 0; z < 2; z++)
      for (int q = 0; q < 2; q++) {
        const double lZ = fmin(P.hi[4], fmax(P.lo[4], lZs[z]));
        su[ns][0] = als[q];
        su[ns][1] = lv;
        su[ns][2] = lZ;
        sf[ns] = varpro(&P, als[q], lv, lZ, lD0, &A, &B);
        ord[ns] = ns;
        ns++;
        ne++;
      }
  }
  for (int i = 1; i < ns; i++) { /* stable insertion sort by cost */
    const int o = ord[i];
    int j = i - 1;
    while (j >= 0 && sf[ord[j]] > sf[o]) {
      ord[j + 1] = ord[j];
      j--;
    }
    ord[j + 1] = o;
  }
  double best = INFINITY, bth[NP] = {0};
  int iters = 0;
  for (int s = 0; s < nrefine && s < ns; s++) {
    const int o = ord[s];
    double th[NP] = {0, 0, su[o][0], su[o][1], su[o][2], lD0};
    varpro(&P, th[2], th[3], th[4], th[5], &th[0], &th[1]);
    ne++;
    double cst;
    const int it = or_lm_fit(nt, K, d, tau, qn, w, bounds6, th, max_iter, tol, &cst);
    iters += it;
    ne += 1 + it;
    if (cst < best) {
      best = cst;
      memcpy(bth, th, sizeof th);
    }
  }
  memcpy(theta, bth, sizeof bth);
  *cost_out = best;
  if (evals) *evals = ne;
  return iters;
}
