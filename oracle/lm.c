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
