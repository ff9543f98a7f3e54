// The decision layer of the analysis path: the motility fit and verdict of
// motility-ddm's analyzeMotility (motility-ddm/src/motility_fit.js) on a
// Radial record -- special functions, Schulz swimmer ISF kernels (3D closed
// form, 2D Legendre form and its table), exact 2-column NNLS, bounded
// Nelder-Mead, the VarPro model column averaged over each bin's effective-|k|
// nodes, Brownian / Brownian+drift / swimmer fits, the phase-drift LSQ, the
// temporal structure index, the residual autocorrelation and effective N,
// BIC, the q-scaling exponent, and the five falsification gates. Host code in
// FP64, like the reference's worker (motility_fit.js:996-1004); it runs on
// the Radial record the GPU engine produces (ddm_read_radial) and returns the
// reference's result fields (C ABI ddm_analyze_motility).
//
// Published constants that must be identical for FP64 parity: the rational
// J0 approximation (Numerical Recipes' bessj0), the Lanczos g=7, n=9 ln-Gamma
// coefficients, and the gate thresholds (motility_fit.js:28-38).
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/ddm_b200.h"
#include "motility.h"

/* GATES (motility_fit.js:28-38); SWIM_MIN_UM_S comes from mf_options. */
#define TSI_MIN 0.15
#define FLOW_SIGMA 3.0
#define FLOW_MIN_UM_S 2.0
#define DBIC_MIN 10.0
#define ALPHA_MIN 0.05
#define DRIFT_ISF_MAX 0.2

static double js_round(double x) {
  const double f = floor(x);
  return (x - f >= 0.5) ? f + 1.0 : f;
}
static double clampd(double x, double lo, double hi) { /* :493 */
  return fmin(hi, fmax(lo, x));
}

/* ---------------------------------------------------------- special functions */

double mf_bessel_j0(double x) { /* :54-68 */
  const double ax = fabs(x);
  if (ax < 8) {
    const double y = x * x;
    const double a1 = 57568490574.0 + y * (-13362590354.0 + y * (651619640.7 + y * (-11214424.18 + y * (77392.33017 + y * -184.9052456))));
    const double a2 = 57568490411.0 + y * (1029532985.0 + y * (9494680.718 + y * (59272.64853 + y * (267.8532712 + y))));
    return a1 / a2;
  }
  const double z = 8 / ax;
  const double y = z * z;
  const double xx = ax - 0.785398164;
  const double a1 = 1 + y * (-0.1098628627e-2 + y * (0.2734510407e-4 + y * (-0.2073370639e-5 + y * 0.2093887211e-6)));
  const double a2 = -0.1562499995e-1 + y * (0.1430488765e-3 + y * (-0.6911147651e-5 + y * (0.7621095161e-6 - y * 0.934935152e-7)));
  return sqrt(0.636619772 / ax) * (cos(xx) * a1 - z * sin(xx) * a2);
}

double mf_ln_gamma(double x) { /* :74-86 */
  static const double c[9] = {
      0.99999999999980993, 676.5203681218851, -1259.1392167224028,
      771.32342877765313, -176.61502916214059, 12.507343278686905,
      -0.13857109526572012, 9.9843695780195716e-6, 1.5056327351493116e-7};
  if (x < 0.5) return log(M_PI / fabs(sin(M_PI * x))) - mf_ln_gamma(1 - x);
  x -= 1;
  double a = c[0];
  const double t = x + 7.5;
  for (int i = 1; i < 9; i++) a += c[i] / (x + i);
  return 0.5 * log(2 * M_PI) + (x + 0.5) * log(t) - t + log(a);
}

double mf_schulz_pdf(double v, double vbar, double Z) { /* :95-99 */
  if (v <= 0) return 0;
  const double b = (Z + 1) / vbar;
  return exp(Z * log(v) - mf_ln_gamma(Z + 1) + (Z + 1) * log(b) - b * v);
}

/* Laplace's first integral by the trapezoid rule (:120-132). */
double mf_legendre_p(double nu, double c) {
  const double s = sqrt(fmax(0, 1 - c * c));
  const int n = 16 + (int)ceil(nu * atan2(s, c));
  double sum = 0;
  for (int i = 0; i <= n; i++) {
    const double phi = (M_PI * i) / n;
    const double im = s * cos(phi);
    const double r2 = c * c + im * im;
    const double val = exp(0.5 * nu * log(r2)) * cos(nu * atan2(im, c));
    sum += (i == 0 || i == n) ? 0.5 * val : val;
  }
  return sum / n;
}

double mf_isf3d(double x, double Z) { /* :140-144 */
  const double L = x / (Z + 1);
  if (L < 1e-4) return 1 - (x * x * (Z + 2)) / (6 * (Z + 1));
  return sin(Z * atan(L)) / (Z * L * exp(0.5 * Z * log1p(L * L)));
}

double mf_isf2d(double x, double Z) { /* :152-159 */
  const double L = x / (Z + 1);
  if (L < 1e-4) return 1 - (x * x * (Z + 2)) / (4 * (Z + 1));
  const double u = 1 + L * L;
  const double lnPre = -0.5 * (Z + 1) * log(u);
  if (lnPre < -25) return 0;
  return mf_legendre_p(Z, 1 / sqrt(u)) * exp(lnPre);
}

/* Tabulated 2D kernel (:168-220): rows uniform in ln Z, Catmull-Rom along
 * ln Lambda, quadratic Lagrange across ln Z. */
#define T2D_NZ 72
#define LSER 1e-4
typedef struct {
  double Z, u0, du;
  int n;
  double *v;
} t2d_row;
static t2d_row t2d_rows[T2D_NZ];
static double t2d_lz0, t2d_dlz;
static pthread_once_t t2d_once = PTHREAD_ONCE_INIT;

static double isf2d_exact_lambda(double L, double Z) { /* :186-191 */
  const double u = 1 + L * L;
  const double lnPre = -0.5 * (Z + 1) * log(u);
  if (lnPre < -25) return 0;
  return mf_legendre_p(Z, 1 / sqrt(u)) * exp(lnPre);
}

static void build_table2d(void) { /* :171-184 */
  t2d_lz0 = log(0.5);
  const double lz1 = log(100);
  t2d_dlz = (lz1 - t2d_lz0) / (T2D_NZ - 1);
  for (int i = 0; i < T2D_NZ; i++) {
    const double Z = exp(t2d_lz0 + i * t2d_dlz);
    const double Lc = fmin(1e4, sqrt(expm1(50 / (Z + 1))));
    const double u0 = log(LSER), u1 = log(Lc);
    const double du = fmin(0.04, 0.1 / ((Z + 0.5) / 2));
    const int n = (int)ceil((u1 - u0) / du) + 1;
    double *v = (double *)malloc(sizeof(double) * (n + 2));
    for (int k = 0; k < n + 2; k++) v[k] = isf2d_exact_lambda(exp(u0 + k * du), Z);
    t2d_rows[i].Z = Z;
    t2d_rows[i].u0 = u0;
    t2d_rows[i].du = du;
    t2d_rows[i].n = n;
    t2d_rows[i].v = v;
  }
}

static double row_eval(const t2d_row *r, double x) { /* :193-204 */
  const double L = x / (r->Z + 1);
  if (L < LSER) return 1 - (x * x * (r->Z + 2)) / (4 * (r->Z + 1));
  const double f = (log(L) - r->u0) / r->du;
  if (f >= r->n - 1) return 0;
  const int i = (int)floor(f);
  const double t = f - i;
  const double *v = r->v;
  const double p1 = v[i], p2 = v[i + 1], p3 = v[i + 2];
  const double p0 = i > 0 ? v[i - 1] : 2 * p1 - p2;
  return p1 + 0.5 * t * (p2 - p0 + t * (2 * p0 - 5 * p1 + 4 * p2 - p3 + t * (3 * (p1 - p2) + p3 - p0)));
}

double mf_isf2d_fast(double x, double Z) { /* :212-220 */
  pthread_once(&t2d_once, build_table2d);
  const double zf = (log(fmin(100, fmax(0.5, Z))) - t2d_lz0) / t2d_dlz;
  int i0 = (int)js_round(zf) - 1;
  if (i0 < 0) i0 = 0;
  if (i0 > T2D_NZ - 3) i0 = T2D_NZ - 3;
  const double t = zf - i0;
  const double g0 = row_eval(&t2d_rows[i0], x);
  const double g1 = row_eval(&t2d_rows[i0 + 1], x);
  const double g2 = row_eval(&t2d_rows[i0 + 2], x);
  return 0.5 * (t - 1) * (t - 2) * g0 - t * (t - 2) * g1 + 0.5 * t * (t - 1) * g2;
}

typedef double (*kernel_fn)(double, double);
static kernel_fn swimmer_kernel(int geometry2d) { /* :227-229 */
  return geometry2d ? mf_isf2d_fast : mf_isf3d;
}

/* ---------------------------------------------------------- NNLS (3 columns) */

/* Gaussian elimination with partial pivoting, k <= 3; 0 if singular
 * (:270-291). */
static int solve_small(int k, double A[3][3], const double *b, double *x) {
  double M[3][4];
  double scale = 1e-300;
  for (int i = 0; i < k; i++) {
    for (int j = 0; j < k; j++) M[i][j] = A[i][j];
    M[i][k] = b[i];
  }
  {
    double mx = -INFINITY;
    for (int i = 0; i < k; i++) mx = fmax(mx, fabs(A[i][i]));
    scale = fmax(mx, 1e-300);
  }
  for (int c = 0; c < k; c++) {
    int p = c;
    for (int r = c + 1; r < k; r++)
      if (fabs(M[r][c]) > fabs(M[p][c])) p = r;
    if (fabs(M[p][c]) < 1e-11 * scale) return 0;
    if (p != c)
      for (int j = 0; j <= k; j++) {
        const double t = M[c][j];
        M[c][j] = M[p][j];
        M[p][j] = t;
      }
    for (int r = c + 1; r < k; r++) {
      const double f = M[r][c] / M[c][c];
      for (int j = c; j <= k; j++) M[r][j] -= f * M[c][j];
    }
  }
  for (int r = k - 1; r >= 0; r--) {
    double s = M[r][k];
    for (int j = r + 1; j < k; j++) s -= M[r][j] * x[j];
    x[r] = s / M[r][r];
  }
  return 1;
}

/* Exact NNLS by enumerating supports (:243-263). */
double mf_nnls3(const double *G, const double *h, double dd, double *a) {
  double best_rss = dd;
  a[0] = a[1] = a[2] = 0;
  for (int mask = 1; mask < 8; mask++) {
    int idx[3], k = 0;
    for (int i = 0; i < 3; i++)
      if (mask & (1 << i)) idx[k++] = i;
    double A[3][3], b[3], x[3];
    for (int i = 0; i < k; i++) {
      for (int j = 0; j < k; j++) A[i][j] = G[3 * idx[i] + idx[j]];
      b[i] = h[idx[i]];
    }
    if (!solve_small(k, A, b, x)) continue;
    int neg = 0;
    for (int i = 0; i < k; i++)
      if (x[i] < 0) neg = 1;
    if (neg) continue;
    double rss = dd;
    for (int i = 0; i < k; i++) rss -= x[i] * b[i];
    if (rss < best_rss) {
      a[0] = a[1] = a[2] = 0;
      for (int i = 0; i < k; i++) a[idx[i]] = x[i];
      best_rss = fmax(rss, 0);
    }
  }
  return best_rss;
}

/* ---------------------------------------------------------- Nelder-Mead */

typedef double (*objective)(const double *u, void *ctx);

/* Bounded Nelder-Mead (:302-350); bounds are clamps inside f. n <= 4. */
static double nelder_mead(objective f, void *ctx, int n, const double *x0,
                          const double *step, int maxIter, double tol,
                          double *xout) {
  double S[5][4], fs[5];
  for (int j = 0; j < n; j++) S[0][j] = x0[j];
  for (int i = 0; i < n; i++) {
    for (int j = 0; j < n; j++) S[i + 1][j] = x0[j];
    S[i + 1][i] += step[i];
  }
  for (int i = 0; i <= n; i++) fs[i] = f(S[i], ctx);
  for (int it = 0; it < maxIter; it++) {
    /* stable ascending sort of the vertices by f (V8's sort is stable) */
    for (int i = 1; i <= n; i++) {
      double fv = fs[i], xv[4];
      memcpy(xv, S[i], sizeof(double) * n);
      int j = i - 1;
      while (j >= 0 && fs[j] - fv > 0) {
        fs[j + 1] = fs[j];
        memcpy(S[j + 1], S[j], sizeof(double) * n);
        j--;
      }
      fs[j + 1] = fv;
      memcpy(S[j + 1], xv, sizeof(double) * n);
    }
    if (fabs(fs[n] - fs[0]) <= tol * (fabs(fs[0]) + 1e-30)) break;
    double c[4] = {0, 0, 0, 0};
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) c[j] += S[i][j] / n;
    double xr[4], xe[4], xc[4];
    for (int j = 0; j < n; j++) xr[j] = c[j] + -1.0 * (S[n][j] - c[j]);
    const double fr = f(xr, ctx);
    if (fr < fs[0]) {
      for (int j = 0; j < n; j++) xe[j] = c[j] + -2.0 * (S[n][j] - c[j]);
      const double fe = f(xe, ctx);
      if (fe < fr) {
        memcpy(S[n], xe, sizeof(double) * n);
        fs[n] = fe;
      } else {
        memcpy(S[n], xr, sizeof(double) * n);
        fs[n] = fr;
      }
    } else if (fr < fs[n - 1]) {
      memcpy(S[n], xr, sizeof(double) * n);
      fs[n] = fr;
    } else {
      const int outside = fr < fs[n];
      const double t = outside ? -0.5 : 0.5;
      for (int j = 0; j < n; j++) xc[j] = c[j] + t * (S[n][j] - c[j]);
      const double fc = f(xc, ctx);
      if (fc < (outside ? fr : fs[n])) {
        memcpy(S[n], xc, sizeof(double) * n);
        fs[n] = fc;
      } else {
        for (int i = 1; i <= n; i++) {
          for (int j = 0; j < n; j++) S[i][j] = S[0][j] + 0.5 * (S[i][j] - S[0][j]);
          fs[i] = f(S[i], ctx);
        }
      }
    }
  }
  int ib = 0;
  for (int i = 1; i <= n; i++)
    if (fs[i] < fs[ib]) ib = i;
  memcpy(xout, S[ib], sizeof(double) * n);
  return fs[ib];
}

/* ---------------------------------------------------------- data preparation */

int mf_lag_grid(int L, int *lags) { /* :358-369 */
  int n = 0;
  for (int t = 1; t <= (L - 1 < 10 ? L - 1 : 10); t++) lags[n++] = t;
  double x = 10;
  for (;;) {
    x *= 1.08;
    const int t = (int)js_round(x);
    if (t > L - 1) break;
    if (n == 0 || t > lags[n - 1]) lags[n++] = t;
  }
  return n;
}

#define MAXQN 16
typedef struct {
  int b;
  double q, w;
  int nq;
  double qn[MAXQN];
  double *d;
} pbin;

typedef struct {
  int nbins, nt, L;
  pbin *bins;
  int *lags;
  double *tau;
  double dt, tauMax;
  double swimMin;
} prepared;

static void prepare(const mf_radial *r, const mf_options *opt, prepared *pr) {
  /* :383-401 */
  const int L = r->L, NB = r->NB;
  pr->dt = 1 / opt->fps;
  pr->lags = (int *)malloc(sizeof(int) * (L + 16));
  pr->nt = mf_lag_grid(L, pr->lags);
  pr->tau = (double *)malloc(sizeof(double) * (pr->nt + 1));
  for (int j = 0; j < pr->nt; j++) pr->tau[j] = pr->lags[j] * pr->dt;
  pr->bins = (pbin *)calloc(NB > 0 ? NB : 1, sizeof(pbin));
  pr->nbins = 0;
  pr->L = L;
  pr->tauMax = (L - 1) * pr->dt;
  pr->swimMin = opt->swimMin;
  const int K = r->knodes;
  for (int b = 0; b < NB; b++) {
    if (r->nModes[b] < 3) continue;
    double scale = -INFINITY;
    int nan = 0;
    for (int j = 0; j < pr->nt; j++) {
      const double v = r->D[b * L + pr->lags[j]];
      if (isnan(v)) nan = 1;
      scale = fmax(scale, v);
    }
    if (nan) scale = NAN;
    if (!(scale > 0) || !isfinite(scale)) continue;
    pbin *pb = &pr->bins[pr->nbins++];
    const double qs = (2 * M_PI) / (r->N * opt->dxUm);
    pb->b = b;
    pb->q = qs * r->kCenter[b];
    if (K > 0) {
      pb->nq = K;
      for (int n = 0; n < K; n++) pb->qn[n] = r->kNodes[b * K + n] * qs;
    } else {
      pb->nq = 1;
      pb->qn[0] = pb->q;
    }
    pb->d = (double *)malloc(sizeof(double) * pr->nt);
    for (int j = 0; j < pr->nt; j++) pb->d[j] = r->D[b * L + pr->lags[j]];
    pb->w = 1 / scale;
  }
}

static void free_prepared(prepared *pr) {
  for (int i = 0; i < pr->nbins; i++) free(pr->bins[i].d);
  free(pr->bins);
  free(pr->lags);
  free(pr->tau);
}

/* ---------------------------------------------------------- models */

typedef struct {
  double vbar, Z, Dd, Vmag, alpha;
} params;

/* c_b(tau) = 1 - <E (1 - alpha + alpha g)>_nodes (:417-432) */
static void model_column(const prepared *pr, const pbin *bin, const params *p,
                         kernel_fn kernel, int swim, double *out) {
  const double inv = 1.0 / bin->nq;
  const double alpha = swim ? p->alpha : 0;
  for (int j = 0; j < pr->nt; j++) {
    const double t = pr->tau[j];
    double f = 0;
    for (int n = 0; n < bin->nq; n++) {
      const double q = bin->qn[n];
      double E = exp(-p->Dd * q * q * t);
      if (p->Vmag > 0) E *= mf_bessel_j0(q * p->Vmag * t);
      f += alpha > 0 ? E * (1 - alpha + alpha * kernel(q * p->vbar * t, p->Z)) : E;
    }
    out[j] = 1 - f * inv;
  }
}

/* VarPro: exact NNLS amplitudes A_b, B_b >= 0 per bin (:450-474).
 * amps[2*i] = A, amps[2*i+1] = B. */
static double eval_model(const prepared *pr, const params *p, kernel_fn kernel,
                         int swim, double *amps) {
  const int nt = pr->nt;
  double c[512];
  double rss = 0;
  for (int i = 0; i < pr->nbins; i++) {
    const pbin *bin = &pr->bins[i];
    model_column(pr, bin, p, kernel, swim, c);
    double g11 = 0, g12 = 0, h1 = 0, h2 = 0, dd = 0;
    for (int j = 0; j < nt; j++) {
      g11 += c[j] * c[j];
      g12 += c[j];
      h1 += c[j] * bin->d[j];
      h2 += bin->d[j];
      dd += bin->d[j] * bin->d[j];
    }
    const double G[9] = {g11, g12, 0, g12, (double)nt, 0, 0, 0, 0};
    const double h[3] = {h1, h2, 0};
    double a[3];
    const double r = mf_nnls3(G, h, dd, a);
    rss += r * bin->w * bin->w;
    if (amps) {
      amps[2 * i] = a[0];
      amps[2 * i + 1] = a[1];
    }
  }
  return rss;
}

typedef struct {
  double vmin, vmax, Dmin, Dmax, Zmin, Zmax;
} bounds_t;

static bounds_t bounds(const prepared *pr) { /* :480-491 */
  double qmin = INFINITY, qmax = -INFINITY;
  for (int i = 0; i < pr->nbins; i++) {
    qmin = fmin(qmin, pr->bins[i].q);
    qmax = fmax(qmax, pr->bins[i].q);
  }
  bounds_t B;
  B.vmin = fmax(pr->swimMin, 0.3 / (qmax * pr->tauMax));
  B.vmax = 3 / (qmin * pr->dt);
  B.Dmin = 0.01 / (qmax * qmax * pr->tauMax);
  B.Dmax = 10 / (qmin * qmin * pr->dt);
  B.Zmin = 0.5;
  B.Zmax = 100;
  return B;
}

typedef struct {
  const prepared *pr;
  bounds_t B;
  double Vmag, vlo, vhi;
  kernel_fn kernel;
} fit_ctx;

static double f_brownian(double lnD, fit_ctx *cx) {
  params p = {0, 1, exp(lnD), cx->Vmag, 0};
  return eval_model(cx->pr, &p, mf_isf3d, 0, NULL);
}

/* Brownian-only: 49-point ln D scan + golden section (:500-536). */
static mf_fit fit_brownian(const prepared *pr, double Vmag) {
  fit_ctx cx = {pr, bounds(pr), Vmag, 0, 0, NULL};
  const double lo = log(cx.B.Dmin), hi = log(cx.B.Dmax);
  const int n = 48;
  int bi = 0;
  double bf = INFINITY, xs[49];
  for (int i = 0; i <= n; i++) {
    const double x = lo + ((hi - lo) * i) / n;
    xs[i] = x;
    const double v = f_brownian(x, &cx);
    if (v < bf) {
      bf = v;
      bi = i;
    }
  }
  double a = xs[bi - 1 > 0 ? bi - 1 : 0], b = xs[bi + 1 < n ? bi + 1 : n];
  const double gr = (sqrt(5) - 1) / 2;
  double c = b - gr * (b - a), d = a + gr * (b - a);
  double fc = f_brownian(c, &cx), fd = f_brownian(d, &cx);
  for (int it = 0; it < 60 && b - a > 1e-6; it++) {
    if (fc < fd) {
      b = d;
      d = c;
      fd = fc;
      c = b - gr * (b - a);
      fc = f_brownian(c, &cx);
    } else {
      a = c;
      c = d;
      fc = fd;
      d = a + gr * (b - a);
      fd = f_brownian(d, &cx);
    }
  }
  const double lnD = fc < fd ? c : d;
  mf_fit out;
  out.Dd = exp(lnD);
  out.vbar = 0;
  out.Z = 1;
  out.Vmag = Vmag;
  out.alpha = 0;
  params p = {0, 1, out.Dd, Vmag, 0};
  out.rss = eval_model(pr, &p, mf_isf3d, 0, NULL);
  return out;
}

static params unpack_bd(const double *u, const fit_ctx *cx) { /* :547-553 */
  params p;
  p.vbar = 0;
  p.Z = 1;
  p.Dd = exp(clampd(u[0], log(cx->B.Dmin), log(cx->B.Dmax)));
  p.Vmag = clampd(u[1], cx->vlo, cx->vhi);
  p.alpha = 0;
  return p;
}
static double f_bd(const double *u, void *ctx) {
  fit_ctx *cx = (fit_ctx *)ctx;
  params p = unpack_bd(u, cx);
  return eval_model(cx->pr, &p, mf_isf3d, 0, NULL);
}

/* Passive null with uniform drift in [vlo, vhi] (:545-568). */
static mf_fit fit_brownian_drift(const prepared *pr, double vlo, double vhi) {
  fit_ctx cx = {pr, bounds(pr), 0, vlo, vhi, NULL};
  const double lDmin = log(cx.B.Dmin), lDmax = log(cx.B.Dmax);
  double bu[2] = {0, 0}, bfv = 0;
  int have = 0;
  for (int i = 0; i <= 24; i++) {
    const double lD = lDmin + ((lDmax - lDmin) * i) / 24;
    for (int j = 0; j <= 6; j++) {
      const double u[2] = {lD, vlo + ((vhi - vlo) * j) / 6};
      const double v = f_bd(u, &cx);
      if (!have || v < bfv) {
        have = 1;
        bfv = v;
        bu[0] = u[0];
        bu[1] = u[1];
      }
    }
  }
  const double step[2] = {0.2, fmax((vhi - vlo) / 6, 1e-3)};
  double x[2];
  nelder_mead(f_bd, &cx, 2, bu, step, 200, 1e-10, x);
  params p = unpack_bd(x, &cx);
  mf_fit out = {p.vbar, p.Z, p.Dd, p.Vmag, p.alpha, 0};
  out.rss = eval_model(pr, &p, mf_isf3d, 0, NULL);
  return out;
}

static params unpack_sw(const double *u, const fit_ctx *cx) { /* :581-587 */
  params p;
  p.vbar = exp(clampd(u[0], log(cx->B.vmin), log(cx->B.vmax)));
  p.Z = exp(clampd(u[1], log(cx->B.Zmin), log(cx->B.Zmax)));
  p.Dd = exp(clampd(u[2], log(cx->B.Dmin), log(cx->B.Dmax)));
  p.Vmag = cx->Vmag;
  p.alpha = clampd(u[3], 0, 1);
  return p;
}
static double f_sw(const double *u, void *ctx) {
  fit_ctx *cx = (fit_ctx *)ctx;
  params p = unpack_sw(u, cx);
  return eval_model(cx->pr, &p, cx->kernel, 1, NULL);
}

typedef struct {
  double u[4], f;
} start_t;

/* Swimmer VarPro over (ln vbar, ln Z, ln D, alpha), 64 starts, best 3
 * refined by Nelder-Mead (:577-611). */
static mf_fit fit_swimmer(const prepared *pr, int geometry2d, double Vmag,
                          double Dstart) {
  fit_ctx cx = {pr, bounds(pr), Vmag, 0, 0, swimmer_kernel(geometry2d)};
  const bounds_t B = cx.B;
  const double D0 = Dstart > 0 ? clampd(Dstart, B.Dmin, B.Dmax) : sqrt(B.Dmin * B.Dmax);
  start_t starts[64];
  int ns = 0;
  const int nv = 16;
  const double lZs[2] = {log(1.5), log(8)};
  const double a0s[2] = {0.3, 0.8};
  for (int i = 0; i < nv; i++) {
    const double lv = log(B.vmin) + ((log(B.vmax) - log(B.vmin)) * (i + 0.5)) / nv;
    for (int zi = 0; zi < 2; zi++)
      for (int ai = 0; ai < 2; ai++) {
        start_t s;
        s.u[0] = lv;
        s.u[1] = lZs[zi];
        s.u[2] = log(D0);
        s.u[3] = a0s[ai];
        s.f = f_sw(s.u, &cx);
        starts[ns++] = s;
      }
  }
  /* stable sort by f (V8's Array.prototype.sort is stable) */
  for (int i = 1; i < ns; i++) {
    start_t v = starts[i];
    int j = i - 1;
    while (j >= 0 && starts[j].f - v.f > 0) {
      starts[j + 1] = starts[j];
      j--;
    }
    starts[j + 1] = v;
  }
  const double step[4] = {0.3, 0.7, 0.7, 0.2};
  double bx[4], bf = 0;
  int have = 0;
  for (int s = 0; s < 3 && s < ns; s++) {
    double x[4];
    const double fv = nelder_mead(f_sw, &cx, 4, starts[s].u, step, 400, 1e-10, x);
    if (!have || fv < bf) {
      have = 1;
      bf = fv;
      memcpy(bx, x, sizeof bx);
    }
  }
  params p = unpack_sw(bx, &cx);
  mf_fit out = {p.vbar, p.Z, p.Dd, p.Vmag, p.alpha, 0};
  out.rss = eval_model(pr, &p, cx.kernel, 1, NULL);
  return out;
}

static double bic(double rss, double n, double k, double nRaw) { /* :620-622 */
  return n * log(fmax(rss, 1e-300) / nRaw) + k * log(n);
}

/* Pooled lag-1 autocorrelation of the normalised residuals (:634-651). */
static double residual_autocorr(const prepared *pr, const params *p,
                                kernel_fn kernel, int swim) {
  double *amps = (double *)malloc(sizeof(double) * 2 * (pr->nbins + 1));
  eval_model(pr, p, kernel, swim, amps);
  double c[512];
  double num = 0, den = 0;
  for (int i = 0; i < pr->nbins; i++) {
    const pbin *bin = &pr->bins[i];
    const double A = amps[2 * i], Bv = amps[2 * i + 1];
    model_column(pr, bin, p, kernel, swim, c);
    double prev = 0;
    for (int j = 0; j < pr->nt; j++) {
      const double r = (bin->d[j] - (A * c[j] + Bv)) * bin->w;
      den += r * r;
      if (j > 0) num += prev * r;
      prev = r;
    }
  }
  free(amps);
  return den > 0 ? fmin(0.99, fmax(0, num / den)) : 0;
}

static double effective_n(double n, double rho) { /* :654-656 */
  return fmax(2, (n * (1 - rho)) / (1 + rho));
}

typedef struct {
  double Vx, Vy, mag, sigma, angleDeg;
  int significant, pairs;
  double samples;
} drift_t;

/* Weighted LSQ for a uniform drift from phase increments (:672-725). */
static drift_t estimate_drift(const mf_radial *r, const prepared *pr,
                              const mf_options *opt, int use_swimmer,
                              double svbar, double sZ) {
  const int L = r->L, N = r->N;
  kernel_fn kernel = swimmer_kernel(opt->geometry2d);
  double S[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double modesUsed = 0;
  int pairs = 0;
  for (int i = 0; i < pr->nbins; i++) {
    const pbin *bin = &pr->bins[i];
    const int b = bin->b;
    int usedHere = 0;
    for (int tau = 1; tau < L - 1; tau++) {
      if (use_swimmer) {
        const double g = kernel(bin->q * svbar * tau * pr->dt, sZ);
        if (!(fabs(g) < DRIFT_ISF_MAX)) continue;
      }
      const double *o = r->drift + (size_t)(b * L + tau) * 8;
      if (!(o[0] > 0)) continue;
      for (int c = 0; c < 8; c++) S[c] += o[c];
      usedHere = 1;
      pairs++;
    }
    if (usedHere) modesUsed += r->nModes[b];
  }
  const double Sw = S[0], Sxx = S[1], Sxy = S[2], Syy = S[3], Rx = S[4],
               Ry = S[5], Rpp = S[6], n = S[7];
  const double det = Sxx * Syy - Sxy * Sxy;
  drift_t out = {0, 0, 0, INFINITY, 0, 0, pairs, n};
  if (n < 10 || !(det > 1e-12 * Sxx * Syy) || !(Sw > 0)) return out;
  const double bx = (Syy * Rx - Sxy * Ry) / det;
  const double by = (Sxx * Ry - Sxy * Rx) / det;
  const double rss = fmax(Rpp - bx * Rx - by * Ry, 0);
  const double inflate = fmax(1, n / fmax(modesUsed, 1));
  const double s2 = (rss / (n - 2)) * inflate;
  const double cxx = (s2 * Syy) / det, cyy = (s2 * Sxx) / det,
               cxy = (-s2 * Sxy) / det;
  const double conv = -(N * opt->dxUm) / (2 * M_PI * pr->dt);
  const double Vx = conv * bx, Vy = conv * by;
  const double mag = hypot(Vx, Vy);
  double varAlong;
  if (mag > 0) {
    const double ux = Vx / mag, uy = Vy / mag;
    varAlong = conv * conv * (ux * ux * cxx + 2 * ux * uy * cxy + uy * uy * cyy);
  } else
    varAlong = (conv * conv * (cxx + cyy)) / 2;
  const double sigma = sqrt(fmax(varAlong, 0));
  out.Vx = Vx;
  out.Vy = Vy;
  out.mag = mag;
  out.sigma = sigma;
  out.angleDeg = (atan2(Vy, Vx) * 180) / M_PI;
  out.significant = mag > FLOW_SIGMA * sigma;
  return out;
}

static int cmp_desc(const void *a, const void *b) {
  const double x = *(const double *)a, y = *(const double *)b;
  return (x < y) - (x > y);
}

double mf_temporal_structure_index(const mf_radial *r) { /* :735-749 */
  const int NB = r->NB, L = r->L;
  double *v = (double *)malloc(sizeof(double) * (NB + 1));
  int nv = 0;
  for (int b = 0; b < NB; b++) {
    if (r->nModes[b] < 3) continue;
    double late = 0;
    int n = 0;
    for (int t = L >> 1; t < L; t++) {
      late += r->D[b * L + t];
      n++;
    }
    late /= n;
    if (!(late > 0)) continue;
    v[nv++] = (late - r->D[b * L + 1]) / late;
  }
  qsort(v, nv, sizeof(double), cmp_desc);
  const int top = nv < 4 ? nv : 4;
  double s = 0;
  for (int i = 0; i < top; i++) s += v[i];
  free(v);
  return top ? fmax(0, s / top) : 0;
}

/* tau_1/2(q) and the exponent mu (:771-804); amps are the best model's. */
static double scaling_exponent(const mf_radial *r, const prepared *pr,
                               const double *amps) {
  const int L = r->L;
  double *lq = (double *)malloc(sizeof(double) * (pr->nbins + 1));
  double *lt = (double *)malloc(sizeof(double) * (pr->nbins + 1));
  int cnt = 0;
  for (int i = 0; i < pr->nbins; i++) {
    const pbin *bin = &pr->bins[i];
    const double A = amps[2 * i], B = amps[2 * i + 1];
    if (!(A > 0.2 * (A + B))) continue;
    double prev = 1;
    int prevT = 0;
    for (int t = 1; t < L; t++) {
      const double f = 1 - (r->D[bin->b * L + t] - B) / A;
      if (f <= 0.5) {
        double tt;
        if (t == 1)
          tt = 1;
        else {
          const double lt0 = log((double)prevT), lt1 = log((double)t);
          tt = exp(lt0 + ((prev - 0.5) / (prev - f)) * (lt1 - lt0));
        }
        lq[cnt] = bin->q;
        lt[cnt] = tt * pr->dt;
        cnt++;
        break;
      }
      prev = f;
      prevT = t;
    }
  }
  double mu = NAN;
  if (cnt >= 3) {
    double mx = 0, my = 0;
    for (int i = 0; i < cnt; i++) mx += log(lq[i]);
    for (int i = 0; i < cnt; i++) my += log(lt[i]);
    mx /= cnt;
    my /= cnt;
    double sxy = 0, sxx = 0;
    for (int i = 0; i < cnt; i++) {
      const double x = log(lq[i]), y = log(lt[i]);
      sxy += (x - mx) * (y - my);
      sxx += (x - mx) * (x - mx);
    }
    if (sxx > 0) mu = -sxy / sxx;
  }
  free(lq);
  free(lt);
  return mu;
}

/* ---------------------------------------------------------- top level */

static void finish(mf_result *o, int insufficient, int exposureLocked) {
  /* :918-990 */
  const int g1 = o->TSI >= TSI_MIN;
  int verdict;
  if (insufficient) {
    verdict = MF_NO_DYNAMICS;
  } else {
    const int flow = o->driftMag > FLOW_SIGMA * o->driftSigma &&
                     o->driftMag > FLOW_MIN_UM_S;
    const int g3 = o->dBIC > DBIC_MIN;
    const int g4 = o->alpha > ALPHA_MIN && o->alphaResolved;
    if (!g1)
      verdict = MF_NO_DYNAMICS;
    else if (flow)
      verdict = MF_DIRECTED_TRANSPORT;
    else if (!g3 || !g4)
      verdict = MF_NOT_MOTILE;
    else
      verdict = MF_MOTILE;
  }
  o->physicsVerdict = verdict;
  o->verdict = exposureLocked ? verdict : MF_UNLOCKED_EXPOSURE;
}

void mf_analyze_motility(const mf_radial *r, const mf_options *opt,
                         mf_result *o) { /* :870-912 */
  memset(o, 0, sizeof(*o));
  o->mu = NAN;
  prepared pr;
  prepare(r, opt, &pr);
  o->TSI = mf_temporal_structure_index(r);
  o->nbins = pr.nbins;
  o->nlags = pr.nt;
  if (pr.nbins < 4) {
    o->insufficient = 1;
    finish(o, 1, opt->exposureLocked);
    free_prepared(&pr);
    return;
  }
  const int nData = pr.nbins * pr.nt;
  kernel_fn kernel = swimmer_kernel(opt->geometry2d);
  mf_fit brown = fit_brownian(&pr, 0);
  double kBrown = 1 + 2 * pr.nbins;
  mf_fit swim = fit_swimmer(&pr, opt->geometry2d, 0, brown.Dd);
  int hasSwim = swim.alpha > 0.01;
  drift_t drift = estimate_drift(r, &pr, opt, hasSwim, swim.vbar, swim.Z);
  int driftParams = 0;
  if (drift.significant && drift.mag > 0) {
    const double half = FLOW_SIGMA * drift.sigma + 0.25 * drift.mag;
    brown = fit_brownian_drift(&pr, fmax(0, drift.mag - half), drift.mag + half);
    kBrown = 2 + 2 * pr.nbins;
    swim = fit_swimmer(&pr, opt->geometry2d, brown.Vmag, brown.Dd);
    driftParams = 1;
    hasSwim = swim.alpha > 0.01;
    drift_t d2 = estimate_drift(r, &pr, opt, hasSwim, swim.vbar, swim.Z);
    if (d2.samples >= 10) drift = d2;
  }
  params ps = {swim.vbar, swim.Z, swim.Dd, swim.Vmag, swim.alpha};
  const double rho = residual_autocorr(&pr, &ps, kernel, 1);
  const double nEff = effective_n(nData, rho);
  const double kSwim = 4 + 2 * pr.nbins;
  const double bicS = bic(swim.rss, nEff, kSwim + driftParams, nData);
  const double bicB = bic(brown.rss, nEff, kBrown, nData);
  const double dBIC = bicB - bicS;
  int resolved = 0; /* motileShare :759-762 */
  for (int i = 0; i < pr.nbins; i++) {
    const double q = pr.bins[i].q;
    if (q * swim.vbar * pr.dt <= 0.5 && q * swim.vbar * pr.tauMax >= 3) resolved++;
  }
  double *amps = (double *)malloc(sizeof(double) * 2 * (pr.nbins + 1));
  if (dBIC > 0)
    eval_model(&pr, &ps, kernel, 1, amps);
  else {
    params pb = {0, 1, brown.Dd, brown.Vmag, 0};
    eval_model(&pr, &pb, mf_isf3d, 0, amps);
  }
  o->mu = scaling_exponent(r, &pr, amps);
  free(amps);
  o->alpha = swim.alpha;
  o->alphaResolved = resolved > 0;
  o->resolvedBins = resolved;
  o->vbar = swim.vbar;
  o->sigmaV = swim.vbar / sqrt(swim.Z + 1);
  o->Z = swim.Z;
  o->Ddiff = swim.Dd;
  o->DdiffBrownian = brown.Dd;
  o->dBIC = dBIC;
  o->driftVx = drift.Vx;
  o->driftVy = drift.Vy;
  o->driftMag = drift.mag;
  o->driftSigma = drift.sigma;
  o->driftAngleDeg = drift.angleDeg;
  o->driftSignificant = drift.significant;
  o->driftPairs = drift.pairs;
  o->driftSamples = drift.samples;
  o->nData = nData;
  o->nEff = nEff;
  o->rho = rho;
  o->swim = swim;
  o->brown = brown;
  finish(o, 0, opt->exposureLocked);
  free_prepared(&pr);
}

/* ---------------------------------------------------------- C ABI */

extern "C" int ddm_analyze_motility(const ddm_radial_view *r, const ddm_motility_options *opt,
                                    ddm_motility_result *out) {
  if (!r || !opt || !out || !r->kCenter || !r->nModes || !r->D || !r->P || !r->drift || r->NB < 1 || r->L < 3 ||
      r->N < 8 || (r->knodes > 0 && !r->kNodes) || !(opt->dxUm > 0) || !(opt->fps > 0))
    return DDM_ERR_ARG;
  mf_analyze_motility(r, opt, out);
  return DDM_OK;
}
