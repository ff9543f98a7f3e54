/*
 * FP64 CPU oracle for the motility-ddm analysis path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker: the tests, the smoke
 * check and the CPU-baseline leg of bench.py call it to produce the FP64
 * reference answers that the CUDA path is compared against. Nothing in the
 * product (hackathon_b200/) links or calls it.
 *
 * It restates, in C, the reference's own CPU implementation of the path:
 *   motility-ddm/src/fft.js          (FFT, DFT, window, half-plane 2D spectrum)
 *   motility-ddm/src/ddm_ref.js      (bins, history ring, masked Wiener-Khinchin,
 *                                     radial reduction, temporal metadata)
 *   motility-ddm/src/motility_fit.js (ISF kernels, NNLS, Nelder-Mead, VarPro
 *                                     fits, drift, gates, verdict)
 *   motility-ddm/test/sim.mjs        (seeded synthetic movies)
 * Each function cites the file:line it follows. Operation order is kept where
 * it decides FP64 rounding (Stockham pass order, RNG streams, quantisation),
 * so the oracle reproduces the reference's FP64 numbers, not just its maths.
 *
 * The reference is JavaScript and no JS runtime exists where this is built, so
 * the oracle is pinned against the reference's own known-answer tests
 * (test/t_fft.mjs, test/t_kernels.mjs, test/t_drift_phase.mjs) and the
 * published validation-matrix outputs (README.md section 6); see tests/.
 *
 * Extensions beyond the reference (marked "extension" where they appear):
 * arbitrary power-of-two N, T, TPAD, L; temporal metadata for any T/TPAD/L.
 */
#ifndef DDM_ORACLE_H
#define DDM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------ fft.js */
void or_fft(double *data, int n, int inverse);                  /* fft.js:59-93   */
void or_dft(const double *in, double *out, int n, int inverse); /* fft.js:101-119 */
void or_blackman_harris(double *w, int n);                      /* fft.js:126-133 */
void or_spectrum2d_half(const double *img, int N, const double *win,
                        double *out);                           /* fft.js:149-183 */
/* Extension: spatial pixel mask (mean over smask != 0, masked pixels zero). */
void or_spectrum2d_half_masked(const double *img, int N, const double *win,
                               const uint8_t *smask, double *out);

/* ------------------------------------------------------------ ddm_ref.js */
int or_window_leakage(int N, double step, double *d, double *p); /* ddm_ref.js:40-55 */
void or_mode_k(int m, int N, int *kx, int *ky);                  /* ddm_ref.js:63-69 */
/* Number of binned modes for a geometry (first half of makeBins). */
int or_make_bins_count(int N, int NB, double kmin, double kmax);
/* ddm_ref.js:84-170. binModes holds 4 int32 per entry: mode, kx, ky, 0. */
void or_make_bins(int N, int NB, double kmin, double kmax, int knodes,
                  uint32_t *binOffsets, int32_t *binModes, double *kCenter,
                  uint32_t *nModes, double *kNodes);

/* History ring hist[(mode*T + slot)*2 + {re,im}] (ddm_ref.js:178-206).
 * Transforms `nframes` luma frames into the given slots (OpenMP over frames).
 * spec_out, if not NULL, receives the last frame's spectrum. */
void or_history_ingest(double *hist, int N, int T, const double *luma,
                       const int *slots, int nframes);
/* Same with the spatial-mask extension (smask N*N bytes, NULL = none). */
void or_history_ingest_masked(double *hist, int N, int T, const double *luma,
                              const uint8_t *smask, const int *slots, int nframes);

/* ddm_ref.js:229-288, with n = TPAD (the reference uses 2T). */
double or_temporal_mode(const double *hist, int mode, int T, int TPAD,
                        const uint32_t *order, const double *mask, int L,
                        double *outD, double *outC);
/* ddm_ref.js:306-333 */
double or_temporal_mode_direct(const double *hist, int mode, int T,
                               const uint32_t *order, const double *mask,
                               int L, double *outD, double *outC);

/* ddm_ref.js:425-437 (binned modes only, reduced straight to radial sums).
 * D[NB*L], P[NB], drift[NB*L*8]; OpenMP over bins. */
void or_analyze_radial(const double *hist, int N, int T, int TPAD,
                       const uint32_t *order, const double *mask, int NB,
                       const uint32_t *binOffsets, const int32_t *binModes,
                       const uint32_t *nModes, int L, double *D, double *P,
                       double *drift, int threads);
/* ddm_ref.js:450-463 for an explicit mode list: D[n*L], C[n*2L], P[n]. */
void or_analyze_modes(const double *hist, int T, int TPAD,
                      const uint32_t *order, const double *mask, int L,
                      const int32_t *modes, int nmodes, double *D, double *C,
                      double *P, int threads);
/* ddm_ref.js:474-487. fullD[modes*L], fullC[modes*2L], fullP[modes]
 * (float arrays accepted as double). */
void or_radial_from_full(const double *fullD, const double *fullC,
                         const double *fullP, int NB,
                         const uint32_t *binOffsets, const int32_t *binModes,
                         const uint32_t *nModes, int L, double *D, double *P,
                         double *drift);
/* ddm_ref.js:538-560, generalised to T/TPAD/L (extension). npairs[L],
 * mspec[2*TPAD] (FP64, before the reference's f32 rounding). */
void or_temporal_meta(const uint32_t *order, const double *mask, int T,
                      int TPAD, int L, double *npairs, double *mspec);

/* ------------------------------------------------------------ motility_fit.js */
double or_bessel_j0(double x);               /* :54-68   */
double or_ln_gamma(double x);                /* :74-86   */
double or_schulz_pdf(double v, double vbar, double Z); /* :95-99 */
double or_legendre_p(double nu, double c);   /* :120-132 */
double or_isf3d(double x, double Z);         /* :140-144 */
double or_isf2d(double x, double Z);         /* :152-159 */
double or_isf2d_fast(double x, double Z);    /* :168-220 */
/* :243-263. a[3] out; returns rss. */
double or_nnls3(const double *G, const double *h, double dd, double *a);
int or_lag_grid(int L, int *lags);           /* :358-369, returns count */

typedef struct {
  int N, NB, L, knodes;
  const double *kCenter; /* NB */
  const double *kNodes;  /* NB*knodes */
  const uint32_t *nModes;
  const double *D;     /* NB*L */
  const double *P;     /* NB */
  const double *drift; /* NB*L*8 */
} or_radial;

typedef struct {
  double dxUm, fps;
  int geometry2d;     /* 0 = '3d', 1 = '2d' */
  int exposureLocked; /* 1 = locked */
  double swimMin;     /* GATES.SWIM_MIN_UM_S (2 in the reference) */
} or_options;

typedef struct {
  double vbar, Z, Dd, Vmag, alpha, rss;
} or_fit;

enum {
  OR_MOTILE = 0,
  OR_NOT_MOTILE = 1,
  OR_DIRECTED_TRANSPORT = 2,
  OR_NO_DYNAMICS = 3,
  OR_UNLOCKED_EXPOSURE = 4
};

typedef struct {
  int verdict, physicsVerdict, insufficient;
  double TSI, alpha;
  int alphaResolved, resolvedBins;
  double vbar, sigmaV, Z, Ddiff, DdiffBrownian, dBIC;
  double driftVx, driftVy, driftMag, driftSigma, driftAngleDeg;
  int driftSignificant, driftPairs;
  double driftSamples;
  double mu;
  int nData;
  double nEff, rho;
  int nbins, nlags;
  or_fit swim, brown;
} or_result;

/* :870-912 + finish :918-990 */
void or_analyze_motility(const or_radial *r, const or_options *opt,
                         or_result *out);
/* Pieces used by the known-answer tests (t_kernels.mjs, t_drift_phase.mjs). */
void or_fit_brownian_swimmer(const or_radial *r, const or_options *opt,
                             or_fit *brown, or_fit *swim);
void or_estimate_drift(const or_radial *r, const or_options *opt,
                       int use_swimmer, double vbar, double Z, double *out8);
double or_temporal_structure_index(const or_radial *r); /* :735-749 */
/* Model column of one bin (:417-432) on the reference's lag grid. */
int or_model_column(const or_radial *r, const or_options *opt, int bin,
                    double vbar, double Z, double Dd, double Vmag,
                    double alpha, int swim, double *out);
/* VarPro objective (:450-474) at given parameters; amps[2*nbins] (A, B). */
double or_eval_model(const or_radial *r, const or_options *opt, double vbar,
                     double Z, double Dd, double Vmag, double alpha, int swim,
                     double *amps);

/* ------------------------------------------------------------ per-bin LM (new) */
/* FP64 Levenberg-Marquardt on one bin (see lm.c). bounds6 = (vmin, vmax,
 * Zmin, Zmax, Dmin, Dmax); theta = (A, B, alpha, ln vbar, ln Z, ln D) in/out.
 * Returns the iteration count. */
int or_lm_fit(int nt, int K, const double *d, const double *tau, const double *qn, double w,
              const double *bounds6, double *theta, int max_iter, double tol, double *cost_out);
void or_lm_model(int nt, int K, const double *tau, const double *qn, const double *theta,
                 double *y);
/* LM from start4 = (alpha, vbar, Z, D) with VarPro amplitudes. */
int or_lm_fit_start(int nt, int K, const double *d, const double *tau, const double *qn, double w,
                    const double *bounds6, const double *start4, int max_iter, double tol,
                    double *theta, double *cost_out);
/* LM from the reference's start strategy (Brownian scan, 64 starts, best
 * nrefine refined). */
/* Brownian model per bin (fitBrownian's search, alpha = 0) -> cost. */
double or_lm_fit_brownian(int nt, int K, const double *d, const double *tau, const double *qn, double w,
                          const double *bounds6, double *theta);
int or_lm_fit_plain(int nt, int K, const double *d, const double *tau, const double *qn, double w,
                    const double *bounds6, int max_iter, double tol, int nrefine, double *theta,
                    double *cost_out, int *evals);

/* ------------------------------------------------------------ sim.mjs */
typedef struct {
  int N, T;
  double fps, dxUm;
  uint32_t seed;
  int nSwim;
  double swimVbar, swimSigma;
  int swim2d;
  int nPassive;
  double Dum2s;
  int nFixed;
  int hasDrift;
  double driftSpeed, driftAngleDeg;
  double dropFrac;
  int dropExact;
  double blobSigmaPx, amp, background, noise;
} or_sim_params;

/* sim.mjs:90-186. frames[T*N*N] u8, valid[T] (1/0). truth[4]: meanSpeed,
 * Vx, Vy, D. */
void or_simulate(const or_sim_params *p, uint8_t *frames, uint8_t *valid,
                 double *truth);
/* sim.mjs:14-23: fills out[n] with successive mulberry32 draws. */
void or_mulberry32(uint32_t seed, double *out, int n);
/* sim.mjs:26-63: normals and gammas from makeRng(seed). */
void or_rng_normals(uint32_t seed, double *out, int n);
void or_rng_gammas(uint32_t seed, double k, double theta, double *out, int n);
/* ddm_ref.js:510-519 with rand = mulberry32(seed). */
void or_shuffle_order(uint32_t *order, double *mask, int T, uint32_t seed);

#ifdef __cplusplus
}
#endif
#endif
