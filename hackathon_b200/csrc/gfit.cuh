// Global VarPro fits of the motility model on the device (gfit.cu): types
// shared with the host analysis (analysis.cpp).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "isf.cuh"

namespace ddm {

// physical parameters of a fit: phi = (ln vbar, ln Z, ln D, alpha, |V|)
enum { GP_LV = 0, GP_LZ = 1, GP_LD = 2, GP_AL = 3, GP_V = 4, GP_N = 5 };
// models: which parameters move (the others stay at the job's values)
enum { GF_BROWN = 0,   // ln D                       (fitBrownian, motility_fit.js:500-536)
       GF_DRIFT = 1,   // ln D, |V|                  (fitBrownianDrift, :545-568)
       GF_SWIM = 2 };  // ln vbar, ln Z, ln D, alpha (fitSwimmer, :577-611)
// job kinds
enum { GJ_EVAL = 0,    // the VarPro cost at phi
       GJ_LM = 1,      // bounded Levenberg-Marquardt from phi
       GJ_FINAL = 2,   // at phi: per-bin amplitudes, residual lag-1 sums, drift-lag mask
       GJ_NM = 3,      // the reference's Nelder-Mead from phi (nelderMead, motility_fit.js:302-350)
       GJ_GOLDEN = 4 }; // golden section of ln D on [lo, hi] (fitBrownian's, :514-533)

constexpr int GF_MAX_LAGS = 128;  // 4 per lane
constexpr int GF_MAX_NODES = 8;

// One prepared Radial record (prepare, motility_fit.js:383-401) in device memory.
struct GfitProblem {
  int nb, nt, K;          // usable bins, lags of the fit grid, q-nodes per bin
  int geometry2d;         // swimmer kernel: 0 = 3D closed form, 1 = 2D table
  const double* tau;      // [nt] lag times (s)
  const double* d;        // [nb][nt] D_b(tau_j)
  const double* w;        // [nb] 1 / max_j D_b(tau_j)
  const double* qn;       // [nb][K] effective-|q| nodes
  const double* qc;       // [nb] bin-centre q (drift-lag mask)
  double dt;              // frame interval (s)
  int Lr;                 // lags of the Radial record (drift-lag mask covers 1..Lr-2)
  double* amps;           // [nb][2] out (GJ_FINAL): A_b, B_b
  uint8_t* dmask;         // [nb][Lr] out (GJ_FINAL, swimmer): |g(q_b vbar tau dt; Z)| < 0.2
};

struct GfitJob {
  int prob, model, kind;
  int max_iter;           // GJ_NM: iteration cap (0: the launch's)
  double phi[GP_N];       // start (LM, NM) or evaluation point
  double lo[GP_N], hi[GP_N];  // box of the moving parameters (NM: clamps inside the objective)
  double step[4];         // GJ_NM: initial simplex steps along the moving parameters
  double tol;             // GJ_NM: relative spread of the simplex costs that ends it
};

struct GfitResult {
  double phi[GP_N];
  double cost;            // weighted RSS (evalModel's rss)
  double num, den;        // GJ_FINAL: lag-1 residual products and squares
  int iters, status;      // iterations (LM, NM, golden) / evaluations (NM); bit 0: converged (not the cap)
  int evals, pad;
};

struct GfitLaunch {
  const GfitProblem* probs;
  const GfitJob* jobs;
  GfitResult* res;
  int njobs, max_iter;
  double tol;             // relative cost decrease that counts as no progress
  Isf2dTable tab;
  int max_bins;           // the most bins of any problem of the launch (sizes the clusters)
};

// One thread-block cluster per job (bins split across the cluster, sums
// combined through distributed shared memory); every job of a launch has the
// same model.
cudaError_t launch_gfit_model(int model, const GfitLaunch& a, cudaStream_t s);

}  // namespace ddm
