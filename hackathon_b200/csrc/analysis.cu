// analyzeMotility (motility-ddm/src/motility_fit.js:870-990) over Radial
// records, with every model fit on the GPU (gfit.cu).
//
// The analysis of a record is a fixed sequence of stages. Records are
// analysed together: each stage collects the device jobs of every record
// still in play and runs them as ONE launch per model (scan points and start
// sets are independent jobs), so a batch of records costs about as many
// launches as one record. What stays on the host is O(bins x lags) or less:
// preparing the record (prepare, lagGrid), the temporal structure index, the
// phase-drift least squares, BIC with the AR(1) effective sample size, the
// identifiability count of alpha, the q-scaling exponent and the gates.
//
// Stages (pass 2 only for records whose drift is significant):
//   Brownian null   49-point ln D scan, then golden section inside the
//                   bracket of the best scan point (fitBrownian :500-536)
//   swimmer         64 starts, Nelder-Mead from the 3 best by cost, lowest
//                   cost kept                 (fitSwimmer       :577-611)
//   final swimmer   amplitudes, lag-1 residual sums, drift-lag mask
//   drift           phase-drift LSQ on the host (estimateDrift :672-725)
//   [pass 2]        Brownian + drift: 25 x 7 grid in (ln D, |V|) over the
//                   phase band, then Nelder-Mead (fitBrownianDrift :545-568);
//                   swimmer again at that |V|; drift again
//   final Brownian  amplitudes of the null model (q-scaling when it wins)
// The searches are the reference's own (same starts, steps, tolerances and
// iteration caps), so the fits follow its path. Option optimizer = 1 replaces
// golden section and Nelder-Mead by a bounded Levenberg-Marquardt iteration
// from the same starts (gfit.cu): several times faster, and on flat,
// non-identifiable surfaces (a swimmer fit of a sample with no swimmers) it
// can end at a lower cost than the reference's search, at other parameters.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/ddm_b200.h"
#include "gfit.cuh"

extern std::string& ddm_detached_error();  // message slot of calls without an engine (engine.cu)

namespace ddm {
namespace {

// falsification gate thresholds (GATES, motility_fit.js:28-38); the swimmer
// speed floor comes from the options; the drift-lag threshold 0.2 is applied
// on the device (gfit.cu)
constexpr double TSI_MIN = 0.15, FLOW_SIGMA = 3.0, FLOW_MIN = 2.0, DBIC_MIN = 10.0, ALPHA_MIN = 0.05;
constexpr int MAX_ITER = 200;
constexpr double LM_TOL = 1e-12;
constexpr int SWIM_STARTS = 64, SWIM_REFINE = 3, BROWN_SCAN = 49, DRIFT_GD = 25, DRIFT_GV = 7;

// ------------------------------------------------------------------ preparation

// every lag 1..10, then steps of 8 % (rounded half up) up to L - 1 (:358-369)
std::vector<int> fit_lags(int L) {
  std::vector<int> out;
  for (int t = 1; t <= std::min(10, L - 1); t++) out.push_back(t);
  for (double x = 10.0;;) {
    x *= 1.08;
    const int t = (int)std::floor(x + 0.5);
    if (t > L - 1) break;
    if (out.empty() || t > out.back()) out.push_back(t);
  }
  return out;
}

struct Record {
  // inputs
  const ddm_radial_view* r = nullptr;
  ddm_motility_options opt{};
  ddm_motility_result* out = nullptr;
  // prepared data (prepare, :383-401): bins with >= 3 modes and a positive,
  // finite largest D over the fit lags
  std::vector<int> bin;           // Radial bin index
  std::vector<double> q, qn, d, w;
  std::vector<int> lags;
  std::vector<double> tau;
  int nb = 0, nt = 0, K = 1;
  double dt = 0, tau_max = 0;
  // box (bounds, :480-491)
  double lo[GP_N]{}, hi[GP_N]{};
  // device problem entries: [0] swimmer amplitudes + drift mask, [1] Brownian amplitudes
  int prob = -1;
  // fits
  double brown[GP_N]{}, swim[GP_N]{};
  double brown_rss = 0, swim_rss = 0;
  int drift_params = 0;
  bool pass2 = false;
  double num = 0, den = 0;
  std::vector<double> amps_swim, amps_brown;
  std::vector<uint8_t> dmask;
  ddm_motility_fit fs{}, fb{};
};

void prepare(Record& R) {
  const ddm_radial_view& r = *R.r;
  R.dt = 1.0 / R.opt.fps;
  R.lags = fit_lags(r.L);
  R.nt = (int)R.lags.size();
  R.tau.resize(R.nt);
  for (int j = 0; j < R.nt; j++) R.tau[j] = R.lags[j] * R.dt;
  R.tau_max = (r.L - 1) * R.dt;
  R.K = r.knodes > 0 && r.kNodes ? r.knodes : 1;
  const double qs = 2.0 * M_PI / (r.N * R.opt.dxUm);
  for (int b = 0; b < r.NB; b++) {
    if (r.nModes[b] < 3) continue;
    double mx = -INFINITY;
    for (int j = 0; j < R.nt; j++) {
      const double v = r.D[(size_t)b * r.L + R.lags[j]];
      mx = std::isnan(v) || std::isnan(mx) ? NAN : std::max(mx, v);  // a NaN poisons the maximum
    }
    if (!(mx > 0) || !std::isfinite(mx)) continue;
    R.bin.push_back(b);
    const double qb = qs * r.kCenter[b];
    R.q.push_back(qb);
    for (int n = 0; n < R.K; n++) R.qn.push_back(r.knodes > 0 && r.kNodes ? r.kNodes[(size_t)b * R.K + n] * qs : qb);
    for (int j = 0; j < R.nt; j++) R.d.push_back(r.D[(size_t)b * r.L + R.lags[j]]);
    R.w.push_back(1.0 / mx);
  }
  R.nb = (int)R.bin.size();
  if (R.nb == 0) return;
  const double qmin = *std::min_element(R.q.begin(), R.q.end());
  const double qmax = *std::max_element(R.q.begin(), R.q.end());
  const double vmin = std::max(R.opt.swimMin, 0.3 / (qmax * R.tau_max)), vmax = 3.0 / (qmin * R.dt);
  const double Dmin = 0.01 / (qmax * qmax * R.tau_max), Dmax = 10.0 / (qmin * qmin * R.dt);
  // clamp(x, lo, hi) = min(hi, max(lo, x)): an inverted range collapses on hi
  auto setbox = [&](int k, double a, double b) {
    R.lo[k] = std::min(a, b);
    R.hi[k] = b;
  };
  setbox(GP_LV, std::log(vmin), std::log(vmax));
  setbox(GP_LZ, std::log(0.5), std::log(100.0));
  setbox(GP_LD, std::log(Dmin), std::log(Dmax));
  setbox(GP_AL, 0.0, 1.0);
  setbox(GP_V, 0.0, 0.0);
}

// mean over the 4 largest bins of (D_late - D(1)) / D_late, D_late the mean
// over lags L/2..L-1, bins with >= 3 modes (:735-749)
double structure_index(const ddm_radial_view& r) {
  std::vector<double> s;
  for (int b = 0; b < r.NB; b++) {
    if (r.nModes[b] < 3) continue;
    const double* D = r.D + (size_t)b * r.L;
    double late = 0;
    int n = 0;
    for (int t = r.L / 2; t < r.L; t++, n++) late += D[t];
    late /= n;
    if (late > 0) s.push_back((late - D[1]) / late);
  }
  std::sort(s.begin(), s.end(), [](double a, double b) { return a > b; });
  const size_t k = std::min<size_t>(4, s.size());
  if (!k) return 0.0;
  double acc = 0;
  for (size_t i = 0; i < k; i++) acc += s[i];
  return std::max(0.0, acc / k);
}

// ------------------------------------------------------------------ drift

struct DriftFit {
  double Vx = 0, Vy = 0, mag = 0, sigma = INFINITY, angle = 0;
  bool significant = false;
  int pairs = 0;
  double samples = 0;
};

// Weighted LSQ of phi ~ kx bx + ky by over the (bin, lag) drift sums, using
// only lags where the swimmer ISF has decayed (mask != nullptr), then
// V = -(N dx / (2 pi dt)) b and its standard error along V, the covariance
// inflated by the mean number of lag pairs per mode (:672-725).
DriftFit drift_lsq(const Record& R, const uint8_t* mask) {
  const ddm_radial_view& r = *R.r;
  double S[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double modes = 0;
  DriftFit f;
  for (int i = 0; i < R.nb; i++) {
    const int b = R.bin[i];
    bool used = false;
    for (int t = 1; t < r.L - 1; t++) {
      if (mask && !mask[(size_t)i * r.L + t]) continue;
      const double* s = r.drift + ((size_t)b * r.L + t) * 8;
      if (!(s[0] > 0)) continue;
      for (int c = 0; c < 8; c++) S[c] += s[c];
      used = true;
      f.pairs++;
    }
    if (used) modes += r.nModes[b];
  }
  const double Sw = S[0], Sxx = S[1], Sxy = S[2], Syy = S[3], Rx = S[4], Ry = S[5], Rpp = S[6], n = S[7];
  f.samples = n;
  const double det = Sxx * Syy - Sxy * Sxy;
  if (n < 10 || !(det > 1e-12 * Sxx * Syy) || !(Sw > 0)) return f;  // no estimate
  const double bx = (Syy * Rx - Sxy * Ry) / det, by = (Sxx * Ry - Sxy * Rx) / det;
  const double rss = std::max(Rpp - bx * Rx - by * Ry, 0.0);
  const double s2 = rss / (n - 2) * std::max(1.0, n / std::max(modes, 1.0));
  const double cxx = s2 * Syy / det, cyy = s2 * Sxx / det, cxy = -s2 * Sxy / det;
  const double conv = -(r.N * R.opt.dxUm) / (2.0 * M_PI * R.dt);
  f.Vx = conv * bx;
  f.Vy = conv * by;
  f.mag = std::hypot(f.Vx, f.Vy);
  double var;
  if (f.mag > 0) {
    const double ux = f.Vx / f.mag, uy = f.Vy / f.mag;
    var = conv * conv * (ux * ux * cxx + 2 * ux * uy * cxy + uy * uy * cyy);
  } else {
    var = conv * conv * (cxx + cyy) / 2;
  }
  f.sigma = std::sqrt(std::max(var, 0.0));
  f.angle = std::atan2(f.Vy, f.Vx) * 180.0 / M_PI;
  f.significant = f.mag > FLOW_SIGMA * f.sigma;
  return f;
}

// ------------------------------------------------------------------ q-scaling

// tau_1/2 per bin from the data normalised by the fit's amplitudes
// (log-linear interpolation of the half crossing), then the slope of
// ln tau_1/2 against ln q: mu (:771-804)
double scaling_mu(const Record& R, const std::vector<double>& amps) {
  const ddm_radial_view& r = *R.r;
  std::vector<double> lq, lt;
  for (int i = 0; i < R.nb; i++) {
    const double A = amps[2 * i], B = amps[2 * i + 1];
    if (!(A > 0.2 * (A + B))) continue;
    const double* D = r.D + (size_t)R.bin[i] * r.L;
    double prev = 1, prev_t = 0;
    for (int t = 1; t < r.L; t++) {
      const double f = 1 - (D[t] - B) / A;
      if (f <= 0.5) {
        double th = 1;
        if (t > 1) {
          const double l0 = std::log(prev_t), l1 = std::log((double)t);
          th = std::exp(l0 + (prev - 0.5) / (prev - f) * (l1 - l0));
        }
        lq.push_back(std::log(R.q[i]));
        lt.push_back(std::log(th * R.dt));
        break;
      }
      prev = f;
      prev_t = t;
    }
  }
  if (lq.size() < 3) return NAN;
  const double mx = std::accumulate(lq.begin(), lq.end(), 0.0) / lq.size();
  const double my = std::accumulate(lt.begin(), lt.end(), 0.0) / lt.size();
  double sxy = 0, sxx = 0;
  for (size_t i = 0; i < lq.size(); i++) {
    sxy += (lq[i] - mx) * (lt[i] - my);
    sxx += (lq[i] - mx) * (lq[i] - mx);
  }
  return sxx > 0 ? -sxy / sxx : NAN;
}

// ------------------------------------------------------------------ device

struct Device {
  cudaStream_t s = nullptr;
  Isf2dTable tab{};
  GfitProblem* probs = nullptr;  // device table
  GfitJob* jobs = nullptr;
  GfitResult* res = nullptr;
  double* dbuf = nullptr;
  uint8_t* mbuf = nullptr;
  int max_jobs = 0;
  std::vector<GfitProblem> hprobs;
  int max_bins = 1;
  cudaError_t err = cudaSuccess;

  ~Device() {
    for (void* p : {(void*)probs, (void*)jobs, (void*)res, (void*)dbuf, (void*)mbuf})
      if (p) cudaFree(p);
    if (s) cudaStreamDestroy(s);
  }
  bool ok(cudaError_t e) {
    if (err == cudaSuccess && e != cudaSuccess) err = e;
    return err == cudaSuccess;
  }

  // device copies of every record's prepared data; two problem entries per
  // record (swimmer / Brownian amplitude outputs)
  bool upload(std::vector<Record*>& recs) {
    if (!ok(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking))) return false;
    if (!ok(isf2d_table(&tab))) return false;
    size_t nd = 0, nm = 0;
    for (Record* R : recs) {
      nd += R->nt + (size_t)R->nb * (R->nt + 1 + R->K + 1 + 4);
      nm += (size_t)R->nb * R->r->L;
    }
    if (!ok(cudaMalloc((void**)&dbuf, sizeof(double) * std::max<size_t>(nd, 1)))) return false;
    if (!ok(cudaMalloc((void**)&mbuf, std::max<size_t>(nm, 1)))) return false;
    std::vector<double> h(nd);
    size_t o = 0, om = 0;
    hprobs.clear();
    for (Record* R : recs) {
      GfitProblem P{};
      P.nb = R->nb;
      P.nt = R->nt;
      P.K = R->K;
      P.geometry2d = R->opt.geometry2d;
      P.dt = R->dt;
      P.Lr = R->r->L;
      auto put = [&](const std::vector<double>& v) {
        std::copy(v.begin(), v.end(), h.begin() + o);
        const double* p = dbuf + o;
        o += v.size();
        return p;
      };
      P.tau = put(R->tau);
      P.d = put(R->d);
      P.w = put(R->w);
      P.qn = put(R->qn);
      P.qc = put(R->q);
      P.amps = dbuf + o;
      o += 2 * (size_t)R->nb;
      P.dmask = mbuf + om;
      om += (size_t)R->nb * R->r->L;
      R->prob = (int)hprobs.size();
      max_bins = std::max(max_bins, R->nb);
      hprobs.push_back(P);
      P.amps = dbuf + o;  // the Brownian entry: its own amplitudes, no mask
      o += 2 * (size_t)R->nb;
      P.dmask = nullptr;
      hprobs.push_back(P);
    }
    if (!ok(cudaMemcpyAsync(dbuf, h.data(), sizeof(double) * nd, cudaMemcpyHostToDevice, s))) return false;
    if (!ok(cudaMalloc((void**)&probs, sizeof(GfitProblem) * hprobs.size()))) return false;
    if (!ok(cudaMemcpyAsync(probs, hprobs.data(), sizeof(GfitProblem) * hprobs.size(), cudaMemcpyHostToDevice, s)))
      return false;
    max_jobs = std::max<int>(1, (int)recs.size() * DRIFT_GD * DRIFT_GV);
    if (!ok(cudaMalloc((void**)&jobs, sizeof(GfitJob) * max_jobs))) return false;
    if (!ok(cudaMalloc((void**)&res, sizeof(GfitResult) * max_jobs))) return false;
    return ok(cudaStreamSynchronize(s));  // h goes out of scope
  }

  // one launch of same-model jobs; results back on the host
  bool run(int model, const std::vector<GfitJob>& J, std::vector<GfitResult>& out) {
    out.resize(J.size());
    if (J.empty()) return true;
    if ((int)J.size() > max_jobs) return ok(cudaErrorInvalidValue);
    if (!ok(cudaMemcpyAsync(jobs, J.data(), sizeof(GfitJob) * J.size(), cudaMemcpyHostToDevice, s))) return false;
    GfitLaunch a{};
    a.probs = probs;
    a.jobs = jobs;
    a.res = res;
    a.njobs = (int)J.size();
    a.max_iter = MAX_ITER;
    a.tol = LM_TOL;
    a.tab = tab;
    a.max_bins = max_bins;
    if (!ok(launch_gfit_model(model, a, s))) return false;
    if (!ok(cudaMemcpyAsync(out.data(), res, sizeof(GfitResult) * J.size(), cudaMemcpyDeviceToHost, s))) return false;
    return ok(cudaStreamSynchronize(s));
  }

  bool read_amps(const Record& R, int entry, std::vector<double>& amps) {
    amps.resize(2 * (size_t)R.nb);
    return ok(cudaMemcpy(amps.data(), hprobs[R.prob + entry].amps, sizeof(double) * amps.size(),
                         cudaMemcpyDeviceToHost));
  }
  bool read_mask(const Record& R, std::vector<uint8_t>& m) {
    m.resize((size_t)R.nb * R.r->L);
    return ok(cudaMemcpy(m.data(), hprobs[R.prob].dmask, m.size(), cudaMemcpyDeviceToHost));
  }
};

GfitJob make_job(const Record& R, int model, int kind, const double* phi, int entry = 0) {
  GfitJob j{};
  j.prob = R.prob + entry;
  j.model = model;
  j.kind = kind;
  for (int k = 0; k < GP_N; k++) {
    j.phi[k] = phi[k];
    j.lo[k] = R.lo[k];
    j.hi[k] = R.hi[k];
  }
  return j;
}

bool use_lm(const Record& R) { return R.opt.optimizer == 1; }

// the search from a start: the reference's Nelder-Mead (steps, cap, tolerance
// of its caller) or LM
void to_search(const Record& R, GfitJob& j, const double* step, int max_iter) {
  if (use_lm(R)) {
    j.kind = GJ_LM;
    return;
  }
  j.kind = GJ_NM;
  j.max_iter = max_iter;
  j.tol = 1e-10;
  for (int k = 0; k < 4; k++) j.step[k] = step[k];
}

double clampd(double x, double lo, double hi) { return std::min(hi, std::max(lo, x)); }

// Brownian null at fixed |V| for each record: scan, then LM inside the bracket
bool fit_brownian(Device& dev, std::vector<Record*>& recs, const std::vector<double>& V) {
  std::vector<GfitJob> J;
  for (size_t i = 0; i < recs.size(); i++) {
    const Record& R = *recs[i];
    for (int k = 0; k < BROWN_SCAN; k++) {
      double phi[GP_N] = {R.lo[GP_LV], 0.0, R.lo[GP_LD] + (R.hi[GP_LD] - R.lo[GP_LD]) * k / (BROWN_SCAN - 1), 0.0,
                          V[i]};
      J.push_back(make_job(R, GF_BROWN, GJ_EVAL, phi, 1));
    }
  }
  std::vector<GfitResult> out;
  if (!dev.run(GF_BROWN, J, out)) return false;
  std::vector<GfitJob> L;
  for (size_t i = 0; i < recs.size(); i++) {
    const Record& R = *recs[i];
    int bi = 0;
    for (int k = 1; k < BROWN_SCAN; k++)
      if (out[i * BROWN_SCAN + k].cost < out[i * BROWN_SCAN + bi].cost) bi = k;
    const double span = R.hi[GP_LD] - R.lo[GP_LD];
    GfitJob j = J[i * BROWN_SCAN + bi];
    j.kind = use_lm(R) ? GJ_LM : GJ_GOLDEN;
    j.lo[GP_LD] = R.lo[GP_LD] + span * std::max(0, bi - 1) / (BROWN_SCAN - 1);
    j.hi[GP_LD] = R.lo[GP_LD] + span * std::min(BROWN_SCAN - 1, bi + 1) / (BROWN_SCAN - 1);
    L.push_back(j);
  }
  if (!dev.run(GF_BROWN, L, out)) return false;
  for (size_t i = 0; i < recs.size(); i++) {
    Record& R = *recs[i];
    std::copy(out[i].phi, out[i].phi + GP_N, R.brown);
    R.brown_rss = out[i].cost;
  }
  return true;
}

// Brownian null with a drift speed refined inside [vlo, vhi]: grid, then LM
bool fit_brownian_drift(Device& dev, std::vector<Record*>& recs, const std::vector<double>& vlo,
                        const std::vector<double>& vhi) {
  std::vector<GfitJob> J;
  const int G = DRIFT_GD * DRIFT_GV;
  for (size_t i = 0; i < recs.size(); i++) {
    Record& R = *recs[i];
    R.lo[GP_V] = vlo[i];
    R.hi[GP_V] = vhi[i];
    for (int a = 0; a < DRIFT_GD; a++)
      for (int b = 0; b < DRIFT_GV; b++) {
        double phi[GP_N] = {R.lo[GP_LV], 0.0, R.lo[GP_LD] + (R.hi[GP_LD] - R.lo[GP_LD]) * a / (DRIFT_GD - 1), 0.0,
                            vlo[i] + (vhi[i] - vlo[i]) * b / (DRIFT_GV - 1)};
        J.push_back(make_job(R, GF_DRIFT, GJ_EVAL, phi, 1));
      }
  }
  std::vector<GfitResult> out;
  if (!dev.run(GF_DRIFT, J, out)) return false;
  std::vector<GfitJob> L;
  for (size_t i = 0; i < recs.size(); i++) {
    int bi = 0;
    for (int k = 1; k < G; k++)
      if (out[i * G + k].cost < out[i * G + bi].cost) bi = k;
    GfitJob j = J[i * G + bi];
    const double step[4] = {0.2, std::max((vhi[i] - vlo[i]) / 6, 1e-3), 0, 0};
    to_search(*recs[i], j, step, 200);
    L.push_back(j);
  }
  if (!dev.run(GF_DRIFT, L, out)) return false;
  for (size_t i = 0; i < recs.size(); i++) {
    Record& R = *recs[i];
    std::copy(out[i].phi, out[i].phi + GP_N, R.brown);
    R.brown_rss = out[i].cost;
  }
  return true;
}

// swimmer model at fixed |V| from the 64 starts around D0; LM from the best 3
bool fit_swimmer(Device& dev, std::vector<Record*>& recs, const std::vector<double>& V,
                 const std::vector<double>& D0) {
  std::vector<GfitJob> J;
  for (size_t i = 0; i < recs.size(); i++) {
    const Record& R = *recs[i];
    const double d0 = D0[i] > 0 ? clampd(D0[i], std::exp(R.lo[GP_LD]), std::exp(R.hi[GP_LD]))
                                : std::sqrt(std::exp(R.lo[GP_LD]) * std::exp(R.hi[GP_LD]));
    const double lzs[2] = {std::log(1.5), std::log(8.0)}, als[2] = {0.3, 0.8};
    for (int k = 0; k < SWIM_STARTS / 4; k++)
      for (int z = 0; z < 2; z++)
        for (int a = 0; a < 2; a++) {
          const double lv = R.lo[GP_LV] + (R.hi[GP_LV] - R.lo[GP_LV]) * (k + 0.5) / (SWIM_STARTS / 4);
          double phi[GP_N] = {lv, lzs[z], std::log(d0), als[a], V[i]};
          for (int p = 0; p < 4; p++) phi[p] = clampd(phi[p], R.lo[p], R.hi[p]);
          J.push_back(make_job(R, GF_SWIM, GJ_EVAL, phi, 0));
        }
  }
  std::vector<GfitResult> out;
  if (!dev.run(GF_SWIM, J, out)) return false;
  std::vector<GfitJob> L;
  for (size_t i = 0; i < recs.size(); i++) {
    std::vector<int> ord(SWIM_STARTS);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
      return out[i * SWIM_STARTS + a].cost < out[i * SWIM_STARTS + b].cost;
    });
    for (int r = 0; r < SWIM_REFINE; r++) {
      GfitJob j = J[i * SWIM_STARTS + ord[r]];
      const double step[4] = {0.3, 0.7, 0.7, 0.2};
      to_search(*recs[i], j, step, 400);
      L.push_back(j);
    }
  }
  if (!dev.run(GF_SWIM, L, out)) return false;
  for (size_t i = 0; i < recs.size(); i++) {
    Record& R = *recs[i];
    int best = 0;
    for (int r = 1; r < SWIM_REFINE; r++)
      if (out[i * SWIM_REFINE + r].cost < out[i * SWIM_REFINE + best].cost) best = r;
    std::copy(out[i * SWIM_REFINE + best].phi, out[i * SWIM_REFINE + best].phi + GP_N, R.swim);
    R.swim_rss = out[i * SWIM_REFINE + best].cost;
  }
  return true;
}

// final swimmer evaluation: amplitudes, lag-1 residual sums, drift-lag mask
bool final_swimmer(Device& dev, std::vector<Record*>& recs) {
  std::vector<GfitJob> J;
  for (Record* R : recs) J.push_back(make_job(*R, GF_SWIM, GJ_FINAL, R->swim, 0));
  std::vector<GfitResult> out;
  if (!dev.run(GF_SWIM, J, out)) return false;
  for (size_t i = 0; i < recs.size(); i++) {
    Record& R = *recs[i];
    R.num = out[i].num;
    R.den = out[i].den;
    if (!dev.read_amps(R, 0, R.amps_swim) || !dev.read_mask(R, R.dmask)) return false;
  }
  return true;
}

bool final_brownian(Device& dev, std::vector<Record*>& recs) {
  std::vector<GfitJob> J;
  for (Record* R : recs) J.push_back(make_job(*R, GF_BROWN, GJ_FINAL, R->brown, 1));
  std::vector<GfitResult> out;
  if (!dev.run(GF_BROWN, J, out)) return false;
  for (Record* R : recs)
    if (!dev.read_amps(*R, 1, R->amps_brown)) return false;
  return true;
}

DriftFit drift_of(const Record& R) {
  // a swimmer component (alpha > 0.01) restricts the drift sums to the lags
  // where its self-ISF has decayed
  return drift_lsq(R, R.swim[GP_AL] > 0.01 ? R.dmask.data() : nullptr);
}

void set_verdict(ddm_motility_result* o, bool insufficient, bool exposure_locked) {
  // G1 TSI, G2 uniform flow, G3 Delta BIC, G4 alpha resolved; G5 exposure
  int v;
  if (insufficient || !(o->TSI >= TSI_MIN)) {
    v = 3;  // NO_DYNAMICS
  } else if (o->driftMag > FLOW_SIGMA * o->driftSigma && o->driftMag > FLOW_MIN) {
    v = 2;  // DIRECTED_TRANSPORT
  } else if (!(o->dBIC > DBIC_MIN) || !(o->alpha > ALPHA_MIN && o->alphaResolved)) {
    v = 1;  // NOT_MOTILE
  } else {
    v = 0;  // MOTILE
  }
  o->physicsVerdict = v;
  o->verdict = exposure_locked ? v : 4;  // UNLOCKED_EXPOSURE overrides
}

int analyze(int n, const ddm_radial_view* radials, const ddm_motility_options* opts, ddm_motility_result* results) {
  std::vector<Record> recs(n);
  std::vector<Record*> fit;
  for (int i = 0; i < n; i++) {
    Record& R = recs[i];
    R.r = &radials[i];
    R.opt = opts[i];
    R.out = &results[i];
    std::memset(R.out, 0, sizeof(*R.out));
    R.out->mu = NAN;
    prepare(R);
    R.out->TSI = structure_index(*R.r);
    R.out->nbins = R.nb;
    R.out->nlags = R.nt;
    if (R.nb < 4) {
      R.out->insufficient = 1;
      set_verdict(R.out, true, R.opt.exposureLocked != 0);
      continue;
    }
    if (R.nt > GF_MAX_LAGS || R.K > GF_MAX_NODES) {
      ddm_detached_error() = "ddm_analyze_motility: at most 128 fit lags (L <= 4096) and 8 q-nodes per bin";
      return DDM_ERR_ARG;
    }
    fit.push_back(&R);
  }
  if (fit.empty()) return DDM_OK;
  Device dev;
  auto cuda_fail = [&]() {
    ddm_detached_error() = std::string("ddm_analyze_motility: ") + cudaGetErrorString(dev.err);
    return dev.err == cudaErrorNoDevice || dev.err == cudaErrorInsufficientDriver ? DDM_ERR_NODEV : DDM_ERR_CUDA;
  };
  if (!dev.upload(fit)) return cuda_fail();
  // pass 1: no drift in the models
  std::vector<double> zero(fit.size(), 0.0), d0(fit.size());
  if (!fit_brownian(dev, fit, zero)) return cuda_fail();
  for (size_t i = 0; i < fit.size(); i++) d0[i] = std::exp(fit[i]->brown[GP_LD]);
  if (!fit_swimmer(dev, fit, zero, d0) || !final_swimmer(dev, fit)) return cuda_fail();
  std::vector<DriftFit> drift(fit.size());
  for (size_t i = 0; i < fit.size(); i++) drift[i] = drift_of(*fit[i]);
  // pass 2: a significant uniform drift joins the null model, its speed
  // refined inside the phase band |V| +/- (3 sigma + 25 %); the swimmer model
  // reuses that speed
  std::vector<Record*> p2;
  std::vector<double> vlo, vhi, V2, D2;
  for (size_t i = 0; i < fit.size(); i++) {
    if (!(drift[i].significant && drift[i].mag > 0)) continue;
    const double half = FLOW_SIGMA * drift[i].sigma + 0.25 * drift[i].mag;
    fit[i]->pass2 = true;
    fit[i]->drift_params = 1;
    p2.push_back(fit[i]);
    vlo.push_back(std::max(0.0, drift[i].mag - half));
    vhi.push_back(drift[i].mag + half);
  }
  if (!p2.empty()) {
    if (!fit_brownian_drift(dev, p2, vlo, vhi)) return cuda_fail();
    for (Record* R : p2) {
      V2.push_back(R->brown[GP_V]);
      D2.push_back(std::exp(R->brown[GP_LD]));
    }
    if (!fit_swimmer(dev, p2, V2, D2) || !final_swimmer(dev, p2)) return cuda_fail();
    for (size_t i = 0; i < fit.size(); i++) {
      if (!fit[i]->pass2) continue;
      const DriftFit d = drift_of(*fit[i]);
      if (d.samples >= 10) drift[i] = d;
    }
  }
  if (!final_brownian(dev, fit)) return cuda_fail();
  // statistics and gates
  for (size_t i = 0; i < fit.size(); i++) {
    Record& R = *fit[i];
    ddm_motility_result* o = R.out;
    const int nData = R.nb * R.nt;
    const double rho = R.den > 0 ? std::min(0.99, std::max(0.0, R.num / R.den)) : 0.0;  // residualAutocorr :634-651
    const double nEff = std::max(2.0, nData * (1 - rho) / (1 + rho));                  // effectiveN :654-656
    auto bic = [&](double rss, double k) {                                              // :620-622
      return nEff * std::log(std::max(rss, 1e-300) / nData) + k * std::log(nEff);
    };
    const double kS = 4 + 2.0 * R.nb + R.drift_params, kB = (R.pass2 ? 2 : 1) + 2.0 * R.nb;
    const double dBIC = bic(R.brown_rss, kB) - bic(R.swim_rss, kS);
    const double v = std::exp(R.swim[GP_LV]), Z = std::exp(R.swim[GP_LZ]);
    int resolved = 0;  // motileShare :759-762
    for (int b = 0; b < R.nb; b++)
      if (R.q[b] * v * R.dt <= 0.5 && R.q[b] * v * R.tau_max >= 3) resolved++;
    o->mu = scaling_mu(R, dBIC > 0 ? R.amps_swim : R.amps_brown);
    o->alpha = R.swim[GP_AL];
    o->alphaResolved = resolved > 0;
    o->resolvedBins = resolved;
    o->vbar = v;
    o->sigmaV = v / std::sqrt(Z + 1);  // schulzSigma
    o->Z = Z;
    o->Ddiff = std::exp(R.swim[GP_LD]);
    o->DdiffBrownian = std::exp(R.brown[GP_LD]);
    o->dBIC = dBIC;
    o->driftVx = drift[i].Vx;
    o->driftVy = drift[i].Vy;
    o->driftMag = drift[i].mag;
    o->driftSigma = drift[i].sigma;
    o->driftAngleDeg = drift[i].angle;
    o->driftSignificant = drift[i].significant;
    o->driftPairs = drift[i].pairs;
    o->driftSamples = drift[i].samples;
    o->nData = nData;
    o->nEff = nEff;
    o->rho = rho;
    o->swim = ddm_motility_fit{v, Z, std::exp(R.swim[GP_LD]), R.swim[GP_V], R.swim[GP_AL], R.swim_rss};
    o->brown = ddm_motility_fit{0.0, 1.0, std::exp(R.brown[GP_LD]), R.brown[GP_V], 0.0, R.brown_rss};
    set_verdict(o, false, R.opt.exposureLocked != 0);
  }
  return DDM_OK;
}

bool valid_record(const ddm_radial_view* r, const ddm_motility_options* o) {
  return r && o && r->kCenter && r->nModes && r->D && r->P && r->drift && r->NB >= 1 && r->L >= 3 && r->N >= 8 &&
         (r->knodes <= 0 || r->kNodes) && o->dxUm > 0 && o->fps > 0 && (o->geometry2d == 0 || o->geometry2d == 1) &&
         (o->optimizer == 0 || o->optimizer == 1);
}

}  // namespace
}  // namespace ddm

extern "C" int ddm_analyze_motility(const ddm_radial_view* r, const ddm_motility_options* opt,
                                    ddm_motility_result* out) {
  ddm_detached_error().clear();
  if (!out || !ddm::valid_record(r, opt)) {
    ddm_detached_error() = "ddm_analyze_motility: invalid Radial record or options";
    return DDM_ERR_ARG;
  }
  return ddm::analyze(1, r, opt, out);
}

extern "C" int ddm_analyze_motility_batch(int32_t n, const ddm_radial_view* radials,
                                          const ddm_motility_options* opts, ddm_motility_result* out) {
  ddm_detached_error().clear();
  if (n < 0 || (n > 0 && (!radials || !opts || !out))) {
    ddm_detached_error() = "ddm_analyze_motility_batch: need n >= 0 and non-null arrays";
    return DDM_ERR_ARG;
  }
  for (int i = 0; i < n; i++)
    if (!ddm::valid_record(&radials[i], &opts[i])) {
      ddm_detached_error() = "ddm_analyze_motility_batch: record " + std::to_string(i) + " is invalid";
      return DDM_ERR_ARG;
    }
  return n ? ddm::analyze(n, radials, opts, out) : DDM_OK;
}

// ------------------------------------------------------------------ host statistics on their own
// The host half of the analysis, callable without a device (the q-bins are
// those prepare() keeps).

extern "C" double ddm_temporal_structure_index(const ddm_radial_view* r) {
  if (!r || !r->D || !r->nModes || r->NB < 1 || r->L < 3) return NAN;
  return ddm::structure_index(*r);
}

extern "C" int ddm_estimate_drift(const ddm_radial_view* r, const ddm_motility_options* opt,
                                  const uint8_t* lag_mask, double* out) {
  ddm_detached_error().clear();
  if (!out || !ddm::valid_record(r, opt)) {
    ddm_detached_error() = "ddm_estimate_drift: invalid Radial record or options";
    return DDM_ERR_ARG;
  }
  ddm::Record R;
  R.r = r;
  R.opt = *opt;
  ddm::prepare(R);
  const ddm::DriftFit f = ddm::drift_lsq(R, lag_mask);
  const double v[8] = {f.Vx, f.Vy, f.mag, f.sigma, f.angle, f.significant ? 1.0 : 0.0, (double)f.pairs, f.samples};
  for (int i = 0; i < 8; i++) out[i] = v[i];
  return DDM_OK;
}

extern "C" int ddm_scaling_exponent(const ddm_radial_view* r, const ddm_motility_options* opt, const double* amps,
                                    double* mu) {
  ddm_detached_error().clear();
  if (!mu || !amps || !ddm::valid_record(r, opt)) {
    ddm_detached_error() = "ddm_scaling_exponent: invalid Radial record, options or amplitudes";
    return DDM_ERR_ARG;
  }
  ddm::Record R;
  R.r = r;
  R.opt = *opt;
  ddm::prepare(R);
  *mu = ddm::scaling_mu(R, std::vector<double>(amps, amps + 2 * (size_t)R.nb));
  return DDM_OK;
}

extern "C" int ddm_prepared_bins(const ddm_radial_view* r, const ddm_motility_options* opt, int32_t* bins,
                                 int32_t* nbins, int32_t* nlags) {
  ddm_detached_error().clear();
  if (!nbins || !ddm::valid_record(r, opt)) {
    ddm_detached_error() = "ddm_prepared_bins: invalid Radial record or options";
    return DDM_ERR_ARG;
  }
  ddm::Record R;
  R.r = r;
  R.opt = *opt;
  ddm::prepare(R);
  *nbins = R.nb;
  if (nlags) *nlags = R.nt;
  if (bins)
    for (int i = 0; i < R.nb; i++) bins[i] = R.bin[i];
  return DDM_OK;
}
