/*
 * ddm_b200 — C ABI of the B200 (sm_100a) DDM analysis library.
 *
 * Drop-in for the operator surface of motility-ddm's WebGPU engine
 * (class DdmEngine, motility-ddm/src/ddm-engine.ts:62-426): the same calls,
 * argument meanings, data layouts and error behaviour, behind plain C types so
 * an N-API addon (Node), ctypes (Python) or any FFI can bind it. Each entry
 * point names the reference member it replaces.
 *
 * Layouts (identical to the reference):
 *   history   hist[(mode*T + slot)*2 + {re,im}], mode = ky*(N/2+1) + kx
 *             (ddm_ref.js:175-206)
 *   full      D[mode*L + tau], C[(mode*L + tau)*2 + {re,im}], P[mode]
 *             (ddm-engine.ts:403-408)
 *   radial    D[b*L + tau], P[b], drift[(b*L + tau)*8 + c] with
 *             c = Sw, Sxx, Sxy, Syy, Rx, Ry, Rpp, count (ddm_ref.js:336-348)
 *   bins      binOffsets[NB+1], binModes[4*i] = (mode, kx, ky, 0),
 *             kCenter[NB], nModes[NB], kNodes[NB*knodes] (ddm_ref.js:84-170)
 *
 * Conventions: every call returns DDM_OK (0) or an error code; the message is
 * available from ddm_last_error(). Input arrays are copied before a call
 * returns (the reference's queue.writeBuffer semantics); read functions fill
 * caller-owned arrays. One engine is single-threaded (like the reference's JS
 * event loop); distinct engines are independent.
 */
#ifndef DDM_B200_H
#define DDM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ddm_engine ddm_engine;

/* Geometry. The reference freezes N=256, T=256, TPAD=512, L=128, NB=32,
 * KMIN=4, KMAX=100, KNODES=4 (ddm_ref.js:18-31); here they are parameters.
 * Supported: N a power of two in {64..2048} or 384 or 768 (mixed-radix
 * transforms), TPAD a power of two in {128..8192}, 2 <= L <= T <= TPAD/2. */
typedef struct ddm_geometry {
  int32_t N;       /* ROI side in pixels: a power of two in [64, 2048], or 384 or 768 */
  int32_t T;       /* history slots (frames) */
  int32_t TPAD;    /* temporal FFT length; 0 = smallest power of two >= max(2T, 128) */
  int32_t L;       /* lags 0..L-1 */
  int32_t NB;      /* radial q-bins */
  double kmin;     /* inner edge of the first bin, FFT index units */
  double kmax;     /* outer edge of the last bin */
  int32_t knodes;  /* effective-|k| quadrature nodes per bin (4) */
  int32_t reserved;
} ddm_geometry;

enum ddm_dtype { DDM_U8 = 0, DDM_U16 = 1, DDM_F32 = 2 };

enum ddm_status {
  DDM_OK = 0,
  DDM_ERR_ARG = 1,     /* invalid argument (the reference throws) */
  DDM_ERR_CUDA = 2,    /* CUDA runtime failure */
  DDM_ERR_STATE = 3,   /* call not valid in the engine's state */
  DDM_ERR_NOMEM = 4,   /* device allocation failed */
  DDM_ERR_NODEV = 5,   /* no usable sm_100 device */
  DDM_ERR_TOO_LARGE = 6 /* request exceeds a fixed maximum (ddm_spectra_noalloc) */
};

/* DdmEngine.create (ddm-engine.ts:125-149): device buffers, bin table
 * (makeBins, ddm_ref.js:84-170), window and twiddle tables. */
int ddm_create(const ddm_geometry *geometry, ddm_engine **out);
/* DdmEngine.destroy (ddm-engine.ts:421-425). NULL is ignored. */
void ddm_destroy(ddm_engine *h);
/* Message of the last failed call on this engine ("" if none). */
const char *ddm_last_error(const ddm_engine *h);
/* Message of the last failed call that has no engine on this thread:
 * ddm_create or ddm_spectra_noalloc. */
const char *ddm_create_error(void);

/* Large videos (no counterpart in the reference, whose ring is fixed at
 * 256^2 x 256): an engine whose history holds only a band of spectrum
 * columns at a time, sized to history_budget_bytes (whole pairs of columns of
 * N * T complex values each; the whole half-plane if it fits). Such an engine
 * analyses a video only through ddm_analyze_banded, reads its record with
 * ddm_read_radial; the per-frame ingest, computeTemporal, readHistory and the
 * full outputs answer DDM_ERR_STATE. */
int ddm_create_banded(const ddm_geometry *geometry, uint64_t history_budget_bytes,
                      ddm_engine **out);
/* Bands of a banded engine and the spectrum columns each holds (1 and N/2+1
 * for an ordinary engine). */
int ddm_get_bands(const ddm_engine *h, int32_t *nbands, int32_t *band_cols);
/* The analysis of one video on a banded engine: for each band, the spatial
 * pass of all n frames writing that band's history (host frames stream
 * through the engine's pinned staging once per band; on_device = 1: the
 * frames are in device memory), then the band's masked Wiener-Khinchin pass
 * (order, mask as ddm_compute_temporal), its radial sums added to the record
 * band after band. Blocks until the record is ready. */
int ddm_analyze_banded(ddm_engine *h, const void *frames, int32_t dtype, int32_t n,
                       const int32_t *slots, float scale, const uint32_t *order,
                       const float *mask, int32_t on_device);

/* Resolved geometry (TPAD filled in). */
int ddm_get_geometry(const ddm_engine *h, ddm_geometry *out);
/* DdmEngine.bins (ddm-engine.ts:69): number of binned modes, then the table. */
int ddm_bins_count(const ddm_engine *h);
int ddm_get_bins(const ddm_engine *h, uint32_t *binOffsets, int32_t *binModes,
                 double *kCenter, uint32_t *nModes, double *kNodes);

/* DdmEngine.ingestLuma (ddm-engine.ts:308-324): one N*N row-major luma frame
 * (host memory) into ring slot `slot % T`. Returns DDM_OK, or sets *accepted
 * to 0 and counts a throttled frame when more than 2 ingests are still in
 * flight (the reference's MAX_PENDING back-pressure, ddm-engine.ts:46). */
int ddm_ingest_luma(ddm_engine *h, const float *luma, int32_t slot,
                    int32_t *accepted);

/* Raw-frame ingest (replaces DdmEngine.ingestFrame, ddm-engine.ts:258-302,
 * whose VideoFrame/external-texture import is a graphics path). `frames`
 * holds n frames of N*N pixels of `dtype` in HOST memory; frame i goes to
 * slot slots[i] % T with luma = value * scale (the reference's lumaOf uses
 * 1/255 for 8-bit frames, test/sim.mjs:189-193). Slots within one call must
 * be distinct. Pinned host memory is copied asynchronously, overlapped with
 * the transforms of the previous chunk; the call returns once the frames have
 * been copied off the caller's buffer. */
int ddm_ingest_frames(ddm_engine *h, const void *frames, int32_t dtype,
                      int32_t n, const int32_t *slots, float scale);
/* Same, with `frames` already in device memory (cudaMalloc / torch; 16-byte
 * aligned, else DDM_ERR_ARG). Work is queued on the engine's stream; the
 * buffer must stay valid until it runs. */
int ddm_ingest_frames_device(ddm_engine *h, const void *frames, int32_t dtype,
                             int32_t n, const int32_t *slots, float scale);
/* ddm_ingest_frames without the final wait (no counterpart in the reference,
 * whose writeBuffer copies at call time): returns once the copies and
 * transforms are queued, so a host with a stream of videos keeps the PCIe
 * link busy while it prepares the next call. The host buffer must stay
 * unchanged until ddm_ingest_wait returns (or a later synchronous ingest,
 * ddm_idle or ddm_destroy). Pinned memory is needed for the copies to be
 * asynchronous at all. */
int ddm_ingest_frames_async(ddm_engine *h, const void *frames, int32_t dtype,
                            int32_t n, const int32_t *slots, float scale);
/* Waits until the frames of every earlier ingest have been copied off the
 * caller's buffers. */
int ddm_ingest_wait(ddm_engine *h);

/* Spatial ROI mask (extension; the reference has none): N*N bytes, 1 = pixel
 * used. Masked pixels are excluded from the frame mean and zeroed before the
 * window. NULL restores the full frame. */
int ddm_set_spatial_mask(ddm_engine *h, const uint8_t *mask);

/* DdmEngine.computeTemporal (ddm-engine.ts:331-365): order[j] = ring slot of
 * time index j, mask[j] = 1 if time index j holds a valid frame (length T;
 * temporalMeta, ddm_ref.js:538-560). full = 0 computes the radial record
 * only (binned modes, the reference's analyzeRadial, ddm_ref.js:425-437);
 * full = 1 also keeps per-mode D, C, P for every mode (analyzeFull,
 * ddm_ref.js:450-463). Blocks until the results are ready. */
int ddm_compute_temporal(ddm_engine *h, const uint32_t *order,
                         const float *mask, int32_t full);
/* Same, without waiting: the work is queued on the engine's stream. */
int ddm_compute_temporal_async(ddm_engine *h, const uint32_t *order,
                               const float *mask, int32_t full);
/* Live analysis: the dashboard's analysis tick (main.ts:366-398) with
 * computeTemporal running while frames keep arriving (ddm-engine.ts:331-365).
 * The snapshot holds every frame queued before the call; the analysis runs
 * on the engine's analysis stream and returns at once, so later ingests
 * proceed concurrently. Ring slots those ingests overwrite must be masked
 * out of `mask` (the guard of FrameClock.snapshot, camera.ts:408-425).
 * DDM_ERR_STATE "computeTemporal is already running" while the previous
 * live analysis is in flight (ddm-engine.ts:332). The result stays readable
 * (ddm_read_radial, ddm_read_temporal_full) until the next computeTemporal,
 * whatever is ingested meanwhile. */
int ddm_compute_temporal_live(ddm_engine *h, const uint32_t *order,
                              const float *mask, int32_t full);
/* *done = 1 once no live analysis is in flight (surfacing its device error). */
int ddm_analysis_poll(ddm_engine *h, int32_t *done);
/* Waits for the live analysis in flight, if any. */
int ddm_wait_analysis(ddm_engine *h);

/* DdmEngine.readRadial (ddm-engine.ts:391-395) + radialFromGpu
 * (ddm_ref.js:584-590): D[NB*L], P[NB], drift[NB*L*8] in FP64. */
int ddm_read_radial(ddm_engine *h, double *D, double *P, double *drift);
/* DdmEngine.readHistory (ddm-engine.ts:398-400): modes*T*2 floats. */
int ddm_read_history(ddm_engine *h, float *out);
/* DdmEngine.readTemporalFull (ddm-engine.ts:403-408); needs a preceding
 * ddm_compute_temporal with full = 1, else DDM_ERR_STATE. */
int ddm_read_temporal_full(ddm_engine *h, float *D, float *C, float *P);
/* DdmEngine.readMean (ddm-engine.ts:411-414): last ingested frame's mean
 * luma (over the spatial mask when one is set). */
int ddm_read_mean(ddm_engine *h, double *mean);
/* DdmEngine.idle (ddm-engine.ts:417-419): waits for all queued work. */
int ddm_idle(ddm_engine *h);

/* Back-pressure state (ddm-engine.ts:120-124, 216-224, 107). */
int ddm_pending(ddm_engine *h);
int ddm_wait_for_capacity(ddm_engine *h);
int64_t ddm_throttled(const ddm_engine *h);

/* Run the engine's work on a caller's CUDA stream (cudaStream_t as void*),
 * e.g. to time it with events on that stream. NULL restores the engine's own
 * stream. */
int ddm_set_stream(ddm_engine *h, void *stream);
/* Autotuner (no reference counterpart): times the engine's kernels on this
 * device for its geometry and keeps the fastest spatial chunk (frames per
 * row/column launch pair), temporal work-unit size (modes per unit) and
 * temporal kernel variant (0: one group of TPAD/8 threads, radix-8 stages;
 * 1: two groups of TPAD/16 threads, radix-16 stages, TPAD 1024..4096). The
 * timing runs overwrite the history ring: call it right after ddm_create,
 * before ingesting and before ddm_batch_create over the engine. `report`
 * (may be NULL) receives a JSON summary of every candidate's time. */
int ddm_autotune(ddm_engine *h, char *report, int32_t report_len);
/* The temporal pass of an analysis whose 0/1 mask drops few time indices
 * (a recording with a few missing frames) computes A + B of the masked
 * Wiener-Khinchin formula from FP64 prefix sums and the masked set instead
 * of two transforms, and pairs the modes' |Y|^2 in one inverse transform:
 * 1.5 transforms per mode instead of 2.5. "Few": at most 64 zeros for TPAD
 * 256..4096; at TPAD 8192, 256 divided by the lags per thread (L/512 rounded
 * up to 1, 2, 4 or 8) while the tables fit shared memory. A batch takes it
 * when every video qualifies and its first engine has it enabled. enable = 0
 * keeps the transform path for every mask. Default 1. */
int ddm_set_sparse(ddm_engine *h, int32_t enable);
/* Short lag ranges on long series (no counterpart in the reference): at TPAD
 * 8192 with L <= 128 the fused path assembles every correlation from
 * 128-sample blocks with 256-point transforms (DDM_TK_BLOCKED) instead of
 * 8192-point ones. enable = 0 keeps the TPAD 8192 kernels. Default 1. */
int ddm_set_blocked(ddm_engine *h, int32_t enable);
/* The temporal kernel of the engine's last computeTemporal: DDM_TK_RADIX8
 * (one-group radix-8 transforms), DDM_TK_RADIX16 (two-group radix-16),
 * DDM_TK_SPARSE (sparse-mask kernel), DDM_TK_BIG (TPAD 8192),
 * DDM_TK_SPARSE_BIG (sparse-mask kernel at TPAD 8192), DDM_TK_BLOCKED (TPAD
 * 8192 with L <= 128: correlations from 128-sample blocks); -1 before the first
 * analysis (instrumentation). */
enum { DDM_TK_RADIX8 = 0, DDM_TK_RADIX16 = 1, DDM_TK_SPARSE = 2, DDM_TK_BIG = 3, DDM_TK_SPARSE_BIG = 4,
       DDM_TK_BLOCKED = 5 };
int ddm_last_temporal_kernel(const ddm_engine *h);
/* The engine's current chunk, unit size and variant; set them without
 * timing (e.g. from a cached autotune report; chunk/unit 0 and variant -1
 * keep a value). */
int ddm_get_tuning(const ddm_engine *h, int32_t *chunk, int32_t *unit_size, int32_t *variant);
int ddm_set_tuning(ddm_engine *h, int32_t chunk, int32_t unit_size, int32_t variant);

/* Kernels launched by this engine so far (instrumentation). */
int64_t ddm_kernel_launches(const ddm_engine *h);

/* ---------------------------------------------------------------------------
 * Decision layer: analyzeMotility (motility-ddm/src/motility_fit.js:870-990)
 * on a Radial record -- Brownian, Brownian+drift and swimmer fits of ONE
 * parameter set shared by all q-bins (the reference's VarPro objective,
 * evalModel :450-474, with its start sets: fitBrownian :500-536,
 * fitBrownianDrift :545-568, fitSwimmer :577-611), phase drift, temporal
 * structure index, BIC with the residual autocorrelation, q-scaling, and the
 * five gates -> verdict. The fits run on the current CUDA device in FP64:
 * scans and start sets as parallel jobs, each search a bounded
 * Levenberg-Marquardt iteration by one thread-block cluster (the reference
 * uses Nelder-Mead on one CPU thread). The Radial record is the one
 * ddm_read_radial returns with the engine's bins. The first call on a device
 * builds the 2D swimmer-ISF table (a kernel launch and a synchronisation). */
typedef struct ddm_radial_view {
  int32_t N, NB, L, knodes;
  const double *kCenter;   /* [NB] */
  const double *kNodes;    /* [NB*knodes] */
  const uint32_t *nModes;  /* [NB] */
  const double *D;         /* [NB*L] */
  const double *P;         /* [NB] */
  const double *drift;     /* [NB*L*8] */
} ddm_radial_view;

typedef struct ddm_motility_options {
  double dxUm, fps;        /* pixel pitch (um) and frame rate (1/s) */
  int32_t geometry2d;      /* 0: 3D swimmers ('3d'), 1: in-plane ('2d') */
  int32_t exposureLocked;  /* 0 gives UNLOCKED_EXPOSURE (gate G5) */
  double swimMin;          /* GATES.SWIM_MIN_UM_S, 2 in the reference */
  int32_t optimizer;       /* 0: the reference's searches (golden section, Nelder-Mead);
                              1: bounded Levenberg-Marquardt from the same starts (extension) */
  int32_t reserved;
} ddm_motility_options;

typedef struct ddm_motility_fit {
  double vbar, Z, Dd, Vmag, alpha, rss;
} ddm_motility_fit;

/* verdict: 0 MOTILE, 1 NOT_MOTILE, 2 DIRECTED_TRANSPORT, 3 NO_DYNAMICS,
 * 4 UNLOCKED_EXPOSURE (motility_fit.js:40-46); fields as the reference's
 * result object (motility_fit.js:918-990). */
typedef struct ddm_motility_result {
  int32_t verdict, physicsVerdict, insufficient;
  double TSI, alpha;
  int32_t alphaResolved, resolvedBins;
  double vbar, sigmaV, Z, Ddiff, DdiffBrownian, dBIC;
  double driftVx, driftVy, driftMag, driftSigma, driftAngleDeg;
  int32_t driftSignificant, driftPairs;
  double driftSamples;
  double mu;
  int32_t nData;
  double nEff, rho;
  int32_t nbins, nlags;
  ddm_motility_fit swim, brown;
} ddm_motility_result;

int ddm_analyze_motility(const ddm_radial_view *radial, const ddm_motility_options *opt,
                         ddm_motility_result *out);
/* analyzeMotility of n records at once (no counterpart in the reference,
 * which analyses one record per worker message, motility_fit.js:996-1004):
 * each stage of the analysis runs the device jobs of every record in one
 * launch. out[i] equals ddm_analyze_motility(&radials[i], &opts[i]). */
int ddm_analyze_motility_batch(int32_t n, const ddm_radial_view *radials,
                               const ddm_motility_options *opts, ddm_motility_result *out);
/* The swimmer self-ISF kernels as the fits evaluate them, for n points of
 * host arrays x = q vbar tau and Z: g, x dg/dx and Z dg/dZ (the last two may
 * be NULL). geometry2d 0: isf3d (motility_fit.js:140-144); 1: the 2D kernel
 * isf2d (:152-159) read from the device table that replaces the reference's
 * isf2dFast (:168-220). */
int ddm_isf_eval(int32_t n, int32_t geometry2d, const double *x, const double *Z,
                 double *g, double *xdgdx, double *Zdgdz);
/* Batched zero-padded 2048-point DFT on the tensor cores (no reference
 * counterpart; a measured reference point for the temporal stage's forward
 * transforms, not on the analysis path): X[i][k] = sum_{t<1024} x[i*ld + t]
 * exp(-2 pi i t k / 2048), k < 2048, for n series. x: DEVICE complex64, ld
 * >= 1024 elements between series; X: DEVICE complex64 [n][2048]. tcgen05
 * BF16 products with a three-term split, FP32 accumulation: within ~2e-5 of
 * each series' RMS spectrum. Queued on `stream` (cudaStream_t as void*) and
 * waited for; errors via ddm_create_error(). */
int ddm_dft2048_tc(const void *x, int64_t ld, int32_t n, void *X, void *stream);
/* The host half of the analysis on its own (no device needed). The q-bins
 * are those prepare() keeps (motility_fit.js:383-401): ddm_prepared_bins
 * returns their Radial indices (bins may be NULL to query the count; up to
 * NB values) and the number of fit lags (lagGrid, :358-369). */
int ddm_prepared_bins(const ddm_radial_view *radial, const ddm_motility_options *opt,
                      int32_t *bins, int32_t *nbins, int32_t *nlags);
/* temporalStructureIndex (:735-749); NaN for an invalid record. */
double ddm_temporal_structure_index(const ddm_radial_view *radial);
/* estimateDrift (:672-725). lag_mask [nbins][L] (prepared bins; 1 = use the
 * lag) restricts the drift sums to lags where the swimmer ISF has decayed,
 * NULL = every lag. out[8] = Vx, Vy, |V|, sigma, angle (deg), significant,
 * pairs, samples. */
int ddm_estimate_drift(const ddm_radial_view *radial, const ddm_motility_options *opt,
                       const uint8_t *lag_mask, double *out);
/* scalingExponent's mu (:771-804) from per-prepared-bin amplitudes
 * amps[2*i] = A, amps[2*i+1] = B; NaN when fewer than 3 bins cross half. */
int ddm_scaling_exponent(const ddm_radial_view *radial, const ddm_motility_options *opt,
                         const double *amps, double *mu);

/* ---------------------------------------------------------------------------
 * Batches: many videos of uneven size and frame count analysed together (no
 * counterpart in the reference, whose engine holds one video). A batch
 * borrows existing engines (any geometries, one device; the caller keeps
 * them alive and destroys them after the batch). Every engine's spatial
 * chunks are queued on the batch stream without host synchronisation, and
 * the temporal analysis of ALL videos is one persistent launch over the
 * concatenated work units of every engine, at the batch's largest TPAD (zero
 * padding beyond T + L - 1 leaves every lag < L exact: each video's radial
 * record, read with ddm_read_radial on its engine, equals what its own
 * engine computes). The whole step can be captured once into a CUDA graph
 * and replayed. Errors via ddm_batch_last_error(b) (NULL after a failed
 * create). */
typedef struct ddm_batch ddm_batch;
int ddm_batch_create(ddm_engine *const *engines, int32_t n, ddm_batch **out);
void ddm_batch_destroy(ddm_batch *b);
const char *ddm_batch_last_error(const ddm_batch *b);
/* The stream the batch queues its work on (NULL = its own stream). */
int ddm_batch_set_stream(ddm_batch *b, void *stream);
/* Spatial stage of every video from DEVICE frames (16-byte aligned):
 * frames[i] holds n[i] frames of engine i (dtype dtypes[i]), slots[i][n[i]],
 * luma scale scales[i]. Queued, no host synchronisation (a changed scale is
 * uploaded first, which synchronises). */
int ddm_batch_ingest(ddm_batch *b, const void *const *frames, const int32_t *dtypes,
                     const int32_t *n, const int32_t *const *slots, const float *scales);
/* Temporal analysis of every video in one launch; orders[i] and masks[i] of
 * length T_i (as ddm_compute_temporal). Computes the per-video tables on the
 * host, then queues the copies, the launch and the per-video reductions. */
int ddm_batch_compute_temporal(ddm_batch *b, const uint32_t *const *orders,
                               const float *const *masks);
/* The queued part of ddm_batch_compute_temporal alone, from the tables the
 * last ddm_batch_compute_temporal filled in. */
int ddm_batch_enqueue_temporal(ddm_batch *b);
/* Waits for the batch stream; surfaces device-side error words. */
int ddm_batch_sync(ddm_batch *b);
/* Captures ddm_batch_ingest(frames...) + ddm_batch_enqueue_temporal into a
 * CUDA graph (after one ddm_batch_compute_temporal); ddm_batch_launch_graph
 * replays it on the batch stream (new orders/masks: call
 * ddm_batch_compute_temporal's table step again first -- it also runs the
 * step once). */
int ddm_batch_capture(ddm_batch *b, const void *const *frames, const int32_t *dtypes,
                      const int32_t *n, const int32_t *const *slots, const float *scales);
int ddm_batch_launch_graph(ddm_batch *b);

/* Batched per-bin Levenberg-Marquardt fit of the motility model (the fit
 * stage of analyzeMotility, motility-ddm/src/motility_fit.js:577-611, per
 * q-bin). The reference fits (alpha, vbar, Z, D) globally by VarPro +
 * Nelder-Mead and has no LM; this solves, for each of nfit bins, one warp per
 * bin,
 *   min sum_j (w (A c(tau_j) + B - d_j))^2,
 *   c = 1 - <exp(-D q^2 tau) (1 - alpha + alpha g(q vbar tau; Z))>_nodes
 * (modelColumn, motility_fit.js:417-432, 3D Schulz swimmer ISF g; see
 * ddm_fit_lm_model for the 2D kernel and the drift factor) over
 * theta = (A, B, alpha, ln vbar, ln Z, ln D), A, B >= 0, alpha in [0, 1], the
 * rest clamped to bounds[6*i..] = (vmin, vmax, Zmin, Zmax, Dmin, Dmax)
 * (bounds(), :480-491). Model in FP32, normal equations (J^T J + lambda I,
 * Marquardt scaling) and the Cholesky solve in FP64.
 *   mode 0: the reference's start strategy per bin -- 49-point ln D Brownian
 *           scan + golden section (fitBrownian :500-536), then 64 starts
 *           (16 vbar x Z in {1.5, 8} x alpha in {0.3, 0.8}, fitSwimmer
 *           :589-601) ranked by VarPro cost, LM from the best `nrefine`.
 *   mode 1: LM from start[4*i..] = (alpha, vbar, Z, D) (e.g. the surrogate's
 *           prediction), amplitudes from VarPro.
 *   mode 2: as mode 1; a fit whose LM did not converge (stopped at
 *           max_iter) or whose cost exceeds a coarse 17-point Brownian
 *           (alpha = 0) scan -- impossible at a global optimum, since the
 *           Brownian model is nested -- also runs mode 0 and keeps the lower
 *           cost (the reference's starts as the fallback).
 *   mode 4: as mode 1; the fallback to mode 0 is decided by the cost alone:
 *           it runs when the seeded cost exceeds the bin's Brownian optimum
 *           (mode 3's search, FP64 model). A seeded LM stopped at max_iter
 *           below that bound is kept.
 *   mode 3: the Brownian model alone, A (1 - <exp(-D q_n^2 tau)>) + B, one D
 *           per bin by fitBrownian's search (the 49-point scan + golden
 *           section of mode 0); theta = (A, B, 0, ln vmin, ln Zmin, ln D),
 *           status bit 0 = the golden-section bracket closed.
 * Arrays: nt[nfit] lags per fit (<= nt_max <= 128), d and tau [nfit][nt_max],
 * qn [nfit][K] (K <= 8), w[nfit], bounds [nfit][6], start [nfit][4];
 * out theta [nfit][6], cost[nfit], iters/evals/status [nfit] (may be NULL;
 * status bit 0 = converged, bit 1 = fell back to mode 0).
 * on_device = 0: host arrays, blocks until done; 1: device arrays, queued on
 * `stream` (cudaStream_t as void*). Errors via ddm_create_error(). */
int ddm_fit_lm(int32_t nfit, int32_t nt_max, int32_t K, const int32_t *nt, const float *d,
               const float *tau, const float *qn, const float *w, const float *bounds,
               const float *start, int32_t mode, int32_t max_iter, double tol, int32_t nrefine,
               double *theta, double *cost, int32_t *iters, int32_t *evals, int32_t *status,
               int32_t on_device, void *stream);
/* ddm_fit_lm with the rest of modelColumn (motility_fit.js:417-432): the
 * swimmer kernel of the geometry (geometry2d 0: isf3d :140-144; 1: the 2D
 * kernel isf2d :152-159 from the device table, swimmerKernel :227-229) and
 * the drift factor J0(q |V| tau) with vmag[nfit] the known drift speed of
 * each fit (NULL: no factor; host or device array like the others). The
 * first 2D call on a device builds the table (a kernel launch and a
 * synchronisation: make it before any stream capture). ddm_fit_lm is this
 * call with geometry2d = 0 and vmag = NULL. */
int ddm_fit_lm_model(int32_t nfit, int32_t nt_max, int32_t K, const int32_t *nt, const float *d,
                     const float *tau, const float *qn, const float *w, const float *bounds,
                     const float *start, int32_t mode, int32_t max_iter, double tol, int32_t nrefine,
                     int32_t geometry2d, const float *vmag, double *theta, double *cost,
                     int32_t *iters, int32_t *evals, int32_t *status, int32_t on_device, void *stream);

/* Model curves for training and evaluation data (no reference counterpart):
 * y[i][j] = (A c(tau_j) + B) (1 + noise * n_ij), c the model column above
 * (FP32), n_ij standard normal from a counter-based generator keyed by
 * (seed, i, j). theta [n][6] = (A, B, alpha, vbar, Z, D) (linear units),
 * qn [n][K], tau [nt] shared; tau_e[i] (may be NULL) = the first lag where
 * c reaches 1 - 1/e (noise-free). DEVICE arrays, queued on `stream`. */
int ddm_model_curves(int32_t n, int32_t K, const float *qn, const float *theta, int32_t nt,
                     const float *tau, float noise, uint64_t seed, float *y, float *tau_e,
                     void *stream);

/* ---------------------------------------------------------------------------
 * Learned seed for the fit: a BF16 tensor-core MLP (no counterpart in the
 * reference). Input: 65 features per q-bin -- the bin's D(q, tau) at 64
 * log-spaced lags divided by its maximum, and ln(q)/4; output: 5 motility
 * parameters in normalised units (see hackathon_b200/surrogate.py);
 * 65 -> 256 -> 256 -> 256 -> 256 -> 5 with GELU. All products run on tcgen05
 * tensor cores (BF16 operands, FP32 accumulators in tensor memory); FP32
 * master weights with Adam. Its prediction only seeds ddm_fit_lm (mode 1).
 * x, y and out are DEVICE arrays (row-major [n][65], [n][5], [n][5]); n is a
 * multiple of 8 and at most batch_max. Work is queued on the caller's
 * `stream` (cudaStream_t as void*, NULL = the legacy default stream), in
 * order with the caller's other work there; one model serves one stream at
 * a time. Errors via ddm_mlp_last_error(h)
 * (or with h = NULL after a failed create). Parameters travel as one flat
 * FP32 array: per layer W [out][in] row-major, then b [out]. */
typedef struct ddm_mlp ddm_mlp;
int ddm_mlp_create(int32_t batch_max, uint64_t seed, ddm_mlp **out);
void ddm_mlp_destroy(ddm_mlp *h);
const char *ddm_mlp_last_error(const ddm_mlp *h);
int32_t ddm_mlp_param_count(void);
int ddm_mlp_get_params(ddm_mlp *h, float *params);
int ddm_mlp_set_params(ddm_mlp *h, const float *params);
/* Inference. */
int ddm_mlp_forward(ddm_mlp *h, const float *x, int32_t n, float *out, void *stream);
/* Forward + backward of the mean-squared error; host grads in the parameter
 * layout and the loss (may be NULL). Blocks. */
int ddm_mlp_gradients(ddm_mlp *h, const float *x, const float *y, int32_t n, float *grads,
                      float *loss, void *stream);
/* One Adam step (lr; beta 0.9, 0.999). loss != NULL blocks and returns it. */
int ddm_mlp_train_step(ddm_mlp *h, const float *x, const float *y, int32_t n, float lr,
                       float *loss, void *stream);
/* Waits for `stream`; surfaces the model's device-side error words. */
int ddm_mlp_sync(ddm_mlp *h, void *stream);

/* Allocation-free spatial stage. No counterpart in the reference (its WebGPU
 * engine allocates all buffers at create time); this is for callers that may
 * not allocate device memory at all -- a host framework that owns every
 * device allocation and only lends its plugins planned buffers, or a capture
 * loop that must not enter cudaMalloc, which can stall on device-wide
 * synchronisation. Needs no engine.
 *
 * Transforms n frames (DEVICE memory, 16-byte aligned, N*N pixels of `dtype` each, luma =
 * value * scale) exactly as ddm_ingest_frames_device does and writes frame i
 * into ring slot slots[i] % T of the caller's DEVICE history `hist`
 * (float2 [N*(N/2+1)][T], the readHistory layout), on `stream`
 * (cudaStream_t as void*; NULL = legacy default stream). No spatial mask.
 * It calls no cudaMalloc/cudaFree: its scratch is a fixed 8 MiB file-scope
 * device array (plus < 1 MiB of tables) that every GPU loading the library
 * holds until exit, so N is limited to 64..512 (DDM_ERR_TOO_LARGE above).
 * The first call on a device, and any call that changes N or scale, does
 * set-up (symbol lookups, table uploads, a stream synchronisation): make the
 * first call before any stream capture. All calls share the scratch: calls
 * whose work overlaps on the GPU race, so serialise them. Errors: DDM_ERR_ARG,
 * DDM_ERR_TOO_LARGE, DDM_ERR_CUDA, DDM_ERR_NODEV; message from
 * ddm_create_error(). The call returns once its work is queued; a bounded
 * wait for a staged copy that gave up on the device is reported by
 * ddm_spectra_noalloc_status. */
int ddm_spectra_noalloc(const void *frames, int32_t dtype, int32_t n, int32_t N,
                        int32_t T, const int32_t *slots, float scale, void *hist,
                        void *stream);
/* Completion status of the last ddm_spectra_noalloc call queued on `stream`
 * on the current device: waits for the stream, then returns DDM_OK, or
 * DDM_ERR_CUDA when one of its kernels recorded a staged copy that did not
 * complete in time (the ring is then partly written; the device word is
 * cleared). Allocates nothing. No counterpart in the reference (its WebGPU
 * queue reports validation errors through onError, ddm-engine.ts:28). */
int ddm_spectra_noalloc_status(void *stream);

/* ------------------------------------------------------------------ movies
 * The reference's seeded movie generator (test/sim.mjs:90-186: mulberry32
 * stream, polar normals, Marsaglia-Tsang gammas, periodic Gaussian blobs, u8
 * quantisation, drop masks) on the GPU, for training data and large inputs.
 * Same seed, same random streams: frames equal the reference's up to one grey
 * level where a pixel sits on a rounding boundary (exp/log within an ulp).
 * Field names follow SimParams (sim.mjs:66-84); swimmers/passive/fixed/drift
 * are flattened. */
typedef struct ddm_sim_params {
  int32_t N, T;             /* frame size (multiple of 16), frames */
  double fps, dxUm;
  uint32_t seed;
  int32_t nSwim;            /* swimmers: count, mean speed, speed sd, 2-D flag */
  double swimVbar, swimSigma;
  int32_t swim2d;
  int32_t nPassive;         /* Brownian particles */
  double Dum2s;             /* diffusion coefficient, um^2/s */
  int32_t nFixed;           /* particles stuck to the glass */
  int32_t hasDrift;
  double driftSpeed, driftAngleDeg;
  double dropFrac;          /* random frame drops (frame 0 always kept) */
  int32_t dropExact;        /* exactly this many drops instead, if > 0 */
  double blobSigmaPx, amp, background, noise;
} ddm_sim_params;

/* frames: T*N*N u8 (device memory if frames_on_device, else host); valid[T]
 * 1/0; truth[4] (may be NULL): mean swim speed, Vx, Vy, D. Runs on `stream`
 * (NULL: the legacy default stream) and returns when the movie is complete. */
int ddm_simulate(const ddm_sim_params *p, uint8_t *frames, int32_t frames_on_device,
                 uint8_t *valid, double *truth, void *stream);
const char *ddm_simulate_error(void);

#ifdef __cplusplus
}
#endif
#endif /* DDM_B200_H */
