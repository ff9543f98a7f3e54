"""Benchmark of the DDM analysis hot path: frames/s at 512^2 x 1024 uint16.

One step = one full pass of the path over one video (1024 frames of 512^2
u16): spatial FFT of every frame into the mode-major history, masked
Wiener-Khinchin temporal analysis of every binned mode (TPAD 2048, L = 512
lags), radial reduction into 256 q-bins (the reference's History.ingest ->
analyzeRadial, motility-ddm/src/ddm_ref.js:196-206, 425-437).

  value  frames/s with the frames already in HBM (device-timed, CUDA events on
         the engine's stream, max over ranks, summed over ranks)
  e2e    the same through the C ABI from pinned HOST frames: every step copies
         its frames host->device and reads the radial record back; three
         engines take the videos in turn, so one video's copies overlap the
         previous videos' temporal analyses
Under torchrun each rank analyses its own video (weak scaling, no collective
on the data path).

  roofline  the dominant kernel (the temporal kernel the engine ran: with 2 %
         dropped frames the sparse-mask kernel) against the HBM peak, with
         its FP32 rate beside it, both stages' figures, and cuFFT running just
         the stages' transforms on device-resident data as a library
         reference point

  fit    (rank 0) q-fits/s of the batched GPU LM on 10^5 held-out q-curves:
         plain (the reference's start strategy), seeded by the tensor-core
         surrogate (trained in the run on 2^20 curves: 2^19 analytic + 2^19
         radial curves the engine produces from seeded 512^2 x 1024 videos;
         also evaluated on held-out pipeline curves), and seeded with the plain
         strategy as fallback; fit error as the share of curves whose cost is
         within 1e-3 of the plain LM's, and agreement with the FP64 LM oracle
         on a bounded sample.

--impl reference times the reference's CPU algorithm on the host cores: the
reference is JavaScript with no runtime on this machine, so its FP64 C
restatement (oracle/, test infrastructure) stands in, on a bounded sample.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N, T, TPAD, L, NB, KMIN, KMAX = 512, 1024, 2048, 512, 256, 4.0, 200.0
METRIC = "DDM frames/s at 512²×1024"
WORKLOAD = ("512x512x1024 u16 video: 2000 blobs sigma 2 px, 30% Brownian D=0.2 px^2/frame, 70% "
            "straight swimmers Schulz vbar=1.5 px/frame Z=4 (+D=0.2), Poisson noise mean 400 "
            "counts, circular ROI r=230 px, 2% dropped frames; TPAD=2048, L=512 lags, 256 q-bins "
            "(kmin 4, kmax 200)")
# nominal FP32 CUDA-core peak: 148 SMs x 128 lanes x 2 FLOP x 1.965 GHz
FP32_NOMINAL_TFLOPS = 74.4
# algorithmic HBM bytes per frame: u16 input + spectrum write + spectrum read
BYTES_PER_FRAME_IN = N * N * 2
BYTES_PER_MODE_SLOT = 8


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled every 5 ms during
    the timed region, through NVML (the counters nvidia-smi's
    clocks.sm / clocks_event_reasons.* report). Read-only: no setting of the
    GPU is changed."""

    REASONS = (("hw_slowdown", 0x8), ("sw_thermal_slowdown", 0x20), ("hw_thermal_slowdown", 0x40),
               ("sw_power_cap", 0x4))

    def __init__(self, cuda_index):
        self.cuda_index = cuda_index
        self.samples = []
        self.window = None
        self._stop = threading.Event()
        self.t = None

    def _handle(self, nv):
        import torch
        try:
            return nv.nvmlDeviceGetHandleByUUID("GPU-" + str(torch.cuda.get_device_properties(self.cuda_index).uuid))
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.cuda_index)

    def start(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv, self.h = nv, self._handle(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
        except Exception:
            self.nv = None
            return
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def _run(self):
        nv, h = self.nv, self.h
        while not self._stop.is_set():
            try:
                self.samples.append((time.perf_counter(), nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM),
                                     nv.nvmlDeviceGetCurrentClocksEventReasons(h)))
            except Exception:
                return
            time.sleep(0.005)

    def mark(self, t0, t1):
        """Host-time window of the timed region; only samples inside it count
        (all samples, if none fell inside)."""
        self.window = (t0, t1)

    def stop(self):
        if self.t is None:
            return None
        self._stop.set()
        self.t.join(timeout=2)
        w = self.window
        inside = [s for s in self.samples if w and w[0] <= s[0] <= w[1]]
        use = inside or self.samples
        if not use:
            return None
        reasons = sorted({nm for _, _, r in use for nm, bit in self.REASONS if r & bit})
        return {"sm_mhz": statistics.median(m for _, m, _ in use), "sm_max_mhz": float(self.max_mhz),
                "reasons": reasons, "samples": len(use), "samples_inside_timed_region": len(inside),
                "source": "NVML, 5 ms period"}


def _profile_traffic():
    """DRAM bytes (read + write) per launch of the dominant kernel from the
    committed ncu summary (profiles/ncu_traffic.txt, 'key value' lines), or
    None."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.txt")
    if not os.path.exists(p):
        return None
    out = {}
    for ln in open(p):
        parts = ln.split()
        if len(parts) == 2 and not ln.startswith("#"):
            try:
                out[parts[0]] = float(parts[1])
            except ValueError:
                pass
    return out


# the CPU baseline's temporal sample: the modes of every CPU_BIN_STRIDE-th
# q-bin from bin 3 on (25.2 % of the binned modes at 256 bins), on the
# video's real history
CPU_BIN_STRIDE = 4
E2E_ENGINES = 3  # engines taking videos in turn in the e2e measurement


def _sampled_bins(bins, stride):
    off = bins["binOffsets"]
    sel = np.arange(stride - 1, bins["NB"], stride)
    rows = [bins["binModes"][off[b]:off[b + 1]] for b in sel]
    sub = dict(bins)
    sub.update(NB=len(sel), binModes=np.ascontiguousarray(np.concatenate(rows)),
               binOffsets=np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.uint32),
               nModes=np.ascontiguousarray(bins["nModes"][sel]).astype(np.uint32))
    return sel, sub


def cpu_baseline(frames_u16, valid, roi, threads=None, gpu_radial=None, one_core=False, reps=1):
    """The reference's CPU algorithm (its FP64 C restatement, oracle/) on this
    very video, timed on the host cores. Both arms call it with the same
    sample:
      spatial   every valid frame of the video (History.ingest,
                ddm_ref.js:196-206, with the ROI pixel mask the engine applies)
                -- the real history, not a sample;
      temporal  the masked Wiener-Khinchin analysis and radial sums
                (analyzeRadial, ddm_ref.js:425-437) of every CPU_BIN_STRIDE-th
                q-bin's modes of that history, scaled to all binned modes.
    frames/s = T / (spatial time + temporal time / sampled share of modes);
    `reps` timings, the median kept. With gpu_radial, the sampled bins' radial
    D is compared with the GPU's record (max |dD| / bin scale); one_core adds
    a single-thread figure from 16 frames and every 16th sampled mode."""
    import oracle as O
    threads = threads or os.cpu_count()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    idx = np.nonzero(valid)[0]
    order, mask = O.linear_order(valid)
    bins = O.make_bins(N, NB, KMIN, KMAX)
    nbinned = int(bins["binOffsets"][-1])
    sel, sub = _sampled_bins(bins, CPU_BIN_STRIDE)
    frac = sub["binModes"].shape[0] / nbinned
    runs = []
    hist = ro = None
    for _ in range(reps):
        hist = np.zeros((N * (N // 2 + 1), T), np.complex128)
        t0 = time.perf_counter()
        for c in range(0, idx.size, 64):
            k = idx[c:c + 64]
            O.history_ingest(frames_u16[k].astype(np.float64) * (1.0 / 65535), k.astype(np.int32), T, hist=hist,
                             smask=roi)
        t_sp = time.perf_counter() - t0
        t0 = time.perf_counter()
        ro = O.analyze_radial(hist, order, mask, sub, L, TPAD=TPAD, threads=threads)
        t_tm = time.perf_counter() - t0
        runs.append((T / (t_sp + t_tm / frac), t_sp, t_tm))
    runs.sort()
    v, t_sp, t_tm = runs[len(runs) // 2]
    out = {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
           "sample": f"spatial: all {idx.size} valid frames of the video; temporal: the {sub['binModes'].shape[0]} "
                     f"modes of every {CPU_BIN_STRIDE}th q-bin ({frac:.1%} of the {nbinned} binned modes) on the "
                     f"video's own FP64 history, scaled to all binned modes; TPAD={TPAD}, L={L}, FP64",
           "sample_mode_frac": frac, "spatial_s": t_sp, "temporal_s_sampled": t_tm, "reps": reps}
    if gpu_radial is not None:
        # the same record's motility analysis by the oracle (one thread, like
        # the reference's worker), beside the GPU's
        rec = O.Radial(gpu_radial.N, gpu_radial.NB, gpu_radial.L, np.asarray(gpu_radial.kCenter, np.float64),
                       np.asarray(gpu_radial.kNodes, np.float64), np.asarray(gpu_radial.nModes, np.uint32),
                       np.asarray(gpu_radial.D, np.float64), np.asarray(gpu_radial.P, np.float64),
                       np.asarray(gpu_radial.drift, np.float64))
        t0 = time.perf_counter()
        ores = O.analyze_motility(rec, **MOTILITY_OPTS)
        ta = time.perf_counter() - t0
        out["analysis"] = {"what": "analyzeMotility of the GPU's radial record, FP64 oracle, one thread",
                           "s_per_record": ta, "records_per_s": 1.0 / ta,
                           "result": {k: ores[k] for k in ("verdict", "alpha", "vbar", "Z", "Ddiff", "dBIC")}}
        Dg = gpu_radial.D2()[sel]
        sc = np.where(ro["D"].max(axis=1) > 0, ro["D"].max(axis=1), 1)
        out["agreement"] = {"what": "GPU radial record vs this run's FP64 radial, sampled bins",
                            "bins": int(len(sel)),
                            "D_max_rel_to_bin_scale": float((np.abs(Dg - ro["D"]).max(axis=1) / sc).max()),
                            "P_max_rel": float(np.abs(gpu_radial.P[sel] / np.where(ro["P"] > 0, ro["P"], 1) - 1).max())}
    if one_core:
        os.environ["OMP_NUM_THREADS"] = "1"
        k = idx[:16]
        h1 = np.zeros((N * (N // 2 + 1), T), np.complex128)
        t0 = time.perf_counter()
        O.history_ingest(frames_u16[k].astype(np.float64) * (1.0 / 65535), k.astype(np.int32), T, hist=h1, smask=roi)
        sp1 = (time.perf_counter() - t0) / k.size
        del h1
        m1 = sub["binModes"][::16, 0].astype(np.int32)
        t0 = time.perf_counter()
        O.analyze_modes(hist, order, mask, L, m1, TPAD=TPAD, threads=1)
        tm1 = (time.perf_counter() - t0) / m1.size
        out["value_1core"] = 1.0 / (sp1 * idx.size / T + tm1 * nbinned / T)
        out["sample_1core"] = f"{k.size} frames + {m1.size} modes on one thread, scaled to the video"
        os.environ["OMP_NUM_THREADS"] = str(threads)
    del hist
    return out


# the motility analysis of the 512^2 x 1024 record: pixel/frame units; the
# reference's 2 um/s swimmer floor (GATES.SWIM_MIN_UM_S) is lowered to 0.1
# px/frame because this workload's mean swim speed, 1.5 px/frame, lies below it
MOTILITY_OPTS = dict(dxUm=1.0, fps=1.0, geometry="3d", swimMin=0.1)


def motility_benchmark(radial, truth, n_batch=48, reps=5):
    """analyzeMotility (motility_fit.js:870-990) on the video's radial
    record: every model fit on the GPU (csrc/gfit.cu), the statistics on the
    host. Wall-clock per call through the C ABI (host record in, result out):
    one record at a time, and n_batch records in one batched call (one launch
    per stage for all records)."""
    from hackathon_b200.motility import analyze_motility, analyze_motility_batch
    analyze_motility(radial, **MOTILITY_OPTS)  # context and 2D table set-up, outside the timing
    t = []
    res = None
    for _ in range(reps):
        t0 = time.perf_counter()
        res = analyze_motility(radial, **MOTILITY_OPTS)
        t.append(time.perf_counter() - t0)
    analyze_motility_batch([radial] * 2, **MOTILITY_OPTS)
    t0 = time.perf_counter()
    batch = analyze_motility_batch([radial] * n_batch, **MOTILITY_OPTS)
    tb = time.perf_counter() - t0
    same = all(b["alpha"] == res["alpha"] and b["vbar"] == res["vbar"] for b in batch)
    return {"what": "analyzeMotility of the video's radial record (Brownian, swimmer and drift fits of one "
                    "parameter set over all q-bins on the GPU; drift LSQ, BIC and gates on the host), "
                    "wall clock through the C ABI",
            "records_per_s": 1.0 / statistics.median(t), "ms_per_record": 1e3 * statistics.median(t),
            "batch": {"records": n_batch, "records_per_s": n_batch / tb, "equal_to_single": bool(same)},
            "options": MOTILITY_OPTS, "nbins": res["nbins"], "nlags": res["nlags"],
            "result": {k: res[k] for k in ("verdict", "alpha", "vbar", "Z", "Ddiff", "DdiffBrownian", "dBIC",
                                           "driftMag", "mu", "TSI")},
            "generator_truth": {"swimmer_share": 1 - truth["frac_brownian"], "vbar": truth["vbar"],
                                "Z": truth["Z"], "D": truth["D"]}}


# the surrogate's training videos: 512^2 x 1024, 1024 q-bins over the network's
# q range, until 2^19 pipeline curves (half of the 2^20-curve training set)
PIPELINE = dict(N=512, T=1024, NB=1024, kmin=4.0, kmax=60.0, max_curves=1 << 19)


def fit_benchmark(n_eval=100000, n_train=1 << 19, n_videos=2000, epochs=8, oracle_sample=256, pipeline=PIPELINE,
                  heldout_videos=24):
    """q-fits/s of the batched LM on held-out q-curves: plain (the reference's
    start strategy), surrogate-seeded, and surrogate-seeded with the plain
    strategy as fallback; the surrogate trained here on the GPU (analytic
    curves + the engine's own radial curves of seeded videos). Fit error:
    share of curves whose cost is within 1e-3 of the plain LM's (or lower),
    and, on a bounded sample, cost and parameter agreement with the FP64 LM
    oracle (reference start strategy, on the host)."""
    import torch
    from hackathon_b200 import surrogate_train as ST
    t0 = time.perf_counter()
    net = ST.build_and_train(n_analytic=n_train, n_videos=n_videos, epochs=epochs, seed=0, batch_max=8192,
                             pipeline=pipeline, log=lambda m: print(m, file=sys.stderr, flush=True))
    t_train = time.perf_counter() - t0
    held = ST.analytic_set(n_eval, seed=12345)
    bnds = ST.swim_bounds(held["qn"])
    summary, res = ST.compare_fits(net, held, bnds)
    # FP64 oracle on a bounded sample (host)
    import oracle as O
    d = held["d"].cpu().numpy().astype(np.float64)
    tau = ST.lm_tau().astype(np.float64)
    idx = np.arange(0, n_eval, n_eval // oracle_sample)[:oracle_sample]
    t1 = time.perf_counter()
    oc = np.array([O.lm_fit_plain(d[i], tau, held["qn"][i].astype(np.float64), 1 / d[i].max(),
                                  bnds.astype(np.float64))[1] for i in idx])
    t_or = time.perf_counter() - t1
    fb = res["fallback"]
    summary.update({
        "train_curves": int(n_train), "train_videos": int(n_videos), "train_s": t_train,
        "train_set": getattr(net, "train_info", None),
        "oracle_sample": int(len(idx)), "oracle_qfits_per_s_1core": len(idx) / t_or,
        # equal fit error: cost within 1e-3 of the FP64 oracle's, or lower
        "fallback_frac_equal_or_better_than_fp64_oracle": float((fb["cost"][idx] <= oc * (1 + 1e-3)).mean()),
        "seeded_frac_equal_or_better_than_fp64_oracle": float(
            (res["seeded"]["cost"][idx] <= oc * (1 + 1e-3)).mean()),
        "plain_frac_cost_within_1e-3_of_fp64_oracle": float(
            (np.abs(res["plain"]["cost"][idx] - oc) <= 1e-3 * oc).mean())})
    if heldout_videos:
        # held-out curves from the pipeline itself (fresh videos and seeds)
        hp = ST.pipeline_set(heldout_videos, 777, label="truth",
                             **{k: v for k, v in (pipeline or {}).items() if k != "max_curves"})
        ps, pres = ST.compare_fits(net, hp, ST.swim_bounds(hp["qn"]))
        summary["heldout_pipeline"] = {k: v for k, v in ps.items()}
    net.close()
    torch.cuda.synchronize()
    return summary


def run_reference(args, rank, world):
    if rank != 0:
        return
    import torch
    from hackathon_b200 import synth
    spec = synth.config2(seed=1)
    frames, valid, _ = synth.generate(spec, device="cuda" if torch.cuda.is_available() else "cpu")
    fr = frames.view(torch.int16).cpu().numpy().view(np.uint16)
    roi = synth.roi_mask(spec)
    del frames
    for _ in range(args.warmup):
        cpu_baseline(fr, valid, roi)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_baseline(fr, valid, roi))
    wall = time.perf_counter() - t0
    v = statistics.median(x["value"] for x in vals)
    line = {"metric": METRIC, "value": v, "unit": "frames/s", "impl": "reference", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": WORKLOAD},
            "cpu_baseline": {"value": v, "unit": "frames/s", "cores": vals[0]["cores"], "kind": "port",
                             "sample": vals[0]["sample"], "sample_mode_frac": vals[0]["sample_mode_frac"]},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference path is JavaScript (motility-ddm/src/ddm_ref.js, fft.js); no JS "
                    "runtime exists on this box, so its FP64 C restatement runs on the host cores; "
                    "each step is the same measurement as the GPU arm's cpu_baseline"}
    print(json.dumps(line), flush=True)


LARGE = dict(N=2048, T=4096, TPAD=8192, L=128, NB=1024, KMIN=4.0, KMAX=800.0)
LARGE_METRIC = "DDM frames/s at 2048²×4096 (large streamed run)"
LARGE_WORKLOAD = ("2048x2048x4096 u16 video: 40,000 blobs sigma 2 px with the 512x1024 workload's motility "
                  "statistics, 5% stuck pixels excluded by a pixel mask, Poisson noise mean 400 counts, 2% "
                  "dropped frames; TPAD=8192, L=128 lags, 1024 q-bins (kmin 4, kmax 800)")


def run_large(args, rank, world, dist, quiet=False):
    """The large streamed configuration: one 2048^2 x 4096 video per GPU
    (68.8 GB history). value: frames already in HBM; e2e: the frames streamed
    from host memory through the engine's pinned staging, radial read back.
    Full-size checks: fused radial == radial of the full per-mode outputs,
    D(q, 0) = 0, all finite."""
    import psutil
    import torch

    import hackathon_b200 as H
    from hackathon_b200 import replicas as R
    from hackathon_b200 import synth
    g = dict(LARGE)
    if args.roi:  # a smaller ROI, same q range per pixel and blob density (profiling)
        f = args.roi / g["N"]
        g.update(N=args.roi, KMAX=g["KMAX"] * f)
    if args.frames:  # a shorter video of the same frames (profiling, smoke runs)
        g["T"] = args.frames
        g["TPAD"] = max(128, 1 << (2 * args.frames - 1).bit_length())
    N, T, L, NB = g["N"], g["T"], g["L"], g["NB"]
    L = g["L"] = min(L, T)
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    spec = synth.large(seed=R.rank_seed(1, rank))
    spec.T = T
    if N != spec.N:
        spec.n_blobs = int(round(spec.n_blobs * (N / spec.N) ** 2))
        spec.N = N
    t_gen = time.perf_counter()
    frames, valid, _ = synth.generate(spec)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    slots = np.arange(T, dtype=np.int32)
    order = np.arange(T, dtype=np.uint32)
    tmask = valid.astype(np.float32)
    eng = H.DdmEngine.create(N=N, T=T, TPAD=g["TPAD"], L=L, NB=NB, kmin=g["KMIN"], kmax=g["KMAX"])
    eng.set_spatial_mask(synth.hot_mask(spec))
    tune = eng.autotune()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
    scale = 1.0 / 65535
    for _ in range(max(args.warmup, 3)):
        eng.ingest_frames(frames, slots, scale)
        eng.compute_temporal(order, tmask, full=False, wait=False)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    l0 = eng.kernel_launches
    ev = [tuple(torch.cuda.Event(enable_timing=True) for _ in range(3)) for _ in range(args.steps)]
    h0 = time.perf_counter()
    for i in range(args.steps):
        ev[i][0].record(stream)
        eng.ingest_frames(frames, slots, scale)
        ev[i][1].record(stream)
        eng.compute_temporal(order, tmask, full=False, wait=False)
        ev[i][2].record(stream)
    torch.cuda.synchronize()
    clocks.mark(h0, time.perf_counter())
    launches = eng.kernel_launches - l0
    clk = clocks.stop()
    ms = ev[0][0].elapsed_time(ev[-1][2])
    t_sp = statistics.mean(a.elapsed_time(b) for a, b, _ in ev)
    t_tm = statistics.mean(b.elapsed_time(c) for _, b, c in ev)
    ms_step = R.max_over_ranks(ms, dist, device="cuda") / args.steps
    value = R.weak_scaling_throughput(T, ms_step, world)
    fused = eng.read_radial()
    fused_bins = eng.bins
    large_tk = eng.last_temporal_kernel

    # full-size consistency: the full-output path's radial equals the fused one
    eng.compute_temporal(order, tmask, full=True)
    full = eng.read_radial()
    D1, D2 = fused.D2(), full.D2()
    sc = np.abs(D1).max(axis=1, keepdims=True)
    checks = {"finite": bool(np.isfinite(D1).all() and np.isfinite(fused.P).all() and np.isfinite(fused.drift).all()),
              "fused_vs_full_D_max_rel": float((np.abs(D1 - D2) / np.where(sc > 0, sc, 1)).max()),
              "fused_vs_full_P_max_rel": float(np.abs(fused.P / np.where(full.P > 0, full.P, 1) - 1)[full.P > 0].max()),
              "D0_max_rel": float((np.abs(D1[:, 0:1]) / np.where(sc > 0, sc, 1)).max())}

    # e2e from host memory: the whole video in pageable host memory when it
    # fits, streamed by the engine's pinned staging (frames -> HBM) each step
    need = frames.numel() * 2
    avail = psutil.virtual_memory().available
    e2e = None
    if args.e2e_steps > 0 and avail > 1.5 * need:
        host = frames.view(torch.int16).cpu()
        pinned = avail > 3 * need
        if pinned:  # page-locked: the copies run at the link's rate
            host = host.pin_memory()
        rad_bytes = 8 * (NB * L + NB + NB * L * 8)
        eng.ingest_frames(host[:64], slots[:64], scale)  # staging warm
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.e2e_steps):
            eng.ingest_frames(host, slots, scale)
            eng.compute_temporal(order, tmask, full=False, wait=False)
            eng.read_radial()
        e1.record(stream)
        torch.cuda.synchronize()
        ms_e2e = R.max_over_ranks(e0.elapsed_time(e1), dist, device="cuda")
        e2e = {"value": R.weak_scaling_throughput(T * args.e2e_steps, ms_e2e, world), "unit": "frames/s",
               "h2d_bytes_per_step": int(need), "d2h_bytes_per_step": rad_bytes,
               "host_memory": "pinned" if pinned else "pageable, staged through the engine's pinned ring"}
        banded = None
        if args.band_budget_gb > 0:
            # the same video with the history held one band of spectrum columns
            # at a time, sized to the stated budget: per band the frames
            # stream from host memory through the spatial pass again
            eng.destroy()
            eng = None
            torch.cuda.empty_cache()
            budget = int(args.band_budget_gb * 2**30)
            beng = H.DdmEngine.create_banded(budget, N=N, T=T, TPAD=g["TPAD"], L=L, NB=NB, kmin=g["KMIN"],
                                             kmax=g["KMAX"])
            beng.set_spatial_mask(synth.hot_mask(spec))
            beng.set_tuning(tune["best_chunk"], tune["best_unit"], tune["best_variant"])
            beng.set_stream(stream.cuda_stream)
            nbands, bcols = beng.bands
            beng.analyze_banded(host, slots, order, tmask, scale)  # warm
            torch.cuda.synchronize()
            b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            b0.record(stream)
            beng.analyze_banded(host, slots, order, tmask, scale)
            b1.record(stream)
            torch.cuda.synchronize()
            ms_b = R.max_over_ranks(b0.elapsed_time(b1), dist, device="cuda")
            rb = beng.read_radial()
            Db = rb.D2()
            banded = {"what": "the history held one band of spectrum columns at a time (ddm_create_banded), "
                              "the frames streamed from host memory through the spatial pass once per band",
                      "history_budget_bytes": budget, "bands": nbands, "band_columns": bcols,
                      "history_bytes_on_device": int(bcols) * N * T * 8,
                      "value": R.weak_scaling_throughput(T, ms_b, world), "unit": "frames/s",
                      "ms_per_video": ms_b, "h2d_bytes_per_step": int(need) * nbands,
                      "host_memory": "pinned" if pinned else "pageable",
                      "checks": {"banded_vs_resident_D_max_rel": float(
                          (np.abs(Db - D1) / np.where(sc > 0, sc, 1)).max()),
                                 "banded_vs_resident_P_max_rel": float(
                          np.abs(rb.P / np.where(fused.P > 0, fused.P, 1) - 1)[fused.P > 0].max())}}
            beng.destroy()
        e2e["banded"] = banded
        del host
    else:
        e2e = {"value": None, "unit": "frames/s",
               "unavailable": "no e2e steps requested" if args.e2e_steps <= 0 else
               f"host memory {avail / 2**30:.0f} GiB < 1.5 x video"}

    peak, peak_kind = _peaks()
    nbinned = int(fused_bins["binOffsets"][-1])
    sp_bytes = T * (N * N * 2 + N * (N // 2 + 1) * BYTES_PER_MODE_SLOT)
    tm_bytes = nbinned * T * BYTES_PER_MODE_SLOT
    TP = g["TPAD"]
    tk = large_tk  # 1.5 transforms per mode for the sparse-mask kernels, else 2.5
    per_mode = 1.5 if tk in ("temporal_sparse_kernel", "temporal_sparse_big_kernel") else 2.5
    tm_flop = nbinned * per_mode * 5 * TP * np.log2(TP)
    if tk == "temporal_blocked_kernel":
        # 256-point transforms: one per 128-sample block of x, one per two
        # blocks of p, two inverse transforms
        nblk = -(-T // 128)
        tm_flop = nbinned * (nblk + -(-nblk // 2) + 2) * 5 * 256 * 8
    stages = {"spatial": {"ms": t_sp, "bytes": sp_bytes, "GBps": sp_bytes / (t_sp * 1e6),
                          "gflop": T * (N + 1) * 5 * N * np.log2(N) / 1e9},
              "temporal": {"ms": t_tm, "bytes": tm_bytes, "GBps": tm_bytes / (t_tm * 1e6), "kernel": tk,
                           "gflop": tm_flop / 1e9}}
    for s in stages.values():
        s["frac"] = s["GBps"] / peak
        s["fp32_frac_of_nominal"] = s["gflop"] / s["ms"] / FP32_NOMINAL_TFLOPS
    tm = stages["temporal"]
    roof = {"bound": "hbm", "kernel": tk, "achieved": tm["GBps"], "peak": peak, "unit": "GB/s",
            "frac": tm["frac"], "peak_source": peak_kind, "traffic": None, "algorithmic_bytes": tm_bytes,
            "stages": stages}
    line = None
    if rank == 0:
        metric = LARGE_METRIC if (N, T) == (LARGE["N"], LARGE["T"]) else \
            f"DDM frames/s at {N}²×{T} (large streamed run, reduced)"
        line = {"metric": metric, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded GPU generator, hackathon_b200/synth.py large())",
                "config": {"workload": LARGE_WORKLOAD, **{k.lower(): v for k, v in g.items()},
                           "binned_modes": nbinned, "history_bytes": N * (N // 2 + 1) * T * 8,
                           "l2": "inputs larger than L2", "generation_s": t_gen,
                           "autotuned": {"chunk": tune["best_chunk"], "unit": tune["best_unit"],
                                         "temporal_variant": tune["best_variant"]}},
                "e2e": e2e, "gpu_launches": int(launches), "roofline": roof, "clocks": clk, "checks": checks}
        if not quiet:
            print(json.dumps(line), flush=True)
    if eng is not None:
        eng.destroy()
    return line


BATCH_METRIC = "DDM frames/s, 48 uneven videos in one persistent launch"
BATCH_WORKLOAD = ("48 seeded u16 videos, N in {256, 384, 512, 768}, "
                  "T uniform in [300, 2000], per-video motile fraction in [0, 0.9], mean speed in [0.3, 3] "
                  "px/frame, D in [0.05, 0.5] px^2/frame, circular ROI of random radius, 2% dropped frames; "
                  "L = min(512, T/2), NB = N/4, kmin 4, kmax 0.39 N; one batched ingest + ONE temporal launch "
                  "over all videos, replayed from a CUDA graph; all q-bins of all videos in one LM launch")


def run_batch(args, rank, world, dist):
    """The batched-videos configuration: every video's spatial chunks and one
    persistent temporal launch over the work units of all videos, captured
    once into a CUDA graph and replayed (value), then all q-bins of all
    videos fitted by one batched LM launch (q-fits/s). Tile shapes come from
    the autotuner (one engine of each size, applied to the others)."""
    import torch

    import hackathon_b200 as H
    from hackathon_b200 import fit as F
    from hackathon_b200 import replicas as R
    from hackathon_b200 import synth
    from hackathon_b200.batch import DdmBatch
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    rng = np.random.default_rng(R.rank_seed(7, rank))
    nvid = args.videos or 48
    vids, engines, tuned = [], [], {}
    t_gen = time.perf_counter()
    for i in range(nvid):
        N = int(rng.choice([256, 384, 512, 768]))
        T = int(rng.integers(300, 2001)) // 2 * 2
        al, vb, Dd = rng.uniform(0, 0.9), rng.uniform(0.3, 3.0), rng.uniform(0.05, 0.5)
        spec = synth.VideoSpec(N=N, T=T, n_blobs=int(2000 * (N / 512) ** 2), frac_brownian=1 - al, D=Dd, vbar=vb,
                               roi_radius=float(rng.uniform(0.30, 0.48)) * N, drop_frac=0.02,
                               seed=int(R.rank_seed(1000, rank) * 100 + i))
        frames, valid, _ = synth.generate(spec)
        L, NB = min(512, T // 2), N // 4
        e = H.DdmEngine.create(N=N, T=T, L=L, NB=NB, kmin=4.0, kmax=0.39 * N)
        e.set_spatial_mask(synth.roi_mask(spec))
        if N not in tuned:
            tuned[N] = e.autotune()
        else:
            t = tuned[N]
            e.set_tuning(t["best_chunk"], t["best_unit"], t["best_variant"])
        vids.append(dict(frames=frames.contiguous(), valid=valid, T=T, N=N))
        engines.append(e)
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t_gen
    total = sum(v["T"] for v in vids)
    slots = [np.arange(v["T"], dtype=np.int32) for v in vids]
    orders = [np.arange(v["T"], dtype=np.uint32) for v in vids]
    masks = [v["valid"].astype(np.float32) for v in vids]
    scales = [1.0 / 65535] * nvid
    frames = [v["frames"] for v in vids]
    batch = DdmBatch(engines)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    batch.set_stream(stream.cuda_stream)
    batch.ingest(frames, slots, scales)
    batch.compute_temporal(orders, masks)  # per-video tables, then the launch
    batch.sync()
    l0 = sum(e.kernel_launches for e in engines)
    batch.ingest(frames, slots, scales)    # one step outside the graph: its launch count
    batch.enqueue_temporal()
    batch.sync()
    per_step = sum(e.kernel_launches for e in engines) - l0
    batch.capture(frames, slots, scales)   # ingest + temporal of all videos as one graph
    for _ in range(max(args.warmup, 3)):
        batch.launch_graph()
    batch.sync()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    steps = max(1, min(args.steps, 10))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    h0 = time.perf_counter()
    e0.record(stream)
    for _ in range(steps):
        batch.launch_graph()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks.mark(h0, time.perf_counter())
    clk = clocks.stop()
    ms_step = R.max_over_ranks(e0.elapsed_time(e1), dist, device="cuda") / steps
    value = R.weak_scaling_throughput(total, ms_step, world)
    radials = batch.read_radials()
    # all q-bins of all videos: one LM launch (host arrays in and out)
    torch.cuda.synchronize()
    f0 = time.perf_counter()
    fits = batch.fit_all(radials, swim_min=0.0)
    f_s = time.perf_counter() - f0
    nfit = sum(len(p.bins) for p, _ in fits)
    finite = all(np.isfinite(r.cost).all() for _, r in fits)
    if rank == 0:
        line = {"metric": BATCH_METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": steps,
                "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded GPU generator, hackathon_b200/synth.py)",
                "config": {"workload": BATCH_WORKLOAD, "videos": nvid, "frames_per_step": total,
                           "sizes": {str(n): sum(v["N"] == n for v in vids) for n in (256, 384, 512, 768)},
                           "l2": "inputs larger than L2", "generation_s": t_gen,
                           "temporal_kernel": engines[0].last_temporal_kernel,
                           "autotuned": {str(n): {k: t[k] for k in ("best_chunk", "best_unit", "best_variant")}
                                         for n, t in tuned.items()}},
                "e2e": {"value": None, "unit": "frames/s",
                        "unavailable": "the batched ingest takes frames already on the device"},
                "gpu_launches": int(per_step * steps), "clocks": clk,
                "fit": {"qfits": nfit, "one_launch_s_host_timed": f_s, "qfits_per_s": nfit / f_s,
                        "all_finite": bool(finite)}}
        print(json.dumps(line), flush=True)
    batch.destroy()
    for e in engines:
        e.destroy()



SURROGATE_METRIC = "q-fits/s learned+LM vs plain LM at equal fit error (surrogate trained on 2^20 curves)"


def run_surrogate(args, rank, world, dist):
    """The learned-surrogate configuration at its stated size: the network is
    trained on the GPU on 2^20 curves, 2^19 analytic model curves with 1 %
    noise and 2^19 radial curves the engine itself produces from seeded
    512^2 x 1024 videos (1024 q-bins over the network's q range, each video
    labelled with its generator's parameters), then evaluated as the LM's
    initial guess against plain LM on 10^5 held-out analytic curves and on
    held-out pipeline curves of fresh videos."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    half = 1 << 19
    pipe = PIPELINE
    t0 = time.perf_counter()
    fit = fit_benchmark(n_train=half, n_videos=args.videos or 2000, pipeline=pipe, heldout_videos=24)
    if rank == 0:
        line = {"metric": SURROGATE_METRIC, "value": fit["seeded_qfits_per_s"], "unit": "q-fits/s",
                "n_gpus": 1, "higher_is_better": True, "dtype": "bf16 network, f32/f64 LM",
                "data": "synthetic (analytic model curves + the engine's radial curves of seeded videos)",
                "config": {"workload": "surrogate: 2^19 analytic + 2^19 pipeline training curves "
                                       "(512^2 x 1024 videos, 1024 q-bins, k in [4, 60]); 10^5 held-out analytic "
                                       "curves + held-out pipeline curves of 24 fresh videos",
                           "pipeline": {k: v for k, v in pipe.items()}},
                "vs_baseline": None, "total_s": time.perf_counter() - t0, "fit": fit}
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=12)
    ap.add_argument("--no-fit", action="store_true", help="skip the q-fits/s (surrogate + LM) section")
    ap.add_argument("--tuning", default="", help="chunk,unit[,variant]: apply instead of autotuning")
    ap.add_argument("--workload", default="config2", choices=["config2", "large", "batch", "surrogate"],
                    help="large: one 2048^2 x 4096 video per GPU (68.8 GB history), its own JSON line")
    ap.add_argument("--frames", type=int, default=0, help="large workload: frames per video (default 4096)")
    ap.add_argument("--band-budget-gb", type=float, default=24.0,
                    help="large workload: device history budget of the banded streamed run (0: skip it)")
    ap.add_argument("--no-large", action="store_true",
                    help="skip the large streamed run nested in the 512^2 x 1024 line")
    ap.add_argument("--roi", type=int, default=0, help="large workload: ROI size (default 2048)")
    ap.add_argument("--videos", type=int, default=0,
                    help="batch workload: number of videos (48); surrogate: cap on pipeline videos (2000)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "ours" and args.workload in ("large", "batch", "surrogate"):
        {"large": run_large, "batch": run_batch, "surrogate": run_surrogate}[args.workload](args, rank, world, dist)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    import hackathon_b200 as H
    from hackathon_b200 import synth

    from hackathon_b200 import replicas as R
    torch.cuda.set_device(local)
    spec = synth.config2(seed=R.rank_seed(1, rank))
    frames, valid, truth = synth.generate(spec)
    mask_roi = synth.roi_mask(spec)
    slots = np.arange(T, dtype=np.int32)
    order = np.arange(T, dtype=np.uint32)
    tmask = valid.astype(np.float32)
    eng = H.DdmEngine.create(N=N, T=T, TPAD=TPAD, L=L, NB=NB, kmin=KMIN, kmax=KMAX)
    eng.set_spatial_mask(mask_roi)
    if args.tuning:  # a cached autotune result "chunk,unit[,variant]"
        vals = [int(x) for x in args.tuning.split(",")]
        c, u, var = (vals + [0])[:3]
        eng.set_tuning(c, u, var)
        tune = {"best_chunk": c, "best_unit": u, "best_variant": var}
    else:
        tune = eng.autotune()  # set-up, outside the timed region
    # a dedicated stream: the engine queues its kernels there and the CUDA
    # events below are recorded on the same stream
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    assert stream.cuda_stream != 0
    eng.set_stream(stream.cuda_stream)
    scale = 1.0 / 65535

    def step():
        eng.ingest_frames(frames, slots, scale)
        eng.compute_temporal(order, tmask, full=False, wait=False)

    # stage timing events (spatial, temporal) inside the timed region
    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)  # sampler running before the timed region
    l0 = eng.kernel_launches
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    torch.cuda.synchronize()
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    h0 = time.perf_counter()
    start.record(stream)
    for i in range(args.steps):
        ev[i][0].record(stream)
        eng.ingest_frames(frames, slots, scale)
        ev[i][1].record(stream)
        eng.compute_temporal(order, tmask, full=False, wait=False)
        ev[i][2].record(stream)
    end.record(stream)
    torch.cuda.synchronize()
    clocks.mark(h0, time.perf_counter())
    if dist:
        dist.barrier()
    launches = eng.kernel_launches - l0
    clk = clocks.stop()
    ms = start.elapsed_time(end)
    t_sp = statistics.mean(a.elapsed_time(b) for a, b, _ in ev)
    t_tm = statistics.mean(b.elapsed_time(c) for _, b, c in ev)
    ms = R.max_over_ranks(ms, dist, device="cuda")
    ms_step = ms / args.steps
    value = R.weak_scaling_throughput(T, ms_step, world)

    # ---------------- e2e: pinned host frames through the C ABI. Three
    # engines take videos in turn (a user with a stream of videos): while one
    # video's temporal analysis runs, the next video's frames already cross
    # PCIe into the next engine; every video's radial record is read back,
    # two videos behind the ingest, so the host's reads and queueing never
    # wait on an analysis that is still running. (Measured on one B200 at
    # 512^2 x 1024: two engines 94.7-96.3K frames/s, three 101.2K; no faster:
    # two host threads, one per engine; ddm_ingest_frames_async with the
    # host's set-up overlapping the copies; four staging buffers instead of
    # two.)
    host = frames.view(torch.int16).cpu().pin_memory()
    rad_bytes = 8 * (NB * L + NB + NB * L * 8)
    eng.set_stream(stream.cuda_stream)
    engs, e2e_streams = [eng], [stream]
    for _ in range(E2E_ENGINES - 1):
        ex = H.DdmEngine.create(N=N, T=T, TPAD=TPAD, L=L, NB=NB, kmin=KMIN, kmax=KMAX)
        ex.set_spatial_mask(mask_roi)
        ex.set_tuning(tune["best_chunk"], tune["best_unit"], tune["best_variant"])
        sx = torch.cuda.Stream()
        ex.set_stream(sx.cuda_stream)
        engs.append(ex)
        e2e_streams.append(sx)

    # the radial records come back into pinned host buffers reused across
    # videos (read_radial(out=...)): 9.4 MB at the link's rate, 0.2 ms
    # against 0.64 ms through the pageable path, during which the link idles
    rad_out = [torch.empty(n, dtype=torch.float64).pin_memory().numpy() for n in (NB * L, NB, NB * L * 8)]

    def e2e_run(n):
        pending, radial = [], None
        for i in range(n):
            x = engs[i % len(engs)]
            x.ingest_frames(host, slots, scale)
            x.compute_temporal(order, tmask, full=False, wait=False)
            pending.append(x)
            if len(pending) == len(engs):  # the engine the next video goes to
                radial = pending.pop(0).read_radial(out=rad_out)
        while pending:
            radial = pending.pop(0).read_radial(out=rad_out)
        return radial

    e2e_run(E2E_ENGINES)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for sx in e2e_streams[1:]:
        sx.wait_stream(stream)
    radial = e2e_run(args.e2e_steps)
    for sx in e2e_streams[1:]:
        stream.wait_stream(sx)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e0.elapsed_time(e1)
    for ex in engs[1:]:
        ex.destroy()
    ms_e2e = R.max_over_ranks(ms_e2e, dist, device="cuda")
    e2e = R.weak_scaling_throughput(T * args.e2e_steps, ms_e2e, world)
    # the link's ceiling for context: one plain pinned host->device copy of a video
    dev_copy = torch.empty_like(host, device="cuda")
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    dev_copy.copy_(host, non_blocking=True)
    torch.cuda.synchronize()
    c0.record(stream)
    dev_copy.copy_(host, non_blocking=True)
    c1.record(stream)
    torch.cuda.synchronize()
    h2d_gbps = host.numel() * 2 / (c0.elapsed_time(c1) * 1e6)
    del dev_copy

    # ---------------- roofline of the dominant stage
    peak, peak_kind = _peaks()
    nbinned = int(eng.bins["binOffsets"][-1])
    modes = eng.modes
    sp_bytes = T * (BYTES_PER_FRAME_IN + modes * BYTES_PER_MODE_SLOT)  # read frames, write history
    tm_bytes = nbinned * T * BYTES_PER_MODE_SLOT                       # read binned series
    stages = {
        "spatial": {"ms": t_sp, "bytes": sp_bytes, "GBps": sp_bytes / (t_sp * 1e6)},
        "temporal": {"ms": t_tm, "bytes": tm_bytes, "GBps": tm_bytes / (t_tm * 1e6)},
    }
    for s in stages.values():
        s["frac"] = s["GBps"] / peak
    # FP32 work, 5 n log2 n per complex FFT of n points
    fl_sp = T * (N // 2 + N // 2 + 1) * 5 * N * np.log2(N)
    # transforms per mode of the kernel that ran: 2.5 (masked WK by
    # transforms), 1.5 (sparse-mask kernel: A + B from prefix sums)
    tk = eng.last_temporal_kernel
    fl_tm = nbinned * (1.5 if tk == "temporal_sparse_kernel" else 2.5) * 5 * TPAD * np.log2(TPAD)
    stages["spatial"]["gflop"] = fl_sp / 1e9
    stages["temporal"]["gflop"] = fl_tm / 1e9
    stages["temporal"]["kernel"] = tk
    # a library reference point for the temporal stage's transform work:
    # cuFFT (torch.fft) running just the same number of TPAD-point complex
    # transforms over device-resident series (one forward per mode from T
    # samples, plus the inverse transforms: one per mode pair for the
    # sparse-mask kernel, 1.5 per mode for the transform kernels), with none
    # of the masked Wiener-Khinchin arithmetic or the radial epilogue
    lib = None
    try:
        x = torch.randn((nbinned, T), dtype=torch.complex64, device="cuda")
        n_inv = nbinned // 2 if tk == "temporal_sparse_kernel" else (3 * nbinned) // 2
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        times = []
        for r in range(4):
            torch.cuda.synchronize()
            f0.record()
            y = torch.fft.fft(x, n=TPAD, dim=1)
            z = torch.fft.ifft(y[:n_inv] if n_inv <= nbinned else torch.cat([y, y[:n_inv - nbinned]]), dim=1)
            f1.record()
            torch.cuda.synchronize()
            if r:
                times.append(f0.elapsed_time(f1))
            del y, z
        lib = {"temporal": {"what": f"torch.fft (cuFFT): {nbinned} forward + {n_inv} inverse {TPAD}-point C2C "
                                    "transforms, device-resident, no other work",
                            "ms": statistics.median(times)}}
        if T == 1024 and TPAD == 2048:
            # the forward transforms alone on the tensor cores (ddm_dft2048_tc,
            # BF16 three-term split) against cuFFT's forward transforms alone
            import ctypes
            from hackathon_b200 import _lib as LIB
            lib_so = LIB.load()
            X = torch.empty((nbinned, TPAD), dtype=torch.complex64, device="cuda")
            tf, tt = [], []
            for r in range(4):
                torch.cuda.synchronize()
                f0.record()
                y = torch.fft.fft(x, n=TPAD, dim=1)
                f1.record()
                torch.cuda.synchronize()
                if r:
                    tf.append(f0.elapsed_time(f1))
                f0.record()
                rc = lib_so.ddm_dft2048_tc(ctypes.c_void_p(x.data_ptr()), T, nbinned, ctypes.c_void_p(X.data_ptr()),
                                           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
                f1.record()
                torch.cuda.synchronize()
                if rc:
                    raise RuntimeError(lib_so.ddm_create_error().decode())
                if r:
                    tt.append(f0.elapsed_time(f1))
            s64 = slice(0, 64)
            rms = torch.sqrt(torch.mean(torch.abs(y[s64]) ** 2, dim=1))
            err = float((torch.abs(X[s64] - y[s64]).max(dim=1).values / rms).max())
            lib["tensor_core_forward"] = {
                "what": f"{nbinned} forward {TPAD}-point transforms of {T} samples, FP32 in and out: tcgen05 "
                        "four-step DFT (BF16 three-term split) against cuFFT",
                "tcgen05_ms": statistics.median(tt), "cufft_ms": statistics.median(tf),
                "max_err_vs_cufft_of_rms": err}
            del X, y
        del x
        # and the spatial stage's: a 2D real-to-half-plane FFT of every frame
        # already in FP32 (no conversion, window, mean or transposed store)
        x = torch.randn((T, N, N), dtype=torch.float32, device="cuda")
        times = []
        for r in range(4):
            torch.cuda.synchronize()
            f0.record()
            y = torch.fft.rfft2(x)
            f1.record()
            torch.cuda.synchronize()
            if r:
                times.append(f0.elapsed_time(f1))
            del y
        lib["spatial"] = {"what": f"torch.fft.rfft2 (cuFFT) of {T} FP32 {N}x{N} frames, device-resident, no other work",
                          "ms": statistics.median(times)}
        del x
    except RuntimeError as e:  # e.g. out of memory on a shared device
        lib = {"unavailable": str(e)[:120]}
    # dominant kernel: the temporal kernel (one launch per step, the largest
    # single kernel; the spatial stage is 3 kernels x 16 chunk launches)
    traffic = _profile_traffic() or {}
    tm = stages["temporal"]
    roof = {"bound": "hbm", "kernel": tk, "achieved": tm["GBps"], "peak": peak,
            "unit": "GB/s", "frac": tm["frac"], "peak_source": peak_kind,
            "traffic": traffic.get(f"{tk}_bytes_per_launch"),
            "algorithmic_bytes": tm["bytes"],
            "timed_span": f"temporal stage on the engine stream: meta upload + {tk} + reduce_kernel",
            "fp32_tflops": tm["gflop"] / tm["ms"], "fp32_frac_of_nominal": tm["gflop"] / tm["ms"] / FP32_NOMINAL_TFLOPS,
            "library_fft_reference": lib,
            "pipeline_GBps": (sp_bytes + tm_bytes) / (ms_step * 1e6),
            "pipeline_frac": (sp_bytes + tm_bytes) / (ms_step * 1e6) / peak,
            "stages": stages}

    # full-size checks on this video (outside the timed regions): the fused
    # radial record equals the record of the full per-mode outputs, D(q, 0) = 0,
    # everything finite; the CPU baseline below adds the FP64 comparison
    eng.compute_temporal(order, tmask, full=False)
    fused = eng.read_radial()
    eng.compute_temporal(order, tmask, full=True)
    fullr = eng.read_radial()
    D1, D2 = fused.D2(), fullr.D2()
    sc = np.abs(D1).max(axis=1, keepdims=True)
    checks = {"finite": bool(np.isfinite(D1).all() and np.isfinite(fused.P).all() and np.isfinite(fused.drift).all()),
              "fused_vs_full_D_max_rel": float((np.abs(D1 - D2) / np.where(sc > 0, sc, 1)).max()),
              "fused_vs_full_P_max_rel": float(np.abs(fused.P / np.where(fullr.P > 0, fullr.P, 1) - 1)[fullr.P > 0].max()),
              "D0_max_rel": float((np.abs(D1[:, 0:1]) / np.where(sc > 0, sc, 1)).max()),
              "kernel": eng.last_temporal_kernel}
    del fullr

    motility = motility_benchmark(fused, truth) if rank == 0 else None

    fit = None
    if rank == 0 and not args.no_fit:
        fit = fit_benchmark()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        fr = frames.view(torch.int16).cpu().numpy().view(np.uint16)
        cpu = cpu_baseline(fr, valid, mask_roi, gpu_radial=radial, one_core=True, reps=3)

    # the large streamed configuration (2048^2 x 4096, resident and banded),
    # summarised in this line so that one run records both workloads
    large = None
    eng.destroy()
    eng = None
    if rank == 0 and world == 1 and not args.no_large:
        del frames
        torch.cuda.empty_cache()
        la = argparse.Namespace(**vars(args))
        la.steps, la.warmup, la.e2e_steps = 2, 3, 1
        try:
            ll = run_large(la, 0, 1, None, quiet=True)
            large = {k: ll[k] for k in ("metric", "value", "unit", "ms_per_step", "e2e", "checks", "clocks",
                                        "gpu_launches")}
            large["roofline"] = {k: ll["roofline"][k] for k in ("kernel", "achieved", "peak", "frac", "unit")}
            large["stages"] = {k: {"ms": v["ms"], "frac": v["frac"]} for k, v in ll["roofline"]["stages"].items()}
            large["config"] = {k: ll["config"][k] for k in ("workload", "history_bytes", "binned_modes",
                                                            "generation_s")}
        except Exception as e:  # e.g. too little host memory for the pinned video
            large = {"unavailable": f"{type(e).__name__}: {str(e)[:200]}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded GPU generator, hackathon_b200/synth.py)",
                "config": {"workload": WORKLOAD, "N": N, "T": T, "TPAD": TPAD, "L": L, "NB": NB,
                           "frames_dtype": "u16", "parallelism": f"replicas x{world} (one video per GPU)",
                           "l2": "inputs larger than L2 (537 MB frames, 1.08 GB history per video)",
                           "autotuned": {"chunk": tune["best_chunk"], "unit": tune["best_unit"],
                                         "temporal_variant": tune["best_variant"]}},
                "e2e": {"value": e2e, "unit": "frames/s", "pipeline": f"{E2E_ENGINES} engines take videos in turn",
                        "h2d_GBps": host.numel() * 2 * args.e2e_steps / (ms_e2e * 1e6),
                        "h2d_GBps_plain_copy": h2d_gbps,
                        "h2d_bytes_per_step": int(host.numel() * 2),
                        "d2h_bytes_per_step": rad_bytes},
                "gpu_launches": int(launches),
                "roofline": roof,
                "clocks": clk,
                "cpu_baseline": cpu,
                "checks": checks,
                "motility": motility,
                "large": large,
                "binned_modes": nbinned,
                "fit": fit}
        print(json.dumps(line), flush=True)
    if eng is not None:
        eng.destroy()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
