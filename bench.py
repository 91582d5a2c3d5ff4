#!/usr/bin/env python
"""Benchmark of one EMC iteration (expand -> maximize -> compress).

A step is one iteration -- maximize (slices, E-step with pruning, per-frame
normalisation, M-step, merge, scale update) + update_model + normalize_scale,
launched as one CUDA graph (dfg_run_iteration) -- on the production-size plain
workload:

  260 x 257 flat pnCCD-like detector, 6-row panel gap (rows 127-132), radius-10
  central hole; 201^3 model from 2000 Gaussian atoms in a radius-30 sphere;
  num_div = 10 (50100 orientations); 200000 frames with lognormal fluence
  (median 300 photons, sigma 0.5); scale update on; beta from 0.01, x sqrt(2)
  every 5 iterations, capped at 1.

Data are seeded synthetic inputs of that shape (no dataset is involved);
frames are simulated on the GPU by the library. Every input (frames, log-slices,
per-pair buffers) is far larger than the 126 MB L2, so no flush is needed
between iterations.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's own CPU engine (dragonfly/src compiled
into oracle/_ref) on the host cores, on a bounded frame sample of the same
workload. With N > 1 each rank runs an independent replica (the iteration
needs no collective); rank 0 prints the JSON line.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(name="plain EMC: 260x257 pnCCD-like detector, 201^3 model, 50100 orientations, "
                     "200000 frames, median 300 photons, scale update, beta 0.01 x sqrt2 / 5",
                det=(260, 257), gap_rows=list(range(127, 133)), hole=10., size=201, qmax=100.,
                n_atoms=2000, atom_radius=30., num_div=10, n_frames=200000, median_photons=300.,
                fluence_sigma=0.5, beta=0.01, beta_jump=math.sqrt(2.), beta_period=5)
METRIC = "frame x orientation pairs per second of one plain EMC iteration"
UNIT = "pairs/s"


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------
def build_inputs(w, seed=1234):
    """Host-side inputs: detector, intensity model, orientations, per-frame
    orientations and fluence, start model."""
    from dragonfly_b200 import synth
    from dragonfly_b200.quatgen import quat_gen
    rng = np.random.default_rng(seed)
    intens = synth.gaussian_atom_intensity(w["n_atoms"], w["atom_radius"], w["size"], rng)
    qvals, corr, mask, detd, ewald = synth.flat_detector(w["det"][0], w["det"][1], w["qmax"], w["size"],
                                                         hole_radius=w["hole"], gap_rows=w["gap_rows"])
    intens *= w["median_photons"] / synth.model_mean_count(intens, qvals, corr, mask, rng, n_orient=48)
    quats = quat_gen(w["num_div"])
    n = w["n_frames"]
    frame_q = synth.random_quaternions(n, rng)
    phi = np.exp(rng.normal(0., w["fluence_sigma"], n))
    model_mean = w["median_photons"] * math.exp(w["fluence_sigma"] ** 2 / 2) / (mask == 0).sum() * 2.
    start = rng.random((1,) + (w["size"],) * 3) * model_mean
    return dict(qvals=qvals, corr=corr, mask=mask, intens=intens, quats=quats, frame_q=frame_q, phi=phi,
                start=start)


def clock_sampler(device_index):
    """Starts nvidia-smi sampling clocks every 200 ms; returns (proc, path)."""
    fd, path = tempfile.mkstemp(suffix=".csv")
    os.close(fd)
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    try:
        proc = subprocess.Popen(["nvidia-smi", "--id=%d" % device_index, "--query-gpu=" + q,
                                 "--format=csv,noheader,nounits", "-lms", "200"],
                                stdout=open(path, "w"), stderr=subprocess.DEVNULL)
    except OSError:
        proc = None
    return proc, path


def clock_summary(proc, path):
    if proc is None:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
    proc.terminate()
    proc.wait()
    sm, smax, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for ln in open(path):
        f = [x.strip() for x in ln.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            smax.append(float(f[2]))
        except ValueError:
            continue
        for k, v in zip(names, f[5:9]):
            if v.lower().startswith("active"):
                reasons.add(k)
    os.unlink(path)
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p["hbm_gbs"], "of measured"
    except Exception:
        return 6650., "of fallback"


# DRAM bytes of one launch of the gather kernels, as fractions of their
# compulsory streams, from ncu captures of the 3240-orientation x 8000-frame
# case (dram__bytes_read.sum + dram__bytes_write.sum): the row gathers
# themselves are served by L2 (95 % hit), so DRAM traffic follows the streams
# below and not the number of gathers.
#   E-step: reads 0.85 of the tile's log-slices, writes 0.97 of the log-likelihoods
#   M-step: reads 0.85 of tomograms + probability rows, writes 0.72 of tomograms
TRAFFIC_FRACTIONS = {"estep": (0.85, 0.97), "mstep": (0.85, 0.72)}


def measured_tensor_peak():
    """Measured sustained dense BF16 rate (TFLOP/s) for a kernel timed inside a
    long step, else the fallback figure."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops_sustained"]), "of measured (sustained)"
    except (OSError, KeyError, ValueError):
        return 1400., "of fallback (sustained)"


def roofline_traffic(kernel, R_pad, P, Nc):
    """Modelled DRAM bytes of one launch of `kernel` (None for other kernels)."""
    if kernel == "estep":
        rd, wr = TRAFFIC_FRACTIONS["estep"]
        return rd * 4. * R_pad * (P + 1) + wr * 8. * R_pad * Nc
    if kernel == "mstep":
        rd, wr = TRAFFIC_FRACTIONS["mstep"]
        tomo = 4. * R_pad * P
        return rd * (tomo + 4. * R_pad * (Nc + 1)) + wr * tomo
    return None


def max_over_ranks(x, world, device):
    """Maximum of a per-rank number over all ranks (the slowest replica sets
    the job time). device: where the collective's tensor lives ("cpu" for
    gloo, "cuda:i" for nccl)."""
    if world <= 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# reference engine on the host cores
# ---------------------------------------------------------------------------
def reference_threads(w):
    """Host threads for the reference engines: every core, unless the private
    model copies of the packaged engine (maximize.c:103-104) would not fit in
    half of the available memory. Returns (threads, nproc)."""
    nproc = os.cpu_count() or 1
    n = nproc
    try:
        import psutil
        avail = psutil.virtual_memory().available
        per_thread = 2 * w["size"] ** 3 * 8 * 1.3  # private model + weight copies (maximize.c:103-104)
        n = max(1, min(n, int(avail * 0.5 // per_thread)))
    except Exception:
        pass
    return n, nproc


class FrameStock:
    """Frames of the workload sampled on the host for the CPU engines, grown
    on demand (a sample of n frames is the first n): each frame at a random
    orientation with the workload's lognormal fluence, Poisson counts of the
    FP64 slice (the oracle's slice_gen, the reference's geometry) on the
    pixels with mask <= 1."""

    def __init__(self, w, inp, seed):
        from oracle.oracle import EMCProblem, OracleEngine
        from dragonfly_b200 import synth
        self.w, self.inp = w, inp
        self.rng = np.random.default_rng(seed)
        self.synth = synth
        z = np.zeros(1, np.int32)
        e = np.zeros(0, np.int32)
        self.slicer = OracleEngine(EMCProblem(inp["qvals"], inp["corr"], inp["mask"], z, z, e, e, e,
                                              np.array([[1., 0., 0., 0., 1.]]), inp["intens"][None]))
        self.good = inp["mask"] <= 1
        self.ones, self.multi, self.po, self.pm, self.cm = [], [], [], [], []

    def _grow(self, n):
        while len(self.ones) < n:
            q = self.synth.random_quaternions(1, self.rng)[0]
            phi = np.exp(self.rng.normal(0., self.w["fluence_sigma"]))
            lam = self.slicer.slice_gen(np.append(q, 1.)) * phi
            lam[~self.good] = 0.
            c = self.rng.poisson(np.maximum(lam, 0.))
            p1, pmu = np.nonzero(c == 1)[0], np.nonzero(c > 1)[0]
            self.ones.append(p1.size)
            self.multi.append(pmu.size)
            self.po.append(p1.astype(np.int32))
            self.pm.append(pmu.astype(np.int32))
            self.cm.append(c[pmu].astype(np.int32))

    def problem(self, n):
        """An EMCProblem of the first n frames at the workload's orientations,
        start model and schedule (need_scaling, update_scale)."""
        from oracle.oracle import EMCProblem
        self._grow(n)
        cat = lambda xs: np.concatenate(xs[:n]).astype(np.int32)
        inp, w = self.inp, self.w
        return EMCProblem(inp["qvals"], inp["corr"], inp["mask"], np.array(self.ones[:n], np.int32),
                          np.array(self.multi[:n], np.int32), cat(self.po), cat(self.pm), cat(self.cm),
                          inp["quats"], inp["start"], need_scaling=1, update_scale=1, beta=w["beta"],
                          beta_jump=w["beta_jump"], beta_period=w["beta_period"])


def reference_step(w, inp, n_frames, seed, threads, engine="packaged", iteration=1, stock=None):
    """One iteration of a reference engine (maximize + update_model +
    normalize_scale) on n_frames frames at the full orientation set, from the
    workload's start model, at the given iteration index (its beta and
    whether the scale factors enter the likelihood). engine "packaged" is
    dragonfly/src (the engine behind the Python API), "legacy" is src/ (the
    `emc` binary). Returns seconds."""
    from oracle.oracle import LegacyEngine, ReferenceEngine
    stock = stock or FrameStock(w, inp, seed)
    prob = stock.problem(n_frames)
    eng = ReferenceEngine(prob, num_threads=threads, fast=True) if engine == "packaged" else \
        LegacyEngine(prob, num_threads=threads)
    t0 = time.perf_counter()
    eng.run_iteration(iteration)
    t = time.perf_counter() - t0
    eng.close()
    return t


def reference_throughput(w, inp, threads, budget_s=40., steps=2, engine="packaged", iteration=1, seed=11,
                         stock=None):
    """Reference pairs/s at the full frame count, extrapolated from frame
    samples: t(n) = a + b n through a small sample (64 frames: mostly the
    per-iteration slice work a) and a sample grown by 4x until its time is at
    least three times the small one's (so that the frame-dependent part b n
    dominates the difference) or the budget is spent; that sample is timed
    steps - 1 times. The samples are prefixes of one host-sampled frame
    stream (stock, a FrameStock; one is made when None)."""
    R = inp["quats"].shape[0]
    kw = dict(engine=engine, iteration=iteration, stock=stock)
    n1 = 64
    t1 = reference_step(w, inp, n1, seed, threads, **kw)
    spent, n2, t2 = t1, n1, t1
    while n2 < 16384:
        nxt = 4 * n2
        if n2 > n1:  # predicted time of the next sample from the line so far
            pred = t1 + (t2 - t1) * (nxt - n1) / (n2 - n1)
            if spent + pred > budget_s:
                break
        t2 = reference_step(w, inp, nxt, seed, threads, **kw)
        n2 = nxt
        spent += t2
        if t2 >= 3. * t1:
            break
    reps = [t2]
    for k in range(max(0, steps - 2)):
        if spent + t2 > budget_s:
            break
        reps.append(reference_step(w, inp, n2, seed, threads, **kw))
        spent += reps[-1]
    t2 = float(np.mean(reps))
    b = max((t2 - t1) / (n2 - n1), 1e-12)
    a = max(t1 - b * n1, 0.)
    N = w["n_frames"]
    t_full = a + b * N
    return dict(value=R * N / t_full, t_full=t_full, fixed_s=a, per_frame_s=b, samples={n1: t1, n2: t2},
                raw_sample_pairs_s=R * n2 / t2, cores=threads, frame_share=(t2 - t1) / t2, engine=engine,
                iteration=iteration)


def reference_engines(w, inp, threads, nproc, budget_s, steps, iteration):
    """Both reference engines timed as above at one iteration index; the
    faster is the baseline. Returns the cpu_baseline object."""
    from oracle.oracle import legacy_available
    stock = FrameStock(w, inp, 11)
    res = {"packaged": reference_throughput(w, inp, threads, budget_s, steps, "packaged", iteration, stock=stock)}
    if legacy_available():
        res["legacy"] = reference_throughput(w, inp, threads, budget_s, steps, "legacy", iteration, stock=stock)
    best = max(res, key=lambda k: res[k]["value"])
    beta = min(1., w["beta"] * w["beta_jump"] ** ((iteration - 1) // w["beta_period"]))
    names = {"packaged": "dragonfly/src (the engine behind the Python API)", "legacy": "src/ (the emc binary)"}
    r = res[best]
    return {"value": r["value"], "unit": UNIT, "cores": threads, "nproc": nproc, "kind": "reference",
            "engine": best,
            "sample": "reference engine %s, -O3 -march=native, OpenMP %d threads of %d cores, iteration %d "
                      "(beta %.4g) from the workload's start model, on %s host-sampled frames at all %d "
                      "orientations; t(n) = a + b n fitted and extrapolated to %d frames; the faster of the "
                      "two reference engines" % (names[best], threads, nproc, iteration, beta,
                                                 "/".join(str(k) for k in r["samples"]), inp["quats"].shape[0],
                                                 w["n_frames"]),
            "engines": {k: {"value": v["value"], "fixed_s": v["fixed_s"], "per_frame_s": v["per_frame_s"],
                            "samples_s": {str(n): t for n, t in v["samples"].items()},
                            "frame_share": v["frame_share"]} for k, v in res.items()}}


# iterations of the parity block: beta 0.01 from the start model (rescale in
# the likelihood), then beta 0.01 x sqrt(2) with the scale factors
PARITY_ITERATIONS = (1, 6)


def parity_block(w, inp, n_frames, iterations):
    """The product's graph-launched iteration against the FP64 oracle
    (bit-identical to the reference engine with one thread) on n_frames
    frames simulated at the workload's geometry and fluence, at all of its
    orientations; run after the timed region, on the host cores and the GPU.
    Returns the per-iteration deviations and whether each meets the bar."""
    from oracle.parity import BAR, compare_runs, simulated_subset
    t0 = time.perf_counter()
    prob = simulated_subset(inp, w, n_frames, seed=4242)
    devs = compare_runs(prob, iterations, graph=True)
    keep = ("iteration", "beta", "model_rel_l2", "ll_rel", "mi_rel", "rmax_agree", "scale_rel",
            "frame_ll_max_rel", "within_bar")
    return {"frames": n_frames, "orientations": int(inp["quats"].shape[0]),
            "oracle": "FP64 restatement of dragonfly/src, bit-identical to the reference engine with one thread",
            "bar": BAR, "iterations": [{k: d[k] for k in keep} for d in devs],
            "all_within_bar": all(d["within_bar"] for d in devs), "seconds": time.perf_counter() - t0}


# ---------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    from dragonfly_b200._lib import Context
    import torch
    w = dict(WORKLOAD)
    if args.frames:
        w["n_frames"] = args.frames
    if args.num_div:
        w["num_div"] = args.num_div
    if args.median_photons > 0:
        w["median_photons"] = args.median_photons
    if args.fluence_sigma >= 0:
        w["fluence_sigma"] = args.fluence_sigma
    if w != WORKLOAD:
        w["name"] = ("plain EMC: 260x257 pnCCD-like detector, 201^3 model, num_div %d, %d frames, median %g "
                     "photons (sigma %g), scale update, beta 0.01 x sqrt2 / 5"
                     % (w["num_div"], w["n_frames"], w["median_photons"], w["fluence_sigma"]))
    t_setup = time.perf_counter()
    inp = build_inputs(w)
    ctx = Context(local_rank)
    ctx.set_detector(inp["qvals"], inp["corr"], inp["mask"])
    tot = ctx.simulate_frames(inp["intens"], inp["frame_q"], inp["phi"], seed=777 + rank)
    ctx.set_quaternions(inp["quats"])
    ctx.set_model(inp["start"])
    ctx.calc_beta(w["beta"], 1)
    R = inp["quats"].shape[0]
    N = w["n_frames"]
    # the library's autotuner picks the slice block and the E-step form
    # (sparse gathers or tensor-core products) on these inputs, before timing
    tpar = ctx.params(1, need_scaling=1, update_scale=1, beta_jump=w["beta_jump"], beta_period=w["beta_period"])
    tune = ctx.autotune(tpar)
    if args.estep_form == "auto":
        ctx.set_option("autotune", 1)
    else:
        ctx.set_option("slice_block", tune["slice_block"])
        ctx.set_option("estep_form", 1 if args.estep_form == "dense" else 0)
        ctx.set_option("mstep_form", tune["mstep_form"])
        tune["estep_form"] = 1 if args.estep_form == "dense" else 0
    setup_s = time.perf_counter() - t_setup

    def params(it):
        return ctx.params(it, need_scaling=1, update_scale=1, known_scale=0, beta_jump=w["beta_jump"],
                          beta_period=w["beta_period"], beta_factor=1.)

    def step(it):
        # maximize + update_model + normalize_scale, captured as one CUDA graph
        ctx.run_iteration(params(it), 0.)

    it = 1
    for _ in range(args.warmup):
        step(it)
        it += 1
    wl = ctx.workload()
    # the ceiling of the gather kernels' access pattern on this device: random
    # 512-byte rows of a table the size of one log-slice tile (E-step) and of
    # one probability tile (M-step), measured before the timed region
    gather_peak = {"estep": ctx.measure_gather_rate(inp["qvals"].shape[0] + 1),
                   "mstep": ctx.measure_gather_rate(wl["chunk_frames"] + 1)}

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # timed region: K iterations bracketed by events on the library's stream
    ctx.set_option("timing", 1)
    ctx.reset_phase_times()
    launches0 = ctx.workload()["launches"]
    proc, cpath = clock_sampler(local_rank)
    barrier()
    torch.cuda.synchronize()
    ctx.event_record(0)
    for _ in range(args.steps):
        step(it)
        it += 1
    ctx.event_record(1)
    total_ms = ctx.event_elapsed_ms(0, 1)
    torch.cuda.synchronize()
    barrier()
    clocks = clock_summary(proc, cpath)
    launches = ctx.workload()["launches"] - launches0
    phases = ctx.phase_times()
    ctx.set_option("timing", 0)
    total_ms = max_over_ranks(total_ms, world, "cuda:%d" % local_rank)
    ms_per_step = total_ms / args.steps
    value = world * R * N / (ms_per_step / 1e3)

    # end to end through the host-buffer entry point: model in pinned host
    # memory uploaded, iteration, model + rmax + likelihood read back, per step
    model_h = torch.empty(inp["start"].shape, dtype=torch.float64, pin_memory=True).numpy()
    rmax_h = torch.empty(N, dtype=torch.int32, pin_memory=True).numpy()
    ll_h = torch.empty(N, dtype=torch.float64, pin_memory=True).numpy()
    m1, _, _ = ctx.model()
    model_h[...] = m1
    barrier()
    e2e = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ctx.run_iteration_host(params(it), model_h, 0., rmax_h, ll_h)
        e2e.append(time.perf_counter() - t0)
        it += 1
    e2e_s = max_over_ranks(float(np.mean(e2e)), world, "cuda:%d" % local_rank)

    # roofline of the dominant kernel (per-launch CUDA-event durations)
    dom = max(phases, key=lambda k: phases[k][0])
    ms, nl = phases[dom]
    peak, peak_src = measured_peaks()
    E, EM = wl["estep_entries"], wl["mstep_entries"]
    chunks = max(wl["chunks"], 1)
    algo = {  # algorithmic bytes per launch
        "estep": 4. * R * E / chunks,             # one FP32 log-slice value per orientation x photon entry
        "mstep": 4. * R * EM / chunks,            # one FP32 probability per orientation x photon entry
        "slice": (4. * R * inp["qvals"].shape[0]) / 3,  # log-slice output, over 3 launches
        "norm": (2 * 8. + 4.) * R * N / chunks,   # two passes over FP64 log-likelihoods, FP32 P written
        "psum": 4. * R * N / chunks / 2,
        "merge": 8. * inp["start"].size,
        "update": 8. * inp["start"].size,
    }
    per_launch_s = (ms / 1e3) / max(nl, 1)
    dense_bits = {"estep": 1, "mstep": 2}.get(dom, 0)
    if wl["dense_estep"] & dense_bits:
        # tensor-core E-step or M-step: 2 x R_pad x frames x K_pad x 2 (hi, lo)
        # FLOP per chunk over the phase time per chunk (the E-step phase
        # includes the count densification, the M-step phase the probability
        # split)
        tpeak, tsrc = measured_tensor_peak()
        flop = 2. * (-(-R // 128) * 128) * wl["chunk_frames"] * wl["k_pad"] * 2
        achieved = flop / ((ms / 1e3) / (args.steps * chunks)) / 1e12
        roof = {"kernel": dom + " (dense, tensor cores)", "bound": "tensor", "achieved": achieved, "peak": tpeak,
                "unit": "TFLOP/s", "frac": achieved / tpeak, "peak_source": tsrc, "traffic": None,
                "phase_ms_per_step": {k: v[0] / args.steps for k, v in phases.items()}}
    elif dom in gather_peak:
        # the row gathers are served by L2 / L1 (the tile stays resident while
        # its warps run): the roofline is the measured gather ceiling of the
        # same access pattern; the DRAM side is reported beside it
        achieved = algo[dom] / per_launch_s / 1e9
        traffic = roofline_traffic(dom, -(-R // 128) * 128, inp["qvals"].shape[0], wl["chunk_frames"])
        dram = traffic / per_launch_s / 1e9
        roof = {"kernel": dom, "bound": "l2", "achieved": achieved, "peak": gather_peak[dom], "unit": "GB/s",
                "frac": achieved / gather_peak[dom],
                "peak_source": "measured in this run on this GPU: uniformly random 512-byte rows of a table the "
                               "size of the kernel's tile (dfg_measure_gather_rate)",
                "algorithmic_bytes_per_launch": algo[dom], "launch_ms": per_launch_s * 1e3,
                "traffic": traffic,
                "traffic_note": "modelled from ncu DRAM bytes of a small capture (compulsory streams)",
                "dram": {"achieved": dram, "peak": peak, "frac": dram / peak, "peak_source": peak_src},
                "gather_peaks": gather_peak,
                "phase_ms_per_step": {k: v[0] / args.steps for k, v in phases.items()}}
    else:
        achieved = algo[dom] / per_launch_s / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_src,
                "traffic": roofline_traffic(dom, -(-R // 128) * 128, inp["qvals"].shape[0], wl["chunk_frames"]),
                "phase_ms_per_step": {k: v[0] / args.steps for k, v in phases.items()}}

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64 accumulate / f32 log-slices",
           "data": "synthetic (seeded; frames simulated on the GPU)",
           "config": {"workload": w["name"], "num_orientations": R, "num_frames": N,
                      "photons_per_frame_mean": tot[2] / N, "detector_pixels": int(inp["qvals"].shape[0]),
                      "model": "%d^3 x %d mode" % (w["size"], 1), "frame_chunks": wl["chunks"],
                      "l2": "inputs larger than L2 (no flush needed)",
                      "parallelism": "replicas x%d" % world if world > 1 else "single GPU",
                      "autotuned": {"slice_block": tune["slice_block"],
                                    "estep_form": ["sparse", "dense"][tune["estep_form"]],
                                    "mstep_form": ["sparse", "dense"][tune["mstep_form"]],
                                    "estep_blocks_per_sm": tune["estep_blocks_per_sm"],
                                    "mstep_blocks_per_sm": tune["mstep_blocks_per_sm"],
                                    "ms_first_chunk": {k: None if tune[k] is None else round(float(tune[k]), 2)
                                                       for k in ("estep_sparse_ms", "estep_dense_ms",
                                                                 "mstep_sparse_ms", "mstep_dense_ms")},
                                    "ms_by_blocks_per_sm": {
                                        "estep": {str(k): round(v, 2)
                                                  for k, v in tune["estep_ms_by_blocks_per_sm"].items()},
                                        "mstep": {str(k): round(v, 2)
                                                  for k, v in tune["mstep_ms_by_blocks_per_sm"].items()}}},
                      "setup_s": setup_s},
           "s_per_iteration": ms_per_step / 1e3,
           "clocks": clocks,
           "e2e": {"value": world * R * N / e2e_s, "unit": UNIT,
                   "h2d_bytes_per_step": int(model_h.nbytes),
                   "d2h_bytes_per_step": int(model_h.nbytes + rmax_h.nbytes + ll_h.nbytes),
                   "s_per_iteration": e2e_s},
           "gpu_launches": int(launches),
           "roofline": roof}
    ctx.close()
    return out, inp, w


# ---------------------------------------------------------------------------
# batched form: several reconstructions iterated together
# ---------------------------------------------------------------------------
# independent reconstructions: (model size, frames, num_div, median photons)
BATCH_RECONS = [(51, 5000, 4, 50.), (65, 10000, 5, 100.), (81, 20000, 6, 150.), (95, 40000, 7, 200.),
                (111, 80000, 8, 300.), (125, 60000, 6, 400.), (141, 30000, 5, 500.), (151, 15000, 4, 250.)]
# four heterogeneous modes: a shared 1000-atom density with a 50-atom domain
# shifted by 0, 2, 4 and 6 voxels; frames mixed 4:3:2:1
BATCH_MODES = dict(size=125, atoms=1000, domain=50, shifts=(0, 2, 4, 6), frames=300000, mix=(4, 3, 2, 1),
                   median=200., num_div=6)


def _intensity(pos, size, sigma=1.0):
    rho = np.zeros((size, size, size))
    idx = np.rint(pos).astype(np.int64) % size
    np.add.at(rho, (idx[:, 0], idx[:, 1], idx[:, 2]), 1.0)
    f = np.fft.fftn(rho)
    k = np.fft.fftfreq(size)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    f *= np.exp(-2. * np.pi ** 2 * sigma ** 2 * k2)
    return np.fft.fftshift(np.abs(f) ** 2)


def _batch_context(Context, device, size, num_div, models, frame_sets, budget_mb, seed):
    """One reconstruction: flat size x size detector (edge |q| = (size - 3) / 2),
    num_div orientations, frames simulated from models (one per mode, mode m
    for frame_sets[m] frames) at lognormal fluence."""
    from dragonfly_b200 import synth
    from dragonfly_b200.quatgen import quat_gen
    rng = np.random.default_rng(seed)
    qmax = (size - 3) / 2.
    qvals, corr, mask, _, _ = synth.flat_detector(size, size, qmax, size, hole_radius=size / 25.)
    ctx = Context(device)
    ctx.set_option("pair_budget_mb", budget_mb)
    ctx.set_option("autotune", 1)
    ctx.set_detector(qvals, corr, mask)
    parts = []
    for m, (intens, (n, median)) in enumerate(zip(models, frame_sets)):
        intens = intens * (median / synth.model_mean_count(intens, qvals, corr, mask, rng, n_orient=32))
        ctx.simulate_frames(intens, synth.random_quaternions(n, rng), np.exp(rng.normal(0., 0.3, n)), seed + m)
        parts.append(ctx.get_frames())
    if len(parts) > 1:
        cat = [np.concatenate([p[k] for p in parts]) for k in range(5)]
        ctx.set_frames(*cat)
    quats = quat_gen(num_div)
    ctx.set_quaternions(quats)
    M = len(models)
    ctx.set_model(rng.random((M, size, size, size)) * frame_sets[0][1] / (mask == 0).sum() * 2.)
    ctx.calc_beta(0.01, 1)
    n = sum(f[0] for f in frame_sets)
    return ctx, M * quats.shape[0] * n


def run_batched(args):
    """The batched workload: the four-mode reconstruction and the eight
    independent ones, one iteration each, as one batched graph launch
    (dfg_batch_run) against the same iterations one reconstruction after
    another (each its own graph); both timed on the device over the same
    contexts. Prints one JSON line."""
    from dragonfly_b200._lib import Batch, Context
    from dragonfly_b200 import synth
    import torch
    rng = np.random.default_rng(4321)
    t0 = time.perf_counter()
    ctxs, pairs = [], []
    B = BATCH_MODES
    base = synth.atom_positions(B["atoms"], 0.15 * B["size"], rng)
    dom = synth.atom_positions(B["domain"], 0.05 * B["size"], rng) + np.array([0.08 * B["size"], 0., 0.])
    models = [_intensity(np.concatenate([base, dom + np.array([s, 0., 0.])]), B["size"]) for s in B["shifts"]]
    tot = sum(B["mix"])
    sets = [(B["frames"] * k // tot, B["median"]) for k in B["mix"]]
    c, n = _batch_context(Context, 0, B["size"], B["num_div"], models, sets, 40000., 100)
    ctxs.append(c)
    pairs.append(n)
    for i, (size, frames, nd, median) in enumerate(BATCH_RECONS):
        intens = synth.gaussian_atom_intensity(1000, 0.15 * size, size, rng)
        c, n = _batch_context(Context, 0, size, nd, [intens], [(frames, median)], 12000., 200 + i)
        ctxs.append(c)
        pairs.append(n)
    setup_s = time.perf_counter() - t0
    par = lambda c, it: c.params(it, need_scaling=1, update_scale=1, beta_jump=math.sqrt(2.), beta_period=5)
    batch = Batch(ctxs)
    it = 1
    for _ in range(args.warmup):            # tunes every context, builds the graphs
        batch.run([par(c, it) for c in ctxs])
        for c in ctxs:
            c.run_iteration(par(c, it), 0.)
        it += 1
    timer = ctxs[0]
    torch.cuda.synchronize()
    seq_ms, lane_ms = [], {1: [], len(ctxs): []}
    for _ in range(args.steps):
        timer.event_record(0)
        for c in ctxs:
            c.run_iteration(par(c, it), 0.)
        timer.event_record(1)
        seq_ms.append(timer.event_elapsed_ms(0, 1))
        it += 1
        for lanes in lane_ms:
            batch.set_lanes(lanes)
            timer.event_record(2)
            batch.run([par(c, it) for c in ctxs])
            timer.event_record(3)
            lane_ms[lanes].append(timer.event_elapsed_ms(2, 3))
            it += 1
    total = float(sum(pairs))
    seq = float(np.mean(seq_ms))
    lane_mean = {k: float(np.mean(v)) for k, v in lane_ms.items()}
    best_lanes = min(lane_mean, key=lane_mean.get)
    bat = lane_mean[best_lanes]
    out = {"metric": "frame x orientation pairs per second, batched reconstructions", "value": total / (bat / 1e3),
           "unit": "pairs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": bat,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 accumulate / f32 log-slices",
           "data": "synthetic (seeded; frames simulated on the GPU)",
           "config": {"workload": "batched: 4-mode 125^3 (shared 1000-atom density, 50-atom domain shifted 0/2/4/6 "
                                  "voxels), 300000 frames mixed 4:3:2:1 at median 200, num_div 6; plus 8 independent "
                                  "reconstructions " + ", ".join("%d^3/%d frames/num_div %d/median %g" % r
                                                                for r in BATCH_RECONS),
                      "pairs_per_step": total, "setup_s": setup_s,
                      "autotuned": [c.tune_report() for c in ctxs]},
           "sequential": {"ms_per_step": seq, "value": total / (seq / 1e3)},
           "batch_lanes": {str(k): {"ms_per_step": v, "value": total / (v / 1e3)} for k, v in lane_mean.items()},
           "lanes": best_lanes,
           "speedup_vs_sequential": seq / bat,
           "batch_graph": batch.stats()}
    print(json.dumps(out))
    batch.close()
    for c in ctxs:
        c.close()


# learned-proposal workload: the production detector and 201^3 model,
# num_div 20 (400200 orientations), 500000 frames at median 300 photons; a
# network over 3240 coarse cells (num_div 4), top 16 refined at full
# resolution, 1 % of the frames searched in full and watched
PROPOSALS = dict(num_div=20, n_frames=500000, coarse_div=4, K=16, held_out=0.01, threshold=0.99,
                 train_frames=100000, epochs=2, rounds=10, lr=5e-4, lr_end=1e-4, full_fracs=(8, 4))


def _full_search_ms(w, inp, stride, steps, warmup):
    """Device ms of one full-search iteration (graph, autotuned) over every
    stride-th orientation of the workload (the full set's log-slices and
    tomograms, 4 B x R x P each, do not fit one GPU at num_div 20)."""
    from dragonfly_b200._lib import Context
    c = Context(0)
    c.set_detector(inp["qvals"], inp["corr"], inp["mask"])
    c.simulate_frames(inp["intens"], inp["frame_q"], inp["phi"], seed=777)
    q = np.ascontiguousarray(inp["quats"][::stride])
    q[:, 4] = 1. / q.shape[0]
    c.set_quaternions(q)
    c.set_model(inp["intens"][None])
    c.set_scale(inp["phi"])
    c.calc_beta(1., 1)
    c.set_option("autotune", 1)
    par = lambda it: c.params(it, 1, 1, 1, w["beta_jump"], w["beta_period"], 1.)
    for it in range(1, warmup + 1):
        c.run_iteration(par(it), 0.)
    ms = []
    for it in range(warmup + 1, warmup + 1 + steps):
        c.event_record(0)
        c.run_iteration(par(it), 0.)
        c.event_record(1)
        ms.append(c.event_elapsed_ms(0, 1))
    R = q.shape[0]
    c.close()
    return R, float(np.mean(ms))


def run_proposals(args):
    """The learned-proposal workload: proposal-restricted iterations over pair
    lists (network images and top-K, restriction lists, iteration; wall clock)
    against the plain full search, whose time is measured on every 8th and
    every 4th orientation and extrapolated linearly to all of them. Prints one
    JSON line."""
    import torch
    from dragonfly_b200._lib import Context
    from dragonfly_b200.proposals import LearnedProposals, sort_by_coarse
    P_ = dict(PROPOSALS)
    w = dict(WORKLOAD)
    w.update(num_div=P_["num_div"], n_frames=args.frames or P_["n_frames"])
    if args.num_div:
        w["num_div"] = args.num_div
    t0 = time.perf_counter()
    inp = build_inputs(w)
    R = inp["quats"].shape[0]
    N = w["n_frames"]
    # the full search at two orientation subsets
    full = {}
    full_ms = None
    if not args.no_full_search:
        for stride in P_["full_fracs"]:
            full[stride] = _full_search_ms(w, inp, stride, 1, 1)
        (Ra, ta), (Rb, tb) = full[P_["full_fracs"][0]], full[P_["full_fracs"][1]]
        slope = (tb - ta) / (Rb - Ra)
        full_ms = tb + slope * (R - Rb)
    torch.cuda.synchronize()
    # the proposal form at the full orientation set
    c = Context(0)
    c.set_detector(inp["qvals"], inp["corr"], inp["mask"])
    c.simulate_frames(inp["intens"], inp["frame_q"], inp["phi"], seed=777)
    fine, _, _ = sort_by_coarse(inp["quats"], P_["coarse_div"], c)
    c.set_quaternions(fine)
    c.set_model(inp["intens"][None])
    c.set_scale(inp["phi"])
    c.calc_beta(1., 1)
    setup_s = time.perf_counter() - t0
    lp = LearnedProposals(c, inp["qvals"], fine, coarse_div=P_["coarse_div"], K=P_["K"], held_out=P_["held_out"],
                          threshold=P_["threshold"], seed=5, pair_lists=True, retrain_epochs=args.retrain_epochs,
                          K_max=args.proposal_kmax or None, mass=args.proposal_mass or None,
                          retrain_lr=args.retrain_lr)
    t1 = time.perf_counter()
    if args.train_rounds:
        P_["rounds"] = args.train_rounds
    loss = lp.train_simulated(inp["intens"], n_frames=P_["train_frames"], epochs=P_["epochs"], lr=P_["lr"],
                              lr_end=P_["lr_end"], rounds=P_["rounds"],
                              phi=np.exp(np.random.default_rng(9).normal(0., w["fluence_sigma"],
                                                                          P_["train_frames"])))
    train_s = time.perf_counter() - t1
    # hit rate of the true orientation's cell
    cells = c.voronoi_subset(lp.coarse, np.pad(inp["frame_q"][:, :4], ((0, 0), (0, 1))))
    par = lambda it: c.params(it, 1, 1, 1, w["beta_jump"], w["beta_period"], 1.)
    runs = []
    c.set_option("timing", 1)
    for it in range(1, args.warmup + args.steps + 1):
        if it == args.warmup + 1:
            c.reset_phase_times()
        torch.cuda.synchronize()
        ts = time.perf_counter()
        out = lp.proposal_iteration(par(it), 0.)
        torch.cuda.synchronize()
        runs.append(dict(wall_ms=1e3 * (time.perf_counter() - ts), mass=out["captured_mass"],
                         min_mass=out["min_mass"], propose_ms=1e3 * out["propose_s"], lists_ms=1e3 * out["lists_s"],
                         iterate_ms=1e3 * out["iterate_s"], fallback_next=lp.full_next))
    phases = {k: round(v[0] / args.steps, 1) for k, v in c.phase_times().items()}
    top = lp.propose()
    hit = float(np.mean(np.any(top == cells[:, None], axis=1)))
    loop = None
    if args.loop:
        # the fallback: a full search over all orientations (in orientation
        # blocks) keeping its probabilities, the network retrained on them;
        # then a proposal iteration, compared with a full search from the same
        # state
        it = args.warmup + args.steps + 1
        lp.full_next = True
        c.reset_phase_times()
        f = lp.iteration(par(it), 0.)
        full_phases = {k: round(v[0], 1) for k, v in c.phase_times().items()}
        wl_full = c.workload()
        m0, _, _ = c.model()
        s0 = c.frame_params()["scale"]
        p_ = lp.proposal_iteration(par(it + 1), 0.)
        p_fallback = lp.full_next
        mp, _, _ = c.model()
        rp = c.frame_results()["rmax"].copy()
        c.set_model(m0)
        c.set_scale(s0)
        c.set_refinement(None)
        t0 = time.perf_counter()
        c.run_iteration(par(it + 1), 0.)
        t_same = time.perf_counter() - t0
        mf, _, _ = c.model()
        rf = c.frame_results()["rmax"]
        # further proposal iterations after the retraining: their captured
        # mass, and the loop's time per iteration amortised over the fallback
        # (full search + retraining) and every proposal iteration
        more = []
        for k in range(args.loop_iterations):
            q_ = lp.iteration(par(it + 2 + k), 0.)
            more.append({"mode": q_["mode"], "captured_mass": q_.get("captured_mass"),
                         "wall_s": q_.get("propose_s", 0.) + q_.get("lists_s", 0.) + q_["iterate_s"] +
                         q_.get("retrain_s", 0.)})
        t_loop = f["iterate_s"] + f["retrain_s"] + p_["propose_s"] + p_["lists_s"] + p_["iterate_s"] + \
            sum(x["wall_s"] for x in more)
        n_loop = 2 + len(more)
        loop = {"full_search_s": f["iterate_s"], "full_search_phases_ms": full_phases,
                "more_iterations": more,
                "amortised_s_per_iteration": t_loop / n_loop,
                "amortised_speedup_vs_full_search": f["iterate_s"] / (t_loop / n_loop),
                "full_search_chunks": wl_full["chunks"], "retrain_s": f["retrain_s"],
                "retrain": "%d epochs (lr %g) on the %d frames against the full search's probabilities per cell" % (
                    lp.retrain_epochs, lp.retrain_lr, N),
                "proposal_after_retrain": {"captured_mass": p_["captured_mass"], "min_mass": p_["min_mass"],
                                           "wall_s": p_["propose_s"] + p_["lists_s"] + p_["iterate_s"],
                                           "fallback_next": p_fallback},
                "vs_full_search_same_state": {"model_rel_l2": float(np.linalg.norm(mp - mf) / np.linalg.norm(mf)),
                                              "rmax_agreement": float(np.mean(rp == rf)),
                                              "full_search_s": t_same}}
    wl = c.workload()
    timed = runs[args.warmup:]
    ms = float(np.mean([r["wall_ms"] for r in timed]))
    it_ms = float(np.mean([r["iterate_ms"] for r in timed]))
    tiles = -(-R // 128)
    out = {"metric": "s per EMC iteration, learned-proposal form vs plain full search",
           "value": ms / 1e3, "unit": "s/iteration", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
           "dtype": "bf16 network / f64 accumulate / f32 log-slices",
           "data": "synthetic (seeded; frames simulated on the GPU; model at the truth, true scales, beta 1)",
           "config": {"workload": "learned proposals: 260x257 pnCCD-like detector, 201^3 model, num_div %d (%d "
                                  "orientations), %d frames, median %g photons (lognormal sigma %g); %d coarse "
                                  "cells (num_div %d), top %d%s, %g %% held out" % (
                                      w["num_div"], R, N, w["median_photons"], w["fluence_sigma"], lp.nc,
                                      P_["coarse_div"], P_["K"],
                                      "" if lp.mass is None else " and more up to %d until the network's probability "
                                      "reaches %g" % (lp.K_max, lp.mass), 100 * P_["held_out"]),
                      "setup_s": setup_s, "train_s": train_s,
                      "training": "%d rounds x %d epochs of %d newly simulated frames, lr %g -> %g" % (
                          P_["rounds"], P_["epochs"], P_["train_frames"], P_["lr"], P_["lr_end"]),
                      "train_loss": loss},
           "proposal": {"wall_ms": ms, "iteration_ms": it_ms, "phases_ms": phases, "runs": timed,
                        "live_pairs": wl["live_pairs"], "block_tiles": wl["block_tiles"],
                        "live_fraction_of_tiles": wl["live_pairs"] / float(tiles * N),
                        "top_k_hit_rate": hit, "evaluated_fraction_of_cells": out["evaluated_fraction"]},
           "full_search": {"ms_extrapolated": full_ms,
                           "measured": {str(Rx): tx for Rx, tx in full.values()},
                           "rule": "t(R) linear in R through the two measured subsets"},
           "speedup_vs_full_search": full_ms / ms if full_ms else None,
           "loop": loop,
           "effective_pairs_per_s": R * N / (ms / 1e3),
           # the (orientation, frame) pairs the proposal iteration evaluates:
           # every orientation of each live (tile, frame) pair
           "evaluated_pairs_per_s": wl["live_pairs"] * 128 / (it_ms / 1e3)}
    print(json.dumps(out))
    lp.close()
    c.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=0, help="override the frame count (testing)")
    ap.add_argument("--num-div", type=int, default=0, help="override num_div (testing)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the parity block (GPU iteration against the oracle on a frame subset)")
    ap.add_argument("--parity-frames", type=int, default=512, help="frames of the parity block")
    ap.add_argument("--median-photons", type=float, default=0., help="override the median photons per frame")
    ap.add_argument("--fluence-sigma", type=float, default=-1., help="override the lognormal fluence sigma")
    ap.add_argument("--estep-form", default="auto", choices=["auto", "sparse", "dense"],
                    help="E-step photon term: autotuned (default), sparse gathers or tensor-core products")
    ap.add_argument("--train-rounds", type=int, default=0,
                    help="proposals: rounds of network training (default 10; fewer for profiling runs)")
    ap.add_argument("--retrain-epochs", type=int, default=3,
                    help="proposals --loop: epochs of retraining on the fallback full search's probabilities")
    ap.add_argument("--retrain-lr", type=float, default=1e-3, help="proposals --loop: retraining rate")
    ap.add_argument("--proposal-kmax", type=int, default=0,
                    help="proposals: mass-covering proposals with at most this many cells per frame (0: exactly K)")
    ap.add_argument("--proposal-mass", type=float, default=0.,
                    help="proposals: the network probability a frame's cells must cover (with --proposal-kmax)")
    ap.add_argument("--loop-iterations", type=int, default=2,
                    help="proposals --loop: proposal iterations after the retraining, for the amortised time")
    ap.add_argument("--loop", action="store_true",
                    help="proposals: also run the fallback full search (orientation blocks), retrain on its "
                         "probabilities and compare the next proposal iteration with a full search")
    ap.add_argument("--no-full-search", action="store_true",
                    help="proposals: skip timing the full search (profiling runs)")
    ap.add_argument("--workload", default="plain", choices=["plain", "batched", "proposals"],
                    help="plain: the production-size iteration (default); batched: nine reconstructions "
                         "iterated together against one after another; proposals: the learned-proposal "
                         "form at num_div 20 against the full search")
    args = ap.parse_args()
    if args.warmup < 3:
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "proposals":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned-proposal "
                                  "form, and its full search at 400200 orientations x 500000 frames would run "
                                  "for days on the host cores"}))
            return
        if rank == 0:
            run_proposals(args)
        return
    if args.workload == "batched":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the batched workload has no counterpart in "
                                  "the reference (one reconstruction per process)"}))
            return
        if rank == 0:
            run_batched(args)
        return

    if args.impl == "reference":
        if rank != 0:
            return
        w = dict(WORKLOAD)
        if args.frames:
            w["n_frames"] = args.frames
        if args.num_div:
            w["num_div"] = args.num_div
        from oracle.oracle import reference_available, build_oracle
        if not reference_available(fast=True):
            try:
                build_oracle()
            except Exception:
                pass
        if not reference_available(fast=True):
            print(json.dumps({"impl": "reference", "unavailable":
                              "reference engine library oracle/_ref/libdragonfly_ref_fast.so not built"}))
            return
        inp = build_inputs(w)
        threads, nproc = reference_threads(w)
        # the middle of the timed iterations of the GPU arm (warm-up steps
        # first), i.e. the same iteration index and beta
        iteration = args.warmup + 1 + args.steps // 2
        cb = reference_engines(w, inp, threads, nproc, budget_s=110., steps=max(2, args.steps), iteration=iteration)
        t_full = inp["quats"].shape[0] * w["n_frames"] / cb["value"]
        out = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_full * 1e3,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic (seeded)", "impl": "reference",
               "config": {"workload": w["name"], "num_orientations": int(inp["quats"].shape[0]),
                          "num_frames": w["n_frames"], "parallelism": "host cores"},
               "cpu_baseline": cb,
               "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return

    import torch
    if world > 1:
        torch.cuda.set_device(local_rank)
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    out, inp, w = run_ours(args, rank, world, local_rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.oracle import reference_available
        if reference_available(fast=True):
            threads, nproc = reference_threads(w)
            out["cpu_baseline"] = reference_engines(w, inp, threads, nproc, budget_s=60., steps=2,
                                                    iteration=args.warmup + 1 + args.steps // 2)
        else:
            out["cpu_baseline"] = None
        if not args.no_parity:
            out["parity"] = parity_block(w, inp, args.parity_frames, PARITY_ITERATIONS)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
