"""The product's iteration compared with the FP64 oracle. TEST INFRASTRUCTURE ONLY.

Used by tests/ (which assert the bar) and by bench.py's CPU-baseline leg
(which reports the deviations next to the reference's timing, outside the
timed region). The product never imports it.

Bar of the plain GPU form against the FP64 oracle (one-thread semantics of
the reference engine, dragonfly/src/maximize.c:8-56 with recon.pyx:112-149 and
iterate.pyx:361-384): model relative L2 <= 1e-5 after every iteration,
average log-likelihood and mutual information within 1e-6 relative, the same
most likely orientation for >= 99.9 % of frames (exact ties of the oracle's
log-likelihoods count as agreeing), scale factors within 1e-5 relative.
"""
import numpy as np

from .oracle import EMCProblem, OracleEngine

BAR = dict(model_rel_l2=1e-5, ll_rel=1e-6, mi_rel=1e-6, rmax_agree=0.999, scale_rel=1e-5)


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rel(a, b):
    return float(abs(a - b) / max(abs(b), 1e-300))


class GPUEngine:
    """The product path (libdfgpu.so through dragonfly_b200._lib) run with the
    same steps as OracleEngine.run_iteration: maximize, update_model and, for
    need_scaling volumes, normalize_scale. With as_graph=True the three run as
    the one CUDA graph of dfg_run_iteration (the form bench.py times).
    Keyword options are set_option keys."""

    def __init__(self, prob, device=0, as_graph=False, **options):
        from dragonfly_b200._lib import Context
        self.prob = p = prob
        self.as_graph = as_graph
        self.ctx = c = Context(device)
        for k, v in options.items():
            c.set_option(k, v)
        c.set_detector(p.qvals, p.corr, p.mask)
        c.set_frames(p.ones, p.multi, p.place_ones, p.place_multi, p.count_multi)
        c.set_quaternions(p.quats)
        if p.model_type != "3d":
            c.set_model_type(p.model_type, p.friedel_sym)
            c.set_detector_distance(p.detd)
        c.set_model(p.model1)
        if p.scale is not None:
            c.set_scale(p.scale)
        if p.blacklist is not None:
            c.set_blacklist(p.blacklist)
        c.calc_beta(p.beta, p.need_scaling)

    def run_iteration(self, iteration):
        p, c = self.prob, self.ctx
        par = c.params(iteration, p.need_scaling, p.update_scale, p.known_scale, p.beta_jump,
                       p.beta_period, p.beta_factor)
        if self.as_graph:
            out = c.run_iteration(par, p.alpha)
            res = dict(c.frame_results())
            res["u"], res["psum_r"] = c.orientation_results()
            res["num_prob"] = c.num_prob()
            res.update(rescale=out["rescale"], mutual_info=out["mutual_info"],
                       avg_likelihood=out["avg_likelihood"], rms_change=out["rms_change"])
            fp = c.frame_params()
            res["scale"], res["beta"] = fp["scale"], fp["beta"]
            m1, m2n, _ = c.model()
            res["model1"], res["model2"] = m1, m2n
            return res
        avg_ll = c.maximize(par)
        res = dict(c.frame_results())
        res["u"], res["psum_r"] = c.orientation_results()
        res["quat_norm"] = c.quat_norm()
        res["num_prob"] = c.num_prob()
        sc = c.scalars()
        res.update(rescale=sc["rescale"], mutual_info=sc["mutual_info"], avg_likelihood=avg_ll)
        _, m2, w = c.model()
        res["model2_sum"], res["inter_weight"] = m2, w
        rms = c.update_model(p.alpha)
        if p.need_scaling and p.model_type == "3d":   # recon.pyx:102-103
            c.normalize_scale()
            rms = c.scalars()["rms_change"]
        fp = c.frame_params()
        res["scale"], res["beta"] = fp["scale"], fp["beta"]
        res["rms_change"] = rms
        m1, m2n, _ = c.model()
        res["model1"], res["model2"] = m1, m2n
        return res

    def close(self):
        self.ctx.close()


def pair_loglik(prob, model, r, d, u_r, s_d):
    """FP64 log-likelihood of frame d at orientation r under model, in the
    reference's order (max_prob.c:122-171), from the oracle's slice."""
    M = prob.num_modes
    orc = OracleEngine(prob)
    orc._model1 = np.ascontiguousarray(model)
    with np.errstate(divide="ignore"):
        logw = np.log(orc.slice_gen(prob.quats[r // M], r % M))
    oo = int(prob.ones[:d].sum())
    mo = int(prob.multi[:d].sum())
    pval = np.log(prob.quats[r // M, 4]) - u_r * s_d
    for p in prob.place_ones[oo:oo + prob.ones[d]]:
        if prob.mask[p] < 1:
            pval += logw[p]
    for p, c in zip(prob.place_multi[mo:mo + prob.multi[d]], prob.count_multi[mo:mo + prob.multi[d]]):
        if prob.mask[p] < 1:
            pval += c * logw[p]
    return pval


def rmax_agreement(a, b, prob, model_before, it, scale_before=None, max_checks=200):
    """Fraction of good frames whose most likely orientation is the oracle's,
    counting as agreeing the frames where the two choices are exact ties: the
    oracle's log-likelihoods of both orientations equal within 1e-9 relative
    (e.g. frames without photons, ranked by u_r alone, when a symmetry of the
    detector and the Friedel-symmetric model maps one orientation onto the
    other -- the reference then picks by rounding noise). At most max_checks
    mismatches are examined (the rest count as disagreeing). Returns
    (agreement, number of tie frames)."""
    good = np.ones(prob.num_data, bool) if prob.blacklist is None else prob.blacklist == 0
    if not good.any():
        return 1., 0
    mism = np.nonzero((a["rmax"] != b["rmax"]) & good)[0]
    ties = 0
    use_scale = prob.need_scaling and (it > 1 or prob.known_scale)
    for d in mism[:max_checks]:
        ra, rb = int(a["rmax"][d]), int(b["rmax"][d])
        if ra < 0 or rb < 0:
            continue
        s_d = scale_before[d] if use_scale else b["rescale"]
        la = pair_loglik(prob, model_before, ra, d, b["u"][ra], s_d)
        lb = pair_loglik(prob, model_before, rb, d, b["u"][rb], s_d)
        if abs(la - lb) <= 1e-9 * max(1., abs(lb)):
            ties += 1
    return float(1. - (len(mism) - ties) / good.sum()), ties


def deviations(a, b, prob, it, model_before=None, scale_before=None):
    """Deviations of GPU result a from oracle result b (dicts of one
    iteration's outputs), in the terms of BAR, plus the per-frame
    log-likelihood error."""
    good = np.ones(prob.num_data, bool) if prob.blacklist is None else prob.blacklist == 0
    out = {}
    out["model_rel_l2"] = rel_l2(a["model1"], b["model1"])
    out["ll_rel"] = rel(a["avg_likelihood"], b["avg_likelihood"])
    out["mi_rel"] = rel(a["mutual_info"], b["mutual_info"]) if b["mutual_info"] != 0 else \
        float(abs(a["mutual_info"]))
    out["rmax_agree"] = float(np.mean(a["rmax"][good] == b["rmax"][good])) if good.any() else 1.
    out["rmax_ties"] = 0
    if out["rmax_agree"] < BAR["rmax_agree"] and model_before is not None:
        out["rmax_agree"], out["rmax_ties"] = rmax_agreement(a, b, prob, model_before, it, scale_before)
    out["rmax_blacklisted_equal"] = bool(np.all(a["rmax"][~good] == b["rmax"][~good]))
    if prob.need_scaling:
        sa, sb = a["scale"][good], b["scale"][good]
        out["scale_rel"] = float(np.max(np.abs(sa - sb) / np.abs(sb)))
    la, lb = a["likelihood"][good], b["likelihood"][good]
    fin = np.isfinite(lb)
    out["frame_ll_max_abs"] = float(np.max(np.abs(la[fin] - lb[fin]))) if fin.any() else 0.
    out["frame_ll_max_rel"] = float(np.max(np.abs(la[fin] - lb[fin]) / np.maximum(np.abs(lb[fin]), 1.))) \
        if fin.any() else 0.
    return out


def within_bar(dev, prob, check_model=True):
    """True when the deviations meet BAR."""
    ok = dev["ll_rel"] <= BAR["ll_rel"] and dev["mi_rel"] <= BAR["mi_rel"] and \
        dev["rmax_agree"] >= BAR["rmax_agree"] and dev["rmax_blacklisted_equal"]
    if check_model:
        ok = ok and dev["model_rel_l2"] <= BAR["model_rel_l2"]
    if prob.need_scaling:
        ok = ok and dev["scale_rel"] <= BAR["scale_rel"]
    return bool(ok)


def probability_deviations(gpu_sparse, orc_sparse, num_rot):
    """Errors of the GPU's per-frame probabilities (pairs with P > 1e-6, the
    keep_prob lists) against the oracle's kept lists: the largest absolute
    error over the union of both sets of pairs above 1e-6, and the mean over
    frames of the L1 distance between the two distributions."""
    go, gp, gv = gpu_sparse
    oo, op, ov = orc_sparse
    n = len(go) - 1
    gkey = np.repeat(np.arange(n, dtype=np.int64), np.diff(go)) * num_rot + gp
    okey = np.repeat(np.arange(n, dtype=np.int64), np.diff(oo)) * num_rot + op
    sel = ov > 1e-6
    okey, ovs = okey[sel], ov[sel]
    keys = np.union1d(gkey, okey)
    pa = np.zeros(keys.size)
    pb = np.zeros(keys.size)
    pa[np.searchsorted(keys, gkey)] = gv
    pb[np.searchsorted(keys, okey)] = ovs
    diff = np.abs(pa - pb)
    frame = keys // num_rot
    l1 = np.bincount(frame, weights=diff, minlength=n)
    return {"prob_max_abs": float(diff.max()) if diff.size else 0., "prob_l1_mean": float(l1.mean()),
            "prob_pairs_gpu": int(gkey.size), "prob_pairs_oracle": int(okey.size)}


def simulated_subset(inp, w, n_frames, seed, device=0):
    """An EMCProblem of n_frames frames of the workload w (bench.py's
    WORKLOAD layout) with inputs inp (bench.build_inputs): the workload's
    detector, orientations and start model, frames simulated by the library
    on the GPU at random orientations with the workload's lognormal fluence
    and read back, need_scaling and update_scale on, the workload's beta
    schedule."""
    from dragonfly_b200._lib import Context
    from dragonfly_b200 import synth
    rng = np.random.default_rng(seed)
    fq = synth.random_quaternions(n_frames, rng)
    phi = np.exp(rng.normal(0., w["fluence_sigma"], n_frames))
    c = Context(device)
    try:
        c.set_detector(inp["qvals"], inp["corr"], inp["mask"])
        c.simulate_frames(inp["intens"], fq, phi, seed)
        fr = c.get_frames()
    finally:
        c.close()
    return EMCProblem(inp["qvals"], inp["corr"], inp["mask"], *fr, inp["quats"], inp["start"],
                      need_scaling=1, update_scale=1, beta=w["beta"], beta_jump=w["beta_jump"],
                      beta_period=w["beta_period"])


def compare_runs(prob, iterations, graph=True, probabilities=False, **options):
    """Runs the GPU path (options as set_option keys) and the oracle through
    the same iteration indices from the same start and returns one record of
    deviations per iteration (with a 'within_bar' flag each)."""
    import time
    gpu = GPUEngine(prob, as_graph=graph and not probabilities, **options)
    if probabilities:
        gpu.ctx.set_option("keep_prob", 1)
    orc = OracleEngine(prob)
    orc.set_save_prob(probabilities)
    out = []
    try:
        for it in iterations:
            model_before, scale_before = orc.model1(), orc.scale.copy()
            t0 = time.perf_counter()
            a = gpu.run_iteration(it)
            if probabilities:
                gsp = gpu.ctx.sparse_prob()
            t1 = time.perf_counter()
            b = orc.run_iteration(it)
            t2 = time.perf_counter()
            dev = deviations(a, b, prob, it, model_before, scale_before)
            if probabilities:
                dev.update(probability_deviations(gsp, b["sparse_prob"], prob.num_modes * prob.num_rot))
            dev["within_bar"] = within_bar(dev, prob)
            dev["iteration"] = int(it)
            dev["beta"] = float(b["beta"][0])
            dev["gpu_s"] = t1 - t0
            dev["oracle_s"] = t2 - t1
            out.append(dev)
    finally:
        gpu.close()
    return out
