"""Shared helpers of the test suite: golden cases, engines and tolerances."""
import os

import numpy as np

from oracle.oracle import EMCProblem, OracleEngine

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("beta1", "scaling", "edge", "modes2")

# Parity bar of the plain GPU form against the FP64 oracle (one-thread
# semantics of the reference engine):
MODEL_REL_L2 = 1e-5      # model after each iteration
SCALAR_REL = 1e-6        # average log-likelihood and mutual information
RMAX_AGREE = 0.999       # fraction of frames with the same most likely orientation
SCALE_REL = 1e-5         # per-frame scale factors (max relative deviation)


def load_case(name):
    g = np.load(os.path.join(GOLDEN, name + ".npz"))
    pp = g["prob_params"]
    bl = g["blacklist"]
    prob = EMCProblem(g["qvals"], g["corr"], g["mask"], g["ones"], g["multi"], g["place_ones"],
                      g["place_multi"], g["count_multi"], g["quats"], g["model_start"],
                      need_scaling=int(pp[0]), update_scale=int(pp[1]), known_scale=int(pp[2]),
                      alpha=pp[3], beta=pp[4], beta_jump=pp[5], beta_period=int(pp[6]),
                      beta_factor=pp[7], blacklist=bl if bl.any() else None)
    return prob, g


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


class GPUEngine:
    """The product path (libdfgpu.so through dragonfly_b200._lib) run with the
    same steps as oracle.OracleEngine.run_iteration."""

    def __init__(self, prob, device=0, **options):
        from dragonfly_b200._lib import Context
        self.prob = p = prob
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


def rmax_agreement(a, b, prob, model_before, it, scale_before=None):
    """Fraction of good frames whose most likely orientation is the oracle's,
    counting as agreeing the frames where the two choices are exact ties: the
    oracle's log-likelihoods of both orientations equal within 1e-9 relative
    (e.g. frames without photons, ranked by u_r alone, when a symmetry of the
    detector and the Friedel-symmetric model maps one orientation onto the
    other -- the reference then picks by rounding noise). Returns
    (agreement, number of tie frames)."""
    good = np.ones(prob.num_data, bool) if prob.blacklist is None else prob.blacklist == 0
    if not good.any():
        return 1., 0
    mism = np.nonzero((a["rmax"] != b["rmax"]) & good)[0]
    ties = 0
    use_scale = prob.need_scaling and (it > 1 or prob.known_scale)
    for d in mism:
        ra, rb = int(a["rmax"][d]), int(b["rmax"][d])
        if ra < 0 or rb < 0:
            continue
        s_d = scale_before[d] if use_scale else b["rescale"]
        la = pair_loglik(prob, model_before, ra, d, b["u"][ra], s_d)
        lb = pair_loglik(prob, model_before, rb, d, b["u"][rb], s_d)
        if abs(la - lb) <= 1e-9 * max(1., abs(lb)):
            ties += 1
    return float(1. - (len(mism) - ties) / good.sum()), ties


def compare_iteration(a, b, prob, it, check_model=True, model_before=None, scale_before=None):
    """Checks GPU result a against oracle result b; returns a dict of the
    measured deviations (asserts the parity bar). model_before / scale_before
    (the oracle's inputs of this iteration) let exact ties of the most likely
    orientation be recognised."""
    good = np.ones(prob.num_data, bool) if prob.blacklist is None else prob.blacklist == 0
    out = {}
    out["model_rel_l2"] = rel_l2(a["model1"], b["model1"])
    out["ll_rel"] = rel(a["avg_likelihood"], b["avg_likelihood"])
    out["mi_rel"] = rel(a["mutual_info"], b["mutual_info"]) if b["mutual_info"] != 0 else \
        abs(a["mutual_info"])
    out["rmax_agree"] = float(np.mean(a["rmax"][good] == b["rmax"][good])) if good.any() else 1.
    out["rmax_ties"] = 0
    if out["rmax_agree"] < RMAX_AGREE and model_before is not None:
        out["rmax_agree"], out["rmax_ties"] = rmax_agreement(a, b, prob, model_before, it, scale_before)
    out["rmax_blacklisted_equal"] = bool(np.all(a["rmax"][~good] == b["rmax"][~good]))
    if prob.need_scaling:
        sa, sb = a["scale"][good], b["scale"][good]
        out["scale_rel"] = float(np.max(np.abs(sa - sb) / np.abs(sb)))
    msg = "iteration %d: %s" % (it, out)
    if check_model:
        assert out["model_rel_l2"] <= MODEL_REL_L2, msg
    assert out["ll_rel"] <= SCALAR_REL, msg
    assert out["mi_rel"] <= SCALAR_REL, msg
    assert out["rmax_agree"] >= RMAX_AGREE, msg
    assert out["rmax_blacklisted_equal"], msg
    if prob.need_scaling:
        assert out["scale_rel"] <= SCALE_REL, msg
    return out
