"""Shared helpers of the test suite: golden cases, engines and tolerances."""
import os

import numpy as np

from oracle.oracle import EMCProblem, OracleEngine  # noqa: F401
from oracle.parity import (GPUEngine, deviations, pair_loglik, rel, rel_l2,  # noqa: F401
                           rmax_agreement)

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


def compare_iteration(a, b, prob, it, check_model=True, model_before=None, scale_before=None):
    """Checks GPU result a against oracle result b; returns a dict of the
    measured deviations (asserts the parity bar). model_before / scale_before
    (the oracle's inputs of this iteration) let exact ties of the most likely
    orientation be recognised."""
    out = deviations(a, b, prob, it, model_before, scale_before)
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


def two_detector_problems(seed, **kw):
    """Two EMCProblems sharing orientations and model, each with its own
    detector (different geometry and pixel count) and frames
    (synth.two_detector_problem); kw are EMCProblem parameters; with
    known_scale each detector's frames get seeded uniform [0.5, 1.5) scales."""
    from dragonfly_b200 import synth
    dets, sh = synth.two_detector_problem(seed=seed)
    probs = []
    for k, d in enumerate(dets):
        scale = None
        if kw.get("known_scale"):
            scale = np.random.default_rng(seed + k).uniform(0.5, 1.5, d["ones"].size)
        probs.append(EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"],
                                d["place_multi"], d["count_multi"], sh["quats"], sh["model_start"], scale=scale,
                                **kw))
    return probs
