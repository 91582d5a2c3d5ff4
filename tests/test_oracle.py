"""The CPU oracle, pinned against the reference engine.

* golden vectors (tests/golden/*.npz, produced by the reference's own C engine
  with one thread by tests/golden/make_golden.py): the oracle must reproduce
  them bit for bit;
* where the reference sources were compiled here (oracle/_ref), a live
  comparison on fresh seeded inputs, also bit for bit.
"""
import hashlib

import numpy as np
import pytest

from common import CASES, load_case, two_detector_problems
from oracle.oracle import EMCProblem, OracleEngine, ReferenceEngine, reference_available


def sha(m):
    return hashlib.sha256(np.ascontiguousarray(m, np.float64).tobytes()).hexdigest()


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden(name, oracle_built):
    prob, g = load_case(name)
    eng = OracleEngine(prob)
    np.testing.assert_array_equal(eng.fcounts, g["fcounts"])
    np.testing.assert_array_equal(eng.sum_fact, g["sum_fact"])
    np.testing.assert_array_equal(eng.beta_start, g["beta_start"])
    for it in range(1, int(g["iters"]) + 1):
        r = eng.run_iteration(it)
        k = "it%d_" % it
        sc = g[k + "scalars"]
        assert r["avg_likelihood"] == sc[0]
        assert r["mutual_info"] == sc[1]
        assert r["rms_change"] == sc[2]
        assert r["rescale"] == sc[3]
        for key in ("rmax", "info", "likelihood", "max_exp", "p_norm", "psum_d", "u"):
            np.testing.assert_array_equal(r[key], g[k + key], err_msg=key)
        # the reference never writes beta of blacklisted frames (malloc'd,
        # iterate.c:70; skipped at recon.pyx:166-167)
        good = g["blacklist"] == 0
        np.testing.assert_array_equal(r["beta"][good], g[k + "beta"][good])
        if prob.num_modes > 1:
            np.testing.assert_array_equal(r["quat_norm"], g[k + "quat_norm"])
        if prob.need_scaling:
            np.testing.assert_array_equal(r["scale"], g[k + "scale"])
        assert sha(r["model2_sum"]) == str(g[k + "model2_sum_sha256"])
        assert sha(r["inter_weight"]) == str(g[k + "weight_sha256"])
        assert sha(r["model1"]) == str(g[k + "model_sha256"])
    np.testing.assert_array_equal(r["model1"], g["final_model1"])


def test_golden_edge_case_contents():
    """The edge case really exercises what it claims to."""
    prob, g = load_case("edge")
    assert prob.num_pix % 64 != 0 and prob.num_rot % 32 != 0
    assert (g["blacklist"] == 1).sum() == 10
    assert (prob.ones == 0).sum() >= 2
    assert prob.count_multi.max() > 1023
    rmax = g["it1_rmax"]
    assert ((rmax == -1) & (g["blacklist"] == 0)).sum() > 0  # frames with every pval = -inf


@pytest.mark.skipif(not reference_available(), reason="reference sources not compiled here")
@pytest.mark.parametrize("seed,prob_kw", [
    (11, dict(beta=1.)),
    (12, dict(beta=0.02, beta_jump=2., beta_period=1, need_scaling=1, update_scale=1)),
    (13, dict(beta=0.3, need_scaling=1, update_scale=0, known_scale=1, alpha=0.25)),
])
def test_oracle_matches_live_reference(seed, prob_kw, oracle_built):
    from dragonfly_b200 import synth
    d = synth.small_problem(seed=seed, det_side=28, size=33, qmax=15., n_atoms=80, atom_radius=6.,
                            num_div=2, n_frames=160, mean_count=40.)
    scale = None
    if prob_kw.get("known_scale"):
        scale = np.random.default_rng(seed).uniform(0.5, 1.5, d["ones"].size)
    p = EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"],
                   d["place_multi"], d["count_multi"], d["quats"], d["model_start"], scale=scale, **prob_kw)
    ref = ReferenceEngine(p, num_threads=1)
    orc = OracleEngine(p)
    for it in (1, 2, 3):
        a = ref.run_iteration(it)
        b = orc.run_iteration(it)
        for k in ("avg_likelihood", "mutual_info", "rms_change", "rescale"):
            assert a[k] == b[k], k
        for k in ("rmax", "info", "likelihood", "max_exp", "p_norm", "psum_d", "u", "model1", "model2"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        if p.need_scaling:
            np.testing.assert_array_equal(a["scale"], b["scale"])
    ref.close()


@pytest.mark.skipif(not reference_available(), reason="reference sources not compiled here")
def test_oracle_slice_ops_match_reference(oracle_built):
    prob, _ = load_case("beta1")
    ref = ReferenceEngine(prob, num_threads=1)
    orc = OracleEngine(prob)
    for r in (0, 17, 200, 419):
        np.testing.assert_array_equal(ref.slice_gen(prob.quats[r]), orc.slice_gen(prob.quats[r]))
    ref.close()


@pytest.mark.skipif(not reference_available(), reason="reference sources not compiled here")
def test_oracle_probability_lists_match_reference(oracle_built):
    """The kept (orientation, probability) lists of one iteration equal the
    reference's save_prob lists (max_prob.c:294-325) bit for bit."""
    prob, _ = load_case("scaling")
    ref = ReferenceEngine(prob, num_threads=1)
    orc = OracleEngine(prob)
    ref.set_save_prob(True)
    orc.set_save_prob(True)
    for it in (1, 2):
        a = ref.run_iteration(it)["sparse_prob"]
        b = orc.run_iteration(it)["sparse_prob"]
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
    ref.close()


_THREADS_SCRIPT = """
import sys, hashlib
import numpy as np
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[1] + "/tests")
from common import load_case
from oracle.oracle import OracleEngine
prob, _ = load_case("modes2")
eng = OracleEngine(prob)
h = hashlib.sha256()
for it in (1, 2):
    r = eng.run_iteration(it)
    for k in ("rmax", "likelihood", "p_norm", "psum_r", "model2_sum", "inter_weight", "model1"):
        h.update(np.ascontiguousarray(r[k]).tobytes())
print(h.hexdigest())
"""


def test_oracle_results_do_not_depend_on_its_thread_count(oracle_built):
    """The oracle parallelises only where every sum keeps its order (frames,
    orientations, and the merge's grid planes), so 1 and 5 OpenMP threads
    give the same bytes."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = []
    for n in ("1", "5"):
        env = dict(os.environ, OMP_NUM_THREADS=n)
        r = subprocess.run([sys.executable, "-c", _THREADS_SCRIPT, root], env=env, capture_output=True,
                           text=True, check=True)
        out.append(r.stdout.strip().splitlines()[-1])
    assert out[0] == out[1]


@pytest.mark.skipif(not reference_available(), reason="reference sources not compiled here")
def test_legacy_engine_driver_agrees_with_packaged_engine(oracle_built):
    """The legacy engine (src/max_emc.c through legacy_driver.c, the second
    timed CPU baseline) computes the same E-step as the packaged engine when
    every mask-0 pixel lies inside a positive model: the same average
    log-likelihood in the first iteration; the model differs only by the
    legacy update order (divide, then Friedel average: src/recon_emc.c:137-149
    against recon.pyx:120-140)."""
    from dragonfly_b200 import synth
    from oracle.oracle import LegacyEngine, legacy_available
    if not legacy_available():
        pytest.skip("legacy engine library not built")
    d = synth.small_problem(seed=17, det_side=28, size=33, qmax=15., n_atoms=80, atom_radius=6.,
                            num_div=2, n_frames=160, mean_count=40.)
    p = EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"],
                   d["place_multi"], d["count_multi"], d["quats"], d["model_start"], beta=0.3, need_scaling=1,
                   update_scale=1)
    ref = ReferenceEngine(p, num_threads=1)
    leg = LegacyEngine(p)
    try:
        a = ref.run_iteration(1)
        b = leg.run_iteration(1)
        assert abs(a["avg_likelihood"] - b) <= 1e-10 * abs(b), (a["avg_likelihood"], b)
        m = leg.model1()
        assert np.linalg.norm(m - a["model1"]) <= 0.05 * np.linalg.norm(a["model1"])
    finally:
        leg.close()
        ref.close()


@pytest.mark.skipif(not reference_available(), reason="reference sources not compiled here")
@pytest.mark.parametrize("seed,prob_kw", [
    (21, dict(beta=1.)),
    (22, dict(beta=0.05, beta_jump=2., beta_period=1, need_scaling=1, update_scale=1)),
    (23, dict(beta=0.3, need_scaling=1, update_scale=0, known_scale=1)),
])
def test_oracle_two_detectors_match_live_reference(seed, prob_kw, oracle_built):
    """Two detectors of different geometry and pixel count, each with its own
    dataset (the reference's in_detector_list: u, rescale, psum_r and the
    tomograms per detector, merges per orientation in detector order): the
    oracle against the reference engine run with both detectors, bit for
    bit, over three iterations."""
    p0, p1 = two_detector_problems(seed, **prob_kw)
    ref = ReferenceEngine(p0, num_threads=1)
    ref.add_detector(p1)
    orc = OracleEngine(p0, extra=[p1])
    assert ref.num_data == orc.det_of.size == p0.num_data + p1.num_data
    for it in (1, 2, 3):
        a = ref.run_iteration(it)
        b = orc.run_iteration(it)
        for k in ("avg_likelihood", "mutual_info", "rms_change"):
            assert a[k] == b[k], k
        np.testing.assert_array_equal(a["rescale_det"], b["rescale_det"])
        np.testing.assert_array_equal(a["mean_count_det"], b["mean_count_det"])
        np.testing.assert_array_equal(a["u_det"], b["u_det"])
        for k in ("rmax", "info", "likelihood", "max_exp", "p_norm", "psum_d", "model1", "model2", "beta"):
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        if p0.need_scaling:
            np.testing.assert_array_equal(a["scale"], b["scale"])
    # the two detectors see different things: their rescale factors differ
    assert abs(b["rescale_det"][0] - b["rescale_det"][1]) > 1e-3 * abs(b["rescale_det"][0])
    ref.close()


def test_oracle_matches_two_detector_golden(oracle_built):
    """The two-detector fixture (tests/golden/detectors2.npz, made by the
    reference engine run with both detectors): the oracle bit for bit, three
    iterations with scale updates."""
    import os
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "detectors2.npz"))
    pp = g["prob_params"]
    kw = dict(need_scaling=int(pp[0]), update_scale=int(pp[1]), known_scale=int(pp[2]), alpha=pp[3],
              beta=pp[4], beta_jump=pp[5], beta_period=int(pp[6]), beta_factor=pp[7])
    probs = [EMCProblem(*(g["d%d_%s" % (k, key)] for key in ("qvals", "corr", "mask", "ones", "multi",
                                                             "place_ones", "place_multi", "count_multi")),
                        g["quats"], g["model_start"], **kw) for k in (0, 1)]
    eng = OracleEngine(probs[0], extra=probs[1:])
    np.testing.assert_array_equal(eng.fcounts, g["fcounts"])
    np.testing.assert_array_equal(eng.sum_fact, g["sum_fact"])
    np.testing.assert_array_equal(eng.beta_start, g["beta_start"])
    for it in range(1, int(g["iters"]) + 1):
        r = eng.run_iteration(it)
        k = "it%d_" % it
        sc = g[k + "scalars"]
        assert (r["avg_likelihood"], r["mutual_info"], r["rms_change"]) == tuple(sc)
        np.testing.assert_array_equal(r["rescale_det"], g[k + "rescale_det"])
        np.testing.assert_array_equal(r["mean_count_det"], g[k + "mean_count_det"])
        np.testing.assert_array_equal(r["u_det"], g[k + "u_det"])
        for key in ("rmax", "info", "likelihood", "max_exp", "p_norm", "psum_d", "beta", "scale"):
            np.testing.assert_array_equal(r[key], g[k + key], err_msg=key)
        assert sha(r["model2_sum"]) == str(g[k + "model2_sum_sha256"])
        assert sha(r["inter_weight"]) == str(g[k + "weight_sha256"])
        assert sha(r["model1"]) == str(g[k + "model_sha256"])
    np.testing.assert_array_equal(r["model1"], g["final_model1"])
