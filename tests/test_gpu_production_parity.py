"""Parity at the benchmarked geometries, on frame subsets the oracle finishes
in about a minute per iteration.

* Plain form at the production workload (the one bench.py times): 260 x 257
  pnCCD-like detector (66820 pixels, 6-row gap, radius-10 hole), 201^3 model,
  all 50100 orientations (num_div 10), lognormal fluence (median 300 photons,
  sigma 0.5), need_scaling and update_scale on, beta 0.01 x sqrt(2) every 5
  iterations; 1024 frames simulated by the library, iterations 1, 2 and 11
  (beta 0.01, 0.01 with the scale factors in the likelihood, 0.02).
* Tensor-core form at the precision workload: the same detector and model,
  86520 orientations (num_div 12), median 1500 photons (sigma 0.3); 384
  frames, both the E-step photon term and the tomogram update as BF16 hi/lo
  tcgen05 products; the model, per-frame log-likelihood and per-frame
  probabilities compared with the FP64 oracle, within the form's own stated
  error bounds.

The oracle is bit-identical to the reference engine with one thread
(tests/test_oracle.py), at any thread count of its own.
"""
import math

import pytest

from oracle.parity import BAR, compare_runs, simulated_subset

pytestmark = pytest.mark.gpu


def _inputs(**override):
    from bench import WORKLOAD, build_inputs
    w = dict(WORKLOAD)
    w.update(override)
    return w, build_inputs(w)


def test_production_workload_subset_matches_oracle(oracle_built):
    w, inp = _inputs()
    assert inp["quats"].shape[0] == 50100 and inp["qvals"].shape[0] == 66820
    prob = simulated_subset(inp, w, 1024, seed=31)
    devs = compare_runs(prob, (1, 2, 11), graph=True)
    print("production workload, 1024 frames x 50100 orientations:", devs)
    assert [round(d["beta"], 6) for d in devs] == [0.01, 0.01, round(0.01 * math.sqrt(2.) ** 2, 6)]
    for d in devs:
        assert d["within_bar"], d
        assert d["model_rel_l2"] <= BAR["model_rel_l2"]


def test_precision_workload_dense_subset_matches_oracle(oracle_built):
    """Errors of the tensor-core form against the FP64 oracle at the
    precision workload's geometry and fluence. The log-slices enter the
    products as BF16 hi + lo (|x - hi - lo| <= 2^-17 |x|), so a frame of 1500
    photons carries an absolute log-likelihood error of order
    1500 x 2^-17 x |log W| (about 0.1 nats): the form has its own error
    profile, stated here (measured: model 3.7e-7, average log-likelihood 9e-6,
    mutual information 2.2e-5, per-frame log-likelihood 1.5e-5, per-pair
    probabilities 1e-8 absolute and 2e-5 per frame in L1, most likely
    orientation 99.2-99.7 %) and bounded with margin."""
    w, inp = _inputs(num_div=12, median_photons=1500., fluence_sigma=0.3, n_frames=100000)
    assert inp["quats"].shape[0] == 86520
    prob = simulated_subset(inp, w, 384, seed=32)
    devs = compare_runs(prob, (1, 2), probabilities=True, estep_form=1, mstep_form=1)
    print("precision workload (tensor-core form), 384 frames x 86520 orientations:", devs)
    for d in devs:
        assert d["model_rel_l2"] <= 2e-6, d
        assert d["ll_rel"] <= 3e-5 and d["mi_rel"] <= 1e-4, d
        assert d["frame_ll_max_rel"] <= 5e-5, d
        assert d["rmax_agree"] >= 0.98, d
        assert d["scale_rel"] <= 1e-6, d
        assert d["prob_max_abs"] <= 1e-6 and d["prob_l1_mean"] <= 1e-4, d
