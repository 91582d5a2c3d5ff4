"""Dense (tensor-core) form of the E-step photon term against the sparse form
and the FP64 oracle.

The dense form computes sum_k count * logW as BF16 products of the hi / lo
split of the log-slices (|x - hi - lo| <= 2^-17 |x|) with FP32 accumulation,
so each log-likelihood carries an absolute error of order 1e-4 x the photon
count; the bounds below state what that does to every reported result.
"""
import numpy as np
import pytest

from common import GPUEngine, load_case, rel_l2
from oracle.oracle import EMCProblem, OracleEngine

pytestmark = pytest.mark.gpu

# measured on these cases: <= 5e-6 per photon, 8.5e-7, 6.3e-6, 1.0
MAXEXP_ABS_PER_PHOTON = 2e-5   # |max_r pval| error per photon of the frame
LL_REL = 5e-6                  # average log-likelihood
MODEL_REL_L2 = 5e-5            # model after each iteration, against the oracle
RMAX_AGREE = 0.999             # most likely orientation


def _synth():
    from dragonfly_b200 import synth
    d = synth.small_problem(seed=21, det_side=48, size=41, qmax=19., n_atoms=120, atom_radius=7., num_div=4,
                            n_frames=700, mean_count=300., hole_radius=3.)
    return EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"], d["place_multi"],
                      d["count_multi"], d["quats"], d["model_start"], beta=1.)


@pytest.mark.parametrize("forms", [(1, 0), (0, 1), (1, 1)], ids=["estep", "mstep", "both"])
@pytest.mark.parametrize("case", ["beta1", "scaling", "modes2", "synth300"])
def test_dense_estep_matches_sparse_and_oracle(oracle_built, case, forms):
    prob = _synth() if case == "synth300" else load_case(case)[0]
    sparse = GPUEngine(prob)
    dense = GPUEngine(prob, estep_form=forms[0], mstep_form=forms[1])
    orc = OracleEngine(prob)
    mo = np.concatenate([[0], np.cumsum(prob.multi)])
    cm = np.concatenate([[0], np.cumsum(prob.count_multi)])
    photons = np.asarray(prob.ones, np.float64) + (cm[mo[1:]] - cm[mo[:-1]])
    for it in (1, 2):
        a = dense.run_iteration(it)
        b = sparse.run_iteration(it)
        o = orc.run_iteration(it)
        good = np.asarray(b["rmax"]) >= 0
        mx = np.abs(np.asarray(a["max_exp"]) - np.asarray(b["max_exp"]))[good]
        per_photon = float((mx / np.maximum(photons[good], 1.)).max())
        ll = abs(a["avg_likelihood"] - o["avg_likelihood"]) / abs(o["avg_likelihood"])
        dev = rel_l2(a["model1"], o["model1"])
        dev_sparse = rel_l2(b["model1"], o["model1"])
        agree = float(np.mean(np.asarray(a["rmax"]) == np.asarray(o["rmax"])))
        print("dense %s %s iteration %d: max_exp %.2e / photon, ll %.2e, model %.2e (sparse %.2e), rmax %.4f"
              % (forms, case, it, per_photon, ll, dev, dev_sparse, agree))
        assert per_photon <= MAXEXP_ABS_PER_PHOTON, per_photon
        assert ll <= LL_REL and dev <= MODEL_REL_L2 and agree >= RMAX_AGREE, (ll, dev, agree)
        # both engines continue from the oracle's model, so the errors do not compound
        for e in (dense, sparse):
            e.ctx.set_model(o["model1"])
            if prob.need_scaling:
                e.ctx.set_scale(o["scale"])
    for e in (dense, sparse):
        e.close()


@pytest.mark.parametrize("case", ["scaling", "synth300"])
def test_autotuner_times_both_forms_and_keeps_the_fastest(oracle_built, case):
    prob = _synth() if case == "synth300" else load_case(case)[0]
    tuned = GPUEngine(prob, autotune=1)
    c = tuned.ctx
    par = c.params(1, prob.need_scaling, prob.update_scale, prob.known_scale, prob.beta_jump, prob.beta_period,
                   prob.beta_factor)
    rep = c.autotune(par)
    print("autotune %s:" % case, rep)
    assert set(rep["slice_ms"]) == {128, 64, 32, 16} and all(v > 0 for v in rep["slice_ms"].values())
    assert rep["slice_block"] == min(rep["slice_ms"], key=rep["slice_ms"].get)
    assert rep["estep_sparse_ms"] > 0 and rep["estep_dense_ms"] is not None and rep["estep_dense_ms"] > 0
    assert rep["estep_form"] == int(rep["estep_dense_ms"] < rep["estep_sparse_ms"])
    assert rep["mstep_sparse_ms"] > 0 and rep["mstep_dense_ms"] > 0
    assert rep["mstep_form"] == int(rep["mstep_dense_ms"] < rep["mstep_sparse_ms"])
    # where the sparse gathers win, their resident blocks per SM are tuned too
    if rep["estep_form"] == 0:
        t = rep["estep_ms_by_blocks_per_sm"]
        assert set(t) == {2, 3, 4} and rep["estep_blocks_per_sm"] == min(t, key=t.get)
    if rep["mstep_form"] == 0:
        t = rep["mstep_ms_by_blocks_per_sm"]
        assert set(t) == {3, 4, 5} and rep["mstep_blocks_per_sm"] == min(t, key=t.get)
    # iterations with the tuned choice agree with the plain sparse form
    plain = GPUEngine(prob)
    orc = OracleEngine(prob)
    for it in (1, 2):
        a = tuned.run_iteration(it)
        b = orc.run_iteration(it)
        assert rel_l2(a["model1"], b["model1"]) <= MODEL_REL_L2
        assert np.mean(np.asarray(a["rmax"]) == np.asarray(b["rmax"])) >= RMAX_AGREE
    tuned.close()
    plain.close()


@pytest.mark.parametrize("forms", [(1, 0), (0, 1)], ids=["estep", "mstep"])
def test_dense_pipeline_wait_gives_up_and_the_context_recovers(oracle_built, forms):
    """Failure detection of the tensor-core kernels without a GPU fault: with
    one stage's copies withheld (test hook) every wait on that stage runs out
    after a short limit, the kernels set the error flag, drain their copies,
    free their TMEM and return, and maximize reports DFG_ERR_CUDA; the next
    call on the same context, with the hook off, succeeds and matches the
    oracle."""
    from dragonfly_b200._lib import DFG_ERR_CUDA, DFGError
    prob = _synth()
    gpu = GPUEngine(prob, estep_form=forms[0], mstep_form=forms[1])
    c = gpu.ctx
    par = c.params(1, prob.need_scaling, prob.update_scale, prob.known_scale, prob.beta_jump, prob.beta_period,
                   prob.beta_factor)
    c.set_option("dense_wait_cycles", 2e7)        # about 10 ms per wait
    c.set_option("dense_withhold_stage", 1)
    with pytest.raises(DFGError) as e:
        c.maximize(par)
    assert e.value.code == DFG_ERR_CUDA and "gave up" in str(e.value)
    c.set_option("dense_withhold_stage", -1)
    c.set_option("dense_wait_cycles", 2e9)
    a = gpu.run_iteration(1)
    b = OracleEngine(prob).run_iteration(1)
    assert rel_l2(a["model1"], b["model1"]) <= MODEL_REL_L2
    assert np.mean(np.asarray(a["rmax"]) == np.asarray(b["rmax"])) >= RMAX_AGREE
    gpu.close()
