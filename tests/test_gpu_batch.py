"""Batches of independent reconstructions (dfg_batch_run): every context's
iteration as one branch of a single CUDA graph. Each reconstruction's results
equal those of running it alone (up to the run-to-run order of the merge's
FP64 atomics)."""
import numpy as np
import pytest

from common import GPUEngine, load_case, rel_l2

pytestmark = pytest.mark.gpu


def _problems():
    from dragonfly_b200 import synth
    from oracle.oracle import EMCProblem
    probs = [load_case(c)[0] for c in ("beta1", "scaling", "modes2")]
    d = synth.small_problem_2d(seed=8)
    probs.append(EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"],
                            d["place_multi"], d["count_multi"], d["quats"], d["model_start"], beta=1.,
                            model_type="2d"))
    return probs


def _params(c, p, it):
    return c.params(it, p.need_scaling, p.update_scale, p.known_scale, p.beta_jump, p.beta_period, p.beta_factor)


@pytest.mark.parametrize("keep_prob", [0, 1])
def test_batch_equals_separate_runs(oracle_built, keep_prob):
    from dragonfly_b200._lib import Batch
    probs = _problems()
    alone = [GPUEngine(p) for p in probs]
    batched = [GPUEngine(p, keep_prob=keep_prob if i == 1 else 0) for i, p in enumerate(probs)]
    batch = Batch([e.ctx for e in batched])
    for it in (1, 2, 3):
        outs = batch.run([_params(e.ctx, p, it) for e, p in zip(batched, probs)], [p.alpha for p in probs])
        for p, a, e, o in zip(probs, alone, batched, outs):
            r = a.ctx.run_iteration(_params(a.ctx, p, it), p.alpha)
            m_a, _, _ = a.ctx.model()
            m_b, _, _ = e.ctx.model()
            assert rel_l2(m_b, m_a) <= 1e-10
            assert abs(o["avg_likelihood"] - r["avg_likelihood"]) <= 1e-10 * abs(r["avg_likelihood"])
            assert np.mean(e.ctx.frame_results()["rmax"] == a.ctx.frame_results()["rmax"]) >= 0.999
    st = batch.stats()
    if keep_prob:
        assert st["launches"] == 0          # the keep_prob context needs the host: no graph
    else:
        assert st["launches"] == 3 and st["instantiations"] == 1, st
    batch.close()
    for e in alone + batched:
        e.close()
