"""The whole iteration as one CUDA graph (dfg_run_iteration): the same
kernels as the step-wise calls (maximize, update_model, normalize_scale), so
the results agree to the run-to-run spread of the merge's FP64 atomic
additions (their order varies between any two runs, ~1e-15 relative); later
iterations update the captured graph in place rather than instantiating it
again."""
import numpy as np
import pytest

from common import GPUEngine, load_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["beta1", "scaling"])
def test_graph_iteration_equals_stepwise(oracle_built, case):
    prob, _ = load_case(case)
    step = GPUEngine(prob)
    graph = GPUEngine(prob)
    plain = GPUEngine(prob, graph=0)
    for it in (1, 2, 3):
        a = step.run_iteration(it)
        outs = []
        for eng in (graph, plain):
            c = eng.ctx
            par = c.params(it, prob.need_scaling, prob.update_scale, prob.known_scale, prob.beta_jump,
                           prob.beta_period, prob.beta_factor)
            outs.append(c.run_iteration(par, prob.alpha))
        for eng, o in zip((graph, plain), outs):
            m1, _, _ = eng.ctx.model()
            np.testing.assert_allclose(m1, a["model1"], rtol=1e-10, atol=1e-12 * np.abs(a["model1"]).max())
            fr = eng.ctx.frame_results()
            assert np.mean(fr["rmax"] == a["rmax"]) >= 0.999
            for k in ("avg_likelihood", "rms_change", "mutual_info"):
                assert abs(o[k] - a[k]) <= 1e-10 * abs(a[k]), (k, o[k], a[k])
            if prob.need_scaling:
                np.testing.assert_allclose(eng.ctx.frame_params()["scale"], a["scale"], rtol=1e-10)
    st = graph.ctx.graph_stats()
    assert st["launches"] == 3 and st["instantiations"] == 1 and st["updates"] == 2, st
    assert plain.ctx.graph_stats()["launches"] == 0
    for e in (step, graph, plain):
        e.close()


def test_graph_phase_timing(oracle_built):
    """Phase timing (option timing) inside the captured graph: every phase of
    the iteration is timed, from event records in the graph."""
    prob, _ = load_case("scaling")
    g = GPUEngine(prob, timing=1)
    c = g.ctx
    for it in (1, 2):
        par = c.params(it, prob.need_scaling, prob.update_scale, prob.known_scale, prob.beta_jump,
                       prob.beta_period, prob.beta_factor)
        c.run_iteration(par, prob.alpha)
    ph = c.phase_times()
    assert c.graph_stats()["launches"] == 2
    for k in ("slice", "estep", "norm", "psum", "mstep", "merge", "update"):
        ms, n = ph[k]
        assert ms > 0. and n > 0, (k, ph[k])
    # the step-wise calls time the same phases outside a graph
    c.reset_phase_times()
    par = c.params(3, prob.need_scaling, prob.update_scale, prob.known_scale, prob.beta_jump,
                   prob.beta_period, prob.beta_factor)
    c.maximize(par)
    c.update_model(prob.alpha)
    c.normalize_scale()
    ph2 = c.phase_times()
    for k in ("slice", "estep", "norm", "psum", "mstep", "merge", "update"):
        assert ph2[k][0] > 0. and ph2[k][1] == ph[k][1] // 2, (k, ph2[k], ph[k])
    g.close()
