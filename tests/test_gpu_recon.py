"""The reference-facing Python API end to end on the GPU: a config file,
Iterate, EMCRecon.run_iteration (recon.pyx:72-110), outputs and the log,
checked against the oracle on the same inputs."""
import os

import numpy as np
import pytest

from common import MODEL_REL_L2, SCALAR_REL, rel, rel_l2
from oracle.oracle import EMCProblem, OracleEngine
from test_api_host import write_problem

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("need_scaling", [0, 1])
def test_emcrecon_run_iteration_matches_oracle(tmp_path, need_scaling, oracle_built):
    from dragonfly_b200 import Iterate
    from dragonfly_b200.recon import EMCRecon
    d, cfg = write_problem(tmp_path, need_scaling=need_scaling, extra="update_scale = 1\n")
    itr = Iterate(cfg)
    start = itr.model.model1.copy()
    recon = EMCRecon()
    recon.set_iterate(itr)
    recon.save_initial_model()

    prob = EMCProblem(itr.dets[0].qvals, itr.dets[0].corr, itr.dets[0].raw_mask, d["ones"], d["multi"],
                      d["place_ones"], d["place_multi"], d["count_multi"], itr.quat.quats, start,
                      need_scaling=need_scaling, update_scale=1, beta=0.5, beta_jump=2., beta_period=3)
    orc = OracleEngine(prob)
    for it in (1, 2, 3, 4):
        itr.params.iteration = it
        ll = recon.run_iteration()
        b = orc.run_iteration(it)
        assert rel_l2(itr.model.model1, b["model1"]) <= MODEL_REL_L2
        assert rel(ll, b["avg_likelihood"]) <= SCALAR_REL
        assert rel(itr.mutual_info, b["mutual_info"]) <= SCALAR_REL
        assert np.mean(recon.rmax == b["rmax"]) >= 0.999
        np.testing.assert_allclose(itr.beta, b["beta"], rtol=0)
        if need_scaling:
            np.testing.assert_allclose(itr.scale, b["scale"], rtol=1e-6)
        assert abs(itr.rms_change - b["rms_change"]) <= 1e-5 * abs(b["rms_change"])
    out = itr.params.output_folder
    names = sorted(os.listdir(out))
    assert any(n.startswith("output_000") for n in names) and any(n.startswith("output_004") for n in names)
    log = open(itr.params.log_fname).read().splitlines()
    assert log[-1].split()[0] == "4" and "num_rot = 420" in "\n".join(log)
    recon.free()


def test_model_slice_api_on_gpu(oracle_built):
    from common import load_case
    from dragonfly_b200 import CDetector, Model
    prob, _ = load_case("beta1")
    det = CDetector()
    det.qvals, det.corr, det.raw_mask = prob.qvals, prob.corr, prob.mask
    m = Model(prob.size)
    m.model1 = prob.model1.copy()
    m.model2 = np.zeros_like(m.model1)
    m.inter_weight = np.zeros_like(m.model1)
    orc = OracleEngine(prob)
    s = m.slice_gen(prob.quats[3], det)
    np.testing.assert_array_equal(s, orc.slice_gen(prob.quats[3]))
    m.slice_merge(prob.quats[3], s, det)
    assert m.inter_weight.sum() > 0


def test_emcrecon_refinement_from_a_coarse_run(tmp_path, oracle_built):
    """num_div = "2 1" with probs_file naming a coarse run's output: the fine
    orientations map to their nearest coarse one (voronoi_subset) and each
    frame evaluates those whose coarse cell carries probability in the
    coarse run (src/iterate.c:103-130), checked against the reference engine
    with the same lists."""
    from dragonfly_b200 import Iterate
    from dragonfly_b200.recon import EMCRecon
    from oracle.oracle import ReferenceEngine, reference_available, voronoi_subset_reference
    if not reference_available():
        pytest.skip("reference engine library not built")
    d, cfg = write_problem(tmp_path, extra="save_prob = 1\n")
    text = open(cfg).read()
    open(cfg, "w").write(text.replace("num_div = 2", "num_div = 1"))
    itr = Iterate(cfg)
    recon = EMCRecon()
    recon.set_iterate(itr)
    for it in (1, 2):
        itr.params.iteration = it
        recon.run_iteration()
    coarse_out = [n for n in os.listdir(itr.params.output_folder) if n.startswith("output_002")][0]
    recon.free()

    fine_cfg = tmp_path / "fine.ini"
    fine_cfg.write_text(text.replace("num_div = 2", "num_div = 2 1").replace("save_prob = 1", "")
                        .replace("output_folder = out/", "output_folder = fine/")
                        .replace("log_file = out/EMC.log", "log_file = fine/EMC.log")
                        + "probs_file = out/%s\n" % coarse_out)
    itr = Iterate(str(fine_cfg))
    assert itr.params.refine and itr.quat.num_rot == 420 and itr.quat.num_rot_coarse == 60
    np.testing.assert_array_equal(itr.quat.quat_mapping, voronoi_subset_reference(1, itr.quat.quats))
    assert len(itr.rel_quat) == d["ones"].size and sum(len(x) for x in itr.rel_quat) > d["ones"].size
    start = itr.model.model1.copy()
    recon = EMCRecon()
    recon.set_iterate(itr)
    prob = EMCProblem(itr.dets[0].qvals, itr.dets[0].corr, itr.dets[0].raw_mask, d["ones"], d["multi"],
                      d["place_ones"], d["place_multi"], d["count_multi"], itr.quat.quats, start,
                      beta=0.5, beta_jump=2., beta_period=3)
    ref = ReferenceEngine(prob)
    ref.set_refinement(itr.quat.quat_mapping, itr.rel_quat)
    for it in (1, 2):
        itr.params.iteration = it
        ll = recon.run_iteration()
        b = ref.run_iteration(it)
        assert rel_l2(itr.model.model1, b["model1"]) <= MODEL_REL_L2
        assert rel(ll, b["avg_likelihood"]) <= SCALAR_REL
        assert np.mean(recon.rmax == b["rmax"]) >= 0.999
        assert all(r < 0 or itr.quat.quat_mapping[r] in itr.rel_quat[i] for i, r in enumerate(recon.rmax))
    recon.free()
    ref.close()


def test_emcrecon_2d_from_config(tmp_path, oracle_built):
    """recon_type = 2d: the detector's q vectors projected to the detector
    plane (CDetector._convert_2d, detector.pyx:128-134), num_rot in-plane
    angles over [0, pi) with friedel_sym (quaternion.pyx:70-74), a
    [modes, S, S] image, and the iteration against the reference engine."""
    from dragonfly_b200 import Iterate
    from dragonfly_b200.recon import EMCRecon
    from oracle.oracle import ReferenceEngine, reference_available
    if not reference_available():
        pytest.skip("reference engine library not built")
    d, cfg = write_problem(tmp_path, extra="recon_type = 2d\nnum_rot = 48\nfriedel_sym = 1\n")
    itr = Iterate(cfg)
    assert itr.model.mtype == "MODEL_2D" and itr.model.model1.ndim == 3
    assert itr.quat.num_rot == 48 and itr.quat.quats[:, 0].max() < np.pi
    assert np.abs(itr.dets[0].qvals[:, :2]).max() > np.abs(d["qvals"][:, :2]).max()   # pixel units
    start = itr.model.model1.copy()
    recon = EMCRecon()
    recon.set_iterate(itr)
    prob = EMCProblem(itr.dets[0].qvals, itr.dets[0].corr, itr.dets[0].raw_mask, d["ones"], d["multi"],
                      d["place_ones"], d["place_multi"], d["count_multi"], itr.quat.quats, start,
                      beta=0.5, beta_jump=2., beta_period=3, model_type="2d", friedel_sym=1)
    ref = ReferenceEngine(prob)
    for it in (1, 2, 3):
        itr.params.iteration = it
        ll = recon.run_iteration()
        b = ref.run_iteration(it)
        assert rel_l2(itr.model.model1, b["model1"]) <= MODEL_REL_L2
        assert rel(ll, b["avg_likelihood"]) <= SCALAR_REL
        assert np.mean(recon.rmax == b["rmax"]) >= 0.999
    recon.free()
    ref.close()
