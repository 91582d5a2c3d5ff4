"""Several detectors in one reconstruction (dfg_group_*, the reference's
in_detector_list) against the oracle's restatement with two detectors, which
is pinned bit for bit to the reference engine run with two detectors
(tests/test_oracle.py). Per detector: u and the rescale factor; shared: the
model after each iteration, the average log-likelihood and mutual
information over all frames, the per-frame most likely orientations and
scale factors, at the plain form's parity bar."""
import numpy as np
import pytest

from common import MODEL_REL_L2, SCALAR_REL, SCALE_REL, two_detector_problems
from oracle.oracle import OracleEngine

pytestmark = pytest.mark.gpu


def _group(probs, orc, **options):
    from dragonfly_b200._lib import Context, DetectorGroup
    ctxs, o = [], 0
    for p in probs:
        c = Context(0)
        for k, v in options.items():
            c.set_option(k, v)
        c.set_detector(p.qvals, p.corr, p.mask)
        c.set_frames(p.ones, p.multi, p.place_ones, p.place_multi, p.count_multi)
        c.set_quaternions(p.quats)
        c.set_model(p.model1)
        if p.scale is not None:
            c.set_scale(p.scale)
        # calc_beta over all detectors' frames (iterate.c:66-83: the
        # empirical start from detector 0's mean count)
        c.set_beta_start(orc.beta_start[o:o + p.num_data])
        o += p.num_data
        ctxs.append(c)
    return ctxs, DetectorGroup(ctxs)


def _rel(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


@pytest.mark.parametrize("seed,prob_kw", [
    (21, dict(beta=1.)),
    (22, dict(beta=0.05, beta_jump=2., beta_period=1, need_scaling=1, update_scale=1)),
    (23, dict(beta=0.3, need_scaling=1, update_scale=0, known_scale=1, alpha=0.25)),
])
def test_two_detectors_match_oracle(seed, prob_kw, oracle_built):
    probs = two_detector_problems(seed, **prob_kw)
    p0 = probs[0]
    orc = OracleEngine(p0, extra=probs[1:])
    ctxs, g = _group(probs, orc)
    for it in (1, 2, 3):
        par = ctxs[0].params(it, p0.need_scaling, p0.update_scale, p0.known_scale, p0.beta_jump, p0.beta_period,
                             p0.beta_factor)
        out = g.run_iteration(par, p0.alpha)
        b = orc.run_iteration(it)
        fr = g.frame_results()
        dev = dict(model=_rel(g.model()[0], b["model1"]),
                   ll=abs(out["avg_likelihood"] - b["avg_likelihood"]) / abs(b["avg_likelihood"]),
                   mi=abs(out["mutual_info"] - b["mutual_info"]) / max(abs(b["mutual_info"]), 1e-300),
                   rmax=float(np.mean(fr["rmax"] == b["rmax"])),
                   rescale=max(abs(c.scalars()["rescale"] - r) / r for c, r in zip(ctxs, b["rescale_det"])),
                   u=max(_rel(c.orientation_results()[0], u) for c, u in zip(ctxs, b["u_det"])))
        print("iteration %d:" % it, dev)
        assert dev["model"] <= MODEL_REL_L2 and dev["ll"] <= SCALAR_REL and dev["mi"] <= SCALAR_REL, dev
        # u_r: the device sums FP64 slice values over pixels in another
        # order (and iteration 2's model carries the merge's deviation)
        assert dev["rmax"] >= 0.99 and dev["rescale"] <= 1e-7 and dev["u"] <= 1e-7, dev
        if p0.need_scaling:
            sc = np.concatenate([c.frame_params()["scale"] for c in ctxs])
            assert np.max(np.abs(sc - b["scale"]) / b["scale"]) <= SCALE_REL
        # every member holds the shared model
        np.testing.assert_array_equal(ctxs[1].model()[0], g.model()[0])
    g.close()
    for c in ctxs:
        c.close()


def test_group_of_one_detector_equals_the_context(oracle_built):
    """A group with one member runs the same iteration as the context alone."""
    from common import load_case
    from dragonfly_b200._lib import Context, DetectorGroup
    prob, _ = load_case("scaling")
    outs = []
    for grouped in (False, True):
        c = Context(0)
        c.set_option("graph", 0)
        c.set_detector(prob.qvals, prob.corr, prob.mask)
        c.set_frames(prob.ones, prob.multi, prob.place_ones, prob.place_multi, prob.count_multi)
        c.set_quaternions(prob.quats)
        c.set_model(prob.model1)
        c.calc_beta(prob.beta, prob.need_scaling)
        g = DetectorGroup([c]) if grouped else None
        for it in (1, 2):
            par = c.params(it, prob.need_scaling, prob.update_scale, prob.known_scale, prob.beta_jump,
                           prob.beta_period, prob.beta_factor)
            out = g.run_iteration(par, prob.alpha) if grouped else c.run_iteration(par, prob.alpha)
        outs.append((out, c.model()[0], c.frame_params()["scale"]))
        if g is not None:
            g.close()
        c.close()
    (a, ma, sa), (b, mb, sb) = outs
    assert abs(a["avg_likelihood"] - b["avg_likelihood"]) <= 1e-12 * abs(a["avg_likelihood"])
    assert _rel(mb, ma) <= 1e-12 and _rel(sb, sa) <= 1e-12


def test_group_rejects_mismatched_members(oracle_built):
    from dragonfly_b200._lib import Context, DetectorGroup, DFGError
    probs = two_detector_problems(24, beta=1.)
    ctxs = []
    for k, p in enumerate(probs):
        c = Context(0)
        c.set_detector(p.qvals, p.corr, p.mask)
        c.set_frames(p.ones, p.multi, p.place_ones, p.place_multi, p.count_multi)
        c.set_quaternions(p.quats if k == 0 else p.quats[:-1])
        c.set_model(p.model1)
        c.calc_beta(1., 0)
        ctxs.append(c)
    g = DetectorGroup(ctxs)
    with pytest.raises(DFGError, match="orientation count"):
        g.maximize(ctxs[0].params(1))
    g.close()
    for c in ctxs:
        c.close()


def test_emcrecon_detector_list_matches_oracle(tmp_path, oracle_built):
    """EMCRecon on an Iterate read from a config with in_detector_list and
    in_photons_list (file i seen by detector i; detector 0 is the file name
    first in sorted order, here the second file's): two iterations against
    the oracle with the same detectors, frames and start model."""
    from dragonfly_b200 import Detector, Iterate, synth
    from dragonfly_b200.recon import EMCRecon
    from dragonfly_b200.emcfile import write_emc
    from oracle.oracle import EMCProblem
    dets, sh = synth.two_detector_problem(seed=8, n_frames=(300, 200))
    names = ["det_z.npz", "det_a.npz"]
    for k, dd in enumerate(dets):
        det = Detector()
        det.qvals, det.corr, det.raw_mask = dd["qvals"], dd["corr"], dd["mask"]
        det.detd, det.ewald_rad = dd["detd"], 1.
        det.write(str(tmp_path / names[k]))
        write_emc(str(tmp_path / ("photons%d.emc" % k)), dd["qvals"].shape[0], dd["ones"], dd["multi"],
                  dd["place_ones"], dd["place_multi"], dd["count_multi"])
    (tmp_path / "dets.txt").write_text("\n".join(names) + "\n")
    (tmp_path / "photons.txt").write_text("photons0.emc\nphotons1.emc\n")
    (tmp_path / "config.ini").write_text("""[emc]
in_photons_list = photons.txt
in_detector_list = dets.txt
num_div = 2
output_folder = out/
log_file = out/EMC.log
beta = 0.5
need_scaling = 1
""")
    itr = Iterate(str(tmp_path / "config.ini"))
    assert itr.num_det == 2
    model0 = itr.model.model1.copy()
    # the oracle: detector 0 (det_a, the second file's frames) first
    probs = []
    for k, src in ((0, 1), (1, 0)):
        dt, dd = itr.dets[k], dets[src]
        probs.append(EMCProblem(dt.qvals, dt.corr, dt.raw_mask, dd["ones"], dd["multi"], dd["place_ones"],
                                dd["place_multi"], dd["count_multi"], itr.quat.quats, model0, beta=0.5,
                                need_scaling=1, update_scale=1))
    orc = OracleEngine(probs[0], extra=probs[1:])
    perm = np.concatenate([itr.member_index(0), itr.member_index(1)])   # oracle frame -> global frame
    recon = EMCRecon()
    recon.set_iterate(itr)
    for it in (1, 2):
        itr.params.iteration = it
        recon.run_iteration()
        b = orc.run_iteration(it)
        dev = _rel(itr.model.model1, b["model1"])
        agree = float(np.mean(recon.rmax[perm] == b["rmax"]))
        ll = abs(itr.likelihood - b["avg_likelihood"]) / abs(b["avg_likelihood"])
        print("iteration %d: model %.2e, rmax %.4f, log-likelihood %.2e, rescale %s / %s"
              % (it, dev, agree, ll, itr.rescale, b["rescale_det"]))
        assert dev <= MODEL_REL_L2 and agree >= 0.99 and ll <= SCALAR_REL
        np.testing.assert_allclose(itr.rescale, b["rescale_det"], rtol=1e-9)
        np.testing.assert_allclose(itr.scale[perm], b["scale"], rtol=SCALE_REL)
        assert len(recon.u) == 2
    assert (tmp_path / "out" / "EMC.log").exists()
    recon.free()
