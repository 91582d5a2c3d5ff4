"""Learned orientation proposals end to end: the network trained on frames
simulated from the model at known orientations, frames restricted to their
top-K coarse cells, a held-out share searched in full and watched. Against a
full search over the same frames from the same model: the captured
probability mass, the most likely orientations and the model, and what the
network gains over proposals without it (random cells). A first full
search retrains the network on its probabilities per coarse cell; the next
proposal iterations then capture more than the threshold and each must stay
within 1e-3 (model) and 99 % (most likely orientations) of a full search
from the same state. The proposals are mass-covering: at least K cells per
frame, more (up to K_max) where the network's probabilities of the frame's
cells fall short of a target mass. The network trains on the tensor cores
(mixed precision)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("pair_lists", [False, True])
def test_learned_proposals_against_full_search(pair_lists):
    from dragonfly_b200 import synth
    from dragonfly_b200._lib import Context
    from dragonfly_b200.proposals import LearnedProposals, sort_by_coarse
    from dragonfly_b200.quatgen import quat_gen
    d = synth.small_problem(seed=9, det_side=64, size=61, qmax=29., n_atoms=200, atom_radius=10., num_div=6,
                            n_frames=4000, mean_count=300., hole_radius=3.)
    ctxs = []
    for k in range(2):
        c = Context(0)
        c.set_detector(d["qvals"], d["corr"], d["mask"])
        c.set_frames(d["ones"], d["multi"], d["place_ones"], d["place_multi"], d["count_multi"])
        ctxs.append(c)
    full, restr = ctxs
    fine, _, qmap = sort_by_coarse(quat_gen(6), 2, full)
    for c in ctxs:
        c.set_quaternions(fine)
        c.set_model(d["model_true"][None])
        c.calc_beta(1., 0)
    # a 64 x 64 detector and 420 classes: the whole detector as the image and
    # a larger rate than the production detector's 3240 classes want
    # at least 24 cells per frame, more where the network is unsure, until
    # its probabilities of the frame's cells reach 0.999999 (at most 128).
    # Measured on this case (one B200), after the first full search and the
    # retraining on it: the model within 6.6-8.4e-4 of a full search from the
    # same state, most likely orientations 99.88-99.975 %, 16.7-18 % of the
    # pairs evaluated, captured mass 0.9995-0.9998. At 0.99999 the retrained
    # network's proposals hold 11.6-12.2 % of the pairs and the model stays
    # 1.0-1.3e-3 away (so does a fixed 24 cells, 7.6 %, at 0.9985-0.999
    # captured mass): an orientation whose probability comes mostly from
    # frames that did not propose it gets another tomogram, and every merged
    # tomogram weighs the same in the model
    lp = LearnedProposals(restr, d["qvals"], fine, coarse_div=2, K=24, held_out=0.02, threshold=0.99, seed=1,
                          pair_lists=pair_lists, zoom=1.0, retrain_epochs=40, K_max=128, mass=0.999999)
    loss = lp.train_simulated(d["model_true"], n_frames=30000, epochs=4, lr=2e-3)
    # the network's gain: top-K hit rate of the true orientations' cells
    cells = full.voronoi_subset(quat_gen(2), np.pad(d["frame_quats"][:, :4], ((0, 0), (0, 1))))
    lp.net.load_frames(restr)
    top = lp.net.topk(lp.K)
    hit = float(np.mean([cells[i] in top[i] for i in range(len(cells))]))
    chance = lp.K / lp.nc
    print("training loss %.3f; top-%d hit rate %.3f (random cells %.3f)" % (loss, lp.K, hit, chance))
    assert hit >= 0.9 and hit > 10 * chance
    # the first iteration is a full search: the network is retrained on its
    # probabilities per coarse cell (simulated frames alone leave 25 of the
    # full search's orientations without a frame that proposes them here)
    lp.full_next = True
    masses, devs = [], []
    for it in (1, 2, 3, 4):
        # both iterations start from the proposal context's model, so that the
        # comparison is one proposal (or fallback) iteration against one full
        # search from the same state
        m0, _, _ = restr.model()
        full.set_model(m0)
        par = full.params(it)
        t0 = time.time()
        a = full.run_iteration(par, 0.)
        t1 = time.time()
        b = lp.iteration(restr.params(it), 0.)
        t2 = time.time()
        ma, _, _ = full.model()
        mb, _, _ = restr.model()
        dev = float(np.linalg.norm(ma - mb) / np.linalg.norm(ma))
        agree = float(np.mean(full.frame_results()["rmax"] == restr.frame_results()["rmax"]))
        print("iteration %d (%s): captured mass %s, evaluated %.3f of the pairs, model %.2e, rmax %.4f, "
              "full %.0f ms, proposal %.0f ms" % (it, b["mode"], b["captured_mass"], b["evaluated_fraction"], dev,
                                                 agree, 1e3 * (t1 - t0), 1e3 * (t2 - t1)))
        if b["mode"] == "proposal":
            masses.append(b["captured_mass"])
            assert b["evaluated_fraction"] < 0.35
            if b["captured_mass"] >= lp.threshold:
                devs.append(dev)
                # the bar: within 1e-3 of a full search from the same state,
                # most likely orientations >= 99 %
                assert dev <= 1e-3 and agree >= 0.99, (dev, agree)
            else:
                assert lp.full_next          # the next iteration falls back to full search
    print("captured mass per proposal iteration:", ["%.4f" % m for m in masses])
    assert len(devs) >= 3 and masses[-1] >= lp.threshold, (masses, devs)
    lp.close()
    for c in ctxs:
        c.close()
