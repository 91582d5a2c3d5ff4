"""The GPU frame simulator (dfg_simulate_frames) against the rules of the
reference's gen_and_save_dataset (dragonfly/utils/src/make_data.c:115-326):
a slice of the intensity at the frame's orientation times the frame's scale
is the Poisson mean of every pixel with mask <= 1 (make_data.c:182-189);
count-1 pixels go to place_ones and larger counts to place_multi /
count_multi (:191-198), pixels in ascending order within a frame.

The Poisson means come from the oracle's slice (orc_slice_gen3d, FP64, the
reference's geometry), so the checks are statistical: z-scores of per-pixel
means and per-frame totals against their Poisson spread.
"""
import numpy as np
import pytest

from oracle.oracle import EMCProblem, OracleEngine

pytestmark = pytest.mark.gpu


def _setup(seed=3):
    from dragonfly_b200 import synth
    from dragonfly_b200._lib import Context
    rng = np.random.default_rng(seed)
    size = 33
    intens = synth.gaussian_atom_intensity(80, 6., size, rng)
    qvals, corr, mask, _, _ = synth.flat_detector(32, 32, 15., size, hole_radius=3.)
    ctx = Context(0)
    ctx.set_detector(qvals, corr, mask)
    return ctx, intens, qvals, corr, mask, rng


def _lambda(intens, qvals, corr, mask, quat):
    """Per-pixel Poisson mean at phi = 1: the oracle's slice (DBL_MIN outside
    the model, i.e. no photons)."""
    z = np.zeros(1, np.int32)
    prob = EMCProblem(qvals, corr, mask, z, z, np.zeros(0, np.int32), np.zeros(0, np.int32),
                      np.zeros(0, np.int32), np.array([[1., 0., 0., 0., 1.]]), intens[None])
    q = np.append(np.asarray(quat, np.float64)[:4], 1.)
    lam = OracleEngine(prob).slice_gen(q)
    lam[lam < 1e-300] = 0.
    return lam


def _dense(ones, multi, po, pm, cm, P):
    n = len(ones)
    out = np.zeros((n, P), np.int64)
    oo = np.concatenate([[0], np.cumsum(ones)])
    mo = np.concatenate([[0], np.cumsum(multi)])
    for d in range(n):
        out[d, po[oo[d]:oo[d + 1]]] += 1
        out[d, pm[mo[d]:mo[d + 1]]] += cm[mo[d]:mo[d + 1]]
    return out


def test_simulated_layout_mask_and_sorted_places(oracle_built):
    ctx, intens, qvals, corr, mask, rng = _setup()
    from dragonfly_b200 import synth
    n = 400
    intens = intens * (60. / synth.model_mean_count(intens, qvals, corr, mask, rng, n_orient=16))
    q = synth.random_quaternions(n, rng)
    tot = ctx.simulate_frames(intens, q, np.ones(n), seed=11)
    ones, multi, po, pm, cm = ctx.get_frames()
    assert (int(ones.sum()), int(multi.sum()), int(ones.sum() + cm.sum())) == tuple(tot)
    assert ones.sum() > 0 and multi.sum() > 0
    assert np.all(cm >= 2)                                       # count 1 lives in place_ones
    assert np.all(mask[po] <= 1) and np.all(mask[pm] <= 1)       # make_data.c:183-184
    oo = np.concatenate([[0], np.cumsum(ones)])
    mo = np.concatenate([[0], np.cumsum(multi)])
    for d in range(n):
        a, b = po[oo[d]:oo[d + 1]], pm[mo[d]:mo[d + 1]]
        assert np.all(np.diff(a) > 0) and np.all(np.diff(b) > 0)  # ascending, no repeats
        assert np.intersect1d(a, b).size == 0
    # the same seed draws the same frames; another seed others
    ctx.simulate_frames(intens, q, np.ones(n), seed=11)
    again = ctx.get_frames()
    for x, y in zip((ones, multi, po, pm, cm), again):
        np.testing.assert_array_equal(x, y)
    ctx.simulate_frames(intens, q, np.ones(n), seed=12)
    assert not np.array_equal(ctx.get_frames()[2][:50], po[:50])
    ctx.close()


def test_simulated_pixel_means_follow_the_slice(oracle_built):
    """20000 frames at one orientation and phi = 2: every pixel's mean count
    is 2 W_p within its Poisson spread, and its variance equals its mean."""
    ctx, intens, qvals, corr, mask, rng = _setup(5)
    n, phi = 20000, 2.
    quat = np.array([0.8, 0.2, -0.5, 0.26])
    quat /= np.linalg.norm(quat)
    lam = phi * _lambda(intens, qvals, corr, mask, quat)
    scale = 3. / lam[mask <= 1].mean()          # about 3 photons per pixel
    lam *= scale
    ctx.simulate_frames(intens * scale, np.tile(quat, (n, 1)), np.full(n, phi), seed=21)
    counts = _dense(*ctx.get_frames(), qvals.shape[0])
    assert np.all(counts[:, mask > 1] == 0)
    good = (mask <= 1) & (lam > 0)
    mean = counts[:, good].mean(0)
    z = (mean - lam[good]) / np.sqrt(lam[good] / n)
    print("per-pixel z: max |z| %.2f, mean z^2 %.3f over %d pixels" % (np.abs(z).max(), (z ** 2).mean(), z.size))
    assert np.abs(z).max() < 5.5
    assert 0.85 < (z ** 2).mean() < 1.15
    disp = counts[:, good].var(0) / lam[good]        # Poisson: variance = mean
    assert 0.9 < np.median(disp) < 1.1
    assert np.all(counts[:, (mask <= 1) & (lam == 0)] == 0)
    ctx.close()


def test_simulated_frame_totals_follow_the_scale(oracle_built):
    """Frames at random orientations with lognormal scales: each frame's
    photon count is Poisson with mean phi_d sum_p W_p(q_d)."""
    from dragonfly_b200 import synth
    ctx, intens, qvals, corr, mask, rng = _setup(7)
    n = 600
    intens = intens * (80. / synth.model_mean_count(intens, qvals, corr, mask, rng, n_orient=16))
    q = synth.random_quaternions(n, rng)
    phi = np.exp(rng.normal(0., 0.5, n))
    ctx.simulate_frames(intens, q, phi, seed=31)
    ones, multi, po, pm, cm = ctx.get_frames()
    mo = np.concatenate([[0], np.cumsum(multi)])
    cms = np.concatenate([[0], np.cumsum(cm)])
    photons = ones + (cms[mo[1:]] - cms[mo[:-1]])
    mu = np.array([phi[d] * _lambda(intens, qvals, corr, mask, q[d])[mask <= 1].sum() for d in range(n)])
    z = (photons - mu) / np.sqrt(mu)
    print("frame totals: mean z %.3f, var z %.3f, corr(photons, phi) %.3f"
          % (z.mean(), z.var(), np.corrcoef(photons, phi)[0, 1]))
    assert abs(z.mean()) < 0.2 and 0.8 < z.var() < 1.25
    assert np.corrcoef(np.log(photons), np.log(phi))[0, 1] > 0.9
    ctx.close()
