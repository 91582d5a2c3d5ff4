"""Sparse probability lists (EMCRecon.prob / place_prob with save_prob) and
per-orientation photon tomograms against the reference engine.

The reference forms the lists in combine_information_omp (max_prob.c:294-325):
per frame the pairs with P > 1e-6, in ascending orientation order. The GPU
forms them with the same gate from its own P; pairs whose P lies within the
tolerance of the 1e-6 gate may fall on either side, everything else must
agree.
"""
import numpy as np
import pytest

from common import GPUEngine, load_case
from oracle.oracle import ReferenceEngine, reference_available

PROB_MIN = 1e-6
# Per-pair P, relative. Log-slices are FP32 (relative 6e-8 per value), so a
# frame with K photons carries about K * 6e-8 * |log W| of absolute error in
# its log-likelihood and beta times that in P; the aggregate bounds of the
# parity contract (model 1e-5, likelihood and information 1e-6) are tested
# elsewhere, this bound is for single pairs at beta = 1.
P_REL = 1e-4
TOMO_REL = 1e-4   # tomograms: FP32 accumulation of P with the same error


def _frame_photons(prob):
    """Per frame: (pixel, count) of the photons on mask < 2 pixels."""
    out = []
    o1 = np.concatenate([[0], np.cumsum(prob.ones)])
    om = np.concatenate([[0], np.cumsum(prob.multi)])
    for d in range(prob.num_data):
        pix = list(prob.place_ones[o1[d]:o1[d + 1]])
        cnt = [1] * len(pix)
        pix += list(prob.place_multi[om[d]:om[d + 1]])
        cnt += list(prob.count_multi[om[d]:om[d + 1]])
        pix, cnt = np.asarray(pix, np.int64), np.asarray(cnt, np.float64)
        keep = prob.mask[pix] < 2
        out.append((pix[keep], cnt[keep]))
    return out


def _compare_lists(gpu_sp, ref_sp, n):
    go, gp, gv = gpu_sp
    ro, rp, rv = ref_sp
    flips, worst = 0, 0.
    for d in range(n):
        a = dict(zip(gp[go[d]:go[d + 1]].tolist(), gv[go[d]:go[d + 1]].tolist()))
        b = dict(zip(rp[ro[d]:ro[d + 1]].tolist(), rv[ro[d]:ro[d + 1]].tolist()))
        assert (np.diff(gp[go[d]:go[d + 1]]) > 0).all(), "orientations not ascending in frame %d" % d
        for r in a.keys() & b.keys():
            worst = max(worst, abs(a[r] - b[r]) / abs(b[r]))
            assert abs(a[r] - b[r]) <= P_REL * abs(b[r]), (d, r, a[r], b[r])
        for r in a.keys() ^ b.keys():
            v = a.get(r, b.get(r))
            assert v <= PROB_MIN * (1 + P_REL), ("pair far above the gate missing", d, r, v)
            flips += 1
    print("sparse prob: worst relative P deviation %.2e, gate flips %d" % (worst, flips))
    return flips


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["beta1", "scaling"])
def test_gpu_sparse_prob_and_tomograms_match_reference(oracle_built, case):
    if not reference_available():
        pytest.skip("reference engine library not built")
    prob, _ = load_case(case)
    gpu = GPUEngine(prob, keep_prob=1)
    ref = ReferenceEngine(prob)
    ref.set_save_prob(1)
    photons = _frame_photons(prob)
    total_pairs = 0
    for it in (1, 2):
        gpu.run_iteration(it)
        b = ref.run_iteration(it)
        sp = gpu.ctx.sparse_prob()
        total_pairs += int(sp[0][-1])
        flips = _compare_lists(sp, b["sparse_prob"], prob.num_data)
        assert flips <= 1e-4 * max(int(sp[0][-1]), 1), flips

        # tomograms of a few orientations: sum_d count * P_dr over the listed
        # pairs (P > 1e-6 gate of update_tomogram_nobg, max_update.c:181-210)
        _, psum_r = gpu.ctx.orientation_results()
        ro, rp, rv = b["sparse_prob"]
        rs = sorted(set([0, 1, 2, prob.num_rot * prob.num_modes - 1] + list(rp[ro[0]:ro[0] + 3])))
        expect = np.zeros((len(rs), prob.num_pix))
        where = {r: k for k, r in enumerate(rs)}
        for d in range(prob.num_data):
            for r, v in zip(rp[ro[d]:ro[d + 1]], rv[ro[d]:ro[d + 1]]):
                if r in where:
                    pix, cnt = photons[d]
                    np.add.at(expect[where[r]], pix, cnt * v)
        for k, r in enumerate(rs):
            got = gpu.ctx.tomograms(int(r), 1)[0]
            ref_row = expect[k] / psum_r[r] if psum_r[r] > 0 else expect[k]
            scale = max(np.abs(ref_row).max(), 1e-300)
            assert np.abs(got - ref_row).max() <= TOMO_REL * scale, (it, r)
    assert total_pairs > 0
    with pytest.raises(Exception):
        gpu.ctx.tomograms(prob.num_rot * prob.num_modes, 1)
    gpu.close()
    ref.close()
