"""Host-side logic of the learned proposals (no GPU): the soft targets a
full search's probabilities give per coarse cell, and the per-frame
restriction lists of a proposal iteration, against direct loops."""
import numpy as np

from dragonfly_b200._lib import _csr
from dragonfly_b200.proposals import cell_targets, restriction_lists


def test_cell_targets_match_loops():
    rng = np.random.default_rng(3)
    N, R, nc = 60, 500, 37
    qmap = rng.integers(0, nc, R)
    lens = rng.integers(0, 30, N)
    lens[5] = 0
    off = np.zeros(N + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    place = np.concatenate([np.sort(rng.choice(R, k, replace=False)) for k in lens]).astype(np.int32)
    prob = rng.random(off[-1]) ** 4
    t_off, cells, w = cell_targets(off, place, prob, qmap, nc, min_share=1e-2)
    assert t_off[0] == 0 and t_off[-1] == cells.size == w.size
    for d in range(N):
        mass = {}
        for j in range(off[d], off[d + 1]):
            mass[qmap[place[j]]] = mass.get(qmap[place[j]], 0.) + prob[j]
        tot = sum(mass.values())
        kept = {c: m for c, m in mass.items() if m >= 1e-2 * tot}
        kt = sum(kept.values())
        got_c = cells[t_off[d]:t_off[d + 1]]
        got_w = w[t_off[d]:t_off[d + 1]]
        assert list(got_c) == sorted(kept)
        np.testing.assert_allclose(got_w, [kept[c] / kt for c in sorted(kept)], rtol=1e-6)
        if len(got_w):
            assert abs(float(got_w.sum()) - 1.) < 1e-5


def test_restriction_lists():
    rng = np.random.default_rng(4)
    N, K, nc = 50, 6, 40
    top = np.stack([rng.choice(nc, K, replace=False) for _ in range(N)]).astype(np.int32)
    watch = np.array([3, 17, 49])
    off, flat = restriction_lists(top, watch, nc)
    for d in range(N):
        got = flat[off[d]:off[d + 1]]
        if d in watch:
            assert list(got) == list(range(nc))
        else:
            assert list(got) == list(top[d])


def test_csr_forms_agree():
    lists = [np.array([3, 1]), np.array([], np.int32), np.array([7])]
    off, flat = _csr(lists)
    assert list(off) == [0, 2, 2, 3] and list(flat) == [3, 1, 7]
    off2, flat2 = _csr((off, flat))
    assert np.array_equal(off, off2) and np.array_equal(flat, flat2)
    off3, flat3 = _csr(np.array([[1, 2], [3, 4]]))
    assert list(off3) == [0, 2, 4] and list(flat3) == [1, 2, 3, 4]
