"""Coarse-to-fine orientation refinement (params.refine).

CPU: the oracle's restatement of voronoi_subset against the reference's own
(quaternion.c:844-862, compiled), and the per-frame coarse lists read back
from a coarse run's output or the binary format (parse_rel_quat,
src/iterate.c:364-527). GPU: dfg_voronoi_subset against the reference, and
refined iterations against the reference engine with quat_mapping /
rel_quat filled as the legacy engine's setup does (src/iterate.c:103-130);
the packaged engine then skips the pairs at max_prob.c:110-120.
"""
import os

import numpy as np
import pytest

from common import GPUEngine, MODEL_REL_L2, RMAX_AGREE, SCALAR_REL, rel_l2
from oracle.oracle import (EMCProblem, ReferenceEngine, reference_available, voronoi_subset_port,
                           voronoi_subset_reference)
from dragonfly_b200.quatgen import quat_gen


@pytest.mark.parametrize("coarse_div,fine_div", [(1, 3), (2, 4)])
def test_voronoi_port_matches_reference(oracle_built, coarse_div, fine_div):
    if not reference_available():
        pytest.skip("reference engine library not built")
    fine = quat_gen(fine_div)
    ref = voronoi_subset_reference(coarse_div, fine)
    port = voronoi_subset_port(quat_gen(coarse_div), fine)
    np.testing.assert_array_equal(port, ref)
    # every coarse cell is used, and fine vertices that coincide with coarse
    # ones map onto them
    assert np.unique(ref).size == quat_gen(coarse_div).shape[0]


def _iterate_stub(n):
    from dragonfly_b200.iterate import Iterate
    itr = Iterate()
    itr.tot_num_data = n
    return itr


def test_parse_rel_quat_binary_and_output(tmp_path):
    rng = np.random.default_rng(3)
    n, nc = 50, 60
    lists = [np.sort(rng.choice(nc, rng.integers(0, 5), replace=False)).astype(np.int32) for _ in range(n)]
    # binary: num_data, num_rot, then at byte 1024 the counts and the lists
    fn = str(tmp_path / "rel.bin")
    with open(fn, "wb") as f:
        np.array([n, nc], np.int32).tofile(f)
        f.seek(1024)
        np.array([len(x) for x in lists], np.int32).tofile(f)
        for x in lists:
            x.tofile(f)
    itr = _iterate_stub(n)
    got = itr.parse_rel_quat(fn, nc)
    assert all(np.array_equal(a, b) for a, b in zip(got, lists))
    with pytest.raises(ValueError):
        itr.parse_rel_quat(fn, nc + 1)
    # an output file with saved probabilities
    off = np.zeros(n + 1, np.int64)
    off[1:] = np.cumsum([len(x) for x in lists])
    fn2 = str(tmp_path / "out.npz")
    np.savez(fn2, probabilities__num_rot=np.array([nc]), probabilities__offsets=off,
             probabilities__place=np.concatenate(lists), orientations=np.zeros(n, np.int32))
    got = itr.parse_rel_quat(fn2, nc)
    assert all(np.array_equal(a, b) for a, b in zip(got, lists))
    # without probabilities: the most likely orientation of each frame
    rmax = rng.integers(0, nc, n).astype(np.int32)
    fn3 = str(tmp_path / "out3.npz")
    np.savez(fn3, orientations=rmax)
    got = itr.parse_rel_quat(fn3, nc)
    assert [int(x[0]) for x in got] == rmax.tolist()


@pytest.mark.gpu
@pytest.mark.parametrize("coarse_div,fine_div", [(2, 4), (4, 8)])
def test_gpu_voronoi_matches_reference(oracle_built, coarse_div, fine_div):
    if not reference_available():
        pytest.skip("reference engine library not built")
    from dragonfly_b200.quaternion import Quaternion
    q = Quaternion(num_div=fine_div)
    got = q.voronoi_subset(coarse_div)
    ref = voronoi_subset_reference(coarse_div, q.quats)
    np.testing.assert_array_equal(got, ref)
    assert q.num_rot_coarse == quat_gen(coarse_div).shape[0]


def _rel_lists(rng, n, nc, true_cell, mode, allow_empty):
    out = []
    for d in range(n):
        if mode == "rmax":
            out.append(np.array([true_cell[d]], np.int32))
        else:
            k = int(rng.integers(0 if allow_empty else 1, 6))   # some frames may get an empty list
            extra = rng.choice(nc, k, replace=False)
            cells = extra if (k == 0 or rng.random() < 0.2) else np.append(extra, true_cell[d])
            out.append(np.unique(cells).astype(np.int32))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("mode,need_scaling", [("rmax", 0), ("lists", 0), ("lists", 1)])
def test_gpu_refinement_matches_reference(oracle_built, mode, need_scaling):
    if not reference_available():
        pytest.skip("reference engine library not built")
    from dragonfly_b200 import synth
    d = synth.small_problem(seed=9, det_side=48, size=41, qmax=19., n_atoms=120, atom_radius=7., num_div=4,
                            n_frames=500, mean_count=80., hole_radius=3.)
    fine = quat_gen(4)
    qmap = voronoi_subset_reference(2, fine)
    nc = quat_gen(2).shape[0]
    # the coarse cell of a fine orientation near each frame's true one
    rng = np.random.default_rng(17)
    true_cell = qmap[rng.integers(0, fine.shape[0], d["ones"].size)]
    # with scale updates an empty list leaves psum_d = 0 and phi_d = fcounts / 0
    # in both engines (max_scale.c:3-19), so those frames are left out there
    rel = _rel_lists(rng, d["ones"].size, nc, true_cell, mode, allow_empty=not need_scaling)
    prob = EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"], d["place_multi"],
                      d["count_multi"], fine, d["model_start"], beta=1., need_scaling=need_scaling,
                      update_scale=need_scaling)
    ref = ReferenceEngine(prob)
    ref.set_refinement(qmap, rel)
    ref.set_save_prob(True)
    gpu = GPUEngine(prob, keep_prob=1)
    gpu.ctx.set_refinement(nc, qmap, rel)
    for it in (1, 2):
        a = gpu.run_iteration(it)
        b = ref.run_iteration(it)
        dev = rel_l2(a["model1"], b["model1"])
        ll = abs(a["avg_likelihood"] - b["avg_likelihood"]) / abs(b["avg_likelihood"])
        mi = abs(a["mutual_info"] - b["mutual_info"]) / max(abs(b["mutual_info"]), 1e-300)
        agree = float(np.mean(np.asarray(a["rmax"]) == np.asarray(b["rmax"])))
        # the per-frame lists of pairs with P > 1e-6 (save_prob path)
        off_a, place_a, _ = gpu.ctx.sparse_prob()
        off_b, place_b, _ = b["sparse_prob"]
        nprob = float(np.mean(np.diff(off_a) == np.diff(off_b)))
        if np.array_equal(off_a, off_b):
            assert np.array_equal(place_a, place_b)
        assert all(qmap[place_a[j]] in rel[i] for i in range(len(rel)) for j in range(off_a[i], off_a[i + 1]))
        print("refinement (%s, scaling %d) iteration %d: model %.2e, ll %.2e, mi %.2e, rmax %.4f, num_prob %.4f"
              % (mode, need_scaling, it, dev, ll, mi, agree, nprob))
        assert dev <= MODEL_REL_L2 and ll <= SCALAR_REL and mi <= SCALAR_REL, (dev, ll, mi)
        assert agree >= RMAX_AGREE and nprob >= RMAX_AGREE, (agree, nprob)
        # frames with no relevant orientation have none: rmax -1, as the reference
        empty = np.array([len(x) == 0 for x in rel])
        assert (np.asarray(a["rmax"])[empty] == -1).all()
        # every most likely orientation lies in one of the frame's coarse cells
        r = np.asarray(a["rmax"])
        ok = [r[i] < 0 or qmap[r[i]] in rel[i] for i in range(len(rel))]
        assert all(ok)
    gpu.close()
    ref.close()


@pytest.mark.gpu
@pytest.mark.parametrize("need_scaling,block_mb", [(0, 0.), (1, 6.)])
def test_gpu_pair_lists_match_reference(oracle_built, need_scaling, block_mb):
    """Pair lists (option pair_lists): only the live (tile, frame) pairs are
    stored, orientations in blocks of whole tiles (block_budget_mb 6: five
    tiles per block at this detector, six blocks). Against the reference
    engine with the same lists, and against the dense restricted path: the
    same log-likelihood sums and kept sets (identical rmax, p_norm and
    likelihood to FP64 rounding), tomograms scattered with FP32 atomics."""
    if not reference_available():
        pytest.skip("reference engine library not built")
    from dragonfly_b200 import synth
    d = synth.small_problem(seed=9, det_side=48, size=41, qmax=19., n_atoms=120, atom_radius=7., num_div=4,
                            n_frames=500, mean_count=80., hole_radius=3.)
    fine = quat_gen(4)
    qmap = voronoi_subset_reference(2, fine)
    order = np.lexsort((np.arange(fine.shape[0]), qmap))   # cells contiguous, as proposals use them
    fine, qmap = np.ascontiguousarray(fine[order]), np.ascontiguousarray(qmap[order])
    nc = quat_gen(2).shape[0]
    rng = np.random.default_rng(17)
    true_cell = qmap[rng.integers(0, fine.shape[0], d["ones"].size)]
    rel = _rel_lists(rng, d["ones"].size, nc, true_cell, "lists", allow_empty=not need_scaling)
    prob = EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"], d["place_multi"],
                      d["count_multi"], fine, d["model_start"], beta=1., need_scaling=need_scaling,
                      update_scale=need_scaling)
    ref = ReferenceEngine(prob)
    ref.set_refinement(qmap, rel)
    opts = dict(pair_lists=1)
    if block_mb:
        opts["block_budget_mb"] = block_mb
    gpu = GPUEngine(prob, **opts)
    gpu.ctx.set_refinement(nc, qmap, rel)
    dense = GPUEngine(prob)
    dense.ctx.set_refinement(nc, qmap, rel)
    for it in (1, 2):
        a = gpu.run_iteration(it)
        b = ref.run_iteration(it)
        c = dense.run_iteration(it)
        dev = rel_l2(a["model1"], b["model1"])
        ll = abs(a["avg_likelihood"] - b["avg_likelihood"]) / abs(b["avg_likelihood"])
        mi = abs(a["mutual_info"] - b["mutual_info"]) / max(abs(b["mutual_info"]), 1e-300)
        agree = float(np.mean(np.asarray(a["rmax"]) == np.asarray(b["rmax"])))
        dd = rel_l2(a["model1"], c["model1"])
        print("pair lists (scaling %d, block %g MB) iteration %d: vs reference model %.2e, ll %.2e, mi %.2e, "
              "rmax %.4f; vs dense restricted path model %.2e" % (need_scaling, block_mb, it, dev, ll, mi, agree, dd))
        assert dev <= MODEL_REL_L2 and ll <= SCALAR_REL and mi <= SCALAR_REL, (dev, ll, mi)
        assert agree >= RMAX_AGREE, agree
        np.testing.assert_array_equal(a["rmax"], c["rmax"])
        # iteration 1 starts from the same model: equal sums; later the
        # models differ by the tomograms' atomic rounding (about 1e-9), which
        # moves log-likelihoods of about 200 by about 2e-7 and probabilities
        # by as much relative
        tol = 1e-12 if it == 1 else 1e-7
        np.testing.assert_allclose(a["likelihood"], c["likelihood"], rtol=tol, atol=tol)
        np.testing.assert_allclose(a["psum_r"], c["psum_r"], rtol=1e-12 if it == 1 else 1e-5, atol=1e-300)
        assert dd <= 1e-6, dd
        empty = np.array([len(x) == 0 for x in rel])
        assert (np.asarray(a["rmax"])[empty] == -1).all()
    with pytest.raises(RuntimeError):
        gpu.ctx.tomograms(0, 1)        # not kept with pair lists
    for e in (gpu, dense):
        e.close()
    ref.close()
