"""Point-group and axial model symmetries.

CPU: the orientation reductions to the octahedral (S4) and icosahedral (A5)
asymmetric units (Quaternion.reduce_octahedral / reduce_icosahedral,
quaternion.pyx:177-255). GPU: update_model with each symmetry against the
reference engine's own symmetrize_octahedral / symmetrize_icosahedral /
symmetrize_axial (model.c:527-757), over two full iterations.
"""
import itertools

import numpy as np
import pytest

from common import GPUEngine, rel_l2
from dragonfly_b200.quaternion import Quaternion
from oracle.oracle import EMCProblem, ReferenceEngine, reference_available


def test_octahedral_quaternions_as_the_reference_builds_them():
    # restated from quaternion.pyx:227-241 (identity first; the sign choices
    # matter because the reduction uses Euclidean distances)
    cq = np.zeros((24, 4))
    cq[:4] = np.identity(4)
    signs3 = np.stack(np.meshgrid([-1., 1.], [-1., 1.], [-1., 1.], indexing="ij"), -1).reshape(-1, 3)
    cq[4:12] = 0.5
    cq[4:12, 1:] *= signs3
    v = np.sqrt(0.5)
    cq[12:18, 0] = v
    cq[12:15, 1:] = np.identity(3) * v
    cq[15:18, 1:] = -np.identity(3) * v
    for i, pos in enumerate(itertools.permutations(range(3), 2)):
        cq[18 + i, np.array(pos) + 1] = [v, -v] if pos[0] < pos[1] else [v, v]
    np.testing.assert_array_equal(Quaternion.octahedral_quaternions(), cq)


@pytest.mark.parametrize("group", ["A5", "S4"])
def test_reduction_keeps_a_subset_with_its_weights(group):
    full = Quaternion(num_div=4)
    q = Quaternion(num_div=4)
    n = q.reduce_icosahedral() if group == "A5" else q.reduce_octahedral()
    assert n == q.num_rot and q.reduced
    rows = {tuple(r) for r in full.quats}
    assert all(tuple(r) in rows for r in q.quats)          # rows (weights included) unchanged
    if group == "A5":
        np.testing.assert_array_equal(q.quats[0], full.quats[8])   # the identity vertex first
    # the kept set is the cell of the identity: about 1/24 of the octahedral
    # orientations, and at most 1/32 of the 600-cell's for A5
    ratio = full.num_rot / n
    assert (40 < ratio < 50) if group == "A5" else (20 < ratio < 26)
    assert q.reduce_octahedral() == n                        # already reduced: unchanged


@pytest.mark.gpu
@pytest.mark.parametrize("point_group,axial", [(1, 0), (2, 0), (0, 4), (1, 2)])
def test_gpu_symmetrised_update_matches_reference(oracle_built, point_group, axial):
    if not reference_available():
        pytest.skip("reference engine library not built")
    from dragonfly_b200 import synth
    d = synth.small_problem(seed=5, det_side=48, size=41, qmax=19., n_atoms=120, atom_radius=7., num_div=4,
                            n_frames=600, mean_count=80., hole_radius=3.)
    q = Quaternion(num_div=4)
    if point_group == 1:
        q.reduce_octahedral()
    elif point_group == 2:
        q.reduce_icosahedral()
    prob = EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"], d["place_multi"],
                      d["count_multi"], q.quats, d["model_start"], beta=1.)
    ref = ReferenceEngine(prob)
    ref.set_symmetry(point_group, axial)
    gpu = GPUEngine(prob)
    gpu.ctx.set_symmetry(point_group, axial)
    for it in (1, 2):
        a = gpu.run_iteration(it)
        b = ref.run_iteration(it)
        dev = rel_l2(a["model1"], b["model1"])
        ll = abs(a["avg_likelihood"] - b["avg_likelihood"]) / abs(b["avg_likelihood"])
        print("symmetry (%d, %d) iteration %d: model %.2e, likelihood %.2e" % (point_group, axial, it, dev, ll))
        assert dev <= 1e-5 and ll <= 1e-6, (dev, ll)
    gpu.close()
    ref.close()


def _ref_lib():
    import ctypes as C
    from oracle.oracle import LIB_REF
    lib = C.CDLL(LIB_REF)
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    lib.rotate_model.argtypes = [dp, dp, C.c_int, C.c_int, dp]
    for n in ("symmetrize_octahedral", "symmetrize_icosahedral"):
        getattr(lib, n).argtypes = [dp, dp, C.c_int]
    lib.symmetrize_axial.argtypes = [dp, dp, C.c_int, C.c_int]
    return lib


@pytest.mark.gpu
@pytest.mark.parametrize("size,max_r", [(33, 0), (34, 10), (21, 3)])
def test_gpu_rotate_model_matches_reference(oracle_built, size, max_r):
    """Model.rotate_model on the GPU (dfg_model_rotate) equals the reference's
    rotate_model (model.c:381-425) bit for bit, added into a given array."""
    if not reference_available():
        pytest.skip("reference engine library not built")
    from dragonfly_b200.model import Model
    rng = np.random.default_rng(size + max_r)
    m = rng.random((size,) * 3)
    q = rng.normal(size=4)
    rot = np.ascontiguousarray(Model.make_rot_quat(q / np.linalg.norm(q)), np.float64)
    start = rng.random((size,) * 3)
    ref = start.copy()
    _ref_lib().rotate_model(rot, m, size, max_r, ref)
    out = Model.rotate_model(m, rot, max_r, start.copy())
    np.testing.assert_array_equal(out, ref)
    zero = np.zeros((size,) * 3)
    _ref_lib().rotate_model(rot, m, size, max_r, zero)
    np.testing.assert_array_equal(Model.rotate_model(m, rot, max_r), zero)


@pytest.mark.gpu
@pytest.mark.parametrize("group", ["octahedral", "icosahedral", "axial"])
def test_gpu_model_symmetrize_matches_reference(oracle_built, group):
    """Model.symmetrize_* on the GPU (dfg_model_symmetrize) against the
    reference's symmetrize_octahedral / icosahedral / axial (model.c:527-757)
    on the same un-normalised volume and weights. The groups' rotations are
    summed in another order (and A5's are exact where the reference's table
    has 11 decimals), so the bound is relative, not bitwise."""
    if not reference_available():
        pytest.skip("reference engine library not built")
    from dragonfly_b200.model import Model
    rng = np.random.default_rng(7)
    size = 31
    m = rng.random((size,) * 3)
    w = rng.random((size,) * 3) + 0.1
    a, wa, b, wb = m.copy(), w.copy(), m.copy(), w.copy()
    lib = _ref_lib()
    if group == "axial":
        lib.symmetrize_axial(a, wa, size, 5)
        Model.symmetrize_axial(b, wb, 5)
    else:
        getattr(lib, "symmetrize_" + group)(a, wa, size)
        getattr(Model, "symmetrize_" + group)(b, wb)
    tol = 1e-9 if group == "icosahedral" else 1e-13
    assert rel_l2(wb, wa) <= tol and rel_l2(b, a) <= tol, (rel_l2(wb, wa), rel_l2(b, a))
    if group != "icosahedral":
        assert np.all((wa > 0) == (wb > 0))
