"""2-D and RZ models (enum model_type, model.h:13).

CPU: Model.symmetrize_friedel2d against the reference's symmetrize_friedel2d
(model.c:495-515, compiled). GPU: one-slice slice_gen / slice_merge of 2-D
and RZ models against the reference's slice_gen2d / slice_merge2d /
slice_genrz / slice_mergerz (model.c:65-150, 254-340), and 2-D iterations
(recon_type = 2d: recon.pyx:86-91 selects slice_gen2d / slice_merge2d; update
with symmetrize_friedel2d when friedel_sym, recon.pyx:118-119; no
normalize_scale, :102-103) against the reference engine.
"""
import ctypes as C

import numpy as np
import pytest

from common import GPUEngine, MODEL_REL_L2, RMAX_AGREE, SCALAR_REL, rel_l2
from oracle.oracle import LIB_REF, EMCProblem, ReferenceEngine, reference_available


def _ref_lib():
    if not reference_available():
        pytest.skip("reference engine library not built")
    return C.CDLL(LIB_REF)


@pytest.mark.parametrize("size", [21, 24])
def test_friedel2d_matches_reference(oracle_built, size):
    from dragonfly_b200.model import Model
    L = _ref_lib()
    L.symmetrize_friedel2d.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    rng = np.random.default_rng(size)
    m = rng.random((3, size, size))
    w = rng.random((3, size, size)) * (rng.random((3, size, size)) > 0.3)
    ref = m.copy()
    L.symmetrize_friedel2d(ref.ctypes.data, w.ctypes.data, 3, size)
    ours = m.copy()
    Model.symmetrize_friedel2d(ours, w)
    np.testing.assert_array_equal(ours, ref)


def _problem(model_type="2d", friedel=0, need_scaling=0, seed=4, **kw):
    from dragonfly_b200 import synth
    d = synth.small_problem_2d(seed=seed, **kw)
    if friedel:
        # with friedel_sym, Quaternion.from_config generates angles in [0, pi)
        # (point group '2', quaternion.pyx:70-74): 180-degree turns of a
        # centrosymmetric image would otherwise tie
        n = d["quats"].shape[0]
        d["quats"][:, 0] = np.arange(n) * (np.pi / n)
    return d, EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"],
                         d["place_multi"], d["count_multi"], d["quats"], d["model_start"], beta=1.,
                         need_scaling=need_scaling, update_scale=need_scaling, model_type=model_type,
                         friedel_sym=friedel, detd=60.)


@pytest.mark.gpu
@pytest.mark.parametrize("model_type", ["2d", "rz"])
def test_gpu_one_slice_2d_rz_matches_reference(oracle_built, model_type):
    _ref_lib()
    d, prob = _problem(model_type)
    ref = ReferenceEngine(prob)
    gpu = GPUEngine(prob)
    rng = np.random.default_rng(1)
    model = d["model_true"][None] if model_type == "2d" else rng.random((1,) + d["model_true"].shape)
    gpu.ctx.set_model(model)
    ref.lib.ref_set_model1(ref.h, np.ascontiguousarray(model).reshape(-1))
    size = model.shape[-1]
    for k in range(6):
        o = np.array([rng.random() * 2 * np.pi]) if model_type == "2d" else rng.random(2) * np.pi
        a = gpu.ctx.slice_gen(o)
        b = np.zeros(prob.num_pix)
        ref.lib.ref_slice_gen(ref.h, np.ascontiguousarray(o), 0, b)
        np.testing.assert_array_equal(a, b)
        assert (b > 1e-300).sum() > prob.num_pix // 4      # most pixels inside the image
        m2a, wa = np.zeros((1, size, size)), np.zeros((1, size, size))
        gpu.ctx.slice_merge(o, b, m2a, wa)
        m2b, wb = np.zeros((1, size, size)), np.zeros((1, size, size))
        ref.lib.ref_slice_merge(ref.h, np.ascontiguousarray(o), 0, b, m2b.reshape(-1), wb.reshape(-1))
        # atomic additions on the GPU: same terms, order may differ
        np.testing.assert_allclose(m2a, m2b, rtol=1e-12, atol=1e-12 * np.abs(m2b).max())
        np.testing.assert_allclose(wa, wb, rtol=1e-12, atol=1e-14)
    gpu.close()
    ref.close()


@pytest.mark.gpu
@pytest.mark.parametrize("friedel,need_scaling", [(0, 0), (1, 0), (0, 1)])
def test_gpu_2d_iterations_match_reference(oracle_built, friedel, need_scaling):
    _ref_lib()
    d, prob = _problem("2d", friedel, need_scaling)
    ref = ReferenceEngine(prob)
    gpu = GPUEngine(prob)
    for it in (1, 2, 3):
        a = gpu.run_iteration(it)
        b = ref.run_iteration(it)
        dev = rel_l2(a["model1"], b["model1"])
        ll = abs(a["avg_likelihood"] - b["avg_likelihood"]) / abs(b["avg_likelihood"])
        mi = abs(a["mutual_info"] - b["mutual_info"]) / max(abs(b["mutual_info"]), 1e-300)
        agree = float(np.mean(np.asarray(a["rmax"]) == np.asarray(b["rmax"])))
        print("2-D (friedel %d, scaling %d) iteration %d: model %.2e, ll %.2e, mi %.2e, rmax %.4f"
              % (friedel, need_scaling, it, dev, ll, mi, agree))
        assert dev <= MODEL_REL_L2 and ll <= SCALAR_REL and mi <= SCALAR_REL, (dev, ll, mi)
        assert agree >= RMAX_AGREE, agree
        if need_scaling:
            np.testing.assert_allclose(a["scale"], b["scale"], rtol=1e-6)
    # the reconstruction moves towards the true image (up to rotation)
    gpu.close()
    ref.close()
