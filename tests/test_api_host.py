"""Host-side parts of the reference-facing API, on CPU: file formats, config
parsing, per-frame statistics, Friedel symmetrisation, rotation matrices."""
import ctypes as C
import os

import numpy as np
import pytest

from common import load_case
from dragonfly_b200 import CDataset, CDetector, Detector, EMCParams, EMCReader, EMCWriter, Iterate, Model, \
    Quaternion, synth
from dragonfly_b200.emcfile import read_emc, write_emc
from oracle.oracle import OracleEngine, _load, LIB_ORACLE


def write_problem(tmp_path, seed=5, need_scaling=0, extra=""):
    d = synth.small_problem(seed=seed, det_side=24, size=29, qmax=13., n_atoms=40, atom_radius=5., num_div=1,
                            n_frames=60, mean_count=20.)
    det = Detector()
    det.qvals = d["qvals"]
    det.corr = d["corr"]
    det.raw_mask = d["mask"]
    det.detd, det.ewald_rad = d["detd"], d["ewald_rad"]
    det.write(str(tmp_path / "det.npz"))
    write_emc(str(tmp_path / "photons.emc"), d["qvals"].shape[0], d["ones"], d["multi"], d["place_ones"],
              d["place_multi"], d["count_multi"])
    cfg = tmp_path / "config.ini"
    cfg.write_text("""[files]
det = det.npz

[emc]
in_photons_file = photons.emc
in_detector_file = files:::det
num_div = 2
output_folder = out/
log_file = out/EMC.log
need_scaling = %d
beta = 0.5
beta_schedule = 2. 3
alpha = 0.
%s
""" % (need_scaling, extra))
    return d, str(cfg)


def test_emc_binary_round_trip(tmp_path):
    d = synth.small_problem(seed=3, det_side=16, size=21, qmax=9., n_atoms=20, atom_radius=4., num_div=1,
                            n_frames=40, mean_count=30.)
    fn = str(tmp_path / "a.emc")
    with EMCWriter(fn, 256, hdf5=False) as w:
        oo = np.concatenate([[0], np.cumsum(d["ones"])])
        mo = np.concatenate([[0], np.cumsum(d["multi"])])
        for i in range(d["ones"].size):
            w.write_sparse_frame(d["place_ones"][oo[i]:oo[i + 1]], d["place_multi"][mo[i]:mo[i + 1]],
                                 d["count_multi"][mo[i]:mo[i + 1]])
    num_pix, ones, multi, po, pm, cm = read_emc(fn)
    assert num_pix == 256
    for a, b in ((ones, d["ones"]), (multi, d["multi"]), (po, d["place_ones"]), (pm, d["place_multi"]),
                 (cm, d["count_multi"])):
        np.testing.assert_array_equal(a, b)
    assert os.path.getsize(fn) == 1024 + 4 * (2 * ones.size + po.size + 2 * pm.size)
    # dense frame writer and reader agree
    frame = np.zeros(256, np.int32)
    frame[[3, 7, 9]] = [1, 4, 1]
    fn2 = str(tmp_path / "b.emc")
    with EMCWriter(fn2, 256, hdf5=False) as w:
        w.write_frame(frame)
        w.write_frame(frame * 0)
    det = CDetector()
    det.raw_mask = np.zeros(256, np.uint8)
    r = EMCReader(fn2, det)
    np.testing.assert_array_equal(r.get_frame(0, raw=True), frame)
    assert r.get_frame(1, raw=True).sum() == 0
    ds = CDataset(fn2, det)
    assert ds.num_data == 2 and ds.ones_total == 2 and ds.multi_total == 1
    np.testing.assert_array_equal(ds.ones_accum, [0, 2])


def test_emc_truncated_file_is_rejected(tmp_path):
    fn = str(tmp_path / "t.emc")
    write_emc(fn, 100, np.array([3], np.int32), np.array([0], np.int32), np.array([1, 2, 3], np.int32),
              np.zeros(0, np.int32), np.zeros(0, np.int32))
    data = open(fn, "rb").read()
    open(fn, "wb").write(data[:-4])
    with pytest.raises(ValueError, match="truncated"):
        read_emc(fn)


def test_detector_file_and_coords(tmp_path):
    q, corr, mask, detd, ewald = synth.flat_detector(20, 18, 12., 27, hole_radius=2.)
    det = Detector()
    det.qvals, det.corr, det.raw_mask = q, corr * 3., mask
    det.detd, det.ewald_rad = detd, ewald
    fn = str(tmp_path / "d.npz")
    det.write(fn)
    back = CDetector(fn)  # norm=True divides corr by its mean
    np.testing.assert_allclose(back.corr, corr / corr.mean())
    np.testing.assert_array_equal(back.raw_mask, mask)
    assert abs(back.qmax() - 12.) < 1e-9
    # calc_from_coords reproduces the generator's qvals
    d2 = Detector()
    cx, cy = np.meshgrid(np.arange(20) - 9.5, np.arange(18) - 8.5, indexing="ij")
    d2.cx, d2.cy, d2.detd, d2.ewald_rad = cx, cy, detd, ewald
    d2.calc_from_coords("x")
    np.testing.assert_allclose(d2.qvals, q, rtol=1e-13, atol=1e-13)
    full = Detector(fn)
    assert full.frame_shape == (20, 18)
    with pytest.raises(ValueError):
        det.corr = np.ones(5)


def test_params_from_config(tmp_path):
    _, cfg = write_problem(tmp_path)
    p = EMCParams()
    assert p.beta_factor == -1. and p.update_scale == 1 and p.num_modes == 1
    p.from_config(cfg)
    assert p.beta_jump == 2. and p.beta_period == 3 and p.beta_factor == 1.
    assert p.output_folder.endswith("out/") and p.log_fname.endswith("out/EMC.log")
    assert p.verbosity == 9 and p.sigmasq == 0.


def test_iterate_from_config_frame_stats(tmp_path, oracle_built):
    d, cfg = write_problem(tmp_path, need_scaling=1)
    itr = Iterate(cfg)
    assert itr.tot_num_data == d["ones"].size
    assert itr.model.size == Iterate.calculate_size(itr.dets[0].qmax())
    assert itr.quat.num_rot == 420
    np.testing.assert_array_equal(itr.scale, np.ones(itr.tot_num_data))
    # fcounts, sum_fact, mean_count as the reference's iterate.c (through the oracle)
    L = _load(LIB_ORACLE)
    n = itr.tot_num_data
    fc = np.zeros(n, np.int32)
    sf = np.zeros(n)
    mc = C.c_double()
    ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
    L.orc_frame_stats.argtypes = [C.c_int, ip, ip, ip, ip, ip,
                                  np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS"), ip,
                                  np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS"), C.POINTER(C.c_double)]
    L.orc_frame_stats(n, d["ones"], d["multi"], d["place_ones"], d["place_multi"], d["count_multi"],
                      np.ascontiguousarray(itr.dets[0].raw_mask), fc, sf, C.byref(mc))
    np.testing.assert_array_equal(itr.fcounts, fc)
    np.testing.assert_array_equal(itr.sum_fact, sf)
    assert itr.mean_count[0] == mc.value
    np.testing.assert_array_equal(itr.beta_start, np.full(n, 0.5))
    # empirical beta rule when 'beta' is auto and need_scaling
    itr.calc_beta()
    np.testing.assert_allclose(itr.beta_start, np.exp(-6.5 * (fc * 1e-5) ** 0.15))
    # odd_only selection
    itr.parse_blacklist("", "odd_only", refresh=True)
    assert itr.blacklist[0] == 0 and itr.blacklist[1] == 1


def test_normalize_scale_matches_reference_rule():
    itr = Iterate()
    itr.scale = np.array([1., 2., 3., 6.])
    itr.blacklist = np.array([0, 0, 1, 0], np.uint8)
    itr.model = Model(3)
    itr.model.model1 = np.ones((1, 3, 3, 3))
    itr.rms_change = 1.
    m = itr.normalize_scale()
    assert m == 3.
    np.testing.assert_allclose(itr.scale, [1 / 3., 2 / 3., 3., 2.])
    assert itr.model.model1[0, 0, 0, 0] == 3. and itr.rms_change == 3.


@pytest.mark.parametrize("size", [9, 10, 35])
def test_symmetrize_friedel_matches_oracle(size, oracle_built):
    rng = np.random.default_rng(size)
    m = rng.random((size, size, size))
    w = rng.random((size, size, size)) * (rng.random((size, size, size)) > 0.2)
    a = m.copy()
    Model.symmetrize_friedel(a, w)
    b = m.copy().reshape(-1)
    L = _load(LIB_ORACLE)
    dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
    L.orc_symmetrize_friedel.argtypes = [dp, dp, C.c_int]
    L.orc_symmetrize_friedel(b, np.ascontiguousarray(w).reshape(-1), size)
    np.testing.assert_array_equal(a.reshape(-1), b)


def test_make_rot_quat_and_quaternion_api():
    q = Quaternion(num_div=2)
    assert q.num_rot == 420
    R = Model.make_rot_quat(q.quats[7])
    np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-14)
    assert q.divide(0, 3) == 140 and q.divide(2, 4) == 105
    # voronoi_subset runs on the GPU: tests/test_refinement.py
    q2 = Quaternion(num_rot=36, point_group="1")
    assert q2.quats.shape == (36, 5)


def test_iterate_detector_list(tmp_path, oracle_built):
    """in_detector_list / in_photons_list (iterate.pyx:61-101, 432-456):
    file i is seen by detector i; the unique detectors are ordered by file
    name, so here the second file's detector is detector 0. Frame counts,
    sum_fact and the per-detector mean counts as the oracle forms them for
    each detector's frames; the model is sized by the largest qmax."""
    dets, sh = synth.two_detector_problem(seed=7)
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
    cfg = tmp_path / "config.ini"
    cfg.write_text("""[emc]
in_photons_list = photons.txt
in_detector_list = dets.txt
num_div = 2
output_folder = out/
log_file = out/EMC.log
beta = 0.5
""")
    itr = Iterate(str(cfg))
    n0, n1 = dets[0]["ones"].size, dets[1]["ones"].size
    assert itr.num_det == 2 and itr.tot_num_data == n0 + n1
    np.testing.assert_array_equal(itr.det_mapping, [1, 0])
    assert itr.dets[0].fname.endswith("det_a.npz") and itr.dets[1].fname.endswith("det_z.npz")
    np.testing.assert_array_equal(itr.member_index(0), np.arange(n0, n0 + n1))
    np.testing.assert_array_equal(itr.member_index(1), np.arange(n0))
    for k, key in enumerate(("ones", "multi", "place_ones", "place_multi", "count_multi")):
        np.testing.assert_array_equal(itr.member_frames(0)[k], dets[1][key])
    fcs, mcs = [], []
    for dd in dets:
        p = EMCProblem_from(dd, sh)
        orc = OracleEngine(p)
        fcs.append(orc.fcounts)
        mcs.append(orc.mean_count)
    np.testing.assert_array_equal(itr.fcounts, np.concatenate(fcs))
    assert itr.mean_count[0] == mcs[1] and itr.mean_count[1] == mcs[0]
    qmax = max(np.linalg.norm(dd["qvals"], axis=1).max() for dd in dets)
    assert itr.model.size == Iterate.calculate_size(qmax)
    # calc_beta's empirical start uses detector 0's mean count (iterate.c:72-73)
    itr.calc_beta()
    np.testing.assert_allclose(itr.beta_start, np.exp(-6.5 * (itr.mean_count[0] * 1e-5) ** 0.15), rtol=1e-14)
    # a background list needs one entry per detector (iterate.pyx:109-127),
    # in the detector list's order (det_z first), whatever their sorted order
    for k, dd in enumerate(dets):
        np.savez(str(tmp_path / ("bg%d.npz" % k)), background=np.full(dd["qvals"].shape[0], 0.1 * (k + 1)))
    (tmp_path / "bg1.txt").write_text("bg0.npz\n")
    (tmp_path / "bg2.txt").write_text("bg0.npz\nbg1.npz\n")
    base = cfg.read_text()
    cfg.write_text(base + "background_list = bg1.txt\n")
    with pytest.raises(ValueError, match="Background list has 1 entries but there are 2 unique detectors"):
        Iterate(str(cfg))
    cfg.write_text(base + "background_list = bg2.txt\n")
    itr2 = Iterate(str(cfg))
    assert all(d.with_bg for d in itr2.dets)
    assert itr2.dets[0].background[0] == 0.2 and itr2.dets[1].background[0] == 0.1
    # a single photons file with a detector list uses the first detector
    cfg.write_text(base.replace("in_photons_list = photons.txt", "in_photons_file = photons0.emc"))
    itr1 = Iterate(str(cfg))
    assert itr1.num_det == 1 and itr1.dets[0].fname.endswith("det_z.npz")


def EMCProblem_from(dd, sh):
    from oracle.oracle import EMCProblem
    return EMCProblem(dd["qvals"], dd["corr"], dd["mask"], dd["ones"], dd["multi"], dd["place_ones"],
                      dd["place_multi"], dd["count_multi"], sh["quats"], sh["model_start"])
