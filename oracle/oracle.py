"""ctypes front end of the CPU oracle. TEST INFRASTRUCTURE ONLY.

Two engines with one interface:

* ``OracleEngine`` -- our own C restatement (``liboracle.so``,
  source ``emc_oracle.c``; OpenMP, bit-identical to the reference with one
  thread at any thread count) of duaneloh/Dragonfly's packaged EMC engine;
* ``ReferenceEngine`` -- the reference's own C engine compiled from its sources
  (``_ref/libdragonfly_ref.so``, driver ``ref_driver.c``).

Both run ``run_iteration`` the way ``EMCRecon.run_iteration`` does
(dragonfly/recon.pyx:72-110): update_beta, maximize, update_model and, when
need_scaling is set, Iterate.normalize_scale (dragonfly/iterate.pyx:361-384,
restated here in numpy as in the reference).

Only tests/, ``__graft_entry__.smoke`` and bench.py's CPU-baseline leg import
this module; the product never does.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_ORACLE = os.path.join(HERE, "liboracle.so")
LIB_REF = os.path.join(HERE, "_ref", "libdragonfly_ref.so")
LIB_REF_FAST = os.path.join(HERE, "_ref", "libdragonfly_ref_fast.so")
LIB_LEGACY_FAST = os.path.join(HERE, "_ref", "libdragonfly_legacy_fast.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build_oracle():
    """Builds liboracle.so (and the reference libraries when the reference
    sources are present) with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load(path):
    if not os.path.exists(path):
        build_oracle()
    return C.CDLL(path)


def reference_available(fast=False):
    return os.path.exists(LIB_REF_FAST if fast else LIB_REF)


def legacy_available():
    return os.path.exists(LIB_LEGACY_FAST)


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


MODEL_TYPES = {"3d": 0, "2d": 1, "rz": 2}   # enum model_type, model.h:13


class EMCProblem:
    """Inputs of an EMC reconstruction in the reference's layouts.

    Attributes mirror the reference structs: detector (``qvals [P,3]``, ``corr``,
    ``mask``), sparse frames (``ones``, ``multi``, ``place_ones``,
    ``place_multi``, ``count_multi``), ``quats [R,5]``, model1
    ``[M, S, S, S]`` (``model_type`` "3d") or ``[M, S, S]`` ("2d", "rz"; the
    orientation is then the angle in column 0, or (phi, beta) for RZ) and the
    [emc] parameters used by the iteration.
    """

    def __init__(self, qvals, corr, mask, ones, multi, place_ones, place_multi, count_multi,
                 quats, model1, need_scaling=0, update_scale=1, known_scale=0, alpha=0.,
                 beta=1., beta_jump=1., beta_period=100, beta_factor=1., scale=None,
                 blacklist=None, model_type="3d", friedel_sym=0, detd=0.):
        self.model_type = model_type
        self.friedel_sym = int(friedel_sym)
        self.detd = float(detd)
        self.qvals = _c(qvals, np.float64).reshape(-1, 3)
        self.corr = _c(corr, np.float64)
        self.mask = _c(mask, np.uint8)
        self.ones = _c(ones, np.int32)
        self.multi = _c(multi, np.int32)
        self.place_ones = _c(place_ones, np.int32)
        self.place_multi = _c(place_multi, np.int32)
        self.count_multi = _c(count_multi, np.int32)
        self.quats = _c(quats, np.float64).reshape(-1, 5)
        m = _c(model1, np.float64)
        nd = 3 if model_type == "3d" else 2
        self.model1 = m.reshape((-1,) + m.shape[-nd:]) if m.ndim >= nd else m
        self.need_scaling = int(need_scaling)
        self.update_scale = int(update_scale)
        self.known_scale = int(known_scale)
        self.alpha = float(alpha)
        self.beta = float(beta)
        self.beta_jump = float(beta_jump)
        self.beta_period = int(beta_period)
        self.beta_factor = float(beta_factor)
        self.scale = None if scale is None else _c(scale, np.float64)
        self.blacklist = None if blacklist is None else _c(blacklist, np.uint8)

    @property
    def num_pix(self):
        return self.corr.shape[0]

    @property
    def num_data(self):
        return self.ones.shape[0]

    @property
    def num_rot(self):
        return self.quats.shape[0]

    @property
    def num_modes(self):
        return self.model1.shape[0]

    @property
    def size(self):
        return self.model1.shape[-1]


def normalize_scale(scale, blacklist, model1, rms):
    """Iterate.normalize_scale (dragonfly/iterate.pyx:361-384): numpy mean of
    the good frames' scale, model1 of mode 0 multiplied by it, scale divided."""
    if blacklist is None:
        mean_scale = scale.mean()
        scale /= mean_scale
    else:
        mean_scale = scale[blacklist == 0].mean()
        scale[blacklist == 0] /= mean_scale
    vol = model1[0].size
    model1.reshape(-1)[:vol] *= mean_scale
    return rms * mean_scale, mean_scale


class IterationResult(dict):
    """Outputs of one iteration, keyed like the reference's properties."""
    __getattr__ = dict.__getitem__


class ReferenceEngine:
    """The reference C engine (dragonfly/src) driven through ref_driver.c."""

    def __init__(self, prob, num_threads=1, fast=False):
        self.lib = _load(LIB_REF_FAST if fast else LIB_REF)
        L = self.lib
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, _dp, _dp, _up, C.c_int, _ip, _ip, _ip, _ip, _ip,
                                 C.c_int, _dp, C.c_long, C.c_int, C.c_int, _dp,
                                 C.c_int, C.c_int, C.c_int, C.c_double,
                                 C.c_double, C.c_double, C.c_int, C.c_double,
                                 C.c_void_p, C.c_void_p, C.c_int]
        L.ref_maximize.restype = C.c_double
        L.ref_maximize.argtypes = [C.c_void_p, C.c_int]
        L.ref_update_model.restype = C.c_double
        L.ref_update_model.argtypes = [C.c_void_p]
        for n in ("ref_get_model1", "ref_set_model1", "ref_get_model2", "ref_get_weight",
                  "ref_get_quat_norm", "ref_get_u", "ref_set_scale", "ref_get_scalars"):
            getattr(L, n).argtypes = [C.c_void_p, _dp]
        L.ref_get_frame_arrays.argtypes = [C.c_void_p, _ip, _dp, _dp, _dp, _dp, _dp]
        L.ref_get_iter_arrays.argtypes = [C.c_void_p, _ip, _dp, _dp, _dp, _dp]
        L.ref_set_rms.argtypes = [C.c_void_p, C.c_double]
        L.ref_slice_gen.argtypes = [C.c_void_p, _dp, C.c_int, _dp]
        L.ref_slice_merge.argtypes = [C.c_void_p, _dp, C.c_int, _dp, _dp, _dp]
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_set_save_prob.argtypes = [C.c_void_p, C.c_int]
        L.ref_set_symmetry.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.ref_set_background.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_get_powder.argtypes = [C.c_void_p, _dp]
        L.ref_get_frame_prob.restype = C.c_int
        L.ref_get_frame_prob.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.ref_set_refinement.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_set_friedel_detd.argtypes = [C.c_void_p, C.c_int, C.c_double]
        L.ref_add_detector.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _up, C.c_int, _ip, _ip, _ip, _ip, _ip,
                                       C.c_void_p, C.c_void_p]
        L.ref_get_u_det.argtypes = [C.c_void_p, C.c_int, _dp]
        L.ref_get_det_scalars.argtypes = [C.c_void_p, _dp, _dp]
        self.save_prob = False
        self.extra = []
        self.prob = p = prob
        self._scale_buf = p.scale
        self._bl_buf = p.blacklist
        self.h = L.ref_create(
            p.num_pix, p.qvals.reshape(-1), p.corr, p.mask, p.num_data, p.ones, p.multi,
            p.place_ones, p.place_multi, p.count_multi, p.num_rot, p.quats.reshape(-1),
            p.size, p.num_modes, MODEL_TYPES[p.model_type], p.model1.reshape(-1), p.need_scaling, p.update_scale,
            p.known_scale, p.alpha, p.beta, p.beta_jump, p.beta_period, p.beta_factor,
            None if p.scale is None else p.scale.ctypes.data,
            None if p.blacklist is None else p.blacklist.ctypes.data, int(num_threads))
        L.ref_set_friedel_detd(self.h, int(p.friedel_sym), float(p.detd))

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def add_detector(self, det):
        """Another detector and the frames it sees (see ref_add_detector):
        det is an EMCProblem whose detector and frames are used (its scale and
        blacklist, if any, give those frames' values); its frames follow the
        frames so far."""
        self.extra.append(det)
        self.lib.ref_add_detector(
            self.h, det.num_pix, det.qvals.reshape(-1), det.corr, det.mask, det.num_data, det.ones, det.multi,
            det.place_ones, det.place_multi, det.count_multi,
            None if det.scale is None else det.scale.ctypes.data,
            None if det.blacklist is None else det.blacklist.ctypes.data)

    @property
    def num_data(self):
        return self.prob.num_data + sum(d.num_data for d in self.extra)

    @property
    def num_det(self):
        return 1 + len(self.extra)

    @property
    def blacklist(self):
        if self.prob.blacklist is None and all(d.blacklist is None for d in self.extra):
            return None
        return np.concatenate([q.blacklist if q.blacklist is not None else np.zeros(q.num_data, np.uint8)
                               for q in [self.prob] + self.extra])

    def _arr(self, fn, shape, dt=np.float64):
        out = np.zeros(shape, dtype=dt)
        fn(self.h, out.reshape(-1))
        return out

    def model1(self):
        p = self.prob
        return self._arr(self.lib.ref_get_model1, p.model1.shape)

    def iter_arrays(self):
        n = self.num_data
        fc = np.zeros(n, np.int32)
        sf, sc, be, bs = (np.zeros(n) for _ in range(4))
        self.lib.ref_get_iter_arrays(self.h, fc, sf, sc, be, bs)
        return dict(fcounts=fc, sum_fact=sf, scale=sc, beta=be, beta_start=bs)

    def slice_gen(self, quat, mode=0):
        out = np.zeros(self.prob.num_pix)
        self.lib.ref_slice_gen(self.h, _c(quat, np.float64), int(mode), out)
        return out

    def set_background(self, background, bgscale=None):
        """Background-aware model (see ref_set_background); bgscale defaults
        to ones (iterate.pyx:290-296)."""
        p = self.prob
        bg = _c(background, np.float64)
        bs = _c(np.ones(p.num_data) if bgscale is None else bgscale, np.float64)
        self.lib.ref_set_background(self.h, bg, bs)

    def powder(self):
        return self._arr(self.lib.ref_get_powder, self.prob.num_pix)

    def set_symmetry(self, point_group=0, axial_order=0):
        """Model symmetries of update_model: point_group 1 = S4, 2 = A5."""
        self.lib.ref_set_symmetry(self.h, int(point_group), int(axial_order))

    def set_refinement(self, quat_mapping=None, rel_quat=None):
        """Coarse-to-fine refinement (see ref_set_refinement): quat_mapping
        [num_rot] nearest coarse orientation, rel_quat a per-frame sequence of
        relevant coarse orientations; None switches it off."""
        if quat_mapping is None:
            self.lib.ref_set_refinement(self.h, None, None, None)
            return
        self._qmap = _c(quat_mapping, np.int32)
        lens = np.array([len(x) for x in rel_quat], np.int64)
        self._rel_off = np.zeros(len(lens) + 1, np.int64)
        np.cumsum(lens, out=self._rel_off[1:])
        self._rel = _c(np.concatenate([np.asarray(x, np.int32).ravel() for x in rel_quat]) if lens.sum()
                       else np.zeros(1, np.int32), np.int32)
        self.lib.ref_set_refinement(self.h, self._qmap.ctypes.data, self._rel_off.ctypes.data,
                                    self._rel.ctypes.data)

    def set_save_prob(self, on):
        """Makes maximize form the combined per-frame probability lists
        (save_prob path, max_prob.c:294-325); run_iteration then returns them
        as res["sparse_prob"] = (offsets, place, prob)."""
        self.save_prob = bool(on)
        self.lib.ref_set_save_prob(self.h, int(bool(on)))

    def _sparse_prob(self):
        n = self.num_data
        counts = np.array([self.lib.ref_get_frame_prob(self.h, d, None, None) for d in range(n)], np.int64)
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum(counts)
        place = np.zeros(int(off[-1]), np.int32)
        prob = np.zeros(int(off[-1]))
        for d in range(n):
            if counts[d]:
                self.lib.ref_get_frame_prob(self.h, d, place[off[d]:].ctypes.data, prob[off[d]:].ctypes.data)
        return off, place, prob

    def run_iteration(self, iteration):
        p = self.prob
        L = self.lib
        avg_ll = L.ref_maximize(self.h, int(iteration))
        n = self.num_data
        res = IterationResult()
        if self.save_prob:
            res["sparse_prob"] = self._sparse_prob()
        rmax = np.zeros(n, np.int32)
        info, ll, mx, pn, pd = (np.zeros(n) for _ in range(5))
        L.ref_get_frame_arrays(self.h, rmax, info, ll, mx, pn, pd)
        res.update(rmax=rmax, info=info, likelihood=ll, max_exp=mx, p_norm=pn, psum_d=pd)
        res["u"] = self._arr(L.ref_get_u, p.num_modes * p.num_rot)
        res["quat_norm"] = self._arr(L.ref_get_quat_norm, (n, p.num_modes))
        sc = np.zeros(5)
        L.ref_get_scalars(self.h, sc)
        res["rescale"], res["mean_count"], res["mutual_info"] = sc[0], sc[1], sc[2]
        res["avg_likelihood"] = avg_ll
        if self.extra:
            K = self.num_det
            res["u_det"] = np.zeros((K, p.num_modes * p.num_rot))
            for k in range(K):
                L.ref_get_u_det(self.h, k, res["u_det"][k])
            res["rescale_det"], res["mean_count_det"] = np.zeros(K), np.zeros(K)
            L.ref_get_det_scalars(self.h, res["rescale_det"], res["mean_count_det"])
        res["model2_sum"] = self._arr(L.ref_get_model2, p.model1.shape)
        res["inter_weight"] = self._arr(L.ref_get_weight, p.model1.shape)
        rms = L.ref_update_model(self.h)
        res["model2"] = self._arr(L.ref_get_model2, p.model1.shape)
        it = self.iter_arrays()
        res["beta"] = it["beta"]
        res["scale"] = it["scale"]
        if p.need_scaling and p.model_type == "3d":   # recon.pyx:102-103
            scale = it["scale"]
            model1 = self.model1()
            rms, _ = normalize_scale(scale, self.blacklist, model1, rms)
            L.ref_set_scale(self.h, scale)
            L.ref_set_model1(self.h, model1.reshape(-1))
            L.ref_set_rms(self.h, rms)
            res["scale"] = scale
        res["rms_change"] = rms
        res["model1"] = self.model1()
        return res


class LegacyEngine:
    """The reference's legacy engine (src/max_emc.c, the `emc` binary's
    maximize) driven through legacy_driver.c: one iteration of
    src/recon_emc.c:102-131 per run_iteration (update_beta, maximize,
    divide-then-Friedel update_model, normalize_scale). It keeps its state in
    the library's globals, so only one LegacyEngine exists at a time. Used as
    a timed CPU baseline; OpenMP threads from OMP_NUM_THREADS / num_threads."""

    _live = None

    def __init__(self, prob, num_threads=None):
        if LegacyEngine._live is not None:
            raise RuntimeError("one LegacyEngine at a time (the legacy engine keeps global state)")
        self.lib = L = _load(LIB_LEGACY_FAST)
        L.leg_create.restype = C.c_int
        L.leg_create.argtypes = [C.c_int, _dp, _dp, _up, C.c_int, _ip, _ip, _ip, _ip, _ip, C.c_int, _dp, C.c_long,
                                 _dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int]
        L.leg_run_iteration.restype = C.c_double
        L.leg_run_iteration.argtypes = [C.c_int]
        L.leg_get_model1.argtypes = [_dp]
        L.leg_set_scale.argtypes = [_dp]
        p = self.prob = prob
        if p.num_modes != 1 or p.model_type != "3d" or p.blacklist is not None:
            raise ValueError("the legacy driver takes one 3-D mode and no blacklist")
        if num_threads:
            omp = C.CDLL(L._name)
            try:
                omp.omp_set_num_threads(int(num_threads))
            except AttributeError:
                pass
        rc = L.leg_create(p.num_pix, p.qvals.reshape(-1), p.corr, p.mask, p.num_data, p.ones, p.multi,
                          p.place_ones, p.place_multi, p.count_multi, p.num_rot, p.quats.reshape(-1), p.size,
                          p.model1.reshape(-1), p.need_scaling, p.update_scale, p.beta, p.beta_jump,
                          p.beta_period)
        if rc != 0:
            raise RuntimeError("leg_create failed")
        if p.scale is not None:
            L.leg_set_scale(p.scale)
        LegacyEngine._live = self

    def run_iteration(self, iteration):
        return self.lib.leg_run_iteration(int(iteration))

    def model1(self):
        out = np.zeros(self.prob.model1.shape)
        self.lib.leg_get_model1(out.reshape(-1))
        return out

    def close(self):
        if LegacyEngine._live is self:
            self.lib.leg_destroy()
            LegacyEngine._live = None

    def __del__(self):
        self.close()


class OracleEngine:
    """Our own C restatement (emc_oracle.c), same interface as ReferenceEngine.
    extra: more detectors, each an EMCProblem whose detector and frames are
    used (as ReferenceEngine.add_detector); their frames follow prob's."""

    def __init__(self, prob, extra=()):
        self.lib = L = _load(LIB_ORACLE)
        L.orc_maximize.restype = C.c_double
        L.orc_maximize.argtypes = [C.c_int, _dp, _dp, _up, C.c_int, _ip, _ip, _ip, _ip, _ip,
                                   C.c_int, C.c_int, _dp, C.c_long, _dp,
                                   _dp, _dp, _dp, _ip, _up, C.c_double,
                                   C.c_int, C.c_int, C.c_int, C.c_int,
                                   _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _dp]
        L.orc_update_model.restype = C.c_double
        L.orc_update_model.argtypes = [C.c_long, C.c_int, _dp, _dp, _dp, C.c_double]
        L.orc_frame_stats.argtypes = [C.c_int, _ip, _ip, _ip, _ip, _ip, _up, _ip, _dp,
                                      C.POINTER(C.c_double)]
        L.orc_calc_beta.argtypes = [C.c_int, C.c_double, C.c_int, C.c_double, _ip, _dp]
        L.orc_slice_gen3d.argtypes = [_dp, C.c_int, _dp, C.c_int, _dp, _dp, C.c_long, C.c_long, _dp]
        L.orc_slice_merge3d.argtypes = [_dp, C.c_int, _dp, _dp, _dp, C.c_long, C.c_int, _dp, _dp, _up]
        L.orc_set_keep_prob.argtypes = [C.c_int]
        L.orc_kept_prob.restype = C.c_int
        L.orc_kept_prob.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        PP = C.POINTER(C.c_void_p)
        L.orc_maximize_dets.restype = C.c_double
        L.orc_maximize_dets.argtypes = [C.c_int, _ip, PP, PP, PP, _ip, C.c_int, _ip, _ip, _ip, _ip, _ip,
                                        C.c_int, C.c_int, _dp, C.c_long, _dp,
                                        _dp, _dp, _dp, _ip, _up, _dp,
                                        C.c_int, C.c_int, C.c_int, C.c_int,
                                        _dp, _dp, _dp, _dp, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _ip, _dp, _dp]
        self.save_prob = False
        self.prob = p = prob
        self.dets = dets = [p] + list(extra)
        # per detector: fcounts, sum_fact over its mask (calc_frame_counts,
        # calc_sum_fact, iterate.c:3-117), mean_count over its frames
        fcs, sfs, mcs = [], [], []
        for q in dets:
            fc, sf, mc = np.zeros(q.num_data, np.int32), np.zeros(q.num_data), C.c_double(0.)
            L.orc_frame_stats(q.num_data, q.ones, q.multi, q.place_ones, q.place_multi, q.count_multi,
                              q.mask, fc, sf, C.byref(mc))
            fcs.append(fc)
            sfs.append(sf)
            mcs.append(mc.value)
        n = sum(q.num_data for q in dets)
        self.fcounts = np.concatenate(fcs)
        self.sum_fact = np.concatenate(sfs)
        self.mean_count_det = np.array(mcs)
        self.mean_count = mcs[0]
        self.det_of = np.concatenate([np.full(q.num_data, k, np.int32) for k, q in enumerate(dets)])
        self.beta_start = np.zeros(n)
        # calc_beta's empirical start uses detector 0's mean count (iterate.c:72-73)
        L.orc_calc_beta(n, p.beta, p.need_scaling, self.mean_count, self.fcounts, self.beta_start)
        self.beta = np.zeros(n)
        self.blacklist = np.concatenate([q.blacklist if q.blacklist is not None else np.zeros(q.num_data, np.uint8)
                                         for q in dets])
        self.scale = np.concatenate([q.scale.copy() if q.scale is not None else np.ones(q.num_data)
                                     for q in dets]) if p.need_scaling else np.ones(n)
        self._model1 = p.model1.copy()
        if len(dets) > 1:
            self.frames = {k: np.concatenate([getattr(q, k) for q in dets]).astype(np.int32)
                           for k in ("ones", "multi", "place_ones", "place_multi", "count_multi")}

    def model1(self):
        return self._model1.copy()

    def set_save_prob(self, on):
        """Makes run_iteration return the per-frame probability lists as
        res["sparse_prob"] = (offsets, place, prob), the layout of
        ReferenceEngine.set_save_prob."""
        self.save_prob = bool(on)

    def _sparse_prob(self):
        L = self.lib
        n = self.det_of.size
        counts = np.array([max(L.orc_kept_prob(d, None, None), 0) for d in range(n)], np.int64)
        off = np.zeros(n + 1, np.int64)
        off[1:] = np.cumsum(counts)
        place = np.zeros(int(off[-1]), np.int32)
        prob = np.zeros(int(off[-1]))
        for d in range(n):
            if counts[d]:
                L.orc_kept_prob(d, place[off[d]:].ctypes.data, prob[off[d]:].ctypes.data)
        return off, place, prob

    def slice_gen(self, quat, mode=0):
        p = self.prob
        out = np.zeros(p.num_pix)
        self.lib.orc_slice_gen3d(_c(quat, np.float64), int(mode), out, p.num_pix,
                                 p.qvals.reshape(-1), p.corr, p.size, p.size // 2,
                                 self._model1.reshape(-1))
        return out

    def update_beta(self, iteration):
        """recon.pyx:151-174"""
        p = self.prob
        factor = p.beta_jump ** ((iteration - 1) // p.beta_period)
        factor *= p.beta_factor
        good = self.blacklist != 1
        self.beta[good] = np.minimum(self.beta_start[good] * factor, 1.)

    def run_iteration(self, iteration):
        p = self.prob
        L = self.lib
        n, M, K = self.det_of.size, p.num_modes, len(self.dets)
        self.update_beta(iteration)
        shape = self._model1.shape
        model2 = np.zeros(shape)
        weight = np.zeros(shape)
        u = np.zeros((K, M * p.num_rot))
        psum_r = np.zeros((K, M * p.num_rot))
        rmax = np.zeros(n, np.int32)
        info, ll, mx, pn, pd = (np.zeros(n) for _ in range(5))
        qn = np.zeros((n, M))
        nprob = np.zeros(n, np.int32)
        L.orc_set_keep_prob(int(self.save_prob))
        if K == 1:
            sc = np.zeros(3)
            avg_ll = L.orc_maximize(
                p.num_pix, p.qvals.reshape(-1), p.corr, p.mask, n, p.ones, p.multi, p.place_ones,
                p.place_multi, p.count_multi, p.num_rot, M, p.quats.reshape(-1), p.size,
                self._model1.reshape(-1), self.scale, self.beta, self.sum_fact, self.fcounts,
                self.blacklist, self.mean_count, p.need_scaling, p.update_scale, p.known_scale,
                int(iteration), model2.reshape(-1), weight.reshape(-1), u[0], psum_r[0], rmax, info, ll,
                mx, pn, pd, qn.reshape(-1), nprob, sc)
            rescale_det, mi = sc[:1], sc[1]
        else:
            PA = C.c_void_p * K
            qv = PA(*[q.qvals.ctypes.data for q in self.dets])
            co = PA(*[q.corr.ctypes.data for q in self.dets])
            mk = PA(*[q.mask.ctypes.data for q in self.dets])
            npix = np.array([q.num_pix for q in self.dets], np.int32)
            f = self.frames
            rescale_det, sc = np.zeros(K), np.zeros(2)
            avg_ll = L.orc_maximize_dets(
                K, npix, qv, co, mk, self.det_of, n, f["ones"], f["multi"], f["place_ones"], f["place_multi"],
                f["count_multi"], p.num_rot, M, p.quats.reshape(-1), p.size, self._model1.reshape(-1), self.scale,
                self.beta, self.sum_fact, self.fcounts, self.blacklist, self.mean_count_det, p.need_scaling,
                p.update_scale, p.known_scale, int(iteration), model2.reshape(-1), weight.reshape(-1),
                u.reshape(-1), psum_r.reshape(-1), rmax, info, ll, mx, pn, pd, qn.reshape(-1), nprob,
                rescale_det, sc)
            mi = sc[0]
        res = IterationResult(rmax=rmax, info=info, likelihood=ll, max_exp=mx, p_norm=pn,
                              psum_d=pd, u=u[0], psum_r=psum_r[0], quat_norm=qn, num_prob=nprob,
                              rescale=rescale_det[0], mutual_info=mi, avg_likelihood=avg_ll,
                              mean_count=self.mean_count, beta=self.beta.copy())
        if K > 1:
            res.update(u_det=u, psum_r_det=psum_r, rescale_det=rescale_det, mean_count_det=self.mean_count_det)
        if self.save_prob:
            res["sparse_prob"] = self._sparse_prob()
            L.orc_set_keep_prob(0)
        res["model2_sum"] = model2.copy()
        res["inter_weight"] = weight
        rms = L.orc_update_model(p.size, M, self._model1.reshape(-1), model2.reshape(-1),
                                 weight.reshape(-1), p.alpha)
        res["model2"] = model2
        if p.need_scaling:
            rms, _ = normalize_scale(self.scale, self.blacklist if K > 1 else p.blacklist, self._model1, rms)
            res["scale"] = self.scale.copy()
        res["rms_change"] = rms
        res["model1"] = self.model1()
        return res


def quat_gen_reference(num_div):
    """Quaternions from the reference's quat_gen (quaternion.c:811-842)."""
    L = _load(LIB_REF)
    L.ref_quat_gen.restype = C.c_int
    L.ref_quat_gen.argtypes = [C.c_int, C.c_void_p]
    n = L.ref_quat_gen(int(num_div), None)
    out = np.zeros((n, 5))
    L.ref_quat_gen(int(num_div), out.ctypes.data)
    return out


def voronoi_subset_reference(coarse_div, fine):
    """Nearest coarse (num_div = coarse_div) orientation of every fine one,
    from the reference's voronoi_subset (quaternion.c:844-862)."""
    L = _load(LIB_REF)
    L.ref_voronoi_subset.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p]
    f = _c(fine, np.float64)
    out = np.full(f.shape[0], -1, np.int32)
    L.ref_voronoi_subset(int(coarse_div), f.shape[0], f.ctypes.data, out.ctypes.data)
    return out


def voronoi_subset_port(coarse, fine):
    """Restatement of voronoi_subset (quaternion.c:844-862) in numpy: for each
    fine orientation the coarse one with the smallest 1 - d^2, d the dot
    product of (q0..q3) summed in component order without fused multiply-add
    (numpy elementwise operations, no BLAS), first index on ties."""
    c = np.asarray(coarse, np.float64)[:, :4]
    f = np.asarray(fine, np.float64)[:, :4]
    out = np.empty(f.shape[0], np.int32)
    for s in range(0, f.shape[0], 2048):
        q = f[s:s + 2048]
        d = q[:, 0:1] * c[None, :, 0]
        for k in range(1, 4):
            d = d + q[:, k:k + 1] * c[None, :, k]
        out[s:s + 2048] = np.argmin(1. - d * d, axis=1)
    return out
