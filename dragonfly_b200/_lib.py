"""ctypes binding of libdfgpu.so, the C ABI in include/dragonfly_b200.h.

The library is the only compute path of this package: if it cannot be loaded
(not built, or no CUDA driver) every call raises; there is no CPU fallback.
"""
import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdfgpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "dragonfly_b200.h")

DFG_OK, DFG_ERR_ARG, DFG_ERR_CUDA, DFG_ERR_STATE, DFG_ERR_NOMEM = range(5)
PHASES = ("slice", "estep", "norm", "psum", "mstep", "merge", "update")


TUNE_REPORT = 18   # DFG_TUNE_REPORT, values of an autotuner report


class DFGError(RuntimeError):
    """A call into libdfgpu.so returned an error code."""

    def __init__(self, code, msg):
        super().__init__("dragonfly_b200 error %d: %s" % (code, msg))
        self.code = code


class IterParams(C.Structure):
    _fields_ = [("iteration", C.c_int), ("need_scaling", C.c_int), ("update_scale", C.c_int),
                ("known_scale", C.c_int), ("beta_jump", C.c_double), ("beta_period", C.c_int),
                ("beta_factor", C.c_double)]


_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
_U8 = C.POINTER(C.c_uint8)
_V = C.c_void_p

_SIGS = {
    "dfg_version": (C.c_char_p, []),
    "dfg_create": (C.c_int, [C.c_int, C.POINTER(_V)]),
    "dfg_destroy": (None, [_V]),
    "dfg_last_error": (C.c_char_p, [_V]),
    "dfg_set_detector": (C.c_int, [_V, C.c_int, _D, _D, _U8]),
    "dfg_set_frames": (C.c_int, [_V, C.c_int, _I, _I, _I, _I, _I]),
    "dfg_set_quaternions": (C.c_int, [_V, C.c_int, _D]),
    "dfg_set_model": (C.c_int, [_V, C.c_long, C.c_int, _D]),
    "dfg_set_scale": (C.c_int, [_V, _D]),
    "dfg_set_blacklist": (C.c_int, [_V, _U8]),
    "dfg_set_beta_start": (C.c_int, [_V, _D]),
    "dfg_calc_beta": (C.c_int, [_V, C.c_double, C.c_int]),
    "dfg_maximize": (C.c_int, [_V, C.POINTER(IterParams), _D]),
    "dfg_update_model": (C.c_int, [_V, C.c_double, _D]),
    "dfg_normalize_scale": (C.c_int, [_V, _D]),
    "dfg_get_frame_results": (C.c_int, [_V, _I, _D, _D, _D, _D, _D]),
    "dfg_get_quat_norm": (C.c_int, [_V, _D]),
    "dfg_get_orientation_results": (C.c_int, [_V, _D, _D]),
    "dfg_get_model": (C.c_int, [_V, _D, _D, _D]),
    "dfg_get_frame_params": (C.c_int, [_V, _D, _D, _D, _I, _D, _U8]),
    "dfg_get_scalars": (C.c_int, [_V, _D]),
    "dfg_get_num_prob": (C.c_int, [_V, _I]),
    "dfg_set_background": (C.c_int, [_V, _D]),
    "dfg_load_emc": (C.c_int, [_V, C.c_int, C.POINTER(C.c_char_p)]),
    "dfg_save_emc": (C.c_int, [_V, C.c_char_p]),
    "dfg_set_symmetry": (C.c_int, [_V, C.c_int, C.c_int]),
    "dfg_set_refinement": (C.c_int, [_V, C.c_int, _I, C.POINTER(C.c_longlong), _I]),
    "dfg_set_refinement_topk": (C.c_int, [_V, C.c_int, _I, C.c_int, _I, C.c_int, _I]),
    "dfg_set_model_type": (C.c_int, [_V, C.c_int, C.c_int]),
    "dfg_run_iteration": (C.c_int, [_V, C.POINTER(IterParams), C.c_double, _D]),
    "dfg_get_graph_stats": (C.c_int, [_V, C.POINTER(C.c_long)]),
    "dfg_autotune": (C.c_int, [_V, C.POINTER(IterParams), _D]),
    "dfg_get_autotune_report": (C.c_int, [_V, _D]),
    "dfg_batch_create": (C.c_int, [C.POINTER(_V), C.c_int, C.POINTER(_V)]),
    "dfg_batch_run": (C.c_int, [_V, C.POINTER(IterParams), _D, _D]),
    "dfg_batch_last_error": (C.c_char_p, [_V]),
    "dfg_batch_set_lanes": (C.c_int, [_V, C.c_int]),
    "dfg_batch_stats": (C.c_int, [_V, C.POINTER(C.c_long)]),
    "dfg_batch_destroy": (None, [_V]),
    "dfg_group_create": (C.c_int, [C.POINTER(_V), C.c_int, C.POINTER(_V)]),
    "dfg_group_destroy": (None, [_V]),
    "dfg_group_last_error": (C.c_char_p, [_V]),
    "dfg_group_maximize": (C.c_int, [_V, C.POINTER(IterParams), _D]),
    "dfg_group_update_model": (C.c_int, [_V, C.c_double, _D]),
    "dfg_group_normalize_scale": (C.c_int, [_V, _D]),
    "dfg_group_run_iteration": (C.c_int, [_V, C.POINTER(IterParams), C.c_double, _D]),
    "dfg_pnet_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_ulonglong, C.POINTER(_V)]),
    "dfg_pnet_destroy": (None, [_V]),
    "dfg_pnet_last_error": (C.c_char_p, [_V]),
    "dfg_pnet_num_params": (C.c_longlong, [_V]),
    "dfg_pnet_get_params": (C.c_int, [_V, C.POINTER(C.c_float)]),
    "dfg_pnet_set_params": (C.c_int, [_V, C.POINTER(C.c_float)]),
    "dfg_pnet_set_bins": (C.c_int, [_V, C.c_int, _I]),
    "dfg_pnet_load_frames": (C.c_int, [_V, _V]),
    "dfg_pnet_set_images": (C.c_int, [_V, C.c_longlong, C.POINTER(C.c_float)]),
    "dfg_pnet_get_images": (C.c_int, [_V, C.POINTER(C.c_float)]),
    "dfg_pnet_train": (C.c_int, [_V, _I, C.c_int, C.c_double, C.c_ulonglong, _D]),
    "dfg_pnet_topk": (C.c_int, [_V, C.c_int, _I]),
    "dfg_pnet_topk_mass": (C.c_int, [_V, C.c_int, C.c_int, C.c_double, _I]),
    "dfg_pnet_set_tensor_cores": (C.c_int, [_V, C.c_int]),
    "dfg_pnet_set_option": (C.c_int, [_V, C.c_char_p, C.c_double]),
    "dfg_pnet_set_targets": (C.c_int, [_V, C.POINTER(C.c_longlong), _I, C.POINTER(C.c_float)]),
    "dfg_pnet_logits": (C.c_int, [_V, C.POINTER(C.c_float)]),
    "dfg_pnet_gradients": (C.c_int, [_V, _I, C.POINTER(C.c_float), _D]),
    "dfg_set_detector_distance": (C.c_int, [_V, C.c_double]),
    "dfg_voronoi_subset": (C.c_int, [_V, C.c_int, _D, C.c_int, _D, _I]),
    "dfg_set_watch": (C.c_int, [_V, C.c_int, _I, C.POINTER(C.c_longlong), _I]),
    "dfg_get_watch_mass": (C.c_int, [_V, _D]),
    "dfg_set_bgscale": (C.c_int, [_V, _D]),
    "dfg_get_sparse_prob_offsets": (C.c_int, [_V, C.POINTER(C.c_longlong)]),
    "dfg_get_sparse_prob": (C.c_int, [_V, _I, _D]),
    "dfg_get_tomograms": (C.c_int, [_V, C.c_int, C.c_int, _D]),
    "dfg_slice_gen": (C.c_int, [_V, _D, C.c_int, _D]),
    "dfg_slice_merge": (C.c_int, [_V, _D, C.c_int, _D, _D, _D]),
    "dfg_slice_gen_noalloc": (C.c_int, [_V, _D, C.c_int, _D]),
    "dfg_run_iteration_host": (C.c_int, [_V, C.POINTER(IterParams), C.c_double, _D, _I, _D, _D, _D]),
    "dfg_set_option": (C.c_int, [_V, C.c_char_p, C.c_double]),
    "dfg_get_phase_times": (C.c_int, [_V, _D, C.POINTER(C.c_long), C.c_int]),
    "dfg_phase_name": (C.c_char_p, [C.c_int]),
    "dfg_reset_phase_times": (C.c_int, [_V]),
    "dfg_get_workload": (C.c_int, [_V, C.POINTER(C.c_longlong)]),
    "dfg_simulate_frames": (C.c_int, [_V, C.c_long, _D, C.c_int, _D, _D, C.c_ulonglong,
                                      C.POINTER(C.c_longlong)]),
    "dfg_get_frames": (C.c_int, [_V, _I, _I, _I, _I, _I]),
    "dfg_event_record": (C.c_int, [_V, C.c_int]),
    "dfg_event_elapsed": (C.c_int, [_V, C.c_int, C.c_int, _D]),
    "dfg_measure_gather_rate": (C.c_int, [_V, C.c_longlong, C.c_int, _D]),
    "dfg_model_rotate": (C.c_int, [_V, _D, C.c_int, C.c_int, _D, _D]),
    "dfg_model_symmetrize": (C.c_int, [_V, C.c_int, C.c_int, C.c_int, _D, _D]),
}

_lib = None


def header_symbols():
    """Entry points declared in include/dragonfly_b200.h."""
    with open(HEADER) as f:
        return re.findall(r"^DFG_API[^(]*?\b(dfg_\w+)\s*\(", f.read(), flags=re.M)


def load():
    """Loads libdfgpu.so (raises OSError if it is missing or does not load)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libdfgpu.so is not built (run python -m dragonfly_b200.build): %s" % LIB_PATH)
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def ptr(a, ctype):
    """Pointer to a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data_as(C.POINTER(ctype))


def _csr(lists):
    """(offsets int64 [n + 1], flat int32) of per-item lists given as a
    sequence of arrays, a 2-D array (equal lengths) or an (offsets, flat)
    tuple."""
    if isinstance(lists, tuple):
        off, flat = lists
        return np.ascontiguousarray(off, np.int64), np.ascontiguousarray(flat, np.int32)
    if isinstance(lists, np.ndarray) and lists.ndim == 2:
        n, k = lists.shape
        return np.arange(n + 1, dtype=np.int64) * k, np.ascontiguousarray(lists, np.int32).ravel()
    lens = np.array([len(x) for x in lists], np.int64)
    off = np.zeros(len(lens) + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    flat = np.ascontiguousarray(np.concatenate([np.asarray(x, np.int32).ravel() for x in lists])
                                if len(lens) else np.zeros(0, np.int32), np.int32)
    return off, flat


def _quat5(quat):
    """An orientation as the five doubles the slice entry points read: a
    quaternion (q0..q3, weight 1 appended when absent), an angle (2-D: the
    angle, then zeros) or (phi, beta) (RZ)."""
    q = np.ascontiguousarray(np.atleast_1d(quat), np.float64).ravel()
    if q.size == 4:
        q = np.append(q, 1.)
    elif q.size in (1, 2):
        q = np.concatenate([q, np.zeros(5 - q.size)])
    if q.size != 5:
        raise ValueError("an orientation is 1 (angle), 2 (phi, beta), 4 or 5 numbers, got %d" % q.size)
    return q


class Context:
    """Owner of one dfg_ctx (one GPU's resident inputs and work buffers)."""

    def __init__(self, device=0):
        self.lib = load()
        h = _V()
        rc = self.lib.dfg_create(int(device), C.byref(h))
        if rc != DFG_OK:
            raise DFGError(rc, "dfg_create(device=%d) failed (no usable CUDA device?)" % device)
        self.h = h
        self.device = device

    def close(self):
        if getattr(self, "h", None):
            self.lib.dfg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc):
        if rc != DFG_OK:
            raise DFGError(rc, self.lib.dfg_last_error(self.h).decode())
        return rc

    def call(self, name, *args):
        return self.check(getattr(self.lib, name)(self.h, *args))

    # -- inputs ------------------------------------------------------------
    def set_detector(self, qvals, corr, mask):
        q = np.ascontiguousarray(qvals, np.float64).reshape(-1)
        c = np.ascontiguousarray(corr, np.float64)
        m = np.ascontiguousarray(mask, np.uint8)
        if q.size != 3 * c.size or m.size != c.size:
            raise ValueError("qvals must be [P,3], corr and mask [P]")
        self.call("dfg_set_detector", c.size, ptr(q, C.c_double), ptr(c, C.c_double), ptr(m, C.c_uint8))
        self.num_pix = c.size
        self._qvals, self._corr, self._mask = q.reshape(-1, 3), c, m

    def set_frames(self, ones, multi, place_ones, place_multi, count_multi):
        a = [np.ascontiguousarray(x, np.int32) for x in (ones, multi, place_ones, place_multi, count_multi)]
        if a[1].size != a[0].size or a[4].size != a[3].size:
            raise ValueError("ones/multi and place_multi/count_multi lengths differ")
        if a[2].size != int(a[0].sum()) or a[3].size != int(a[1].sum()):
            raise ValueError("place arrays do not match the per-frame counts")
        self.call("dfg_set_frames", a[0].size, *[ptr(x, C.c_int) for x in a])
        self.num_data = a[0].size

    def set_quaternions(self, quats):
        q = np.ascontiguousarray(quats, np.float64).reshape(-1, 5)
        self.call("dfg_set_quaternions", q.shape[0], ptr(q, C.c_double))
        self.num_rot = q.shape[0]

    def set_model(self, model1):
        """model1 [modes, S, S, S] (3-D) or [modes, S, S] (2-D / RZ); one
        mode may omit the leading axis."""
        m = np.ascontiguousarray(model1, np.float64)
        if m.ndim == (3 if getattr(self, "model_type", 0) == 0 else 2):
            m = m[None]
        self.call("dfg_set_model", m.shape[-1], m.shape[0], ptr(m, C.c_double))
        self.model_shape = m.shape

    def load_emc(self, paths):
        """Frames from binary .emc files (sparse, or dense integer made
        sparse), concatenated in order; replaces set_frames."""
        paths = [paths] if isinstance(paths, (str, bytes, os.PathLike)) else list(paths)
        arr = (C.c_char_p * len(paths))(*[os.fsencode(p) for p in paths])
        self.call("dfg_load_emc", len(paths), arr)
        self.num_data = int(self.workload()["num_data"])

    def save_emc(self, path):
        """The context's frames as one sparse binary .emc file."""
        self.call("dfg_save_emc", os.fsencode(path))

    def set_symmetry(self, point_group=0, axial_order=0):
        """Model symmetries of update_model: point_group 0 (Friedel only),
        1 (S4) or 2 (A5); axial_order > 1 adds the axial symmetry."""
        self.call("dfg_set_symmetry", int(point_group), int(axial_order))

    def set_model_type(self, model_type, friedel_sym=0):
        """0 / "3d" (volume), 1 / "2d" (stack of images, angle orientations)
        or 2 / "rz"; friedel_sym: 2-D Friedel average in update_model. Call
        set_model afterwards."""
        mt = {"3d": 0, "2d": 1, "rz": 2}.get(str(model_type).lower(), model_type)
        self.call("dfg_set_model_type", int(mt), int(friedel_sym))
        self.model_type = int(mt)

    def set_detector_distance(self, detd):
        self.call("dfg_set_detector_distance", float(detd))

    def set_refinement(self, num_coarse=0, quat_mapping=None, rel_quat=None):
        """Coarse-to-fine refinement: frame d evaluates orientation r only
        when quat_mapping[r] is in rel_quat[d] (a sequence of per-frame
        coarse-orientation lists, a 2-D array with one row per frame, or a
        tuple (offsets [N + 1], flat lists)). quat_mapping None switches it
        off."""
        if quat_mapping is None:
            self.call("dfg_set_refinement", 0, None, None, None)
            return
        qm = np.ascontiguousarray(quat_mapping, np.int32).ravel()
        off, flat = _csr(rel_quat)
        self.call("dfg_set_refinement", int(num_coarse), ptr(qm, C.c_int), ptr(off, C.c_longlong),
                  ptr(flat, C.c_int))

    def set_refinement_topk(self, num_coarse, quat_mapping, top, all_frames=()):
        """Refinement from a top-K array [N, K] of coarse cells per frame; the
        frames in all_frames evaluate every orientation."""
        qm = np.ascontiguousarray(quat_mapping, np.int32).ravel()
        t = np.ascontiguousarray(top, np.int32)
        af = np.ascontiguousarray(all_frames, np.int32).ravel()
        if t.ndim != 2 or t.shape[0] != getattr(self, "num_data", -1):
            raise ValueError("top must be [num_frames, K] with one row per frame of the context")
        if qm.size != getattr(self, "num_rot", -1):
            raise ValueError("quat_mapping must have one entry per orientation")
        self.call("dfg_set_refinement_topk", int(num_coarse), ptr(qm, C.c_int), int(t.shape[1]), ptr(t, C.c_int),
                  int(af.size), ptr(af, C.c_int) if af.size else None)

    def set_watch(self, frames, cells):
        """Watched frames (ascending) with a coarse-cell list each (lists, a
        2-D array or (offsets, flat) as set_refinement); None clears."""
        if frames is None or len(frames) == 0:
            self.call("dfg_set_watch", 0, None, None, None)
            self._n_watch = 0
            return
        fr = np.ascontiguousarray(frames, np.int32)
        off, flat = _csr(cells)
        self.call("dfg_set_watch", fr.size, ptr(fr, C.c_int), ptr(off, C.c_longlong), ptr(flat, C.c_int))
        self._n_watch = fr.size

    def watch_mass(self):
        out = np.zeros(self._n_watch)
        self.call("dfg_get_watch_mass", ptr(out, C.c_double))
        return out

    def voronoi_subset(self, coarse, fine):
        """Nearest coarse orientation of every fine one (rows of five)."""
        c = np.ascontiguousarray(coarse, np.float64)
        f = np.ascontiguousarray(fine, np.float64)
        out = np.empty(f.shape[0], np.int32)
        self.call("dfg_voronoi_subset", c.shape[0], ptr(c, C.c_double), f.shape[0], ptr(f, C.c_double),
                  ptr(out, C.c_int))
        return out

    def set_background(self, background):
        """Per-pixel background (None: none); with need_scaling the iteration
        then takes the background-aware updates."""
        b = None if background is None else np.ascontiguousarray(background, np.float64).ravel()
        self.call("dfg_set_background", ptr(b, C.c_double))

    def set_bgscale(self, bgscale):
        """Per-frame background scales (None: ones)."""
        b = None if bgscale is None else np.ascontiguousarray(bgscale, np.float64).ravel()
        self.call("dfg_set_bgscale", ptr(b, C.c_double))

    def set_scale(self, scale):
        s = np.ascontiguousarray(scale, np.float64)
        self.call("dfg_set_scale", ptr(s, C.c_double))

    def set_blacklist(self, blacklist):
        b = np.ascontiguousarray(blacklist, np.uint8)
        self.call("dfg_set_blacklist", ptr(b, C.c_uint8))

    def set_beta_start(self, beta_start):
        b = np.ascontiguousarray(beta_start, np.float64)
        self.call("dfg_set_beta_start", ptr(b, C.c_double))

    def calc_beta(self, start, need_scaling):
        self.call("dfg_calc_beta", float(start), int(need_scaling))

    def set_option(self, key, value):
        self.call("dfg_set_option", key.encode(), float(value))

    # -- iteration ---------------------------------------------------------
    @staticmethod
    def params(iteration, need_scaling=0, update_scale=1, known_scale=0, beta_jump=1.,
               beta_period=100, beta_factor=1.):
        return IterParams(int(iteration), int(need_scaling), int(update_scale), int(known_scale),
                          float(beta_jump), int(beta_period), float(beta_factor))

    def maximize(self, par):
        ll = C.c_double(0.)
        self.call("dfg_maximize", C.byref(par), C.byref(ll))
        return ll.value

    def update_model(self, alpha=0.):
        rms = C.c_double(0.)
        self.call("dfg_update_model", float(alpha), C.byref(rms))
        return rms.value

    def normalize_scale(self):
        m = C.c_double(0.)
        self.call("dfg_normalize_scale", C.byref(m))
        return m.value

    def run_iteration(self, par, alpha=0.):
        """maximize + update_model (+ normalize_scale for need_scaling and
        volumes) with one synchronisation, as a CUDA graph where possible.
        Returns dict(avg_likelihood, rms_change, mutual_info, rescale,
        mean_scale)."""
        out = np.zeros(5)
        self.call("dfg_run_iteration", C.byref(par), float(alpha), ptr(out, C.c_double))
        return dict(zip(("avg_likelihood", "rms_change", "mutual_info", "rescale", "mean_scale"), out.tolist()))

    @staticmethod
    def _tune_dict(out):
        opt = lambda v: float(v) if v >= 0 else None
        return dict(slice_ms={b: float(out[i]) for i, b in enumerate((128, 64, 32, 16)) if out[i] >= 0},
                    estep_sparse_ms=float(out[4]), estep_dense_ms=opt(out[5]),
                    slice_block=int(out[6]), estep_form=int(out[7]) & 1, mstep_form=int(out[7]) >> 1,
                    mstep_sparse_ms=opt(out[8]), mstep_dense_ms=opt(out[9]),
                    estep_ms_by_blocks_per_sm={b: float(out[10 + i]) for i, b in enumerate((2, 3, 4))
                                               if out[10 + i] >= 0},
                    mstep_ms_by_blocks_per_sm={b: float(out[13 + i]) for i, b in enumerate((3, 4, 5))
                                               if out[13 + i] >= 0},
                    estep_blocks_per_sm=int(out[16]), mstep_blocks_per_sm=int(out[17]))

    def autotune(self, par):
        """Times the slice blocks, both E-step and M-step forms and the
        sparse forms' blocks per SM on the current inputs and keeps the
        fastest (used by later iterations with option autotune). Returns the
        measurements and the choice."""
        out = np.zeros(TUNE_REPORT)
        self.call("dfg_autotune", C.byref(par), ptr(out, C.c_double))
        return self._tune_dict(out)

    def tune_report(self):
        """The autotuner's last report for the current inputs (None if not tuned)."""
        out = np.zeros(TUNE_REPORT)
        if self.lib.dfg_get_autotune_report(self.h, ptr(out, C.c_double)) != DFG_OK:
            return None
        return self._tune_dict(out)

    def graph_stats(self):
        out = (C.c_long * 3)()
        self.call("dfg_get_graph_stats", out)
        return dict(launches=out[0], instantiations=out[1], updates=out[2])

    def run_iteration_host(self, par, model1, alpha=0., rmax=None, likelihood=None):
        """model1 (float64, C order) is updated in place."""
        ll = C.c_double(0.)
        rms = C.c_double(0.)
        self.call("dfg_run_iteration_host", C.byref(par), float(alpha), ptr(model1, C.c_double),
                  ptr(rmax, C.c_int), ptr(likelihood, C.c_double), C.byref(ll), C.byref(rms))
        return ll.value, rms.value

    # -- results -----------------------------------------------------------
    def frame_results(self):
        n = self.num_data
        rmax = np.zeros(n, np.int32)
        info, ll, mx, pn, pd = (np.zeros(n) for _ in range(5))
        self.call("dfg_get_frame_results", ptr(rmax, C.c_int), ptr(info, C.c_double), ptr(ll, C.c_double),
                  ptr(mx, C.c_double), ptr(pn, C.c_double), ptr(pd, C.c_double))
        return dict(rmax=rmax, info=info, likelihood=ll, max_exp=mx, p_norm=pn, psum_d=pd)

    def num_prob(self):
        out = np.zeros(self.num_data, np.int32)
        self.call("dfg_get_num_prob", ptr(out, C.c_int))
        return out

    def sparse_prob(self):
        """(offsets [N+1] int64, place_prob int32, prob float64) of the last
        maximize run with option keep_prob: frame d's pairs with P > 1e-6 are
        [offsets[d], offsets[d+1]) in orientation order."""
        off = np.zeros(self.num_data + 1, np.int64)
        self.call("dfg_get_sparse_prob_offsets", ptr(off, C.c_longlong))
        place = np.zeros(max(int(off[-1]), 1), np.int32)
        prob = np.zeros(max(int(off[-1]), 1), np.float64)
        self.call("dfg_get_sparse_prob", ptr(place, C.c_int), ptr(prob, C.c_double))
        n = int(off[-1])
        return off, place[:n], prob[:n]

    def tomograms(self, r0, n):
        """Photon tomograms of orientations r0 .. r0+n-1 (each / psum_r where
        positive) as [n, num_pix] float64."""
        out = np.zeros((n, self.num_pix))
        self.call("dfg_get_tomograms", int(r0), int(n), ptr(out, C.c_double))
        return out

    def quat_norm(self):
        out = np.zeros((self.num_data, self.model_shape[0]))
        self.call("dfg_get_quat_norm", ptr(out, C.c_double))
        return out

    def orientation_results(self):
        R = self.model_shape[0] * self.num_rot
        u, pr = np.zeros(R), np.zeros(R)
        self.call("dfg_get_orientation_results", ptr(u, C.c_double), ptr(pr, C.c_double))
        return u, pr

    def model(self):
        m1, m2, w = (np.zeros(self.model_shape) for _ in range(3))
        self.call("dfg_get_model", ptr(m1, C.c_double), ptr(m2, C.c_double), ptr(w, C.c_double))
        return m1, m2, w

    def frame_params(self):
        n = self.num_data
        sc, be, bs, sf = (np.zeros(n) for _ in range(4))
        fc = np.zeros(n, np.int32)
        bl = np.zeros(n, np.uint8)
        self.call("dfg_get_frame_params", ptr(sc, C.c_double), ptr(be, C.c_double), ptr(bs, C.c_double),
                  ptr(fc, C.c_int), ptr(sf, C.c_double), ptr(bl, C.c_uint8))
        return dict(scale=sc, beta=be, beta_start=bs, fcounts=fc, sum_fact=sf, blacklist=bl)

    def scalars(self):
        out = np.zeros(5)
        self.call("dfg_get_scalars", ptr(out, C.c_double))
        return dict(rescale=out[0], mutual_info=out[1], avg_likelihood=out[2], mean_count=out[3],
                    rms_change=out[4])

    def slice_gen(self, quat, mode=0):
        """Slice at a quaternion (3-D), an angle (2-D) or (phi, beta) (RZ)."""
        q = _quat5(quat)
        out = np.zeros(self.num_pix)
        self.call("dfg_slice_gen", ptr(q, C.c_double), int(mode), ptr(out, C.c_double))
        return out

    def slice_gen_noalloc(self, quat, mode=0):
        """slice_gen through the entry point that allocates no device memory
        (its scratch is a fixed device array of DFG_NOALLOC_MAX_PIXELS)."""
        q = _quat5(quat)
        out = np.zeros(self.num_pix)
        self.call("dfg_slice_gen_noalloc", ptr(q, C.c_double), int(mode), ptr(out, C.c_double))
        return out

    def slice_merge(self, quat, view, model2, inter_weight, mode=0):
        q = _quat5(quat)
        v = np.ascontiguousarray(view, np.float64)
        self.call("dfg_slice_merge", ptr(q, C.c_double), int(mode), ptr(v, C.c_double),
                  ptr(model2, C.c_double), ptr(inter_weight, C.c_double))

    def phase_times(self):
        ms = np.zeros(len(PHASES))
        la = (C.c_long * len(PHASES))()
        self.check(0 if self.lib.dfg_get_phase_times(self.h, ptr(ms, C.c_double), la, len(PHASES)) >= 0 else 1)
        return {PHASES[i]: (ms[i], la[i]) for i in range(len(PHASES))}

    def reset_phase_times(self):
        self.call("dfg_reset_phase_times")

    def simulate_frames(self, intens, quats4, phi, seed):
        """Poisson frames of intens at quats4 [N,4] times phi [N]; they become
        this context's frames. Returns (ones_total, multi_total, photons)."""
        m = np.ascontiguousarray(intens, np.float64)
        q = np.ascontiguousarray(np.asarray(quats4)[:, :4], np.float64)
        f = np.ascontiguousarray(phi, np.float64)
        tot = (C.c_longlong * 3)()
        self.call("dfg_simulate_frames", m.shape[-1], ptr(m, C.c_double), q.shape[0], ptr(q, C.c_double),
                  ptr(f, C.c_double), int(seed), tot)
        self.num_data = q.shape[0]
        self._frame_totals = (tot[0], tot[1])
        return tuple(tot)

    def get_frames(self):
        """The context's sparse frames (ones, multi, place_ones, place_multi, count_multi)."""
        n = self.num_data
        ones, multi = np.zeros(n, np.int32), np.zeros(n, np.int32)
        self.call("dfg_get_frames", ptr(ones, C.c_int), ptr(multi, C.c_int), None, None, None)
        po = np.zeros(int(ones.sum()), np.int32)
        pm = np.zeros(int(multi.sum()), np.int32)
        cm = np.zeros(int(multi.sum()), np.int32)
        self.call("dfg_get_frames", None, None, ptr(po, C.c_int), ptr(pm, C.c_int), ptr(cm, C.c_int))
        return ones, multi, po, pm, cm

    def event_record(self, slot):
        self.call("dfg_event_record", int(slot))

    def event_elapsed_ms(self, a, b):
        ms = C.c_double(0.)
        self.call("dfg_event_elapsed", int(a), int(b), C.byref(ms))
        return ms.value

    def model_rotate(self, model, rot, max_r=0, rotmodel=None):
        """rotate_model on the GPU: rotmodel (zeros when None) += model
        interpolated at rot v + c over the cube [-max_r, max_r)^3; returns
        rotmodel."""
        m = np.ascontiguousarray(model, np.float64)
        if m.ndim != 3 or len(set(m.shape)) != 1:
            raise ValueError("model must be [S, S, S]")
        r = np.ascontiguousarray(rot, np.float64).reshape(3, 3)
        out = np.zeros(m.shape) if rotmodel is None else rotmodel
        if out.shape != m.shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("rotmodel must be a C-contiguous float64 array shaped like model")
        self.call("dfg_model_rotate", ptr(r, C.c_double), m.shape[0], int(max_r), ptr(m, C.c_double),
                  ptr(out, C.c_double))
        return out

    def model_symmetrize(self, group, model, weights, order=0):
        """In-place point-group (group "S4" / "A5") or axial ("axial", order)
        symmetrisation of a model and its weights [S, S, S] (float64,
        C-contiguous)."""
        g = {"S4": 1, "A5": 2, "axial": 3}[group]
        for a in (model, weights):
            if a.ndim != 3 or len(set(a.shape)) != 1 or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("model and weights must be C-contiguous float64 [S, S, S]")
        if model.shape != weights.shape:
            raise ValueError("model and weights differ in shape")
        self.call("dfg_model_symmetrize", g, int(order), model.shape[0], ptr(model, C.c_double),
                  ptr(weights, C.c_double))

    def measure_gather_rate(self, rows, reps=5):
        """GB/s of uniformly random 512-byte row reads from a device table of
        `rows` rows: the ceiling of the E-step / M-step gather pattern."""
        out = C.c_double(0.)
        self.call("dfg_measure_gather_rate", int(rows), int(reps), C.byref(out))
        return out.value

    def workload(self):
        out = (C.c_longlong * 11)()
        self.call("dfg_get_workload", out)
        keys = ("num_orient", "num_data", "estep_entries", "mstep_entries", "chunks", "chunk_frames",
                "launches", "k_pad", "dense_estep", "live_pairs", "block_tiles")
        return dict(zip(keys, list(out)))


class Batch:
    """Independent reconstructions (Contexts on one GPU) iterated together as
    one CUDA graph with a branch per reconstruction (dfg_batch_run)."""

    def __init__(self, contexts):
        self.lib = load()
        self.contexts = list(contexts)
        arr = (_V * len(self.contexts))(*[c.h for c in self.contexts])
        h = _V()
        rc = self.lib.dfg_batch_create(arr, len(self.contexts), C.byref(h))
        if rc != DFG_OK:
            raise DFGError(rc, "dfg_batch_create failed (contexts must be distinct and on one device)")
        self.h = h

    def run(self, pars, alphas=None):
        """One iteration of every reconstruction; pars: one IterParams each.
        Returns a list of dicts as Context.run_iteration's."""
        n = len(self.contexts)
        parr = (IterParams * n)(*pars)
        al = None if alphas is None else np.ascontiguousarray(alphas, np.float64)
        out = np.zeros((n, 5))
        rc = self.lib.dfg_batch_run(self.h, parr, ptr(al, C.c_double), ptr(out, C.c_double))
        if rc != DFG_OK:
            raise DFGError(rc, self.lib.dfg_batch_last_error(self.h).decode())
        keys = ("avg_likelihood", "rms_change", "mutual_info", "rescale", "mean_scale")
        return [dict(zip(keys, row.tolist())) for row in out]

    def set_lanes(self, lanes):
        """Concurrent branches (1: one reconstruction after another)."""
        rc = self.lib.dfg_batch_set_lanes(self.h, int(lanes))
        if rc != DFG_OK:
            raise DFGError(rc, "lanes must be >= 1")

    def stats(self):
        out = (C.c_long * 3)()
        self.lib.dfg_batch_stats(self.h, out)
        return dict(launches=out[0], instantiations=out[1], updates=out[2])

    def close(self):
        if getattr(self, "h", None):
            self.lib.dfg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DetectorGroup:
    """Several detectors in one reconstruction (dfg_group_*): one Context per
    detector holding that detector and the frames it sees, all with the same
    orientations, model and parameters. The model lives in member 0."""

    def __init__(self, contexts):
        self.lib = load()
        self.contexts = list(contexts)
        arr = (_V * len(self.contexts))(*[c.h for c in self.contexts])
        h = _V()
        rc = self.lib.dfg_group_create(arr, len(self.contexts), C.byref(h))
        if rc != DFG_OK:
            raise DFGError(rc, "dfg_group_create failed")
        self.h = h

    def call(self, name, *args):
        rc = getattr(self.lib, name)(self.h, *args)
        if rc != DFG_OK:
            raise DFGError(rc, "%s: %s" % (name, self.lib.dfg_group_last_error(self.h).decode()))

    def maximize(self, par):
        ll = C.c_double(0.)
        self.call("dfg_group_maximize", C.byref(par), C.byref(ll))
        return ll.value

    def update_model(self, alpha=0.):
        rms = C.c_double(0.)
        self.call("dfg_group_update_model", float(alpha), C.byref(rms))
        return rms.value

    def normalize_scale(self):
        m = C.c_double(0.)
        self.call("dfg_group_normalize_scale", C.byref(m))
        return m.value

    def run_iteration(self, par, alpha=0.):
        """As Context.run_iteration, over all detectors."""
        out = np.zeros(5)
        self.call("dfg_group_run_iteration", C.byref(par), float(alpha), ptr(out, C.c_double))
        return dict(zip(("avg_likelihood", "rms_change", "mutual_info", "rescale", "mean_scale"), out.tolist()))

    def model(self):
        return self.contexts[0].model()

    def frame_results(self):
        """Per-frame results of all members, member 0's frames first."""
        parts = [c.frame_results() for c in self.contexts]
        return {k: np.concatenate([p[k] for p in parts]) for k in parts[0]}

    def close(self):
        if getattr(self, "h", None):
            self.lib.dfg_group_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ProposalNet:
    """Orientation-proposal network on the GPU (dfg_pnet_*): 32 x 32 binned
    log(1 + photons) frame images -> logits over num_classes coarse
    orientations; trained and evaluated by the library's own kernels."""

    IMG = 32

    def __init__(self, num_classes, batch=256, seed=1, device=0):
        self.lib = load()
        h = _V()
        rc = self.lib.dfg_pnet_create(int(device), int(num_classes), int(batch), int(seed), C.byref(h))
        if rc != DFG_OK:
            raise DFGError(rc, "dfg_pnet_create failed")
        self.h = h
        self.num_classes = int(num_classes)
        self.n_images = 0

    def _call(self, name, *args):
        rc = getattr(self.lib, name)(self.h, *args)
        if rc != DFG_OK:
            raise DFGError(rc, self.lib.dfg_pnet_last_error(self.h).decode())

    @property
    def num_params(self):
        return int(self.lib.dfg_pnet_num_params(self.h))

    def params(self):
        out = np.zeros(self.num_params, np.float32)
        self._call("dfg_pnet_get_params", ptr(out, C.c_float))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        self._call("dfg_pnet_set_params", ptr(p, C.c_float))

    @staticmethod
    def pixel_bins(qvals, qmax=None):
        """Bin of every pixel on a 32 x 32 grid over the detector plane
        (qx, qy within +-qmax), -1 outside."""
        q = np.asarray(qvals, np.float64).reshape(-1, 3)
        qmax = float(np.abs(q[:, :2]).max()) * 1.0001 if qmax is None else float(qmax)
        ix = np.floor((q[:, 0] + qmax) / (2 * qmax) * ProposalNet.IMG).astype(np.int64)
        iy = np.floor((q[:, 1] + qmax) / (2 * qmax) * ProposalNet.IMG).astype(np.int64)
        ok = (ix >= 0) & (ix < ProposalNet.IMG) & (iy >= 0) & (iy < ProposalNet.IMG)
        return np.where(ok, ix * ProposalNet.IMG + iy, -1).astype(np.int32)

    def set_bins(self, pixel_bin):
        b = np.ascontiguousarray(pixel_bin, np.int32)
        self._call("dfg_pnet_set_bins", b.size, ptr(b, C.c_int))

    def load_frames(self, ctx):
        self._call("dfg_pnet_load_frames", ctx.h)
        self.n_images = int(ctx.num_data)

    def set_images(self, images):
        x = np.ascontiguousarray(images, np.float32).reshape(-1, self.IMG * self.IMG)
        self._call("dfg_pnet_set_images", x.shape[0], ptr(x, C.c_float))
        self.n_images = x.shape[0]

    def images(self):
        out = np.zeros((self.n_images, self.IMG * self.IMG), np.float32)
        self._call("dfg_pnet_get_images", ptr(out, C.c_float))
        return out

    def set_targets(self, offsets, classes, weights):
        """Soft targets of the loaded images (CSR: image i's classes
        classes[offsets[i]:offsets[i + 1]] with weights summing to 1); train()
        and gradients() without labels use them."""
        off = np.ascontiguousarray(offsets, np.int64)
        cls = np.ascontiguousarray(classes, np.int32)
        w = np.ascontiguousarray(weights, np.float32)
        self._call("dfg_pnet_set_targets", ptr(off, C.c_longlong), ptr(cls, C.c_int), ptr(w, C.c_float))

    def train(self, labels=None, epochs=1, lr=1e-3, seed=0):
        """Epochs of Adam against labels, or (labels None) against the soft
        targets of set_targets. Returns the last epoch's mean loss."""
        lab = None if labels is None else np.ascontiguousarray(labels, np.int32)
        loss = C.c_double(0.)
        self._call("dfg_pnet_train", ptr(lab, C.c_int), int(epochs), float(lr), int(seed), C.byref(loss))
        return loss.value

    def set_option(self, key, value):
        self._call("dfg_pnet_set_option", key.encode(), float(value))

    def set_tensor_cores(self, on):
        """Inference products on the tcgen05 tensor cores (default) or the
        FP32 path (CUDA-core products, FP32 activations). Training has its
        own switch, set_option("tensor_core_training", 0 or 1)."""
        self._call("dfg_pnet_set_tensor_cores", 1 if on else 0)

    def topk(self, K):
        out = np.zeros((self.n_images, int(K)), np.int32)
        self._call("dfg_pnet_topk", int(K), ptr(out, C.c_int))
        return out

    def topk_mass(self, K_min, K_max, mass):
        """[n, K_max]: per image the classes by decreasing logit, K_min and
        then more until their softmax probabilities sum to mass (at most
        K_max); unused slots -1."""
        out = np.zeros((self.n_images, int(K_max)), np.int32)
        self._call("dfg_pnet_topk_mass", int(K_min), int(K_max), float(mass), ptr(out, C.c_int))
        return out

    def logits(self):
        out = np.zeros((self.n_images, self.num_classes), np.float32)
        self._call("dfg_pnet_logits", ptr(out, C.c_float))
        return out

    def gradients(self, labels=None):
        lab = None if labels is None else np.ascontiguousarray(labels, np.int32)
        g = np.zeros(self.num_params, np.float32)
        loss = C.c_double(0.)
        self._call("dfg_pnet_gradients", ptr(lab, C.c_int), ptr(g, C.c_float), C.byref(loss))
        return g, loss.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.dfg_pnet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
