"""State of an EMC reconstruction (mirror of dragonfly.iterate.Iterate,
dragonfly/iterate.pyx:21-592).

Holds the detector(s), the photon datasets, orientations, model, parameters
and the per-frame arrays (fcounts, scale, beta, beta_start, sum_fact,
blacklist) on the host; EMCRecon uploads them to the GPU. Several detectors
(in_detector_list) map each dataset to one of the unique detectors as the
reference's _gen_detlist does (iterate.pyx:432-456); the frames seen by
detector k are member_frames(k) / member_index(k).
"""
import configparser
import ctypes
import ctypes.util
import math
import os.path as op
import re

import numpy as np

from .detector import CDetector
from .emcfile import CDataset
from .model import Model
from .params import MyConfigParser, EMCParams, RECON3D, RECON2D, RECONRZ
from .quaternion import Quaternion

try:
    import h5py
except ImportError:
    h5py = None


_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.lgamma.restype = ctypes.c_double
_libm.lgamma.argtypes = [ctypes.c_double]


def ln_factorial(c):
    """ln(c!) as the C library's lgamma(c + 1), which the device library and
    the oracle also use (Python's math.lgamma rounds differently)."""
    return _libm.lgamma(float(c) + 1.0)


def frame_stats(dsets, mask, det_mapping=None, num_det=1):
    """fcounts, sum_fact and mean_count over mask == 0 pixels (calc_frame_counts
    and calc_sum_fact, dragonfly/src/iterate.c:3-117; ln c! = lgamma(c + 1)).
    mask: one array, or one per detector with det_mapping giving each
    dataset's detector; mean_count is then per detector (an array)."""
    fc, sf = [], []
    for i, d in enumerate(dsets):
        m = mask if det_mapping is None else mask[det_mapping[i]]
        n = d.num_data
        good1 = m[d.place_ones] < 1
        good_m = m[d.place_multi] < 1
        fid1 = np.repeat(np.arange(n), d.ones)
        fidm = np.repeat(np.arange(n), d.multi)
        f = np.bincount(fid1[good1], minlength=n).astype(np.int64)
        f += np.bincount(fidm[good_m], weights=d.count_multi[good_m], minlength=n).astype(np.int64)
        lf = np.array([ln_factorial(c) for c in d.count_multi], np.float64)
        s = np.zeros(n)
        # sequential per-frame sums, in file order, as the reference adds them
        for i in np.nonzero(good_m)[0]:
            s[fidm[i]] += lf[i]
        fc.append(f.astype(np.int32))
        sf.append(s)
    fcounts = np.concatenate(fc)
    if det_mapping is None:
        mean_count = float(np.cumsum(fcounts.astype(np.float64))[-1] / fcounts.size) if fcounts.size else 0.
        return fcounts, np.concatenate(sf), mean_count
    # per detector: the sequential sum over its frames in dataset order
    # (cumsum adds in order, as the reference's loop), then / count
    mean_count = np.zeros(num_det)
    for k in range(num_det):
        parts = [f for i, f in enumerate(fc) if det_mapping[i] == k]
        v = np.concatenate(parts).astype(np.float64) if parts else np.zeros(0)
        mean_count[k] = np.cumsum(v)[-1] / v.size if v.size else 0.
    return fcounts, np.concatenate(sf), mean_count


class Iterate:
    def __init__(self, config_fname="", section_name="emc", resume=False):
        self.params = EMCParams()
        self.dets = []
        self.data = None
        self.quat = None
        self.model = None
        self.tot_num_data = 0
        self.num_blacklist = 0
        self.fcounts = self.scale = self.bgscale = self.beta = self.beta_start = None
        self.sum_fact = self.blacklist = None
        self.rel_quat = None  # relevant coarse orientations per frame (refinement)
        self.mean_count = None
        self.rescale = None
        self.likelihood = 0.
        self.mutual_info = 0.
        self.rms_change = 0.
        if config_fname != "":
            self.from_config(config_fname, section_name, resume=resume)

    # -- construction --------------------------------------------------------
    def from_config(self, config_fname, section_name="emc", resume=False):
        """iterate.pyx:40-182"""
        param = EMCParams()
        param.from_config(config_fname, section_name)
        self.set_params(param)
        rtype = {RECON3D: "3d", RECON2D: "2d", RECONRZ: "rz"}[param.rtype]
        if rtype == "rz":
            # recon.pyx:86-91 selects no slice functions for RZ iterations
            raise NotImplementedError("RZ reconstructions: Model.slice_gen / slice_merge only")
        print("Doing %s recon from %s" % (rtype.upper(), config_fname))
        folder = op.dirname(config_fname)
        config = MyConfigParser()
        config.read(config_fname)

        def chained(key):
            v = config.get(section_name, key, fallback=None)
            if v is not None and ":::" in v:
                s, o = re.split(":::", v)
                v = config.get(s, o)
            return v

        det_fname, det_flist = chained("in_detector_file"), chained("in_detector_list")
        if det_fname is not None and det_flist is not None:
            raise ValueError("Both in_detector_file and in_detector_list specified. Pick one.")
        if det_fname is not None:
            dets = [CDetector(op.join(folder, det_fname), norm=True, rtype=rtype)]
        elif det_flist is not None:
            with open(op.join(folder, det_flist)) as f:
                dets = [CDetector(op.join(folder, ln.strip()), norm=True, rtype=rtype) for ln in f.readlines()]
        else:
            raise ValueError("Need either in_detector_file or in_detector_list.")

        ph_fname, ph_flist = chained("in_photons_file"), chained("in_photons_list")
        if ph_fname is not None and ph_flist is not None:
            raise ValueError("Both in_photons_file and in_photons_list specified. Pick one.")
        if ph_fname is not None:
            if len(dets) > 1:
                print("WARNING: Multiple detectors but only one photons file. Using first detector")
            frames = CDataset(op.join(folder, ph_fname), dets[0])
        elif ph_flist is not None:
            with open(op.join(folder, ph_flist)) as f:
                fnames = [op.join(folder, ln.strip()) for ln in f.readlines()]
            # file i is seen by detector i with a detector list, else by the one
            frames = CDataset(fnames[0], dets[0])
            for i, fn in enumerate(fnames[1:], 1):
                frames.append(CDataset(fn, dets[i] if len(dets) > 1 else dets[0]))
        else:
            raise ValueError("Need either in_photons_file or in_photons_list.")
        # per-pixel background (iterate.pyx:109-127): one file, or a list with
        # one entry per detector
        bg_file = config.get(section_name, "background_file", fallback=None)
        bg_list = config.get(section_name, "background_list", fallback=None)
        if bg_file is not None and bg_list is not None:
            raise ValueError("Both background_file and background_list specified. Pick one.")
        if bg_list is not None:
            bg_list = op.join(folder, bg_list)
            with open(bg_list) as f:
                lines = [ln.strip() for ln in f if ln.strip()]
            if len(lines) != len(dets):
                raise ValueError("Background list has %d entries but there are %d unique detectors"
                                 % (len(lines), len(dets)))
            for det, ln in zip(dets, lines):
                det.parse_background(op.join(op.dirname(bg_list), ln))
        elif bg_file is not None:
            for det in dets:
                det.parse_background(op.join(folder, bg_file))
        self.set_data(frames)

        quat = Quaternion()
        quat.from_config(config_fname, section_name)
        self.set_quat(quat)

        def fname_opt(key):
            try:
                return config.get_filename(section_name, key)
            except configparser.NoOptionError:
                return ""
        model_file, scale_file = fname_opt("start_model_file"), fname_opt("scale_file")
        bgscale_file = fname_opt("bgscale_file")
        probs_file = fname_opt("probs_file")
        if resume:
            with open(param.log_fname) as f:
                last_iter = int(f.readlines()[-1].split()[0])
            self.params.start_iter = last_iter + 1
            ext = ".h5" if h5py is not None else ".npz"
            model_file = op.join(param.output_folder, "output_%.3d%s" % (last_iter, ext))
            scale_file = model_file
            if param.refine and not probs_file:
                probs_file = model_file
            print("Resuming from iteration", self.params.start_iter)
        # refinement (src/iterate.c:103-130): fine orientations mapped to their
        # nearest coarse one, relevant coarse orientations per frame from an
        # earlier coarse run
        if param.refine:
            if not probs_file:
                raise ValueError("Need coarse probabilities in probs_file to do refinement")
            if quat.quat_mapping is None:
                quat.voronoi_subset(param.coarse_div)
            self.parse_rel_quat(probs_file, quat.num_rot_coarse)

        qmax = max(det.qmax() for det in self.dets)
        model = Model(self.calculate_size(qmax), param.num_modes, rtype)
        model_mean = self.mean_count[0] / (self.dets[0].raw_mask == 0).sum() * 2.
        model.allocate(model_file, model_mean, fixed_seed=bool(param.fixed_seed))
        self.set_model(model)
        if param.need_scaling == 1:
            self.parse_scale(scale_file)
            self.parse_scale(bgscale_file, bg=True)
        sel_string = config.get(section_name, "selection", fallback=None)
        self.parse_blacklist(fname_opt("blacklist_file"), sel_string)
        beta_str = config.get(section_name, "beta", fallback="auto")
        self.calc_beta() if beta_str == "auto" else self.calc_beta(float(beta_str))

    def set_model(self, model):
        self.model = model

    def set_quat(self, quat):
        self.quat = quat

    def set_params(self, param):
        self.params = param

    def set_data(self, in_dset):
        """iterate.pyx:241-266"""
        if self.tot_num_data != 0:
            raise ValueError("Please use update_data() to change dataset")
        self._attach(in_dset)

    def update_data(self, in_dset):
        self._attach(in_dset)
        if self.params.need_scaling == 1:
            self.parse_scale("")
        self.calc_beta()

    def _attach(self, in_dset):
        """Iterate.set_data's bookkeeping (iterate.pyx:241-266): frame
        offsets, the unique detectors and each dataset's detector
        (_gen_detlist, iterate.pyx:432-456: unique detector file names in
        sorted order; datasets without a detector use the first), frame
        counts, sum_fact and per-detector mean counts."""
        self.data = in_dset
        dsets = list(in_dset)
        dets = [d.det if d.det is not None else (self.dets[0] if self.dets else None) for d in dsets]
        if dets[0] is None:
            raise AttributeError("Set a detector for the dataset")
        # one key per distinct detector: its file name, else the object
        keys = [dt.fname if dt.fname else "<%d>" % id(dt) for dt in dets]
        uniq, first, mapping = np.unique(np.array(keys, dtype=object), return_index=True, return_inverse=True)
        self.dets = [dets[i] for i in first]
        self._det_mapping = np.asarray(mapping, np.int32).ravel()
        self.tot_num_data = sum(d.num_data for d in dsets)
        fc, sf, mc = frame_stats(dsets, [dt.raw_mask for dt in self.dets], self._det_mapping, len(self.dets))
        self.fcounts, self.sum_fact = fc, sf
        self.mean_count = mc
        self.rescale = np.zeros(len(self.dets))
        self.blacklist = np.zeros(self.tot_num_data, np.uint8)

    def member_index(self, k):
        """Global indices of the frames seen by detector k, in frame order."""
        ds = list(self.data)
        off = np.concatenate([[0], np.cumsum([d.num_data for d in ds])])
        parts = [np.arange(off[i], off[i + 1]) for i in range(len(ds)) if self._det_mapping[i] == k]
        return np.concatenate(parts).astype(np.int64) if parts else np.zeros(0, np.int64)

    def member_frames(self, k):
        """The datasets seen by detector k as one set of sparse arrays."""
        ds = [d for i, d in enumerate(self.data) if self._det_mapping[i] == k]
        cat = lambda key: np.concatenate([getattr(d, key) for d in ds]).astype(np.int32)
        return tuple(cat(key) for key in ("ones", "multi", "place_ones", "place_multi", "count_multi"))

    def merged_frames(self):
        """The linked datasets as one set of sparse arrays (one detector)."""
        ds = list(self.data)
        cat = lambda k: np.concatenate([getattr(d, k) for d in ds]).astype(np.int32)
        return tuple(cat(k) for k in ("ones", "multi", "place_ones", "place_multi", "count_multi"))

    # -- per-frame parameters -------------------------------------------------
    def parse_scale(self, fname, bg=False):
        """iterate.pyx:284-315; bg selects the per-frame background scales."""
        if not fname or not op.isfile(fname):
            if self.tot_num_data == 0:
                raise AttributeError("Need tot_num_data to initialize scale factors")
            scale = np.ones(self.tot_num_data)
        elif fname.endswith(".npz") or h5py is None:
            scale = np.load(fname)["scale"]
        else:
            with h5py.File(fname, "r") as f:
                scale = f["scale"][:]
        scale = np.asarray(scale, np.float64)
        if self.tot_num_data == 0:
            self.tot_num_data = scale.shape[0]
        elif self.tot_num_data < scale.shape[0]:
            print("More scale factors than required. Taking only first", self.tot_num_data)
            scale = scale[:self.tot_num_data]
        elif self.tot_num_data > scale.shape[0]:
            print("Insufficient scale factors in file. Setting rest to unity")
            scale = np.append(scale, np.ones(self.tot_num_data - scale.shape[0]))
        if bg:
            self.bgscale = scale.copy()
        else:
            self.scale = scale.copy()

    def parse_rel_quat(self, fname, num_rot_coarse):
        """Relevant coarse orientations per frame for refinement
        (parse_rel_quat, src/iterate.c:364-527). From an output file of an
        earlier (coarse) run: the saved probability lists when there are any
        (their orientation count must be num_rot_coarse), else the most
        likely orientation of each frame. From a binary file: int32 num_data
        and num_rot at the start, then from byte 1024 int32 counts [num_data]
        followed by each frame's list. Sets ``rel_quat`` (list of int32
        arrays)."""
        if fname.endswith(".npz") or fname.endswith(".h5"):
            if fname.endswith(".npz"):
                f = np.load(fname)
                get = lambda k: f[k.replace("/", "__")] if k.replace("/", "__") in f.files else None
            else:
                if h5py is None:
                    raise ImportError("h5py is needed to read " + fname)
                h = h5py.File(fname, "r")
                get = lambda k: h[k][()] if k in h else None
            num_rot = get("probabilities/num_rot")
            if num_rot is None:
                print("No probabilities saved. Using most likely orientations")
                rmax = np.asarray(get("orientations"), np.int32)
                if rmax.shape[0] != self.tot_num_data:
                    raise ValueError("num_data of orientations (%d) does not match %d"
                                     % (rmax.shape[0], self.tot_num_data))
                rel = [rmax[d:d + 1] for d in range(rmax.shape[0])]
            else:
                if int(np.ravel(num_rot)[0]) != num_rot_coarse:
                    raise ValueError("Rotation sampling in probs file does not match num_rot_coarse: %d vs %d"
                                     % (int(np.ravel(num_rot)[0]), num_rot_coarse))
                off = np.asarray(get("probabilities/offsets"), np.int64)
                place = np.asarray(get("probabilities/place"), np.int32)
                if off.shape[0] - 1 != self.tot_num_data:
                    raise ValueError("num_data of rel_quat (%d) does not match %d"
                                     % (off.shape[0] - 1, self.tot_num_data))
                rel = [place[off[d]:off[d + 1]] for d in range(off.shape[0] - 1)]
            if not fname.endswith(".npz"):
                h.close()
        else:
            with open(fname, "rb") as f:
                num_data, num_rot = np.fromfile(f, np.int32, 2)
                if num_data != self.tot_num_data:
                    raise ValueError("num_data of rel_quat (%d) does not match" % num_data)
                if num_rot != num_rot_coarse:
                    raise ValueError("Rotation sampling in probs file does not match num_rot_coarse: %d vs %d"
                                     % (num_rot, num_rot_coarse))
                f.seek(1024)
                counts = np.fromfile(f, np.int32, num_data)
                flat = np.fromfile(f, np.int32, int(counts.sum()))
            off = np.zeros(num_data + 1, np.int64)
            np.cumsum(counts, out=off[1:])
            rel = [flat[off[d]:off[d + 1]] for d in range(num_data)]
        self.rel_quat = rel
        return rel

    def parse_blacklist(self, fname, sel_string=None, refresh=False):
        """iterate.pyx:317-359 (num_blacklist is left at 0, as there)."""
        if self.tot_num_data == 0:
            raise AttributeError("Need to define tot_num_data before generating blacklist")
        if self.blacklist is None or refresh:
            self.blacklist = np.zeros(self.tot_num_data, np.uint8)
        if fname and op.isfile(fname):
            arr = np.loadtxt(fname, dtype="u1")
            if arr.shape[0] != self.tot_num_data:
                raise ValueError("Mismatched number of frames in blacklist file")
            self.blacklist[:] = arr
        if sel_string is None:
            return
        if sel_string == "odd_only":
            curr = 0
        elif sel_string == "even_only":
            curr = 1
        else:
            raise ValueError("Unrecognized sel_string, %s" % sel_string)
        for d in range(self.tot_num_data):
            if self.blacklist[d] == 0:
                self.blacklist[d] = curr
                curr = 1 - curr

    def calc_beta(self, setval=None):
        """iterate.pyx:386-402 -> iterate.c:66-83"""
        if self.data is None:
            raise AttributeError("Add data first before calculating beta for each frame")
        start = -1. if setval is None else float(setval)
        if not self.params.need_scaling and start < 0:
            start = math.exp(-6.5 * math.pow(self.mean_count[0] * 1.e-5, 0.15))
        if start > 0:
            self.beta_start = np.full(self.tot_num_data, start)
        else:
            self.beta_start = np.array([math.exp(-6.5 * math.pow(f * 1.e-5, 0.15)) for f in self.fcounts])
        self.beta = self.beta_start.copy()

    def normalize_scale(self):
        """iterate.pyx:361-384"""
        blist = self.blacklist
        mean_scale = self.scale.mean() if blist is None else self.scale[blist == 0].mean()
        if self.model is not None and self.model.model1 is not None:
            self.model.model1.reshape(-1)[:self.model.vol] *= mean_scale
        if blist is None:
            self.scale /= mean_scale
        else:
            self.scale[blist == 0] /= mean_scale
        self.rms_change *= mean_scale
        return mean_scale

    def free(self):
        pass

    @staticmethod
    def calculate_size(qmax):
        """iterate.pyx:458-468"""
        return int(2 * np.ceil(qmax) + 3)

    @property
    def det(self):
        return self.dets[0] if self.dets else None

    @property
    def num_det(self):
        return len(self.dets)

    @property
    def num_dfiles(self):
        return 0 if self.data is None else len(list(self.data))

    @property
    def det_mapping(self):
        if self.data is None:
            return None
        return self._det_mapping.copy()
