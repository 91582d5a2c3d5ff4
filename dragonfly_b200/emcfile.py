"""Sparse photon files (mirror of dragonfly.emcfile, dragonfly/emcfile.pyx).

Binary .emc layout (dragonfly/src/emcfile.c:3-38, writer emcfile.pyx:491-532):
a 1024-byte header of int32 (num_data, num_pix, ftype = 0 for sparse), then
int32 ones[num_data], multi[num_data], place_ones[sum ones],
place_multi[sum multi], count_multi[sum multi]. HDF5 .emc files (vlen
place_ones / place_multi / count_multi and num_pix) are read and written when
h5py is importable.
"""
import os
import os.path as op

import numpy as np

try:
    import h5py
except ImportError:
    h5py = None

HEADER_BYTES = 1024
SPARSE, DENSE_INT, DENSE_DOUBLE = 0, 1, 2


def read_emc(fname):
    """(num_pix, ones, multi, place_ones, place_multi, count_multi) of a sparse
    .emc file."""
    if h5py is not None and h5py.is_hdf5(fname):
        with h5py.File(fname, "r") as f:
            num_pix = int(np.asarray(f["num_pix"][()]).ravel()[0])
            po = [np.asarray(x, np.int32) for x in f["place_ones"][:]]
            pm = [np.asarray(x, np.int32) for x in f["place_multi"][:]]
            cm = [np.asarray(x, np.int32) for x in f["count_multi"][:]]
        ones = np.array([len(x) for x in po], np.int32)
        multi = np.array([len(x) for x in pm], np.int32)
        cat = lambda xs: np.concatenate(xs).astype(np.int32) if xs else np.zeros(0, np.int32)
        return num_pix, ones, multi, cat(po), cat(pm), cat(cm)
    with open(fname, "rb") as f:
        head = np.fromfile(f, np.int32, 3)
        if head.size < 3:
            raise ValueError("%s: truncated header" % fname)
        num_data, num_pix, ftype = (int(x) for x in head)
        if ftype != SPARSE:
            raise ValueError("%s: only sparse .emc files are supported (ftype %d)" % (fname, ftype))
        if num_data < 0 or num_pix <= 0:
            raise ValueError("%s: bad header (num_data %d, num_pix %d)" % (fname, num_data, num_pix))
        f.seek(HEADER_BYTES)
        ones = np.fromfile(f, np.int32, num_data)
        multi = np.fromfile(f, np.int32, num_data)
        if ones.size != num_data or multi.size != num_data:
            raise ValueError("%s: truncated ones/multi arrays" % fname)
        no, nm = int(ones.sum()), int(multi.sum())
        po = np.fromfile(f, np.int32, no)
        pm = np.fromfile(f, np.int32, nm)
        cm = np.fromfile(f, np.int32, nm)
        if po.size != no or pm.size != nm or cm.size != nm:
            raise ValueError("%s: truncated photon arrays" % fname)
    return num_pix, ones, multi, po, pm, cm


def write_emc(fname, num_pix, ones, multi, place_ones, place_multi, count_multi, header_nums=None):
    header = np.zeros(HEADER_BYTES // 4, np.int32)
    header[0] = len(ones)
    header[1] = num_pix
    if header_nums is not None:
        h = np.asarray(header_nums).astype("i4")[:254]
        header[2:2 + h.size] = h
    with open(fname, "wb") as f:
        header.tofile(f)
        for a in (ones, multi, place_ones, place_multi, count_multi):
            np.asarray(a, np.int32).tofile(f)


class CDataset:
    """A sparse photon dataset, optionally linked to further datasets
    (emcfile.pyx:18-149)."""

    def __init__(self, fname=None, det=None):
        self._det = det
        self._fname = ""
        self._next = None
        self.num_pix = 0
        self.ftype = "sparse"
        self._set_arrays(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32),
                         np.zeros(0, np.int32), np.zeros(0, np.int32))
        if fname is not None:
            self.parse(fname)

    @classmethod
    def from_arrays(cls, ones, multi, place_ones, place_multi, count_multi, det=None, num_pix=None):
        """A dataset from in-memory sparse arrays."""
        d = cls(det=det)
        d._set_arrays(ones, multi, place_ones, place_multi, count_multi)
        d.num_pix = num_pix if num_pix is not None else (det.num_pix if det is not None else 0)
        return d

    def _set_arrays(self, ones, multi, po, pm, cm):
        self.ones = np.ascontiguousarray(ones, np.int32)
        self.multi = np.ascontiguousarray(multi, np.int32)
        self.place_ones = np.ascontiguousarray(po, np.int32)
        self.place_multi = np.ascontiguousarray(pm, np.int32)
        self.count_multi = np.ascontiguousarray(cm, np.int32)
        if self.ones.size != self.multi.size:
            raise ValueError("ones and multi lengths differ")
        if self.place_ones.size != int(self.ones.sum()) or self.place_multi.size != int(self.multi.sum()) \
                or self.count_multi.size != self.place_multi.size:
            raise ValueError("photon arrays do not match the per-frame counts")

    def parse(self, fname):
        if self._det is None:
            raise AttributeError("Set detector before parsing")
        num_pix, *arrs = read_emc(fname)
        self._fname = fname
        self.num_pix = num_pix
        if num_pix != self._det.num_pix:
            print("WARNING! The detector file and photons file %s do not have the same number of pixels"
                  % fname)
        self._set_arrays(*arrs)

    def append(self, next_dset):
        curr = self
        while curr._next is not None:
            curr = curr._next
        curr._next = next_dset

    def free(self):
        pass

    def __iter__(self):
        curr = self
        while curr is not None:
            yield curr
            curr = curr._next

    @property
    def fname(self):
        return self._fname

    @property
    def num_data(self):
        return int(self.ones.size)

    @property
    def det(self):
        return self._det

    @det.setter
    def det(self, det):
        self._det = det

    @property
    def next(self):
        return self._next

    @property
    def ones_total(self):
        return int(self.place_ones.size)

    @property
    def multi_total(self):
        return int(self.place_multi.size)

    @property
    def ones_accum(self):
        return (np.cumsum(self.ones, dtype=np.int64) - self.ones).astype(np.int64)

    @property
    def multi_accum(self):
        return (np.cumsum(self.multi, dtype=np.int64) - self.multi).astype(np.int64)


class EMCReader:
    """Random access to frames of one or more sparse .emc files
    (emcfile.pyx:151-400)."""

    def __init__(self, photons_list, det_list, dset_list=None, det_mapping=None):
        if isinstance(photons_list, str):
            photons_list = [photons_list]
        if not isinstance(det_list, (list, tuple)):
            det_list = [det_list]
        self.flist = list(photons_list)
        self.dets = list(det_list)
        self.det_mapping = list(det_mapping) if det_mapping is not None else \
            [0 if len(self.dets) == 1 else i for i in range(len(self.flist))]
        self._data = [read_emc(f) for f in self.flist]
        self.num_frames = sum(d[1].size for d in self._data)
        self._starts = np.cumsum([0] + [d[1].size for d in self._data])

    def _locate(self, num):
        if num < 0 or num >= self.num_frames:
            raise IndexError("frame %d out of range" % num)
        k = int(np.searchsorted(self._starts, num, side="right") - 1)
        return k, num - int(self._starts[k])

    def get_frame(self, num, raw=False, sparse=False, **kwargs):
        k, i = self._locate(num)
        num_pix, ones, multi, po, pm, cm = self._data[k]
        o0 = int(ones[:i].sum())
        m0 = int(multi[:i].sum())
        p1 = po[o0:o0 + ones[i]]
        p2 = pm[m0:m0 + multi[i]]
        c2 = cm[m0:m0 + multi[i]]
        if sparse:
            return p1, p2, c2
        frame = np.zeros(num_pix, np.int32)
        frame[p1] = 1
        frame[p2] = c2
        if raw:
            return frame
        det = self.dets[self.det_mapping[k]]
        if hasattr(det, "assemble_frame"):
            return det.assemble_frame(frame, **kwargs)
        return frame

    def get_powder(self, raw=False, **kwargs):
        out = None
        for k, (num_pix, ones, multi, po, pm, cm) in enumerate(self._data):
            p = np.bincount(po, minlength=num_pix).astype(np.float64)
            p += np.bincount(pm, weights=cm, minlength=num_pix)
            out = p if out is None else out + p
        if raw or not hasattr(self.dets[0], "assemble_frame"):
            return out
        return self.dets[0].assemble_frame(out, **kwargs)


class EMCWriter:
    """Writes sparse frames (emcfile.pyx:259-440)."""

    def __init__(self, out_fname, num_pix, hdf5=True):
        self.h5_output = bool(hdf5) and h5py is not None
        self.out_fname = out_fname
        self.num_data = 0
        self.num_pix = num_pix
        self.mean_count = 0.
        self.ones, self.multi = [], []
        self._po, self._pm, self._cm = [], [], []

    def __enter__(self):
        return self

    def __exit__(self, etype, val, traceback):
        self.finish_write()

    def write_frame(self, frame, fraction=1., partition=1):
        frame = np.asarray(frame)
        if frame.ndim != 1 or not np.issubdtype(frame.dtype, np.integer):
            raise ValueError("write_frame needs 1D array of integers: %s %s" % (frame.shape, frame.dtype))
        if fraction < 1. or partition > 1:
            raise NotImplementedError("photon sub-sampling (fraction / partition) is not supported")
        place_ones = np.where(frame == 1)[0]
        place_multi = np.where(frame > 1)[0]
        self._update(place_ones, place_multi, frame[place_multi])

    def write_sparse_frame(self, place_ones, place_multi, count_multi):
        if len(place_multi) != len(count_multi):
            raise ValueError("place_multi and count_multi should have equal lengths")
        a = [np.asarray(x) for x in (place_ones, place_multi, count_multi)]
        if not all(np.issubdtype(x.dtype, np.integer) or x.size == 0 for x in a):
            raise ValueError("Arrays should be of integer type")
        self._update(*a)

    def _update(self, po, pm, cm):
        self.num_data += 1
        self.mean_count += len(po) + int(np.sum(cm))
        self.ones.append(len(po))
        self.multi.append(len(pm))
        self._po.append(np.asarray(po, np.int32))
        self._pm.append(np.asarray(pm, np.int32))
        self._cm.append(np.asarray(cm, np.int32))

    def finish_write(self, header_nums=None):
        if self.num_data == 0:
            print("No frames to write")
            return
        mean = self.mean_count / self.num_data
        print("num_data = %d, mean_count = %.4e" % (self.num_data, mean))
        if self.h5_output:
            with h5py.File(self.out_fname, "w") as f:
                f["num_pix"] = [self.num_pix]
                vl = h5py.special_dtype(vlen=np.int32)
                for name, lst in (("place_ones", self._po), ("place_multi", self._pm), ("count_multi", self._cm)):
                    ds = f.create_dataset(name, (self.num_data,), dtype=vl)
                    for i, x in enumerate(lst):
                        ds[i] = x
        else:
            write_emc(self.out_fname, self.num_pix, np.array(self.ones, np.int32), np.array(self.multi, np.int32),
                      np.concatenate(self._po), np.concatenate(self._pm), np.concatenate(self._cm), header_nums)
        self.num_data = 0
        self.ones, self.multi, self._po, self._pm, self._cm = [], [], [], [], []
