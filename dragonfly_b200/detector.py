"""Detector objects (mirror of dragonfly.detector, dragonfly/detector.pyx).

CDetector holds what the iteration uses: per-pixel q-vectors in voxel units
(qvals [P,3]), solid-angle/polarisation corrections (corr), the raw mask
(0 good, 1 merge only, 2 bad), detector distance and Ewald radius. Detector
adds the 2-D pixel geometry used to assemble frames.

Files: the reference's HDF5 layout (datasets qx, qy, qz, corr, mask, detd,
ewald_rad, optional background) when h5py is importable; otherwise, and for
names ending in .npz, the same keys in a numpy .npz archive.
"""
import numpy as np

try:
    import h5py
except ImportError:  # h5py is optional
    h5py = None


def _read_arrays(fname, keys):
    if fname.endswith(".npz") or h5py is None:
        with np.load(fname) as f:
            return {k: (f[k] if k in f else None) for k in keys}
    if not h5py.is_hdf5(fname):
        raise TypeError("Need HDF5 format detector file")
    with h5py.File(fname, "r") as f:
        return {k: (f[k][()] if k in f else None) for k in keys}


class CDetector:
    """Detector as the iteration sees it (detector.pyx:15-222)."""

    def __init__(self, fname=None, **kwargs):
        self._fname = ""
        self._qvals = None
        self._corr = None
        self._raw_mask = None
        self._background = None
        self.with_bg = 0
        self.detd = 0.
        self.ewald_rad = 0.
        if fname is not None:
            self.parse(fname, **kwargs)

    def parse(self, fname, norm=True, rtype="3d"):
        """Reads a detector file; corr is divided by its mean when norm
        (detector.pyx:55-57)."""
        a = _read_arrays(fname, ("qx", "qy", "qz", "corr", "mask", "detd", "ewald_rad"))
        self._fname = fname
        qx, qy, qz = (np.asarray(a[k], np.float64).ravel() for k in ("qx", "qy", "qz"))
        corr = np.asarray(a["corr"], np.float64).ravel().copy()
        self.detd = float(a["detd"])
        self.ewald_rad = float(a["ewald_rad"])
        self.with_bg = 0
        if norm:
            corr /= corr.mean()
        if rtype == "2d":
            qx, qy, qz = self._convert_2d(qx, qy, qz)
        self._qvals = np.ascontiguousarray(np.stack([qx, qy, qz], axis=1))
        self._corr = corr
        self._raw_mask = np.asarray(a["mask"]).astype(np.uint8).ravel()

    def free(self):
        self._qvals = self._corr = self._raw_mask = self._background = None

    def parse_background(self, fname):
        a = _read_arrays(fname, ("background",))
        self.background = np.asarray(a["background"], np.float64).ravel()
        self.with_bg = 1

    def qmax(self):
        """Largest |q| over pixels (detector.pyx:106-117)."""
        return float(np.sqrt((self._qvals ** 2).sum(1).max()))

    def _convert_2d(self, qx, qy, qz):
        if qz.mean() > 0:
            f = self.detd / (self.ewald_rad - qz)
        else:
            f = self.detd / (self.ewald_rad + qz)
        return qx * f, qy * f, np.zeros_like(qz)

    def _check_len(self, n):
        if self.num_pix > 0 and n != self.num_pix:
            raise ValueError("num_pix mismatch with other data (%d vs %d)" % (n, self.num_pix))

    @property
    def fname(self):
        return self._fname

    @property
    def num_pix(self):
        for a in (self._qvals, self._corr, self._raw_mask):
            if a is not None:
                return a.shape[0]
        return 0

    @property
    def qvals(self):
        return self._qvals

    @qvals.setter
    def qvals(self, arr):
        arr = np.asarray(arr)
        if arr.ndim != 2 or arr.shape[1] != 3:
            raise ValueError("qvals must be  2D array of shape (N, 3)")
        if arr.dtype != np.float64:
            raise TypeError("qvals must be double precision floats (float64)")
        self._check_len(arr.shape[0])
        self._qvals = np.ascontiguousarray(arr).copy()

    @property
    def corr(self):
        return self._corr

    @corr.setter
    def corr(self, arr):
        arr = np.asarray(arr)
        if arr.ndim != 1 or arr.dtype != np.float64:
            raise ValueError("corr must be  1D array of float64 dtype")
        self._check_len(arr.shape[0])
        self._corr = arr.copy()

    @property
    def raw_mask(self):
        return self._raw_mask

    @raw_mask.setter
    def raw_mask(self, arr):
        arr = np.asarray(arr)
        if arr.ndim != 1 or arr.dtype != np.uint8:
            raise ValueError("raw_mask must be  1D array of uint8 dtype")
        self._check_len(arr.shape[0])
        self._raw_mask = arr.copy()

    @property
    def background(self):
        return self._background

    @background.setter
    def background(self, arr):
        arr = np.asarray(arr)
        if arr.ndim != 1 or arr.dtype != np.float64:
            raise ValueError("background must be  1D array of float64 dtype")
        self._check_len(arr.shape[0])
        self._background = arr.copy()


class Detector(CDetector):
    """Detector with 2-D pixel geometry (detector.pyx:224-449)."""

    def __init__(self, fname=None, **kwargs):
        self._qrad = None
        super().__init__(fname, **kwargs)

    def parse(self, fname, mask_flag=True, keep_mask_1=True, **kwargs):
        super().parse(fname, **kwargs)
        self._process_det(mask_flag=mask_flag, keep_mask_1=keep_mask_1)

    def write(self, fname):
        """Writes the detector (HDF5 with h5py and a non-.npz name, else .npz)."""
        for a in ("qvals", "corr", "raw_mask"):
            if getattr(self, a) is None:
                raise AttributeError("Detector attributes not populated. Cannot write to file")
        d = dict(qx=self.qvals[:, 0].astype("f8"), qy=self.qvals[:, 1].astype("f8"),
                 qz=self.qvals[:, 2].astype("f8"), corr=self.corr.astype("f8"),
                 mask=self.raw_mask.astype("u1"), detd=float(self.detd), ewald_rad=float(self.ewald_rad))
        if self.background is not None:
            d["background"] = self.background.astype("f8")
        if h5py is None or fname.endswith(".npz"):
            np.savez(fname, **d)
        else:
            with h5py.File(fname, "w") as f:
                for k, v in d.items():
                    f[k] = v

    def calc_from_coords(self, pol="x"):
        """qvals and corr from pixel coordinates cx, cy, detd and ewald_rad
        (detector.pyx:317-352)."""
        cx = np.asarray(self.cx, np.float64).ravel()
        cy = np.asarray(self.cy, np.float64).ravel()
        if self.detd == 0. or self.ewald_rad == 0.:
            raise AttributeError("Need cx, cy, detd and ewald_rad to be defined")
        self.cx, self.cy = cx, cy
        fac = np.sqrt(cx ** 2 + cy ** 2 + self.detd ** 2)
        q = np.empty(cx.shape + (3,))
        q[:, 0] = cx * self.ewald_rad / fac
        q[:, 1] = cy * self.ewald_rad / fac
        q[:, 2] = self.ewald_rad * (self.detd / fac - 1.)
        if pol.lower() == "x":
            corr = self.detd / fac ** 3 * (1. - cx ** 2 / fac ** 2)
        elif pol.lower() == "y":
            corr = self.detd / fac ** 3 * (1. - cy ** 2 / fac ** 2)
        else:
            corr = self.detd / fac ** 3 * (1. - (cx ** 2 + cy ** 2) / 2 / fac ** 2)
        self._qvals = None
        self._corr = None
        self.qvals = q
        self.corr = corr

    def remask(self, qradius):
        """Good pixels beyond qradius become merge-only (detector.pyx:354-364)."""
        if self._qrad is None:
            self._qrad = np.linalg.norm(self.qvals, axis=1)
        self.raw_mask[(self.raw_mask == 0) & (self._qrad > qradius)] = 1

    def _process_det(self, mask_flag, keep_mask_1):
        if mask_flag:
            if keep_mask_1:
                mask = (self.raw_mask < 2)
            else:
                mask = (self.raw_mask == 0)
        else:
            self._raw_mask = np.zeros(self.num_pix, np.uint8)
            mask = np.ones(self.num_pix, bool)
        qz = self.qvals[:, 2]
        den = (self.ewald_rad - qz) if qz.mean() > 0 else (self.ewald_rad + qz)
        self.cx = self.qvals[:, 0] * self.detd / den
        self.cy = self.qvals[:, 1] * self.detd / den
        self.x = np.round(self.cx - self.cx.min()).astype("i4")
        self.y = np.round(self.cy - self.cy.min()).astype("i4")
        self.mask = mask.ravel().astype(bool)
        self.frame_shape = (int(self.x.max()) + 1, int(self.y.max()) + 1)
        self.mask_assem = np.zeros(self.frame_shape, np.uint8)
        self.mask_assem[self.x, self.y] = self.mask
        xs, ys = self.x[self.mask], self.y[self.mask]
        self.zoom_bounds = (xs.min(), xs.max() + 1, ys.min(), ys.max() + 1)

    def assemble_frame(self, data, zoomed=False, avg=False):
        """2-D image of per-pixel values (masked outside good pixels)."""
        img = np.ma.masked_array(np.zeros(self.frame_shape), mask=1 - self.mask_assem)
        np.add.at(img.data, (self.x, self.y), data * self.mask)
        if avg:
            cnt = np.zeros(self.frame_shape)
            np.add.at(cnt, (self.x, self.y), self.mask)
            img.data[cnt > 0] /= cnt[cnt > 0]
        if zoomed:
            b = self.zoom_bounds
            return img[b[0]:b[1], b[2]:b[3]]
        return img

    @property
    def coords_xy(self):
        return self.cx, self.cy

    @property
    def indices_xy(self):
        return self.x, self.y
