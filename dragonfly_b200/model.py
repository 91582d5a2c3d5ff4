"""Intensity model (mirror of dragonfly.model.Model, dragonfly/model.pyx:18-313).

model1 is the current intensity [num_modes, size, size, size] (MODEL_3D) or
[num_modes, size, size] (MODEL_2D, MODEL_RZ) (float64, C order, centre
size // 2); model2 / inter_weight hold the last iteration's merged model and
interpolation weights. slice_gen / slice_merge run on the GPU through the C
ABI (dfg_slice_gen / dfg_slice_merge); the orientation is a quaternion (3-D),
an angle (2-D) or (phi, beta) (RZ, which uses the detector's detd). The
volume operations rotate_model and symmetrize_octahedral / icosahedral /
axial run on the GPU too (dfg_model_rotate, dfg_model_symmetrize).
"""
import os

import numpy as np

try:
    import h5py
except ImportError:
    h5py = None

_MODEL_TYPES = {"3d": "MODEL_3D", "2d": "MODEL_2D", "rz": "MODEL_RZ"}
_slice_ctx = None


_TYPE_CODES = {"MODEL_3D": 0, "MODEL_2D": 1, "MODEL_RZ": 2}


def _slice_context(det, model):
    """A shared GPU context holding det and this Model's model1, for
    one-slice calls."""
    c = _device_context()
    key = (id(det.qvals), id(det.corr), id(det.raw_mask))
    if c._det_id != key:
        c.set_detector(det.qvals, det.corr, det.raw_mask)
        c._det_id = key
    c.set_model_type(_TYPE_CODES[model.mtype])
    c.set_detector_distance(getattr(det, "detd", 0.))
    c.set_model(model.model1)
    return c


def _device_context():
    """The shared GPU context of the one-slice calls, for the volume
    operations that need no detector (rotation, symmetrisation)."""
    global _slice_ctx
    from ._lib import Context
    if _slice_ctx is None:
        _slice_ctx = Context(int(os.environ.get("LOCAL_RANK", "0")))
        _slice_ctx._det_id = None
    return _slice_ctx


class Model:
    def __init__(self, size=0, num_modes=1, model_type="3d"):
        if model_type.lower() not in _MODEL_TYPES:
            raise ValueError("Unknown model_type %s" % model_type)
        self.mtype = _MODEL_TYPES[model_type.lower()]
        self._size = 0
        self.center = 0
        self.num_modes = num_modes
        self.model1 = self.model2 = self.inter_weight = None
        if size > 0:
            self.size = size

    @property
    def ndim(self):
        return 3 if self.mtype == "MODEL_3D" else 2

    @property
    def size(self):
        return self._size

    @size.setter
    def size(self, val):
        self._size = int(val)
        self.center = self._size // 2

    @property
    def vol(self):
        return self._size ** self.ndim

    @property
    def shape(self):
        return (self.num_modes,) + (self._size,) * self.ndim

    def allocate(self, fname, model_mean=1., rank=0, fixed_seed=False):
        """model1 from a file (HDF5 'intens', .npy, or raw float64), or uniform
        random times model_mean (model.pyx:43-103); fixed_seed seeds numpy's
        global generator with 0x5EED as the reference does."""
        shape = self.shape
        self.model2 = np.zeros(shape)
        self.inter_weight = np.zeros(shape)
        if fname and os.path.isfile(fname):
            if fname.endswith(".npy"):
                m = np.load(fname)
            elif h5py is not None and h5py.is_hdf5(fname):
                with h5py.File(fname, "r") as f:
                    m = f["intens"][:]
            elif fname.endswith(".npz"):
                m = np.load(fname)["intens"]
            else:
                m = np.fromfile(fname, np.float64)
                n = int(np.rint((m.size) ** (1. / 3)))
                if n != self._size:
                    raise ValueError("Wrong volume size in binary file (%d)" % n, n)
            m = np.asarray(m, np.float64)
            if m.shape[1:] != shape[1:] and m.shape != shape[1:]:
                raise ValueError("Input model has wrong size")
            m = m.reshape((-1,) + shape[1:])
            out = np.empty(shape)
            k = min(m.shape[0], shape[0])
            out[:k] = m[:k]
            if k < shape[0]:
                out[k:] = np.random.random((shape[0] - k,) + shape[1:]) * model_mean
            self.model1 = out
        else:
            if fixed_seed:
                np.random.seed(0x5EED)
            self.model1 = np.random.random(shape) * model_mean

    def slice_gen(self, quat, det, mode=0, view=None):
        """Slice of model1 at quat on det (slice_gen3d / slice_gen2d /
        slice_genrz, model.c:11-150), on the GPU."""
        if self.model1 is None:
            raise AttributeError("Allocate model1 first")
        out = _slice_context(det, self).slice_gen(quat, mode)
        if view is not None:
            view[...] = out
            return view
        return out

    def slice_merge(self, quat, view, det, mode=0):
        """Merges view into model2 / inter_weight (slice_merge3d / 2d / rz,
        model.c:171-340), on the GPU."""
        if self.model2 is None:
            raise AttributeError("Allocate model2 first")
        _slice_context(det, self).slice_merge(quat, view, self.model2, self.inter_weight, mode)

    def free(self):
        self.model1 = self.model2 = self.inter_weight = None

    @staticmethod
    def make_rot_quat(quaternion):
        """Rotation matrix of a quaternion (model.c:759-786)."""
        q0, q1, q2, q3 = (float(x) for x in quaternion[:4])
        return np.array([
            [1. - 2. * (q2 * q2 + q3 * q3), 2. * (q1 * q2 + q0 * q3), 2. * (q1 * q3 - q0 * q2)],
            [2. * (q1 * q2 - q0 * q3), 1. - 2. * (q1 * q1 + q3 * q3), 2. * (q0 * q1 + q2 * q3)],
            [2. * (q0 * q2 + q1 * q3), 2. * (q2 * q3 - q0 * q1), 1. - 2. * (q1 * q1 + q2 * q2)]])

    @staticmethod
    def symmetrize_friedel(model, weights):
        """In-place Friedel average of model with weights (model.c:470-490):
        I(q), I(-q) <- (I(q) w(q) + I(-q) w(-q)) / (w(q) + w(-q)), visiting
        z <= centre like the reference (pairs inside the z = centre plane are
        averaged twice)."""
        size = model.shape[0]
        c = size // 2
        lo = 1 if size % 2 == 0 else 0

        def avg(a1, w1, a2, w2):
            a = 0.5 * (a1 * w1 + a2 * w2)
            ws = 0.5 * (w1 + w2)
            with np.errstate(invalid="ignore", divide="ignore"):
                return np.where(ws > 0, a / np.where(ws > 0, ws, 1.), 0.)

        r = np.arange(lo, size)
        x, y, z = np.meshgrid(r, r, np.arange(lo, c), indexing="ij")
        m, w = model, weights
        a = avg(m[x, y, z], w[x, y, z], m[2 * c - x, 2 * c - y, 2 * c - z], w[2 * c - x, 2 * c - y, 2 * c - z])
        m[x, y, z] = a
        m[2 * c - x, 2 * c - y, 2 * c - z] = a
        x, y = np.meshgrid(r, r, indexing="ij")
        x, y = x.ravel(), y.ravel()
        first = (x < 2 * c - x) | ((x == 2 * c - x) & (y <= 2 * c - y))
        x, y = x[first], y[first]
        xm, ym = 2 * c - x, 2 * c - y
        w1, w2 = w[x, y, c], w[xm, ym, c]
        a = avg(m[x, y, c], w1, m[xm, ym, c], w2)
        same = (x == xm) & (y == ym)
        a = np.where(same, a, avg(a, w2, a, w1))
        m[x, y, c] = a
        m[xm, ym, c] = a

    @staticmethod
    def symmetrize_friedel2d(model, weights):
        """In-place Friedel average of every layer of a [layers, S, S] stack
        (model.c:495-515), visiting z <= centre like the reference (pairs on
        the z = centre line are averaged twice)."""
        size = model.shape[-1]
        c = size // 2
        lo = 1 if size % 2 == 0 else 0

        def avg(a1, w1, a2, w2):
            a = 0.5 * (a1 * w1 + a2 * w2)
            ws = 0.5 * (w1 + w2)
            with np.errstate(invalid="ignore", divide="ignore"):
                return np.where(ws > 0, a / np.where(ws > 0, ws, 1.), 0.)

        r = np.arange(lo, size)
        for m, w in zip(model.reshape(-1, size, size), weights.reshape(-1, size, size)):
            y, z = np.meshgrid(r, np.arange(lo, c), indexing="ij")
            a = avg(m[y, z], w[y, z], m[2 * c - y, 2 * c - z], w[2 * c - y, 2 * c - z])
            m[y, z] = a
            m[2 * c - y, 2 * c - z] = a
            y = r[r <= 2 * c - r]
            ym = 2 * c - y
            w1, w2 = w[y, c], w[ym, c]
            a = avg(m[y, c], w1, m[ym, c], w2)
            a = np.where(y == ym, a, avg(a, w2, a, w1))
            m[y, c] = a
            m[ym, c] = a

    @staticmethod
    def symmetrize_octahedral(model, weights):
        """In-place octahedral (S4, 48 rotations) symmetrisation of a volume
        and its weights on the GPU (model.pyx:175-184 -> model.c:695-729)."""
        _device_context().model_symmetrize("S4", model, weights)

    @staticmethod
    def symmetrize_icosahedral(model, weights):
        """In-place icosahedral (A5, 60 rotations) symmetrisation on the GPU
        (model.pyx:186-195 -> model.c:731-757)."""
        _device_context().model_symmetrize("A5", model, weights)

    @staticmethod
    def symmetrize_axial(model, weights, order):
        """In-place order-fold symmetrisation about z on the GPU
        (model.pyx:197-207 -> model.c:527-571)."""
        _device_context().model_symmetrize("axial", model, weights, order=int(order))

    @staticmethod
    def rotate_model(model, rot, max_r=0, rotmodel=None):
        """Rotated copy of a volume on the GPU (model.pyx:226-254 ->
        model.c:381-425): rotmodel (zeros when None) += model interpolated at
        rot v + c for v in [-max_r, max_r)^3 (max_r 0: size // 2)."""
        return _device_context().model_rotate(model, rot, max_r, rotmodel)
