"""Orientation sets (mirror of dragonfly.quaternion.Quaternion,
dragonfly/quaternion.pyx:25-342). Quaternions are rows (q0, q1, q2, q3, w)
with weights summing to one; generate_3d uses the 600-cell refinement of
quatgen.py, identical to the reference's quat_gen."""
import configparser
import os.path as op
import sys

import numpy as np

from .quatgen import quat_gen

try:
    import h5py
except ImportError:
    h5py = None


class Quaternion:
    def __init__(self, num_div=0, num_rot=0, point_group=""):
        self.octahedral_flag = point_group == "S4"
        self.icosahedral_flag = point_group == "A5"
        self.num_rot_p = 0
        self.num_div = 0
        self._quats = None
        self.reduced = False
        self.quat_mapping = None  # nearest coarse orientation (voronoi_subset)
        self.coarse_div = 0
        self.num_rot_coarse = 0
        if num_div > 0 and num_rot > 0:
            raise ValueError("Cannot specify both num_div and num_rot")
        elif num_div > 0:
            self.generate_3d(num_div)
        elif num_rot > 0:
            self.generate_2d(num_rot, point_group)

    def from_config(self, config_fname, section_name="emc"):
        config = configparser.ConfigParser()
        config.read(config_fname)
        rtype = config.get(section_name, "recon_type", fallback="3d").lower()
        if rtype == "2d":
            num_rot = config.getint(section_name, "num_rot")
            friedel = config.getboolean(section_name, "friedel_sym", fallback=False)
            self.generate_2d(num_rot, "2" if friedel else "1")
        elif rtype == "3d":
            num_div = config.get(section_name, "num_div", fallback="0").split()
            self.generate_3d(int(num_div[0]))
            if len(num_div) == 2:
                self.voronoi_subset(int(num_div[1]))
            point_group = config.get(section_name, "point_group", fallback="1")
            if point_group == "A5":
                print("Reducing to A5 sub-group")
                self.reduce_icosahedral()
                self.icosahedral_flag = True
            elif point_group == "S4":
                print("Reducing to S4 sub-group")
                self.reduce_octahedral()
                self.octahedral_flag = True
            elif point_group != "1":
                raise ValueError("Unknown point group: " + point_group)

    def generate_3d(self, num_div):
        self.num_div = int(num_div)
        self.reduced = False
        self._quats = quat_gen(num_div)

    def generate_2d(self, num_rot, point_group):
        if point_group == "":
            point_group = "1"
        max_angle = 2 * np.pi / int(point_group)
        q = np.zeros((num_rot, 5))
        q[:, 0] = np.arange(0, max_angle, max_angle / num_rot)[:num_rot]
        q[:, 4] = 1. / num_rot
        self._quats = q

    def save(self, fname):
        if self._quats is None:
            raise AttributeError("Generate quaternion first before saving")
        if h5py is None or fname.endswith(".npz"):
            np.savez(fname, quaternions=self._quats)
        else:
            with h5py.File(fname, "w") as f:
                f["quaternions"] = self._quats

    def parse(self, fname):
        if h5py is None or fname.endswith(".npz"):
            quats = np.load(fname)["quaternions"]
        else:
            with h5py.File(fname, "r") as f:
                quats = f["quaternions"][:]
        quats = np.asarray(quats, np.float64)
        if quats.shape[1] == 4:
            quats = np.pad(quats, ((0, 0), (0, 1)), constant_values=1. / quats.shape[0])
        elif quats.shape[1] == 5:
            quats = quats.copy()
            quats[:, 4] /= quats[:, 4].sum()
        else:
            raise ValueError("Need 4- or 5-dimensional quaternions")
        self._quats = np.ascontiguousarray(quats)

    def divide(self, rank, num_proc, num_modes=1, num_nonrot_modes=0):
        """Orientations handled by one rank (quaternion.pyx:156-175)."""
        tot = num_modes * self.num_rot + num_nonrot_modes
        self.num_rot_p = tot // num_proc + (1 if rank < tot % num_proc else 0)
        if num_proc > 1:
            sys.stderr.write("%d: num_rot_p = %d/%d\n" % (rank, self.num_rot_p, tot))
        return self.num_rot_p

    def voronoi_subset(self, coarse_div, ctx=None):
        """Nearest coarse (num_div = coarse_div) orientation of every fine one,
        by 1 - (q.q')^2 with ties to the first (voronoi_subset,
        quaternion.c:844-862; Quaternion.voronoi_subset, quaternion.pyx:257-281),
        computed on the GPU (dfg_voronoi_subset) of ``ctx`` or of a temporary
        context on device 0. The result is kept as ``quat_mapping`` with
        ``coarse_div`` and ``num_rot_coarse`` for refinement."""
        if self._quats is None:
            print("Generate fine quaternions first")
            return None
        from ._lib import Context
        coarse = quat_gen(coarse_div)
        own = ctx is None
        c = Context(0) if own else ctx
        try:
            out = c.voronoi_subset(coarse, self._quats)
        finally:
            if own:
                c.close()
        self.quat_mapping = out
        self.coarse_div = int(coarse_div)
        self.num_rot_coarse = coarse.shape[0]
        return out

    def reduce_icosahedral(self, return_sym=False):
        """Keep the orientations whose nearest (Euclidean, first on ties) of
        the 60 vertex quaternions of the 600-cell is vertex 8, the identity;
        it goes first, and weights are kept (quaternion.pyx:177-209)."""
        from scipy.spatial import distance
        if self._quats is None:
            raise AttributeError("Generate quaternion first before reducing")
        if self.reduced:
            print("Already reduced")
            return self.num_rot
        quats = self._quats
        sel = np.where(distance.cdist(quats[:60, :4], quats[60:, :4]).argmin(axis=0) == 8)[0]
        self._quats = np.ascontiguousarray(np.concatenate([quats[8:9], quats[60 + sel]]))
        if self.quat_mapping is not None:
            self.quat_mapping = np.concatenate([self.quat_mapping[8:9], self.quat_mapping[60 + sel]])
        self.reduced = True
        return quats[:60, :4].copy() if return_sym else self.num_rot

    @staticmethod
    def octahedral_quaternions():
        """The 24 unit quaternions of the octahedral rotation group, with the
        signs and order of quaternion.pyx:227-241 (the identity first): the
        four axes, (1, +-1, +-1, +-1) / 2, the 90-degree turns
        (1, +-e_i) / sqrt 2 and the six edge turns (0, e_i +- e_j) / sqrt 2."""
        q = np.zeros((24, 4))
        q[:4] = np.identity(4)
        v = np.sqrt(0.5)
        for k, (a, b, c) in enumerate(np.ndindex(2, 2, 2)):
            q[4 + k] = [0.5, (a * 2 - 1) * 0.5, (b * 2 - 1) * 0.5, (c * 2 - 1) * 0.5]
        for i in range(3):
            q[12 + i, 0] = q[12 + i, 1 + i] = v
            q[15 + i, 0], q[15 + i, 1 + i] = v, -v
        k = 18
        for i in range(3):
            for j in range(3):
                if i != j:
                    q[k, 1 + i], q[k, 1 + j] = v, (-v if i < j else v)
                    k += 1
        return q

    def reduce_octahedral(self, return_sym=False):
        """Keep the orientations whose nearest (Euclidean, first on ties) of
        the 24 octahedral-group quaternions is the identity; weights are
        kept (quaternion.pyx:211-255)."""
        from scipy.spatial import distance
        if self._quats is None:
            raise AttributeError("Generate quaternion first before reducing")
        if self.reduced:
            print("Already reduced")
            return self.num_rot
        cube = self.octahedral_quaternions()
        sel = np.where(distance.cdist(cube, self._quats[:, :4]).argmin(axis=0) == 0)[0]
        self._quats = np.ascontiguousarray(self._quats[sel])
        if self.quat_mapping is not None:
            self.quat_mapping = self.quat_mapping[sel]
        self.reduced = True
        return cube if return_sym else self.num_rot

    def free(self):
        self._quats = None

    @property
    def num_rot(self):
        return 0 if self._quats is None else int(self._quats.shape[0])

    @property
    def quats(self):
        return self._quats

    @quats.setter
    def quats(self, arr):
        arr = np.asarray(arr, np.float64)
        if arr.ndim != 2 or arr.shape[1] != 5:
            raise ValueError("quats must be [num_rot, 5]")
        self._quats = np.ascontiguousarray(arr).copy()
