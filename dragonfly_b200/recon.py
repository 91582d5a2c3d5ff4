"""EMC reconstruction driver (mirror of dragonfly.recon, dragonfly/recon.pyx).

EMCRecon keeps the reference's interface -- set_iterate, run_iteration,
update_model, update_beta, save_output, save_initial_model and the read-only
result properties -- but the iteration runs on one GPU through the C ABI of
libdfgpu.so (include/dragonfly_b200.h). The Iterate's host arrays stay the
source of truth between iterations: run_iteration uploads model1 and the
per-frame parameters, runs the iteration on the device and writes model1,
model2, inter_weight, scale and beta back, so code that edits them between
iterations keeps working as with the reference.

Outputs: output_%03d.h5 with the reference's keys when h5py is importable,
otherwise output_%03d.npz with the same keys; the EMC.log format is the
reference's (recon.pyx:182-228).
"""
import os
import time

import numpy as np

from .iterate import Iterate
from .params import RECON2D, RECON3D

try:
    import h5py
except ImportError:
    h5py = None


class EMCRecon:
    """Runs EMC iterations on the GPU (recon.pyx:19-415).

    Args:
        num_threads (int): accepted for interface compatibility; the GPU path
            does not use host threads.
        device (int): CUDA device (default: LOCAL_RANK or 0).
    """

    def __init__(self, num_threads=-1, device=None):
        self.num_threads = num_threads if num_threads > 0 else (os.cpu_count() or 1)
        self.device = int(os.environ.get("LOCAL_RANK", "0")) if device is None else device
        self.ctx = None
        # several detectors: one context per detector (ctx is the first, which
        # holds the model), run together as a DetectorGroup
        self.ctxs = []
        self.group = None
        self._index = []
        self._iter = None
        self.refinement = 0
        self.within_openmp = 0
        self._results = {}

    # -- setup ---------------------------------------------------------------
    def set_iterate(self, itr):
        """Uploads the detector, frames, orientations and model (recon.pyx:48-70)."""
        if itr.data is None:
            print("Set data for iterate first")
            return
        if itr.model is None:
            print("Set model for iterate first")
            return
        if itr.quat is None:
            print("Set quat for iterate first")
            return
        two_d = itr.params.rtype == RECON2D
        if not ((itr.params.rtype == RECON3D and itr.model.mtype == "MODEL_3D")
                or (two_d and itr.model.mtype == "MODEL_2D")):
            # recon.pyx:86-91 selects slice functions for 3-D and 2-D only
            raise NotImplementedError("3-D and 2-D reconstructions are supported (RZ: Model.slice_gen / "
                                      "slice_merge only)")
        if two_d and (itr.params.axial_sym > 1 or itr.quat.icosahedral_flag or itr.quat.octahedral_flag):
            raise NotImplementedError("point-group and axial symmetries apply to 3-D models")
        if itr.params.nonrot_modes:
            raise NotImplementedError("non-rotating modes are not supported")
        from ._lib import Context, DetectorGroup
        K = itr.num_det
        if K > 1 and any(d.with_bg for d in itr.dets):
            raise NotImplementedError("background-aware updates with several detectors are not supported")
        while len(self.ctxs) < K:
            self.ctxs.append(Context(self.device))
        while len(self.ctxs) > K:
            self.ctxs.pop().close()
        self.ctx = self.ctxs[0]
        self._index = [itr.member_index(k) for k in range(K)]
        if itr.params.refine and (itr.quat.quat_mapping is None or itr.rel_quat is None):
            raise ValueError("refinement needs quat.voronoi_subset() and Iterate.parse_rel_quat()")
        pg = 2 if itr.quat.icosahedral_flag else (1 if itr.quat.octahedral_flag else 0)
        for k, c in enumerate(self.ctxs):
            det = itr.dets[k]
            c.set_detector(det.qvals, det.corr, det.raw_mask)
            c.set_frames(*itr.member_frames(k))
            # background-aware updates (max_update.c:232-543, max_scale.c:21-288)
            c.set_background(det.background if det.with_bg else None)
            c.set_quaternions(itr.quat.quats)
            # 2-D: angles in quats[:, 0], images [modes, S, S], Friedel average
            # when params.friedel_sym (recon.pyx:118-119)
            c.set_model_type(1 if two_d else 0, itr.params.friedel_sym if two_d else 0)
            c.set_model(itr.model.model1)
            # refinement (max_prob.c:110-120 with src/iterate.c:103-130)
            if itr.params.refine:
                c.set_refinement(itr.quat.num_rot_coarse, itr.quat.quat_mapping,
                                 [itr.rel_quat[i] for i in self._index[k]])
                self.refinement = 1
            # update_model's symmetries (recon.pyx:120-134)
            if not two_d:
                c.set_symmetry(pg, itr.params.axial_sym if itr.params.axial_sym > 1 else 0)
        if self.group is not None:
            self.group.close()
        self.group = DetectorGroup(self.ctxs) if K > 1 else None
        itr.quat.divide(0, 1, itr.params.num_modes, itr.params.nonrot_modes)
        itr.params.rank, itr.params.num_proc = 0, 1
        self._iter = itr

    # -- one iteration ---------------------------------------------------------
    def run_iteration(self, dynamic=False):
        """update_beta, maximize, update_model, normalize_scale, output
        (recon.pyx:72-110)."""
        itr = self._iter
        if itr is None:
            print("Set iterate first")
            return
        par = itr.params
        stime = time.time()
        if par.iteration == 1:
            self.write_log_file_header()
        for c, idx in zip(self.ctxs, self._index):
            c.set_model(itr.model.model1)
            c.set_blacklist(itr.blacklist[idx])
            c.set_beta_start(itr.beta_start[idx])
            if par.need_scaling:
                c.set_scale(itr.scale[idx])
                if itr.dets[0].with_bg:
                    c.set_bgscale(itr.bgscale[idx])
            # the per-frame probability lists are formed only when they are
            # saved (combine_information_omp, max_prob.c:294-325)
            c.set_option("keep_prob", 1 if par.save_prob else 0)
        beta_mean = self.update_beta()
        p = self.ctx.params(par.iteration, par.need_scaling, par.update_scale, par.known_scale, par.beta_jump,
                            par.beta_period, par.beta_factor)
        if self.group is not None:
            likelihood = self.group.maximize(p)
        else:
            likelihood = self.ctx.maximize(p)
        self.update_model()
        # recon.pyx:102-103: volumes only
        if par.need_scaling == 1 and itr.model.mtype == "MODEL_3D":
            itr.normalize_scale()
        beta = self._gather(lambda c: c.frame_params()["beta"])
        itr.beta[itr.blacklist == 0] = beta[itr.blacklist == 0]
        for k, c in enumerate(self.ctxs):
            itr.rescale[k] = c.scalars()["rescale"]
        if self.group is not None:
            n = itr.tot_num_data
            itr.mutual_info = float(sum(c.scalars()["mutual_info"] * c.num_data for c in self.ctxs) / n)
        else:
            itr.mutual_info = self.ctx.scalars()["mutual_info"]
        itr.likelihood = likelihood
        self._results = {}
        if par.rank == 0:
            self.save_output(dynamic)
            self.update_log_file(likelihood, beta_mean, time.time() - stime)
        if par.verbosity > 0:
            print("Finished iteration", par.iteration, "(%e)" % itr.rms_change)
        return likelihood

    def update_model(self):
        """Friedel-symmetrise, divide, rms change, model1 <- model2
        (recon.pyx:112-149), on the device; results copied to the Iterate.
        When need_scaling, the scale update of maximize is copied too."""
        itr = self._iter
        c = self.ctx
        if self.group is not None:
            itr.rms_change = self.group.update_model(itr.params.alpha)
        else:
            itr.rms_change = c.update_model(itr.params.alpha)
        m1, m2, w = c.model()
        itr.model.model1 = m1
        itr.model.model2 = m2
        itr.model.inter_weight = w
        if itr.params.need_scaling:
            itr.scale = self._gather(lambda cc: cc.frame_params()["scale"])

    def _gather(self, fn, dtype=None):
        """Per-frame values of every detector's context in global frame
        order."""
        if len(self.ctxs) == 1:
            return fn(self.ctx)
        parts = [fn(c) for c in self.ctxs]
        out = np.zeros((self._iter.tot_num_data,) + parts[0].shape[1:], dtype or parts[0].dtype)
        for idx, a in zip(self._index, parts):
            out[idx] = a
        return out

    def update_beta(self):
        """Mean of beta_d = min(1, beta_start_d * factor) over good frames
        (recon.pyx:151-174); the device applies the same rule in maximize."""
        itr = self._iter
        par = itr.params
        factor = par.beta_jump ** ((par.iteration - 1) // par.beta_period)
        factor *= par.beta_factor
        print("beta factor =", factor)
        good = itr.blacklist != 1
        beta = np.minimum(itr.beta_start[good] * factor, 1.)
        return float(beta.sum() / (itr.tot_num_data - itr.num_blacklist))

    def free(self):
        if self.group is not None:
            self.group.close()
            self.group = None
        for c in self.ctxs:
            c.close()
        self.ctxs = []
        self.ctx = None

    # -- output ----------------------------------------------------------------
    def write_log_file_header(self):
        itr = self._iter
        par = itr.params
        d = os.path.dirname(par.log_fname)
        if d and not os.path.exists(d):
            os.makedirs(d)
        with open(par.log_fname, "w") as fp:
            fp.write("Cryptotomography with the EMC algorithm using MPI+OpenMP\n\n")
            fp.write("Data parameters:\n")
            fp.write("\tnum_data = %d\n\tmean_count = %f\n\n" % (itr.tot_num_data, itr.mean_count[0]))
            fp.write("System size:\n")
            fp.write("\tnum_rot = %d\n\tnum_pix = %d/%d\n\t" % (itr.quat.num_rot, (itr.dets[0].raw_mask == 0).sum(),
                                                            itr.dets[0].num_pix))
            m = itr.model
            fp.write("system_volume = %d X %ld X %ld X %ld\n\n" % (m.num_modes, m.size, m.size, m.size))
            fp.write("Reconstruction parameters:\n")
            fp.write("\tnum_threads = %d\n\tnum_proc = %d\n\talpha = %.6f\n\tbeta = %.6f\n\tneed_scaling = %s"
                     % (self.num_threads, par.num_proc, par.alpha, itr.beta_start[0],
                        "yes" if par.need_scaling == 1 else "no"))
            fp.write("\n\nIter\ttime\trms_change\tinfo_rate\tlog-likelihood\tnum_rot\tbeta\n")

    def update_log_file(self, likelihood, beta, iter_time):
        itr = self._iter
        with open(itr.params.log_fname, "a") as fp:
            fp.write("%d\t" % itr.params.iteration)
            fp.write("%4.2f\t" % iter_time)
            fp.write("%1.4e\t%f\t%.6e\t%-7d\t%f\n" % (itr.rms_change, itr.mutual_info, likelihood,
                                                     itr.quat.num_rot, beta))

    def _output_dict(self):
        itr = self._iter
        par = itr.params
        out = {}
        for k, v in vars(par).items():
            if not k.startswith("_") and not callable(v):
                out["params/" + k] = v
        out["params/mtype"] = itr.model.mtype
        out["params/num_rot"] = itr.quat.num_rot
        out["params/num_div"] = itr.quat.num_div
        out["orientations"] = self.rmax
        out["mutual_info"] = self.info
        out["likelihood"] = self.likelihood
        if itr.model.num_modes > 1:
            out["occupancies"] = self.quat_norm
        out["intens"] = itr.model.model1
        out["inter_weight"] = itr.model.inter_weight
        if par.need_scaling != 0:
            out["scale"] = itr.scale
        out["quaternions"] = itr.quat.quats
        if par.save_prob != 0:
            # vlen datasets in the reference (recon.pyx:270-279): stored here as
            # flat arrays with per-frame offsets
            off, place, prob = self._sparse()
            out["probabilities/num_rot"] = [itr.quat.num_rot]
            out["probabilities/offsets"] = off
            out["probabilities/place"] = place
            out["probabilities/prob"] = prob
        return out

    def _write(self, fname_noext, d):
        if h5py is not None:
            with h5py.File(fname_noext + ".h5", "w") as f:
                for k, v in d.items():
                    f[k] = v
        else:
            np.savez(fname_noext + ".npz", **{k.replace("/", "__"): np.asarray(v) for k, v in d.items()})

    def save_output(self, dynamic=False):
        par = self._iter.params
        if not os.path.exists(par.output_folder):
            os.makedirs(par.output_folder)
        name = "output_dynamic" if dynamic else "output_%.3d" % par.iteration
        self._write(os.path.join(par.output_folder, name), self._output_dict())

    def save_initial_model(self):
        itr = self._iter
        par = itr.params
        if not os.path.exists(par.output_folder):
            os.makedirs(par.output_folder)
        d = {"intens": itr.model.model1}
        if par.need_scaling != 0:
            d["scale"] = itr.scale
        self._write(os.path.join(par.output_folder, "output_000"), d)

    # -- results ---------------------------------------------------------------
    def _frame(self, key):
        if key not in self._results:
            if len(self.ctxs) > 1:
                parts = [c.frame_results() for c in self.ctxs]
                for k in parts[0]:
                    self._results[k] = self._gather(lambda c, k=k: parts[self.ctxs.index(c)][k])
            else:
                self._results.update(self.ctx.frame_results())
        return self._results[key]

    @property
    def iter(self):
        return self._iter

    @property
    def rmax(self):
        return self._frame("rmax")

    @property
    def info(self):
        return self._frame("info")

    @property
    def likelihood(self):
        return self._frame("likelihood")

    @property
    def max_exp(self):
        return self._frame("max_exp")

    @property
    def p_norm(self):
        return self._frame("p_norm")

    @property
    def psum_d(self):
        return self._frame("psum_d")

    @property
    def max_exp_p(self):
        return self._frame("max_exp")

    @property
    def quat_norm(self):
        return self._gather(lambda c: c.quat_norm())

    @property
    def num_prob(self):
        """Length of each frame's probability list: the pairs with P > 1e-6
        when save_prob is set, zeros otherwise (the reference forms the lists
        only to save them, max_prob.c:294-325)."""
        if self._iter is not None and self._iter.params.save_prob:
            off = self._sparse()[0]
            return np.diff(off).astype(np.int32)
        return np.zeros(self._iter.tot_num_data, np.int32)

    @property
    def u(self):
        """u_r per detector (max_prob.c:31-42)."""
        return [c.orientation_results()[0] for c in self.ctxs]

    @property
    def psum_r(self):
        """psum_r of the first detector (per detector: psum_r_det)."""
        return self.ctx.orientation_results()[1]

    @property
    def psum_r_det(self):
        return [c.orientation_results()[1] for c in self.ctxs]

    @property
    def model(self):
        return self._iter.model.model2

    @property
    def weight(self):
        return self._iter.model.inter_weight

    def _sparse(self):
        if "sparse" not in self._results:
            if len(self.ctxs) == 1:
                self._results["sparse"] = self.ctx.sparse_prob()
            else:
                # every frame's list from its detector's context, in global
                # frame order
                n = self._iter.tot_num_data
                lists = [None] * n
                for c, idx in zip(self.ctxs, self._index):
                    off, place, prob = c.sparse_prob()
                    for j, d in enumerate(idx):
                        lists[d] = (place[off[j]:off[j + 1]], prob[off[j]:off[j + 1]])
                counts = np.array([a.size for a, _ in lists], np.int64)
                off = np.zeros(n + 1, np.int64)
                np.cumsum(counts, out=off[1:])
                place = np.concatenate([a for a, _ in lists]).astype(np.int32) if n else np.zeros(0, np.int32)
                prob = np.concatenate([b for _, b in lists]) if n else np.zeros(0)
                self._results["sparse"] = (off, place, prob)
        return self._results["sparse"]

    @property
    def all_views(self):
        """Photon tomogram of every orientation (divided by psum_r where it is
        positive) as [num_rot * num_modes, num_pix]; see tomograms() for a
        range of orientations."""
        c = self.ctx
        n = c.num_rot * c.model_shape[0]
        if n * c.num_pix * 8 > (2 << 30):
            raise MemoryError("all_views of %d orientations x %d pixels exceeds 2 GiB; use tomograms(r0, n)"
                              % (n, c.num_pix))
        return c.tomograms(0, n)

    def tomograms(self, r0, n):
        return self.ctx.tomograms(r0, n)

    @property
    def prob(self):
        """Per-frame probabilities P > 1e-6 in orientation order (save_prob
        runs only, as in recon.pyx:409-411)."""
        if self._iter is None or not self._iter.params.save_prob:
            return None
        off, _, prob = self._sparse()
        return [prob[off[d]:off[d + 1]] if off[d + 1] > off[d] else None for d in range(len(off) - 1)]

    @property
    def place_prob(self):
        """Orientation indices of prob (recon.pyx:412-415)."""
        if self._iter is None or not self._iter.params.save_prob:
            return None
        off, place, _ = self._sparse()
        return [place[off[d]:off[d + 1]] for d in range(len(off) - 1)]


def main():
    """Command line: dragonfly_b200.recon niter [-c config] [-r] [-t threads]
    (recon.pyx:418-445)."""
    import argparse
    parser = argparse.ArgumentParser(description="Cryptotomography with the EMC algorithm on a B200 GPU")
    parser.add_argument("niter", help="Number of iterations", type=int)
    parser.add_argument("-c", "--config_file", help="Path to configuration file. Default: config.ini",
                        default="config.ini")
    parser.add_argument("-r", "--resume", help="Whether to resume from last iteration", action="store_true")
    parser.add_argument("-t", "--threads", help="Accepted for compatibility", type=int, default=-1)
    args = parser.parse_args()
    recon = EMCRecon(args.threads)
    itr = Iterate(args.config_file, resume=args.resume)
    itr.params.num_iter = args.niter
    recon.set_iterate(itr)
    st = itr.params.start_iter
    en = st + itr.params.num_iter
    if st == 1:
        recon.save_initial_model()
    for itr.params.iteration in range(st, en):
        recon.run_iteration()
    if itr.params.verbosity > 0:
        print("Finished all iterations")


if __name__ == "__main__":
    main()
