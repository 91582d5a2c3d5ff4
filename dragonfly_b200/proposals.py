"""Learned orientation proposals for the E-step (no counterpart in the
reference, whose E-step searches every orientation of every frame).

A small network (``_lib.ProposalNet``, trained and run on the GPU by the
library's own kernels) maps each frame's photon image to logits over a coarse
orientation set (``quat_gen(coarse_div)``); a frame's E-step then evaluates
only the fine orientations whose nearest coarse orientation is among its top
K (``Context.set_refinement`` with the coarse map of ``voronoi_subset``; with
the fine orientations sorted by coarse cell, the skipped orientations form
whole tiles that every phase of the iteration skips). Each iteration a
held-out share of the frames is searched in full and watched: the probability
mass its proposals would have captured (``Context.watch_mass``) measures the
network, and when it falls below ``threshold`` the next iteration is a full
search and the network is trained again, on frames simulated from the
current model at known orientations and on the last full search's most likely
orientations.
"""
import numpy as np

from .quatgen import quat_gen


def cell_targets(offsets, place, prob, qmap, num_cells, min_share=1e-3):
    """Soft targets per frame from a full search's sparse probabilities
    (frame d's pairs [offsets[d], offsets[d + 1]) with orientation indices
    place and probabilities prob): the probability summed per coarse cell
    (qmap[orientation]), cells below min_share of their frame's total dropped,
    the rest renormalised. Returns (t_off [N + 1], cells, weights), cells
    ascending within a frame."""
    off = np.asarray(offsets, np.int64)
    N = off.size - 1
    frame = np.repeat(np.arange(N, dtype=np.int64), np.diff(off))
    key = frame * num_cells + np.asarray(qmap)[np.asarray(place, np.int64)]
    uk, inv = np.unique(key, return_inverse=True)
    mass = np.bincount(inv, weights=np.asarray(prob, np.float64))
    f, c = uk // num_cells, uk % num_cells
    tot = np.bincount(f, weights=mass, minlength=N)
    keep = mass >= min_share * tot[f]
    f, c, mass = f[keep], c[keep], mass[keep]
    tot = np.bincount(f, weights=mass, minlength=N)
    t_off = np.zeros(N + 1, np.int64)
    np.cumsum(np.bincount(f, minlength=N), out=t_off[1:])
    return t_off, c.astype(np.int32), (mass / tot[f]).astype(np.float32)


def restriction_lists(top, watch, num_cells):
    """Per-frame coarse-cell lists of a proposal iteration as (offsets, flat):
    frame d's top-K cells (top [N, K]), every cell for the watched frames."""
    top = np.asarray(top, np.int32)
    N, K = top.shape
    watch = np.asarray(watch, np.int64)
    lens = np.full(N, K, np.int64)
    lens[watch] = num_cells
    off = np.zeros(N + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    flat = np.empty(int(off[-1]), np.int32)
    keep = np.ones(N, bool)
    keep[watch] = False
    flat[(off[:-1][keep][:, None] + np.arange(K)).ravel()] = top[keep].ravel()
    flat[(off[:-1][watch][:, None] + np.arange(num_cells)).ravel()] = np.tile(np.arange(num_cells, dtype=np.int32),
                                                                            watch.size)
    return off, flat


def sort_by_coarse(fine, coarse_div, ctx):
    """Fine orientations [R, 5] ordered by their nearest coarse orientation
    (stable), so that a coarse cell's orientations are contiguous. Returns
    (sorted quaternions, order, coarse map of the sorted list)."""
    coarse = quat_gen(coarse_div)
    qmap = ctx.voronoi_subset(coarse, fine)
    order = np.lexsort((np.arange(fine.shape[0]), qmap))
    return np.ascontiguousarray(fine[order]), order, np.ascontiguousarray(qmap[order])


class LearnedProposals:
    """Drives proposal-restricted iterations of one reconstruction context.

    Args:
        ctx: the reconstruction's ``_lib.Context`` (detector, frames and the
            fine orientations already set; one model mode).
        qvals: the detector's q vectors (image binning).
        fine: the context's orientation list [R, 5] (ideally from
            ``sort_by_coarse``).
        coarse_div: num_div of the coarse orientation set (the classes).
        K: coarse cells kept per frame (the least, with mass).
        K_max, mass: mass-covering proposals: after its K best cells a frame
            keeps further cells, by decreasing network probability, until
            the network's probabilities of its cells sum to mass, at most
            K_max (None: exactly K cells per frame).
        held_out: share of frames searched in full and watched each iteration.
        threshold: mean captured probability mass below which the next
            iteration searches in full and the network is retrained.
        zoom: the image grid covers q within zoom times the detector's
            largest |qx|, |qy| (most photons and the speckle detail are at
            low q; 0.3 triples the top-16 accuracy of the whole-detector grid
            at the production detector).
        pair_lists: run proposal iterations over pair lists (option
            pair_lists: only the live (tile, frame) pairs are stored and the
            orientations are processed in blocks, so that neither all
            log-slices nor all tomograms need to be resident).
    """

    def __init__(self, ctx, qvals, fine, coarse_div=4, K=16, held_out=0.01, threshold=0.99, batch=256, seed=0,
                 pair_lists=False, zoom=0.3, retrain_epochs=3, retrain_lr=1e-3, K_max=None, mass=None):
        from ._lib import Context, ProposalNet
        self.ctx = ctx
        ctx.set_option("pair_lists", 1 if pair_lists else 0)
        self.coarse = quat_gen(coarse_div)
        self.nc = self.coarse.shape[0]
        self.K = int(K)
        self.K_max = int(K_max) if K_max is not None else self.K
        self.mass = None if mass is None else float(mass)
        self.held_out = float(held_out)
        self.threshold = float(threshold)
        self.qmap = np.ascontiguousarray(ctx.voronoi_subset(self.coarse, fine), np.int32)
        self.net = ProposalNet(self.nc, batch=batch, seed=seed, device=ctx.device)
        q = np.asarray(qvals, np.float64).reshape(-1, 3)
        self.net.set_bins(ProposalNet.pixel_bins(q, qmax=float(zoom) * float(np.abs(q[:, :2]).max())))
        self.sim = Context(ctx.device)          # frames simulated for training
        self.sim.set_detector(qvals, ctx._corr, ctx._mask)
        self.rng = np.random.default_rng(seed)
        self.full_next = False
        self.retrain_epochs = int(retrain_epochs)
        self.retrain_lr = float(retrain_lr)
        self.history = []

    def train_simulated(self, model, n_frames=20000, epochs=3, lr=5e-4, phi=None, rounds=1, lr_end=None):
        """Trains on frames simulated from model at uniformly random
        orientations (label: their nearest coarse orientation): `rounds`
        rounds of `epochs` epochs, each round on n_frames newly simulated
        frames, the learning rate going geometrically from lr to lr_end
        (default lr) over the rounds. phi: per-frame fluence factors (default
        ones; one is drawn per frame from them when their count differs).
        Returns the last round's mean loss. A large class count wants a small
        rate (3240 classes stay at chance for epochs at 2e-3)."""
        from . import synth
        lr_end = lr if lr_end is None else lr_end
        loss = None
        for k in range(int(rounds)):
            q = synth.random_quaternions(int(n_frames), self.rng)
            if phi is None:
                f = np.ones(len(q))
            else:
                f = np.asarray(phi, np.float64)
                if f.size != len(q):
                    f = self.rng.choice(f, len(q))
            self.sim.simulate_frames(model, q, f, int(self.rng.integers(1 << 30)))
            labels = self.sim.voronoi_subset(self.coarse, np.pad(q[:, :4], ((0, 0), (0, 1))))
            self.net.load_frames(self.sim)
            rate = lr * (lr_end / lr) ** (k / max(1, int(rounds) - 1))
            loss = self.net.train(labels, epochs=epochs, lr=rate, seed=int(self.rng.integers(1 << 30)))
        return loss

    def train_full_search(self, rmax, epochs=1, lr=1e-3):
        """Trains on the context's own frames labelled by the coarse cell of a
        full search's most likely orientation (frames with none are left out)."""
        ok = np.asarray(rmax) >= 0
        if not ok.any():
            return None
        self.net.load_frames(self.ctx)
        labels = np.where(ok, self.qmap[np.maximum(rmax, 0)], 0).astype(np.int32)
        return self.net.train(labels, epochs=epochs, lr=lr, seed=int(self.rng.integers(1 << 30)))

    def train_full_search_probs(self, offsets, place, prob, epochs=3, lr=1e-3, min_share=1e-3):
        """Trains on the context's own frames against a full search's
        probabilities summed per coarse cell (the per-frame lists of pairs
        with P > 1e-6: offsets [N + 1], orientation indices, P), keeping the
        cells with at least min_share of their frame's mass, renormalised."""
        if np.asarray(offsets)[-1] == 0:
            return None
        t_off, cells, w = cell_targets(offsets, place, prob, self.qmap, self.nc, min_share)
        self.net.load_frames(self.ctx)
        self.net.set_targets(t_off, cells, w)
        return self.net.train(None, epochs=epochs, lr=lr, seed=int(self.rng.integers(1 << 30)))

    def propose(self):
        """Proposed coarse cells of every frame of the context: [N, K] (or
        [N, K_max] with -1 in unused slots for mass-covering proposals)."""
        self.net.load_frames(self.ctx)
        if self.mass is None:
            return self.net.topk(self.K)
        return self.net.topk_mass(self.K, self.K_max, self.mass)

    def iteration(self, par, alpha=0.):
        """One iteration: proposal-restricted (held-out frames in full and
        watched), or a full search when the last captured mass was too low. Returns
        the iteration's results with 'mode', 'captured_mass' and
        'evaluated_fraction'."""
        import time
        ctx = self.ctx
        if self.full_next:
            # the full search keeps its probabilities, and the network learns
            # their distribution over the coarse cells
            ctx.set_refinement(None)
            ctx.set_option("keep_prob", 1)
            t0 = time.perf_counter()
            out = dict(ctx.run_iteration(par, alpha))
            t1 = time.perf_counter()
            off, place, prob = ctx.sparse_prob()
            ctx.set_option("keep_prob", 0)
            self.train_full_search_probs(off, place, prob, epochs=self.retrain_epochs, lr=self.retrain_lr)
            info = dict(mode="full", captured_mass=None, evaluated_fraction=1., iterate_s=t1 - t0,
                        retrain_s=time.perf_counter() - t1)
            self.full_next = False
            out.update(info)
            self.history.append(info)
            return out
        return self.proposal_iteration(par, alpha)

    def proposal_iteration(self, par, alpha=0.):
        """A proposal-restricted iteration: every frame limited to its top-K
        cells, a held-out share searched in full and watched; sets full_next
        when their mean captured mass is below the threshold. Returns the
        iteration's results with 'mode', 'captured_mass', 'min_mass',
        'evaluated_fraction' and the wall-clock seconds of its parts
        ('propose_s': images and top-K, 'lists_s': the restriction lists,
        'iterate_s': the iteration)."""
        import time
        ctx = self.ctx
        N = ctx.num_data
        t0 = time.perf_counter()
        top = self.propose()
        t1 = time.perf_counter()
        n_watch = max(1, int(round(self.held_out * N)))
        watch = np.sort(self.rng.choice(N, n_watch, replace=False)).astype(np.int32)
        ctx.set_refinement_topk(self.nc, self.qmap, top, watch)
        ctx.set_watch(watch, [row[row >= 0] for row in top[watch]])
        t2 = time.perf_counter()
        out = dict(ctx.run_iteration(par, alpha))
        t3 = time.perf_counter()
        mass = ctx.watch_mass()
        per_frame = (top >= 0).sum(1)
        per_frame[watch] = self.nc
        frac = float(per_frame.sum()) / float(self.nc * N)
        info = dict(mode="proposal", captured_mass=float(mass.mean()), min_mass=float(mass.min()),
                    evaluated_fraction=frac, propose_s=t1 - t0, lists_s=t2 - t1, iterate_s=t3 - t2)
        self.full_next = bool(mass.mean() < self.threshold)
        out.update(info)
        self.history.append(info)
        return out

    def close(self):
        self.net.close()
        self.sim.close()
