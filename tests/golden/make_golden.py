"""Generates the golden vectors in this directory from the reference engine.

The reference (duaneloh/Dragonfly) ships no tests, fixtures or golden vectors,
so these are produced by running its own C engine (dragonfly/src, compiled
from its sources by oracle/Makefile into oracle/_ref/libdragonfly_ref.so) with
one OpenMP thread on small seeded inputs, through EMCRecon.run_iteration's
steps (oracle/ref_driver.c, oracle/oracle.py). Needs the reference sources,
so it runs only where they are present:

    python tests/golden/make_golden.py

    python tests/golden/make_golden.py detectors2     # only the named cases

Each case file <name>.npz holds the inputs and, per iteration, the outputs:
scalars, per-frame arrays and the SHA-256 of model1's bytes (bit-exact pin),
plus the final model1. quat_gen.npz holds the reference's quat_gen lists.
detectors2.npz is a reconstruction with two detectors (each with its own
dataset; inputs of detector k under d<k>_*), run through the reference with
both detectors (ref_add_detector).
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dragonfly_b200 import synth  # noqa: E402
from oracle.oracle import EMCProblem, ReferenceEngine, quat_gen_reference  # noqa: E402

GEOM = dict(det_side=32, size=35, qmax=17., n_atoms=100, atom_radius=6., num_div=2, n_frames=300,
            mean_count=30.)

CASES = {
    # beta = 1, no scaling (the small configuration's settings)
    "beta1": dict(seed=1, geom=GEOM, prob=dict(beta=1.), iters=3),
    # scale update on, beta schedule
    "scaling": dict(seed=2, geom=GEOM, prob=dict(beta=0.05, beta_jump=1.41421356, beta_period=2,
                                                 need_scaling=1, update_scale=1), iters=3),
    # ragged sizes and edge cases: P = 480 and R = 60 (no tile multiples),
    # blacklisted and empty frames, a count above 1023, a zero shell in the
    # start model (frames whose every orientation has log-likelihood -inf)
    "edge": dict(seed=3, geom=dict(det_side=24, size=31, qmax=14., n_atoms=60, atom_radius=5., num_div=1,
                                   n_frames=200, mean_count=25.), prob=dict(beta=0.5), iters=2, edge=True),
    # two modes
    "modes2": dict(seed=4, geom=dict(det_side=24, size=31, qmax=14., n_atoms=60, atom_radius=5., num_div=2,
                                     n_frames=200, mean_count=25.), prob=dict(beta=1.), iters=2, modes=2),
}


def model_hash(m):
    return hashlib.sha256(np.ascontiguousarray(m, np.float64).tobytes()).hexdigest()


def make_inputs(spec):
    g = dict(spec["geom"])
    d = synth.small_problem(seed=spec["seed"], **g)
    if g["det_side"] == 24:  # make the detector 24 x 20
        keep = np.arange(24 * 24).reshape(24, 24)[:, :20].ravel()
        remap = -np.ones(24 * 24, np.int64)
        remap[keep] = np.arange(keep.size)
        d["qvals"], d["corr"], d["mask"] = d["qvals"][keep], d["corr"][keep], d["mask"][keep]
        # rebuild the frames on the cropped detector: drop photons off it
        po, pm, cm, ones, multi = [], [], [], [], []
        oo = np.concatenate([[0], np.cumsum(d["ones"])])
        mo = np.concatenate([[0], np.cumsum(d["multi"])])
        for i in range(d["ones"].size):
            a = remap[d["place_ones"][oo[i]:oo[i + 1]]]
            b = remap[d["place_multi"][mo[i]:mo[i + 1]]]
            c = d["count_multi"][mo[i]:mo[i + 1]]
            po.append(a[a >= 0]); pm.append(b[b >= 0]); cm.append(c[b >= 0])
            ones.append((a >= 0).sum()); multi.append((b >= 0).sum())
        d["place_ones"] = np.concatenate(po).astype(np.int32)
        d["place_multi"] = np.concatenate(pm).astype(np.int32)
        d["count_multi"] = np.concatenate(cm).astype(np.int32)
        d["ones"] = np.array(ones, np.int32)
        d["multi"] = np.array(multi, np.int32)
    model = d["model_start"]
    blacklist = None
    if spec.get("modes", 1) > 1:
        rng = np.random.default_rng(spec["seed"] + 100)
        model = np.concatenate([model, rng.random(model.shape)], axis=0)
    if spec.get("edge"):
        n = d["ones"].size
        rng = np.random.default_rng(spec["seed"] + 200)
        size = model.shape[-1]
        c = size // 2
        x = np.arange(size) - c
        rad = np.sqrt(x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2)
        model = model.copy()
        model[0][(rad > 9.) & (rad < 11.)] = 0.
        # empty frames 5 and 6: move their photons nowhere
        oo = np.concatenate([[0], np.cumsum(d["ones"])])
        mo = np.concatenate([[0], np.cumsum(d["multi"])])
        keep_o = np.ones(d["place_ones"].size, bool)
        keep_m = np.ones(d["place_multi"].size, bool)
        for f in (5, 6):
            keep_o[oo[f]:oo[f + 1]] = False
            keep_m[mo[f]:mo[f + 1]] = False
        d["place_ones"] = d["place_ones"][keep_o]
        d["place_multi"] = d["place_multi"][keep_m]
        d["count_multi"] = d["count_multi"][keep_m]
        d["ones"][[5, 6]] = 0
        d["multi"][[5, 6]] = 0
        # frame 7: one pixel with 2000 photons on a mask-0 pixel near the centre
        good = np.nonzero(d["mask"] == 0)[0]
        p = good[np.argmin(np.linalg.norm(d["qvals"][good], axis=1))]
        mo = np.concatenate([[0], np.cumsum(d["multi"])])
        d["place_multi"] = np.insert(d["place_multi"], mo[8], p).astype(np.int32)
        d["count_multi"] = np.insert(d["count_multi"], mo[8], 2000).astype(np.int32)
        d["multi"][7] += 1
        blacklist = np.zeros(n, np.uint8)
        blacklist[rng.choice(n, 10, replace=False)] = 1
    return d, model, blacklist


def run_case(name, spec):
    d, model, blacklist = make_inputs(spec)
    prob = EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"],
                      d["place_multi"], d["count_multi"], d["quats"], model, blacklist=blacklist,
                      **spec["prob"])
    eng = ReferenceEngine(prob, num_threads=1)
    out = dict(qvals=prob.qvals, corr=prob.corr, mask=prob.mask, ones=prob.ones, multi=prob.multi,
               place_ones=prob.place_ones, place_multi=prob.place_multi, count_multi=prob.count_multi,
               quats=prob.quats, model_start=prob.model1,
               blacklist=blacklist if blacklist is not None else np.zeros(prob.num_data, np.uint8),
               prob_params=np.array([prob.need_scaling, prob.update_scale, prob.known_scale, prob.alpha,
                                     prob.beta, prob.beta_jump, prob.beta_period, prob.beta_factor]),
               iters=np.array(spec["iters"]))
    it0 = eng.iter_arrays()
    out["fcounts"], out["sum_fact"], out["beta_start"] = it0["fcounts"], it0["sum_fact"], it0["beta_start"]
    for it in range(1, spec["iters"] + 1):
        r = eng.run_iteration(it)
        k = "it%d_" % it
        out[k + "scalars"] = np.array([r["avg_likelihood"], r["mutual_info"], r["rms_change"], r["rescale"]])
        for key in ("rmax", "info", "likelihood", "max_exp", "p_norm", "psum_d", "u", "beta"):
            out[k + key] = r[key]
        if prob.num_modes > 1:
            out[k + "quat_norm"] = r["quat_norm"]
        if prob.need_scaling:
            out[k + "scale"] = r["scale"]
        out[k + "model_sha256"] = np.array(model_hash(r["model1"]))
        out[k + "model2_sum_sha256"] = np.array(model_hash(r["model2_sum"]))
        out[k + "weight_sha256"] = np.array(model_hash(r["inter_weight"]))
        if it == spec["iters"]:
            out["final_model1"] = r["model1"]
    eng.close()
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path) // 1024, "KB")


def run_two_detectors(name="detectors2", seed=5, iters=3):
    """Two detectors of different geometry, scale updates on (the reference's
    in_detector_list: per-detector u, rescale, psum_r and tomograms)."""
    dets, sh = synth.two_detector_problem(seed=seed)
    kw = dict(beta=0.05, beta_jump=1.41421356, beta_period=2, need_scaling=1, update_scale=1)
    probs = [EMCProblem(d["qvals"], d["corr"], d["mask"], d["ones"], d["multi"], d["place_ones"],
                        d["place_multi"], d["count_multi"], sh["quats"], sh["model_start"], **kw) for d in dets]
    eng = ReferenceEngine(probs[0], num_threads=1)
    eng.add_detector(probs[1])
    out = dict(quats=probs[0].quats, model_start=probs[0].model1, iters=np.array(iters),
               prob_params=np.array([1, 1, 0, 0., kw["beta"], kw["beta_jump"], kw["beta_period"], 1.]))
    for k, p in enumerate(probs):
        for key in ("qvals", "corr", "mask", "ones", "multi", "place_ones", "place_multi", "count_multi"):
            out["d%d_%s" % (k, key)] = getattr(p, key)
    it0 = eng.iter_arrays()
    out["fcounts"], out["sum_fact"], out["beta_start"] = it0["fcounts"], it0["sum_fact"], it0["beta_start"]
    for it in range(1, iters + 1):
        r = eng.run_iteration(it)
        k = "it%d_" % it
        out[k + "scalars"] = np.array([r["avg_likelihood"], r["mutual_info"], r["rms_change"]])
        out[k + "rescale_det"] = r["rescale_det"]
        out[k + "mean_count_det"] = r["mean_count_det"]
        out[k + "u_det"] = r["u_det"]
        for key in ("rmax", "info", "likelihood", "max_exp", "p_norm", "psum_d", "beta", "scale"):
            out[k + key] = r[key]
        out[k + "model_sha256"] = np.array(model_hash(r["model1"]))
        out[k + "model2_sum_sha256"] = np.array(model_hash(r["model2_sum"]))
        out[k + "weight_sha256"] = np.array(model_hash(r["inter_weight"]))
        if it == iters:
            out["final_model1"] = r["model1"]
    eng.close()
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path) // 1024, "KB")


def main(names=None):
    for name, spec in CASES.items():
        if names is None or name in names:
            run_case(name, spec)
    if names is None or "detectors2" in names:
        run_two_detectors()
    if names is None or "quat_gen" in names:
        qg = {"num_div_%d" % n: quat_gen_reference(n) for n in (1, 2, 3, 4)}
        np.savez_compressed(os.path.join(HERE, "quat_gen.npz"), **qg)
        print("wrote quat_gen.npz")


if __name__ == "__main__":
    main(sys.argv[1:] or None)
