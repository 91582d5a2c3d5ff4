"""Seeded synthetic inputs for the EMC iteration.

The reference ships a simulator (dragonfly/utils/make_data.pyx and
utils/src/make_data.c, make_densities.py, make_intensities.py,
make_detector.py); this module is our own, smaller generator of the same kind
of inputs, used by the tests and the benchmark:

* a density of Gaussian atoms placed uniformly in a sphere and its diffraction
  intensity |F(q)|^2 on a model grid centred at size // 2;
* a flat pixel detector whose pixel q-vectors lie on the Ewald sphere, with
  solid-angle and polarisation corrections (the formulas of
  Detector.calc_from_coords, dragonfly/detector.pyx:317-352) and the reference's
  mask semantics (0 good, 1 merge-only, 2 bad);
* frames at uniformly random orientations, Poisson-sampled, stored sparse as
  ones / multi / place_ones / place_multi / count_multi (the .emc layout,
  dragonfly/src/emcfile.c:15-37).

No public dataset is involved: the reference benchmarks on none.
"""
import numpy as np

from .quatgen import quat_gen


# ---------------------------------------------------------------------------
# model
# ---------------------------------------------------------------------------

def atom_positions(n_atoms, radius, rng):
    """Uniform points in a ball of the given radius (voxels), centred at 0."""
    out = np.empty((0, 3))
    while out.shape[0] < n_atoms:
        p = rng.uniform(-radius, radius, size=(2 * n_atoms, 3))
        p = p[(p ** 2).sum(1) <= radius ** 2]
        out = np.concatenate([out, p])
    return out[:n_atoms]


def gaussian_atom_intensity(n_atoms, radius, size, rng, sigma=1.0):
    """|F|^2 of n_atoms Gaussian atoms (width sigma voxels) in a ball, sampled
    on a size^3 grid with q = 0 at index size // 2 (C order, float64)."""
    pos = atom_positions(n_atoms, radius, rng)
    rho = np.zeros((size, size, size))
    idx = np.rint(pos).astype(np.int64) % size
    np.add.at(rho, (idx[:, 0], idx[:, 1], idx[:, 2]), 1.0)
    f = np.fft.fftn(rho)
    k = np.fft.fftfreq(size)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    f *= np.exp(-2. * np.pi ** 2 * sigma ** 2 * k2)
    return np.fft.fftshift(np.abs(f) ** 2)


# ---------------------------------------------------------------------------
# detector
# ---------------------------------------------------------------------------

def flat_detector(nx, ny, qmax, size, hole_radius=0., gap_rows=None, detd=None, pol='x'):
    """Flat detector of nx x ny pixels.

    Returns (qvals [P,3], corr [P] normalised to mean 1, mask [P] u1, detd,
    ewald_rad). The Ewald radius is chosen so that the largest |q| equals qmax
    (voxels). Mask: 2 inside hole_radius pixels of the centre and on gap_rows;
    1 where |q| > size // 2 - 2 (merge-only, keeps every mask-0 pixel inside the
    model); 0 elsewhere.
    """
    cx, cy = np.meshgrid(np.arange(nx) - (nx - 1) / 2., np.arange(ny) - (ny - 1) / 2., indexing='ij')
    cx = cx.ravel()
    cy = cy.ravel()
    if detd is None:
        detd = float(max(nx, ny))
    fac = np.sqrt(cx ** 2 + cy ** 2 + detd ** 2)
    # |q| = E * sqrt(2 - 2 detd / fac); choose E so the maximum is qmax
    ewald_rad = qmax / np.sqrt(2. - 2. * detd / fac.max())
    qvals = np.empty((cx.size, 3))
    qvals[:, 0] = cx * ewald_rad / fac
    qvals[:, 1] = cy * ewald_rad / fac
    qvals[:, 2] = ewald_rad * (detd / fac - 1.)
    if pol == 'x':
        corr = detd / fac ** 3 * (1. - cx ** 2 / fac ** 2)
    elif pol == 'y':
        corr = detd / fac ** 3 * (1. - cy ** 2 / fac ** 2)
    else:
        corr = detd / fac ** 3 * (1. - (cx ** 2 + cy ** 2) / 2 / fac ** 2)
    corr = corr / corr.mean()
    qrad = np.linalg.norm(qvals, axis=1)
    mask = np.zeros(cx.size, dtype=np.uint8)
    mask[qrad > size // 2 - 2] = 1
    mask[np.sqrt(cx ** 2 + cy ** 2) < hole_radius] = 2
    if gap_rows is not None:
        row = np.repeat(np.arange(nx), ny)
        mask[np.isin(row, gap_rows)] = 2
    return qvals, corr, mask, detd, ewald_rad


# ---------------------------------------------------------------------------
# orientations and slices
# ---------------------------------------------------------------------------

def random_quaternions(n, rng):
    """Uniform random unit quaternions by rejection in the 4-ball
    (the method of dragonfly/utils/src/make_data.c:24-40)."""
    out = np.empty((0, 4))
    while out.shape[0] < n:
        q = rng.uniform(-1., 1., size=(2 * n + 8, 4))
        r2 = (q ** 2).sum(1)
        q = q[(r2 <= 1.) & (r2 > 1e-12)]
        out = np.concatenate([out, q / np.linalg.norm(q, axis=1, keepdims=True)])
    return out[:n]


def rotation_matrices(q):
    """Rotation matrices of quaternions q[..., 4] (formula of model.c:759-786)."""
    q0, q1, q2, q3 = q[..., 0], q[..., 1], q[..., 2], q[..., 3]
    rot = np.empty(q.shape[:-1] + (3, 3))
    rot[..., 0, 0] = 1. - 2. * (q2 * q2 + q3 * q3)
    rot[..., 0, 1] = 2. * (q1 * q2 + q0 * q3)
    rot[..., 0, 2] = 2. * (q1 * q3 - q0 * q2)
    rot[..., 1, 0] = 2. * (q1 * q2 - q0 * q3)
    rot[..., 1, 1] = 1. - 2. * (q1 * q1 + q3 * q3)
    rot[..., 1, 2] = 2. * (q0 * q1 + q2 * q3)
    rot[..., 2, 0] = 2. * (q0 * q2 + q1 * q3)
    rot[..., 2, 1] = 2. * (q2 * q3 - q0 * q1)
    rot[..., 2, 2] = 1. - 2. * (q1 * q1 + q2 * q2)
    return rot


def slices(model, quats, qvals, corr):
    """Trilinear slices W[n, P] of a 3-D model at quaternions[n, >=4], times
    corr; zero outside the model (vectorised; used only to simulate data)."""
    size = model.shape[0]
    rot = rotation_matrices(quats)
    pos = np.einsum('nij,pj->npi', rot, qvals) + size // 2
    i0 = np.floor(pos).astype(np.int64)
    f = pos - i0
    ok = np.all((i0 >= 0) & (i0 <= size - 2), axis=-1)
    i0 = np.where(ok[..., None], i0, 0)
    out = np.zeros(pos.shape[:2])
    for dx in (0, 1):
        wx = f[..., 0] if dx else 1. - f[..., 0]
        for dy in (0, 1):
            wy = f[..., 1] if dy else 1. - f[..., 1]
            for dz in (0, 1):
                wz = f[..., 2] if dz else 1. - f[..., 2]
                out += wx * wy * wz * model[i0[..., 0] + dx, i0[..., 1] + dy, i0[..., 2] + dz]
    return np.where(ok, out, 0.) * corr[None, :]


# ---------------------------------------------------------------------------
# frames
# ---------------------------------------------------------------------------

def model_mean_count(model, qvals, corr, mask, rng, n_orient=256):
    """Mean photons per frame over mask <= 1 pixels for random orientations
    (the quantity make_data.c:42-113 rescales to)."""
    q = random_quaternions(n_orient, rng)
    w = slices(model, q, qvals, corr)
    return w[:, mask <= 1].sum(1).mean()


def slices2d(model, angles, qvals, corr):
    """Bilinear slices W[n, P] of a 2-D image at in-plane angles: pixel
    (qx, qy) rotated by [[c, -s], [s, c]] plus the centre, times corr; zero
    outside the image (vectorised; used only to simulate data)."""
    size = model.shape[0]
    c, s = np.cos(angles)[:, None], np.sin(angles)[:, None]
    px = c * qvals[None, :, 0] - s * qvals[None, :, 1] + size // 2
    py = s * qvals[None, :, 0] + c * qvals[None, :, 1] + size // 2
    x0, y0 = np.floor(px).astype(np.int64), np.floor(py).astype(np.int64)
    fx, fy = px - x0, py - y0
    ok = (x0 >= 0) & (x0 <= size - 2) & (y0 >= 0) & (y0 <= size - 2)
    x0, y0 = np.where(ok, x0, 0), np.where(ok, y0, 0)
    out = ((1 - fx) * (1 - fy) * model[x0, y0] + (1 - fx) * fy * model[x0, y0 + 1]
           + fx * (1 - fy) * model[x0 + 1, y0] + fx * fy * model[x0 + 1, y0 + 1])
    return np.where(ok, out, 0.) * corr[None, :]


def sample_frames(model, qvals, corr, mask, n_frames, rng, phi=None, chunk=256, two_d=False):
    """Poisson frames at random orientations (quaternions, or angles in
    [0, 2 pi) for a 2-D image), in the sparse .emc layout.

    Returns dict(ones, multi, place_ones, place_multi, count_multi, quats, phi).
    Pixels with mask == 2 never receive photons."""
    good = mask <= 1
    if two_d:
        quats = rng.random(n_frames) * 2. * np.pi
    else:
        quats = random_quaternions(n_frames, rng)
    if phi is None:
        phi = np.ones(n_frames)
    ones = np.zeros(n_frames, np.int32)
    multi = np.zeros(n_frames, np.int32)
    po, pm, cm = [], [], []
    for s in range(0, n_frames, chunk):
        e = min(n_frames, s + chunk)
        sl = slices2d if two_d else slices
        lam = sl(model, quats[s:e], qvals, corr) * phi[s:e, None]
        lam[:, ~good] = 0.
        counts = rng.poisson(np.maximum(lam, 0.))
        for i in range(e - s):
            c = counts[i]
            p1 = np.nonzero(c == 1)[0]
            pmu = np.nonzero(c > 1)[0]
            ones[s + i] = p1.size
            multi[s + i] = pmu.size
            po.append(p1.astype(np.int32))
            pm.append(pmu.astype(np.int32))
            cm.append(c[pmu].astype(np.int32))
    cat = lambda xs: np.concatenate(xs).astype(np.int32) if xs else np.zeros(0, np.int32)
    return dict(ones=ones, multi=multi, place_ones=cat(po), place_multi=cat(pm),
                count_multi=cat(cm), quats=quats, phi=phi)


# ---------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------

def small_problem(seed=0, det_side=64, size=75, qmax=37., n_atoms=300, atom_radius=12.,
                  num_div=4, n_frames=3000, mean_count=50., hole_radius=4.):
    """Plain-EMC small configuration (defaults: 64x64 detector, 75^3 model,
    num_div 4 = 3240 equal-weight orientations, 3000 frames at 50 photons).

    Returns a dict of reference-layout arrays plus 'model_start' (uniform [0,1)
    from the seed) and 'model_true'."""
    rng = np.random.default_rng(seed)
    intens = gaussian_atom_intensity(n_atoms, atom_radius, size, rng)
    qvals, corr, mask, detd, ewald = flat_detector(det_side, det_side, qmax, size, hole_radius)
    intens *= mean_count / model_mean_count(intens, qvals, corr, mask, rng)
    fr = sample_frames(intens, qvals, corr, mask, n_frames, rng)
    quats = quat_gen(num_div)
    quats[:, 4] = 1. / quats.shape[0]
    model_start = rng.random((1, size, size, size))
    return dict(qvals=qvals, corr=corr, mask=mask, detd=detd, ewald_rad=ewald, quats=quats,
                model_start=model_start, model_true=intens, **{k: fr[k] for k in
                ('ones', 'multi', 'place_ones', 'place_multi', 'count_multi')},
                frame_quats=fr['quats'])


def two_detector_problem(seed=0, size=33, qmax=15., n_atoms=80, atom_radius=6., num_div=2,
                         n_frames=(160, 120), mean_count=(40., 25.), phi_sigma=0.):
    """One model seen by two detectors of different geometry (Iterate with an
    in_detector_list): a 28 x 28 flat detector with a radius-3 hole and a
    20 x 24 detector farther out (detd 40) with a radius-2 hole, x and y
    polarised, each with its own frames (n_frames, mean_count per detector;
    lognormal per-frame fluence when phi_sigma > 0).

    Returns (dets, shared): dets a list of two dicts (qvals, corr, mask and
    the sparse frames, frame_quats, phi), shared a dict of quats (num_div,
    equal weights), model_start (uniform [0, 1) from the seed) and
    model_true."""
    rng = np.random.default_rng(seed)
    intens = gaussian_atom_intensity(n_atoms, atom_radius, size, rng)
    geo = [flat_detector(28, 28, qmax, size, hole_radius=3.),
           flat_detector(20, 24, qmax * 0.8, size, hole_radius=2., detd=40., pol='y')]
    scale0 = mean_count[0] / model_mean_count(intens, geo[0][0], geo[0][1], geo[0][2], rng)
    dets = []
    for k, (qvals, corr, mask, detd, _) in enumerate(geo):
        m = intens * (mean_count[k] / model_mean_count(intens, qvals, corr, mask, rng))
        phi = np.exp(rng.normal(0., phi_sigma, n_frames[k])) if phi_sigma > 0 else None
        fr = sample_frames(m, qvals, corr, mask, n_frames[k], rng, phi=phi)
        dets.append(dict(qvals=qvals, corr=corr, mask=mask, detd=detd, frame_quats=fr["quats"], phi=fr["phi"],
                         **{key: fr[key] for key in ("ones", "multi", "place_ones", "place_multi", "count_multi")}))
    quats = quat_gen(num_div)
    quats[:, 4] = 1. / quats.shape[0]
    return dets, dict(quats=quats, model_start=rng.random((1, size, size, size)), model_true=intens * scale0)


def small_problem_2d(seed=0, det_side=48, n_blobs=30, num_rot=90, n_frames=600, mean_count=80.,
                     hole_radius=3.):
    """A 2-D reconstruction (recon_type = 2d): a det_side^2 flat detector in
    pixel units (qz = 0), an image of n_blobs Gaussian blobs on the
    Iterate.calculate_size grid, num_rot equal-weight in-plane angles
    (Quaternion.generate_2d) and Poisson frames at random angles. Mask: 2
    inside hole_radius, 1 beyond size / 2 - 2 (merged, not in the likelihood)."""
    rng = np.random.default_rng(seed)
    c = (det_side - 1) / 2.
    ix, iy = np.meshgrid(np.arange(det_side) - c, np.arange(det_side) - c, indexing="ij")
    qvals = np.stack([ix.ravel(), iy.ravel(), np.zeros(ix.size)], 1)
    r = np.hypot(qvals[:, 0], qvals[:, 1])
    size = int(2 * np.ceil(r.max()) + 3)
    mask = np.zeros(r.size, np.uint8)
    mask[r > size / 2 - 2] = 1
    mask[r < hole_radius] = 2
    corr = 1. + 0.1 * rng.random(r.size)
    corr /= corr.mean()
    x = np.arange(size) - size // 2
    gx, gy = np.meshgrid(x, x, indexing="ij")
    img = np.zeros((size, size))
    for _ in range(n_blobs):
        cx, cy = rng.normal(0., size / 6., 2)
        sg = 1.5 + 2. * rng.random()
        img += rng.random() * np.exp(-((gx - cx) ** 2 + (gy - cy) ** 2) / (2 * sg * sg))
    lam = slices2d(img, rng.random(64) * 2 * np.pi, qvals, corr)
    img *= mean_count / lam[:, mask <= 1].sum(1).mean()
    fr = sample_frames(img, qvals, corr, mask, n_frames, rng, two_d=True)
    quats = np.zeros((num_rot, 5))
    quats[:, 0] = np.arange(num_rot) * (2 * np.pi / num_rot)
    quats[:, 4] = 1. / num_rot
    model_start = rng.random((1, size, size))
    return dict(qvals=qvals, corr=corr, mask=mask, quats=quats, model_start=model_start, model_true=img,
                **{k: fr[k] for k in ('ones', 'multi', 'place_ones', 'place_multi', 'count_multi')},
                frame_angles=fr['quats'])
