"""Uniform sampling of rotations by refining the 600-cell.

Orientations for the EMC search: the 120 vertices of the 600-cell (unit
quaternions) plus, for ``num_div = n``, the points that subdivide each of its
720 edges, 1200 faces and 600 cells into n parts, projected onto the unit
3-sphere, with a weight per point for the non-uniform density of the
projection. q and -q are the same rotation, so half the points are kept:
those whose first non-zero coordinate is positive. That gives
``10 * (5 n^3 + n)`` rotations (Loh & Elser, Phys. Rev. E 80, 026705 (2009)).

This module follows the construction of duaneloh/Dragonfly's quat_gen
(dragonfly/src/quaternion.c:811-842): the same vertex, edge, face and cell
enumeration order, the same point order and the same weight formula, so the
list is identical, element for element, to the reference's. The order matters:
the most likely orientation of a frame is reported as an index into this list.

Exact arithmetic: every point has coordinates (a + b*tau) / (2 n) with integer
a, b and tau the golden ratio, and is stored as the integer pair (a, b).
"""
import math

import numpy as np

TAU = (np.sqrt(5.) + 1.) / 2.
NUM_VERT, NUM_EDGE, NUM_FACE, NUM_CELL, NNN = 120, 720, 1200, 600, 12

# Even permutations of four coordinates, in the reference's order (quaternion.c:31-33).
_EVEN_PERMS = np.array([[0, 1, 2, 3], [0, 2, 3, 1], [0, 3, 1, 2],
                        [1, 2, 0, 3], [1, 0, 3, 2], [1, 3, 2, 0],
                        [2, 0, 1, 3], [2, 3, 0, 1], [2, 1, 3, 0],
                        [3, 1, 0, 2], [3, 0, 2, 1], [3, 2, 1, 0]])


def _vertices(n):
    """The 120 vertices: float coordinates and integer (a, b) pairs scaled by 2n
    (quaternion.c:27-113)."""
    vf = np.zeros((NUM_VERT, 4))
    vi = np.zeros((NUM_VERT, 4, 2), dtype=np.int64)
    idx = 0
    # 16 vertices (+-1/2, +-1/2, +-1/2, +-1/2)
    for h in range(2):
        for i in range(2):
            for j in range(2):
                for k in range(2):
                    s = np.array([h, i, j, k])
                    vf[idx] = s - 0.5
                    vi[idx, :, 0] = (2 * s - 1) * n
                    idx += 1
    # 8 vertices (+-1, 0, 0, 0) and permutations
    for h in range(2):
        for i in range(4):
            vf[idx, i] = 2 * h - 1.0
            vi[idx, i, 0] = (2 * h - 1) * 2 * n
            idx += 1
    # 96 vertices: even permutations of (+-tau, +-1, +-1/tau, 0) / 2
    for i in range(2):
        for j in range(2):
            for k in range(2):
                base = np.array([(2 * i - 1) * TAU / 2., (2 * j - 1) * 0.5, (2 * k - 1) / (2 * TAU), 0.])
                bint = np.array([[0, (2 * i - 1) * n], [(2 * j - 1) * n, 0],
                                 [-(2 * k - 1) * n, (2 * k - 1) * n], [0, 0]])
                for m in range(12):
                    vf[idx] = base[_EVEN_PERMS[m]]
                    vi[idx] = bint[_EVEN_PERMS[m]]
                    idx += 1
    return vf, vi


def _dist2(a, b):
    """sum_k (a_k - b_k)^2, added in k order from 0 (as the reference's loops)."""
    d = (a - b) ** 2
    return ((d[..., 0] + d[..., 1]) + d[..., 2]) + d[..., 3]


def _topology(vf):
    """Edges, nearest-neighbour lists, faces, cells and the face/edge -> cell
    maps, enumerated in the reference's order (quaternion.c:115-298)."""
    d0 = _dist2(vf[0][None, :], vf[1:])
    min_d2 = min(d0[0], d0[1:].min()) + 1.e-6
    all_d2 = _dist2(vf[:, None, :], vf[None, :, :])
    near = all_d2 < min_d2
    edges = []
    nn = [[] for _ in range(NUM_VERT)]
    for i in range(NUM_VERT):
        for j in range(i + 1, NUM_VERT):
            if near[i, j]:
                edges.append((i, j))
                nn[i].append(j)
                nn[j].append(i)
    edges = np.array(edges)
    nn = np.array(nn)
    le = all_d2 <= min_d2  # "not greater than" tests of make_cell / make_map

    faces = []
    for a, b in edges:
        for c in nn[a]:
            if c <= b:
                continue
            if all_d2[c, b] < min_d2:
                faces.append((a, b, c))
    faces = np.array(faces)

    cells = []
    for a, b, c in faces:
        for d in nn[a]:
            if d <= c:
                continue
            if le[d, b] and le[d, c]:
                cells.append((a, b, c, d))
    cells = np.array(cells)

    face2cell = np.zeros((NUM_FACE, 4), dtype=np.int64)
    for f, (a, b, c) in enumerate(faces):
        for d in nn[a]:
            if d == b or d == c:
                continue
            if le[d, b] and le[d, c]:
                face2cell[f] = (a, b, c, d)
                break

    edge2cell = np.zeros((NUM_EDGE, 4), dtype=np.int64)
    for e, (a, b) in enumerate(edges):
        for jj in range(NNN):
            c = nn[a][jj]
            if c == b or not le[c, b]:
                continue
            edge2cell[e, :3] = (a, b, c)
            for kk in range(jj + 1, NNN):
                d = nn[a][kk]
                if d == b or not le[d, b] or not le[d, c]:
                    continue
                edge2cell[e, 3] = d
                break
            break
    return edges, faces, cells, face2cell, edge2cell


def _weight(vq, vc):
    """Density weight of point vq seen from cell centre vc (quaternion.c:300-318)."""
    sq = vq * vq
    sc = vc * vc
    norm_q = np.sqrt(((sq[..., 0] + sq[..., 1]) + sq[..., 2]) + sq[..., 3])
    norm_c = np.sqrt(((sc[..., 0] + sc[..., 1]) + sc[..., 2]) + sc[..., 3])
    p = vq * vc
    w = ((p[..., 0] + p[..., 1]) + p[..., 2]) + p[..., 3]
    # libm pow, as the reference calls it; numpy's power rounds differently.
    q4 = np.vectorize(math.pow, otypes=[np.float64])(norm_q, 4.)
    return w / (q4 * norm_c)


def _centroid(vf, idx4):
    """Sum of four vertices, added in order from 0."""
    v = vf[idx4]
    return ((v[..., 0, :] + v[..., 1, :]) + v[..., 2, :]) + v[..., 3, :]


def _to_float(vec, n):
    return (vec[..., 0] + TAU * vec[..., 1]) / (2.0 * n)


def _lattice_steps(n, dim):
    """Interior barycentric steps of a dim-simplex subdivided n times, in the
    reference's loop order (quaternion.c:385, 419-420, 460-462)."""
    if dim == 1:
        return [(j,) for j in range(1, n)]
    if dim == 2:
        return [(j, k) for j in range(1, n - 1) for k in range(1, n - j)]
    return [(j, k, m) for j in range(1, n - 2) for k in range(1, n - 1 - j) for m in range(1, n - j - k)]


def _refine(vi, simplices, centroid_cells, vf, n, factor):
    """Points inside each simplex (edge / face / cell), their integer vectors
    and weights, simplex-major then step order (quaternion.c:359-472)."""
    dim = simplices.shape[1] - 1
    steps = np.array(_lattice_steps(n, dim), dtype=np.int64).reshape(-1, dim)
    if steps.shape[0] == 0:
        return np.zeros((0, 4, 2), np.int64), np.zeros(0)
    origin = vi[simplices[:, 0]]                                    # [S,4,2]
    # Vertex coordinates are multiples of n, so the differences divide exactly.
    deltas = np.stack([(vi[simplices[:, e]] - origin) // n for e in range(1, dim + 1)],
                      axis=1)                                         # [S,dim,4,2]
    vec = origin[:, None] + np.einsum('td,sdkc->stkc', steps, deltas)  # [S,T,4,2]
    vq = _to_float(vec, n)
    vc = _centroid(vf, centroid_cells)[:, None, :]
    w = factor * _weight(vq, vc) if factor is not None else _weight(vq, vc)
    return vec.reshape(-1, 4, 2), w.reshape(-1)


def _keep_half(vec):
    """True where the first non-zero integer coordinate is positive
    (quaternion.c:486-510)."""
    flat = vec.reshape(vec.shape[0], 8)
    nz = flat != 0
    first = np.argmax(nz, axis=1)
    val = flat[np.arange(flat.shape[0]), first]
    return nz.any(axis=1) & (val > 0)


def _normalise(vec, n):
    q = _to_float(vec, n)
    sq = q * q
    norm = np.sqrt(((sq[:, 0] + sq[:, 1]) + sq[:, 2]) + sq[:, 3])
    return q / norm[:, None]


def quat_gen(num_div):
    """Returns the [10 (5 n^3 + n), 5] array (q0, q1, q2, q3, weight), weights
    summing to one."""
    n = int(num_div)
    if n < 1:
        raise ValueError('num_div must be >= 1')
    vf, vi = _vertices(n)
    edges, faces, cells, face2cell, edge2cell = _topology(vf)

    # Vertex weights: first cell (in cell order) containing each vertex
    # (quat_setup, quaternion.c:320-357), scaled by 5/6.
    vert_w = np.zeros(NUM_VERT)
    seen = np.zeros(NUM_VERT, dtype=bool)
    for c in cells:
        vc = _centroid(vf, c[None])[0]
        for v in c:
            if seen[v]:
                continue
            seen[v] = True
            vert_w[v] = (5. / 6) * _weight(vf[v], vc)

    groups = [(vi, vert_w)]
    if n > 1:
        groups.append(_refine(vi, edges, edge2cell, vf, n, 35. / 36))
    if n > 2:
        groups.append(_refine(vi, faces, face2cell, vf, n, None))
    if n > 3:
        groups.append(_refine(vi, cells, cells, vf, n, None))

    out = []
    for vec, w in groups:
        keep = _keep_half(vec)
        q = _normalise(vec[keep], n)
        out.append(np.concatenate([q, w[keep][:, None]], axis=1))
    quats = np.concatenate(out, axis=0)
    expected = 10 * (5 * n ** 3 + n)
    if quats.shape[0] != expected:
        raise RuntimeError('quaternion count %d != %d' % (quats.shape[0], expected))
    total = np.cumsum(quats[:, 4])[-1]
    quats[:, 4] *= 1. / total
    return quats
