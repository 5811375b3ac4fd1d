"""Float64 restatement of optode snapping (snap_pos, DOGPUP/dOptode.m:155-190),
point location and the oriented surface faces.

Test infrastructure (never imported by the package): the device path
(dgp_snap_to_surface, dgp_locate_points) is checked against it, and the CPU
baseline of the benchmark places its sources with it.  The nearest boundary
node is the first minimum of the distances (dsearchn, :162); among the surface triangles that contain it (:171) the
closest point wins (first minimum in face order, :173-180), and the normal is
-cross(b - a, c - a) normalised (:181-184).  The closest point on a triangle
is computed here by a different route from the library's Voronoi-region
walk: the orthogonal projection onto the plane when it falls inside the
triangle, else the nearest of the three edge projections.
"""
from __future__ import annotations

import numpy as np


def _closest_on_segment(p, a, b):
    ab = b - a
    t = np.clip((p - a) @ ab / (ab @ ab), 0.0, 1.0)
    return a + t * ab


def closest_point_on_triangle(p, a, b, c):
    n = np.cross(b - a, c - a)
    q = p - ((p - a) @ n) / (n @ n) * n                       # projection onto the plane
    # inside test: q's barycentric weights w.r.t. a, b, c all >= 0
    T = np.stack([b - a, c - a], axis=1)
    uv, *_ = np.linalg.lstsq(T, q - a, rcond=None)
    if uv[0] >= 0 and uv[1] >= 0 and uv.sum() <= 1:
        return q
    cands = [_closest_on_segment(p, a, b), _closest_on_segment(p, b, c), _closest_on_segment(p, c, a)]
    d = [np.linalg.norm(x - p) for x in cands]
    return cands[int(np.argmin(d))]


def snap_pos(node, bnd, face, pos):
    """(surface points [N, 3], inward normals [N, 3], face ids [N], distances [N, k] of every
    candidate face) for positions [N, 3]."""
    node = np.asarray(node, dtype=np.float64)
    face = np.asarray(face, dtype=np.int64)
    bidx = np.nonzero(np.asarray(bnd) != 0)[0]
    pos = np.atleast_2d(np.asarray(pos, dtype=np.float64))
    out, norm, fid, dists = np.empty_like(pos), np.empty_like(pos), np.empty(len(pos), np.int64), []
    for i, p in enumerate(pos):
        nb = bidx[int(np.argmin(((node[bidx] - p) ** 2).sum(1)))]
        fi = np.nonzero((face == nb).any(axis=1))[0]
        qs = [closest_point_on_triangle(p, *node[face[f]]) for f in fi]
        d = np.array([np.linalg.norm(q - p) for q in qs])
        j = int(np.argmin(d))
        out[i], fid[i] = qs[j], fi[j]
        a, b, c = node[face[fi[j]]]
        nv = -np.cross(b - a, c - a)
        norm[i] = nv / np.linalg.norm(nv)
        dists.append(np.sort(d))
    return out, norm, fid, dists


def closest_point_on_triangle_walk(p, a, b, c):
    """Closest point of triangle abc to p by the Voronoi-region walk over vertices,
    edges and face (Ericson, Real-Time Collision Detection, sec. 5.1.5) -- the method
    the device kernel uses, restated here so the two routes can check each other."""
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = ab @ ap, ac @ ap
    if d1 <= 0 and d2 <= 0:
        return a
    bp = p - b
    d3, d4 = ab @ bp, ac @ bp
    if d3 >= 0 and d4 <= d3:
        return b
    vc = d1 * d4 - d3 * d2
    if vc <= 0 and d1 >= 0 and d3 <= 0:
        return a + (d1 / (d1 - d3)) * ab
    cp = p - c
    d5, d6 = ab @ cp, ac @ cp
    if d6 >= 0 and d5 <= d6:
        return c
    vb = d5 * d2 - d1 * d6
    if vb <= 0 and d2 >= 0 and d6 <= 0:
        return a + (d2 / (d2 - d6)) * ac
    va = d3 * d6 - d5 * d4
    if va <= 0 and (d4 - d3) >= 0 and (d5 - d6) >= 0:
        return b + ((d4 - d3) / ((d4 - d3) + (d5 - d6))) * (c - b)
    den = 1.0 / (va + vb + vc)
    return a + ab * (vb * den) + ac * (vc * den)


def surface_faces(node, elem):
    """Boundary triangles (faces owned by one tet) oriented with outward normals, as
    prepare_mesh builds mesh.face (DOGPUP/dMesh.m:964-998): a face whose normal points
    towards the bounding-box centre has its last two nodes swapped."""
    node = np.asarray(node, dtype=np.float64)
    elem = np.asarray(elem, dtype=np.int64)
    faces = np.concatenate([elem[:, [0, 1, 2]], elem[:, [0, 1, 3]], elem[:, [0, 2, 3]], elem[:, [1, 2, 3]]])
    _, ix, cnt = np.unique(np.sort(faces, axis=1), axis=0, return_index=True, return_counts=True)
    face = faces[ix[cnt == 1]].copy()                                   # :964-973
    com = node[face].mean(axis=1)                                       # :983-986
    centre = 0.5 * (node.max(axis=0) + node.min(axis=0))               # :990-992
    nrm = np.cross(node[face[:, 1]] - node[face[:, 0]], node[face[:, 2]] - node[face[:, 0]])
    flip = np.einsum("ij,ij->i", nrm, centre - com) > 0                # :994-997
    face[flip] = face[flip][:, [0, 2, 1]]
    return face


def barycentric(node, elem, e, p):
    """Barycentric weights of points p in elements e (broadcast over leading axes)."""
    v = node[elem[e]]                                                   # [.., 4, 3]
    T = np.stack([v[..., 0, :] - v[..., 3, :], v[..., 1, :] - v[..., 3, :], v[..., 2, :] - v[..., 3, :]], axis=-1)
    l3 = np.linalg.solve(T, (p - v[..., 3, :])[..., None])[..., 0]
    return np.concatenate([l3, 1.0 - l3.sum(axis=-1, keepdims=True)], axis=-1)


def locate_points(node, elem, pts, k=48, eps=1e-9):
    """Containing tetrahedron and barycentric weights of each point (MATLAB
    ``pointLocation``, dOptode.m:88-92, :188) among the k elements with the nearest
    centroids; the candidate whose smallest weight is largest wins and is accepted
    within eps outside (surface points).  Returns (elem id [NP], weights [NP, 4]);
    raises for a point outside the mesh."""
    from scipy.spatial import cKDTree
    node = np.asarray(node, dtype=np.float64)
    elem = np.asarray(elem, dtype=np.int64)
    pts = np.atleast_2d(np.asarray(pts, dtype=np.float64))
    tree = cKDTree(node[elem].mean(axis=1))
    k = min(k, elem.shape[0])
    _, cand = tree.query(pts, k=k)
    cand = np.atleast_2d(cand)
    eid = np.empty(pts.shape[0], dtype=np.int64)
    w = np.empty((pts.shape[0], 4))
    for i in range(pts.shape[0]):
        lam = barycentric(node, elem, cand[i], np.broadcast_to(pts[i], (cand.shape[1], 3)))
        score = lam.min(axis=1)
        j = int(np.argmax(score))
        if score[j] < -eps:
            raise ValueError(f"point {pts[i]} lies outside the mesh")
        eid[i] = cand[i, j]
        w[i] = lam[j]
    return eid, w


def clean_bary(eid, w):
    """Weights below 1e-10 set to zero and renormalised, as [elem id, 4 weights] rows
    (dOptode.m:93-95, :194-197)."""
    w = np.where(w < 1e-10, 0.0, w)
    w = w / w.sum(axis=1, keepdims=True)
    return np.concatenate([np.asarray(eid)[:, None].astype(np.float64), w], axis=1)


def snap2mesh(node, elem, bnd, face, musp, s_pos, d_pos):
    """dOptode.snap2mesh (dOptode.m:77-97): detectors snapped to the surface; sources
    snapped and moved 1/min(musp) inward along the inward normal (:89), then located.
    Returns (s_pos, s_dirs, s_bary, d_pos, d_dirs, d_bary)."""
    dq, dn, _, _ = snap_pos(node, bnd, face, d_pos)
    sq, sn, _, _ = snap_pos(node, bnd, face, s_pos)
    d_bary = clean_bary(*locate_points(node, elem, dq))
    s_bary = clean_bary(*locate_points(node, elem, sq + (1.0 / float(np.min(musp))) * sn))
    return sq, sn, s_bary, dq, dn, d_bary
