"""Float64 restatement of optode snapping (snap_pos, DOGPUP/dOptode.m:155-190).

Test infrastructure: the device path (dgp_snap_to_surface) is checked against
it.  The nearest boundary node is the first minimum of the distances
(dsearchn, :162); among the surface triangles that contain it (:171) the
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
