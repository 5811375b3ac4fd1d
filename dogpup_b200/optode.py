"""Optode set-up: source spectrum, surface snapping, barycentric weights.

Mirrors the ``dOptode`` class (DOGPUP/dOptode.m:34-199).  The Fourier
coefficients of the source pulse come from the device ``td2fc`` kernel; the
geometry (nearest surface point, containing tetrahedron) runs on the device
(``dgp_snap_to_surface``, ``dgp_locate_points``), or on the host with k-d
tree candidates (``snap2mesh(mesh, device=False)``).
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.spatial import cKDTree

from . import api


class DOptode:
    """``dOptode(s_pos, d_pos, link, avgPow, tpsf, tAxis, Nf)``, dOptode.m:34-74.

    ``link`` rows are (source, detector), 0-based here.
    """

    def __init__(self, s_pos, d_pos, link, avg_pow, tpsf, t_axis, nf):
        self.link = np.asarray(link, dtype=np.int64).reshape(-1, 2)
        self.Nf = int(nf)
        t_axis = np.asarray(t_axis, dtype=np.float64)
        self.dt = t_axis[1] - t_axis[0]                                     # :55
        self.tAxis = t_axis
        T = t_axis[-1]                                                      # :57
        w0 = 2 * np.pi / T
        self.fAxis = np.arange(self.Nf) * w0                                # :59
        self.df = self.fAxis[1] - self.fAxis[0] if self.Nf > 1 else w0      # :60
        self.d_positions = np.asarray(d_pos, dtype=np.float64).reshape(-1, 3)
        self.s_positions = np.asarray(s_pos, dtype=np.float64).reshape(-1, 3)
        self.s_avgPow = float(avg_pow)
        tpsf = np.asarray(tpsf, dtype=np.float64)
        self.s_tpsf = tpsf * (avg_pow / tpsf.mean())                        # :69-71
        self.s_fpsf = api.td2fc(torch.as_tensor(self.s_tpsf, device="cuda")[None, :],   # :73
                                torch.as_tensor(self.fAxis), torch.as_tensor(self.tAxis))[0]
        self.s_bary = self.d_bary = None
        self.s_dirs = self.d_dirs = None

    def snap2mesh(self, mesh, device=True):
        """Snap optodes to the surface, move sources 1/min(musp) inward (dOptode.m:77-97).

        device=True: surface search (``dgp_snap_to_surface``) and point location
        (``dgp_locate_points``) on the GPU; device=False: the host k-d tree path."""
        if device:
            return self._snap2mesh_device(mesh)
        self.d_positions, self.d_bary, self.d_dirs = snap_pos(mesh, self.d_positions)
        self.s_positions, _, self.s_dirs = snap_pos(mesh, self.s_positions)
        inset = self.s_positions + (1.0 / float(np.min(mesh.musp_host))) * self.s_dirs   # :89
        eid, w = locate_points(mesh.node_host, mesh.elem_host, inset, mesh.locator())
        self.s_bary = _clean_bary(eid, w)
        return self


    def _snap2mesh_device(self, mesh):
        node = torch.as_tensor(mesh.node_host, device="cuda")
        elem = torch.as_tensor(mesh.elem_host, device="cuda", dtype=torch.int32)
        face = torch.as_tensor(mesh.face_host, device="cuda", dtype=torch.int32)

        def locate(pts):
            eid, w = api.locate_points(node, elem, pts, eps=1e-9)          # pointLocation, :88-92, :188
            eid, w = eid.cpu().numpy(), w.cpu().numpy()
            if (eid < 0).any():
                raise ValueError(f"point {pts[int(np.nonzero(eid < 0)[0][0])].tolist()} lies outside the mesh")
            return _clean_bary(eid, w)

        dpos, ddir, _ = api.snap_to_surface(node, mesh.fem.bnd, face, self.d_positions)
        spos, sdir, _ = api.snap_to_surface(node, mesh.fem.bnd, face, self.s_positions)
        self.d_positions, self.d_dirs = dpos.cpu().numpy(), ddir.cpu().numpy()
        self.s_positions, self.s_dirs = spos.cpu().numpy(), sdir.cpu().numpy()
        self.d_bary = locate(dpos)
        self.s_bary = locate(spos + (1.0 / float(np.min(mesh.musp_host))) * sdir)   # :89
        return self


def _clean_bary(eid, w):
    """Clamp weights below 1e-10 to zero and renormalise (dOptode.m:93-95, :194-197)."""
    w = np.where(w < 1e-10, 0.0, w)
    w = w / w.sum(axis=1, keepdims=True)
    return np.concatenate([eid[:, None].astype(np.float64), w], axis=1)


def closest_point_on_triangle(p, a, b, c):
    """Closest point of triangle abc to p (Voronoi-region walk over vertices,
    edges and face, as in Ericson, Real-Time Collision Detection, sec. 5.1.5)."""
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


def snap_pos(mesh, pos):
    """Nearest surface point, inward normal and barycentric weights (dOptode.m:155-199)."""
    node = mesh.node_host
    face = mesh.face_host
    bidx = np.nonzero(mesh.bnd_host)[0]
    tree = cKDTree(node[bidx])
    _, nb = tree.query(pos)                                                  # dsearchn, :162
    ids = bidx[nb]
    out = np.empty_like(pos)
    norm = np.empty_like(pos)
    for i in range(pos.shape[0]):
        fi = np.nonzero((face == ids[i]).any(axis=1))[0]                   # :171
        best, bpt, bf = np.inf, None, -1
        for f in fi:
            a, b, c = node[face[f]]
            q = closest_point_on_triangle(pos[i], a, b, c)
            d = np.linalg.norm(q - pos[i])
            if d < best:
                best, bpt, bf = d, q, f
        out[i] = bpt                                                        # :180
        a, b, c = node[face[bf]]
        nv = -np.cross(b - a, c - a)                                        # :181-184
        norm[i] = nv / np.linalg.norm(nv)
    eid, w = locate_points(node, mesh.elem_host, out, mesh.locator())
    return out, _clean_bary(eid, w), norm


def barycentric(node, elem, e, p):
    v = node[elem[e]]                                                       # [.., 4, 3]
    T = np.stack([v[..., 0, :] - v[..., 3, :], v[..., 1, :] - v[..., 3, :], v[..., 2, :] - v[..., 3, :]], axis=-1)
    l3 = np.linalg.solve(T, (p - v[..., 3, :])[..., None])[..., 0]
    return np.concatenate([l3, 1.0 - l3.sum(axis=-1, keepdims=True)], axis=-1)


def locate_points(node, elem, pts, tree=None, k=48):
    """Containing tetrahedron and barycentric weights of each point
    (MATLAB ``pointLocation``); points within 1e-9 outside the closest tet are
    accepted (surface points).  Returns (elem_id, weights[., 4])."""
    pts = np.atleast_2d(pts)
    if tree is None:
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
        if score[j] < -1e-9:
            raise ValueError(f"point {pts[i]} lies outside the mesh")
        eid[i] = cand[i, j]
        w[i] = lam[j]
    return eid, w
