"""Float64 restatement of the adjoint absorption Jacobian and the LM step.

``J_complex`` (DOGPUP/dMesh.m:206-247), its time-gated form
(``fc2tg`` applied along the frequency axis, tutorials/tut_2...m:147 and
reconstruction/wghtd_LM_recon.m:61), the vector-Jacobian product of the TG
Jacobian, ``tik_inv`` (reconstruction/tik_inv.m:1-20) with an optional
diagonal data weight W, the voxel basis (mesh2grid, dMesh.m:286-380) and the
sensitivity reshaping weights (target_spots, dMesh.m:250-282; reshape_J,
reconstruction/reshape_J.m:1-17).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from .transforms import fc2tg


def point_location(node, elem, pts, eps=1e-12, chunk=64):
    """Containing tetrahedron and barycentric weights of each point, by testing
    every element (MATLAB ``pointLocation`` in mesh2grid, dMesh.m:311-313).

    The element whose smallest barycentric weight is largest wins (ties: lower
    id); it is accepted when that weight is >= -eps, else the point is outside
    (-1, zero weights).  Returns (eid [NP] int64, w [NP, 4])."""
    node = np.asarray(node, dtype=np.float64)
    elem = np.asarray(elem, dtype=np.int64)
    pts = np.atleast_2d(np.asarray(pts, dtype=np.float64))
    v = node[elem]                                                   # [NE, 4, 3]
    T = np.stack([v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]], axis=-1)
    Ti = np.linalg.inv(T)                                            # [NE, 3, 3]
    eid = np.full(pts.shape[0], -1, dtype=np.int64)
    w = np.zeros((pts.shape[0], 4))
    for c0 in range(0, pts.shape[0], chunk):
        p = pts[c0:c0 + chunk]
        l = np.einsum("eij,pej->pei", Ti, p[:, None, :] - v[None, :, 0])   # [P, NE, 3]
        lam = np.concatenate([1.0 - l.sum(-1, keepdims=True), l], axis=-1)
        score = lam.min(-1)
        j = np.argmax(score, axis=1)                                 # first maximum: lowest id
        best = score[np.arange(p.shape[0]), j]
        ok = best >= -eps
        rows = np.arange(c0, c0 + p.shape[0])[ok]
        eid[rows] = j[ok]
        w[rows] = lam[ok, j[ok]]
    return eid, w


def m2g_matrix(node, elem, grid, eps=1e-12):
    """mesh-to-grid interpolation [NV, NN] and the in-mesh mask (dMesh.m:311-327)."""
    eid, w = point_location(node, elem, grid, eps)
    inm = eid >= 0
    ii = np.repeat(np.nonzero(inm)[0], 4)
    jj = np.asarray(elem, dtype=np.int64)[eid[inm]].ravel()
    return sp.csr_matrix((w[inm].ravel(), (ii, jj)), shape=(grid.shape[0], node.shape[0])), inm


def g2m_matrix(node, axes, inmesh):
    """Grid-to-mesh interpolation [NN, NV] (dMesh.m:330-373).

    The reference locates every node in ``delaunay(grid)`` and keeps the
    barycentric weights of in-mesh voxels (:332-348); a node none of whose
    four voxels is in the mesh takes its nearest in-mesh voxel with weight 1
    (:351-367); rows are normalised (:369-372).  A rectilinear lattice has
    many Delaunay triangulations; this restatement uses the Kuhn split (cell
    corner c, fractions sorted t_a >= t_b >= t_c with ties in axis order,
    simplex c, c+e_a, c+e_a+e_b, c+1).  Nodes outside the lattice take the
    nearest in-mesh voxel.  Nearest ties: lower voxel index."""
    node = np.asarray(node, dtype=np.float64)
    axes = [np.asarray(a, dtype=np.float64).ravel() for a in axes]
    n = [a.size for a in axes]
    o = [a[0] for a in axes]
    d = [a[1] - a[0] if a.size > 1 else 1.0 for a in axes]
    inmesh = np.asarray(inmesh, dtype=bool)
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    grid = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    inm_idx = np.nonzero(inmesh)[0]
    rows, cols, vals = [], [], []
    for r in range(node.shape[0]):
        p = node[r]
        f = [(p[k] - o[k]) / d[k] for k in range(3)]
        in_grid = all(0.0 <= f[k] <= n[k] - 1 for k in range(3))
        kept, ent = 0, []
        if in_grid:
            cell = [min(max(int(np.floor(f[k])), 0), max(n[k] - 2, 0)) for k in range(3)]
            fr = [0.0 if n[k] == 1 else f[k] - cell[k] for k in range(3)]
            order = sorted(range(3), key=lambda k: -fr[k])            # stable: ties keep axis order
            a, b, c = order
            w = [1.0 - fr[a], fr[a] - fr[b], fr[b] - fr[c], fr[c]]
            v = list(cell)
            for q in range(4):
                if q > 0:
                    ax = order[q - 1]
                    v[ax] = min(v[ax] + 1, n[ax] - 1)
                vox = v[0] + n[0] * (v[1] + n[1] * v[2])
                if inmesh[vox]:
                    kept += 1
                    if w[q] != 0.0:
                        ent.append((vox, w[q]))
            s = 0.0
            for _, wq in ent:
                s += wq
            if s != 0.0:
                ent = [(vox, wq / s) for vox, wq in ent]
        if kept == 0 and inm_idx.size:
            d2 = ((grid[inm_idx] - p) ** 2).sum(axis=1)
            ent = [(int(inm_idx[int(np.argmin(d2))]), 1.0)]
        for vox, wq in ent:
            rows.append(r)
            cols.append(vox)
            vals.append(wq)
    return sp.csr_matrix((vals, (rows, cols)), shape=(node.shape[0], grid.shape[0]))


def j_complex(P, w, phi, phiA, link, fpsf):
    """J[m, k, v] = -(P phi_s)[v,k] * (P phiA_d)[v,k] * w[v] / s_fpsf[k], dMesh.m:239-245.

    ``P`` is the [NV, NN] interpolation matrix (``mesh.m2g``, dMesh.m:286-380,
    or the identity for a nodal basis), ``w`` the per-voxel weight
    (``dxyz^3`` for the voxel grid).  ``phi``: [NN, NS, NF], ``phiA``:
    [NN, ND, NF], ``link``: [NM, 2] (source, detector) 0-based.
    Returns [NM, NF, NV] complex128.
    """
    P = sp.csr_matrix(P)
    nn, ns, nf = phi.shape
    pg = (P @ phi.reshape(nn, -1)).reshape(-1, ns, nf)       # :239
    pa = (P @ phiA.reshape(nn, -1)).reshape(-1, phiA.shape[1], nf)   # :240
    w = np.broadcast_to(np.asarray(w, dtype=np.float64), (pg.shape[0],))
    J = -pg[:, link[:, 0], :] * pa[:, link[:, 1], :] * w[:, None, None]   # [NV, NM, NF], :242
    J = np.transpose(J, (1, 2, 0))                          # :244
    return J / np.asarray(fpsf)[None, :, None]              # :245


def j_tg(J, gate_fc, nt):
    """TG Jacobian [NM, NG, NV]: fc2tg along the frequency axis of J."""
    Jm = np.moveaxis(J, 1, -1)                              # [NM, NV, NF]
    out = fc2tg(Jm, gate_fc, np.arange(J.shape[1]), nt)     # [NM, NV, NG]
    return np.moveaxis(out, -1, 1)


def j_tg_vjp(J_tg, g):
    """J^T g for the TG Jacobian: sum over measurements and gates of J[m,g,v] g[m,g]."""
    return np.einsum("mgv,mg->v", J_tg, g)


def target_spots(grid, inmesh, pos, w, kind="gauss"):
    """Sensitivity spots [NS, NV] (dMesh.m:250-282): a Gaussian whose width
    parameter is (2 sqrt(2 ln 2)) w, or a cube of side w, around each spot
    centre, normalised to unit sum over all voxels, negated, and zero outside
    the mesh."""
    grid = np.asarray(grid, dtype=np.float64)
    pos = np.atleast_2d(np.asarray(pos, dtype=np.float64))
    if kind == "gauss":
        s = 2.0 * np.sqrt(2.0 * np.log(2.0)) * w                      # :267
        t = np.exp(-((grid[:, None, 0] - pos[None, :, 0]) ** 2) / (s ** 2 * 2)
                   - ((grid[:, None, 1] - pos[None, :, 1]) ** 2) / (s ** 2 * 2)
                   - ((grid[:, None, 2] - pos[None, :, 2]) ** 2) / (s ** 2 * 2))
    elif kind == "square":
        h = w / 2                                                     # :272
        t = np.ones((grid.shape[0], pos.shape[0]), dtype=bool)
        for d in range(3):
            t &= (grid[:, None, d] <= pos[None, :, d] + h) & (grid[:, None, d] >= pos[None, :, d] - h)
        t = t.astype(np.float64)
    else:
        raise ValueError("Check spot type is gauss or square")
    t = t / t.sum(axis=0)                                             # :279
    t = -t.T
    t[:, ~np.asarray(inmesh, dtype=bool)] = 0.0                        # :281
    return t


def reshape_j(J, Js, lam):
    """w = (Js J^T) / (J J^T + lam max(diag(J J^T)) I)  (reconstruction/reshape_J.m:13-15);
    J [NM, NV], Js [NS, NV]; returns [NS, NM]."""
    A = J @ J.T
    A = A + lam * np.max(np.diag(A)) * np.eye(A.shape[0])
    return np.linalg.solve(A.T, (Js @ J.T).T).T


def tik_inv(J, lam, y, weights=None, diag_mode="max"):
    """Regularised normal-equation step, reconstruction/tik_inv.m:13-20.

    H = J^T W J, H_ii += lam * alpha with alpha = max_j sum_i W_i J_ij^2
    (the reference rule, W = I there); ``diag_mode="diag"`` adds
    lam * H_ii instead.  Returns H^-1 J^T W y.
    """
    J = np.asarray(J, dtype=np.float64)
    Wd = np.ones(J.shape[0]) if weights is None else np.asarray(weights, dtype=np.float64)
    JW = J * Wd[:, None]
    H = J.T @ JW                                            # :14
    if diag_mode == "max":
        alph = np.max((J ** 2 * Wd[:, None]).sum(axis=0))   # :13
        H[np.diag_indices_from(H)] += lam * alph            # :15-16
    else:
        H[np.diag_indices_from(H)] *= (1.0 + lam)
    rhs = JW.T @ y                                          # :19
    L = np.linalg.cholesky(H)                               # :20 (H is SPD: backslash -> Cholesky)
    return np.linalg.solve(L.T, np.linalg.solve(L, rhs))
