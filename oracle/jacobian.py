"""Float64 restatement of the adjoint absorption Jacobian and the LM step.

``J_complex`` (DOGPUP/dMesh.m:206-247), its time-gated form
(``fc2tg`` applied along the frequency axis, tutorials/tut_2...m:147 and
reconstruction/wghtd_LM_recon.m:61), the vector-Jacobian product of the TG
Jacobian, and ``tik_inv`` (reconstruction/tik_inv.m:1-20) with an optional
diagonal data weight W.
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
