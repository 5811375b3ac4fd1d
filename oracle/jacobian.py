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
