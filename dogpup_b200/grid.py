"""Voxel basis of the Jacobian: ``mesh2grid`` (DOGPUP/dMesh.m:286-380).

Builds m2g (mesh -> voxel barycentric interpolation, <= 4 entries per row),
the in-mesh mask and the voxel size, as the reference does once per mesh with
MATLAB's ``pointLocation``; the point location runs on the device
(``dgp_locate_points``) or on the host (k-d tree candidates).  The grid-to-mesh map g2m is built from the
transpose of m2g, row-normalised (a simplification of the reference's
Delaunay-based g2m, used only to map updates back to nodes).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.spatial import cKDTree

from .optode import barycentric


def locate_host(node, elem, grid, tree=None, eps=1e-12):
    """Containing element (-1: none) and barycentric weights of each grid point, on the host
    (candidates: the 32 elements with the nearest centroids)."""
    nv = grid.shape[0]
    if tree is None:
        tree = cKDTree(node[elem].mean(axis=1))
    k = min(32, elem.shape[0])
    _, cand = tree.query(grid, k=k)
    eid = np.full(nv, -1, dtype=np.int64)
    w = np.zeros((nv, 4))
    for c0 in range(0, nv, 4096):
        sl = slice(c0, min(nv, c0 + 4096))
        cc = cand[sl]                                                   # [B, k]
        lam = barycentric(node, elem, cc, np.broadcast_to(grid[sl][:, None, :], cc.shape + (3,)))
        score = lam.min(axis=2)
        j = np.argmax(score, axis=1)
        best = score[np.arange(cc.shape[0]), j]
        ok = best >= -eps
        rows = np.arange(sl.start, sl.stop)[ok]
        eid[rows] = cc[ok, j[ok]]
        w[rows] = lam[ok, j[ok]]
    return eid, w


def mesh2grid(node, elem, x, y, z, tree=None, device=False, dev_mesh=None):
    """Returns dict(grid [NV,3], m2g CSR [NV x NN], gridinmesh [NV], dxyz, size).

    device=True locates the voxel centres with ``dgp_locate_points`` (every
    element whose bounding box touches the point's bin is a candidate);
    dev_mesh = (node, elem) already on the device, optional."""
    node = np.asarray(node, dtype=np.float64)
    elem = np.asarray(elem, dtype=np.int64)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")                      # ndgrid, :308
    grid = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    nv = grid.shape[0]
    if device:
        from . import api
        dn, de = dev_mesh if dev_mesh is not None else (node, elem)
        e_d, w_d = api.locate_points(dn, de, grid, eps=1e-12)
        eid, w = e_d.cpu().numpy(), w_d.cpu().numpy()
    else:
        eid, w = locate_host(node, elem, grid, tree)
    inmesh = eid >= 0                                                   # :315
    ii = np.repeat(np.nonzero(inmesh)[0], 4)
    jj = elem[eid[inmesh]].ravel()
    vv = w[inmesh].ravel()
    m2g = sp.csr_matrix((vv, (ii, jj)), shape=(nv, node.shape[0]))     # :327
    m2g.sort_indices()
    dx = abs(x[1] - x[0])
    g2m = m2g.T.tocsr()
    s = np.asarray(g2m.sum(axis=1)).ravel()
    s[s == 0] = 1.0
    g2m = sp.diags(1.0 / s) @ g2m
    return dict(grid=grid, m2g=m2g, g2m=g2m.tocsr(), gridinmesh=inmesh, dxyz=dx,
                size=(len(x), len(y), len(z)))
