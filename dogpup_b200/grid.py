"""Voxel basis of the Jacobian: ``mesh2grid`` (DOGPUP/dMesh.m:286-380).

Builds m2g (mesh -> voxel barycentric interpolation, <= 4 entries per row),
the in-mesh mask, the voxel size and g2m (voxel -> node interpolation), as
the reference does once per mesh with MATLAB's ``pointLocation`` and
``delaunay``.  The point location (``dgp_locate_points``) and g2m
(``dgp_grid_to_mesh``) run on the device.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp


def m2g_from_location(eid, w, elem, nn):
    """m2g [NV x NN] from each voxel's element and barycentric weights (dMesh.m:315-327);
    zero weights are not stored, as MATLAB's ``sparse`` drops them."""
    inmesh = eid >= 0                                                   # :315
    ii = np.repeat(np.nonzero(inmesh)[0], 4)
    jj = np.asarray(elem, dtype=np.int64)[eid[inmesh]].ravel()
    vv = w[inmesh].ravel()
    m2g = sp.csr_matrix((vv, (ii, jj)), shape=(eid.shape[0], nn))      # :327
    m2g.eliminate_zeros()
    m2g.sort_indices()
    return m2g, inmesh


def g2m_from_rows(col, val, nv):
    """g2m [NN x NV] from the device rows (voxel index or -1, weight) [NN][4]."""
    nn = col.shape[0]
    keep = (col >= 0) & (val != 0)
    ii = np.repeat(np.arange(nn), 4).reshape(nn, 4)[keep]
    g2m = sp.csr_matrix((val[keep], (ii, col[keep])), shape=(nn, nv))
    g2m.sort_indices()
    return g2m


def mesh2grid(node, elem, x, y, z):
    """Returns dict(grid [NV,3], m2g CSR [NV x NN], g2m CSR [NN x NV], gridinmesh [NV], dxyz, size).

    The voxel centres are located with ``dgp_locate_points``; g2m is built on the device
    (``dgp_grid_to_mesh``: Kuhn triangulation of the lattice, in-mesh voxels,
    nearest in-mesh voxel for uncovered nodes, rows normalised)."""
    from . import api
    node = np.asarray(node, dtype=np.float64)
    elem = np.asarray(elem, dtype=np.int64)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")                      # ndgrid, :308
    grid = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    nv = grid.shape[0]
    e_d, w_d = api.locate_points(node, elem, grid, eps=1e-12)
    eid, w = e_d.cpu().numpy(), w_d.cpu().numpy()
    m2g, inmesh = m2g_from_location(eid, w, elem, node.shape[0])
    col, val = api.grid_to_mesh(node, (x, y, z), inmesh)               # :330-373
    g2m = g2m_from_rows(col.cpu().numpy(), val.cpu().numpy(), nv)
    dx = abs(x[1] - x[0])
    return dict(grid=grid, m2g=m2g, g2m=g2m, gridinmesh=inmesh, dxyz=dx, size=(len(x), len(y), len(z)))
