"""``DMesh``: the reference's ``dMesh`` class on the B200 path.

Mirrors DOGPUP/dMesh.m: construction (:48-77), ``update_properties``
(:80-88), ``add_optode`` (:91-96), ``flu_solve`` (:106-141), ``meas_flu``
(:144-171), ``adj_flu_solve`` (:174-202) and ``J_complex`` (:206-247).

Differences of layout: fields are device tensors ``[NF][NN][NS]`` complex128
(harmonic, node, source) instead of MATLAB's ``[NN x NF x NS]``; indices are
0-based.  ``to_reference_layout`` gives the reference's axis order.
"""
from __future__ import annotations

import numpy as np
import torch

from . import api

C_VAC = 2.99792458e11  # mm/s, dMesh.m:42


def surface_faces(node: np.ndarray, elem: np.ndarray) -> np.ndarray:
    """Faces owned by one tet, oriented with outward normals (dMesh.m:964-998)."""
    elem = np.asarray(elem, dtype=np.int64)
    faces = np.concatenate([elem[:, [0, 1, 2]], elem[:, [0, 1, 3]], elem[:, [0, 2, 3]], elem[:, [1, 2, 3]]])
    key = np.sort(faces, axis=1)
    _, ix, cnt = np.unique(key, axis=0, return_index=True, return_counts=True)
    face = faces[ix[cnt == 1]].copy()
    com = node[face].mean(axis=1)
    centre = 0.5 * (node.max(axis=0) + node.min(axis=0))
    vdir = centre - com
    nrm = np.cross(node[face[:, 1]] - node[face[:, 0]], node[face[:, 2]] - node[face[:, 0]])
    flip = np.einsum("ij,ij->i", nrm, vdir) > 0
    face[flip] = face[flip][:, [0, 2, 1]]
    return face


class DMesh:
    def __init__(self, node, elem, nr, props):
        """``dMesh(node, elem, nr, props)``: props = [mua musp] per node or one row."""
        self.node_host = np.asarray(node, dtype=np.float64)
        self.elem_host = np.asarray(elem, dtype=np.int64)
        self.nr = float(nr)
        nn = self.node_host.shape[0]
        props = np.atleast_2d(np.asarray(props, dtype=np.float64))
        if props.shape[0] == 1:
            props = np.repeat(props, nn, axis=0)
        self.fem = api.Fem(torch.as_tensor(self.node_host), torch.as_tensor(self.elem_host), self.nr)
        self.c = self.fem.c
        self.bnd_host = self.fem.bnd.cpu().numpy().astype(bool)
        self.face_host = surface_faces(self.node_host, self.elem_host)
        self.optode = None
        self._solver = None
        self._solver_key = None
        self.update_properties(props)

    # --------------------------------------------------------- properties
    @property
    def nn(self):
        return self.node_host.shape[0]

    def update_properties(self, props=None):
        """Re-assemble K, M on the device (dMesh.m:80-88)."""
        if props is not None:
            props = np.atleast_2d(np.asarray(props, dtype=np.float64))
            if props.shape[0] == 1:
                props = np.repeat(props, self.nn, axis=0)
            self.mua = torch.as_tensor(props[:, 0], device="cuda")
            self.musp = torch.as_tensor(props[:, 1], device="cuda")
            self.musp_host = props[:, 1].copy()
        self.K, self.M = self.fem.assemble(self.mua, self.musp)
        self.props_version = getattr(self, "props_version", 0) + 1
        if self._solver is not None:
            self._solver.update(self.K, self.M)
        return self

    @property
    def kappa(self):
        return 1.0 / (3.0 * (self.mua + self.musp))

    def add_optode(self, optode):
        """Snap optodes to the surface and link them (dMesh.m:91-96)."""
        self.optode = optode.snap2mesh(self)
        self._solver = None
        return self

    # ------------------------------------------------------------ solving
    def solver(self, ns_max=None):
        o = self.optode
        dfc = o.df / self.c                                                     # dMesh.m:1241
        ns_max = int(ns_max or max(o.s_bary.shape[0], o.d_bary.shape[0]))
        key = (o.Nf, ns_max, dfc)
        if self._solver is None or self._solver_key != key:
            self._solver = api.Solver(self.fem.rowptr, self.fem.col, self.K, self.M, dfc, o.Nf, ns_max)
            self._solver_key = key
        return self._solver

    def _sources(self, bary):
        bary = np.asarray(bary)
        nodes = torch.as_tensor(self.elem_host[bary[:, 0].astype(np.int64)].astype(np.int32), device="cuda")
        w = torch.as_tensor(np.ascontiguousarray(bary[:, 1:5]), device="cuda")
        return nodes.contiguous(), w.contiguous()

    def flu_solve(self, precision="fp64", tol=1e-12, maxit=1000, inner_tol=None, stop_rule=None,
                  check_every=None, return_report=False):
        """Fluence for every source x harmonic and the detector data (dMesh.m:106-141)."""
        nodes, w = self._sources(self.optode.s_bary)
        opts = api.make_opts(tol=tol, maxit=maxit, precision=precision, inner_tol=inner_tol, stop_rule=stop_rule,
                             check_every=check_every)
        phi, rep = self.solver().solve_sources(nodes, w, self.optode.s_fpsf.contiguous(), opts)
        data = self.meas_flu(phi)
        return (phi, data, rep) if return_report else (phi, data)

    def adj_flu_solve(self, precision="fp64", tol=1e-12, maxit=1000, inner_tol=None, return_report=False):
        """Adjoint fluence from every detector (dMesh.m:174-202): same A, Q from d_bary x s_fpsf."""
        nodes, w = self._sources(self.optode.d_bary)
        opts = api.make_opts(tol=tol, maxit=maxit, precision=precision, inner_tol=inner_tol)
        phiA, rep = self.solver().solve_sources(nodes, w, self.optode.s_fpsf.contiguous(), opts)
        return (phiA, rep) if return_report else phiA

    def meas_flu(self, phi):
        """Detector data [NM][NF] (dMesh.m:144-171)."""
        nodes, w = self._sources(self.optode.d_bary)
        link = torch.as_tensor(self.optode.link.astype(np.int32), device="cuda").contiguous()
        return api.meas(nodes, w, link, phi)

    # ------------------------------------------------------------ Jacobian
    def mesh2grid(self, x, y, z):
        """Voxel basis of the Jacobian (dMesh.m:286-380): m2g, g2m, gridinmesh, dxyz,
        with the voxel centres located on the device."""
        from .grid import mesh2grid
        g = mesh2grid(self.node_host, self.elem_host, np.asarray(x), np.asarray(y), np.asarray(z))
        self.grid, self.m2g, self.g2m = g["grid"], g["m2g"], g["g2m"]
        self.gridinmesh, self.dxyz, self.gridSize = g["gridinmesh"], g["dxyz"], g["size"]
        self.grid_basis = api.Basis(self.m2g, np.full(self.m2g.shape[0], self.dxyz ** 3))
        return self

    def nodal_basis(self):
        """Nodal basis: J per node weighted by the lumped mass sum_j M_ij."""
        rows = torch.repeat_interleave(torch.arange(self.nn, device="cuda"),
                                       (self.fem.rowptr[1:] - self.fem.rowptr[:-1]).long())
        lump = torch.zeros(self.nn, dtype=torch.float64, device="cuda").index_add_(0, rows, self.M)
        return api.Basis(None, lump, nn=self.nn)

    def _link(self):
        return torch.as_tensor(self.optode.link.astype(np.int32), device="cuda").contiguous()

    def J_complex(self, phi=None, phiA=None, basis=None, **solve_kw):
        """Complex absorption Jacobian J[v][k][m] (dMesh.m:206-247) plus data, phi, phiA."""
        if phiA is None:
            phiA = self.adj_flu_solve(**solve_kw)
        if phi is None:
            phi, _ = self.flu_solve(**solve_kw)
        data = self.meas_flu(phi)
        basis = basis or self.grid_basis
        J = api.jacobian_complex(basis, phi, phiA, self.optode.s_fpsf, self._link())
        return J, data, phi, phiA

    def J_tg(self, gate_fc, phi, phiA, basis=None, rytov=False):
        """Time-gated Jacobian J_tg[v][g][m] (fc2tg of J_complex), optionally / data_tg (Rytov)."""
        basis = basis or self.grid_basis
        nt = len(self.optode.tAxis)
        data_tg = api.fc2tg(self.meas_flu(phi), gate_fc, nt) if rytov else None
        return api.jacobian_tg(basis, phi, phiA, self.optode.s_fpsf, self._link(), gate_fc, nt, data_tg), data_tg


def to_reference_layout(phi: torch.Tensor) -> torch.Tensor:
    """[NF][NN][NS] -> the reference's [NN][NF][NS]."""
    return phi.permute(1, 0, 2)
