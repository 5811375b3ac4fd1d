"""Optode set-up: source spectrum, surface snapping, barycentric weights.

Mirrors the ``dOptode`` class (DOGPUP/dOptode.m:34-199).  The Fourier
coefficients of the source pulse come from the device ``td2fc`` kernel; the
geometry (nearest surface point, containing tetrahedron) runs on the device
(``dgp_snap_to_surface``, ``dgp_locate_points``).
"""
from __future__ import annotations

import numpy as np
import torch

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

    def snap2mesh(self, mesh):
        """Snap optodes to the surface, move sources 1/min(musp) inward (dOptode.m:77-97):
        surface search (``dgp_snap_to_surface``) and point location (``dgp_locate_points``)
        on the GPU."""
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
