"""Weighted Levenberg-Marquardt reconstruction of nodal absorption on the device.

Restates wghtd_LM_recon (DOGPUP/reconstruction/wghtd_LM_recon.m:1-168) with
its helpers id_thresh (DOGPUP/id_thresh.m:1-27) and tik_inv
(DOGPUP/reconstruction/tik_inv.m:1-20), on the library's kernels:

  per iteration   forward + adjoint solves (batched, mixed or FP64)
                  TG Jacobian with Rytov normalisation (dgp_jacobian_tg)
                  H = J^T W J + lam * max diag, r = J^T W y (dgp_normal_eq,
                  split-BF16 tcgen05) and the FP64 Cholesky solve
                  (dgp_cholesky_solve), or all of it in FP64 for comparison
                  property normalisation G = m2g mua and the update map
                  d_mu = g2m (G x) by the library's CSR SpMV (dgp_csr_spmv)
  host            the loop's scalar logic (lambda schedule, step-back on a
                  rising error, exit conditions) on [NM x NG]-sized data

Data weighting: with target spots (``pos_s``) the rows of J and y are
mixed by reshape_J's dense w (wghtd_LM_recon.m:35-37, :72-76;
reconstruction/reshape_J.m:13-15; dMesh.m:250-282), computed on the device:
J J^T + lam2 max diag by the split-BF16 tensor-core kernel (dgp_normal_eq on
J), Js J^T by dgp_times_jt (FP64 accumulation), and w by one FP64 Cholesky
factorisation with one right-hand side per spot (dgp_cholesky_solve_many).  Without spots the
rows are weighted by a diagonal W = 1/sigma^2 or by 1.
"""
from __future__ import annotations

import ctypes as C
import warnings

import numpy as np
import torch

from . import api
from ._lib import lib, check


def id_thresh(data, thresh):
    """Mask of the gated data used by the fit (DOGPUP/id_thresh.m:13-27), data [NM x NG].

    'all': range-normalised value > 1 %.  A number t: on the falling edge
    (gate index >= the curve's maximum) with normalised value in (1 %, t]."""
    d = np.asarray(data, dtype=np.float64)
    lo = d.min(axis=1, keepdims=True)
    rng = d.max(axis=1, keepdims=True) - lo
    rng[rng == 0] = 1.0
    dn = (d - lo) / rng                                        # normalize(data, 2, 'range')
    if isinstance(thresh, str):
        if thresh != "all":
            raise ValueError("thresh must be a number or 'all'")
        return dn > 0.01
    idx = np.arange(d.shape[1])[None, :]
    after = idx >= np.argmax(dn, axis=1)[:, None]
    return after & (dn <= thresh) & (dn > 0.01)


def target_spots(grid, inmesh, pos, w=1.5, kind="gauss"):
    """Sensitivity spots Js [NS][NV] on the device (dMesh.m:250-282): a Gaussian of width
    parameter 2 sqrt(2 ln 2) w ('gauss', w the FWHM) or a cube of side w ('square') around
    each centre pos [NS][3], normalised to unit sum over all voxels, negated, zero outside
    the mesh."""
    g = torch.as_tensor(np.asarray(grid, dtype=np.float64), device="cuda")
    p = torch.as_tensor(np.atleast_2d(np.asarray(pos, dtype=np.float64)), device="cuda")
    diff = g[None, :, :] - p[:, None, :]                               # [NS][NV][3]
    if kind == "gauss":
        s = 2.0 * np.sqrt(2.0 * np.log(2.0)) * w
        t = torch.exp(-(diff * diff).sum(-1) / (s * s * 2))
    elif kind == "square":
        t = (diff.abs() <= w / 2).all(-1).to(torch.float64)
    else:
        raise ValueError("spot type must be 'gauss' or 'square'")
    tot = t.sum(1, keepdim=True)
    if bool((tot == 0).any()):
        raise ValueError("a target spot covers no voxel")
    t = -(t / tot)
    t[:, ~torch.as_tensor(np.asarray(inmesh, dtype=bool), device="cuda")] = 0.0
    return t


def reshape_J(Jt: torch.Tensor, Js: torch.Tensor, lam: float, normal_eq="split_bf16") -> torch.Tensor:
    """w [NS][NM] = (Js J^T)(J J^T + lam max diag I)^-1 (reconstruction/reshape_J.m:13-15).

    Jt [NV][NM] is J transposed (the TG Jacobian's layout), Js [NS][NV] the spots on the
    same voxels.  J J^T: split-BF16 tensor cores (or FP64 for normal_eq='fp64', the all-FP64
    cross-check mode, with torch matrix products); the solve: FP64 Cholesky with one
    right-hand side per spot."""
    nv, nm = Jt.shape
    ns = Js.shape[0]
    A = torch.empty((nm, nm), dtype=torch.float64, device="cuda")
    v = lambda t: C.c_void_p(t.data_ptr())
    if normal_eq == "split_bf16":
        Jf = Jt.to(torch.float32).contiguous()
        J = Jf.t().contiguous()                                           # [NM][NV]: rows of J
        check(lib.dgp_normal_eq(v(J), nm, nv, None, None, float(lam), 0, v(A), nm, None, api.stream_ptr()))
        Jsd = Js.to(torch.float64).contiguous()
        B = torch.empty((ns, nm), dtype=torch.float64, device="cuda")
        check(lib.dgp_times_jt(v(Jsd), ns, nv, v(Jf), nm, v(B), api.stream_ptr()))     # Js J^T
    else:
        Jd = Jt.to(torch.float64)
        A.copy_(Jd.T @ Jd)
        A.diagonal().add_(lam * A.diagonal().max())
        B = (Js.to(torch.float64) @ Jd).contiguous()
    check(lib.dgp_cholesky_solve_many(v(A), nm, nm, v(B), ns, nm, api.stream_ptr()))
    return B


def _flat(x_nm_ng: torch.Tensor) -> torch.Tensor:
    """[NM][NG] -> MATLAB's x(:) order (measurement fastest): index g*NM + m."""
    return x_nm_ng.transpose(0, 1).reshape(-1)


class LMRecon:
    """wghtd_LM_recon on a DMesh with a voxel basis (mesh.mesh2grid called beforehand)."""

    def __init__(self, mesh, gate_fc, precision="mixed", tol=1e-8, normal_eq="split_bf16"):
        if normal_eq not in ("split_bf16", "fp64"):
            raise ValueError("normal_eq must be 'split_bf16' or 'fp64'")
        self.mesh = mesh
        self.gate_fc = torch.as_tensor(gate_fc, device="cuda", dtype=torch.complex128).contiguous()
        self.nt = len(mesh.optode.tAxis)
        self.solve_kw = dict(precision=precision, tol=tol)
        self.normal_eq = normal_eq
        inmesh = np.asarray(mesh.gridinmesh)
        P = mesh.m2g[inmesh]
        self.basis = api.Basis(P, np.full(P.shape[0], mesh.dxyz ** 3))
        self.m2g_in = api.DeviceCsr(P)                                  # in-mesh voxels x nodes
        self.g2m_in = api.DeviceCsr(mesh.g2m[:, np.nonzero(inmesh)[0]])   # nodes x in-mesh voxels
        self.nv = P.shape[0]

    # ----------------------------------------------------------- one model
    def model(self):
        """Time-gated data [NM][NG] and the Rytov-normalised TG Jacobian^T [NV][NG*NM]."""
        m = self.mesh
        phi, data = m.flu_solve(**self.solve_kw)
        phiA = m.adj_flu_solve(**self.solve_kw)
        data_tg = api.fc2tg(data, self.gate_fc, self.nt)
        if self.normal_eq == "split_bf16":
            J = api.jacobian_tg(self.basis, phi, phiA, m.optode.s_fpsf, m._link(), self.gate_fc, self.nt, data_tg)
            Jt = J.reshape(self.nv, -1)
        else:
            Jc = api.jacobian_complex(self.basis, phi, phiA, m.optode.s_fpsf, m._link())   # [NV][NF][NM]
            Jc[:, 0, :] *= 0.5
            Jtg = self.nt * 2.0 * torch.einsum("gk,vkm->vgm", self.gate_fc.conj(), Jc).real   # fc2tg.m:25-32
            del Jc
            Jt = (Jtg / data_tg.transpose(0, 1)[None]).reshape(self.nv, -1)
        return data_tg, Jt

    # --------------------------------------------------------------- step
    def _tik(self, Jt, lam, y, w):
        """update = (J^T W J + lam * max diag)^-1 J^T W y  (tik_inv.m:13-20)."""
        nv = Jt.shape[0]
        if self.normal_eq == "split_bf16":
            # split-BF16 Gram + FP64 Cholesky of the smaller of the two equivalent systems
            Jf = Jt.to(torch.float32).contiguous()
            x = torch.empty(nv, dtype=torch.float64, device="cuda")
            v = lambda t: C.c_void_p(t.data_ptr())
            check(lib.dgp_lm_update(v(Jf), nv, Jf.shape[1], None if w is None else v(w), v(y), float(lam), v(x), 0,
                                    None, api.stream_ptr()))
            return x
        else:
            Jd = Jt.to(torch.float64)
            Jw = Jd if w is None else Jd * w[None, :]
            H = Jw @ Jd.T
            H.diagonal().add_(lam * H.diagonal().max())
            x = Jw @ y
            H = H.contiguous()
        check(lib.dgp_cholesky_solve(C.c_void_p(H.data_ptr()), nv, nv, C.c_void_p(x.data_ptr()), api.stream_ptr()))
        return x

    def run(self, data_m, lam=(1.0, 0.0), sigma=None, thresh=0.8, max_iter=10, truth=None, callback=None,
            pos_s=None, spot_width=1.5, spot_kind="gauss"):
        """Iterates from the mesh's current mua (wghtd_LM_recon.m:25-168); data_m [NM][NG] measured TG data.

        pos_s [NS][3] (or None): centres of the target spots; J and y are then mixed by
        reshape_J's w with regulariser lam[1] at every iteration (wghtd_LM_recon.m:72-76),
        and the misfit is |w y| relative to |w data| (:84-85).

        sigma [NM][NG] (or None): data standard deviations; the fit is on log
        data, so W = (data / sigma)^2 to first order, scaled to unit mean over
        the fitted gates: the reference's damping rule floors lambda at the
        residual norm (wghtd_LM_recon.m:118-120), which keeps its meaning only
        when the weighted norm is on the scale of the unweighted one.
        Returns a history dict; its "exit" names the rule that ended the loop:
        "converged" (:91-95), "max_iter" (:158-161), "nan_update" (:136-141) or
        "negative_mua" (:146-152; both warn and leave mua at the last accepted
        update, as the reference does), or "model_data" (a model gate without a
        logarithm, also recorded under "stopped")."""
        m = self.mesh
        data_m = np.asarray(data_m, dtype=np.float64)
        # gates in the id_thresh window whose measured value has a logarithm (a truncated Fourier
        # series can ring below zero before the pulse arrives; log() of those is undefined)
        mask = id_thresh(data_m, thresh) & (data_m > 0)
        incl = torch.as_tensor(np.nonzero(mask.T.ravel())[0], device="cuda")               # x(:) order
        dm = torch.log(_flat(torch.as_tensor(data_m, device="cuda")))[incl]
        w = None
        Js = None
        if pos_s is not None:
            if sigma is not None:
                raise ValueError("pos_s (reshaping weights) and sigma (diagonal weights) exclude each other")
            inmesh = np.asarray(m.gridinmesh)
            Js = target_spots(m.grid, inmesh, pos_s, spot_width, spot_kind)[:, torch.as_tensor(inmesh, device="cuda")]
            Js = Js.contiguous()
        if sigma is not None:
            rel = np.asarray(sigma, dtype=np.float64) / data_m        # sigma of log data
            w = (1.0 / _flat(torch.as_tensor(rel, device="cuda")) ** 2)[incl]
            w = (w / w.mean()).contiguous()
        k = 10 ** 0.25
        lam1 = lam[0] * k                                             # :38-39
        hist = dict(err=[], err_perc=[], err_del=[], lam=[], mua=[], err_truth=[])
        wn = torch.ones_like(dm) if w is None else w
        count, d_mu, y_prev, J_prev = 0, None, None, None
        while True:
            data_c, Jt = self.model()
            Jt = Jt[:, incl] if incl.numel() != Jt.shape[1] else Jt
            y = dm - torch.log(_flat(data_c))[incl]                   # :60-64
            if not bool(torch.isfinite(y).all()):
                hist["stopped"] = "model data not positive on an included gate"
                hist["exit"] = "model_data"
                break
            if Js is not None:                                        # :72-76
                ws = reshape_J(Jt, Js, lam[1], self.normal_eq)        # [NS][NM]
                Jt = (Jt @ ws.T.to(Jt.dtype)).contiguous()             # rows of w J, transposed
                y = ws @ y
                err = float(torch.linalg.vector_norm(y))
                ref = float(torch.linalg.vector_norm(ws @ dm))
            else:
                err = float(torch.sqrt((wn * y * y).sum()))
                ref = float(torch.sqrt((wn * dm * dm).sum()))
            hist["err"].append(err)
            hist["err_perc"].append(100 * err / ref)
            if truth is not None:
                hist["err_truth"].append(float(torch.linalg.vector_norm(m.mua - truth) /
                                               torch.linalg.vector_norm(truth)))
            if count > 0:
                hist["err_del"].append(hist["err_perc"][-1] - hist["err_perc"][-2])
            if callback:
                callback(count, hist)
            if count > 1 and hist["err_del"][-1] < 0 and (abs(hist["err_del"][-1]) < 0.12 or
                                                           hist["err_perc"][-1] < 1.5):      # :91-95
                hist["exit"] = "converged"
                break
            count += 1
            if count == 1 or hist["err_del"][-1] < 0:                 # :100-106
                G = self.m2g_in @ m.mua
                Jt = (Jt * G[:, None].to(Jt.dtype)).contiguous()      # J .* G.' (property normalisation)
                lam1 = lam1 / k
            else:                                                     # step back (:107-115)
                # the cached J is used as cached, normalised by the G of its own iteration;
                # the new G only rescales the update
                G = self.m2g_in @ (m.mua - d_mu)
                y, Jt = y_prev, J_prev
                lam1 = lam1 * k
            lam1 = max(lam1, err)                                     # :118-120
            hist["lam"].append(lam1)
            upd = self._tik(Jt, lam1, y.contiguous(), None if Js is not None else w)   # :125-127
            x = G * upd                                               # :131
            d_mu = self.g2m_in @ x                                    # :132
            if torch.isnan(d_mu).any():                               # :136-141
                hist["exit"] = "nan_update"
                warnings.warn("LM: NaN absorption update, stopping the reconstruction")
                break
            new_mu = m.mua + d_mu
            if (new_mu < 0).any():                                    # :146-152: the update is not applied
                hist["exit"] = "negative_mua"
                warnings.warn("LM: negative absorption update, stopping the reconstruction")
                break
            m.mua = new_mu.contiguous()
            m.update_properties()                                     # :153
            hist["mua"].append(m.mua.clone())
            if count > max_iter - 1:
                hist["exit"] = "max_iter"
                break
            y_prev, J_prev = y, Jt
        hist["iterations"] = count
        return hist
