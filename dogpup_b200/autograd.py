"""Differentiable time-gated forward model on the device.

``TimeGatedForward(mesh, gate_fc)(mua, musp)`` returns the time-gated detector
data y[m][g] = fc2tg(meas_flu(phi))  (DOGPUP/dMesh.m:80-171 then
DOGPUP/fc2tg.m:25-32) as a torch tensor with a backward pass.  The reference
gets sensitivities from the explicit absorption Jacobian (J_complex,
dMesh.m:206-247, kappa held fixed); here backward is the adjoint method:
one batched solve of A_k lam = dL/dphi per source x harmonic (the same batch
shape as the forward solve), then one element kernel giving dL/dmua and
dL/dmusp exactly for the discrete model (kappa = 1/(3(mua + musp)) included).
The reference's kappa-fixed absorption sensitivity is grad_mua - grad_musp.
"""
from __future__ import annotations

import numpy as np
import torch

from . import api


class TimeGatedForward:
    def __init__(self, mesh, gate_fc, precision="fp64", tol=1e-12, maxit=1000, inner_tol=None, recompute=False):
        """recompute=True keeps no fields between forward and backward: backward solves phi again
        (one extra forward solve for NF x NN x NS x 16 bytes less memory held by the autograd graph)."""
        self.mesh = mesh
        self.recompute = bool(recompute)
        self.gate_fc = torch.as_tensor(gate_fc, device="cuda", dtype=torch.complex128).contiguous()
        self.nt = len(mesh.optode.tAxis)
        self.opts = api.make_opts(tol=tol, maxit=maxit, precision=precision, inner_tol=inner_tol)
        self.src = mesh._sources(mesh.optode.s_bary)
        self.det = mesh._sources(mesh.optode.d_bary)
        self.link = mesh._link()
        self.ns = int(self.src[0].shape[0])
        self.last_reports = []

    def _assemble(self, mua, musp):
        self.mesh.mua = mua.detach().to(device="cuda", dtype=torch.float64).contiguous()
        self.mesh.musp = musp.detach().to(device="cuda", dtype=torch.float64).contiguous()
        self.mesh.update_properties()
        return self.mesh.props_version

    def forward_fields(self, mua, musp):
        state = self._assemble(mua, musp)
        S = self.mesh.solver(ns_max=self.ns)
        phi, rep = S.solve_sources(*self.src, self.mesh.optode.s_fpsf.contiguous(), self.opts)
        data = api.meas(*self.det, self.link, phi)
        y = api.fc2tg(data, self.gate_fc, self.nt)
        self.last_reports = [rep]
        return y, phi, state

    def gradient(self, mua, musp, phi, state, gy):
        """(dL/dmua, dL/dmusp) for L = sum gy * y at the properties the fields were solved for."""
        if phi is None:
            _, phi, state = self.forward_fields(mua, musp)
        elif state != self.mesh.props_version:
            self._assemble(mua, musp)
        S = self.mesh.solver(ns_max=self.ns)
        nf, n, ns = phi.shape
        B = api.tg_adjoint_rhs(*self.det, self.link, self.gate_fc, self.nt, gy, n, nf, ns)
        lam, rep = S.solve(B, self.opts)
        self.last_reports.append(rep)
        return api.fem_adjoint_grad(self.mesh.fem, mua.detach(), musp.detach(), phi, lam)

    def __call__(self, mua: torch.Tensor, musp: torch.Tensor) -> torch.Tensor:
        return _TimeGated.apply(mua, musp, self)


class _TimeGated(torch.autograd.Function):
    @staticmethod
    def forward(ctx, mua, musp, model):
        y, phi, state = model.forward_fields(mua, musp)
        ctx.model, ctx.state = model, state
        ctx.phi = None if model.recompute else phi
        ctx.save_for_backward(mua, musp)
        return y

    @staticmethod
    def backward(ctx, gy):
        mua, musp = ctx.saved_tensors
        gmua, gmusp = ctx.model.gradient(mua, musp, ctx.phi, ctx.state, gy.contiguous())
        return (gmua.to(mua.dtype) if ctx.needs_input_grad[0] else None,
                gmusp.to(musp.dtype) if ctx.needs_input_grad[1] else None, None)


def gate_coefficients(t, centres, fwhm, f):
    """Fourier coefficients of Gaussian gates on the time axis (fc2tg.m gate input)."""
    from . import api as _api
    t = np.asarray(t)
    sd = fwhm / (2 * np.sqrt(2 * np.log(2)))
    gates = np.stack([np.exp(-((t - c) ** 2) / (2 * sd ** 2)) for c in centres])
    return _api.td2fc(torch.as_tensor(gates, device="cuda"), torch.as_tensor(f), torch.as_tensor(t))
