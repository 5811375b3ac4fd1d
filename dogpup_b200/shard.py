"""Harmonic sharding of one mesh's solves over ranks (one process per GPU).

The forward and adjoint solves of different harmonics are independent
(A_k = K + i*k*dfc*M, one FSAI factor per k), so rank r of W owns the
harmonics k = r, r+W, r+2W, ... (interleaved: iteration counts fall with k,
so contiguous blocks would leave the rank with the low harmonics the slowest).
Nothing about the solves is exchanged.  The exchanges are the sums over
harmonics of the time-gate transform (fc2tg.m:25-32):

  data      each rank gates its own harmonics' detector data and one
            all-reduce of the [NM x NG] partial sums gives the time-gated data
            on every rank;
  Jacobian  each rank forms the TG Jacobian of its own harmonics [NV][NG][NM]
            (FP32) and one reduce-scatter over voxels leaves rank r the summed
            rows of voxel block r (the voxel count padded to a multiple of W);
  spectra   the detector data of every harmonic [NM x NF] when wanted, by one
            all-gather of the ranks' column blocks.

Fields and solver state never leave their GPU.  A rank whose share is empty
(W > NF) solves nothing and contributes zeros, so every rank still takes part
in every collective in the same order.  Under a gloo process group (CPU
collectives, used by the tests) device tensors are staged through host memory.
"""
from __future__ import annotations

import numpy as np


def harmonic_shard(nf: int, rank: int, world: int) -> list[int]:
    if not (0 <= rank < world):
        raise ValueError("rank out of range")
    return list(range(rank, nf, world))


def partial_tg(coef, harmonics, gate_fc, nt, fc2tg):
    """This rank's share of fc2tg: coef [NM][len(harmonics)] holds the
    coefficients of ``harmonics``; gate_fc [NG][NF] is the full gate table.
    fc2tg halves the coefficient in column 0 (the DC term); column 0 of a
    shard is harmonic ``harmonics[0]``, which is the DC term only on the rank
    that owns k = 0, so the halving is undone elsewhere.  An empty share
    contributes zeros [NM][NG]."""
    if not harmonics:
        nm, ng = coef.shape[0], gate_fc.shape[0]
        if hasattr(gate_fc, "new_zeros"):
            return gate_fc.real.new_zeros((nm, ng))
        return np.zeros((nm, ng))
    g = gate_fc[:, list(harmonics)]
    if harmonics[0] != 0:
        coef = coef.clone() if hasattr(coef, "clone") else np.array(coef, copy=True)
        coef[..., 0] = coef[..., 0] * 2
    return fc2tg(coef, g, nt)


def _collective(fn, t, group=None):
    """Runs the in-place collective fn(tensor) on t; under a gloo group a device tensor is
    staged through host memory.  Returns the tensor holding the result."""
    import torch.distributed as dist
    if t.is_cuda and dist.get_backend(group) == "gloo":
        h = t.cpu()
        fn(h)
        t.copy_(h)
        return t
    fn(t)
    return t


def sharded_tg_data(coef, harmonics, gate_fc, nt, fc2tg, group=None):
    """Time-gated data summed over the ranks of ``group`` (torch.distributed all-reduce)."""
    import torch
    import torch.distributed as dist
    y = partial_tg(coef, harmonics, gate_fc, nt, fc2tg)
    y = y if isinstance(y, torch.Tensor) else torch.as_tensor(y)
    if dist.is_available() and dist.is_initialized():
        y = _collective(lambda t: dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group), y, group)
    return y


def gather_spectra(data, nf, rank, world, group=None):
    """[NM x NF] detector data from every rank's [NM x len(own harmonics)] block (one
    all-gather of real views; blocks padded to ceil(NF / W) columns)."""
    import torch
    import torch.distributed as dist
    nm = data.shape[0]
    width = -(-nf // world)
    block = torch.zeros((width, nm, 2), dtype=torch.float64, device=data.device)
    own = harmonic_shard(nf, rank, world)
    if own:
        block[:len(own)] = torch.view_as_real(data.transpose(0, 1).contiguous())
    if block.is_cuda and dist.get_backend(group) == "gloo":
        hp = [torch.empty_like(block, device="cpu") for _ in range(world)]
        dist.all_gather(hp, block.cpu(), group=group)
        parts = [p.to(block.device) for p in hp]
    else:
        parts = [torch.empty_like(block) for _ in range(world)]
        dist.all_gather(parts, block, group=group)
    out = torch.empty((nm, nf), dtype=torch.complex128, device=data.device)
    for r in range(world):
        ks = harmonic_shard(nf, r, world)
        if ks:
            out[:, ks] = torch.view_as_complex(parts[r][:len(ks)].contiguous()).transpose(0, 1)
    return out


class ShardedForward:
    """flu_solve + meas_flu + fc2tg for this rank's harmonics of one DMesh (device path)."""

    def __init__(self, mesh, gate_fc, rank, world, precision="mixed", tol=1e-8, group=None, inner_tol=None,
                 ns_max=None):
        import torch
        from . import api
        self.mesh, self.group, self.rank, self.world = mesh, group, rank, world
        o = mesh.optode
        self.nf = o.Nf
        self.harm = harmonic_shard(o.Nf, rank, world)
        self.gate_fc = torch.as_tensor(gate_fc, device="cuda", dtype=torch.complex128)
        self.nt = len(o.tAxis)
        self.src = mesh._sources(o.s_bary)
        self.det = mesh._sources(o.d_bary)
        self.link = mesh._link()
        ns = int(ns_max or self.src[0].shape[0])
        self.solver = None
        if self.harm:
            self.solver = api.Solver(mesh.fem.rowptr, mesh.fem.col, mesh.K, mesh.M, o.df / mesh.c, len(self.harm),
                                     ns, harmonics=self.harm)
        self.fpsf = o.s_fpsf[self.harm].contiguous() if self.harm else None
        self.opts = api.make_opts(tol=tol, precision=precision, inner_tol=inner_tol)

    def update(self):
        """Re-factor after mesh.update_properties() (new K, M)."""
        if self.solver is not None:
            self.solver.update(self.mesh.K, self.mesh.M)

    def solve(self):
        """(phi [own NF][NN][NS] or None, detector data [NM][own NF], report or None)."""
        import torch
        from . import api
        if self.solver is None:
            return None, torch.zeros((int(self.link.shape[0]), 0), dtype=torch.complex128, device="cuda"), None
        phi, rep = self.solver.solve_sources(*self.src, self.fpsf, self.opts)
        return phi, api.meas(*self.det, self.link, phi), rep

    def __call__(self):
        from . import api
        _, data, rep = self.solve()
        return sharded_tg_data(data, self.harm, self.gate_fc, self.nt, api.fc2tg, self.group), rep


class ShardedSensitivity(ShardedForward):
    """Forward + adjoint solves of this rank's harmonics and the TG Jacobian summed over
    all harmonics, reduce-scattered over voxels: rank r returns voxel rows
    [r * NVp / W, (r + 1) * NVp / W) of J_tg [NVp][NG][NM] (NVp = NV padded to a multiple
    of W; padded rows are zero), Rytov-normalised by the full time-gated data when
    ``rytov``."""

    def __init__(self, mesh, gate_fc, rank, world, **kw):
        o = mesh.optode
        super().__init__(mesh, gate_fc, rank, world, ns_max=max(len(o.s_bary), len(o.d_bary)), **kw)

    def __call__(self, basis, rytov=False):
        import torch
        import torch.distributed as dist
        from . import api
        phi, data, rep = self.solve()
        data_tg = sharded_tg_data(data, self.harm, self.gate_fc, self.nt, api.fc2tg, self.group)
        nv, ng, nm = basis.nv, self.gate_fc.shape[0], int(self.link.shape[0])
        nvp = -(-nv // self.world) * self.world
        Jp = torch.zeros((nvp, ng, nm), dtype=torch.float32, device="cuda")
        if self.solver is not None:
            phiA, _ = self.solver.solve_sources(*self.det, self.fpsf, self.opts)
            g = self.gate_fc[:, self.harm].clone()
            if self.harm[0] != 0:
                g[:, 0] *= 2          # the kernel halves its first column (the DC term only on rank 0)
            Jp[:nv] = api.jacobian_tg(basis, phi, phiA, self.mesh.optode.s_fpsf[self.harm].contiguous(), self.link,
                                      g, self.nt, data_tg if rytov else None)
            del phiA
        out = torch.empty((nvp // self.world, ng, nm), dtype=torch.float32, device="cuda")
        if dist.get_backend(self.group) == "gloo":
            # gloo has no reduce-scatter: all-reduce on the host, keep this rank's block
            h = Jp.cpu()
            dist.all_reduce(h, op=dist.ReduceOp.SUM, group=self.group)
            out.copy_(h[self.rank * out.shape[0]:(self.rank + 1) * out.shape[0]])
        else:
            dist.reduce_scatter_tensor(out, Jp, op=dist.ReduceOp.SUM, group=self.group)
        return out, data_tg, rep
