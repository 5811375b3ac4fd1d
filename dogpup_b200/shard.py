"""Harmonic sharding of one mesh's solves over ranks (one process per GPU).

The forward and adjoint solves of different harmonics are independent
(A_k = K + i*k*dfc*M, one FSAI factor per k), so rank r of W owns the
harmonics k = r, r+W, r+2W, ... (interleaved: iteration counts grow with k,
so contiguous blocks would leave the last rank the slowest).  The only
exchange is the time-gate transform, which sums over harmonics
(fc2tg.m:100-111): each rank gates its own harmonics and one all-reduce of
the [NM x NG] partial sums gives the time-gated data.  Fields and solver
state never leave their GPU.
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
    that owns k = 0, so the halving is undone elsewhere."""
    g = gate_fc[:, list(harmonics)]
    if harmonics and harmonics[0] != 0:
        coef = coef.clone() if hasattr(coef, "clone") else np.array(coef, copy=True)
        coef[..., 0] = coef[..., 0] * 2
    return fc2tg(coef, g, nt)


def sharded_tg_data(coef, harmonics, gate_fc, nt, fc2tg, group=None):
    """Time-gated data summed over the ranks of ``group`` (torch.distributed all-reduce)."""
    import torch
    import torch.distributed as dist
    y = partial_tg(coef, harmonics, gate_fc, nt, fc2tg)
    y = y if isinstance(y, torch.Tensor) else torch.as_tensor(y)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(y, op=dist.ReduceOp.SUM, group=group)
    return y


class ShardedForward:
    """flu_solve + meas_flu + fc2tg for this rank's harmonics of one DMesh (device path)."""

    def __init__(self, mesh, gate_fc, rank, world, precision="mixed", tol=1e-8, group=None):
        import torch
        from . import api
        self.mesh, self.group = mesh, group
        o = mesh.optode
        self.harm = harmonic_shard(o.Nf, rank, world)
        self.gate_fc = torch.as_tensor(gate_fc, device="cuda", dtype=torch.complex128)
        self.nt = len(o.tAxis)
        self.src = mesh._sources(o.s_bary)
        self.det = mesh._sources(o.d_bary)
        ns = int(self.src[0].shape[0])
        self.solver = api.Solver(mesh.fem.rowptr, mesh.fem.col, mesh.K, mesh.M, o.df / mesh.c, len(self.harm), ns,
                                 harmonics=self.harm)
        self.fpsf = o.s_fpsf[self.harm].contiguous()
        self.opts = api.make_opts(tol=tol, precision=precision)

    def __call__(self):
        from . import api
        phi, rep = self.solver.solve_sources(*self.src, self.fpsf, self.opts)
        data = api.meas(*self.det, self.mesh._link(), phi)          # [NM][own harmonics]
        return sharded_tg_data(data, self.harm, self.gate_fc, self.nt, api.fc2tg, self.group), rep
