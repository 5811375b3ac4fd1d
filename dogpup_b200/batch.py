"""Uneven batches: many meshes of different sizes, source and harmonic counts on one GPU.

The reference solves one mesh at a time (flu_solve per dMesh object,
DOGPUP/dMesh.m:106-141).  Here a batch of forward (and optional time-gated
vjp) problems is cut into tasks and run concurrently:

* every problem's harmonics are split into contiguous chunks so that one
  chunk's solver plan (FP32 workspace, FP64 output, FSAI factors) fits a
  memory budget -- a 300k-node mesh with 64 sources x 128 harmonics needs
  ~240 GB in one piece, more than the GPU holds;
* tasks run longest-first on ``streams`` worker threads, each with its own
  CUDA stream, so small meshes fill the SMs beside large ones (every
  library call enqueues on the caller's stream and waits only on it);
* per task: a solver plan for the chunk's harmonics
  (``dgp_solver_create_harmonics``), the point-source solve, detector data;
  with gates, also the adjoint solve and the TG Jacobian's vjp, whose sum
  over harmonics is accumulated across the chunks (fc2tg is linear in the
  coefficients; the DC term is halved only in the chunk that holds k = 0).

Results are the same as solving each problem alone (each column's
iteration is independent of the batch; the stop rule is per chunk).
"""
from __future__ import annotations

import threading
from dataclasses import dataclass, field

import numpy as np
import torch

from . import api


def plan_bytes(n: int, nnz: int, nnzG: int, nf: int, ns: int) -> int:
    """Device bytes of one mixed-precision solver plan + its FP64 output (upper estimate)."""
    nsp = 2
    while nsp < ns:
        nsp *= 2
    vec32 = 10 * 8 * nf * n * nsp           # complex-FP32 workspace vectors
    out64 = 16 * nf * n * ns                # FP64 solution
    fsai = (2 * 16 + 2 * 16) * nnzG * nf    # G, G^T in FP64 and FP32 records
    mat = 16 * nnz * 2 + 8 * (n + 1)
    return int(1.15 * (vec32 + out64 + fsai + mat))


def harmonic_chunks(nf: int, n: int, nnz: int, nnzG: int, ns: int, budget: int) -> list[list[int]]:
    """Contiguous harmonic ranges whose plans fit ``budget`` bytes (at least one harmonic each)."""
    per = max(1, plan_bytes(n, nnz, nnzG, 1, ns))
    size = max(1, min(nf, budget // per))
    # balance: equal chunk sizes
    nchunk = -(-nf // size)
    size = -(-nf // nchunk)
    return [list(range(k0, min(nf, k0 + size))) for k0 in range(0, nf, size)]


@dataclass
class Task:
    problem: int
    harmonics: list[int]
    cost: float


@dataclass
class Result:
    data: torch.Tensor                       # [NM][NF] complex128 detector data
    vjp: torch.Tensor | None = None          # [NN] J_tg^T g
    iterations: list[int] = field(default_factory=list)


class UnevenBatch:
    def __init__(self, meshes, budget_bytes: int | None = None, streams: int = 4, precision="mixed", tol=1e-8,
                 gates=None, upstream=None):
        """meshes: DMesh objects with optodes; gates[i]: gate_fc [NG][NF_i] (complex) or None;
        upstream[i]: g [NM_i][NG] for the vjp.  budget_bytes: device memory for the plans in
        flight (default: 70 % of the free memory)."""
        self.meshes = list(meshes)
        free = torch.cuda.mem_get_info()[0]
        self.budget = int(budget_bytes or 0.7 * free)
        self.streams = max(1, int(streams))
        self.opts = dict(precision=precision, tol=tol)
        self.gates = gates
        self.upstream = upstream
        self.tasks = self._plan()

    def _plan(self):
        tasks = []
        per_stream = self.budget // self.streams
        for i, m in enumerate(self.meshes):
            o = m.optode
            ns = max(o.s_bary.shape[0], o.d_bary.shape[0])
            nnz = m.fem.nnz
            for ch in harmonic_chunks(o.Nf, m.nn, nnz, nnz // 2 + m.nn, ns, per_stream):
                cost = float(m.nn) * ns * len(ch) * (1.0 + np.mean(ch) / max(1, o.Nf))
                tasks.append(Task(i, ch, cost))
        tasks.sort(key=lambda t: -t.cost)            # longest first
        return tasks

    def _run_task(self, t: Task, results, lock):
        m = self.meshes[t.problem]
        o = m.optode
        ch = t.harmonics
        ns = max(o.s_bary.shape[0], o.d_bary.shape[0])
        S = api.Solver(m.fem.rowptr, m.fem.col, m.K, m.M, o.df / m.c, len(ch), ns, harmonics=ch)
        opts = api.make_opts(**self.opts)
        fpsf = o.s_fpsf[ch].contiguous()
        src = m._sources(o.s_bary)
        det = m._sources(o.d_bary)
        phi, rep = S.solve_sources(*src, fpsf, opts)
        data = api.meas(*det, m._link(), phi)
        vjp = None
        its = [rep.iterations]
        if self.gates is not None and self.gates[t.problem] is not None:
            phiA, repA = S.solve_sources(*det, fpsf, opts)
            its.append(repA.iterations)
            g = torch.as_tensor(self.gates[t.problem], device="cuda", dtype=torch.complex128)[:, ch].contiguous()
            if ch[0] != 0:
                g[:, 0] *= 2.0                      # the kernel halves slot 0; only harmonic 0 is the DC term
            gin = torch.as_tensor(self.upstream[t.problem], device="cuda", dtype=torch.float64)
            vjp = api.jacobian_tg_vjp(m.nodal_basis(), phi, phiA, fpsf, m._link(), g, len(o.tAxis), gin)
        torch.cuda.current_stream().synchronize()
        del S
        with lock:
            r = results[t.problem]
            r.data[:, ch] = data
            r.iterations.extend(its)
            if vjp is not None:
                r.vjp = vjp if r.vjp is None else r.vjp + vjp

    def run(self) -> list[Result]:
        results = []
        for m in self.meshes:
            nm = m.optode.link.shape[0]
            results.append(Result(torch.zeros((nm, m.optode.Nf), dtype=torch.complex128, device="cuda")))
        lock = threading.Lock()
        queue = list(self.tasks)
        qlock = threading.Lock()
        errors = []
        dev = torch.cuda.current_device()

        def worker():
            torch.cuda.set_device(dev)
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                while True:
                    with qlock:
                        if not queue or errors:
                            return
                        t = queue.pop(0)
                    try:
                        self._run_task(t, results, lock)
                    except Exception as e:  # surfaced after the join
                        errors.append(e)
                        return

        threads = [threading.Thread(target=worker) for _ in range(self.streams)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        torch.cuda.synchronize()
        if errors:
            raise errors[0]
        return results
