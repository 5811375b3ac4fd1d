#!/usr/bin/env python
"""Benchmark of the DOGPUP forward hot path on B200: src.freq FEM solves/s.

Workload (default ``ellipsoid``): ellipsoid head phantom 90x75x70 mm on a
1.2 mm lattice (6 tets per cube, interior nodes jittered 0.2 mm, seeded),
mua = 0.01/mm (1 + 0.2 * smooth Gaussian random field), musp' = 1/mm,
n = 1.4, 64 point sources x 128 harmonics (T = 10 ns), complex-FP32
BiCGSTAB with FP64 iterative refinement to a max relative residual of 1e-8.

One step = device re-assembly of K, M + FSAI factors for all 128 harmonics
+ the batched solve of all 8192 right-hand sides + detector read-out.
Inputs are synthetic (no dataset).  Vectors are ~10 GB each, far larger than
L2, so no flush is needed between iterations.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) every rank solves its own copy of the workload on its
GPU (independent replicas, no data-path collective; weak scaling) and the
step time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ellipsoid", choices=["ellipsoid", "medium", "cylinder", "small"])
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--inner-tol", type=float, default=1e-4)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def log(msg):
    print(msg, file=sys.stderr, flush=True)


def workload(name, seed=1):
    from dogpup_b200 import workloads
    if name == "medium":  # same shape family at a coarser lattice: 19k nodes, 64 x 32 RHS (profiling case)
        return workloads.ellipsoid_fwd(seed=seed, h=2.4, nf=32)
    return {"ellipsoid": workloads.ellipsoid_fwd, "cylinder": workloads.cylinder_fwd,
            "small": workloads.small_fwd}[name](seed=seed)


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling during the timed region (read-only queries)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait(timeout=10)
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------- CPU baseline
def cpu_sample(w, harmonics=(1, 64), ns=8, tol=1e-8):
    """FP64 oracle (the reference algorithm restated: FSAI + BiCGSTAB of
    dMesh.m:1247-1385) on a bounded sample of the workload: ``ns`` sources x
    the given harmonics, on the same mesh and properties.  Assembly is timed
    separately and amortised over the workload's NS*NF right-hand sides."""
    import scipy.sparse as sp
    from oracle import fem, solver
    from dogpup_b200.optode import locate_points
    m = w["mesh"]
    t0 = time.perf_counter()
    geo = fem.prepare_mesh(m.node, m.elem, w["nr"])
    K, M = fem.gen_fwdmat(m.node, m.elem, geo, w["mua"], w["musp"])
    t_asm = time.perf_counter() - t0
    T = w["t"][-1]
    df = 2 * np.pi / T
    dfc = df / geo["c"]
    eid, bw = locate_points(m.node, m.elem, w["src"][:ns] * 0.97)
    nodes = m.elem[eid]
    t1 = time.perf_counter()
    solved = 0
    for k in harmonics:
        A = (K + 1j * k * dfc * M).tocsr()
        At = sp.tril(A).tocsr()
        rg, cg = solver.fsai_pattern(sp.tril(K + 1j * dfc * M).tocsr())
        G = solver.fsai_factor(sp.tril(K).tocsr(), sp.tril(k * dfc * M).tocsr(), rg, cg, 2)[:, 1:2]
        pc = solver.FsaiPrecond.__new__(solver.FsaiPrecond)
        pc.n = K.shape[0]
        pc.K, pc.Mi = K, (k * dfc * M).tocsr()
        pc.rptrG, pc.colsG, pc.G = rg, cg, G
        pc.rptrT, pc.colsT, perm = solver.transpose_pattern(rg, cg, pc.n)
        pc.GT = G[perm]
        pc.fAxis = np.array([1.0])
        Q = np.zeros((pc.n, ns, 1), complex)
        for s in range(ns):
            Q[nodes[s], s, 0] = bw[s]
        solver.bicgstab_fsai(pc, Q, tol, 1000)
        solved += ns
        del At
    t_solve = time.perf_counter() - t1
    per = t_solve / solved + t_asm / (len(w["src"]) * w["nf"])
    return {"value": 1.0 / per, "unit": "src.freq solves/s", "cores": 1, "kind": "port",
            "sample": f"FP64 oracle (numpy/scipy, 1 thread): {ns} sources x harmonics {list(harmonics)} "
                      f"to tol {tol:g} on the full mesh ({m.nn} nodes); assembly {t_asm:.1f}s amortised over "
                      f"{len(w['src']) * w['nf']} RHS", "seconds": t_asm + t_solve}


# --------------------------------------------------------------- our arm
def run_ours(a, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    from dogpup_b200 import workloads
    torch.cuda.set_device(local_rank)
    w = workload(a.workload, seed=1 + rank)
    mesh = workloads.build_dmesh(w)
    ns, nf = len(w["src"]), w["nf"]
    solver = mesh.solver()
    st = torch.cuda.current_stream()
    res = {}

    def step():
        mesh.update_properties()                         # K, M re-assembly + FSAI refactor
        phi, data, rep = mesh.flu_solve(precision="mixed", tol=a.tol, inner_tol=a.inner_tol, return_report=True)
        return rep

    log(f"[rank {rank}] setup done: {mesh.nn} nodes, nnz {mesh.fem.nnz}, solver {solver.memory() / 1e9:.1f} GB")
    for q in range(a.warmup):
        t0 = time.perf_counter()
        rep = step()
        log(f"[rank {rank}] warmup {q}: {time.perf_counter() - t0:.2f}s, {rep.iterations} it, "
            f"{rep.refinements} ref, res {rep.max_rel_residual:.2e}, mem {solver.memory() / 1e9:.1f} GB")
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = Clocks(torch.cuda.current_device()) if rank == 0 else None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(a.steps):
        rep = step()
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clocks = clk.stop() if clk else None
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    ms_step = ms / a.steps
    value = ns * nf * world / (ms_step / 1e3)

    # ---- end to end through the public API with host buffers
    e2e = None
    if not a.no_e2e:
        mua_h = torch.as_tensor(w["mua"]).pin_memory()
        musp_h = torch.as_tensor(w["musp"]).pin_memory()
        data_h = torch.empty((len(w["link"]), nf), dtype=torch.complex128).pin_memory()

        def step_e2e():
            mesh.mua = mua_h.to("cuda", non_blocking=True)
            mesh.musp = musp_h.to("cuda", non_blocking=True)
            mesh.update_properties()
            phi, data = mesh.flu_solve(precision="mixed", tol=a.tol, inner_tol=a.inner_tol)
            data_h.copy_(data, non_blocking=True)

        step_e2e()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0.record(st)
        for _ in range(a.steps):
            step_e2e()
        e1.record(st)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ems], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": ns * nf * world / (ems / a.steps / 1e3), "unit": "src.freq solves/s",
               "h2d_bytes_per_step": 2 * 8 * mesh.nn, "d2h_bytes_per_step": 16 * len(w["link"]) * nf,
               "ms_per_step": ems / a.steps}

    # ---- roofline: the dominant sweep kernel, CUDA-event timed on the solver's stream
    launches = {0: 2, 1: 5, 2: 1, 3: 1}  # per BiCGSTAB iteration: A SpMM x2, G SpMM x5, x/r/p, h/s
    names = {0: "k_spmm_A<float> (K + i w M SpMM)", 1: "k_spmm_G<float> (FSAI apply)",
             2: "k_update_xrp<float>", 3: "k_update_hs<float>"}
    prof = {q: solver.profile_kernel(q, 5) for q in launches}
    dom = max(prof, key=lambda q: prof[q][0] * launches[q])
    pk = json.load(open(ROOT / "MEASURED_PEAKS.json")) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = pk.get("hbm_gbs", 6650.0)
    ach = prof[dom][1] / (prof[dom][0] * 1e-3) / 1e9
    roof = {"bound": "hbm", "kernel": names[dom], "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
            "frac": round(ach / peak, 4), "traffic": None, "peak_source": "measured" if pk else "fallback",
            "per_kernel_ms": {names[q]: round(prof[q][0], 3) for q in prof},
            "per_kernel_gbs": {names[q]: round(prof[q][1] / (prof[q][0] * 1e-3) / 1e9, 1) for q in prof}}
    res.update(ms_per_step=ms_step, value=value, e2e=e2e, rep=rep, clocks=clocks, roof=roof, mesh=mesh, w=w)
    return res


def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        if rank != 0:
            return
        w = workload(a.workload)
        for _ in range(a.warmup):
            pass
        vals = []
        t0 = time.perf_counter()
        for _ in range(max(1, a.steps)):
            vals.append(cpu_sample(w, tol=a.tol))
        el = time.perf_counter() - t0
        v = statistics.median(x["value"] for x in vals)
        cb = dict(vals[0], value=v)
        cb.pop("seconds", None)
        print(json.dumps({"metric": "src.freq FEM solves/s (forward, batched)", "value": v,
                          "unit": "src.freq solves/s", "impl": "reference", "n_gpus": a.gpus, "steps": a.steps,
                          "warmup": a.warmup, "ms_per_step": 1e3 * el / max(1, a.steps),
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
                          "data": "synthetic", "config": {"workload": w["name"], "nodes": w["mesh"].nn,
                                                          "sources": len(w["src"]), "harmonics": w["nf"]},
                          "cpu_baseline": cb, "e2e": {"value": v, "unit": "src.freq solves/s",
                                                      "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local_rank))
    r = run_ours(a, rank, world, local_rank)
    w = r["w"]
    if rank == 0:
        cpu = None if (a.no_cpu or world > 1) else cpu_sample(w, tol=a.tol)
        if cpu:
            cpu.pop("seconds", None)
        rep = r["rep"]
        mesh = r["mesh"]
        line = {
            "metric": "src.freq FEM solves/s (forward, batched)", "value": r["value"], "unit": "src.freq solves/s",
            "n_gpus": world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": r["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c64+f64 refinement",
            "data": "synthetic",
            "config": {"workload": w["name"], "nodes": mesh.nn, "tets": int(w["mesh"].ne), "nnz": mesh.fem.nnz,
                       "sources": len(w["src"]), "harmonics": w["nf"], "tol": a.tol, "inner_tol": a.inner_tol,
                       "iterations": rep.iterations, "refinements": rep.refinements,
                       "max_rel_residual": rep.max_rel_residual, "l2": "inputs larger than L2 (vectors ~GB)",
                       "parallelism": f"replicas x{world}"},
            "e2e": r["e2e"], "roofline": r["roof"], "cpu_baseline": cpu, "clocks": r["clocks"],
            "gpu_launches": None,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
