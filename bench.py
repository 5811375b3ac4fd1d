#!/usr/bin/env python
"""Benchmark of the DOGPUP forward hot path on B200: src.freq FEM solves/s.

Workload (default ``ellipsoid``): ellipsoid head phantom 90x75x70 mm on a
1.2 mm lattice (6 tets per cube, interior nodes jittered 0.2 mm, seeded),
mua = 0.01/mm (1 + 0.2 * smooth Gaussian random field), musp' = 1/mm,
n = 1.4, 64 point sources x 128 harmonics (T = 10 ns), complex-FP32 COCG
(BiCGSTAB with --inner bicgstab) inside FP64 iterative refinement to a max
relative residual of 1e-8.

One step = device re-assembly of K, M + FSAI factors for all 128 harmonics
+ the batched solve of all 8192 right-hand sides + detector read-out.
Inputs are synthetic (no dataset).  Vectors are ~10 GB each, far larger than
L2, so no flush is needed between iterations.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) the harmonics are split over the ranks (rank r owns
k = r, r + N, ...; each GPU re-assembles K, M and factors and solves its own
harmonics) and every step ends with an NCCL all-gather of the detector data
of all harmonics: the total workload is fixed (strong scaling) and the step
time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import datetime
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
    ap.add_argument("--inner-tol", type=float, default=3e-5)
    ap.add_argument("--inner", choices=["cocg", "bicgstab"], default="cocg",
                    help="complex-FP32 inner solver of the mixed solve")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-secondary", action="store_true", help="skip the TG Jacobian / LM / plain-FP64 timings")
    ap.add_argument("--only", choices=["tg", "small", "lm", "recon", "uneven", "grad500k", "tgk", "chol"], default=None,
                    help="run one secondary timing alone and print its JSON (profiling cases)")
    ap.add_argument("--lm-grid-mm", type=float, default=2.0, help="voxel pitch of the LM step's Jacobian basis")
    ap.add_argument("--tgk-h", type=float, default=1.38, help="--only tgk: mesh pitch (mm) of the ellipsoid")
    ap.add_argument("--chol-n", type=int, default=22971, help="--only chol: order of the matrix")
    ap.add_argument("--order", choices=["morton", "lattice"], default="morton", help="mesh node numbering")
    ap.add_argument("--no-autotune", action="store_true", help="keep the built-in SpMM launch shape")
    ap.add_argument("--clock-ms", type=int, default=200, help="nvidia-smi sampling interval in the timed region")
    ap.add_argument("--spmm-vec", type=int, default=0, help="with --no-autotune: gather SpMM complex values per lane")
    ap.add_argument("--spmm-rows", type=int, default=0, help="with --no-autotune: gather SpMM rows per block")
    ap.add_argument("--spmm-kind", type=int, default=0, help="with --no-autotune: gather SpMM inner-loop kind (0-4)")
    ap.add_argument("--host-loop", action="store_true",
                    help="host-polled iteration loop instead of the graph's device-driven WHILE node "
                         "(for launch lists: ncu does not list kernels inside a conditional node)")
    return ap.parse_args()


def log(msg):
    print(msg, file=sys.stderr, flush=True)


def workload(name, seed=1, order="morton"):
    from dogpup_b200 import workloads
    if name == "medium":  # same shape family at a coarser lattice: 19k nodes, 64 x 32 RHS (profiling case)
        return workloads.ellipsoid_fwd(seed=seed, h=2.4, nf=32, order=order)
    return {"ellipsoid": workloads.ellipsoid_fwd, "cylinder": workloads.cylinder_fwd,
            "small": workloads.small_fwd}[name](seed=seed, order=order)


# ------------------------------------------------------------------ clocks
class Clocks:
    """nvidia-smi sampling during the timed region (read-only queries)."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index, interval_ms=200):
        # nvidia-smi numbers the physical GPUs; CUDA numbers the visible ones
        vis = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
        self.index = vis[index] if index < len(vis) else str(index)
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", self.index, f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", str(int(interval_ms))],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def wait_ready(self, samples=5, timeout=30.0):
        """Blocks until nvidia-smi has written `samples` lines: its start-up (device
        enumeration) stalls running GPU work, so it must be over before the timed region."""
        if self.p is None:
            return
        t_end = time.perf_counter() + timeout
        while time.perf_counter() < t_end:
            self.f.flush()
            try:
                n = sum(1 for _ in open(self.f.name))
            except OSError:
                n = 0
            if n >= samples or self.p.poll() is not None:
                break
            time.sleep(0.1)
        time.sleep(0.5)

    def mark(self):
        """Start of the timed region: samples before it are not reported."""
        self.t0 = datetime.datetime.now()

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait(timeout=10)
        self.f.flush()
        rows = []
        t0 = getattr(self, "t0", None)
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 10:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f")
            except ValueError:
                continue
            if t0 is None or ts >= t0:
                rows.append(parts[1:])
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------- CPU baseline
def cpu_sample(w, nharm=5, src_stride=2, tol=1e-8):
    """The reference algorithm on the host: FP64 FSAI + BiCGSTAB (dMesh.m:1247-1385)
    restated in C with OpenMP (oracle/cport), on a bounded sample of the workload:
    `nharm` harmonics spread evenly over the band (iteration counts fall from the
    lowest harmonic to the highest) x every `src_stride`-th source, on the same mesh
    and properties.  The per-RHS time is projected to the whole workload without
    bias: solve time per sampled RHS + FSAI time per harmonic / NS + assembly time /
    (NS * NF), as one GPU step amortises them."""
    import scipy.sparse as sp
    from oracle import cport, fem, solver
    from oracle.optode import locate_points, snap_pos, surface_faces
    m = w["mesh"]
    nf = w["nf"]
    harmonics = sorted({int(round(x)) for x in np.linspace(0, nf - 1, min(nharm, nf))})
    t0 = time.perf_counter()
    geo = fem.prepare_mesh(m.node, m.elem, w["nr"])
    K, M = fem.gen_fwdmat(m.node, m.elem, geo, w["mua"], w["musp"])
    t_asm = time.perf_counter() - t0
    dfc = (2 * np.pi / w["t"][-1]) / geo["c"]
    ns = len(w["src"])
    srcs = list(range(0, ns, src_stride))
    # sources as snap2mesh places them (dOptode.m:77-97): nearest surface point, moved
    # 1/min(musp) inward along the face normal, then located
    spos, sdir, _, _ = snap_pos(m.node, geo["bnd"], surface_faces(m.node, m.elem), w["src"][srcs])
    eid, bw = locate_points(m.node, m.elem, spos + (1.0 / float(np.min(w["musp"]))) * sdir)
    bw = np.where(bw < 1e-10, 0.0, bw)
    bw = bw / bw.sum(axis=1, keepdims=True)
    rg, cg = solver.fsai_pattern(sp.tril(K + 1j * dfc * M).tocsr())
    rt, ct, perm = solver.transpose_pattern(rg, cg, K.shape[0])
    Kt = sp.tril(K).tocsr()
    B = np.zeros((K.shape[0], len(srcs)), complex)
    for j in range(len(srcs)):
        B[m.elem[eid[j]], j] = bw[j]
    t_fsai = t_sol = 0.0
    iters = []
    for k in harmonics:
        t1 = time.perf_counter()
        G = cport.fsai_factor(Kt, sp.tril(k * dfc * M).tocsr(), rg, cg)
        t2 = time.perf_counter()
        _, it = cport.bicgstab(K, M, k * dfc, rg, cg, G, rt, ct, G[perm], B, tol)
        t_sol += time.perf_counter() - t2
        t_fsai += t2 - t1
        iters.append(int(it.max()))
    per = t_sol / (len(srcs) * len(harmonics)) + t_fsai / (len(harmonics) * ns) + t_asm / (ns * nf)
    return {"value": 1.0 / per, "unit": "src.freq solves/s", "cores": cport.threads(), "kind": "port",
            "sample": f"FP64 C/OpenMP restatement: {len(srcs)} of {ns} sources x harmonics {harmonics} of {nf} to "
                      f"tol {tol:g} on the full mesh ({m.nn} nodes; iterations per harmonic {iters}); per-RHS time = "
                      f"solve time per sampled RHS + FSAI time per harmonic / {ns} sources + assembly "
                      f"{t_asm:.1f}s / {ns * nf} RHS", "seconds": t_asm + t_fsai + t_sol}


# ------------------------------------------------------- secondary metrics
def _gates(t, n, width, start, spacing):
    sd = width / (2 * np.sqrt(2 * np.log(2)))
    return np.stack([np.exp(-(t - (start + q * spacing)) ** 2 / (2 * sd ** 2)) for q in range(n)])


def _event_ms(fn, reps):
    """Median over `reps` calls of each call's CUDA-event time (after two untimed calls): a
    single call slowed by the shared node (a driver allocation path that another process
    holds) moves the median of 5 less than the mean of 3."""
    import torch
    st = torch.cuda.current_stream()
    fn()
    fn()  # twice: a call that allocates its output while the previous one lives needs two blocks
    torch.cuda.synchronize()
    times = []
    for _ in range(max(reps, 5)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return float(np.median(times))


def _event_ms_restored(restore, fn, reps):
    """Median over `reps` calls of fn's CUDA-event time (after two untimed calls), restore()
    running before each call outside the timed region (fn overwrites its input in place)."""
    import torch
    st = torch.cuda.current_stream()
    times = []
    for it in range(2 + max(reps, 5)):
        restore()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        if it >= 2:
            times.append(e0.elapsed_time(e1))
    return float(np.median(times))


def plain_fp64_small_bench(tol=1e-10, truth_tol=1e-13):
    """Plain FP64 forward, small: cylinder r30 h60 @1.5 mm (jittered lattice, 6 tets per cube),
    homogeneous mua 0.01 / musp' 1 / n 1.4, 16 sources + 16 detectors on the mid-height ring,
    32 harmonics (100 MHz apart, T = 10 ns), complex FP64 BiCGSTAB + FSAI to `tol` (the
    reference's arithmetic, all right-hand sides batched).  Outputs: detector data, TD curves
    over 0-10 ns (fc2td) and 10 gates of 500 ps (fc2tg).  Each output's error is taken per link
    against the same chain on FP64 fields solved to `truth_tol` (itself checked against a
    sparse-direct solve in tests/test_gpu_fullsize.py): detector data relative to the link's
    norm over harmonics, TD curves and gates relative to the link's peak."""
    import torch
    from dogpup_b200 import api, workloads
    w = workloads.cylinder_fwd()
    mesh = workloads.build_dmesh(w)
    t = torch.as_tensor(w["t"])
    f = torch.as_tensor(mesh.optode.fAxis)
    gates = torch.as_tensor(_gates(w["t"], 10, 500e-12, 0.25e-9, 500e-12), device="cuda")
    nt = len(w["t"])

    def step(tl):
        mesh.update_properties()
        _, data, rep = mesh.flu_solve(precision="fp64", tol=tl, return_report=True)
        gfc = api.td2fc(gates, f, t)
        return data, api.fc2td(data, f, t), api.fc2tg(data, gfc, nt), rep

    step(tol)                                                   # warm-up: plan, graphs
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    data, td, tg, rep = step(tol)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    data0, td0, tg0, rep0 = step(truth_tol)
    per_link = lambda a, b, ref: ((a - b).abs().amax(dim=1) / ref).max().item()
    ns, nf = len(w["src"]), w["nf"]
    out = {"workload": f"{w['name']}, {mesh.nn} nodes, {int(w['mesh'].ne)} tets, {ns}x{len(w['det'])} optodes, "
                       f"{nf} harmonics, FP64 BiCGSTAB + FSAI to {tol:g}",
           "seconds": round(sec, 4), "src_freq_solves_per_s": round(ns * nf / sec, 1),
           "iterations": rep.iterations, "max_rel_residual": rep.max_rel_residual,
           "td_samples": nt, "td_span_ns": float(w["t"][-1] * 1e9), "gates": 10, "gate_width_ps": 500,
           "vs_fp64_to": truth_tol,
           "detector_data_per_link_max": per_link(data, data0, torch.linalg.vector_norm(data0, dim=1)),
           "td_per_link_max": per_link(td, td0, td0.abs().amax(dim=1)),
           "tg_per_link_max": per_link(tg, tg0, tg0.abs().amax(dim=1)),
           "td_peak_ns_link0": float(w["t"][int(td0[0].argmax())] * 1e9),
           "truth_iterations": rep0.iterations}
    mesh._solver = None
    return out


def tg_jacobian_bench(reps=3, tols=(1e-10, 1e-12, 1e-13, 1e-14), truth_tol=1e-14):
    """Sensitivity configuration: ellipsoid at 100k nodes, 32 sources x 32 detectors, 64 harmonics,
    20 gates of 250 ps, nodal basis (J^T is [nodes][20 x 1024] FP32).

    Truth: FP64 forward and adjoint fields solved to `truth_tol` for every source and detector,
    and the detector data, TG data and TG Jacobian formed from them.  For each tolerance in
    `tols` the batched mixed-precision forward + adjoint solves and the TG Jacobian are timed,
    and their errors taken PER LINK over all 1,024 links: detector data |d - d0| / |d0| over the
    link's harmonics, TG data max |y - y0| / max |y0| over its gates, TG Jacobian max |J - J0| /
    max |J0| over its voxels and gates.  The headline compares the fastest tolerance whose
    per-link maxima meet 1e-6 (data) and 1e-5 (Jacobian) with the plain FP64 solve of one
    right-hand side per call at the reference's tolerance 1e-12 (dMesh.m:1342), projected from
    a sample of harmonics spread over the band.  Also times the TG Jacobian's vjp and the
    adjoint gradient of a TG loss."""
    import torch
    from dogpup_b200 import api, workloads
    from dogpup_b200.autograd import TimeGatedForward
    w = workloads.ellipsoid_fwd(seed=3, h=1.38, ns=32, nd=32, nf=64)
    mesh = workloads.build_dmesh(w)
    gfc = api.td2fc(torch.as_tensor(_gates(w["t"], 20, 250e-12, 0.5e-9, 250e-12), device="cuda"),
                    torch.as_tensor(mesh.optode.fAxis), torch.as_tensor(w["t"]))
    nb = mesh.nodal_basis()
    link = mesh._link()
    nt = len(w["t"])
    fpsf = mesh.optode.s_fpsf
    nv, nm, nf = mesh.nn, int(link.shape[0]), w["nf"]
    ns, nd = len(w["src"]), len(w["det"])

    # FP64 truth for every source and detector
    phi0, data0, rep0 = mesh.flu_solve(precision="fp64", tol=truth_tol, maxit=3000, return_report=True)
    phiA0, repA0 = mesh.adj_flu_solve(precision="fp64", tol=truth_tol, maxit=3000, return_report=True)
    tg0 = api.fc2tg(data0, gfc, nt)
    J0 = api.jacobian_tg(nb, phi0, phiA0, fpsf, link, gfc, nt)
    del phi0, phiA0
    jref = J0.abs().amax(dim=(0, 1))                              # [NM]

    def link_errors(data, J):
        tg = api.fc2tg(data, gfc, nt)
        e_d = (torch.linalg.vector_norm(data - data0, dim=1) / torch.linalg.vector_norm(data0, dim=1)).max()
        e_t = ((tg - tg0).abs().amax(dim=1) / tg0.abs().amax(dim=1)).max()
        e_j = ((J - J0).abs().amax(dim=(0, 1)) / jref).max()
        return float(e_d), float(e_t), float(e_j)

    sweep, phi, phiA = {}, None, None
    # the reference's own arithmetic and tolerance (FP64 BiCGSTAB, max-over-columns stop at 1e-12)
    # against the same truth: the accuracy a link of the reference's output has
    phi64, data64 = mesh.flu_solve(precision="fp64", tol=1e-12)
    phiA64 = mesh.adj_flu_solve(precision="fp64", tol=1e-12)
    J64 = api.jacobian_tg(nb, phi64, phiA64, fpsf, link, gfc, nt)
    e_d, e_t, e_j = link_errors(data64, J64)
    sweep["fp64 1e-12"] = {"detector_data_per_link_max": e_d, "tg_data_per_link_max": e_t,
                           "tg_jacobian_per_link_max": e_j}
    del phi64, phiA64, J64
    for tol in tols:
        mesh.flu_solve(precision="mixed", tol=tol)                # warm-up (graphs, workspace)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        phi, data, rf = mesh.flu_solve(precision="mixed", tol=tol, return_report=True)
        phiA, ra = mesh.adj_flu_solve(precision="mixed", tol=tol, return_report=True)
        torch.cuda.synchronize()
        t_solve = time.perf_counter() - t0
        out = {}
        ms = _event_ms(lambda: out.__setitem__("J", api.jacobian_tg(nb, phi, phiA, fpsf, link, gfc, nt)), reps)
        e_d, e_t, e_j = link_errors(data, out["J"])
        del out
        sweep[f"{tol:g}"] = {"forward_and_adjoint_solve_s": round(t_solve, 3), "tg_jacobian_ms": round(ms, 3),
                             "batched_s": round(t_solve + ms * 1e-3, 3),
                             "detector_data_per_link_max": e_d, "tg_data_per_link_max": e_t,
                             "tg_jacobian_per_link_max": e_j,
                             "max_rel_residual": max(rf.max_rel_residual, ra.max_rel_residual),
                             "iterations_refinements": [[rf.iterations, rf.refinements], [ra.iterations, ra.refinements]],
                             "meets_bar": bool(e_d <= 1e-6 and e_j <= 1e-5)}
        log(f"[rank 0] sensitivity at tol {tol:g}: {sweep[f'{tol:g}']}")
    del J0
    ok = [k for k in sweep if sweep[k].get("meets_bar")]
    pick = min(ok, key=lambda k: sweep[k]["batched_s"]) if ok else f"{tols[-1]:g}"

    # kernel timings on the last (tightest) fields
    out = {}
    ms = _event_ms(lambda: out.__setitem__("J", api.jacobian_tg(nb, phi, phiA, fpsf, link, gfc, nt)), reps)
    del out
    g = torch.as_tensor(np.random.default_rng(5).standard_normal((nm, 20)), device="cuda")
    ms_vjp = _event_ms(lambda: api.jacobian_tg_vjp(nb, phi, phiA, fpsf, link, gfc, nt, g), reps)
    # the same two kernels on each engine (dgp_set_jacobian_engine: 1 CUDA cores, 2 tensor cores)
    from dogpup_b200._lib import lib as _dl
    engines = {}
    for eng, name in ((1, "cuda_cores"), (2, "tensor_cores")):
        _dl.dgp_set_jacobian_engine(eng)
        out = {}
        ms_e = _event_ms(lambda: out.__setitem__("J", api.jacobian_tg(nb, phi, phiA, fpsf, link, gfc, nt)), reps)
        del out
        engines[name] = {"ms": round(ms_e, 3),
                         "vjp_ms": round(_event_ms(lambda: api.jacobian_tg_vjp(nb, phi, phiA, fpsf, link, gfc, nt, g),
                                                   reps), 3)}
    _dl.dgp_set_jacobian_engine(0)
    field_bytes = 16.0 * nf * nv * (ns + nd)
    j_bytes = 4.0 * nv * 20 * nm
    flops = 2.0 * nv * nm * nf * (2 + 2 * 20)
    del phi, phiA

    # plain FP64, one right-hand side per solve, at the reference's tolerance (sampled, projected)
    plain = plain_fp64_per_rhs(mesh, nsample=8, tol=1e-12)
    plain_s = (ns + nd) * nf / plain["value"]
    batched_s = sweep[pick]["batched_s"]

    # adjoint gradient of a TG loss (forward + adjoint solve + element kernel), mixed precision
    model = TimeGatedForward(mesh, gfc, precision="mixed", tol=float(pick))
    mua = torch.as_tensor(w["mua"], device="cuda").requires_grad_(True)
    musp = torch.as_tensor(w["musp"], device="cuda")
    (model(mua, musp) * g).sum().backward()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mua.grad = None
    (model(mua, musp) * g).sum().backward()
    torch.cuda.synchronize()
    t_grad = time.perf_counter() - t0
    mesh._solver = None
    return {"workload": f"ellipsoid 90x75x70 @1.38mm, {nv} nodes, 32x32 optodes, 64 harmonics, 20 gates",
            "J_shape": [20 * nm, nv], "ms": round(ms, 3), "vjp_ms": round(ms_vjp, 3),
            "engines": engines, "engine_used": "default: TG Jacobian and vjp on the tensor cores",
            "achieved_gbs": round((field_bytes + j_bytes) / (ms * 1e-3) / 1e9, 1),
            "achieved_tflops_fp32": round(flops / (ms * 1e-3) / 1e12, 2),
            "mixed_vs_fp64": {"truth": f"FP64 fields to {truth_tol:g} (reached {max(rep0.max_rel_residual, repA0.max_rel_residual):.2e}), "
                                       f"all {ns} sources and {nd} detectors, all {nm} links", "by_tol": sweep,
                              "bar": "detector data 1e-6 and TG Jacobian 1e-5 per link"},
            "headline": {"tol": float(pick), "batched_mixed_forward_adjoint_tgJ_s": batched_s,
                         "plain_fp64_per_rhs_s": round(plain_s, 3),
                         "plain_fp64_per_rhs_solves_per_s": round(plain["value"], 2),
                         "plain_sample": plain["sample"] + f", projected to {ns + nd} x {nf} RHS",
                         "plain_projection_rel_spread": plain["rel_spread"],
                         "speedup": round(plain_s / batched_s, 2)},
            "tg_loss_gradient_s": round(t_grad, 3)}


def lm_step_bench(reps=2, grid_mm=2.0):
    """Weighted LM normal-equation step of the 50k-node configuration: cylinder r30 h60 @1.5 mm,
    32 x 32 optodes, 10 gates (10240 measurements), J on the in-mesh voxels of a grid_mm grid."""
    import ctypes as C
    import torch
    from dogpup_b200 import api, workloads
    from dogpup_b200._lib import lib, check
    w = workloads.cylinder_fwd(seed=4, ns=32, nd=32, nf=32)
    mesh = workloads.build_dmesh(w)
    lo, hi = w["mesh"].node.min(0), w["mesh"].node.max(0)
    mesh.mesh2grid(*[np.arange(lo[d], hi[d] + 1e-9, grid_mm) for d in range(3)])
    P = mesh.m2g[mesh.gridinmesh]
    basis = api.Basis(P, np.full(P.shape[0], mesh.dxyz ** 3))
    phi, data = mesh.flu_solve(precision="mixed", tol=1e-8)
    phiA = mesh.adj_flu_solve(precision="mixed", tol=1e-8)
    nt = len(w["t"])
    gfc = api.td2fc(torch.as_tensor(_gates(w["t"], 10, 500e-12, 0.5e-9, 500e-12), device="cuda"),
                    torch.as_tensor(mesh.optode.fAxis), torch.as_tensor(w["t"]))
    data_tg = api.fc2tg(data, gfc, nt)
    J = api.jacobian_tg(basis, phi, phiA, mesh.optode.s_fpsf, mesh._link(), gfc, nt, data_tg)  # Rytov
    nv, nmeas = J.shape[0], J.shape[1] * J.shape[2]
    Jt = J.reshape(nv, nmeas).contiguous()
    del J, phi, phiA
    mesh._solver = None          # release the solver workspace before the dense step
    rng = np.random.default_rng(9)
    W = torch.as_tensor(1.0 / (0.01 * (1 + rng.random(nmeas))) ** 2, device="cuda")
    y = torch.as_tensor(rng.standard_normal(nmeas) * 0.01, device="cuda")
    ld = nv + (nv & 1)                                  # even: 16-byte aligned rows, as dgp_lm_update uses
    H = torch.empty((nv, ld), dtype=torch.float64, device="cuda")
    x = torch.empty(nv, dtype=torch.float64, device="cuda")
    v = lambda t: C.c_void_p(t.data_ptr())
    ms_ne = _event_ms(lambda: check(lib.dgp_normal_eq(v(Jt), nv, nmeas, v(W), v(y), 1e-2, 0, v(H), ld, v(x),
                                                      api.stream_ptr())), reps)
    Hc = H.clone()
    xc = x.clone()

    def restore():                                      # the factorisation overwrites Hc
        Hc.copy_(H)
        xc.copy_(x)
    ms_chol = _event_ms_restored(restore, lambda: check(lib.dgp_cholesky_solve(v(Hc), nv, ld, v(xc),
                                                                              api.stream_ptr())), reps)
    syrk_flops = 3 * 2.0 * nmeas * nv * (nv + 128) / 2
    # the same LM update from all-FP64 normal equations (cuBLAS DGEMM) and the FP64 Cholesky
    Jd = Jt.double()
    Jw = Jd * W[None, :]
    H64 = Jw @ Jd.T
    H64.diagonal().add_(1e-2 * H64.diagonal().max())
    x64 = (Jw @ y).contiguous()
    del Jw, Jd
    H64 = H64.contiguous()
    check(lib.dgp_cholesky_solve(v(H64), nv, nv, v(x64), api.stream_ptr()))
    upd_err = float(torch.linalg.vector_norm(xc - x64) / torch.linalg.vector_norm(x64))
    del H64
    # the same update in one call in the smaller (measurements') form: dgp_lm_update
    xu = torch.empty(nv, dtype=torch.float64, device="cuda")
    used = C.c_int32(0)
    ms_upd = _event_ms(lambda: check(lib.dgp_lm_update(v(Jt), nv, nmeas, v(W), v(y), 1e-2, v(xu), 0, C.byref(used),
                                                       api.stream_ptr())), reps)
    upd_err_u = float(torch.linalg.vector_norm(xu - x64) / torch.linalg.vector_norm(x64))
    # DGEMM peak measured here: the denominator of the Cholesky's FP64 fraction
    a = torch.randn((8192, 8192), dtype=torch.float64, device="cuda")
    ms_dgemm = _event_ms(lambda: a @ a, 3)
    dgemm_tf = 2.0 * 8192 ** 3 / (ms_dgemm * 1e-3) / 1e12
    del a
    pk = json.load(open(ROOT / "MEASURED_PEAKS.json")) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    bf16 = pk.get("bf16_tflops", 1590.0)
    chol_tf = nv ** 3 / 3 / (ms_chol * 1e-3) / 1e12
    syrk_tf = syrk_flops / (ms_ne * 1e-3) / 1e12
    return {"workload": f"cylinder r30 h60 @1.5mm, {mesh.nn} nodes, 32x32 optodes, 10 gates, {nv} voxels "
                        f"({grid_mm:g} mm)",
            "nmeas": nmeas, "nv": nv, "normal_eq_ms": round(ms_ne, 3), "cholesky_solve_ms": round(ms_chol, 3),
            "syrk_tflops_bf16_lower_bound": round(syrk_tf, 1),
            "syrk_frac_of_bf16_peak": round(syrk_tf / bf16, 3),
            "bf16_peak_source": "measured" if "bf16_tflops" in pk else "fallback",
            "cholesky_tflops_fp64": round(chol_tf, 2), "dgemm_tflops_fp64_measured": round(dgemm_tf, 2),
            "cholesky_frac_of_dgemm": round(chol_tf / dgemm_tf, 3),
            "lm_update_rel_err_vs_fp64": upd_err,
            "lm_update_one_call": {"ms": round(ms_upd, 3), "form": "measurements" if used.value == 2 else "unknowns",
                                   "rel_err_vs_fp64": upd_err_u,
                                   "note": "dgp_lm_update: J_w^T (J_w J_w^T + mu I)^-1 W^1/2 y, the same update "
                                           "as the nv x nv normal equations above"}}


def lm_recon_bench(max_iter=10, grid_mm=2.0, seed=7):
    """Weighted LM reconstruction: cylinder r30 h60 @1.5 mm, 32 x 32 optodes, 10 gates of 500 ps;
    truth = two spheres of r = 8 mm with 2x mua at seeded positions; data with 1 % count-scaled
    noise (sigma = 1 % x sqrt(data x the curve's peak)), W = 1/sigma^2.  Runs the loop with
    mixed-precision solves + split-BF16 normal equations, and again all-FP64 (FP64 solves, FP64
    J^T W J); reports per-iteration mua error vs truth and vs the FP64 run, and the time."""
    import torch
    from dogpup_b200 import api, workloads
    from dogpup_b200.recon import LMRecon
    rng = np.random.default_rng(seed)
    w = workloads.cylinder_fwd(seed=4, ns=32, nd=32, nf=32)
    node = w["mesh"].node
    truth = np.full(w["mesh"].nn, 0.01)
    centres = []
    while len(centres) < 2:
        p = np.array([rng.uniform(-12, 12), rng.uniform(-12, 12), rng.uniform(20, 40)])
        if p[0] ** 2 + p[1] ** 2 < 14 ** 2 and all(np.linalg.norm(p - q) > 18 for q in centres):
            centres.append(p)
    for p in centres:
        truth[((node - p) ** 2).sum(1) < 8.0 ** 2] = 0.02
    w["mua"] = truth
    mesh = workloads.build_dmesh(w)
    nt = len(w["t"])
    gfc = api.td2fc(torch.as_tensor(_gates(w["t"], 10, 500e-12, 0.5e-9, 500e-12), device="cuda"),
                    torch.as_tensor(mesh.optode.fAxis), torch.as_tensor(w["t"]))
    _, data = mesh.flu_solve(precision="fp64", tol=1e-12)
    clean = api.fc2tg(data, gfc, nt).cpu().numpy()
    sigma = 0.01 * np.sqrt(np.abs(clean) * np.abs(clean).max(axis=1, keepdims=True))
    data_m = np.abs(clean + sigma * rng.standard_normal(clean.shape))
    lo, hi = node.min(0), node.max(0)
    mesh.mesh2grid(*[np.arange(lo[d], hi[d] + 1e-9, grid_mm) for d in range(3)])
    truth_d = torch.as_tensor(truth, device="cuda")
    out = {}
    for tag, prec, ne in (("mixed_split_bf16", "mixed", "split_bf16"), ("fp64", "fp64", "fp64")):
        mesh.mua = torch.full((mesh.nn,), 0.01, dtype=torch.float64, device="cuda")
        mesh.update_properties()
        rec = LMRecon(mesh, gfc, precision=prec, tol=1e-8 if prec == "mixed" else 1e-10, normal_eq=ne)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = rec.run(data_m, lam=(1.0, 0.0), sigma=sigma, thresh=0.8, max_iter=max_iter, truth=truth_d)
        torch.cuda.synchronize()
        out[tag] = dict(seconds=time.perf_counter() - t0, hist=h)
        mesh._solver = None
    a, b = out["mixed_split_bf16"]["hist"], out["fp64"]["hist"]
    vs64 = [float(torch.linalg.vector_norm(x - y) / torch.linalg.vector_norm(y)) for x, y in zip(a["mua"], b["mua"])]
    return {"workload": f"cylinder r30 h60 @1.5mm, {mesh.nn} nodes, 32x32 optodes, 10 gates, "
                        f"{int(np.asarray(mesh.gridinmesh).sum())} voxels ({grid_mm:g} mm), 2 absorbers r=8 mm 2x",
            "iterations": a["iterations"], "seconds_mixed": round(out["mixed_split_bf16"]["seconds"], 2),
            "seconds_fp64": round(out["fp64"]["seconds"], 2),
            "mua_rel_err_vs_truth_mixed": [round(x, 5) for x in a["err_truth"]],
            "mua_rel_err_vs_truth_fp64": [round(x, 5) for x in b["err_truth"]],
            "mua_rel_diff_mixed_vs_fp64": [float(f"{x:.3e}") for x in vs64],
            "data_misfit_perc_mixed": [round(x, 3) for x in a["err_perc"]]}


def uneven_bench(count=24, seed=11, streams=4):
    """Uneven batch: `count` seeded ellipsoid / cylinder meshes of 5k-300k nodes (log-uniform),
    8-64 sources and detectors, 16-128 harmonics; forward + TG vjp (10 gates of 500 ps, seeded
    upstream gradient) for all of them through the batch executor (mixed precision to 1e-8)."""
    import torch
    from dogpup_b200 import meshgen, workloads
    from dogpup_b200.autograd import gate_coefficients
    from dogpup_b200.batch import UnevenBatch
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    meshes, gates, ups, sizes = [], [], [], []
    for i in range(count):
        target = float(np.exp(rng.uniform(np.log(5e3), np.log(3e5))))
        ns, nd, nf = int(rng.integers(8, 65)), int(rng.integers(8, 65)), int(rng.integers(16, 129))
        t = workloads.time_axis(10e-9)
        if i % 2 == 0:
            h = (4 / 3 * np.pi * 45 * 37.5 * 35 / target) ** (1 / 3)
            m = meshgen.ellipsoid_mesh((90.0, 75.0, 70.0), h, jitter=0.2 * h / 1.2, seed=seed + i)
            src = workloads.ring(ns, np.zeros(3), (45.0, 37.5), 0.0)
            det = workloads.ring(nd, np.zeros(3), (45.0, 37.5), 0.0, phase=np.pi / nd)
        else:
            h = (np.pi * 30 ** 2 * 60 / target) ** (1 / 3)
            m = meshgen.cylinder_mesh(30.0, 60.0, h, jitter=0.2 * h / 1.5, seed=seed + i)
            src = workloads.ring(ns, np.array([0.0, 0.0, 30.0]), (30.0, 30.0), 30.0)
            det = workloads.ring(nd, np.array([0.0, 0.0, 30.0]), (30.0, 30.0), 30.0, phase=np.pi / nd)
        w = dict(name=f"uneven {i}", mesh=m, mua=np.full(m.nn, 0.01), musp=np.full(m.nn, 1.0), nr=1.4, src=src,
                 det=det, link=workloads.all_pairs(ns, nd), t=t, nf=nf)
        mesh = workloads.build_dmesh(w)
        meshes.append(mesh)
        gates.append(gate_coefficients(t, 0.5e-9 + 0.5e-9 * np.arange(10), 500e-12, mesh.optode.fAxis))
        ups.append(rng.standard_normal((ns * nd, 10)))
        sizes.append((m.nn, ns, nd, nf))
    setup_s = time.perf_counter() - t0
    B = UnevenBatch(meshes, streams=streams, precision="mixed", tol=1e-8, gates=gates, upstream=ups)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = B.run()
    torch.cuda.synchronize()
    run_s = time.perf_counter() - t0
    solves = sum((ns + nd) * nf for _, ns, nd, nf in sizes)
    return {"workload": f"{count} meshes, {min(s[0] for s in sizes)}-{max(s[0] for s in sizes)} nodes "
                        f"(total {sum(s[0] for s in sizes)}), 8-64 sources/detectors, 16-128 harmonics, "
                        "forward + adjoint + TG vjp (10 gates)",
            "tasks": len(B.tasks), "streams": streams, "budget_gb": round(B.budget / 1e9, 1),
            "seconds": round(run_s, 2), "src_freq_solves": solves,
            "src_freq_solves_per_s": round(solves / run_s, 1), "host_setup_s": round(setup_s, 1),
            "vjp_finite": bool(all(torch.isfinite(r.vjp).all() for r in res))}


def tg_kernels_bench(h=1.38, reps=5):
    """The TG Jacobian and its vjp alone on both engines (kernel timing and profiling case):
    ellipsoid 90 x 75 x 70 mm at pitch h (h = 1.38 mm: 101,880 nodes; 2.4 mm: 20,497), 32 x 32
    optodes, 64 harmonics, 20 gates of 250 ps, nodal basis, fields from mixed solves to 1e-6.
    The default engine runs first (the tensor cores where the shapes fit)."""
    import torch
    from dogpup_b200 import api, workloads
    from dogpup_b200._lib import lib as _dl
    w = workloads.ellipsoid_fwd(seed=3, h=h, ns=32, nd=32, nf=64)
    mesh = workloads.build_dmesh(w)
    gfc = api.td2fc(torch.as_tensor(_gates(w["t"], 20, 250e-12, 0.5e-9, 250e-12), device="cuda"),
                    torch.as_tensor(mesh.optode.fAxis), torch.as_tensor(w["t"]))
    nb, link, nt, fpsf = mesh.nodal_basis(), mesh._link(), len(w["t"]), mesh.optode.s_fpsf
    phi, _ = mesh.flu_solve(precision="mixed", tol=1e-6)
    phiA = mesh.adj_flu_solve(precision="mixed", tol=1e-6)
    g = torch.as_tensor(np.random.default_rng(5).standard_normal((int(link.shape[0]), 20)), device="cuda")
    res = {"workload": f"ellipsoid 90x75x70 @{h}mm, {mesh.nn} nodes, 32x32 optodes, 64 harmonics, 20 gates"}
    for eng, name in ((0, "default"), (1, "cuda_cores")):
        _dl.dgp_set_jacobian_engine(eng)
        out = {}
        ms = _event_ms(lambda: out.__setitem__("J", api.jacobian_tg(nb, phi, phiA, fpsf, link, gfc, nt)), reps)
        del out
        res[name] = {"tg_jacobian_ms": round(ms, 3),
                     "vjp_ms": round(_event_ms(lambda: api.jacobian_tg_vjp(nb, phi, phiA, fpsf, link, gfc, nt, g),
                                               reps), 3)}
    _dl.dgp_set_jacobian_engine(0)
    return res


def cholesky_bench(n=22971, reps=3):
    """The library's FP64 Cholesky solve alone (kernel timing and profiling case): a random
    diagonally dominant symmetric positive definite matrix of order n, even leading dimension."""
    import ctypes as C
    import torch
    from dogpup_b200._lib import lib, check
    ld = n + (n & 1)
    gen = torch.Generator(device="cuda").manual_seed(3)
    H0 = torch.rand((n, ld), generator=gen, device="cuda", dtype=torch.float64) - 0.5
    H0.diagonal()[:n] += float(n)
    x0 = torch.rand(n, generator=gen, device="cuda", dtype=torch.float64)
    H, x = H0.clone(), x0.clone()

    def restore():                                      # the factorisation overwrites H
        H.copy_(H0)
        x.copy_(x0)
    ms = _event_ms_restored(restore, lambda: check(lib.dgp_cholesky_solve(C.c_void_p(H.data_ptr()), n, ld,
                                                                         C.c_void_p(x.data_ptr()), None)), reps)
    return {"n": n, "ld": ld, "cholesky_solve_ms": round(ms, 3),
            "tflops_fp64": round(n ** 3 / 3 / (ms * 1e-3) / 1e12, 2)}


def grad_big_bench(target_nodes=500_000, ns=32, nd=32, nf=32):
    """End-to-end gradient of a TG least-squares loss w.r.t. nodal mua on a ~500k-node ellipsoid,
    fields recomputed in backward instead of stored; mixed precision vs plain FP64 solves, both to
    the reference's tolerance 1e-12 (a norm-wise 1e-8 leaves detector values far from a source
    inaccurate in either precision: fluence spans ~7 decades over the mesh)."""
    import torch
    from dogpup_b200 import workloads
    from dogpup_b200.autograd import TimeGatedForward, gate_coefficients
    h = (4 / 3 * np.pi * 45 * 37.5 * 35 / target_nodes) ** (1 / 3)
    w = workloads.ellipsoid_fwd(seed=5, h=h, ns=ns, nd=nd, nf=nf)
    mesh = workloads.build_dmesh(w)
    gfc = gate_coefficients(w["t"], 0.5e-9 + 0.5e-9 * np.arange(10), 500e-12, mesh.optode.fAxis)
    rng = np.random.default_rng(2)
    target = None
    out = {}
    for prec, tol in (("mixed", 1e-12), ("fp64", 1e-12)):
        model = TimeGatedForward(mesh, gfc, precision=prec, tol=tol, recompute=True)
        mua = torch.as_tensor(w["mua"], device="cuda").clone().requires_grad_(True)
        musp = torch.as_tensor(w["musp"], device="cuda")
        if target is None:
            with torch.no_grad():
                target = model(mua, musp) * torch.as_tensor(1 + 0.01 * rng.standard_normal((ns * nd, 10)),
                                                            device="cuda")
            # gates above 1 % of each curve's range (id_thresh 'all'): log data is ill-conditioned below
            from dogpup_b200.recon import id_thresh
            mask = torch.as_tensor(id_thresh(target.cpu().numpy(), "all") & (target.cpu().numpy() > 0),
                                   device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        y = model(mua, musp)
        r = torch.where(mask, torch.log(y.clamp_min(1e-300)) - torch.log(target.clamp_min(1e-300)), 0.0)
        loss = (r ** 2).sum()
        loss.backward()
        torch.cuda.synchronize()
        out[prec] = dict(seconds=time.perf_counter() - t0, grad=mua.grad.clone(), loss=float(loss.detach()),
                         iterations=[(rep.iterations, rep.refinements) for rep in model.last_reports])
        mesh._solver = None
    g64, gm = out["fp64"]["grad"], out["mixed"]["grad"]
    return {"workload": f"ellipsoid 90x75x70 @{h:.2f}mm, {mesh.nn} nodes, {ns}x{nd} optodes, {nf} harmonics, "
                        "10 gates, TG log-data least squares, fields recomputed in backward",
            "seconds_mixed": round(out["mixed"]["seconds"], 2), "seconds_fp64": round(out["fp64"]["seconds"], 2),
            "speedup": round(out["fp64"]["seconds"] / out["mixed"]["seconds"], 2),
            "solves_iterations_refinements": {k: out[k]["iterations"] for k in out},
            "gates_in_loss": int(mask.sum()), "loss": {k: out[k]["loss"] for k in out},
            "grad_rel_diff_mixed_vs_fp64": float(torch.linalg.vector_norm(gm - g64) / torch.linalg.vector_norm(g64))}


def plain_fp64_per_rhs(mesh, nsample=4, tol=1e-8):
    """The plain baseline of the path: FP64 BiCGSTAB (reference arithmetic) on ONE right-hand side per
    call (one optode at one harmonic), through the same library, on the given mesh.  Harmonics are
    sampled evenly over the band (iteration counts fall with the harmonic), each with one source
    and one detector solve; solves/s is the sample's count over its summed time, and rel_spread the
    standard error of the mean time per solve over that mean (the projection's uncertainty)."""
    import torch
    from dogpup_b200 import api
    o = mesh.optode
    opt = [mesh._sources(o.s_bary[:1]), mesh._sources(o.d_bary[:1])]
    ks = sorted({int(round(x)) for x in np.linspace(0, o.Nf - 1, nsample)})
    opts = api.make_opts(tol=tol, maxit=1000, precision="fp64")
    times, iters = [], []
    for k in ks:
        S = api.Solver(mesh.fem.rowptr, mesh.fem.col, mesh.K, mesh.M, o.df / mesh.c, 1, 1, harmonics=[k])
        f = o.s_fpsf[k:k + 1].contiguous()
        for nodes, wts in opt:
            S.solve_sources(nodes, wts, f, opts)            # warm-up: workspace, graph capture
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, rep = S.solve_sources(nodes, wts, f, opts)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
            iters.append(rep.iterations)
        del S
    tm = np.asarray(times)
    return {"value": len(tm) / tm.sum(), "unit": "src.freq solves/s", "iterations": iters,
            "rel_spread": float(tm.std(ddof=1) / np.sqrt(len(tm)) / tm.mean()) if len(tm) > 1 else None,
            "sample": f"source 0 and detector 0 at harmonics {ks}, FP64 to {tol:g}, one right-hand side per solve"}


# --------------------------------------------------------------- our arm
def _guarded(name, fn):
    """Runs one secondary measurement with nvidia-smi sampling the clocks meanwhile; an exception
    is reported in its key instead of ending the run (the main line is still printed)."""
    import gc
    import torch
    gc.collect()
    torch.cuda.empty_cache()
    clk = Clocks(torch.cuda.current_device())
    clk.wait_ready()
    clk.mark()
    t0 = time.perf_counter()
    try:
        out = fn()
    except Exception as e:  # noqa: BLE001 -- reported, not swallowed
        import traceback
        traceback.print_exc()
        out = {"error": f"{type(e).__name__}: {e}"}
    if isinstance(out, dict):
        out["clocks"] = clk.stop()      # SM clock and throttle reasons while this measurement ran
    else:
        clk.stop()
    log(f"[rank 0] {name} ({time.perf_counter() - t0:.1f} s): {json.dumps(out)[:2000]}")
    gc.collect()
    torch.cuda.empty_cache()
    return out


def run_ours(a, rank, world, local_rank):
    """One rank of the forward benchmark.  N = 1: the whole workload on one GPU.  N > 1: the
    harmonics are split over the ranks (rank r solves k = r, r + N, ..., shard.py) and every step
    ends with the all-gather of the detector data of all harmonics (NCCL), so `value` is the
    whole job's solves/s at a fixed total workload (strong scaling)."""
    import torch
    import torch.distributed as dist
    from dogpup_b200 import workloads
    from dogpup_b200.shard import ShardedForward, gather_spectra
    torch.cuda.set_device(local_rank)
    w = workload(a.workload, seed=1, order=a.order)
    mesh = workloads.build_dmesh(w)
    ns, nf = len(w["src"]), w["nf"]
    st = torch.cuda.current_stream()
    res = {}
    prec = "mixed" if a.inner == "cocg" else "mixed_bicgstab"
    fw = None
    if world > 1:
        fw = ShardedForward(mesh, np.ones((1, nf), complex), rank, world, precision=prec, tol=a.tol,
                            inner_tol=a.inner_tol)
        solver = fw.solver
    else:
        solver = mesh.solver()

    def step():
        mesh.update_properties()                         # K, M re-assembly (+ FSAI refactor, N = 1)
        if fw is None:
            phi, data, rep = mesh.flu_solve(precision=prec, tol=a.tol, inner_tol=a.inner_tol, return_report=True)
            return rep, data
        fw.update()                                      # FSAI refactor of this rank's harmonics
        _, data, rep = fw.solve()
        return rep, gather_spectra(data, nf, rank, world)   # detector data of every harmonic

    log(f"[rank {rank}] setup done: {mesh.nn} nodes, nnz {mesh.fem.nnz}, harmonics "
        f"{'all' if fw is None else len(fw.harm)}, solver {solver.memory() / 1e9:.1f} GB")
    if a.host_loop:
        solver.set_device_loop(False)
    tuned = None
    if a.no_autotune and a.spmm_vec:
        solver.set_spmm(False, a.spmm_vec, a.spmm_rows)
        solver.set_spmm_kind(a.spmm_kind)
        tuned = dict(solver.spmm_shape(), set_by="command line")
    if not a.no_autotune:
        t0 = time.perf_counter()
        tuned = solver.autotune()                       # one-time plan set-up, outside the timed region
        tuned["seconds"] = round(time.perf_counter() - t0, 2)
        log(f"[rank {rank}] autotune: {tuned}")
    for q in range(a.warmup):
        t0 = time.perf_counter()
        rep, _ = step()
        log(f"[rank {rank}] warmup {q}: {time.perf_counter() - t0:.2f}s, {rep.iterations} it, "
            f"{rep.refinements} ref, res {rep.max_rel_residual:.2e}, mem {solver.memory() / 1e9:.1f} GB")
    # the sampler starts before the timed region (nvidia-smi's start-up talks to the driver and
    # would stall the first timed launches) and keeps sampling through it
    clk = Clocks(torch.cuda.current_device(), a.clock_ms) if rank == 0 else None
    if clk:
        clk.wait_ready()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    from dogpup_b200._lib import lib as _dlib
    if clk:
        clk.mark()
    n_launch0 = _dlib.dgp_kernel_launches()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    marks = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    e0.record(st)
    for q in range(a.steps):
        rep, _ = step()
        marks[q].record(st)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    step_ms = [e0.elapsed_time(marks[0])] + [marks[q - 1].elapsed_time(marks[q]) for q in range(1, a.steps)]
    log(f"[rank {rank}] timed steps (ms): {[round(x, 1) for x in step_ms]}")
    launches = _dlib.dgp_kernel_launches() - n_launch0
    clocks = clk.stop() if clk else None
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)                # the job's time: the slowest rank
        ms = float(t.item())
        lt = torch.tensor([float(launches)], device="cuda")
        dist.all_reduce(lt, op=dist.ReduceOp.SUM)               # kernels launched by all ranks
        launches = int(lt.item())
        dist.barrier()
    ms_step = ms / a.steps
    value = ns * nf / (ms_step / 1e3)                  # the whole job: every source x harmonic once

    # ---- end to end through the public API with host buffers
    e2e = None
    if not a.no_e2e:
        mua_h = torch.as_tensor(w["mua"]).pin_memory()
        musp_h = torch.as_tensor(w["musp"]).pin_memory()
        data_h = torch.empty((len(w["link"]), nf), dtype=torch.complex128).pin_memory()

        def step_e2e():
            mesh.mua = mua_h.to("cuda", non_blocking=True)
            mesh.musp = musp_h.to("cuda", non_blocking=True)
            _, data = step()
            if rank == 0:
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
        e2e = {"value": ns * nf / (ems / a.steps / 1e3), "unit": "src.freq solves/s",
               "h2d_bytes_per_step": world * 2 * 8 * mesh.nn, "d2h_bytes_per_step": 16 * len(w["link"]) * nf,
               "ms_per_step": ems / a.steps}

    # ---- roofline: the dominant sweep kernel, CUDA-event timed on the solver's stream
    # sweeps per inner iteration -- BiCGSTAB: A SpMM x2, G SpMM x5, x/r/p, s; COCG: q = A p with p.q,
    # T = G r with T.T, z = G^T T (the plain G kernel on the G^T records), r update, x/p update
    per_iter = {0: 2, 1: 5, 2: 1, 3: 1} if a.inner == "bicgstab" else {4: 1, 5: 1, 1: 1, 6: 1, 7: 1}
    shp = solver.spmm_shape()
    sv, sk = shp["vec"] or 4, shp["kind"]
    gk = 0 if sk == 4 else sk                       # kind 4 pairs the harmonics of A only
    a0 = f"k_spmm_pair<{sv},0> (K + i w M SpMM, harmonic pairs)" if sk == 4 else f"k_spmm<float,{sv},0,OpA32,{sk}> (K + i w M SpMM)"
    a1 = f"k_spmm_pair<{sv},1> (q = A p, p.q, harmonic pairs)" if sk == 4 else f"k_spmm<float,{sv},1,OpA32,{sk}> (q = A p, p.q)"
    names = {0: a0, 1: f"k_spmm<float,{sv},0,OpG32,{gk}> (FSAI apply)",
             2: "k_update_xrp<float>", 3: "k_update_s<float>",
             4: a1, 5: f"k_spmm<float,{sv},3,OpG32,{gk}> (T = G r, T.T)",
             6: "k_update_r<float>", 7: "k_update_px<float>"}
    prof = {q: solver.profile_kernel(q, 5) for q in per_iter}
    dom = max(prof, key=lambda q: prof[q][0] * per_iter[q])
    pk = json.load(open(ROOT / "MEASURED_PEAKS.json")) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = pk.get("hbm_gbs", 6650.0)
    ach = prof[dom][1] / (prof[dom][0] * 1e-3) / 1e9
    # DRAM bytes (read + write) per launch from one ncu capture of the same kernel and launch
    # shape on the 20,497-node, 32-harmonic ellipsoid, scaled to this launch by nodes x harmonics
    # (the records and vectors all scale with both)
    captured = {0: 659.7e6, 1: 716.4e6, 4: 804.8e6, 5: 797.1e6, 6: 966.3e6, 7: 1626.1e6}
    traffic = traffic_bytes = None
    if dom in captured and a.workload == "ellipsoid":
        traffic_bytes = captured[dom] * (mesh.nn * len(solver.harmonics)) / (20497 * 32)
        traffic = round(traffic_bytes / (prof[dom][0] * 1e-3) / 1e9, 1)
    roof = {"bound": "hbm", "kernel": names[dom], "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
            "frac": round(ach / peak, 4), "traffic": traffic, "traffic_bytes_per_launch": traffic_bytes,
            "algorithmic_bytes_per_launch": prof[dom][1],
            "traffic_note": ("GB/s of DRAM traffic (read + write) per launch: ncu capture of this kernel on the "
                             "20,497-node x 32-harmonic case scaled by nodes x harmonics") if traffic else None,
            "peak_source": "measured" if pk else "fallback",
            "per_kernel_ms": {names[q]: round(prof[q][0], 3) for q in prof},
            "per_kernel_gbs": {names[q]: round(prof[q][1] / (prof[q][0] * 1e-3) / 1e9, 1) for q in prof}}
    res.update(ms_per_step=ms_step, value=value, e2e=e2e, rep=rep, clocks=clocks, roof=roof, mesh=mesh, w=w,
               launches=launches, tuned=tuned)
    # the secondary measurements build plans of their own: release this one's workspace (~80 GB
    # of library allocations) first, and the previous measurement's objects between them
    import gc
    mesh._solver = None
    del solver, fw
    gc.collect()
    if world > 1:
        dist.barrier()
    if rank == 0 and not a.no_secondary:
        res["plain"] = _guarded("plain FP64 per-RHS", lambda: plain_fp64_per_rhs(mesh))
        res["small"] = _guarded("plain FP64 forward, small", plain_fp64_small_bench)
        res["tg"] = _guarded("sensitivity", tg_jacobian_bench)
        res["lm"] = _guarded("LM step", lambda: lm_step_bench(grid_mm=a.lm_grid_mm))
        res["recon"] = _guarded("LM reconstruction", lambda: lm_recon_bench(grid_mm=a.lm_grid_mm))
        res["uneven"] = _guarded("uneven batch", uneven_bench)
        res["grad500k"] = _guarded("500k-node gradient", grad_big_bench)
    return res


def main():
    a = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if a.impl == "reference":
        if rank != 0:
            return
        w = workload(a.workload, order=a.order)
        for _ in range(a.warmup):
            cpu_sample(w, tol=a.tol)
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
    if a.only:
        torch.cuda.set_device(local_rank)
        out = {"tg": tg_jacobian_bench, "small": plain_fp64_small_bench,
               "lm": lambda: lm_step_bench(grid_mm=a.lm_grid_mm),
               "recon": lambda: lm_recon_bench(grid_mm=a.lm_grid_mm), "uneven": uneven_bench,
               "grad500k": grad_big_bench, "tgk": lambda: tg_kernels_bench(h=a.tgk_h),
               "chol": lambda: cholesky_bench(n=a.chol_n)}[a.only]()
        print(json.dumps(out))
        return
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
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
            "higher_is_better": True, "scaling": "strong" if world > 1 else "weak", "vs_baseline": None,
            "dtype": "c64+f64 refinement", "data": "synthetic",
            "config": {"workload": w["name"], "nodes": mesh.nn, "tets": int(w["mesh"].ne), "nnz": mesh.fem.nnz,
                       "sources": len(w["src"]), "harmonics": w["nf"], "tol": a.tol, "inner_tol": a.inner_tol,
                       "inner_solver": a.inner,
                       "iterations": rep.iterations, "refinements": rep.refinements,
                       "max_rel_residual": rep.max_rel_residual, "l2": "inputs larger than L2 (vectors ~GB)",
                       "parallelism": f"harmonics split over {world} GPUs (k = r mod {world}), detector data "
                                      f"all-gathered every step" if world > 1 else "single GPU",
                       "node_order": a.order, "autotuned": r["tuned"],
                       "iteration_loop": "host-polled" if a.host_loop else "device-driven (graph WHILE node)"},
            "e2e": r["e2e"], "roofline": r["roof"], "cpu_baseline": cpu, "clocks": r["clocks"],
            "gpu_launches": r["launches"],
            "plain_fp64_per_rhs": r.get("plain"), "plain_fp64_small": r.get("small"), "tg_jacobian": r.get("tg"),
            "lm_step": r.get("lm"), "lm_recon": r.get("recon"), "uneven": r.get("uneven"),
            "grad500k": r.get("grad500k"),
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
