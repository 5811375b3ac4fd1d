"""Harmonic sharding (dogpup_b200.shard): the partition and its collectives.

On CPU: the partition, empty shares (more ranks than harmonics) and the
all-reduce of partial time-gate sums as gloo ranks, with the transform itself
given by the oracle's fc2tg (same formula, fc2tg.m:25-32) since the device
transform needs a GPU.  On the GPU: the device path itself -- ShardedForward
and ShardedSensitivity with the library's solves, fc2tg and TG Jacobian --
as gloo ranks that share one GPU (their kernels never wait on one another; the
collectives run on the host), against the unsharded result.  Bit-for-bit
agreement is not expected across summation orders: 1e-12 relative for the
transforms, 1e-9 for solved data, 1e-5 for the FP32 Jacobian."""
import os
import socket

import numpy as np
import pytest

from dogpup_b200.shard import harmonic_shard, partial_tg


def _fc2tg(c, gate, nt):
    from oracle.transforms import fc2tg
    return fc2tg(np.asarray(c), gate, None, nt)


def test_harmonic_shard_partitions():
    for nf in (1, 7, 128):
        for world in (1, 2, 3, 8):
            parts = [harmonic_shard(nf, r, world) for r in range(world)]
            assert sorted(sum(parts, [])) == list(range(nf))
            assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        harmonic_shard(8, 2, 2)


def test_partial_tg_sums_to_full_single_process():
    rng = np.random.default_rng(1)
    nm, nf, ng, nt = 5, 11, 3, 201
    c = rng.standard_normal((nm, nf)) + 1j * rng.standard_normal((nm, nf))
    gate = rng.standard_normal((ng, nf)) + 1j * rng.standard_normal((ng, nf))
    full = _fc2tg(c, gate, nt)
    for world in (1, 2, 3):
        tot = sum(partial_tg(c[:, harmonic_shard(nf, r, world)], harmonic_shard(nf, r, world), gate, nt, _fc2tg)
                  for r in range(world))
        assert np.abs(tot - full).max() <= 1e-12 * np.abs(full).max()


def test_empty_share_contributes_zeros():
    """With more ranks than harmonics some shares are empty: their partial sum is zeros of
    the data's shape, and the shares still add up to the full transform."""
    rng = np.random.default_rng(3)
    nm, nf, ng, nt = 3, 2, 4, 51
    c = rng.standard_normal((nm, nf)) + 1j * rng.standard_normal((nm, nf))
    gate = rng.standard_normal((ng, nf)) + 1j * rng.standard_normal((ng, nf))
    world = 3
    assert harmonic_shard(nf, 2, world) == []
    z = partial_tg(c[:, []], [], gate, nt, _fc2tg)
    assert z.shape == (nm, ng) and not z.any()
    tot = sum(partial_tg(c[:, harmonic_shard(nf, r, world)], harmonic_shard(nf, r, world), gate, nt, _fc2tg)
              for r in range(world))
    full = _fc2tg(c, gate, nt)
    assert np.abs(tot - full).max() <= 1e-12 * np.abs(full).max()


def _rank_main(rank, world, port, q, nf=9):
    import torch
    import torch.distributed as dist
    from dogpup_b200.shard import sharded_tg_data
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(7)            # same data on every rank
        nm, ng, nt = 4, 2, 101
        c = rng.standard_normal((nm, nf)) + 1j * rng.standard_normal((nm, nf))
        gate = rng.standard_normal((ng, nf)) + 1j * rng.standard_normal((ng, nf))
        mine = harmonic_shard(nf, rank, world)
        y = sharded_tg_data(c[:, mine], mine, gate, nt, _fc2tg)
        full = _fc2tg(c, gate, nt)
        q.put((rank, float(np.abs(y.numpy() - full).max() / np.abs(full).max())))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spawn(target, world, *args, timeout=120):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = _free_port()
    q = ctx.Queue()
    procs = [ctx.Process(target=target, args=(r, world, port, q) + args) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    return dict(q.get(timeout=5) for _ in procs)


@pytest.mark.parametrize("world,nf", [(2, 9), (3, 2)])
def test_sharded_tg_data_gloo(world, nf):
    """The all-reduce of partial sums as gloo ranks; (3, 2): one rank owns no harmonic and
    still joins the collective with zeros."""
    errs = _spawn(_rank_main, world, nf)
    assert max(errs.values()) <= 1e-12, errs


def _gather_rank_main(rank, world, port, q, nf):
    import torch
    import torch.distributed as dist
    from dogpup_b200.shard import gather_spectra
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(11)
        full = torch.as_tensor(rng.standard_normal((5, nf)) + 1j * rng.standard_normal((5, nf)))
        mine = harmonic_shard(nf, rank, world)
        got = gather_spectra(full[:, mine], nf, rank, world)
        q.put((rank, bool(torch.equal(got, full))))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,nf", [(2, 9), (3, 7), (3, 2)])
def test_gather_spectra_gloo(world, nf):
    """The all-gather of the ranks' harmonic columns rebuilds the full [NM x NF] spectra
    bit for bit on every rank, empty shares included."""
    res = _spawn(_gather_rank_main, world, nf)
    assert all(res.values()), res


@pytest.mark.gpu
def test_sharded_forward_shares_sum_to_full_tg_data():
    """Both shards of a 2-way split run in one process (no process group: each
    returns its partial sum); their sum is the unsharded time-gated data."""
    import torch
    from dogpup_b200 import workloads
    from dogpup_b200.autograd import TimeGatedForward, gate_coefficients
    from dogpup_b200.shard import ShardedForward
    w = workloads.small_fwd(ns=3, nd=4, nf=9)
    mesh = workloads.build_dmesh(w)
    gfc = gate_coefficients(w["t"], [0.4e-9, 0.9e-9], 250e-12, mesh.optode.fAxis)
    full = TimeGatedForward(mesh, gfc, precision="fp64", tol=1e-12).forward_fields(mesh.mua, mesh.musp)[0]
    parts = [ShardedForward(mesh, gfc, r, 2, precision="fp64", tol=1e-12)()[0] for r in range(2)]
    tot = parts[0] + parts[1]
    assert torch.abs(tot - full).max().item() <= 1e-9 * torch.abs(full).max().item()


def _device_rank_main(rank, world, port, q, nf):
    """One gloo rank of the device path on cuda:0: sharded TG data, the all-gathered
    spectra and this rank's voxel block of the reduce-scattered TG Jacobian, each
    against the same quantity computed unsharded in the same process."""
    import torch
    import torch.distributed as dist
    from dogpup_b200 import api, workloads
    from dogpup_b200.autograd import gate_coefficients
    from dogpup_b200.shard import ShardedForward, ShardedSensitivity, gather_spectra
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        w = workloads.small_fwd(ns=3, nd=4, nf=nf)
        mesh = workloads.build_dmesh(w)
        gfc = gate_coefficients(w["t"], [0.4e-9, 0.9e-9, 1.4e-9], 250e-12, mesh.optode.fAxis)
        nt = len(w["t"])
        # unsharded: every harmonic in this process
        phi, data = mesh.flu_solve(precision="fp64", tol=1e-12)
        phiA = mesh.adj_flu_solve(precision="fp64", tol=1e-12)
        tg_full = api.fc2tg(data, gfc, nt)
        J_full = api.jacobian_tg(mesh.nodal_basis(), phi, phiA, mesh.optode.s_fpsf, mesh._link(), gfc, nt, tg_full)
        # sharded: this rank's harmonics, collectives over gloo
        fw = ShardedForward(mesh, gfc, rank, world, precision="fp64", tol=1e-12)
        tg, _ = fw()
        _, own, _ = fw.solve()
        spectra = gather_spectra(own, nf, rank, world)
        sens = ShardedSensitivity(mesh, gfc, rank, world, precision="fp64", tol=1e-12)
        Jblk, tg2, _ = sens(mesh.nodal_basis(), rytov=True)
        nv = mesh.nn
        nb = Jblk.shape[0]
        lo, hi = rank * nb, min((rank + 1) * nb, nv)
        ref = J_full[lo:hi]
        rel = lambda a, b: float(torch.abs(a - b).max() / torch.abs(b).max())
        q.put((rank, {"tg": rel(tg, tg_full), "tg2": rel(tg2, tg_full), "spectra": rel(spectra, data),
                      "J": rel(Jblk[:hi - lo].double(), ref.double()) if hi > lo else 0.0,
                      "pad_zero": bool((Jblk[hi - lo:] == 0).all()), "empty": fw.solver is None}))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("world,nf", [(2, 9), (3, 2)])
def test_sharded_device_path_as_gloo_ranks(world, nf):
    """ShardedForward / ShardedSensitivity on the device under a real process group: TG
    data (all-reduce), spectra (all-gather) and the Rytov TG Jacobian's voxel blocks
    (reduce-scatter) equal the unsharded results; with 3 ranks and 2 harmonics one rank
    owns nothing and contributes zeros."""
    res = _spawn(_device_rank_main, world, nf, timeout=300)
    for r, e in res.items():
        assert e["tg"] <= 1e-9 and e["tg2"] <= 1e-9 and e["spectra"] <= 1e-9, (r, e)
        assert e["J"] <= 1e-5 and e["pad_zero"], (r, e)
    assert any(e["empty"] for e in res.values()) == (world > nf)
