"""Harmonic sharding (dogpup_b200.shard): the partition and the one collective
(all-reduce of partial time-gate sums), as world_size-2 gloo ranks on CPU.
The device transform is stood in for by the oracle's fc2tg (same formula,
fc2tg.m:100-111); bit-for-bit agreement is not expected across summation
orders, so the check is 1e-12 relative."""
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


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from dogpup_b200.shard import sharded_tg_data
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(7)            # same data on every rank
        nm, nf, ng, nt = 4, 9, 2, 101
        c = rng.standard_normal((nm, nf)) + 1j * rng.standard_normal((nm, nf))
        gate = rng.standard_normal((ng, nf)) + 1j * rng.standard_normal((ng, nf))
        mine = harmonic_shard(nf, rank, world)
        y = sharded_tg_data(c[:, mine], mine, gate, nt, _fc2tg)
        full = _fc2tg(c, gate, nt)
        q.put((rank, float(np.abs(y.numpy() - full).max() / np.abs(full).max())))
    finally:
        dist.destroy_process_group()


def test_sharded_tg_data_gloo_world2():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    errs = dict(q.get(timeout=5) for _ in procs)
    assert max(errs.values()) <= 1e-12, errs


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
