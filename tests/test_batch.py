"""Uneven batches (dogpup_b200.batch): the harmonic chunking on the CPU, and on
the GPU a batch of three meshes of different sizes, source and harmonic counts,
chunked by a small memory budget and run on 3 streams, against each problem
solved alone (FP64 to 1e-12: data 1e-9, TG vjp 1e-6 relative)."""
import numpy as np
import pytest

from dogpup_b200.batch import harmonic_chunks, plan_bytes


def test_harmonic_chunks_cover_and_fit():
    n, nnz, nnzG, ns = 50_000, 750_000, 400_000, 64
    for nf in (1, 16, 128):
        for budget in (plan_bytes(n, nnz, nnzG, 1, ns), 3 * plan_bytes(n, nnz, nnzG, 1, ns), 10 ** 12):
            ch = harmonic_chunks(nf, n, nnz, nnzG, ns, budget)
            assert sum(ch, []) == list(range(nf))
            assert all(len(c) >= 1 for c in ch)
            if budget >= plan_bytes(n, nnz, nnzG, 1, ns):
                assert all(plan_bytes(n, nnz, nnzG, len(c), ns) <= budget * 1.0001 or len(c) == 1 for c in ch)
    # tiny budget: one harmonic per chunk
    assert harmonic_chunks(5, n, nnz, nnzG, ns, 1) == [[0], [1], [2], [3], [4]]


@pytest.mark.gpu
def test_uneven_batch_matches_single_solves():
    import torch
    from dogpup_b200 import api, meshgen, workloads
    from dogpup_b200.autograd import gate_coefficients
    from dogpup_b200.batch import UnevenBatch
    cases = [workloads.small_fwd(seed=1, ns=3, nd=4, nf=6), workloads.small_fwd(seed=2, ns=5, nd=2, nf=9)]
    m = meshgen.ellipsoid_mesh((20.0, 16.0, 14.0), 1.5, jitter=0.2, seed=3)
    c3 = dict(cases[0], mesh=m, mua=np.full(m.nn, 0.01), musp=np.full(m.nn, 1.0),
              src=workloads.ring(4, np.zeros(3), (10.0, 8.0), 0.0), det=workloads.ring(3, np.zeros(3), (10.0, 8.0), 0.0, 0.5),
              link=workloads.all_pairs(4, 3), nf=4)
    cases.append(c3)
    meshes = [workloads.build_dmesh(w) for w in cases]
    rng = np.random.default_rng(0)
    gates, ups = [], []
    for w, mesh in zip(cases, meshes):
        gates.append(gate_coefficients(w["t"], [0.5e-9, 1.0e-9], 250e-12, mesh.optode.fAxis))
        ups.append(rng.standard_normal((len(w["link"]), 2)))
    small = max(plan_bytes(mm.nn, mm.fem.nnz, mm.fem.nnz // 2 + mm.nn, 5, 1) for mm in meshes)
    B = UnevenBatch(meshes, budget_bytes=3 * small, streams=3, precision="fp64", tol=1e-12, gates=gates,
                    upstream=ups)
    assert len(B.tasks) > len(meshes)                      # the budget forced harmonic chunks
    res = B.run()
    for mesh, g, u, r in zip(meshes, gates, ups, res):
        phi, data = mesh.flu_solve(precision="fp64", tol=1e-12)
        d0 = data.cpu().numpy()
        assert np.abs(r.data.cpu().numpy() - d0).max() <= 1e-9 * np.abs(d0).max()
        phiA = mesh.adj_flu_solve(precision="fp64", tol=1e-12)
        v0 = api.jacobian_tg_vjp(mesh.nodal_basis(), phi, phiA, mesh.optode.s_fpsf, mesh._link(), g,
                                 len(mesh.optode.tAxis), torch.as_tensor(u, device="cuda")).cpu().numpy()
        assert np.linalg.norm(r.vjp.cpu().numpy() - v0) <= 1e-6 * np.linalg.norm(v0)
