"""Parity at the bench's full size (ellipsoid 90x75x70 mm @1.2 mm, 153,327 nodes,
64 sources x 128 harmonics, mixed precision to 1e-8) through size-independent
properties: the FP64 residual of the returned fluence, recomputed independently
with the standalone FP64 operator, meets tol for every column of sampled
harmonics; the solver's own report agrees; and sampled columns match FP64
solves to 1e-12 within the mixed-precision bar (1e-6 per right-hand side).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HARM = [0, 37, 127]


@pytest.fixture(scope="module")
def full():
    from dogpup_b200 import workloads
    w = workloads.ellipsoid_fwd()
    mesh = workloads.build_dmesh(w)
    phi, data, rep = mesh.flu_solve(precision="mixed", tol=1e-8, inner_tol=3e-5, return_report=True)
    yield dict(w=w, mesh=mesh, phi=phi, data=data, rep=rep)
    mesh._solver = None


def _rhs(mesh, harm, ns):
    """Dense right-hand sides b[h][node][s] = w[s,l] * fpsf[h] of the point sources."""
    import torch
    nodes, wts = mesh._sources(mesh.optode.s_bary)
    fp = mesh.optode.s_fpsf[harm]
    B = torch.zeros((len(harm), mesh.nn, ns), dtype=torch.complex128, device="cuda")
    for s in range(nodes.shape[0]):
        for q in range(4):
            B[:, nodes[s, q], s] += wts[s, q] * fp
    return B


def test_fullsize_residual_recomputed_in_fp64(full):
    import torch
    from dogpup_b200 import api
    from dogpup_b200._lib import lib, check
    mesh, phi, rep = full["mesh"], full["phi"], full["rep"]
    assert mesh.nn == 153327 and phi.shape == (128, 153327, 64)
    assert rep.n_not_converged == 0 and rep.max_rel_residual < 1e-8
    X = phi[HARM].contiguous()
    KM = torch.stack([mesh.K, mesh.M], dim=1).contiguous()
    om = torch.as_tensor(np.array(HARM, dtype=np.float64) * (mesh.optode.df / mesh.c), device="cuda")
    Y = torch.empty_like(X)
    check(lib.dgp_spmm_A(api.ptr(mesh.fem.rowptr), api.ptr(mesh.fem.col), api.ptr(KM), api.ptr(om), mesh.nn,
                         len(HARM), 64, api.ptr(torch.view_as_real(X)), api.ptr(torch.view_as_real(Y)),
                         api.stream_ptr()))
    B = _rhs(mesh, HARM, 64)
    res = torch.linalg.vector_norm(B - Y, dim=1) / torch.linalg.vector_norm(B, dim=1)     # [harm][source]
    assert float(res.max()) < 1e-8, float(res.max())


def test_fullsize_columns_match_fp64(full):
    import torch
    from dogpup_b200 import api
    mesh, phi = full["mesh"], full["phi"]
    S = api.Solver(mesh.fem.rowptr, mesh.fem.col, mesh.K, mesh.M, mesh.optode.df / mesh.c, len(HARM), 2,
                   harmonics=HARM)
    nodes, wts = mesh._sources(mesh.optode.s_bary[[0, 40]])
    ref, rep = S.solve_sources(nodes, wts, mesh.optode.s_fpsf[HARM].contiguous(),
                               api.make_opts(tol=1e-12, precision="fp64"))
    assert rep.n_not_converged == 0
    got = phi[HARM][:, :, [0, 40]]
    err = torch.linalg.vector_norm(got - ref, dim=1) / torch.linalg.vector_norm(ref, dim=1)
    assert float(err.max()) < 1e-6, float(err.max())
