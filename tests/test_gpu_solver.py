"""GPU parity of assembly, FSAI, SpMM and the batched solver against the oracle.

Tolerances: integer/index data (CSR pattern, boundary flags, FSAI pattern)
must match exactly; FP64 values to 1e-12 relative (different summation
order); the FP64 solver to 1e-9 of the oracle's own BiCGSTAB; the
mixed-precision solver to 1e-6 relative fluence error against a sparse-direct
complex128 solve (the accuracy bar of the mixed mode).
"""
import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

C_VAC = 2.99792458e11


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.fixture(scope="module")
def gpu_case(small_case, torch):
    from dogpup_b200 import api
    m = small_case["mesh"]
    fem = api.Fem(torch.as_tensor(m.node), torch.as_tensor(m.elem), 1.4)
    K, M = fem.assemble(torch.as_tensor(small_case["mua"]), torch.as_tensor(small_case["musp"]))
    return dict(fem=fem, K=K, M=M)


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


def test_fem_pattern_and_values(small_case, gpu_case):
    from oracle.fem import robin_faces
    K0, M0 = small_case["K"], small_case["M"]
    fem = gpu_case["fem"]
    assert np.array_equal(fem.rowptr.cpu().numpy(), K0.indptr)
    assert np.array_equal(fem.col.cpu().numpy(), K0.indices)
    assert np.array_equal(fem.bnd.cpu().numpy().astype(bool), small_case["mesh"].bnd)
    assert fem.n_robin_faces == robin_faces(small_case["mesh"].elem, small_case["geo"]["bnd"]).shape[0]
    K, M = gpu_case["K"].cpu().numpy(), gpu_case["M"].cpu().numpy()
    assert np.abs(K - K0.data).max() <= 1e-13 * np.abs(K0.data).max()
    assert np.abs(M - M0.data).max() <= 1e-13 * np.abs(M0.data).max()
    # bitwise-symmetric assembly
    Kg = sp.csr_matrix((K, K0.indices, K0.indptr), shape=K0.shape)
    assert abs(Kg - Kg.T).max() == 0.0


def test_fem_rejects_degenerate_tet(torch):
    from dogpup_b200 import api, DgpError
    node = torch.tensor([[0., 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], dtype=torch.float64)
    elem = torch.tensor([[0, 1, 2, 3]], dtype=torch.int32)
    with pytest.raises(DgpError):
        api.Fem(node, elem, 1.4)


def test_solver_and_fsai_reject_a_bad_pattern(gpu_case, torch):
    """A CSR column outside [0, n) or a decreasing row pointer is DGP_ERR_MESH at solver
    creation, in dgp_fsai_pattern and in dgp_fsai_factor (G pattern), before any kernel
    indexes with it; a row pointer that does not end at nnz is DGP_ERR_MESH at creation."""
    from dogpup_b200 import api, DgpError
    from dogpup_b200._lib import lib
    fem = gpu_case["fem"]
    n = fem.nn
    K, M = gpu_case["K"], gpu_case["M"]
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    bad_col = fem.col.clone()
    bad_col[5] = n
    bad_row = fem.rowptr.clone()
    bad_row[3] = bad_row[4] + 1
    for rp, cl, msg in ((fem.rowptr, bad_col, "column index out of range"), (bad_row, fem.col, "must start at 0")):
        with pytest.raises(DgpError) as ei:
            api.Solver(rp, cl, K, M, dfc, 2, 2)
        assert ei.value.code == 4 and msg in str(ei.value)
        rpg = torch.empty(n + 1, dtype=torch.int32, device="cuda")
        assert lib.dgp_fsai_pattern(api.ptr(rp), api.ptr(cl), api.ptr(K), api.ptr(M), dfc, n, 30, api.ptr(rpg), None,
                                    api.stream_ptr()) == 4
        G = torch.empty((1, int(cl.numel())), dtype=torch.complex128, device="cuda")
        assert lib.dgp_fsai_factor(api.ptr(fem.rowptr), api.ptr(fem.col), api.ptr(K), api.ptr(M), dfc, n, api.ptr(rp),
                                   api.ptr(cl), 1, api.ptr(torch.view_as_real(G)), api.stream_ptr()) == 4
    with pytest.raises(DgpError) as ei:
        api.Solver(fem.rowptr, fem.col[:-1].contiguous(), K, M, dfc, 2, 2)
    assert ei.value.code == 4 and "not at nnz" in str(ei.value)


def test_fsai_pattern_and_factor(small_case, gpu_case, torch):
    from dogpup_b200 import api
    from dogpup_b200._lib import lib, check
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    nf = 5
    fem = gpu_case["fem"]
    n = fem.nn
    rpg = torch.empty(n + 1, dtype=torch.int32, device="cuda")
    check(lib.dgp_fsai_pattern(api.ptr(fem.rowptr), api.ptr(fem.col), api.ptr(gpu_case["K"]), api.ptr(gpu_case["M"]),
                               dfc, n, 30, api.ptr(rpg), None, api.stream_ptr()))
    nnzG = int(rpg[-1].item())
    colg = torch.empty(nnzG, dtype=torch.int32, device="cuda")
    check(lib.dgp_fsai_pattern(api.ptr(fem.rowptr), api.ptr(fem.col), api.ptr(gpu_case["K"]), api.ptr(gpu_case["M"]),
                               dfc, n, 30, api.ptr(rpg), api.ptr(colg), api.stream_ptr()))
    A = sp.tril(K0 + 1j * dfc * M0).tocsr()
    r0, c0 = osv.fsai_pattern(A)
    assert np.array_equal(rpg.cpu().numpy(), r0) and np.array_equal(colg.cpu().numpy(), c0)
    G = torch.empty((nf, nnzG), dtype=torch.complex128, device="cuda")
    check(lib.dgp_fsai_factor(api.ptr(fem.rowptr), api.ptr(fem.col), api.ptr(gpu_case["K"]), api.ptr(gpu_case["M"]),
                              dfc, n, api.ptr(rpg), api.ptr(colg), nf, api.ptr(torch.view_as_real(G)),
                              api.stream_ptr()))
    G0 = osv.fsai_factor(sp.tril(K0).tocsr(), sp.tril(dfc * M0).tocsr(), r0, c0, nf)
    assert rel(G.cpu().numpy().T, G0) < 1e-12


def test_spmm_A_matches_smv(small_case, gpu_case, torch):
    from dogpup_b200 import api
    from dogpup_b200._lib import lib, check
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    dfc = 1e-3
    nf, ns = 4, 8
    n = K0.shape[0]
    rng = np.random.default_rng(5)
    X = rng.standard_normal((nf, n, ns)) + 1j * rng.standard_normal((nf, n, ns))
    KM = torch.stack([gpu_case["K"], gpu_case["M"]], dim=1).contiguous()
    om = torch.arange(nf, dtype=torch.float64, device="cuda") * dfc
    Xd = torch.as_tensor(X, device="cuda")
    Y = torch.empty_like(Xd)
    check(lib.dgp_spmm_A(api.ptr(gpu_case["fem"].rowptr), api.ptr(gpu_case["fem"].col), api.ptr(KM), api.ptr(om), n,
                         nf, ns, api.ptr(torch.view_as_real(Xd)), api.ptr(torch.view_as_real(Y)), api.stream_ptr()))
    Y0 = osv.smv(np.transpose(X, (1, 2, 0)), np.arange(nf, dtype=float), K0, dfc * M0)
    assert rel(np.transpose(Y.cpu().numpy(), (1, 2, 0)), Y0) < 1e-13


def _point_sources(small_case, ns, seed):
    m = small_case["mesh"]
    rng = np.random.default_rng(seed)
    eid = rng.choice(m.ne, ns, replace=False)
    w = rng.random((ns, 4))
    w /= w.sum(axis=1, keepdims=True)
    return m.elem[eid].astype(np.int32), w


@pytest.mark.parametrize("ns", [3, 16])
def test_solver_fp64_matches_oracle_bicgstab(small_case, gpu_case, torch, ns):
    from dogpup_b200 import api
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    nf = 6
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    nodes, w = _point_sources(small_case, ns, 7)
    fpsf = np.exp(-0.2j * np.arange(nf)) * (1.0 + 0.1 * np.arange(nf))
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
    opts = api.make_opts(tol=1e-12, maxit=1000, precision="fp64", check_every=1)
    X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                             torch.as_tensor(fpsf, device="cuda"), opts)
    Q = np.zeros((K0.shape[0], ns, nf), complex)
    for s in range(ns):
        Q[nodes[s], s, :] = w[s][:, None] * fpsf[None, :]
    pc = osv.FsaiPrecond(K0, M0, dfc, nf)
    x0, it0 = osv.bicgstab_fsai(pc, Q, 1e-12, 1000)
    Xh = np.transpose(X.cpu().numpy(), (1, 2, 0))
    assert abs(rep.iterations - it0) <= 1
    assert rel(Xh, x0) < 1e-9
    xd = osv.direct_solve(K0, M0, dfc, Q)
    assert rel(Xh, xd) < 1e-9
    assert rep.max_rel_residual < 1e-10


def test_solver_dense_rhs_and_status(small_case, gpu_case, torch):
    from dogpup_b200 import api
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    nf, ns = 3, 4
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    n = K0.shape[0]
    rng = np.random.default_rng(9)
    B = rng.standard_normal((nf, n, ns)) + 1j * rng.standard_normal((nf, n, ns))
    B[:, :, 2] = 0  # a zero right-hand side column is solved exactly by x = 0
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
    status = torch.full((nf * ns,), -1, dtype=torch.int32, device="cuda")
    X, rep = S.solve(torch.as_tensor(B, device="cuda"), api.make_opts(tol=1e-11, precision="fp64"), status=status)
    xd = osv.direct_solve(K0, M0, dfc, np.transpose(B, (1, 2, 0)))
    assert rel(np.transpose(X.cpu().numpy(), (1, 2, 0)), xd) < 1e-8
    assert (status.cpu().numpy() == 0).all()
    assert np.abs(X[:, :, 2].cpu().numpy()).max() == 0.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_solver_flags_a_nonfinite_column(small_case, gpu_case, torch, precision):
    """A right-hand side column holding a NaN is frozen as DGP_COL_NONFINITE and the call
    returns DGP_ERR_NOT_CONVERGED (reported with the status words, not raised); the other
    columns are unaffected and converge; tol = 0 and maxit = 0 are DGP_ERR_ARG."""
    from dogpup_b200 import api, DgpError
    from dogpup_b200._lib import lib
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    nf, ns = 2, 3
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    n = K0.shape[0]
    rng = np.random.default_rng(4)
    B = rng.standard_normal((nf, n, ns)) + 1j * rng.standard_normal((nf, n, ns))
    B[1, 17, 1] = np.nan
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
    status = torch.full((nf * ns,), -1, dtype=torch.int32, device="cuda")
    Bd = torch.as_tensor(B, device="cuda")
    X = torch.empty_like(Bd)
    rep = api._lib.SolveReport()
    rep.d_status = api.ptr(status)
    o = api.make_opts(tol=1e-10, precision=precision)
    rc = lib.dgp_solve(S._h, api.ptr(api.as_real(Bd)), api.ptr(api.as_real(X)), ns, api.C.byref(o),
                       api.C.byref(rep), api.stream_ptr())
    assert rc == 5 and rep.n_not_converged == 1
    st = status.cpu().numpy().reshape(nf, ns)
    assert st[1, 1] == 4 and (np.delete(st.ravel(), ns + 1) == 0).all()
    B2 = B.copy()
    B2[1, :, 1] = 0
    xd = np.transpose(osv.direct_solve(K0, M0, dfc, np.transpose(B2, (1, 2, 0))), (2, 0, 1))
    Xh = X.cpu().numpy()
    for k in range(nf):
        for s in range(ns):
            if (k, s) != (1, 1):
                assert rel(Xh[k, :, s], xd[k, :, s]) < 1e-6, (k, s)
    for bad in (dict(tol=0.0), dict(tol=1e-10, maxit=0)):
        with pytest.raises(DgpError) as ei:
            S.solve(torch.as_tensor(np.nan_to_num(B), device="cuda"), api.make_opts(precision=precision, **bad))
        assert ei.value.code == 1


@pytest.mark.parametrize("precision", ["mixed", "mixed_bicgstab"])
def test_solver_mixed_precision_accuracy(small_case, gpu_case, torch, precision):
    """Both complex-FP32 inner solvers (COCG, BiCGSTAB) refined in FP64 reach the
    sparse-direct solution."""
    from dogpup_b200 import api
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    nf, ns = 8, 16
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    nodes, w = _point_sources(small_case, ns, 13)
    fpsf = np.exp(-0.3j * np.arange(nf))
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
    opts = api.make_opts(tol=1e-10, precision=precision, inner_tol=1e-4)
    X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                             torch.as_tensor(fpsf, device="cuda"), opts)
    Q = np.zeros((K0.shape[0], ns, nf), complex)
    for s in range(ns):
        Q[nodes[s], s, :] = w[s][:, None] * fpsf[None, :]
    xd = osv.direct_solve(K0, M0, dfc, Q)
    Xh = np.transpose(X.cpu().numpy(), (1, 2, 0))
    # per right-hand side relative error
    err = np.linalg.norm(Xh - xd, axis=0) / np.linalg.norm(xd, axis=0)
    assert err.max() < 1e-6, err.max()
    assert rep.max_rel_residual < 1e-10
    assert rep.refinements >= 2


def test_solver_reports_maxit(small_case, gpu_case, torch):
    from dogpup_b200 import api
    nf, ns = 2, 2
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], 1e-4, nf, ns)
    nodes, w = _point_sources(small_case, ns, 1)
    status = torch.full((nf * ns,), -1, dtype=torch.int32, device="cuda")
    X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                             torch.ones(nf, dtype=torch.complex128, device="cuda"),
                             api.make_opts(tol=1e-14, maxit=2, precision="fp64", check_every=1), status=status)
    assert rep.iterations == 2
    assert (status.cpu().numpy() == 1).all()
    assert np.isfinite(X.cpu().numpy()).all()


@pytest.mark.parametrize("precision", ["mixed", "mixed_bicgstab"])
def test_mixed_solver_stops_at_maxit_with_progress(small_case, gpu_case, torch, precision):
    """maxit reached inside an inner solve: the iterations done so far still enter X (for
    COCG the last x update is applied after the stop), the statuses say maxit and the true
    FP64 residual has fallen."""
    from dogpup_b200 import api
    nf, ns = 4, 4
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
    nodes, w = _point_sources(small_case, ns, 3)
    status = torch.full((nf * ns,), -1, dtype=torch.int32, device="cuda")
    X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                             torch.ones(nf, dtype=torch.complex128, device="cuda"),
                             api.make_opts(tol=1e-12, maxit=5, precision=precision, check_every=1), status=status)
    assert rep.iterations == 5
    assert (status.cpu().numpy() == 1).all()
    assert np.isfinite(X.cpu().numpy()).all() and np.abs(X.cpu().numpy()).max() > 0
    assert rep.max_rel_residual < 0.5


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed_bicgstab"])
def test_solver_harmonic_subset(small_case, gpu_case, torch, precision):
    """A plan over harmonics [5, 0, 9] solves slot j at harmonic h_j: same as the full plan's columns."""
    from dogpup_b200 import api
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    harm = [5, 0, 9]
    ns = 3
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    nodes, w = _point_sources(small_case, ns, 21)
    fpsf_all = np.exp(-0.25j * np.arange(10)) * (1.0 + 0.05 * np.arange(10))
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, len(harm), ns, harmonics=harm)
    opts = api.make_opts(tol=1e-12 if precision == "fp64" else 1e-10, precision=precision)
    X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                             torch.as_tensor(fpsf_all[harm], device="cuda"), opts)
    Q = np.zeros((K0.shape[0], ns, 10), complex)
    for s in range(ns):
        Q[nodes[s], s, :] = w[s][:, None] * fpsf_all[None, :]
    xd = osv.direct_solve(K0, M0, dfc, Q)[:, :, harm]
    Xh = np.transpose(X.cpu().numpy(), (1, 2, 0))
    err = np.linalg.norm(Xh - xd, axis=0) / np.linalg.norm(xd, axis=0)
    assert err.max() < (1e-9 if precision == "fp64" else 1e-6), err.max()
    with pytest.raises(ValueError):
        api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, 2, ns, harmonics=[1])


def test_solver_autotune_then_mixed_accuracy(small_case, gpu_case, torch):
    """The autotuner picks a fitting launch shape; solves after it keep the mixed accuracy bar."""
    from dogpup_b200 import api
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    nf, ns = 6, 16
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    nodes, w = _point_sources(small_case, ns, 31)
    fpsf = np.exp(-0.2j * np.arange(nf))
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
    t = S.autotune()
    assert t["spmm"] in ("tiled", "gather") and t["vec"] in (2, 4, 8) and t["rows"] in (32, 64, 128, 256)
    assert t["kind"] in (0, 1, 2, 3, 4)
    assert t["spmm_ms_per_iteration"] > 0
    opts = api.make_opts(tol=1e-10, precision="mixed")
    X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                             torch.as_tensor(fpsf, device="cuda"), opts)
    Q = np.zeros((K0.shape[0], ns, nf), complex)
    for s in range(ns):
        Q[nodes[s], s, :] = w[s][:, None] * fpsf[None, :]
    xd = osv.direct_solve(K0, M0, dfc, Q)
    err = np.linalg.norm(np.transpose(X.cpu().numpy(), (1, 2, 0)) - xd, axis=0) / np.linalg.norm(xd, axis=0)
    assert err.max() < 1e-6, err.max()


@pytest.mark.parametrize("precision", ["fp64", "mixed", "mixed_bicgstab"])
def test_device_driven_loop_matches_host_polling(small_case, gpu_case, torch, precision):
    """One graph launch per inner solve (WHILE node, the loop ended on the device) against the
    host replaying blocks of iterations and polling the control block: the FP64 solve is the same
    computation (same iteration count, bit-identical fields); the mixed solves may stop their
    inner solves one block apart (the stall guard is checked at block ends on the device), so
    both must meet the 1e-6 fluence bar against the sparse-direct solution."""
    from dogpup_b200 import api
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    nf, ns = 4, 6
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    nodes, w = _point_sources(small_case, ns, 23)
    fpsf = np.exp(-0.1j * np.arange(nf))
    fem = gpu_case["fem"]
    out = {}
    for loop in (True, False):
        S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
        S.set_device_loop(loop)
        X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                                 torch.as_tensor(fpsf, device="cuda"),
                                 api.make_opts(tol=1e-10, precision=precision, check_every=4))
        out[loop] = (X.cpu().numpy(), rep.iterations, rep.max_rel_residual)
        del S
    if precision == "fp64":
        assert out[True][1] == out[False][1]
        assert np.array_equal(out[True][0], out[False][0])
    Q = np.zeros((K0.shape[0], ns, nf), complex)
    for s_ in range(ns):
        Q[nodes[s_], s_, :] = w[s_][:, None] * fpsf[None, :]
    xd = osv.direct_solve(K0, M0, dfc, Q)
    for loop in (True, False):
        x = np.transpose(out[loop][0], (1, 2, 0))
        err = np.linalg.norm(x - xd, axis=0) / np.linalg.norm(xd, axis=0)
        assert err.max() < 1e-6, (loop, err.max())
        assert out[loop][2] < 1e-10


@pytest.mark.parametrize("kind", [1, 2, 3, 4])
@pytest.mark.parametrize("ns,vec", [(3, 2), (16, 4), (40, 8), (64, 4)])
def test_gather_spmm_kinds_solve_to_the_bar(small_case, gpu_case, torch, kind, ns, vec):
    """Each inner-loop kind of the gather SpMM (2 or 4 nonzeros per step with zero-coefficient
    padding, packed FP32 FMAs, harmonic pairs for A -- with 5 harmonics, so the last pair is
    a single harmonic) gives a mixed solve that meets the 1e-6 fluence bar against the
    sparse-direct solution, at lane widths 2, 4, 8 (padded source counts 4, 16, 64); the plan
    reports the kind it was set to."""
    from dogpup_b200 import api
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    nf = 5
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
    S.set_spmm(False, vec=vec, rows=64)
    S.set_spmm_kind(kind)
    assert S.spmm_shape() == {"spmm": "gather", "vec": vec, "rows": 64, "kind": kind}
    nodes, w = _point_sources(small_case, ns, 43)
    fpsf = np.exp(-0.3j * np.arange(nf))
    X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                             torch.as_tensor(fpsf, device="cuda"), api.make_opts(tol=1e-10, precision="mixed"))
    Q = np.zeros((K0.shape[0], ns, nf), complex)
    for s in range(ns):
        Q[nodes[s], s, :] = w[s][:, None] * fpsf[None, :]
    xd = osv.direct_solve(K0, M0, dfc, Q)
    err = np.linalg.norm(np.transpose(X.cpu().numpy(), (1, 2, 0)) - xd, axis=0) / np.linalg.norm(xd, axis=0)
    assert err.max() < 1e-6, err.max()
    with pytest.raises(Exception):
        S.set_spmm_kind(5)


@pytest.mark.parametrize("ns", [3, 16, 40])
def test_tiled_spmm_matches_gather_and_solves(small_case, gpu_case, torch, ns):
    """The tiled SpMM (halo rows in shared memory) equals the gather SpMM up to FP32 summation order,
    and a mixed solve on it meets the 1e-6 fluence bar (padded source counts 4, 16, 64)."""
    from dogpup_b200 import api
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    nf = 5
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
    assert S.check_spmm() < 1e-5
    S.set_spmm(True)
    nodes, w = _point_sources(small_case, ns, 41)
    fpsf = np.exp(-0.4j * np.arange(nf))
    X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                             torch.as_tensor(fpsf, device="cuda"), api.make_opts(tol=1e-10, precision="mixed"))
    Q = np.zeros((K0.shape[0], ns, nf), complex)
    for s in range(ns):
        Q[nodes[s], s, :] = w[s][:, None] * fpsf[None, :]
    xd = osv.direct_solve(K0, M0, dfc, Q)
    err = np.linalg.norm(np.transpose(X.cpu().numpy(), (1, 2, 0)) - xd, axis=0) / np.linalg.norm(xd, axis=0)
    assert err.max() < 1e-6, err.max()
    with pytest.raises(Exception):
        S.set_spmm(False, vec=3)


def test_solver_fp64_per_column_skips_finished_harmonics(small_case, gpu_case, torch):
    """Per-column stopping (columns freeze at tol, finished harmonics leave the sweeps): every column
    still meets tol against the sparse-direct solution, and every status word says converged."""
    from dogpup_b200 import api
    from oracle import solver as osv
    K0, M0 = small_case["K"], small_case["M"]
    nf, ns = 8, 5
    dfc = 2 * np.pi / 10e-9 / (C_VAC / 1.4)
    nodes, w = _point_sources(small_case, ns, 51)
    fpsf = np.exp(-0.3j * np.arange(nf))
    fem = gpu_case["fem"]
    S = api.Solver(fem.rowptr, fem.col, gpu_case["K"], gpu_case["M"], dfc, nf, ns)
    status = torch.full((nf * ns,), -1, dtype=torch.int32, device="cuda")
    X, rep = S.solve_sources(torch.as_tensor(nodes, device="cuda"), torch.as_tensor(w, device="cuda"),
                             torch.as_tensor(fpsf, device="cuda"),
                             api.make_opts(tol=1e-11, precision="fp64", stop_rule="per_column"), status=status)
    Q = np.zeros((K0.shape[0], ns, nf), complex)
    for s in range(ns):
        Q[nodes[s], s, :] = w[s][:, None] * fpsf[None, :]
    xd = osv.direct_solve(K0, M0, dfc, Q)
    err = np.linalg.norm(np.transpose(X.cpu().numpy(), (1, 2, 0)) - xd, axis=0) / np.linalg.norm(xd, axis=0)
    assert err.max() < 1e-8, err.max()
    assert (status.cpu().numpy() == 0).all()
