"""GPU J^T W J (split-BF16 tcgen05), damping, J^T W y and the FP64 Cholesky solve.

Tolerances: H from the three-term BF16 split with FP32 accumulation, 3e-5
norm-wise relative; J^T W y (FP64) 1e-12; the Cholesky solve on an exact
FP64 matrix 1e-10 (one or many right-hand sides); the whole LM step against the all-FP64 oracle
(tik_inv with W), 1e-3.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _v(t):
    return C.c_void_p(t.data_ptr())


def _case(nv, nm, seed):
    rng = np.random.default_rng(seed)
    J = rng.standard_normal((nm, nv)) * np.exp(rng.uniform(-2, 2, nv))[None, :]
    W = rng.uniform(0.5, 2.0, nm)
    y = rng.standard_normal(nm)
    return J, W, y


@pytest.mark.parametrize("nv,nm", [(300, 1000), (128, 64), (257, 777)])
def test_normal_equations_match_fp64(nv, nm):
    import torch
    from dogpup_b200._lib import lib, check
    J, W, y = _case(nv, nm, nv + nm)
    Jt = torch.as_tensor(np.ascontiguousarray(J.T), dtype=torch.float32, device="cuda")
    Jf = Jt.cpu().numpy().T.astype(np.float64)          # the FP32 values actually used
    Wd = torch.as_tensor(W, device="cuda")
    yd = torch.as_tensor(y, device="cuda")
    H = torch.zeros((nv, nv), dtype=torch.float64, device="cuda")
    rhs = torch.zeros(nv, dtype=torch.float64, device="cuda")
    lam = 0.1
    check(lib.dgp_normal_eq(_v(Jt), nv, nm, _v(Wd), _v(yd), lam, 0, _v(H), nv, _v(rhs), None))
    H0 = Jf.T @ (W[:, None] * Jf)
    d = np.diag(H0).copy()
    H0[np.diag_indices(nv)] = d + lam * d.max()
    Hl = np.tril(H.cpu().numpy())
    err = np.linalg.norm(Hl - np.tril(H0)) / np.linalg.norm(np.tril(H0))
    assert err < 3e-5, err
    r0 = Jf.T @ (W * y)
    assert np.linalg.norm(rhs.cpu().numpy() - r0) / np.linalg.norm(r0) < 1e-12


@pytest.mark.parametrize("n,pad", [(333, 0), (1100, 7), (2501, 3), (3333, 0), (128, 0), (129, 1)])
def test_cholesky_solve_exact_matrix(n, pad):
    """n > 128 crosses the 128-column panels (diagonal factor + inverse, panel GEMM, trailing
    lower-triangle GEMM on the FP64 tensor cores) with a partial last panel; n > 1536 crosses the
    outer panels (the rows under each one, their update of the rest); pad > 0 tests ldh > n, and
    an odd ldh (n = 333, 1100, 3333) takes the 8-byte copy path of the GEMM; the strict upper
    triangle holds NaN and must never be read.  Solution 1e-10 against NumPy, L L^T 1e-13."""
    import torch
    from dogpup_b200._lib import lib, check
    rng = np.random.default_rng(3)
    A = rng.standard_normal((n, n))
    H0 = A @ A.T + n * np.eye(n)
    b = rng.standard_normal(n)
    ldh = n + pad
    Hp = np.full((n, ldh), np.nan)
    Hp[:, :n] = np.tril(H0)
    Hp[:, :n][np.triu_indices(n, 1)] = np.nan        # the strict upper triangle is never read
    H = torch.as_tensor(Hp, device="cuda").contiguous()
    x = torch.as_tensor(b, device="cuda").clone()
    check(lib.dgp_cholesky_solve(_v(H), n, ldh, _v(x), None))
    x0 = np.linalg.solve(H0, b)
    assert np.linalg.norm(x.cpu().numpy() - x0) / np.linalg.norm(x0) < 1e-10
    L = np.tril(H.cpu().numpy()[:, :n])
    assert np.linalg.norm(L @ L.T - H0) / np.linalg.norm(H0) < 1e-13


@pytest.mark.parametrize("n,nrhs,padx", [(333, 7, 5), (600, 40, 0)])
def test_cholesky_solve_many_right_hand_sides(n, nrhs, padx):
    """One factorisation, nrhs right-hand sides as the rows of X [nrhs][ldx]; ldx > n keeps
    the pad columns untouched."""
    import torch
    from dogpup_b200._lib import lib, check
    rng = np.random.default_rng(11)
    A = rng.standard_normal((n, n))
    H0 = A @ A.T + n * np.eye(n)
    B = rng.standard_normal((nrhs, n))
    ldx = n + padx
    Xp = np.full((nrhs, ldx), 7.0)
    Xp[:, :n] = B
    H = torch.as_tensor(np.tril(H0), device="cuda").contiguous()
    X = torch.as_tensor(Xp, device="cuda").contiguous()
    check(lib.dgp_cholesky_solve_many(_v(H), n, n, _v(X), nrhs, ldx, None))
    X0 = np.linalg.solve(H0, B.T).T
    Xh = X.cpu().numpy()
    assert np.linalg.norm(Xh[:, :n] - X0) / np.linalg.norm(X0) < 1e-10
    assert (Xh[:, n:] == 7.0).all()


@pytest.mark.parametrize("n,bad", [(70, 0), (600, 530)])
def test_cholesky_rejects_indefinite_matrix(n, bad):
    import torch
    from dogpup_b200._lib import lib
    d = np.ones(n)
    d[bad] = -1.0
    H = torch.as_tensor(np.diag(d), device="cuda").contiguous()
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    assert lib.dgp_cholesky_solve(_v(H), n, n, _v(x), None) == 1


def test_lm_step_against_fp64_tik_inv():
    import torch
    from dogpup_b200._lib import lib, check
    from oracle.jacobian import tik_inv
    nv, nm = 400, 2048
    J, W, y = _case(nv, nm, 7)
    Jt = torch.as_tensor(np.ascontiguousarray(J.T), dtype=torch.float32, device="cuda")
    H = torch.zeros((nv, nv), dtype=torch.float64, device="cuda")
    x = torch.zeros(nv, dtype=torch.float64, device="cuda")
    Wd = torch.as_tensor(W, device="cuda")   # kept alive: the library reads these pointers
    yd = torch.as_tensor(y, device="cuda")
    lam = 1e-2
    check(lib.dgp_normal_eq(_v(Jt), nv, nm, _v(Wd), _v(yd), lam, 0, _v(H), nv, _v(x), None))
    check(lib.dgp_cholesky_solve(_v(H), nv, nv, _v(x), None))
    u0 = tik_inv(Jt.cpu().numpy().T.astype(np.float64), lam, y, weights=W)
    assert np.linalg.norm(x.cpu().numpy() - u0) / np.linalg.norm(u0) < 1e-3


@pytest.mark.parametrize("nv,nm", [(1500, 700), (400, 2048)])
def test_lm_update_both_forms_match_tik_inv(nv, nm):
    """dgp_lm_update in the unknowns' form (nv x nv) and the measurements' form
    (nmeas x nmeas, J_w^T (J_w J_w^T + mu I)^-1 W^1/2 y) gives tik_inv's update
    with W within 1e-3; form 0 picks the smaller system."""
    import ctypes as C
    import torch
    from dogpup_b200._lib import lib, check
    from oracle.jacobian import tik_inv
    J, W, y = _case(nv, nm, 11)
    Jt = torch.as_tensor(np.ascontiguousarray(J.T), dtype=torch.float32, device="cuda")
    Wd = torch.as_tensor(W, device="cuda")
    yd = torch.as_tensor(y, device="cuda")
    lam = 1e-2
    u0 = tik_inv(Jt.cpu().numpy().T.astype(np.float64), lam, y, weights=W)
    for form in (1, 2, 0):
        x = torch.zeros(nv, dtype=torch.float64, device="cuda")
        used = C.c_int32(-1)
        check(lib.dgp_lm_update(_v(Jt), nv, nm, _v(Wd), _v(yd), lam, _v(x), form, C.byref(used), None))
        assert used.value == (form if form else (2 if nm < nv else 1))
        assert np.linalg.norm(x.cpu().numpy() - u0) / np.linalg.norm(u0) < 1e-3, form


def test_lm_update_rejects_bad_weights_in_both_forms():
    """A negative or non-finite data weight is DGP_ERR_ARG in the unknowns' form
    and in the measurements' form alike (the latter takes W^1/2, so an unchecked
    weight would surface as NaN instead)."""
    import torch
    from dogpup_b200._lib import lib
    nv, nm = 300, 200
    J, W, y = _case(nv, nm, 3)
    Jt = torch.as_tensor(np.ascontiguousarray(J.T), dtype=torch.float32, device="cuda")
    yd = torch.as_tensor(y, device="cuda")
    for bad in (-1.0, float("nan")):
        Wb = W.copy()
        Wb[17] = bad
        Wd = torch.as_tensor(Wb, device="cuda")
        for form in (1, 2):
            x = torch.zeros(nv, dtype=torch.float64, device="cuda")
            assert lib.dgp_lm_update(_v(Jt), nv, nm, _v(Wd), _v(yd), 1e-2, _v(x), form, None, None) == 1, (bad, form)


@pytest.mark.parametrize("na,nv,nm", [(1, 5, 3), (6, 1000, 777), (13, 2049, 300)])
def test_times_jt_against_numpy(na, nv, nm):
    """dgp_times_jt (the Js J^T product of reshape_J): FP64 accumulation of an FP64 left factor
    and the FP32 Jacobian, against NumPy in FP64 on the same FP32 values, 1e-12; spot counts
    that are not multiples of its 8-row groups and voxel counts across its 256-voxel chunks."""
    import torch
    from dogpup_b200._lib import lib, check
    rng = np.random.default_rng(na + nv)
    A = rng.standard_normal((na, nv))
    Jt = rng.standard_normal((nv, nm)).astype(np.float32)
    out = torch.empty((na, nm), dtype=torch.float64, device="cuda")
    Ad, Jd = torch.as_tensor(A, device="cuda"), torch.as_tensor(Jt, device="cuda")
    check(lib.dgp_times_jt(_v(Ad), na, nv, _v(Jd), nm, _v(out), None))
    ref = A @ Jt.astype(np.float64)
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max()
