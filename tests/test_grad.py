"""Reverse-mode gradient of time-gated data: oracle pinned by finite differences
(CPU), then the device path against the oracle and against finite differences
of the device forward model (GPU).

Tolerances (relative to max |gradient|): oracle vs central differences 1e-6
(step 1e-4 * mua, sparse-direct solves); device pieces vs oracle on the same
fields 1e-11 (FP64 throughout, only summation order differs); device
autograd vs central differences of the device forward 1e-6 (FP64 BiCGSTAB to
1e-13); mixed-precision solves 1e-4.
"""
import numpy as np
import pytest

from dogpup_b200.meshgen import cylinder_mesh
from oracle import fem, grad, solver

DFC = 2 * np.pi / 10e-9 / (2.99792458e11 / 1.4)


def _tiny_problem(seed=5):
    m = cylinder_mesh(6, 8, 1.5, jitter=0.2, seed=2)
    geo = fem.prepare_mesh(m.node, m.elem, 1.4)
    rng = np.random.default_rng(seed)
    mua = 0.01 * (1 + 0.3 * rng.random(m.nn))
    musp = 1.0 + 0.2 * rng.random(m.nn)

    def bary(n):
        e = rng.integers(0, m.elem.shape[0], n)
        w = rng.random((n, 4))
        w[0, 3] = 0.0        # a zero detector weight, skipped as meas_flu does
        w /= w.sum(1, keepdims=True)
        return np.concatenate([e[:, None].astype(float), w], 1)

    sb, db = bary(2), bary(3)
    link = np.array([[0, 0], [0, 2], [1, 1], [1, 2]])
    nf, ng, nt = 4, 3, 201
    fpsf = rng.standard_normal(nf) + 1j * rng.standard_normal(nf)
    gate = rng.standard_normal((ng, nf)) + 1j * rng.standard_normal((ng, nf))
    g = rng.standard_normal((len(link), ng))
    return dict(m=m, geo=geo, mua=mua, musp=musp, sb=sb, db=db, link=link, nt=nt, fpsf=fpsf, gate=gate, g=g,
                rng=rng)


def test_oracle_adjoint_gradient_matches_finite_differences():
    p = _tiny_problem()
    m, geo = p["m"], p["geo"]
    args = (DFC, p["sb"], p["db"], p["link"], p["fpsf"], p["gate"], p["nt"])
    y, phi, (K, M) = grad.tg_forward(m.node, m.elem, geo, p["mua"], p["musp"], *args)
    B = grad.tg_adjoint_rhs(m.elem, p["db"], p["link"], p["gate"], p["nt"], p["g"], m.nn, 2)
    lam = solver.direct_solve(K, M, DFC, B)
    gm, gs = grad.adjoint_grad(m.node, m.elem, geo, p["mua"], p["musp"], phi, lam)

    def L(a, s):
        return float((p["g"] * grad.tg_forward(m.node, m.elem, geo, a, s, *args)[0]).sum())

    for v in p["rng"].choice(m.nn, 5, replace=False):
        e = np.zeros(m.nn)
        e[v] = 1.0
        d = 1e-4 * p["mua"][v]
        fd_a = (L(p["mua"] + d * e, p["musp"]) - L(p["mua"] - d * e, p["musp"])) / (2 * d)
        fd_s = (L(p["mua"], p["musp"] + d * e) - L(p["mua"], p["musp"] - d * e)) / (2 * d)
        assert abs(gm[v] - fd_a) < 1e-6 * abs(gm).max()
        assert abs(gs[v] - fd_s) < 1e-6 * abs(gs).max()


def test_oracle_kappa_fixed_gradient_is_the_absorption_jacobian():
    """grad_mua - grad_musp equals -Re sum lam^T M_v phi, M_v the consistent absorption mass of node v."""
    p = _tiny_problem(seed=9)
    m, geo = p["m"], p["geo"]
    args = (DFC, p["sb"], p["db"], p["link"], p["fpsf"], p["gate"], p["nt"])
    _, phi, (K, M) = grad.tg_forward(m.node, m.elem, geo, p["mua"], p["musp"], *args)
    B = grad.tg_adjoint_rhs(m.elem, p["db"], p["link"], p["gate"], p["nt"], p["g"], m.nn, 2)
    lam = solver.direct_solve(K, M, DFC, B)
    gm, gs = grad.adjoint_grad(m.node, m.elem, geo, p["mua"], p["musp"], phi, lam)
    # K(mua + e_v, musp - e_v) - K(mua, musp) is linear in e_v: the absorption block of node v
    for v in p["rng"].choice(m.nn, 3, replace=False):
        e = np.zeros(m.nn)
        e[v] = 1.0
        K1, _ = fem.gen_fwdmat(m.node, m.elem, geo, p["mua"] + e, p["musp"] - e)
        dK = (K1 - K).tocsr()
        ref = -sum(np.real((lam[:, s, k] @ (dK @ phi[:, s, k]))) for s in range(2) for k in range(phi.shape[2]))
        assert abs((gm[v] - gs[v]) - ref) < 1e-10 * abs(gm).max()


# ------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def dev_case():
    import torch
    from dogpup_b200 import workloads
    from dogpup_b200.autograd import TimeGatedForward, gate_coefficients
    w = workloads.small_fwd(ns=3, nd=4, nf=8)
    rng = np.random.default_rng(3)
    w["mua"] = 0.01 * (1 + 0.3 * rng.random(w["mesh"].nn))
    w["musp"] = 1.0 + 0.2 * rng.random(w["mesh"].nn)
    mesh = workloads.build_dmesh(w)
    gfc = gate_coefficients(w["t"], [0.4e-9, 0.8e-9, 1.2e-9], 250e-12, mesh.optode.fAxis)
    model = TimeGatedForward(mesh, gfc, precision="fp64", tol=1e-13)
    mua = torch.as_tensor(w["mua"], device="cuda")
    musp = torch.as_tensor(w["musp"], device="cuda")
    g = torch.as_tensor(rng.standard_normal((len(w["link"]), 3)), device="cuda")
    return dict(w=w, mesh=mesh, gfc=gfc, model=model, mua=mua, musp=musp, g=g, rng=rng)


def _oracle_geo(mesh):
    return fem.prepare_mesh(mesh.node_host, mesh.elem_host, mesh.nr)


@pytest.mark.gpu
def test_device_adjoint_pieces_match_oracle(dev_case):
    import torch
    from dogpup_b200 import api
    mesh, model = dev_case["mesh"], dev_case["model"]
    y, phi, _ = model.forward_fields(dev_case["mua"], dev_case["musp"])
    nf, n, ns = phi.shape
    B = api.tg_adjoint_rhs(*model.det, model.link, model.gate_fc, model.nt, dev_case["g"], n, nf, ns)
    B0 = grad.tg_adjoint_rhs(mesh.elem_host, mesh.optode.d_bary, mesh.optode.link, dev_case["gfc"].cpu().numpy(),
                             model.nt, dev_case["g"].cpu().numpy(), n, ns)
    Bh = np.transpose(B.cpu().numpy(), (1, 2, 0))
    assert np.abs(Bh - B0).max() <= 1e-12 * np.abs(B0).max()
    lam = torch.as_tensor(dev_case["rng"].standard_normal(phi.shape) + 1j * dev_case["rng"].standard_normal(phi.shape),
                          device="cuda")
    gm, gs = api.fem_adjoint_grad(mesh.fem, dev_case["mua"], dev_case["musp"], phi, lam)
    tr = lambda t: np.transpose(t.cpu().numpy(), (1, 2, 0))
    gm0, gs0 = grad.adjoint_grad(mesh.node_host, mesh.elem_host, _oracle_geo(mesh), dev_case["w"]["mua"],
                                 dev_case["w"]["musp"], tr(phi), tr(lam))
    assert np.abs(gm.cpu().numpy() - gm0).max() <= 1e-11 * np.abs(gm0).max()
    assert np.abs(gs.cpu().numpy() - gs0).max() <= 1e-11 * np.abs(gs0).max()


@pytest.mark.gpu
def test_device_forward_matches_oracle_forward(dev_case):
    mesh, model = dev_case["mesh"], dev_case["model"]
    y, _, _ = model.forward_fields(dev_case["mua"], dev_case["musp"])
    o = mesh.optode
    y0, _, _ = grad.tg_forward(mesh.node_host, mesh.elem_host, _oracle_geo(mesh), dev_case["w"]["mua"],
                               dev_case["w"]["musp"], o.df / mesh.c, o.s_bary, o.d_bary, o.link,
                               o.s_fpsf.cpu().numpy(), dev_case["gfc"].cpu().numpy(), model.nt)
    assert np.abs(y.cpu().numpy() - y0).max() <= 1e-9 * np.abs(y0).max()


@pytest.mark.gpu
def test_device_autograd_matches_finite_differences(dev_case):
    import torch
    model, g = dev_case["model"], dev_case["g"]
    mua = dev_case["mua"].clone().requires_grad_(True)
    musp = dev_case["musp"].clone().requires_grad_(True)
    L = (model(mua, musp) * g).sum()
    L.backward()
    gm, gs = mua.grad.cpu().numpy(), musp.grad.cpu().numpy()
    n = gm.shape[0]

    def Lf(a, s):
        with torch.no_grad():
            return float((model(a, s) * g).sum())

    for v in dev_case["rng"].choice(n, 4, replace=False):
        e = torch.zeros(n, dtype=torch.float64, device="cuda")
        e[v] = 1.0
        d = 1e-4 * float(dev_case["mua"][v])
        a0, s0 = dev_case["mua"], dev_case["musp"]
        fd_a = (Lf(a0 + d * e, s0) - Lf(a0 - d * e, s0)) / (2 * d)
        fd_s = (Lf(a0, s0 + d * e) - Lf(a0, s0 - d * e)) / (2 * d)
        fd_k = (Lf(a0 + d * e, s0 - d * e) - Lf(a0 - d * e, s0 + d * e)) / (2 * d)
        assert abs(gm[v] - fd_a) < 1e-6 * np.abs(gm).max()
        assert abs(gs[v] - fd_s) < 1e-6 * np.abs(gs).max()
        assert abs((gm[v] - gs[v]) - fd_k) < 1e-6 * np.abs(gm).max()


@pytest.mark.gpu
def test_device_autograd_recompute_equals_stored(dev_case):
    from dogpup_b200.autograd import TimeGatedForward
    rec = TimeGatedForward(dev_case["mesh"], dev_case["gfc"], precision="fp64", tol=1e-13, recompute=True)
    out = []
    for model in (dev_case["model"], rec):
        mua = dev_case["mua"].clone().requires_grad_(True)
        musp = dev_case["musp"].clone().requires_grad_(True)
        (model(mua, musp) * dev_case["g"]).sum().backward()
        out.append((mua.grad.cpu().numpy(), musp.grad.cpu().numpy()))
    # the same solves on the same matrices; only the order of the FP64 atomic
    # partial sums inside the solver's dot products may differ between runs
    for a, b in zip(out[0], out[1]):
        assert np.abs(a - b).max() <= 1e-10 * np.abs(a).max()


@pytest.mark.gpu
def test_device_autograd_mixed_precision(dev_case):
    import torch
    from dogpup_b200.autograd import TimeGatedForward
    ref = dev_case["model"]
    mixed = TimeGatedForward(dev_case["mesh"], dev_case["gfc"], precision="mixed", tol=1e-10)
    out = []
    for model in (ref, mixed):
        mua = dev_case["mua"].clone().requires_grad_(True)
        (model(mua, dev_case["musp"]) * dev_case["g"]).sum().backward()
        out.append(mua.grad.cpu().numpy())
    assert np.abs(out[1] - out[0]).max() <= 1e-4 * np.abs(out[0]).max()
