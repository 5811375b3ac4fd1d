"""LM reconstruction loop (dogpup_b200.recon): id_thresh on the CPU against
its definition; on the GPU a small case with one spherical absorber, where the
loop must reduce the data misfit and the mua error at every iteration, and the
split-BF16 normal equations must track the all-FP64 normal equations (mua
within 1 % relative after each iteration)."""
import numpy as np
import pytest

from dogpup_b200.recon import id_thresh


def test_id_thresh_rules():
    t = np.linspace(0, 1, 11)
    curve = np.exp(-((t - 0.3) / 0.15) ** 2)[None, :] * np.array([[1.0], [5.0]])
    d = curve + 0.5                                   # range normalisation removes offset and scale
    allm = id_thresh(d, "all")
    dn = (curve - curve.min(1, keepdims=True)) / np.ptp(curve, axis=1, keepdims=True)
    assert np.array_equal(allm, dn > 0.01)
    m = id_thresh(d, 0.8)
    peak = np.argmax(dn, axis=1)
    for r in range(2):
        for g in range(11):
            assert m[r, g] == (g >= peak[r] and 0.01 < dn[r, g] <= 0.8)
    with pytest.raises(ValueError):
        id_thresh(d, "some")


@pytest.mark.gpu
def test_lm_recon_reduces_error_and_split_bf16_tracks_fp64():
    import torch
    from dogpup_b200 import api, workloads
    from dogpup_b200.autograd import gate_coefficients
    from dogpup_b200.recon import LMRecon
    w = workloads.small_fwd(ns=8, nd=8, nf=32)
    node = w["mesh"].node
    c = node.mean(0)
    truth = np.full(w["mesh"].nn, 0.01)
    truth[((node - c) ** 2).sum(1) < 4.0 ** 2] = 0.02
    w["mua"] = truth
    mesh = workloads.build_dmesh(w)
    gfc = gate_coefficients(w["t"], 0.6e-9 + 0.25e-9 * np.arange(8), 250e-12, mesh.optode.fAxis)
    _, data = mesh.flu_solve(precision="fp64", tol=1e-12)
    data_m = api.fc2tg(data, gfc, len(w["t"])).cpu().numpy()
    lo, hi = node.min(0), node.max(0)
    mesh.mesh2grid(*[np.arange(lo[d] - 1, hi[d] + 1.001, 2.5) for d in range(3)])
    runs = {}
    for ne in ("split_bf16", "fp64"):
        mesh.mua = torch.full((mesh.nn,), 0.01, dtype=torch.float64, device="cuda")
        mesh.update_properties()
        rec = LMRecon(mesh, gfc, precision="fp64", tol=1e-10, normal_eq=ne)
        runs[ne] = rec.run(data_m, lam=(1e-2, 0), thresh="all", max_iter=3,
                           truth=torch.as_tensor(truth, device="cuda"))
    h = runs["split_bf16"]
    assert "stopped" not in h and len(h["mua"]) >= 2
    # the reference's damping floor (lambda >= residual norm) makes the steps short: the
    # misfit and the mua error must fall monotonically, not by a given factor
    assert all(b < a for a, b in zip(h["err"], h["err"][1:]))
    assert all(b < a for a, b in zip(h["err_truth"], h["err_truth"][1:]))
    for a, b in zip(runs["split_bf16"]["mua"], runs["fp64"]["mua"]):
        assert (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item() < 1e-2


@pytest.mark.gpu
def test_target_spots_and_reshape_weights_against_oracle():
    """Spots on the device equal the oracle's to 1e-14; reshape_J's w from the
    split-BF16 J J^T within 2e-3 (norm-wise relative, lam 0.1), from FP64 1e-9."""
    import torch
    from oracle.jacobian import reshape_j, target_spots as spots0
    from dogpup_b200.recon import reshape_J, target_spots
    g = np.stack(np.meshgrid(np.arange(12.0), np.arange(9.0), np.arange(7.0), indexing="ij"), -1).reshape(-1, 3)
    inm = ((g - [5.5, 4, 3]) ** 2 / [30, 16, 9]).sum(1) < 1
    pos = [[5, 4, 3], [8, 2, 2.5], [3, 6, 4]]
    for kind, wd in (("gauss", 1.5), ("square", 3.0)):
        t = target_spots(g, inm, pos, wd, kind).cpu().numpy()
        assert np.abs(t - spots0(g, inm, pos, wd, kind)).max() < 1e-14
    rng = np.random.default_rng(2)
    nv, nm, ns = 3000, 500, 12
    Jt = torch.as_tensor(rng.standard_normal((nv, nm)), device="cuda", dtype=torch.float32)
    Js = torch.as_tensor(rng.standard_normal((ns, nv)), device="cuda")
    w0 = reshape_j(Jt.double().cpu().numpy().T, Js.cpu().numpy(), 0.1)
    for mode, tol in (("split_bf16", 2e-3), ("fp64", 1e-9)):
        w = reshape_J(Jt if mode == "split_bf16" else Jt.double(), Js, 0.1, mode).cpu().numpy()
        assert np.linalg.norm(w - w0) / np.linalg.norm(w0) < tol, mode


@pytest.mark.gpu
def test_lm_recon_with_target_spots():
    """wghtd_LM_recon's reshaped branch: spots at the absorber and around it; the
    reshaped misfit falls and the split-BF16 run tracks the FP64 one."""
    import torch
    from dogpup_b200 import api, workloads
    from dogpup_b200.autograd import gate_coefficients
    from dogpup_b200.recon import LMRecon
    w = workloads.small_fwd(ns=8, nd=8, nf=32)
    node = w["mesh"].node
    c = node.mean(0)
    truth = np.full(w["mesh"].nn, 0.01)
    truth[((node - c) ** 2).sum(1) < 4.0 ** 2] = 0.02
    w["mua"] = truth
    mesh = workloads.build_dmesh(w)
    gfc = gate_coefficients(w["t"], 0.6e-9 + 0.25e-9 * np.arange(8), 250e-12, mesh.optode.fAxis)
    _, data = mesh.flu_solve(precision="fp64", tol=1e-12)
    data_m = api.fc2tg(data, gfc, len(w["t"])).cpu().numpy()
    lo, hi = node.min(0), node.max(0)
    mesh.mesh2grid(*[np.arange(lo[d] - 1, hi[d] + 1.001, 2.5) for d in range(3)])
    pos = np.array([c, c + [6, 0, 0], c - [6, 0, 0], c + [0, 6, 0], c - [0, 6, 0], c + [0, 0, 4]])
    runs = {}
    for ne in ("split_bf16", "fp64"):
        mesh.mua = torch.full((mesh.nn,), 0.01, dtype=torch.float64, device="cuda")
        mesh.update_properties()
        rec = LMRecon(mesh, gfc, precision="fp64", tol=1e-10, normal_eq=ne)
        runs[ne] = rec.run(data_m, lam=(1e-2, 1e-2), thresh="all", max_iter=3, pos_s=pos)
    h = runs["split_bf16"]
    assert "stopped" not in h and len(h["mua"]) >= 1
    assert h["err"][-1] < h["err"][0]
    assert all(torch.isfinite(m).all() for m in h["mua"])
    for a, b in zip(runs["split_bf16"]["mua"], runs["fp64"]["mua"]):
        assert (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item() < 2e-2


@pytest.mark.gpu
def test_lm_loop_against_oracle_with_two_step_backs_in_a_row():
    """The LM loop's control flow against the oracle's restatement of wghtd_LM_recon
    (oracle/recon.py) on a scripted model whose misfit falls, rises twice in a row, then
    falls: both step-back iterations reuse the Jacobian cached at the last accepted step,
    normalised by that step's G (wghtd_LM_recon.m:103-116, :165-166), and rescale the update
    by the new G.  FP64 normal equations; the device maps m2g / g2m (dgp_csr_spmv) and the
    FP64 Cholesky against NumPy: mua after every update to 1e-10, lambda and misfit exactly
    as the oracle's up to rounding."""
    import types

    import scipy.sparse as sp
    import torch
    from dogpup_b200.recon import LMRecon, _flat
    from oracle.recon import lm_loop

    rng = np.random.default_rng(17)
    nn, nv, nm, ng = 60, 40, 12, 4
    m2g = sp.random(nv, nn, density=0.08, random_state=3, format="csr") + sp.eye(nv, nn, format="csr")
    m2g = sp.diags(1.0 / np.asarray(m2g.sum(1)).ravel()) @ m2g                    # rows sum to 1
    g2m = sp.random(nn, nv, density=0.1, random_state=4, format="csr") + sp.eye(nn, nv, format="csr")
    g2m = sp.diags(1.0 / np.maximum(np.asarray(g2m.sum(1)).ravel(), 1e-300)) @ g2m
    data_m = np.exp(5.0 + 0.5 * rng.standard_normal((nm, ng)))
    r = rng.standard_normal((nm, ng))
    eps = [1.0, 0.6, 0.8, 0.9, 0.4, 0.3, 0.25]           # misfit scale per model call
    Js = [300.0 * rng.standard_normal((nv, ng * nm)) for _ in eps]   # normalised J ~ 3: small steps
    mua0 = 0.01 + 0.002 * rng.random(nn)

    def scripted(q):
        return data_m * np.exp(-eps[q] * r), Js[q]      # data [NM][NG], J^T [NV][NG*NM] in x(:) order

    mesh = types.SimpleNamespace(
        mua=torch.as_tensor(mua0, device="cuda"), gridinmesh=np.ones(nv, bool), m2g=m2g, g2m=g2m, dxyz=1.0,
        optode=types.SimpleNamespace(tAxis=np.arange(11.0)), update_properties=lambda: None)

    class Scripted(LMRecon):
        calls = 0

        def model(self):
            d, J = scripted(self.calls)
            self.calls += 1
            return torch.as_tensor(d, device="cuda"), torch.as_tensor(J, device="cuda")

    rec = Scripted(mesh, np.ones((ng, 8), complex), precision="fp64", normal_eq="fp64")
    h = rec.run(data_m, lam=(1.0, 0.0), thresh="all", max_iter=5)

    mask = id_thresh(data_m, "all") & (data_m > 0)
    incl = np.nonzero(mask.T.ravel())[0]
    dm = np.log(_flat(torch.as_tensor(data_m)).numpy())[incl]
    h0 = lm_loop(lambda q: (_flat(torch.as_tensor(scripted(q)[0])).numpy(), scripted(q)[1].T),
                 mua0, m2g, g2m, dm, incl, 1.0, max_iter=5)
    deltas = np.sign(h0["err_del"])
    assert list(deltas[:3]) == [-1, 1, 1]                # fall, then two rises in a row
    assert h["exit"] == h0["exit"] == "max_iter" and h["iterations"] == h0["iterations"] == 5
    assert np.allclose(h["err"], h0["err"], rtol=1e-12, atol=0)
    assert np.allclose(h["lam"], h0["lam"], rtol=1e-12, atol=0)
    assert len(h["mua"]) == len(h0["mua"]) == 5
    for a, b in zip(h["mua"], h0["mua"]):
        assert np.abs(a.cpu().numpy() - b).max() <= 1e-10 * np.abs(b).max()
