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
