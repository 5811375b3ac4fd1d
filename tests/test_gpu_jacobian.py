"""GPU Jacobian, TG Jacobian and vjp against the oracle's J_complex restatement.

Tolerances (norm-wise relative): complex Jacobian 1e-6 and TG Jacobian 1e-5
(fields are staged in complex FP32, sums accumulate in FP32 / FP64); the vjp
against the explicit J^T g from the same Jacobian, 1e-5.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def jac_case():
    import torch
    from dogpup_b200 import workloads, api
    from oracle.transforms import td2fc
    w = workloads.small_fwd(ns=4, nd=5, nf=16)
    mesh = workloads.build_dmesh(w)
    phi, data = mesh.flu_solve(precision="fp64", tol=1e-12)
    phiA = mesh.adj_flu_solve(precision="fp64", tol=1e-12)
    t = w["t"]
    sd = 250e-12 / (2 * np.sqrt(2 * np.log(2)))
    gates = np.stack([np.exp(-(t - (0.3e-9 + q * 250e-12)) ** 2 / (2 * sd ** 2)) for q in range(20)])
    gfc = td2fc(gates, mesh.optode.fAxis, t)
    lo, hi = w["mesh"].node.min(0), w["mesh"].node.max(0)
    xs = [np.arange(lo[d] - 2, hi[d] + 2.001, 2.0) for d in range(3)]
    mesh.mesh2grid(*xs)
    return dict(w=w, mesh=mesh, phi=phi, phiA=phiA, gfc=gfc, gates=gates,
                gfc_d=torch.as_tensor(gfc, device="cuda"))


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


def _oracle_J(case, P, wts):
    from oracle.jacobian import j_complex
    mesh = case["mesh"]
    phi = np.transpose(case["phi"].cpu().numpy(), (1, 2, 0))     # [NN, NS, NF]
    phiA = np.transpose(case["phiA"].cpu().numpy(), (1, 2, 0))
    return j_complex(P, wts, phi, phiA, mesh.optode.link, mesh.optode.s_fpsf.cpu().numpy())


def test_complex_jacobian_voxel_basis(jac_case):
    mesh = jac_case["mesh"]
    J, data, _, _ = mesh.J_complex(jac_case["phi"], jac_case["phiA"])
    J0 = _oracle_J(jac_case, mesh.m2g, mesh.dxyz ** 3)             # [NM, NF, NV]
    assert rel(np.transpose(J.cpu().numpy(), (2, 1, 0)), J0) < 1e-6


def test_tg_jacobian_and_rytov(jac_case):
    from oracle.jacobian import j_tg
    from oracle.transforms import fc2tg
    mesh = jac_case["mesh"]
    nt = len(mesh.optode.tAxis)
    J0 = j_tg(_oracle_J(jac_case, mesh.m2g, mesh.dxyz ** 3), jac_case["gfc"], nt)   # [NM, NG, NV]
    Jt, _ = mesh.J_tg(jac_case["gfc_d"], jac_case["phi"], jac_case["phiA"])
    assert rel(np.transpose(Jt.cpu().numpy(), (2, 1, 0)), J0) < 1e-5
    Jr, dtg = mesh.J_tg(jac_case["gfc_d"], jac_case["phi"], jac_case["phiA"], rytov=True)
    d0 = fc2tg(mesh.meas_flu(jac_case["phi"]).cpu().numpy(), jac_case["gfc"], None, nt)
    assert rel(dtg.cpu().numpy(), d0) < 1e-12
    assert rel(np.transpose(Jr.cpu().numpy(), (2, 1, 0)), J0 / d0[:, :, None]) < 1e-5


def test_vjp_matches_explicit_jacobian_nodal(jac_case):
    import torch
    from dogpup_b200 import api
    mesh = jac_case["mesh"]
    nb = mesh.nodal_basis()
    nt = len(mesh.optode.tAxis)
    link = mesh._link()
    Jt = api.jacobian_tg(nb, jac_case["phi"], jac_case["phiA"], mesh.optode.s_fpsf, link, jac_case["gfc_d"], nt)
    rng = np.random.default_rng(0)
    g = rng.standard_normal((link.shape[0], 20))
    v = api.jacobian_tg_vjp(nb, jac_case["phi"], jac_case["phiA"], mesh.optode.s_fpsf, link, jac_case["gfc_d"], nt,
                            torch.as_tensor(g))
    explicit = np.einsum("vgm,mg->v", Jt.cpu().numpy().astype(np.float64), g)
    assert rel(v.cpu().numpy(), explicit) < 1e-5
    # nodal basis = the identity interpolation with lumped-mass weights
    lump = nb.w.cpu().numpy()
    import scipy.sparse as sp
    from oracle.jacobian import j_tg
    J0 = j_tg(_oracle_J(jac_case, sp.identity(mesh.nn, format="csr"), lump), jac_case["gfc"], nt)
    assert rel(np.transpose(Jt.cpu().numpy(), (2, 1, 0)), J0) < 1e-5


@pytest.mark.parametrize("ng", [3, 20, 29])
def test_tg_jacobian_odd_sizes(ng):
    """Odd harmonic x optode counts (the staged fields end at an odd complex offset) and gate
    counts that pad to 8, 24 and 32: TG Jacobian and vjp against the oracle."""
    import scipy.sparse as sp
    import torch
    from dogpup_b200 import api, workloads
    from oracle.jacobian import j_complex, j_tg
    from oracle.transforms import td2fc
    w = workloads.small_fwd(ns=3, nd=4, nf=5)
    mesh = workloads.build_dmesh(w)
    phi, _ = mesh.flu_solve(precision="fp64", tol=1e-12)
    phiA = mesh.adj_flu_solve(precision="fp64", tol=1e-12)
    t = w["t"]
    gates = np.stack([np.exp(-(t - (0.3e-9 + q * 150e-12)) ** 2 / (2 * (100e-12) ** 2)) for q in range(ng)])
    gfc = td2fc(gates, mesh.optode.fAxis, t)
    nb = mesh.nodal_basis()
    link = mesh._link()
    nt = len(t)
    Jt = api.jacobian_tg(nb, phi, phiA, mesh.optode.s_fpsf, link, torch.as_tensor(gfc, device="cuda"), nt)
    P = sp.identity(mesh.nn, format="csr")
    J0 = j_tg(j_complex(P, nb.w.cpu().numpy(), np.transpose(phi.cpu().numpy(), (1, 2, 0)),
                        np.transpose(phiA.cpu().numpy(), (1, 2, 0)), mesh.optode.link,
                        mesh.optode.s_fpsf.cpu().numpy()), gfc, nt)
    assert rel(np.transpose(Jt.cpu().numpy(), (2, 1, 0)), J0) < 1e-5
    g = np.random.default_rng(1).standard_normal((link.shape[0], ng))
    v = api.jacobian_tg_vjp(nb, phi, phiA, mesh.optode.s_fpsf, link, torch.as_tensor(gfc, device="cuda"), nt,
                            torch.as_tensor(g))
    assert rel(v.cpu().numpy(), np.einsum("mgv,mg->v", J0, g)) < 1e-5


def test_jacobian_rejects_bad_link_and_basis(jac_case):
    """Link entries outside [0, ns) x [0, nd) are DGP_ERR_ARG; basis columns outside [0, nn)
    and basis rows of more than 8 entries are DGP_ERR_MESH -- all raised before a kernel
    addresses shared memory or the fields with them."""
    import scipy.sparse as sp
    import torch
    from dogpup_b200 import api
    from dogpup_b200._lib import DgpError
    mesh = jac_case["mesh"]
    phi, phiA = jac_case["phi"], jac_case["phiA"]
    nt = len(mesh.optode.tAxis)
    nn, ns, nd = phi.shape[1], phi.shape[2], phiA.shape[2]
    link = mesh._link()
    nb = mesh.nodal_basis()
    for j, bad in ((0, ns), (1, nd), (0, -1)):
        lk = link.clone()
        lk[2, j] = bad
        with pytest.raises(DgpError) as ei:
            api.jacobian_tg(nb, phi, phiA, mesh.optode.s_fpsf, lk, jac_case["gfc_d"], nt)
        assert ei.value.code == 1 and "link index out of range" in str(ei.value)
    P = sp.csr_matrix((np.full(3, 1 / 3), ([0, 1, 2], [0, 1, 2])), shape=(3, nn))
    b = api.Basis(P, np.ones(3))
    b.col[1] = nn
    with pytest.raises(DgpError) as ei:
        api.jacobian_complex(b, phi, phiA, mesh.optode.s_fpsf, link)
    assert ei.value.code == 4 and "column index out of range" in str(ei.value)
    P9 = sp.csr_matrix((np.full(9, 1 / 9), (np.zeros(9, int), np.arange(9))), shape=(2, nn))
    gin = torch.zeros((link.shape[0], jac_case["gfc_d"].shape[0]), dtype=torch.float64)
    with pytest.raises(DgpError) as ei:
        api.jacobian_tg_vjp(api.Basis(P9, np.ones(2)), phi, phiA, mesh.optode.s_fpsf, link, jac_case["gfc_d"], nt, gin)
    assert ei.value.code == 4 and "more than 8 entries" in str(ei.value)
    J = api.jacobian_complex(api.Basis(P, np.ones(3)), phi, phiA, mesh.optode.s_fpsf, link)
    assert torch.isfinite(torch.view_as_real(J)).all()


@pytest.fixture
def cuda_core_engine():
    """use(e) selects the Jacobian engines (1 CUDA cores, 2 tensor cores where the shapes fit);
    the default (0) is restored after the test."""
    from dogpup_b200._lib import lib, check

    def use(engine):
        check(lib.dgp_set_jacobian_engine(engine))
    yield use
    use(0)


@pytest.mark.parametrize("ns,nd,nf,ng,shuffle", [(32, 32, 64, 20, False), (7, 5, 33, 29, True),
                                                 (13, 11, 17, 3, False), (9, 16, 80, 32, True),
                                                 (9, 16, 80, 12, True), (32, 32, 48, 24, True)])
def test_tg_jacobian_tensor_cores_match_cuda_cores_and_oracle(ns, nd, nf, ng, shuffle, cuda_core_engine):
    """The tcgen05 TG Jacobian (3xTF32 split, FP32 accumulate in tensor memory) and the CUDA-core
    FP32 kernel, each against the FP64 oracle: link counts that are not multiples of the 128-link
    tile (1024, 28, 143, 115, 819), harmonic counts that are not multiples of the 16-harmonic
    chunk, gate counts from 3 to 32, and shuffled, partial link tables (not all source-detector
    pairs, in no particular order).  NF = 80 with 32 gates does not fit the tensor-core kernel's
    shared memory, so engine 2 runs the CUDA-core kernel there too.  Bar: 1e-5 norm-wise against the oracle (the
    TG Jacobian's tolerance); between the engines 1e-5 per link, relative to the link's largest
    entry.  The vjp of both engines (the tensor-core one runs for up to 32 sources and detectors)
    against the oracle's J^T g, 1e-5.  (Without the Rytov division: early gates carry TG data
    near zero, where dividing FP32 entries by it magnifies their rounding.)"""
    import scipy.sparse as sp
    import torch
    from dogpup_b200 import api, workloads
    from oracle.jacobian import j_complex, j_tg
    from oracle.transforms import td2fc
    w = workloads.small_fwd(ns=ns, nd=nd, nf=nf)
    if shuffle:
        rng = np.random.default_rng(ns + nd)
        keep = rng.permutation(len(w["link"]))[: max(1, 4 * len(w["link"]) // 5)]
        w["link"] = w["link"][keep]
    mesh = workloads.build_dmesh(w)
    phi, data = mesh.flu_solve(precision="fp64", tol=1e-12)
    phiA = mesh.adj_flu_solve(precision="fp64", tol=1e-12)
    t = w["t"]
    gates = np.stack([np.exp(-(t - (0.3e-9 + q * 120e-12)) ** 2 / (2 * (90e-12) ** 2)) for q in range(ng)])
    gfc = td2fc(gates, mesh.optode.fAxis, t)
    gfc_d = torch.as_tensor(gfc, device="cuda")
    nb = mesh.nodal_basis()
    link = mesh._link()
    nt = len(t)
    cuda_core_engine(2)
    J_tc = api.jacobian_tg(nb, phi, phiA, mesh.optode.s_fpsf, link, gfc_d, nt)
    cuda_core_engine(1)
    J_cc = api.jacobian_tg(nb, phi, phiA, mesh.optode.s_fpsf, link, gfc_d, nt)
    cuda_core_engine(0)
    J0 = j_tg(j_complex(sp.identity(mesh.nn, format="csr"), nb.w.cpu().numpy(),
                        np.transpose(phi.cpu().numpy(), (1, 2, 0)), np.transpose(phiA.cpu().numpy(), (1, 2, 0)),
                        mesh.optode.link, mesh.optode.s_fpsf.cpu().numpy()), gfc, nt)
    e_cc = rel(np.transpose(J_cc.cpu().numpy(), (2, 1, 0)), J0)
    e_tc = rel(np.transpose(J_tc.cpu().numpy(), (2, 1, 0)), J0)
    assert e_cc < 1e-5 and e_tc < 1e-5, (e_cc, e_tc)
    a, b = J_tc.double(), J_cc.double()
    per_link = ((a - b).abs().amax(dim=(0, 1)) / b.abs().amax(dim=(0, 1))).max().item()
    assert per_link < 1e-5, per_link
    g = np.random.default_rng(nf).standard_normal((link.shape[0], ng))
    g_d = torch.as_tensor(g, device="cuda")
    cuda_core_engine(2)
    v_tc = api.jacobian_tg_vjp(nb, phi, phiA, mesh.optode.s_fpsf, link, gfc_d, nt, g_d).cpu().numpy()
    cuda_core_engine(1)
    v_cc = api.jacobian_tg_vjp(nb, phi, phiA, mesh.optode.s_fpsf, link, gfc_d, nt, g_d).cpu().numpy()
    cuda_core_engine(0)
    v0 = np.einsum("mgv,mg->v", J0, g)
    assert rel(v_cc, v0) < 1e-5 and rel(v_tc, v0) < 1e-5, (rel(v_cc, v0), rel(v_tc, v0))


def test_tg_jacobian_engine_switch_rejects_unknown_engines():
    from dogpup_b200._lib import lib
    assert lib.dgp_set_jacobian_engine(3) == 1 and lib.dgp_set_jacobian_engine(-1) == 1
    assert lib.dgp_set_jacobian_engine(2) == 0 and lib.dgp_set_jacobian_engine(0) == 0


def test_vjp_from_several_host_threads(jac_case):
    """Four host threads, each on its own stream, run the CUDA-core vjp on different harmonic
    counts (different dynamic shared-memory sizes of the same kernel) at once, 25 times each:
    every call succeeds and matches the same call made alone (1e-12).  The kernel's shared-memory limit
    is process-wide, so one thread's launch must not depend on the size another thread set."""
    import threading
    import torch
    from dogpup_b200 import api
    from dogpup_b200._lib import lib, check
    mesh = jac_case["mesh"]
    nb = mesh.nodal_basis()
    nt = len(mesh.optode.tAxis)
    link = mesh._link()
    g = torch.as_tensor(np.random.default_rng(4).standard_normal((link.shape[0], 20)))
    fpsf = mesh.optode.s_fpsf
    args = {k: (jac_case["phi"][:k].contiguous(), jac_case["phiA"][:k].contiguous(), fpsf[:k].contiguous(),
                jac_case["gfc_d"][:, :k].contiguous()) for k in (16, 11, 6, 3)}
    check(lib.dgp_set_jacobian_engine(1))
    try:
        alone = {k: api.jacobian_tg_vjp(nb, p, pa, f, link, gf, nt, g).cpu() for k, (p, pa, f, gf) in args.items()}
        errors, results = [], {}

        def work(k):
            try:
                s = torch.cuda.Stream()
                with torch.cuda.stream(s):
                    p, pa, f, gf = args[k]
                    for _ in range(25):
                        v = api.jacobian_tg_vjp(nb, p, pa, f, link, gf, nt, g)
                    s.synchronize()
                    results[k] = v.cpu()
            except Exception as e:          # collected: the assertion below reports it
                errors.append(repr(e))
        threads = [threading.Thread(target=work, args=(k,)) for k in args]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    finally:
        check(lib.dgp_set_jacobian_engine(0))
    assert not errors, errors
    for k in args:
        assert rel(results[k].numpy(), alone[k].numpy()) < 1e-12, k
