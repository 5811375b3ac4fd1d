"""The reference-layout drop-ins (smv_call / FSAImv_call / FSAIP_call) on the GPU.

Each is checked against the oracle and, when the checker library built from
the reference's own CUDA sources (oracle/_ref/libdogpup_ref.so) is present,
against the unmodified reference kernels on identical inputs.  That second
comparison also pins the oracle's smv / fsai_apply / fsai_factor to the
reference.  FP64 tolerance: 1e-12 relative (different summation order).
"""
import ctypes as C
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parent.parent
REF = ROOT / "oracle" / "_ref" / "libdogpup_ref.so"


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.fixture(scope="module")
def ref():
    if not REF.exists():
        pytest.skip("reference-kernel checker not built")
    lib = C.CDLL(str(REF))
    for n in ("ref_smv", "ref_fsaimv", "ref_fsaip"):
        getattr(lib, n).restype = C.c_int
    return lib


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / max(np.linalg.norm(np.ravel(b)), 1e-300)


def planes(torch, x):
    """complex numpy [N, NS, NF] -> (re, im) device planes in MATLAB column-major order."""
    xf = np.asfortranarray(x)
    re = torch.as_tensor(np.ravel(xf.real, order="F").copy(), device="cuda")
    im = torch.as_tensor(np.ravel(xf.imag, order="F").copy(), device="cuda")
    return re, im


def unplanes(re, im, shape):
    return (re.cpu().numpy() + 1j * im.cpu().numpy()).reshape(shape, order="F")


@pytest.fixture(scope="module")
def system(small_case):
    K, M = small_case["K"], small_case["M"]
    dfc = 2 * np.pi / 10e-9 / (2.99792458e11 / 1.4)
    A = (K + 1j * dfc * M).tocsr()
    A.sort_indices()
    return K, M, dfc, A


def _ip(t):
    return C.c_void_p(t.data_ptr())


def test_smv_drop_in(system, torch, ref):
    from dogpup_b200._lib import lib, check
    from oracle import solver as osv
    K, M, dfc, A = system
    n, ns, nf = A.shape[0], 5, 4
    rng = np.random.default_rng(3)
    x = rng.standard_normal((n, ns, nf)) + 1j * rng.standard_normal((n, ns, nf))
    xr, xi = planes(torch, x)
    f = torch.arange(nf, dtype=torch.float64, device="cuda")
    ar = torch.as_tensor(A.data.real.copy(), device="cuda")
    ai = torch.as_tensor(A.data.imag.copy(), device="cuda")
    rp = torch.as_tensor(A.indptr.astype(np.int32), device="cuda")
    cp = torch.as_tensor(A.indices.astype(np.int32), device="cuda")
    outs = []
    for fn in ("dgp", "ref"):
        o_re = torch.zeros(n * ns * nf, dtype=torch.float64, device="cuda")
        o_im = torch.zeros_like(o_re)
        args = [_ip(o_re), _ip(o_im), _ip(xr), _ip(xi), _ip(f), _ip(ar), _ip(ai), _ip(rp), _ip(cp), n, ns, nf]
        if fn == "dgp":
            check(lib.dgp_smv_mex(*args, None))
        else:
            assert ref.ref_smv(*args) == 0
        torch.cuda.synchronize()
        outs.append(unplanes(o_re, o_im, (n, ns, nf)))
    y0 = osv.smv(x, np.arange(nf, dtype=float), K, dfc * M)
    assert rel(outs[1], y0) < 1e-13        # oracle pinned to the reference kernel
    assert rel(outs[0], outs[1]) < 1e-13   # drop-in == reference kernel


def test_fsaip_and_fsaimv_drop_ins(system, torch, ref):
    from dogpup_b200._lib import lib, check
    from oracle import solver as osv
    K, M, dfc, A = system
    n, nf, ns = A.shape[0], 6, 3
    At = sp.tril(A).tocsr()
    At.sort_indices()
    rg, cg = osv.fsai_pattern(At)
    nnzG = cg.shape[0]
    dev = lambda a, dt=torch.float64: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    args_in = [dev(At.data.real), dev(At.data.imag), dev(At.indptr, torch.int32), dev(At.indices, torch.int32),
               dev(rg, torch.int32), dev(cg, torch.int32)]
    outs = []
    for fn in ("dgp", "ref"):
        o_re = torch.zeros(nf * nnzG, dtype=torch.float64, device="cuda")
        o_im = torch.zeros_like(o_re)
        args = [_ip(o_re), _ip(o_im)] + [_ip(t) for t in args_in] + [nf, n]
        if fn == "dgp":
            check(lib.dgp_fsaip_mex(*args, None))
        else:
            assert ref.ref_fsaip(*args) == 0
        torch.cuda.synchronize()
        # [NF x nnzG] column-major == harmonic fastest
        outs.append((o_re.cpu().numpy() + 1j * o_im.cpu().numpy()).reshape(nnzG, nf))
    G0 = osv.fsai_factor(sp.tril(K).tocsr(), sp.tril(dfc * M).tocsr(), rg, cg, nf)
    assert rel(outs[1], G0) < 1e-12        # oracle pinned to the reference FSAI kernel
    assert rel(outs[0], outs[1]) < 1e-12   # drop-in == reference kernel

    # FSAImv with the reference's [nnzG x NF] value layout (dMesh.m:1384)
    G = outs[1]
    rng = np.random.default_rng(4)
    x = rng.standard_normal((n, ns, nf)) + 1j * rng.standard_normal((n, ns, nf))
    xr, xi = planes(torch, x)
    gr = dev(np.ravel(G.real, order="F"))
    gi = dev(np.ravel(G.imag, order="F"))
    ys = []
    for fn in ("dgp", "ref"):
        o_re = torch.zeros(n * ns * nf, dtype=torch.float64, device="cuda")
        o_im = torch.zeros_like(o_re)
        args = [_ip(o_re), _ip(o_im), _ip(xr), _ip(xi), _ip(gr), _ip(gi), _ip(args_in[4]), _ip(args_in[5]), nnzG,
                n, ns, nf]
        if fn == "dgp":
            check(lib.dgp_fsaimv_mex(*args, None))
        else:
            assert ref.ref_fsaimv(*args) == 0
        torch.cuda.synchronize()
        ys.append(unplanes(o_re, o_im, (n, ns, nf)))
    y0 = osv.fsai_apply(x, G, rg, cg, n)
    assert rel(ys[1], y0) < 1e-13
    assert rel(ys[0], ys[1]) < 1e-13
