"""The MATLAB gateways (dogpup_b200/mex) driven through a test double of the
mex / gpuArray runtime (tests/mexshim).

CPU: the gateways and the test double build and export mexFunction, and
argument errors raise MATLAB-style errors before any GPU work.  GPU: each
drop-in gateway against the oracle on MATLAB's layouts (FP64, 1e-12
relative), and bicgstab_fsai_mex -- the one-call replacement of fluGPU --
against a sparse-direct solve (1e-9 FP64 to tol 1e-12; 1e-6 mixed).
"""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
SHIM = HERE / "mexshim"
BUILD = SHIM / "_build"
GATEWAYS = ("smv_mex", "FSAImv_mex", "FSAIP_gen_mex", "bicgstab_fsai_mex")
DOUBLE, INT32 = 6, 12


class Mex:
    def __init__(self):
        if shutil.which("g++") is None:
            pytest.skip("no C++ compiler")
        subprocess.run(["make", "-s", "-C", str(SHIM)], check=True)
        self.shim = C.CDLL(str(BUILD / "libmexshim.so"), mode=C.RTLD_GLOBAL)
        s = self.shim
        s.shim_array.restype = C.c_void_p
        s.shim_array.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_size_t), C.c_void_p]
        s.shim_sparse.restype = C.c_void_p
        s.shim_sparse.argtypes = [C.c_size_t, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
        s.shim_string.restype = C.c_void_p
        s.shim_string.argtypes = [C.c_char_p]
        s.shim_call.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_char_p, C.c_int]
        s.shim_info.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_size_t), C.c_int]
        s.shim_read.argtypes = [C.c_void_p, C.c_void_p]
        s.shim_destroy.argtypes = [C.c_void_p]
        s.shim_warnings.restype = C.c_char_p
        self.gw = {}
        for g in GATEWAYS:
            lib = C.CDLL(str(BUILD / f"{g}.so"))
            self.gw[g] = (lib, C.cast(lib.mexFunction, C.c_void_p).value)
        self.live = []

    # ---- arrays (MATLAB column-major; complex interleaved)
    def array(self, a, gpu=False):
        a = np.asarray(a)
        if a.ndim == 1:
            a = a[:, None]
        dims = (C.c_size_t * a.ndim)(*a.shape)
        if np.iscomplexobj(a):
            buf, cls, cx = np.ravel(a.astype(np.complex128), order="F").view(np.float64).copy(), DOUBLE, 1
        elif a.dtype == np.int32:
            buf, cls, cx = np.ravel(a, order="F").copy(), INT32, 0
        else:
            buf, cls, cx = np.ravel(a.astype(np.float64), order="F").copy(), DOUBLE, 0
        h = self.shim.shim_array(cls, cx, int(gpu), a.ndim, dims, buf.ctypes.data_as(C.c_void_p))
        self.live.append(h)
        return h

    def sparse(self, S):
        S = sp.csc_matrix(S)
        S.sort_indices()
        jc = S.indptr.astype(np.uint64)
        ir = S.indices.astype(np.uint64)
        v = S.data.astype(np.float64)
        h = self.shim.shim_sparse(S.shape[0], S.shape[1], jc.ctypes.data_as(C.c_void_p),
                                  ir.ctypes.data_as(C.c_void_p), v.ctypes.data_as(C.c_void_p))
        self.live.append(h)
        return h

    def string(self, s):
        h = self.shim.shim_string(s.encode())
        self.live.append(h)
        return h

    def read(self, h):
        cls, cx, gpu = C.c_int(), C.c_int(), C.c_int()
        dims = (C.c_size_t * 8)()
        nd = self.shim.shim_info(h, C.byref(cls), C.byref(cx), C.byref(gpu), dims, 8)
        shape = tuple(dims[i] for i in range(nd))
        n = int(np.prod(shape))
        dt = {DOUBLE: np.float64, INT32: np.int32}[cls.value]
        buf = np.empty(n * (2 if cx.value else 1), dtype=dt)
        assert self.shim.shim_read(h, buf.ctypes.data_as(C.c_void_p)) == 0
        out = buf.view(np.complex128) if cx.value else buf
        return out.reshape(shape, order="F"), bool(gpu.value)

    def call(self, name, nlhs, *args):
        plhs = (C.c_void_p * max(nlhs, 1))()
        prhs = (C.c_void_p * len(args))(*args)
        err = C.create_string_buffer(1024)
        rc = self.shim.shim_call(self.gw[name][1], nlhs, plhs, len(args), prhs, err, 1024)
        if rc:
            raise RuntimeError(err.value.decode())
        for i in range(nlhs):
            self.live.append(plhs[i])
        return [plhs[i] for i in range(nlhs)]

    def close(self):
        for h in self.live:
            self.shim.shim_destroy(h)
        self.live = []


@pytest.fixture(scope="module")
def mex():
    m = Mex()
    yield m
    m.close()


def test_gateways_build_and_export_mexFunction(mex):
    for g in GATEWAYS:
        assert mex.gw[g][1], g


def test_gateway_argument_errors_are_matlab_errors(mex):
    x = mex.array(np.zeros((3, 1, 1)))
    with pytest.raises(RuntimeError, match="dogpup_b200:smv_mex:nrhs"):
        mex.call("smv_mex", 1, x)
    with pytest.raises(RuntimeError, match="dogpup_b200:FSAImv_mex:nrhs"):
        mex.call("FSAImv_mex", 1, x, x)
    with pytest.raises(RuntimeError, match="dogpup_b200:FSAIP_gen_mex:nrhs"):
        mex.call("FSAIP_gen_mex", 1, x)
    with pytest.raises(RuntimeError, match="dogpup_b200:bicgstab_fsai_mex:type"):
        mex.call("bicgstab_fsai_mex", 1, x, x, x, mex.array(np.array([1.0])))


# ------------------------------------------------------------------- GPU
@pytest.fixture(scope="module")
def system(small_case):
    K, M = small_case["K"], small_case["M"]
    dfc = 2 * np.pi / 10e-9 / (2.99792458e11 / 1.4)
    A = (K + 1j * dfc * M).tocsr()
    A.sort_indices()
    return K, M, dfc, A


def rel(a, b):
    return np.linalg.norm(np.ravel(a - b)) / np.linalg.norm(np.ravel(b))


@pytest.mark.gpu
def test_smv_and_fsaimv_gateways(mex, system):
    from oracle import solver as osv
    K, M, dfc, A = system
    n, ns, nf = A.shape[0], 3, 5
    rng = np.random.default_rng(4)
    x = rng.standard_normal((n, ns, nf)) + 1j * rng.standard_normal((n, ns, nf))
    rp, cp = A.indptr.astype(np.int32), A.indices.astype(np.int32)
    f = np.arange(nf, dtype=np.float64)[None, :]
    y, on_gpu = mex.read(mex.call("smv_mex", 1, mex.array(x, True), mex.array(f, True), mex.array(A.data, True),
                                  mex.array(rp, True), mex.array(cp, True))[0])
    assert on_gpu and y.shape == (n, ns, nf)
    y0 = np.stack([np.stack([(K + 1j * k * dfc * M) @ x[:, s, k] for s in range(ns)], 1) for k in range(nf)], 2)
    assert rel(y, y0) < 1e-12
    # a real x (MATLAB drops all-zero imaginary parts) is widened to complex
    yr, _ = mex.read(mex.call("smv_mex", 1, mex.array(x.real), mex.array(f), mex.array(A.data), mex.array(rp),
                              mex.array(cp))[0])
    y0r = np.stack([np.stack([(K + 1j * k * dfc * M) @ x[:, s, k].real for s in range(ns)], 1) for k in range(nf)], 2)
    assert rel(yr, y0r) < 1e-12
    # FSAImv on the oracle's FSAI factor
    pc = osv.FsaiPrecond(K, M, dfc, nf)
    G = pc.G                                               # [nnzG, NF]
    rg, cg = pc.rptrG.astype(np.int32), pc.colsG.astype(np.int32)
    z, _ = mex.read(mex.call("FSAImv_mex", 1, mex.array(x, True), mex.array(G, True), mex.array(rg, True),
                             mex.array(cg, True))[0])
    z0 = np.stack([np.stack([sp.csr_matrix((G[:, k], cg, rg), shape=(n, n)) @ x[:, s, k] for s in range(ns)], 1)
                   for k in range(nf)], 2)
    assert rel(z, z0) < 1e-12


@pytest.mark.gpu
def test_fsaip_gateway(mex, system):
    from oracle import solver as osv
    K, M, dfc, A = system
    nf = 4
    At = sp.tril(A).tocsr()
    At.sort_indices()
    pc = osv.FsaiPrecond(K, M, dfc, nf)
    rg, cg = pc.rptrG.astype(np.int32), pc.colsG.astype(np.int32)
    G, on_gpu = mex.read(mex.call("FSAIP_gen_mex", 1, mex.array(At.data), mex.array(At.indptr.astype(np.int32)),
                                  mex.array(At.indices.astype(np.int32)), mex.array(rg), mex.array(cg),
                                  mex.array(np.array([nf], dtype=np.int32)))[0])
    assert not on_gpu and G.shape == (nf, cg.shape[0])     # host [NF x nnzG], as the reference returns
    assert rel(G.T, pc.G) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("precision,gpu_q", [("fp64", False), ("mixed", True)])
def test_bicgstab_fsai_gateway_replaces_flugpu(mex, system, small_case, precision, gpu_q):
    """phi = bicgstab_fsai_mex(Q, triu(K), triu(M), df/c, tol, maxit, precision) with fluGPU's Q layout."""
    from oracle import solver as osv
    K, M, dfc, _ = system
    m = small_case["mesh"]
    n, nf, ns = K.shape[0], 6, 3
    rng = np.random.default_rng(8)
    Q = np.zeros((n, nf, ns), complex)                     # nodes x freqs x sources (fluGPU)
    fpsf = np.exp(-0.3j * np.arange(nf))
    for s in range(ns):
        e = m.elem[rng.integers(0, m.ne)]
        w = rng.random(4)
        Q[e, :, s] = (w / w.sum())[:, None] * fpsf[None, :]
    tol = 1e-12 if precision == "fp64" else 1e-10
    outs = mex.call("bicgstab_fsai_mex", 3, mex.array(Q, gpu_q), mex.sparse(sp.triu(K)), mex.sparse(sp.triu(M)),
                    mex.array(np.array([dfc])), mex.array(np.array([tol])), mex.array(np.array([1000.0])),
                    mex.string(precision))
    phi, on_gpu = mex.read(outs[0])
    assert on_gpu == gpu_q and phi.shape == (n, nf, ns)
    iters = mex.read(outs[1])[0].item()
    relres = mex.read(outs[2])[0].item()
    assert iters > 0 and relres < tol
    xd = osv.direct_solve(K, M, dfc, np.transpose(Q, (0, 2, 1)))   # [N, NS, NF]
    err = np.linalg.norm(np.transpose(phi, (0, 2, 1)) - xd, axis=0) / np.linalg.norm(xd, axis=0)
    assert err.max() < (1e-9 if precision == "fp64" else 1e-6), err.max()
