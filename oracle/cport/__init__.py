"""ctypes wrapper of the oracle's C restatement (oracle_cport.c) -- test/baseline infrastructure.

Builds ``liboracle_cport.so`` with ``make -C oracle cport`` when it is missing.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_LIB = _HERE / "liboracle_cport.so"
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not _LIB.exists():
            subprocess.run(["make", "-s", "-C", str(_HERE.parent), "cport"], check=True)
        _lib = C.CDLL(str(_LIB))
        P = C.c_void_p
        _lib.oc_threads.restype = C.c_int
        _lib.oc_fsai_factor.argtypes = [C.c_int, P, P, P, P, P, P, P]
        _lib.oc_bicgstab.argtypes = [C.c_int, P, P, P, P, C.c_double, P, P, P, P, P, P, C.c_int, P, P,
                                     C.c_double, C.c_int, P]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def threads() -> int:
    return lib().oc_threads()


def fsai_factor(A_tril_re, A_tril_im, rg, cg):
    """G values (complex128, [nnzG]) of tril(A) = re + i*im on the pattern (rg, cg)."""
    re = A_tril_re.tocsr()
    re.sort_indices()
    im = A_tril_im.tocsr()
    im.sort_indices()
    rp = re.indptr.astype(np.int32)
    cl = re.indices.astype(np.int32)
    G = np.zeros(cg.shape[0], dtype=np.complex128)
    rgi, cgi = rg.astype(np.int32), cg.astype(np.int32)
    rc = lib().oc_fsai_factor(re.shape[0], _p(rp), _p(cl), _p(np.ascontiguousarray(re.data)),
                              _p(np.ascontiguousarray(im.data)), _p(rgi), _p(cgi), _p(G))
    if rc:
        raise RuntimeError("oc_fsai_factor: pattern row length outside 1..64")
    return G


def bicgstab(K, M, w, rg, cg, G, rt, ct, GT, B, tol, maxit=1000):
    """Solves (K + i w M) X = B column by column (B: [n, ncol] complex128)."""
    K = K.tocsr(); K.sort_indices()
    M = M.tocsr(); M.sort_indices()
    assert np.array_equal(K.indptr, M.indptr) and np.array_equal(K.indices, M.indices)
    n, ncol = B.shape
    Bc = np.ascontiguousarray(B.T)
    X = np.zeros_like(Bc)
    it = np.zeros(ncol, dtype=np.int32)
    arrs = [K.indptr.astype(np.int32), K.indices.astype(np.int32), np.ascontiguousarray(K.data),
            np.ascontiguousarray(M.data), rg.astype(np.int32), cg.astype(np.int32),
            np.ascontiguousarray(G, dtype=np.complex128), rt.astype(np.int32), ct.astype(np.int32),
            np.ascontiguousarray(GT, dtype=np.complex128)]
    lib().oc_bicgstab(n, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]), _p(arrs[3]), float(w), _p(arrs[4]), _p(arrs[5]),
                      _p(arrs[6]), _p(arrs[7]), _p(arrs[8]), _p(arrs[9]), ncol, _p(Bc), _p(X), float(tol),
                      int(maxit), _p(it))
    return X.T, it
