"""The allocation-free FSAI factor entry point, dgp_fsaip_mex_noalloc.

It exists for callers that may not allocate device memory themselves -- a
MATLAB mex gateway whose device memory must come from MATLAB's gpuArray pool,
or an application whose own pooling allocator owns the GPU.  It must give the
same factor as the allocating dgp_fsaip_mex, call after call, although every
call reuses (and must reset) the same fixed device scratch array.  The
harmonic count below makes the rows go through the scratch array in several
blocks.  This file is named to run last.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

DGP_ERR_ARG = 1


def _vp(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_factor_matches_allocating_entry_point(small_case):
    import torch
    from dogpup_b200._lib import lib, check
    from oracle import solver as osv

    K, M = small_case["K"], small_case["M"]
    dfc = 2 * np.pi / 10e-9 / (2.99792458e11 / 1.4)
    A = sp.tril(K + 1j * dfc * M).tocsr()
    A.sort_indices()
    rg, cg = osv.fsai_pattern(A)
    n, nnzG, nf = A.shape[0], cg.shape[0], 64   # 64 harmonics x 8-entry rows: 2048 rows per scratch block

    def dev(a, dt):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")

    ins = [dev(A.data.real, torch.float64), dev(A.data.imag, torch.float64), dev(A.indptr, torch.int32),
           dev(A.indices, torch.int32), dev(rg, torch.int32), dev(cg, torch.int32)]

    def run(fn):
        re = torch.full((nnzG * nf,), np.nan, dtype=torch.float64, device="cuda")
        im = torch.full_like(re, np.nan)
        check(fn(_vp(re), _vp(im), *[_vp(t) for t in ins], nf, n, None))
        torch.cuda.synchronize()
        return re.cpu().numpy() + 1j * im.cpu().numpy()

    expected = run(lib.dgp_fsaip_mex)
    assert np.isfinite(expected).all()
    free = []
    for call in range(3):
        got = run(lib.dgp_fsaip_mex_noalloc)
        free.append(torch.cuda.mem_get_info()[0])
        err = np.linalg.norm(got - expected) / np.linalg.norm(expected)
        assert err <= 1e-12, (call, err)
    # after the first call (which may load the module) no call changes free device memory
    assert free[1] == free[2]


def test_noalloc_rejects_requests_beyond_its_scratch(small_case):
    import torch
    from dogpup_b200._lib import lib, last_error
    from oracle import solver as osv

    K, M = small_case["K"], small_case["M"]
    A = sp.tril(K + 1j * 1e-3 * M).tocsr()
    A.sort_indices()
    rg, cg = osv.fsai_pattern(A)
    mmax = int(np.diff(rg).max())
    nf = (1 << 20) // mmax + 1
    dev = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device="cuda")
    ins = [dev(A.data.real, torch.float64), dev(A.data.imag, torch.float64), dev(A.indptr, torch.int32),
           dev(A.indices, torch.int32), dev(rg, torch.int32), dev(cg, torch.int32)]
    dummy = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc = lib.dgp_fsaip_mex_noalloc(_vp(dummy), _vp(dummy), *[_vp(t) for t in ins], nf, A.shape[0], None)
    assert rc == DGP_ERR_ARG
    assert "scratch" in last_error()
