"""Child process of tests/test_zz_no_alloc.py: the allocation-free FSAI entry point
used from two CUDA contexts in turn, the first destroyed before the second exists.

A MATLAB session does this between mex calls: reset(gpuDevice) destroys the CUDA
context, and the next call runs in a new one where the library's fixed scratch
array may sit at another address.  The contexts here are made with the driver API
(cuCtxCreate / cuCtxDestroy) and every buffer is allocated in the context that
uses it; no torch is loaded, so no other context exists in this process.

    python noalloc_contexts_child.py case.npz nfreqs      -> one JSON line on stdout
"""
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

from dogpup_b200._lib import lib  # noqa: E402  (loads libdogpup_b200.so)


def main():
    case = np.load(sys.argv[1])
    nf = int(sys.argv[2])
    cu = C.CDLL("libcuda.so.1")
    U64, VP, SZ = C.c_uint64, C.c_void_p, C.c_size_t
    cu.cuInit.argtypes = [C.c_uint]
    cu.cuDeviceGet.argtypes = [C.POINTER(C.c_int), C.c_int]
    cu.cuCtxCreate_v2.argtypes = [C.POINTER(VP), C.c_uint, C.c_int]
    cu.cuCtxDestroy_v2.argtypes = [VP]
    cu.cuCtxSynchronize.argtypes = []
    cu.cuMemAlloc_v2.argtypes = [C.POINTER(U64), SZ]
    cu.cuMemFree_v2.argtypes = [U64]
    cu.cuMemcpyHtoD_v2.argtypes = [U64, VP, SZ]
    cu.cuMemcpyDtoH_v2.argtypes = [VP, U64, SZ]

    def ck(rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: CUresult {rc}")

    ck(cu.cuInit(0), "cuInit")
    dev = C.c_int()
    ck(cu.cuDeviceGet(C.byref(dev), 0), "cuDeviceGet")
    n, nnzG = int(case["n"]), int(case["cg"].shape[0])
    out = []
    for rnd in range(2):
        ctx = VP()
        ck(cu.cuCtxCreate_v2(C.byref(ctx), 0, dev), "cuCtxCreate")      # current on this thread
        bufs = []

        def alloc(nbytes):
            p = U64()
            ck(cu.cuMemAlloc_v2(C.byref(p), nbytes), "cuMemAlloc")
            bufs.append(p)
            return p

        def up(a):
            a = np.ascontiguousarray(a)
            p = alloc(a.nbytes)
            ck(cu.cuMemcpyHtoD_v2(p, a.ctypes.data_as(VP), a.nbytes), "cuMemcpyHtoD")
            return p

        ins = [up(case["re"]), up(case["im"]), up(case["rp"].astype(np.int32)), up(case["cl"].astype(np.int32)),
               up(case["rg"].astype(np.int32)), up(case["cg"].astype(np.int32))]
        res = {}
        for name in ("dgp_fsaip_mex", "dgp_fsaip_mex_noalloc"):
            ore, oim = alloc(8 * nnzG * nf), alloc(8 * nnzG * nf)
            a0 = lib.dgp_device_allocations()
            rc = getattr(lib, name)(VP(ore.value), VP(oim.value), *[VP(p.value) for p in ins], nf, n, None)
            allocs = lib.dgp_device_allocations() - a0
            ck(cu.cuCtxSynchronize(), "cuCtxSynchronize")
            hre, him = np.empty(nnzG * nf), np.empty(nnzG * nf)
            ck(cu.cuMemcpyDtoH_v2(hre.ctypes.data_as(VP), ore, hre.nbytes), "cuMemcpyDtoH")
            ck(cu.cuMemcpyDtoH_v2(him.ctypes.data_as(VP), oim, him.nbytes), "cuMemcpyDtoH")
            res[name] = (rc, allocs, hre + 1j * him)
        (rc0, al0, g0), (rc1, al1, g1) = res["dgp_fsaip_mex"], res["dgp_fsaip_mex_noalloc"]
        err = float(np.linalg.norm(g1 - g0) / np.linalg.norm(g0)) if rc0 == 0 and rc1 == 0 else None
        out.append({"round": rnd, "rc_alloc": rc0, "rc_noalloc": rc1, "allocs_alloc": al0, "allocs_noalloc": al1,
                    "rel_err": err, "finite": bool(np.isfinite(g1).all()),
                    "error": lib.dgp_last_error().decode() if rc1 else ""})
        for p in bufs:
            ck(cu.cuMemFree_v2(p), "cuMemFree")
        ck(cu.cuCtxDestroy_v2(ctx), "cuCtxDestroy")
    print(json.dumps(out))


if __name__ == "__main__":
    main()
