"""Thin, typed wrappers over the C ABI on torch device tensors.

PyTorch only provides device memory and the current stream here; every
operation runs in libdogpup_b200's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import lib, check


def stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def ptr(t: torch.Tensor) -> int:
    if not t.is_cuda:
        raise ValueError("dogpup_b200 operates on CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return t.data_ptr()


def as_real(t: torch.Tensor) -> torch.Tensor:
    """complex tensor -> interleaved real view (no copy)."""
    return torch.view_as_real(t) if t.is_complex() else t


class Fem:
    """Device FEM topology + assembly plan (``prepare_mesh``/``gen_fwdmat``, dMesh.m:945-1235)."""

    def __init__(self, node: torch.Tensor, elem: torch.Tensor, nr: float):
        node = node.to(device="cuda", dtype=torch.float64).contiguous()
        elem = elem.to(device="cuda", dtype=torch.int32).contiguous()
        self.nn, self.ne = int(node.shape[0]), int(elem.shape[0])
        h = C.c_void_p()
        check(lib.dgp_fem_create(C.byref(h), ptr(node), ptr(elem), self.nn, self.ne, float(nr), stream_ptr()))
        self._h = h
        nnz, nf, nb, c = C.c_int64(), C.c_int64(), C.c_int64(), C.c_double()
        check(lib.dgp_fem_info(h, C.byref(nnz), C.byref(nf), C.byref(nb), C.byref(c)))
        self.nnz, self.n_robin_faces, self.n_boundary, self.c = nnz.value, nf.value, nb.value, c.value
        rp, cp = C.c_void_p(), C.c_void_p()
        check(lib.dgp_fem_pattern(h, C.byref(rp), C.byref(cp)))
        # own copies of the pattern as torch tensors
        self.rowptr = torch.empty(self.nn + 1, dtype=torch.int32, device="cuda")
        self.col = torch.empty(self.nnz, dtype=torch.int32, device="cuda")
        _d2d(self.rowptr, rp.value)
        _d2d(self.col, cp.value)
        self.bnd = torch.empty(self.nn, dtype=torch.int32, device="cuda")
        check(lib.dgp_fem_boundary(h, ptr(self.bnd), stream_ptr()))

    def assemble(self, mua: torch.Tensor, musp: torch.Tensor):
        mua = mua.to(device="cuda", dtype=torch.float64).contiguous()
        musp = musp.to(device="cuda", dtype=torch.float64).contiguous()
        K = torch.empty(self.nnz, dtype=torch.float64, device="cuda")
        M = torch.empty(self.nnz, dtype=torch.float64, device="cuda")
        check(lib.dgp_fem_assemble(self._h, ptr(mua), ptr(musp), ptr(K), ptr(M), stream_ptr()))
        return K, M

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:  # lib is None during interpreter shutdown
            lib.dgp_fem_destroy(h)
            self._h = None


def _d2d(dst: torch.Tensor, src_ptr: int):
    """Copy library-owned device memory into a torch tensor of the same size."""
    dst.copy_(_borrow(src_ptr, dst.numel(), dst.dtype))


def _borrow(p: int, n: int, dtype) -> torch.Tensor:
    """Non-owning tensor view of device memory owned by the library."""
    class _Holder:
        def __init__(self, p, n, dtype):
            typestr = {torch.int32: "<i4", torch.float64: "<f8"}[dtype]
            self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (p, False), "version": 3,
                                             "strides": None}
    return torch.as_tensor(_Holder(p, n, dtype), device="cuda")


class Solver:
    """Batched FSAI-BiCGSTAB plan for A_k = K + i*k*dfc*M (gpuBicstab_FSAIP, dMesh.m:1247-1385)."""

    def __init__(self, rowptr, col, K, M, dfc: float, nf: int, ns_max: int, opts: _lib.SolveOpts | None = None,
                 harmonics=None):
        """harmonics: the harmonic index of each of the nf batch slots (default 0 .. nf-1)."""
        self.n = int(rowptr.numel() - 1)
        self.nnz = int(col.numel())
        self.nf, self.ns_max, self.dfc = int(nf), int(ns_max), float(dfc)
        o = opts or _lib.default_opts()
        h = C.c_void_p()
        if harmonics is None:
            check(lib.dgp_solver_create(C.byref(h), ptr(rowptr), ptr(col), self.n, self.nnz, ptr(K), ptr(M),
                                        self.dfc, self.nf, self.ns_max, C.byref(o), stream_ptr()))
            self.harmonics = list(range(self.nf))
        else:
            hl = [int(x) for x in harmonics]
            if len(hl) != self.nf:
                raise ValueError("one harmonic index per batch slot")
            arr = (C.c_int32 * self.nf)(*hl)
            check(lib.dgp_solver_create_harmonics(C.byref(h), ptr(rowptr), ptr(col), self.n, self.nnz, ptr(K),
                                                  ptr(M), self.dfc, arr, self.nf, self.ns_max, C.byref(o),
                                                  stream_ptr()))
            self.harmonics = hl
        self._h = h

    def update(self, K, M):
        check(lib.dgp_solver_update(self._h, ptr(K), ptr(M), stream_ptr()))

    def memory(self) -> int:
        b = C.c_int64()
        check(lib.dgp_solver_memory(self._h, C.byref(b)))
        return b.value

    def autotune(self) -> dict:
        """Pick the complex-FP32 SpMM kind and launch shape for this plan (dgp_solver_autotune)."""
        tl, v, r, ms = C.c_int32(), C.c_int32(), C.c_int32(), C.c_float()
        check(lib.dgp_solver_autotune(self._h, C.byref(tl), C.byref(v), C.byref(r), C.byref(ms), stream_ptr()))
        return dict(self.spmm_shape(), spmm_ms_per_iteration=round(ms.value, 3))

    def spmm_shape(self) -> dict:
        """The plan's complex-FP32 SpMM: tiled or gather, lane width, rows per block, inner-loop kind."""
        tl, v, r, k = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        check(lib.dgp_solver_spmm_shape(self._h, C.byref(tl), C.byref(v), C.byref(r), C.byref(k)))
        return {"spmm": "tiled" if tl.value else "gather", "vec": v.value, "rows": r.value, "kind": k.value}

    def set_spmm(self, tiled: bool, vec: int = 0, rows: int = 0):
        check(lib.dgp_solver_set_spmm(self._h, int(tiled), int(vec), int(rows)))

    def set_device_loop(self, on: bool):
        """True (default): one graph launch per inner solve (device-driven WHILE loop); False: host polling."""
        check(lib.dgp_solver_set_device_loop(self._h, int(bool(on))))

    def set_spmm_kind(self, kind: int):
        """Inner loop of the gather SpMM: 0 one nonzero per step, 1 two, 2 four, 3 four with packed FMAs."""
        check(lib.dgp_solver_set_spmm_kind(self._h, int(kind)))

    def set_dot_rows(self, mult: int):
        """Rows per block of the dot-product SpMM sweeps as a multiple of the plain ones (0 = 4)."""
        check(lib.dgp_solver_set_dot_rows(self._h, int(mult)))

    def check_spmm(self) -> float:
        """max |tiled - gather| / max |value| over A, G, G^T on a test pattern."""
        d = C.c_double()
        check(lib.dgp_solver_check_spmm(self._h, C.byref(d), stream_ptr()))
        return d.value

    def profile_kernel(self, which: int, reps: int = 10):
        """(ms per launch, algorithmic bytes per launch) of one sweep kernel, CUDA-event timed."""
        ms, b = C.c_float(), C.c_double()
        check(lib.dgp_solver_profile_kernel(self._h, which, reps, C.byref(ms), C.byref(b), stream_ptr()))
        return ms.value, b.value

    def solve(self, B: torch.Tensor, opts=None, status=None):
        """X[k] = A_k^-1 B[k], B complex128 [NF][NN][NS]."""
        nf, n, ns = B.shape
        X = torch.empty_like(B)
        rep = _lib.SolveReport()
        if status is not None:
            rep.d_status = ptr(status)
        o = opts or _lib.default_opts()
        rc = lib.dgp_solve(self._h, ptr(as_real(B)), ptr(as_real(X)), ns, C.byref(o), C.byref(rep), stream_ptr())
        check(rc, allow=(_lib.ERR_NOT_CONVERGED,))
        return X, rep

    def solve_sources(self, nodes, w, fpsf, opts=None, status=None, out=None):
        """Point-source right-hand sides b[k][nodes[s,l]][s] = w[s,l]*fpsf[k] (dMesh.m:124-129)."""
        ns = int(nodes.shape[0])
        X = out if out is not None else torch.empty((self.nf, self.n, ns), dtype=torch.complex128, device="cuda")
        rep = _lib.SolveReport()
        if status is not None:
            rep.d_status = ptr(status)
        o = opts or _lib.default_opts()
        rc = lib.dgp_solve_sources(self._h, ptr(nodes), ptr(w), ptr(as_real(fpsf)), ns, ptr(as_real(X)),
                                   C.byref(o), C.byref(rep), stream_ptr())
        check(rc, allow=(_lib.ERR_NOT_CONVERGED,))
        return X, rep

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and lib is not None:  # lib is None during interpreter shutdown
            lib.dgp_solver_destroy(h)
            self._h = None


def make_opts(**kw) -> _lib.SolveOpts:
    o = _lib.default_opts()
    for k, v in kw.items():
        if v is None:
            continue
        if k == "precision" and isinstance(v, str):
            v = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED, "mixed_bicgstab": _lib.PREC_MIXED_BICGSTAB}[v]
        if k == "stop_rule" and isinstance(v, str):
            v = {"max_all": _lib.STOP_MAX_ALL, "per_column": _lib.STOP_PER_COLUMN}[v]
        setattr(o, k, v)
    return o


# ------------------------------------------------------------- transforms
def td2fc(x: torch.Tensor, f: torch.Tensor, t: torch.Tensor) -> torch.Tensor:
    """Fourier-series coefficients along the last axis (td2fc.m:26-32)."""
    x2 = x.to(torch.float64).reshape(-1, x.shape[-1]).contiguous()
    f = f.to(device="cuda", dtype=torch.float64).contiguous()
    t = t.to(device="cuda", dtype=torch.float64).contiguous()
    out = torch.empty((x2.shape[0], f.numel()), dtype=torch.complex128, device="cuda")
    check(lib.dgp_td2fc(ptr(x2), x2.shape[0], x2.shape[1], ptr(t), ptr(f), f.numel(), ptr(as_real(out)),
                        stream_ptr()))
    return out.reshape(*x.shape[:-1], f.numel())


def fc2td(c: torch.Tensor, f: torch.Tensor, t: torch.Tensor) -> torch.Tensor:
    """Time-domain signal from coefficients along the last axis (fc2td.m:24-31)."""
    c2 = c.to(torch.complex128).reshape(-1, c.shape[-1]).contiguous()
    f = f.to(device="cuda", dtype=torch.float64).contiguous()
    t = t.to(device="cuda", dtype=torch.float64).contiguous()
    out = torch.empty((c2.shape[0], t.numel()), dtype=torch.float64, device="cuda")
    check(lib.dgp_fc2td(ptr(as_real(c2)), c2.shape[0], c2.shape[1], ptr(f), ptr(t), t.numel(), ptr(out),
                        stream_ptr()))
    return out.reshape(*c.shape[:-1], t.numel())


def fc2tg(c: torch.Tensor, gate_fc: torch.Tensor, nt: int) -> torch.Tensor:
    """Time-gated data from coefficients along the last axis (fc2tg.m:25-32)."""
    c2 = c.to(torch.complex128).reshape(-1, c.shape[-1]).contiguous()
    g = gate_fc.to(device="cuda", dtype=torch.complex128).contiguous()
    out = torch.empty((c2.shape[0], g.shape[0]), dtype=torch.float64, device="cuda")
    check(lib.dgp_fc2tg(ptr(as_real(c2)), c2.shape[0], c2.shape[1], ptr(as_real(g)), g.shape[0], int(nt),
                        ptr(out), stream_ptr()))
    return out.reshape(*c.shape[:-1], g.shape[0])


class DeviceCsr:
    """A real FP64 CSR matrix on the device with ``A @ x`` through ``dgp_csr_spmv``.

    Built from a SciPy sparse matrix; the pattern is checked once here (row pointer
    from 0, non-decreasing, ending at nnz; columns in range) so the kernel gets a
    well-formed matrix."""

    def __init__(self, A):
        A = A.tocsr()
        A.sort_indices()
        ip, ix = np.asarray(A.indptr, dtype=np.int64), np.asarray(A.indices, dtype=np.int64)
        if ip[0] != 0 or ip[-1] != ix.size or (np.diff(ip) < 0).any() or (ix.size and (ix.min() < 0 or
                                                                                      ix.max() >= A.shape[1])):
            raise ValueError("DeviceCsr: malformed CSR pattern")
        self.shape = A.shape
        self.rowptr = torch.as_tensor(ip.astype(np.int32), device="cuda")
        self.col = torch.as_tensor(ix.astype(np.int32), device="cuda")
        self.val = torch.as_tensor(np.asarray(A.data, dtype=np.float64), device="cuda")

    def __matmul__(self, x: torch.Tensor) -> torch.Tensor:
        x = x.to(device="cuda", dtype=torch.float64).contiguous()
        if x.numel() != self.shape[1]:
            raise ValueError(f"DeviceCsr: x has {x.numel()} entries, the matrix {self.shape[1]} columns")
        y = torch.empty(self.shape[0], dtype=torch.float64, device="cuda")
        check(lib.dgp_csr_spmv(ptr(self.rowptr), ptr(self.col), ptr(self.val), self.shape[0], self.shape[1], ptr(x),
                               ptr(y), stream_ptr()))
        return y


class Basis:
    """Jacobian basis: P = m2g as device CSR (voxel grid) or None (nodal), plus weights w [nv]."""

    def __init__(self, P=None, w=None, nn=None):
        if P is not None:
            P = P.tocsr()
            P.sort_indices()
            self.rowptr = torch.as_tensor(P.indptr.astype("int32"), device="cuda")
            self.col = torch.as_tensor(P.indices.astype("int32"), device="cuda")
            self.val = torch.as_tensor(P.data.astype("float64"), device="cuda")
            self.nv = P.shape[0]
        else:
            self.rowptr = self.col = self.val = None
            self.nv = int(nn)
        self.w = None if w is None else torch.as_tensor(w, dtype=torch.float64, device="cuda").contiguous()

    def args(self):
        p = lambda t: None if t is None else ptr(t)
        return [p(self.rowptr), p(self.col), p(self.val), self.nv, p(self.w)]


def _jac_common(basis, phi, phiA, fpsf, link):
    nf, nn, ns = phi.shape
    nd = phiA.shape[2]
    link = link.to(device="cuda", dtype=torch.int32).contiguous()
    fpsf = fpsf.to(device="cuda", dtype=torch.complex128).contiguous()
    return [*basis.args(), ptr(as_real(phi)), ns, ptr(as_real(phiA)), nd, nn, nf, ptr(as_real(fpsf)), ptr(link),
            int(link.shape[0])], (link, fpsf)


def jacobian_complex(basis, phi, phiA, fpsf, link) -> torch.Tensor:
    """J[v][k][m] (J_complex, dMesh.m:206-247), complex128."""
    args, keep = _jac_common(basis, phi, phiA, fpsf, link)
    out = torch.empty((basis.nv, phi.shape[0], int(link.shape[0])), dtype=torch.complex128, device="cuda")
    check(lib.dgp_jacobian_complex(*args, ptr(as_real(out)), stream_ptr()))
    return out


def jacobian_tg(basis, phi, phiA, fpsf, link, gate_fc, nt, data_tg=None) -> torch.Tensor:
    """Time-gated Jacobian J_tg[v][g][m] float32 (optionally Rytov-normalised by data_tg [nm][ng])."""
    args, keep = _jac_common(basis, phi, phiA, fpsf, link)
    g = gate_fc.to(device="cuda", dtype=torch.complex128).contiguous()
    rt = None if data_tg is None else data_tg.to(device="cuda", dtype=torch.float64).contiguous()
    out = torch.empty((basis.nv, g.shape[0], int(link.shape[0])), dtype=torch.float32, device="cuda")
    check(lib.dgp_jacobian_tg(*args, ptr(as_real(g)), g.shape[0], int(nt), None if rt is None else ptr(rt), ptr(out),
                              stream_ptr()))
    return out


def jacobian_tg_vjp(basis, phi, phiA, fpsf, link, gate_fc, nt, gin, data_tg=None) -> torch.Tensor:
    """J_tg^T g [nv] for an upstream gradient g [nm][ng], without forming J."""
    args, keep = _jac_common(basis, phi, phiA, fpsf, link)
    g = gate_fc.to(device="cuda", dtype=torch.complex128).contiguous()
    rt = None if data_tg is None else data_tg.to(device="cuda", dtype=torch.float64).contiguous()
    gin = gin.to(device="cuda", dtype=torch.float64).contiguous()
    out = torch.empty(basis.nv, dtype=torch.float64, device="cuda")
    check(lib.dgp_jacobian_tg_vjp(*args, ptr(as_real(g)), g.shape[0], int(nt), None if rt is None else ptr(rt),
                                  ptr(gin), ptr(out), stream_ptr()))
    return out


def meas(det_nodes, det_w, link, phi) -> torch.Tensor:
    """Detector data [NM][NF] from phi [NF][NN][NS] (meas_flu, dMesh.m:144-171)."""
    nf, n, ns = phi.shape
    nm = int(link.shape[0])
    out = torch.empty((nm, nf), dtype=torch.complex128, device="cuda")
    check(lib.dgp_meas(ptr(det_nodes), ptr(det_w), int(det_nodes.shape[0]), ptr(link), nm, ptr(as_real(phi)), n,
                       nf, ns, ptr(as_real(out)), stream_ptr()))
    return out


def locate_points(node: torch.Tensor, elem: torch.Tensor, pts, eps: float = 1e-12):
    """(elem id [NP] int64, -1 outside; barycentric weights [NP][4]) of points [NP][3] on the device."""
    node = torch.as_tensor(node).to(device="cuda", dtype=torch.float64).contiguous()
    elem = torch.as_tensor(elem).to(device="cuda", dtype=torch.int32).contiguous()
    pts = torch.as_tensor(pts).to(device="cuda", dtype=torch.float64).reshape(-1, 3).contiguous()
    n = int(pts.shape[0])
    eid = torch.empty(n, dtype=torch.int32, device="cuda")
    w = torch.empty((n, 4), dtype=torch.float64, device="cuda")
    check(lib.dgp_locate_points(ptr(node), ptr(elem), int(node.shape[0]), int(elem.shape[0]), ptr(pts), n,
                                float(eps), ptr(eid), ptr(w), stream_ptr()))
    return eid.long(), w


def snap_to_surface(node, bnd, face, pos):
    """(surface point [N][3], inward normal [N][3], face id [N]) of positions [N][3] on the device
    (snap_pos, dOptode.m:155-190); bnd [NN] flags, face [NF][3] 0-based surface triangles."""
    node = torch.as_tensor(node).to(device="cuda", dtype=torch.float64).contiguous()
    bnd = torch.as_tensor(bnd).to(device="cuda", dtype=torch.int32).contiguous()
    face = torch.as_tensor(face).to(device="cuda", dtype=torch.int32).contiguous()
    pos = torch.as_tensor(pos).to(device="cuda", dtype=torch.float64).reshape(-1, 3).contiguous()
    n = int(pos.shape[0])
    out = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    dirs = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    fid = torch.empty(n, dtype=torch.int32, device="cuda")
    check(lib.dgp_snap_to_surface(ptr(node), int(node.shape[0]), ptr(bnd), ptr(face), int(face.shape[0]), ptr(pos),
                                  n, ptr(out), ptr(dirs), ptr(fid), stream_ptr()))
    return out, dirs, fid.long()


def grid_to_mesh(node: torch.Tensor, axes, inmesh):
    """g2m rows (voxel index [NN][4], -1 = empty; weight [NN][4]) for the lattice of
    voxel centres ``ndgrid(*axes)`` (each axis uniformly spaced) and the in-mesh mask."""
    node = torch.as_tensor(node).to(device="cuda", dtype=torch.float64).contiguous()
    inm = torch.as_tensor(np.asarray(inmesh, dtype=np.uint8)).to("cuda").contiguous()
    o, d, n = [], [], []
    for a in axes:
        a = np.asarray(a, dtype=np.float64).ravel()
        step = a[1] - a[0] if a.size > 1 else 1.0
        if a.size > 1 and np.abs(np.diff(a) - step).max() > 1e-9 * abs(step):
            raise ValueError("grid axes must be uniformly spaced")
        o.append(a[0]); d.append(step); n.append(a.size)
    if int(np.prod(n)) != inm.numel():
        raise ValueError("inmesh must have one flag per voxel")
    o, d, n = (C.c_double * 3)(*o), (C.c_double * 3)(*d), (C.c_int32 * 3)(*n)
    nn = int(node.shape[0])
    col = torch.empty((nn, 4), dtype=torch.int32, device="cuda")
    val = torch.empty((nn, 4), dtype=torch.float64, device="cuda")
    check(lib.dgp_grid_to_mesh(ptr(node), nn, o, d, n, ptr(inm), ptr(col), ptr(val), stream_ptr()))
    return col.long(), val


# ------------------------------------------------------ reverse-mode pieces
def tg_adjoint_rhs(det_nodes, det_w, link, gate_fc, nt, g, n, nf, ns) -> torch.Tensor:
    """dL/dphi [NF][NN][NS] complex128 for L = sum g * fc2tg(meas(phi)), g [NM][NG]."""
    gate = gate_fc.to(device="cuda", dtype=torch.complex128).contiguous()
    g = g.to(device="cuda", dtype=torch.float64).contiguous()
    link = link.to(device="cuda", dtype=torch.int32).contiguous()
    B = torch.empty((nf, n, ns), dtype=torch.complex128, device="cuda")
    check(lib.dgp_tg_adjoint_rhs(ptr(det_nodes), ptr(det_w), int(det_nodes.shape[0]), ptr(link), int(link.shape[0]),
                                 ptr(as_real(gate)), int(gate.shape[0]), int(nt), ptr(g), n, nf, ns, ptr(as_real(B)),
                                 stream_ptr()))
    return B


def fem_adjoint_grad(fem: Fem, mua, musp, phi, lam, want_musp=True):
    """(dL/dmua, dL/dmusp or None) [NN] from forward fields phi and adjoint fields lam [NF][NN][NS]."""
    nf, n, ns = phi.shape
    if lam.shape != phi.shape:
        raise ValueError("phi and lam must have the same shape")
    mua = mua.to(device="cuda", dtype=torch.float64).contiguous()
    musp = musp.to(device="cuda", dtype=torch.float64).contiguous()
    gmua = torch.empty(n, dtype=torch.float64, device="cuda")
    gmusp = torch.empty(n, dtype=torch.float64, device="cuda") if want_musp else None
    check(lib.dgp_fem_adjoint_grad(fem._h, ptr(mua), ptr(musp), ptr(as_real(phi)), ptr(as_real(lam)), nf, ns,
                                   ptr(gmua), None if gmusp is None else ptr(gmusp), stream_ptr()))
    return gmua, gmusp
