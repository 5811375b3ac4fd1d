"""Float64 restatement of DOGPUP's FSAI-preconditioned BiCGSTAB forward solve.

Restates ``fluGPU`` (DOGPUP/dMesh.m:1238-1244), ``gpuBicstab_FSAIP``
(:1247-1348), ``FSAIP_gen`` (:1351-1385), ``sparse_csr`` (:1388-1414), the
three mex kernels' arithmetic (cuda_lib/mex_sources/smv_CUDA.cu:8-54,
FSAImv_CUDA.cu:8-53, FSAIP_CUDA.cu:13-160), the source-vector build of
``flu_solve``/``adj_flu_solve`` (dMesh.m:124-129, :191-196) and ``meas_flu``
(:144-171).

Layout: fields are ``[NN, NS, NF]`` complex128 (the reference's own layout
inside the solver after ``permute(Q,[1 3 2])``, dMesh.m:1258).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


# ----------------------------------------------------------------- CSR helpers
def sparse_csr_from_matrix(A):
    """0-based int32 CSR of a scipy sparse matrix, dMesh.m:1388-1414 (one-argument form)."""
    A = sp.csr_matrix(A)
    A.sort_indices()
    return A.indices.astype(np.int32), A.indptr.astype(np.int32), A.data.copy()


def transpose_pattern(rptr, cols, nrows):
    """CSR of the transpose plus the slot permutation, the three-argument
    ``sparse_csr`` call of dMesh.m:1255-1256 (a stable sort by column)."""
    rows = np.repeat(np.arange(nrows), np.diff(rptr))
    order = np.argsort(cols, kind="stable")
    t_cols = rows[order]
    t_ptr = np.zeros(nrows + 1, dtype=np.int64)
    np.add.at(t_ptr, cols + 1, 1)
    t_ptr = np.cumsum(t_ptr)
    return t_ptr, t_cols, order


# ------------------------------------------------------------- FSAI pattern
def fsai_pattern(A_tril, cap=30):
    """Sparsity pattern of G exactly as ``FSAIP_gen`` selects it, dMesh.m:1361-1380.

    ``A_tril`` is ``tril(A)`` with A = K + i*df/c*M.  Returns (rptr, cols)
    0-based with columns ascending in each row.
    """
    A = sp.csc_matrix(A_tril)
    A.sort_indices()
    # MATLAB find(): column-major order
    j = np.repeat(np.arange(A.shape[1]), np.diff(A.indptr))
    i = A.indices.astype(np.int64)
    v = np.abs(A.data)
    # sortrows([i abs(v)],'descend'), stable (:1367-1368)
    idx = np.lexsort((-v, -i), axis=0)
    si = i[idx]
    d = np.diff(np.concatenate([[si[-1] + 1], si]))             # :1369
    starts = np.nonzero(d)[0] + 1                               # 1-based, :1370
    sel = (starts[None, :] - np.arange(cap)[:, None]).ravel()   # :1371
    sel = np.unique(sel)
    sel = sel[sel > 0]                                          # :1372
    pick = idx[sel - 1]                                         # :1373
    pi, pj = i[pick], j[pick]
    o = np.lexsort((pj, pi))                                    # sortrows, :1375
    pi, pj = pi[o], pj[o]
    n = A.shape[0]
    rptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rptr, pi + 1, 1)
    return np.cumsum(rptr), pj.astype(np.int64)


def fsai_pattern_rowwise(A_tril, cap=30):
    """Per-row statement of the same rule: in each row of tril(A), rank the
    entries by |a_ij| descending (ties by column), keep rank 0 and every rank
    >= n_row - (cap-1).  Rows with <= cap entries keep all of them."""
    A = sp.csr_matrix(A_tril)
    A.sort_indices()
    rptr = [0]
    cols = []
    for r in range(A.shape[0]):
        c = A.indices[A.indptr[r]:A.indptr[r + 1]]
        v = np.abs(A.data[A.indptr[r]:A.indptr[r + 1]])
        n = len(c)
        order = np.lexsort((c, -v))
        keep = [order[t] for t in range(n) if t == 0 or t >= n - (cap - 1)]
        cc = np.sort(c[keep])
        cols.extend(cc.tolist())
        rptr.append(len(cols))
    return np.array(rptr, dtype=np.int64), np.array(cols, dtype=np.int64)


# -------------------------------------------------------------- FSAI factor
def complex_sqrt_ref(z):
    """``complexSqrt`` of FSAIP_CUDA.cu:28-43 (principal square root)."""
    a, b = z.real, z.imag
    m = np.sqrt(a * a + b * b)
    re = np.sqrt((m + a) / 2)
    im = np.where(b > 0, 1.0, -1.0) * np.sqrt(np.maximum((m - a) / 2, 0.0))
    zero_b = b == 0
    neg = zero_b & (a < 0)
    re = np.where(neg, 0.0, re)
    im = np.where(zero_b, np.where(a < 0, np.sqrt(np.abs(a)), 0.0), im)
    return re + 1j * im


def fsai_factor(A_tril_re, A_tril_im, rptrG, colsG, nf):
    """FSAI factor values, the arithmetic of ``FSAI_kernel`` (FSAIP_CUDA.cu:92-160).

    For row i with pattern P_i (m entries, diagonal last) and harmonic
    k = 0..nf-1: S = Re A[P_i,P_i] + i*k*Im A[P_i,P_i] (symmetric fill
    from tril, :117-137), y = S^-1 e_m (:144-150), g_i = y / sqrt(y_m)
    (:152-158).  Returns ``[nnzG, nf]`` complex128 (the layout after the
    transpose at dMesh.m:1384).
    """
    Are = sp.csr_matrix(A_tril_re)
    Aim = sp.csr_matrix(A_tril_im)
    n = Are.shape[0]
    m_row = np.diff(rptrG)
    out = np.zeros((colsG.shape[0], nf), dtype=np.complex128)
    kk = np.arange(nf, dtype=np.float64)
    for m in np.unique(m_row):
        rows = np.nonzero(m_row == m)[0]
        if m == 0:
            continue
        P = np.stack([colsG[rptrG[r]:rptrG[r] + m] for r in rows])          # [R, m]
        aa, bb = np.tril_indices(m)
        ri, ci = P[:, aa], P[:, bb]                                           # ri >= ci
        sre = np.asarray(Are[ri.ravel(), ci.ravel()]).reshape(ri.shape)
        sim = np.asarray(Aim[ri.ravel(), ci.ravel()]).reshape(ri.shape)
        S0 = np.zeros((rows.size, m, m))
        S1 = np.zeros((rows.size, m, m))
        S0[:, aa, bb] = sre; S0[:, bb, aa] = sre
        S1[:, aa, bb] = sim; S1[:, bb, aa] = sim
        S = S0[:, None] + 1j * kk[None, :, None, None] * S1[:, None]          # [R, nf, m, m]
        e = np.zeros((m,), dtype=np.complex128); e[m - 1] = 1.0
        y = np.linalg.solve(S, np.broadcast_to(e, S.shape[:-1])[..., None])[..., 0]  # [R, nf, m]
        g = y / complex_sqrt_ref(y[..., m - 1])[..., None]
        slots = rptrG[rows][:, None] + np.arange(m)[None, :]                   # [R, m]
        out[slots.ravel()] = np.transpose(g, (0, 2, 1)).reshape(-1, nf)
    return out


# ---------------------------------------------------------- mex kernel math
def smv(x, fAxis, K, Mi):
    """``smv_kernel`` (smv_CUDA.cu:8-54): y[:,s,k] = (Re A + i*fAxis[k]*Im A) x[:,s,k]
    with Re A = K and Im A = ``Mi`` (already scaled by df/c)."""
    y = np.empty_like(x)
    for k in range(x.shape[2]):
        y[:, :, k] = K @ x[:, :, k] + 1j * fAxis[k] * (Mi @ x[:, :, k])
    return y


def fsai_apply(x, G, rptr, cols, n):
    """``FSAImv_kernel`` (FSAImv_CUDA.cu:8-53): y[:,s,k] = G_k x[:,s,k], G_k values = G[:, k]."""
    y = np.empty_like(x)
    for k in range(x.shape[2]):
        Gk = sp.csr_matrix((G[:, k], cols, rptr), shape=(n, n))
        y[:, :, k] = Gk @ x[:, :, k]
    return y


# ------------------------------------------------------------------ BiCGSTAB
class FsaiPrecond:
    """G, its transpose and the A operator for all harmonics, dMesh.m:1253-1274."""

    def __init__(self, K, M, dfc, nf, cap=30):
        K = sp.csr_matrix(K); M = sp.csr_matrix(M)
        self.n = K.shape[0]
        self.K, self.Mi = K, (dfc * M).tocsr()
        A_tril = sp.tril(K + 1j * dfc * M).tocsr()
        self.rptrG, self.colsG = fsai_pattern(A_tril, cap)
        self.G = fsai_factor(sp.tril(K).tocsr(), sp.tril(dfc * M).tocsr(), self.rptrG, self.colsG, nf)
        self.rptrT, self.colsT, perm = transpose_pattern(self.rptrG, self.colsG, self.n)
        self.GT = self.G[perm]
        self.fAxis = np.arange(nf, dtype=np.float64)                          # :1260

    def A(self, x):
        return smv(x, self.fAxis, self.K, self.Mi)

    def Gm(self, x):
        return fsai_apply(x, self.G, self.rptrG, self.colsG, self.n)

    def GTm(self, x):
        return fsai_apply(x, self.GT, self.rptrT, self.colsT, self.n)


def _colsum(a):
    return a.sum(axis=0)


def _maxerr(e):
    with np.errstate(invalid="ignore"):
        return np.nan if np.all(np.isnan(e)) else np.nanmax(e)


def bicgstab_fsai(pc: FsaiPrecond, Q, tol=1e-12, maxit=1000, history=None):
    """``gpuBicstab_FSAIP`` (dMesh.m:1247-1348) on Q ``[NN, NS, NF]``.

    Bilinear (unconjugated) dot products, alph = 1/alpha, omega in the
    G-weighted bilinear form, and a stop once the maximum over all columns
    of the relative residual is below ``tol``.  Returns (x, iterations).
    """
    x = np.zeros_like(Q)                                                      # :1283
    r = Q - pc.A(x)                                                           # :1284-1285
    with np.errstate(invalid="ignore", divide="ignore"):
        err0 = np.sqrt(_colsum(np.abs(r) ** 2))                               # :1286
        rhat0 = r.copy()                                                      # :1288
        rho0 = _colsum(rhat0 * r)                                             # :1289
        p = r.copy()                                                          # :1290
        it = 0
        for it in range(1, maxit + 1):                                        # :1293
            h = pc.GTm(pc.Gm(p))                                              # :1295-1296
            v = pc.A(h)                                                       # :1301
            alph = _colsum(v * rhat0) / rho0                                  # :1304
            h = x + h / alph                                                  # :1305
            s = r - v / alph                                                  # :1306
            err = _maxerr(np.sqrt(_colsum(np.abs(s) ** 2)) / err0)            # :1307-1308
            if history is not None:
                history.append(err)
            if err < tol:                                                     # :1310-1313
                x = h
                break
            Gs = pc.Gm(s)                                                     # :1315
            z = pc.GTm(Gs)                                                    # :1316
            t = pc.A(z)                                                       # :1319
            Gtt = pc.Gm(t)                                                    # :1322
            om = _colsum(Gtt * Gs) / _colsum(Gtt * Gtt)                       # :1325
            x = h + om * z                                                    # :1327
            r = s - om * t                                                    # :1328
            p = p - om * v                                                    # :1329
            err = _maxerr(np.sqrt(_colsum(np.abs(r) ** 2)) / err0)            # :1330-1331
            if history is not None:
                history.append(err)
            if err < tol:                                                     # :1333-1335
                break
            rho = _colsum(rhat0 * r)                                          # :1337
            beta = rho / rho0 * (1.0 / (alph * om))                           # :1338
            rho0 = rho                                                        # :1339
            p = r + beta * p                                                  # :1340
    return x, it


def cocg_fsai(pc: FsaiPrecond, Q, tol=1e-12, maxit=4000):
    """Preconditioned COCG (conjugate-orthogonal CG) on the same systems and
    preconditioner as ``bicgstab_fsai``: A_k and M = G^T G are complex
    symmetric, so CG with bilinear dots applies.  Restates the library's
    mixed-precision inner solver (not a reference algorithm): per column
    alpha = (r.z)/(p.Ap), x += alpha p, r -= alpha Ap, z = M r,
    beta = (r.z)'/(r.z), p = z + beta p; stop when the largest relative
    residual is below tol.  Returns (x, iterations)."""
    x = np.zeros_like(Q)
    r = Q.copy()
    with np.errstate(invalid="ignore", divide="ignore"):
        e0 = np.sqrt(_colsum(np.abs(r) ** 2))
        z = pc.GTm(pc.Gm(r))
        p = z.copy()
        rho = _colsum(r * z)
        it = 0
        for it in range(1, maxit + 1):
            q = pc.A(p)
            alpha = rho / _colsum(p * q)
            x = x + alpha * p
            r = r - alpha * q
            if _maxerr(np.sqrt(_colsum(np.abs(r) ** 2)) / e0) < tol:
                break
            z = pc.GTm(pc.Gm(r))
            rn = _colsum(r * z)
            p = z + (rn / rho) * p
            rho = rn
    return x, it


# ------------------------------------------------------- sources / detectors
def source_vectors(elem, bary, fpsf, nn):
    """Q[:, s, k] = barycentric weights of optode s at its tet's nodes times
    s_fpsf[k], dMesh.m:124-129 (and :191-196 for the adjoint).  ``bary`` rows
    are [elem_id (0-based), w1..w4].  Returns ``[NN, NS, NF]``."""
    ns = bary.shape[0]
    q = np.zeros((nn, ns))
    for s in range(ns):
        q[np.asarray(elem)[int(bary[s, 0])], s] = bary[s, 1:5]
    return q[:, :, None] * np.asarray(fpsf)[None, None, :]


def meas_flu(elem, d_bary, link, phi):
    """Detector data ``[NM, NF]``, dMesh.m:144-171.  ``phi`` is ``[NN, NS, NF]``,
    ``link`` rows are (source, detector), 0-based."""
    nd = d_bary.shape[0]
    nn = phi.shape[0]
    D = np.zeros((nd, nn))
    for d in range(nd):
        w = d_bary[d, 1:5]
        nodes = np.asarray(elem)[int(d_bary[d, 0])]
        for l in range(4):
            if w[l] > 0:
                D[d, nodes[l]] += w[l]
    out = np.empty((link.shape[0], phi.shape[2]), dtype=np.complex128)
    for m, (s, d) in enumerate(link):
        out[m] = D[d] @ phi[:, s, :]
    return out


# --------------------------------------------------------------- FP64 truth
def direct_solve(K, M, dfc, Q):
    """Sparse-direct complex128 solve of (K + i*k*dfc*M) x = Q[:, :, k] for
    every harmonic k (the FP64 truth the iterative solves are measured
    against)."""
    K = sp.csc_matrix(K); M = sp.csc_matrix(M)
    x = np.empty_like(Q, dtype=np.complex128)
    for k in range(Q.shape[2]):
        lu = spla.splu((K + 1j * k * dfc * M).tocsc())
        x[:, :, k] = lu.solve(np.ascontiguousarray(Q[:, :, k]).astype(np.complex128))
    return x
