"""Float64 restatement of the reverse-mode gradient of time-gated data (test infrastructure).

The reference forms the absorption Jacobian explicitly (J_complex,
DOGPUP/dMesh.m:206-247) and time-gates it with fc2tg (DOGPUP/fc2tg.m:25-32);
its J holds kappa fixed.  The library's backward pass computes the exact
discrete gradient of

    L(mua, musp) = sum_{m,g} g[m, g] * fc2tg(meas_flu(phi(mua, musp)))[m, g]

by one adjoint solve per source x harmonic.  This module restates that
computation with dense numpy on small meshes, so that the gradient can be
pinned against central finite differences of ``tg_forward`` (which is the
reference's forward chain: gen_fwdmat -> solve -> meas_flu -> fc2tg).

Layouts follow the oracle: fields ``[NN, NS, NF]``; detector data ``[NM, NF]``.
"""
from __future__ import annotations

import numpy as np

from . import fem, solver, transforms


def tg_forward(node, elem, geo, mua, musp, dfc, s_bary, d_bary, link, fpsf, gate_fc, nt):
    """data_tg [NM, NG] and phi [NN, NS, NF] by sparse-direct solves (FP64 truth)."""
    K, M = fem.gen_fwdmat(node, elem, geo, mua, musp)                    # dMesh.m:80-88
    Q = solver.source_vectors(elem, s_bary, fpsf, node.shape[0])         # dMesh.m:124-129
    phi = solver.direct_solve(K, M, dfc, Q)
    data = solver.meas_flu(elem, d_bary, link, phi)                      # dMesh.m:144-171
    f = np.arange(len(fpsf))
    return transforms.fc2tg(data, gate_fc, f, nt), phi, (K, M)


def tg_adjoint_rhs(elem, d_bary, link, gate_fc, nt, g, nn, ns):
    """dL/dphi as right-hand sides B [NN, NS, NF] (chain rule of fc2tg and meas_flu)."""
    nf = gate_fc.shape[1]
    h = np.ones(nf)
    h[0] = 0.5
    c = 2.0 * nt * h[None, :] * (np.asarray(g) @ np.conj(gate_fc))      # [NM, NF]
    B = np.zeros((nn, ns, nf), dtype=np.complex128)
    for m, (s, d) in enumerate(link):
        w = d_bary[d, 1:5]
        nodes = np.asarray(elem)[int(d_bary[d, 0])]
        for l in range(4):
            if w[l] > 0:
                B[nodes[l], s, :] += w[l] * c[m]
    return B


def adjoint_grad(node, elem, geo, mua, musp, phi, lam):
    """(dL/dmua, dL/dmusp) [NN] = -Re sum lam^T (dA/dp) phi through element_matrices."""
    elem = np.asarray(elem, dtype=np.int64)
    nn = node.shape[0]
    xa, ya, za, wt = fem.tet_quad()
    n3 = np.stack([1 - xa - ya - za, xa, ya, za])                       # [4, 5]
    ngrad = np.array([[-1.0, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    vol = geo["vol"]
    grads = np.einsum("eab,ib->eia", geo["gradScale"], ngrad)           # [NE, 4, 3]
    kap = 1.0 / (3.0 * (mua + musp))
    cv = n3 @ wt                                                         # sum_q w_q N_v(x_q)
    dk = -3.0 * kap[elem] ** 2 * cv[None, :] * vol[:, None]             # d(vol * ksum)/dp_v, [NE, 4]
    fe = phi[elem]                                                       # [NE, 4, NS, NF]
    le = lam[elem]
    fq = np.einsum("lq,elsk->eqsk", n3, fe)
    lq = np.einsum("lq,elsk->eqsk", n3, le)
    prod = np.real(lq * fq).sum(axis=(2, 3))                             # [NE, 5]
    absorb = vol[:, None] * np.einsum("q,lq,eq->el", wt, n3, prod)      # [NE, 4]
    gl = np.einsum("eld,elsk->edsk", grads, le)
    gp = np.einsum("eld,elsk->edsk", grads, fe)
    dot = np.real(gl * gp).sum(axis=(1, 2, 3))                           # [NE]
    stiff = dot[:, None] * dk
    gmua = np.zeros(nn)
    gmusp = np.zeros(nn)
    np.add.at(gmua, elem, -(absorb + stiff))
    np.add.at(gmusp, elem, -stiff)
    return gmua, gmusp
