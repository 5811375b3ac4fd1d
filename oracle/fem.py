"""Float64 restatement of DOGPUP's mesh preparation and FEM assembly.

Restates ``prepare_mesh`` (DOGPUP/dMesh.m:945-1030) and ``gen_fwdmat`` with
its quadrature tables (DOGPUP/dMesh.m:1033-1235), vectorised over elements.
Node and element indices are 0-based here (MATLAB's are 1-based).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

C_VAC = 2.99792458e11  # mm/s, DOGPUP/dMesh.m:42


def tet_quad():
    """Keast 5-point rule, DOGPUP/dMesh.m:1197-1216 (weights sum to 1)."""
    xa = np.array([1 / 4, 1 / 2, 1 / 6, 1 / 6, 1 / 6])
    ya = np.array([1 / 4, 1 / 6, 1 / 6, 1 / 6, 1 / 2])
    za = np.array([1 / 4, 1 / 6, 1 / 6, 1 / 2, 1 / 6])
    wt = np.array([-0.8, 0.45, 0.45, 0.45, 0.45])
    return xa, ya, za, wt


def tri_quad():
    """3-point order-2 triangle rule, DOGPUP/dMesh.m:1219-1235."""
    xa = np.array([2 / 3, 1 / 6, 1 / 6])
    ya = np.array([1 / 6, 2 / 3, 1 / 6])
    wt = np.array([1 / 3, 1 / 3, 1 / 3])
    return xa, ya, wt


def robin_factor(nr: float) -> float:
    """Nodal Robin coefficient 1/(2A) for a medium-air boundary, DOGPUP/dMesh.m:1008-1011."""
    r0 = (nr - 1.0) ** 2 / (nr + 1.0) ** 2
    theta_c = np.arcsin(1.0 / nr)
    ct = abs(np.cos(theta_c))
    a = (2.0 / (1.0 - r0) - 1.0 + ct ** 3) / (1.0 - ct ** 2)
    return 1.0 / (2.0 * a)


def prepare_mesh(node: np.ndarray, elem: np.ndarray, nr: float) -> dict:
    """Geometry for assembly, DOGPUP/dMesh.m:945-1030.

    Returns c (speed of light in the medium), vol, the true surface faces,
    the boundary flags ``bnd``, the nodal Robin factor ``R`` and the per-tet
    ``gradScale`` = inv(B^T) with B = [v2-v1, v3-v1, v4-v1].
    """
    node = np.asarray(node, dtype=np.float64)
    elem = np.asarray(elem, dtype=np.int64)
    c = C_VAC / nr                                                      # :949
    a = node[elem[:, 1]] - node[elem[:, 0]]                             # :952-955
    b = node[elem[:, 2]] - node[elem[:, 0]]
    cc = node[elem[:, 3]] - node[elem[:, 0]]
    vol = np.abs(np.einsum("ij,ij->i", np.cross(a, b), cc) / 6.0)
    faces = np.concatenate([elem[:, [0, 1, 2]], elem[:, [0, 1, 3]],     # :964-967
                            elem[:, [0, 2, 3]], elem[:, [1, 2, 3]]])
    _, ix, jx, cnt = np.unique(np.sort(faces, axis=1), axis=0, return_index=True,
                               return_inverse=True, return_counts=True)  # :969-972
    face = faces[ix[cnt == 1]]                                          # :973
    bnd = np.zeros(node.shape[0], dtype=np.int64)                       # :978-980
    bnd[np.unique(face.ravel())] = 1
    R = robin_factor(nr) * bnd                                          # :1008-1011
    B = np.stack([a, b, cc], axis=2)                                    # columns = edge vectors, :1017-1019
    grad_scale = np.linalg.inv(np.transpose(B, (0, 2, 1)))              # inv(B^T), :1020-1023
    return dict(c=c, vol=vol, face=face, bnd=bnd, R=R, gradScale=grad_scale, nr=nr)


def robin_faces(elem: np.ndarray, bnd: np.ndarray) -> np.ndarray:
    """The face set the reference integrates the Robin term over, DOGPUP/dMesh.m:1129-1140.

    Every tet with all 4 nodes on the boundary contributes its 4 faces; every
    tet with exactly 3 boundary nodes contributes the face of those 3 nodes
    (so interior faces whose nodes all lie on the surface are included, and a
    face shared by two such tets appears twice).
    """
    s = np.sort(np.asarray(elem, dtype=np.int64), axis=1)
    flag = np.asarray(bnd)[s] != 0
    cnt = flag.sum(axis=1)
    four = s[cnt == 4]
    f4 = np.concatenate([four[:, [0, 1, 2]], four[:, [0, 1, 3]], four[:, [0, 2, 3]], four[:, [1, 2, 3]]])
    three = s[cnt == 3]
    fl3 = flag[cnt == 3]
    f3 = three[fl3].reshape(-1, 3)          # the 3 flagged ids, ascending
    return np.concatenate([f4, f3]).astype(np.int64)


def element_matrices(node, elem, geo, mua, kappa):
    """Per-tet 4x4 K and M blocks, DOGPUP/dMesh.m:1055-1121."""
    elem = np.asarray(elem, dtype=np.int64)
    xa, ya, za, wt = tet_quad()
    n3 = np.stack([1 - xa - ya - za, xa, ya, za])                    # [4 basis, 5 q], :1060
    ngrad = np.array([[-1.0, -1, -1], [1, 0, 0], [0, 1, 0], [0, 0, 1]])  # :1061
    vol = geo["vol"]
    kq = (kappa[elem] @ n3) * wt                                      # [NE, 5], :1083,1086
    mq = (mua[elem] @ n3) * wt                                        # :1084,1087
    grads = np.einsum("eab,ib->eia", geo["gradScale"], ngrad)         # [NE, 4, 3], :1103-1104
    gg = np.einsum("eia,eja->eij", grads, grads)                      # gradI . gradJ, :1107-1108
    stiff = vol[:, None, None] * gg * kq.sum(axis=1)[:, None, None]   # :1109-1110
    absrp = vol[:, None, None] * np.einsum("eq,iq,jq->eij", mq, n3, n3)   # :1113
    mass = vol[:, None, None] * np.einsum("q,iq,jq->ij", wt, n3, n3)[None]  # :1118
    return stiff + absrp, np.broadcast_to(mass, stiff.shape).copy()


def gen_fwdmat(node, elem, geo, mua, musp, full=True):
    """Assemble K (stiffness + absorption + Robin) and M (mass), DOGPUP/dMesh.m:1033-1194.

    The reference returns ``triu(K)``, ``triu(M)`` (:1189-1190) and later
    symmetrises (:1242); with ``full=True`` the symmetric matrices are
    returned directly as CSR with sorted column indices.
    """
    node = np.asarray(node, dtype=np.float64)
    elem = np.asarray(elem, dtype=np.int64)
    nn = node.shape[0]
    mua = np.asarray(mua, dtype=np.float64) * np.ones(nn)
    musp = np.asarray(musp, dtype=np.float64) * np.ones(nn)
    kappa = 1.0 / (3.0 * (mua + musp))                                # :74, :85
    Ke, Me = element_matrices(node, elem, geo, mua, kappa)
    ii = np.repeat(elem, 4, axis=1).ravel()                           # elemMapI, :1073-1077
    jj = np.tile(elem, (1, 4)).ravel()
    K = sp.coo_matrix((Ke.ravel(), (ii, jj)), shape=(nn, nn)).tocsr()  # :1123
    M = sp.coo_matrix((Me.ravel(), (ii, jj)), shape=(nn, nn)).tocsr()  # :1124
    bf = robin_faces(elem, geo["bnd"])                                # :1129-1140
    if bf.shape[0]:
        a = node[bf[:, 1]] - node[bf[:, 0]]                           # :1143-1146
        b = node[bf[:, 2]] - node[bf[:, 0]]
        area = 0.5 * np.sqrt((np.cross(a, b) ** 2).sum(axis=1))
        xa, ya, wt = tri_quad()
        n2 = np.stack([1 - xa - ya, xa, ya])                          # [3, 3 q], :1063
        rq = (geo["R"][bf] @ n2) * wt                                 # :1159-1163
        Be = area[:, None, None] * np.einsum("fq,iq,jq->fij", rq, n2, n2)  # :1170-1179
        bi = np.repeat(bf, 3, axis=1).ravel()
        bj = np.tile(bf, (1, 3)).ravel()
        K = K + sp.coo_matrix((Be.ravel(), (bi, bj)), shape=(nn, nn)).tocsr()  # :1181
    K = K.tocsr()
    M = M.tocsr()
    K.sort_indices()
    M.sort_indices()
    if not full:
        return sp.triu(K).tocsr(), sp.triu(M).tocsr()
    return K, M


def shared_pattern(K, M):
    """K and M as values on their common CSR pattern.

    Both come from the same element (i, j) pairs and every Robin face lies in
    one tet, so the two patterns are identical; this is asserted.
    """
    assert np.array_equal(K.indptr, M.indptr) and np.array_equal(K.indices, M.indices)
    return K.indptr.astype(np.int64), K.indices.astype(np.int64), K.data.copy(), M.data.copy()
