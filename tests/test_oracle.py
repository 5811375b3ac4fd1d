"""CPU tests of the oracle itself: identities the reference formulation must satisfy."""
import numpy as np
import pytest
import scipy.sparse as sp

from dogpup_b200.meshgen import box_mesh, cylinder_mesh, ellipsoid_mesh
from oracle import fem, solver, transforms, jacobian


def test_mesh_generators_are_conforming():
    for m in (cylinder_mesh(6, 8, 1.5, 0.2, 1), ellipsoid_mesh((12, 10, 8), 1.0, 0.1, 2), box_mesh((4, 3, 5), 1.0)):
        geo = fem.prepare_mesh(m.node, m.elem, 1.4)
        assert (geo["vol"] > 0).all()
        assert np.array_equal(geo["bnd"].astype(bool), m.bnd)
        # every interior face is shared by exactly two tets: surface = faces seen once
        assert geo["face"].shape[0] > 0


def test_mass_matrix_identities(small_case):
    K, M, geo = small_case["K"], small_case["M"], small_case["geo"]
    assert abs(M.sum() - geo["vol"].sum()) < 1e-9 * geo["vol"].sum()
    assert abs(M - M.T).max() < 1e-15 * abs(M).max()
    assert abs(K - K.T).max() < 1e-15 * abs(K).max()
    # P1 consistent mass of one tet: vol/20 (1 + delta_ij)
    m = small_case["mesh"]
    Ke, Me = fem.element_matrices(m.node, m.elem[:1], {"vol": geo["vol"][:1], "gradScale": geo["gradScale"][:1]},
                                  np.zeros(m.nn), np.zeros(m.nn))
    assert np.allclose(Me[0], geo["vol"][0] / 20 * (np.ones((4, 4)) + np.eye(4)), rtol=1e-14)


def test_stiffness_rows_vanish_without_absorption_or_boundary():
    m = box_mesh((3, 3, 3), 1.0, 0.2, 4)
    geo = fem.prepare_mesh(m.node, m.elem, 1.4)
    geo = dict(geo, bnd=np.zeros_like(geo["bnd"]), R=np.zeros(m.nn))
    K, M = fem.gen_fwdmat(m.node, m.elem, geo, 0.0, 1.0)
    assert np.abs(np.asarray(K.sum(axis=1))).max() < 1e-13


def test_absorption_term_equals_mua_times_mass():
    m = box_mesh((3, 3, 3), 1.0, 0.2, 5)
    geo = fem.prepare_mesh(m.node, m.elem, 1.4)
    geo0 = dict(geo, bnd=np.zeros_like(geo["bnd"]), R=np.zeros(m.nn))
    K1, M = fem.gen_fwdmat(m.node, m.elem, geo0, 0.02, 1.0)
    # kappa depends on mua: compare with the stiffness at the same kappa but mua = 0
    kap = 1.0 / (3.0 * (0.02 + 1.0))
    K0, _ = fem.gen_fwdmat(m.node, m.elem, geo0, 0.0, 1.0 / (3 * kap))
    assert abs((K1 - K0) - 0.02 * M).max() < 1e-14


def test_robin_face_rule_counts():
    m = cylinder_mesh(4, 4, 1.0, 0.0, 0)
    geo = fem.prepare_mesh(m.node, m.elem, 1.4)
    f = fem.robin_faces(m.elem, geo["bnd"])
    # includes every true surface face (as node sets)
    surf = {tuple(sorted(x)) for x in geo["face"]}
    rob = {tuple(x) for x in f}
    assert surf <= rob


def test_fsai_pattern_rule_rowwise_equals_global_sort(small_case):
    K, M = small_case["K"], small_case["M"]
    A = sp.tril(K + 1j * 3e-3 * M).tocsr()
    for cap in (30, 5, 3):
        r1, c1 = solver.fsai_pattern(A, cap)
        r2, c2 = solver.fsai_pattern_rowwise(A, cap)
        assert np.array_equal(r1, r2) and np.array_equal(c1, c2)


def test_fsai_identity(small_case):
    K, M = small_case["K"], small_case["M"]
    dfc = 2 * np.pi / 10e-9 / (2.99792458e11 / 1.4)
    pc = solver.FsaiPrecond(K, M, dfc, 6)
    n = K.shape[0]
    for k in range(6):
        Gk = sp.csr_matrix((pc.G[:, k], pc.colsG, pc.rptrG), shape=(n, n))
        d = (Gk @ (K + 1j * k * dfc * M) @ Gk.T).diagonal()
        assert np.abs(d - 1).max() < 1e-12


def test_bicgstab_matches_direct(small_case):
    K, M = small_case["K"], small_case["M"]
    dfc = 2 * np.pi / 10e-9 / (2.99792458e11 / 1.4)
    pc = solver.FsaiPrecond(K, M, dfc, 4)
    rng = np.random.default_rng(0)
    Q = np.zeros((K.shape[0], 3, 4), complex)
    for s in range(3):
        idx = rng.choice(K.shape[0], 4, replace=False)
        Q[idx, s, :] = rng.random(4)[:, None] * np.exp(0.3j * np.arange(4))[None]
    x, it = solver.bicgstab_fsai(pc, Q, 1e-12, 1000)
    xd = solver.direct_solve(K, M, dfc, Q)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-9
    assert 5 < it < 200


def test_cocg_matches_direct_and_bicgstab_iterations(small_case):
    """COCG (the mixed solver's inner method) on the same systems reaches the direct
    solution; per iteration it applies A and G^T G once (BiCGSTAB: twice), and needs
    fewer than twice BiCGSTAB's iterations."""
    K, M = small_case["K"], small_case["M"]
    dfc = 2 * np.pi / 10e-9 / (2.99792458e11 / 1.4)
    pc = solver.FsaiPrecond(K, M, dfc, 4)
    rng = np.random.default_rng(0)
    Q = np.zeros((K.shape[0], 3, 4), complex)
    for s in range(3):
        idx = rng.choice(K.shape[0], 4, replace=False)
        Q[idx, s, :] = rng.random(4)[:, None] * np.exp(0.3j * np.arange(4))[None]
    x, it = solver.cocg_fsai(pc, Q, 1e-12)
    xd = solver.direct_solve(K, M, dfc, Q)
    assert np.linalg.norm(x - xd) / np.linalg.norm(xd) < 1e-9
    _, itb = solver.bicgstab_fsai(pc, Q, 1e-12, 1000)
    assert it < 2 * itb


def test_transform_round_trip_and_gates():
    t = np.arange(0, 141) * 50e-12
    T = t[-1]
    nf = 40
    f = np.arange(nf) * 2 * np.pi / T
    x = transforms.gaussian_tpsf(t, 250e-12)
    c = transforms.td2fc(x, f, t)
    xr = transforms.fc2td(c, f, t)
    assert np.abs(xr - x).max() < 2e-3 * x.max()
    # fc2tg with gate coefficients = Nt * sum over the gate of x * gate / Nt (discrete Parseval)
    gates = np.stack([transforms.gaussian_tpsf(t - 1e-9 * g, 400e-12) for g in range(3)])
    gfc = transforms.td2fc(gates, f, t)
    y = transforms.fc2tg(c, gfc, f, t.size)
    direct = np.array([(gates[g] * x).sum() * (t[1] - t[0]) / T * 1.0 for g in range(3)])
    assert np.allclose(y * (t[1] - t[0]) / T / t.size * T / (t[1] - t[0]), direct, rtol=5e-3, atol=1e-6 * direct.max())


def test_tik_inv_matches_normal_equations():
    rng = np.random.default_rng(1)
    J = rng.standard_normal((40, 12))
    y = rng.standard_normal(40)
    u = jacobian.tik_inv(J, 0.1, y)
    H = J.T @ J + 0.1 * np.max((J ** 2).sum(0)) * np.eye(12)
    assert np.allclose(u, np.linalg.solve(H, J.T @ y), rtol=1e-12)
    w = rng.random(40) + 0.5
    uw = jacobian.tik_inv(J, 0.1, y, weights=w)
    Hw = J.T @ (w[:, None] * J) + 0.1 * np.max((w[:, None] * J ** 2).sum(0)) * np.eye(12)
    assert np.allclose(uw, np.linalg.solve(Hw, J.T @ (w * y)), rtol=1e-12)


def test_c_port_matches_numpy_oracle(small_case):
    """The C/OpenMP restatement used as the CPU baseline agrees with the numpy oracle."""
    from oracle import cport
    K, M = small_case["K"], small_case["M"]
    dfc = 2 * np.pi / 10e-9 / (2.99792458e11 / 1.4)
    k = 3
    A = sp.tril(K + 1j * dfc * M).tocsr()
    rg, cg = solver.fsai_pattern(A)
    G = cport.fsai_factor(sp.tril(K).tocsr(), sp.tril(k * dfc * M).tocsr(), rg, cg)
    G0 = solver.fsai_factor(sp.tril(K).tocsr(), sp.tril(dfc * M).tocsr(), rg, cg, k + 1)[:, k]
    assert np.abs(G - G0).max() <= 1e-12 * np.abs(G0).max()
    rt, ct, perm = solver.transpose_pattern(rg, cg, K.shape[0])
    rng = np.random.default_rng(2)
    B = np.zeros((K.shape[0], 3), complex)
    for c in range(3):
        B[rng.choice(K.shape[0], 4, replace=False), c] = rng.random(4)
    X, it = cport.bicgstab(K, M, k * dfc, rg, cg, G, rt, ct, G[perm], B, 1e-12)
    Xd = solver.direct_solve(K, M, k * dfc, np.stack([B, B], axis=2))[:, :, 1]   # harmonic 1 of k*dfc
    assert np.linalg.norm(X - Xd) / np.linalg.norm(Xd) < 1e-9
    assert (it > 3).all()


def test_morton_and_lattice_orders_are_the_same_mesh():
    a = cylinder_mesh(5, 6, 1.5, jitter=0.2, seed=4, order="lattice")
    b = cylinder_mesh(5, 6, 1.5, jitter=0.2, seed=4, order="morton")
    assert a.nn == b.nn and a.ne == b.ne
    # same node positions under the permutation given by the lattice coordinates
    ka = {tuple(x): i for i, x in enumerate(a.lattice)}
    perm = np.array([ka[tuple(x)] for x in b.lattice])
    assert np.array_equal(a.node[perm], b.node)
    assert np.array_equal(a.bnd[perm], b.bnd)
    ea = {tuple(sorted(e)) for e in a.elem.tolist()}
    eb = {tuple(sorted(perm[e])) for e in b.elem.tolist()}
    assert ea == eb
    # Morton order: consecutive runs of 64 nodes span compact lattice boxes
    spans = [np.ptp(b.lattice[i:i + 64], axis=0).max() for i in range(0, b.nn - 64, 64)]
    assert np.median(spans) <= 7


def test_point_location_oracle_against_kdtree_locator():
    """Brute-force point location vs the oracle's k-d tree candidate locator (two routes):
    the same in-mesh mask and the same interpolation of a linear field."""
    from dogpup_b200.grid import m2g_from_location
    from oracle.optode import locate_points
    m = ellipsoid_mesh((8, 7, 6), 1.2, 0.15, 3)
    lo, hi = m.node.min(0), m.node.max(0)
    xs = [np.arange(lo[d] - 0.7, hi[d] + 0.71, 0.9) for d in range(3)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    grid = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    eid = np.full(len(grid), -1)
    wts = np.zeros((len(grid), 4))
    for i, p in enumerate(grid):
        try:
            e, wi = locate_points(m.node, m.elem, p, k=32, eps=1e-12)
            eid[i], wts[i] = e[0], wi[0]
        except ValueError:
            pass
    m2g_host, inm_host = m2g_from_location(eid, wts, m.elem, m.nn)
    P, inm = jacobian.m2g_matrix(m.node, m.elem, grid)
    assert inm.sum() > 100 and (~inm).sum() > 100
    assert np.array_equal(inm, inm_host)
    f = m.node @ np.array([0.3, -1.1, 0.7]) + 2.0
    fg = grid @ np.array([0.3, -1.1, 0.7]) + 2.0
    assert np.abs(P @ f - np.where(inm, fg, 0)).max() < 1e-11
    assert np.abs(m2g_host @ f - P @ f).max() < 1e-11
    # rows sum to one inside, empty outside
    rs = np.asarray(P.sum(axis=1)).ravel()
    assert np.abs(rs[inm] - 1).max() < 1e-12 and not rs[~inm].any()


def test_g2m_oracle_properties():
    """g2m restatement: rows sum to 1; a node whose lattice cell is all in-mesh
    interpolates a linear voxel field exactly (barycentric weights); uncovered
    nodes take their nearest in-mesh voxel."""
    m = ellipsoid_mesh((8, 7, 6), 1.0, 0.1, 5)
    lo, hi = m.node.min(0), m.node.max(0)
    xs = [np.arange(lo[d] - 0.3, hi[d] + 0.9, 0.8) for d in range(3)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    grid = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    _, inm = jacobian.m2g_matrix(m.node, m.elem, grid)
    G = jacobian.g2m_matrix(m.node, xs, inm)
    assert np.abs(np.asarray(G.sum(axis=1)).ravel() - 1).max() < 1e-14
    assert not G[:, ~inm].count_nonzero()                          # only in-mesh voxels carry weight
    lin = np.array([0.3, -1.1, 0.7])
    fv = grid @ lin + 2.0
    n = [len(a) for a in xs]
    full = []
    for r, p in enumerate(m.node):
        c = [int(np.floor((p[k] - xs[k][0]) / 0.8)) for k in range(3)]
        corners = [c[0] + i + n[0] * (c[1] + j + n[1] * (c[2] + k)) for i in (0, 1) for j in (0, 1) for k in (0, 1)]
        full.append(all(inm[v] for v in corners))
    full = np.array(full)
    assert full.sum() > 50
    assert np.abs((G @ fv)[full] - (m.node[full] @ lin + 2.0)).max() < 1e-12
    single = np.diff(G.indptr) == 1
    for r in np.nonzero(single & ~full)[0][:20]:
        v = G.indices[G.indptr[r]]
        d2 = ((grid[inm] - m.node[r]) ** 2).sum(1)
        assert abs(((grid[v] - m.node[r]) ** 2).sum() - d2.min()) <= 1e-12 * max(1.0, d2.min()) or G.data[G.indptr[r]] == 1


def test_reshape_and_spot_oracles():
    """reshape_J's w solves w (J J^T + lam max diag I) = Js J^T; spots have unit
    (negative) mass over the whole grid and vanish outside the mesh."""
    rng = np.random.default_rng(4)
    J = rng.standard_normal((40, 300))
    Js = rng.standard_normal((6, 300))
    w = jacobian.reshape_j(J, Js, 0.05)
    A = J @ J.T
    A += 0.05 * A.diagonal().max() * np.eye(40)
    assert np.abs(w @ A - Js @ J.T).max() < 1e-10 * np.abs(Js @ J.T).max()
    g = np.stack(np.meshgrid(np.arange(10.0), np.arange(8.0), np.arange(6.0), indexing="ij"), -1).reshape(-1, 3)
    inm = g[:, 0] < 7
    for kind, wd in (("gauss", 1.5), ("square", 3.0)):
        t = jacobian.target_spots(g, np.ones(len(g), bool), [[3, 4, 2], [6.5, 1, 3]], wd, kind)
        assert np.allclose(t.sum(1), -1.0)
        t2 = jacobian.target_spots(g, inm, [[3, 4, 2], [6.5, 1, 3]], wd, kind)
        assert not t2[:, ~inm].any() and np.array_equal(t2[:, inm], t[:, inm])
    assert np.count_nonzero(jacobian.target_spots(g, inm, [[3, 4, 2]], 3.0, "square")) == 27


def test_closest_point_on_triangle_two_methods():
    """The Voronoi-region walk (the device kernel's method) and the projection-or-edges
    route agree."""
    from oracle.optode import closest_point_on_triangle_walk as walk
    from oracle.optode import closest_point_on_triangle as proj
    rng = np.random.default_rng(8)
    for _ in range(400):
        a, b, c = rng.standard_normal((3, 3))
        p = rng.standard_normal(3) * 2
        assert np.abs(walk(p, a, b, c) - proj(p, a, b, c)).max() < 1e-12


def test_grid_matrix_assembly_helpers():
    """m2g from (element, weights) drops zero weights as MATLAB's sparse does and leaves
    out-of-mesh rows empty; g2m from device rows skips -1 slots and zero weights."""
    from dogpup_b200.grid import g2m_from_rows, m2g_from_location
    elem = np.array([[0, 1, 2, 3], [1, 2, 3, 4]])
    eid = np.array([0, -1, 1])
    w = np.array([[0.25, 0.25, 0.5, 0.0], [0, 0, 0, 0], [0.1, 0.2, 0.3, 0.4]])
    P, inm = m2g_from_location(eid, w, elem, 5)
    assert P.shape == (3, 5) and np.array_equal(inm, [True, False, True])
    assert P.nnz == 3 + 4 and P[1].nnz == 0
    assert np.allclose(P.toarray()[2], [0, 0.1, 0.2, 0.3, 0.4]) and np.allclose(P.toarray()[0], [0.25, 0.25, 0.5, 0, 0])
    col = np.array([[3, -1, 5, 7], [-1, -1, -1, -1], [2, 4, 6, 8]])
    val = np.array([[0.5, 0.0, 0.5, 0.0], [0, 0, 0, 0], [0.25, 0.25, 0.25, 0.25]])
    G = g2m_from_rows(col, val, 10)
    assert G.shape == (3, 10) and G.nnz == 2 + 4
    assert np.allclose(G.toarray()[0], np.eye(10)[3] * 0.5 + np.eye(10)[5] * 0.5)
