"""Device point location (dgp_locate_points) against the oracle's brute-force
point location (every element tested), the device grid-to-mesh map
(dgp_grid_to_mesh) against the oracle's g2m, and the device mesh2grid basis.

Element ids must agree wherever the containing element is unique (the
oracle's best score above 1e-9); elsewhere -- points on shared faces, edges
or vertices -- any of the tied elements is correct, so the interpolation of a
linear field is compared instead (1e-11 absolute on O(10) values).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIN = np.array([0.3, -1.1, 0.7])


def _oracle_scores(node, elem, pts, eid):
    from oracle.jacobian import point_location
    e0, w0 = point_location(node, elem, pts)
    return e0, w0


def _check(node, elem, pts):
    from dogpup_b200 import api
    e_d, w_d = api.locate_points(node, elem, pts)
    eid, w = e_d.cpu().numpy(), w_d.cpu().numpy()
    e0, w0 = _oracle_scores(node, elem, pts, eid)
    assert np.array_equal(eid >= 0, e0 >= 0)
    inm = e0 >= 0
    unique = inm & (w0.min(axis=1) > 1e-9)
    assert np.array_equal(eid[unique], e0[unique])
    assert np.abs(w[unique] - w0[unique]).max(initial=0) < 1e-12
    # any tied element interpolates a linear field exactly
    f = node @ LIN + 2.0
    fi = (w[inm] * f[elem[eid[inm]]]).sum(axis=1)
    assert np.abs(fi - (pts[inm] @ LIN + 2.0)).max(initial=0) < 1e-11
    assert not w[~inm].any()
    assert np.abs(w[inm].sum(axis=1) - 1).max(initial=0) < 1e-12
    return eid, inm


def test_locate_ellipsoid_grid_inside_and_outside():
    from dogpup_b200.meshgen import ellipsoid_mesh
    m = ellipsoid_mesh((12, 10, 8), 1.0, 0.15, 7)
    lo, hi = m.node.min(0), m.node.max(0)
    xs = [np.arange(lo[d] - 1.3, hi[d] + 1.31, 0.7) for d in range(3)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    _, inm = _check(m.node, m.elem.astype(np.int64), pts)
    assert inm.sum() > 200 and (~inm).sum() > 200


def test_locate_points_on_vertices_faces_and_far_away():
    from dogpup_b200.meshgen import box_mesh
    m = box_mesh((4, 3, 5), 1.0)                     # lattice: grid points hit vertices, edges and faces
    xs = [np.arange(-0.5, s + 0.51, 0.5) for s in (4, 3, 5)]
    X, Y, Z = np.meshgrid(*xs, indexing="ij")
    pts = np.concatenate([np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1),
                          [[1e6, 0, 0], [-3, -3, -3], [2, 1.5, 1e3], [np.nan, 1, 1]]])
    # the NaN point is outside for the device and the oracle alike
    eid, inm = _check(m.node, m.elem.astype(np.int64), np.nan_to_num(pts, nan=-7.0))
    from dogpup_b200 import api
    e_nan, w_nan = api.locate_points(m.node, m.elem.astype(np.int64), pts[-1:])
    assert int(e_nan[0]) == -1 and not w_nan.any()
    assert (eid[-4:] == -1).all()


def test_locate_empty_and_single_point():
    from dogpup_b200 import api
    from dogpup_b200.meshgen import box_mesh
    m = box_mesh((2, 2, 2), 1.0)
    e, w = api.locate_points(m.node, m.elem.astype(np.int64), np.zeros((0, 3)))
    assert e.shape == (0,) and w.shape == (0, 4)
    _check(m.node, m.elem.astype(np.int64), np.array([[0.25, 0.5, 0.75]]))


def test_dmesh_mesh2grid_device_equals_oracle():
    """DMesh.mesh2grid (device point location) against the oracle's k-d tree host locator:
    the same in-mesh mask and the same interpolation of a linear field."""
    from dogpup_b200 import workloads
    from dogpup_b200.grid import m2g_from_location
    from oracle.jacobian import point_location
    w = workloads.small_fwd(ns=2, nd=2, nf=4)
    mesh = workloads.build_dmesh(w)
    lo, hi = w["mesh"].node.min(0), w["mesh"].node.max(0)
    xs = [np.arange(lo[d] - 2, hi[d] + 2.001, 1.5) for d in range(3)]
    mesh.mesh2grid(*xs)
    P_host, inm_host = m2g_from_location(*point_location(mesh.node_host, mesh.elem_host, mesh.grid, chunk=8),
                                         mesh.elem_host, mesh.nn)
    assert np.array_equal(mesh.gridinmesh, inm_host)
    f = mesh.node_host @ LIN + 2.0
    assert np.abs(mesh.m2g @ f - P_host @ f).max() < 1e-11
    g = mesh.grid @ LIN + 2.0
    assert np.abs((mesh.m2g @ f)[mesh.gridinmesh] - g[mesh.gridinmesh]).max() < 1e-11


def _g2m_check(node, axes, inm):
    """Device g2m rows vs the oracle's g2m: same pattern, weights to 1e-15;
    nearest-voxel rows may differ only between voxels at equal distance."""
    from dogpup_b200 import api
    from dogpup_b200.grid import g2m_from_rows
    from oracle.jacobian import g2m_matrix
    col, val = api.grid_to_mesh(node, axes, inm)
    nv = int(np.prod([len(a) for a in axes]))
    G = g2m_from_rows(col.cpu().numpy(), val.cpu().numpy(), nv)
    _g2m_compare(G, g2m_matrix(node, axes, inm), node, axes)
    return G


def _g2m_compare(G, G0, node, axes):
    # rows sum to 1, or to 0 where the only in-mesh voxels of the node's simplex
    # carry weight 0 (the reference's rule then adds no nearest voxel either)
    rs = np.asarray(G.sum(axis=1)).ravel()
    assert np.minimum(np.abs(rs - 1), np.abs(rs)).max() < 1e-14
    diff = abs(G - G0).tocsr()
    bad = np.nonzero(np.asarray(diff.max(axis=1).todense()).ravel() > 1e-15)[0]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    grid = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    for r in bad:                                   # only nearest-voxel ties may differ
        assert G.indptr[r + 1] - G.indptr[r] == 1 and G0.indptr[r + 1] - G0.indptr[r] == 1
        v, v0 = G.indices[G.indptr[r]], G0.indices[G0.indptr[r]]
        d, d0 = ((grid[v] - node[r]) ** 2).sum(), ((grid[v0] - node[r]) ** 2).sum()
        assert abs(d - d0) <= 1e-12 * max(d0, 1.0)


def test_g2m_ellipsoid_partial_grid():
    """Lattice that stops short of the mesh on two sides: nodes outside it and
    nodes with no in-mesh voxel take the nearest in-mesh voxel."""
    from dogpup_b200.meshgen import ellipsoid_mesh
    from oracle.jacobian import m2g_matrix
    m = ellipsoid_mesh((12, 10, 8), 1.0, 0.15, 9)
    lo, hi = m.node.min(0), m.node.max(0)
    axes = [np.arange(lo[0] + 1.1, hi[0] + 0.8, 0.75), np.arange(lo[1] - 0.4, hi[1] - 0.9, 0.75),
            np.arange(lo[2] - 0.4, hi[2] + 0.8, 0.75)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    grid = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    _, inm = m2g_matrix(m.node, m.elem, grid)
    G = _g2m_check(m.node, axes, inm)
    assert (np.diff(G.indptr) == 1).sum() > 20      # the nearest-voxel rule was exercised


def test_g2m_nodes_on_lattice_points_and_descending_axis():
    from dogpup_b200.meshgen import box_mesh
    from oracle.jacobian import m2g_matrix
    m = box_mesh((4, 3, 5), 1.0)
    axes = [np.arange(4.5, -0.51, -0.5), np.arange(0.0, 3.01, 1.0), np.arange(-0.5, 5.51, 0.5)]
    X, Y, Z = np.meshgrid(*axes, indexing="ij")
    grid = np.stack([X.ravel(order="F"), Y.ravel(order="F"), Z.ravel(order="F")], axis=1)
    _, inm = m2g_matrix(m.node, m.elem, grid)
    _g2m_check(m.node, axes, inm)


def test_dmesh_g2m_is_the_oracle_g2m():
    from dogpup_b200 import workloads
    from oracle.jacobian import g2m_matrix
    w = workloads.small_fwd(ns=2, nd=2, nf=4)
    mesh = workloads.build_dmesh(w)
    lo, hi = w["mesh"].node.min(0), w["mesh"].node.max(0)
    xs = [np.arange(lo[d] - 2, hi[d] + 2.001, 1.5) for d in range(3)]
    mesh.mesh2grid(*xs)
    _g2m_compare(mesh.g2m, g2m_matrix(mesh.node_host, xs, mesh.gridinmesh), mesh.node_host, xs)


def _snap_case(with_w=False):
    from dogpup_b200 import workloads
    w = workloads.small_fwd(ns=8, nd=8, nf=4)
    mesh = workloads.build_dmesh(w)
    if with_w:
        return mesh, w
    rng = np.random.default_rng(5)
    c = w["mesh"].node.mean(0)
    pos = np.concatenate([w["src"], w["det"], c + rng.standard_normal((40, 3)) * [14, 14, 10],
                          mesh.node_host[np.nonzero(mesh.bnd_host)[0][:5]]])      # exactly on boundary nodes
    return mesh, pos


def test_snap_to_surface_against_oracle():
    """Surface points to 1e-12 and normals to 1e-12; where two candidate faces are equally
    close (the point lands on their shared edge) either face's normal is accepted."""
    from dogpup_b200 import api
    from oracle.optode import snap_pos
    mesh, pos = _snap_case()
    q, d, f = api.snap_to_surface(mesh.node_host, mesh.fem.bnd, mesh.face_host, pos)
    q, d, f = q.cpu().numpy(), d.cpu().numpy(), f.cpu().numpy()
    q0, d0, f0, dists = snap_pos(mesh.node_host, mesh.bnd_host, mesh.face_host, pos)
    assert np.abs(q - q0).max() < 1e-12
    for i in range(len(pos)):
        tie = len(dists[i]) > 1 and dists[i][1] - dists[i][0] <= 1e-12 * max(1.0, dists[i][0])
        if not tie:
            assert f[i] == f0[i]
            assert np.abs(d[i] - d0[i]).max() < 1e-12
    assert np.allclose(np.linalg.norm(d, axis=1), 1.0)


def test_snap_rejects_a_mesh_without_boundary():
    from dogpup_b200 import api
    from dogpup_b200._lib import DgpError
    mesh, pos = _snap_case()
    with pytest.raises(DgpError):
        api.snap_to_surface(mesh.node_host, np.zeros(mesh.nn, np.int32), mesh.face_host, pos[:3])


def test_optode_snap_device_equals_oracle():
    """DOptode.snap2mesh on the device against the oracle's snap2mesh on the host: same
    surface points, normals and source/detector points (the weighted vertices of the
    located elements)."""
    from dogpup_b200.optode import DOptode
    from dogpup_b200.workloads import gaussian_pulse
    from oracle.optode import snap2mesh
    mesh, w = _snap_case(with_w=True)
    t = w["t"]
    o_dev = DOptode(w["src"], w["det"], w["link"], 1e3, gaussian_pulse(t), t, w["nf"])
    o_dev.snap2mesh(mesh)
    sq, sn, s_bary, dq, dn, d_bary = snap2mesh(mesh.node_host, mesh.elem_host, mesh.bnd_host, mesh.face_host,
                                               mesh.musp_host, w["src"], w["det"])
    assert np.abs(sq - o_dev.s_positions).max() < 1e-12
    assert np.abs(dq - o_dev.d_positions).max() < 1e-12
    assert np.abs(sn - o_dev.s_dirs).max() < 1e-12
    for b_dev, b_host in ((o_dev.s_bary, s_bary), (o_dev.d_bary, d_bary)):
        pt = lambda b: (b[:, 1:, None] * mesh.node_host[mesh.elem_host[b[:, 0].astype(int)]]).sum(1)
        assert np.abs(pt(b_dev) - pt(b_host)).max() < 1e-9


def test_locate_and_snap_reject_out_of_range_node_ids():
    """An element or face node id outside [0, nn) is DGP_ERR_MESH, raised before any
    kernel indexes the node array with it; a valid call afterwards still works."""
    from dogpup_b200 import api
    from dogpup_b200._lib import DgpError
    from dogpup_b200.meshgen import box_mesh
    m = box_mesh((3, 3, 3), 1.0)
    pts = np.array([[1.5, 1.5, 1.5]])
    for bad in (m.node.shape[0], -1):
        elem = m.elem.astype(np.int64).copy()
        elem[5, 2] = bad
        with pytest.raises(DgpError) as ei:
            api.locate_points(m.node, elem, pts)
        assert ei.value.code == 4 and "node index out of range" in str(ei.value)
    eid, _ = api.locate_points(m.node, m.elem.astype(np.int64), pts)
    assert int(eid[0]) >= 0
    mesh, pos = _snap_case()
    for bad in (mesh.nn, -7):
        face = np.array(mesh.face_host, copy=True)
        face[3, 1] = bad
        with pytest.raises(DgpError) as ei:
            api.snap_to_surface(mesh.node_host, mesh.fem.bnd, face, pos[:3])
        assert ei.value.code == 4 and "node index out of range" in str(ei.value)
