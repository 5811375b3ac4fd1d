"""dMesh / dOptode records (dogpup_b200.caseio): .mat and .npz round trips with MATLAB's
1-based indices on the CPU; on the GPU a DMesh saved and rebuilt from its record gives the
same detector data (identical inputs; only the order of the solver's FP64 atomic dot
partials may differ: 1e-12 relative)."""
import numpy as np
import pytest
import scipy.sparse as sp

from dogpup_b200 import caseio
from dogpup_b200.meshgen import cylinder_mesh


def _record():
    m = cylinder_mesh(5, 6, 1.5, jitter=0.2, seed=1)
    rng = np.random.default_rng(0)
    K = sp.random(m.nn, m.nn, density=0.01, random_state=1, format="csc")
    opt = dict(s_bary=np.c_[rng.integers(0, m.ne, 3), rng.random((3, 4))], d_bary=np.c_[[0, 5], rng.random((2, 4))],
               link=np.array([[0, 0], [2, 1]]), fAxis=np.arange(4) * 0.1, tAxis=np.linspace(0, 1, 5), Nf=4, df=0.1,
               s_fpsf=rng.standard_normal(4) + 1j * rng.standard_normal(4))
    return dict(node=m.node, elem=m.elem.astype(np.int64), nr=1.4, mua=np.full(m.nn, 0.01), musp=np.ones(m.nn),
                K=K, optode=opt)


@pytest.mark.parametrize("fmt", ["mat", "npz"])
def test_record_round_trip(tmp_path, fmt):
    rec = _record()
    p = tmp_path / f"mesh.{fmt}"
    getattr(caseio, f"save_{fmt}")(p, rec)
    back = getattr(caseio, f"load_{fmt}")(p)
    assert np.array_equal(back["elem"], rec["elem"]) and np.allclose(back["node"], rec["node"])
    assert abs(back["K"] - rec["K"]).max() == 0
    o, o0 = back["optode"], rec["optode"]
    assert np.array_equal(np.asarray(o["link"]).reshape(-1, 2), o0["link"])
    assert np.allclose(o["s_bary"], o0["s_bary"]) and np.allclose(o["s_fpsf"], o0["s_fpsf"])


def test_mat_file_uses_one_based_indices(tmp_path):
    import scipy.io
    rec = _record()
    caseio.save_mat(tmp_path / "m.mat", rec)
    raw = scipy.io.loadmat(str(tmp_path / "m.mat"))
    assert raw["elem"].min() == 1 and raw["elem"].max() == rec["elem"].max() + 1


@pytest.mark.gpu
def test_dmesh_record_rebuild_gives_same_data(tmp_path):
    from dogpup_b200 import workloads
    w = workloads.small_fwd(ns=3, nd=3, nf=4)
    mesh = workloads.build_dmesh(w)
    _, d0 = mesh.flu_solve(precision="fp64", tol=1e-12)
    caseio.save_mat(tmp_path / "m.mat", caseio.mesh_record(mesh))
    mesh2 = caseio.dmesh_from_record(caseio.load_mat(tmp_path / "m.mat"))
    _, d1 = mesh2.flu_solve(precision="fp64", tol=1e-12)
    a, b = d0.cpu().numpy(), d1.cpu().numpy()
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()
