"""Case files for the standalone C++ driver (dogpup_b200/driver/dgp_forward.cpp).

``write_case`` stores one forward problem -- mesh, nodal mua / musp, the
snapped optodes' barycentric nodes and weights, links and the source
spectrum -- in the driver's little-endian ``DGPCASE1`` layout; ``read_data``
reads the detector data the driver writes (``DGPDATA1``).  The fields are
those of the reference's dMesh / dOptode objects (DOGPUP/dMesh.m:4-38,
DOGPUP/dOptode.m:5-28) with 0-based indices.
"""
from __future__ import annotations

import numpy as np


def case_arrays(mesh) -> dict:
    """The driver's inputs from a DMesh with optodes attached."""
    o = mesh.optode
    elem = mesh.elem_host

    def bary(b):
        b = np.asarray(b)
        return elem[b[:, 0].astype(np.int64)].astype(np.int32), np.ascontiguousarray(b[:, 1:5], dtype=np.float64)

    sn, sw = bary(o.s_bary)
    dn, dw = bary(o.d_bary)
    return dict(node=mesh.node_host, elem=elem.astype(np.int32), mua=mesh.mua.cpu().numpy(),
                musp=mesh.musp.cpu().numpy(), src_nodes=sn, src_w=sw, det_nodes=dn, det_w=dw,
                link=o.link.astype(np.int32), fpsf=o.s_fpsf.cpu().numpy().astype(np.complex128), nr=mesh.nr,
                dfc=o.df / mesh.c)


def write_case(path, a: dict) -> None:
    nn, ne = a["node"].shape[0], a["elem"].shape[0]
    ns, nd, nm, nf = a["src_nodes"].shape[0], a["det_nodes"].shape[0], a["link"].shape[0], a["fpsf"].shape[0]
    with open(path, "wb") as f:
        f.write(b"DGPCASE1")
        f.write(np.array([nn, ne, ns, nd, nm, nf], dtype="<i8").tobytes())
        f.write(np.array([a["nr"], a["dfc"]], dtype="<f8").tobytes())
        for key, dt in (("node", "<f8"), ("elem", "<i4"), ("mua", "<f8"), ("musp", "<f8"), ("src_nodes", "<i4"),
                        ("src_w", "<f8"), ("det_nodes", "<i4"), ("det_w", "<f8"), ("link", "<i4")):
            f.write(np.ascontiguousarray(a[key], dtype=dt).tobytes())
        f.write(np.ascontiguousarray(a["fpsf"], dtype="<c16").view("<f8").tobytes())


def read_data(path) -> np.ndarray:
    """Detector data [NM][NF] complex128 written by the driver."""
    with open(path, "rb") as f:
        if f.read(8) != b"DGPDATA1":
            raise ValueError("not a DGPDATA1 file")
        nm, nf = np.frombuffer(f.read(16), dtype="<i8")
        return np.frombuffer(f.read(), dtype="<f8").view("<c16").reshape(int(nm), int(nf)).copy()


# ---------------------------------------------------------------- interchange
# dMesh / dOptode property records (DOGPUP/dMesh.m:4-38, DOGPUP/dOptode.m:5-28) for MATLAB
# users: .mat (scipy.io, MATLAB v5) or .npz, with MATLAB's 1-based element / node / optode
# indices, so a record saved here loads into the reference's classes field by field.
_MESH_FIELDS = ("node", "elem", "vol", "face", "bnd", "nr", "c", "mua", "musp", "kappa", "K", "M")
_OPTODE_FIELDS = ("s_dirs", "s_positions", "s_bary", "s_avgPow", "s_tpsf", "s_fpsf", "d_dirs", "d_positions",
                  "d_bary", "dt", "tAxis", "Nf", "df", "fAxis", "link")
_ONE_BASED = {"elem", "face", "link"}           # index arrays
_BARY = {"s_bary", "d_bary"}                     # column 0 is an element index


def mesh_record(mesh) -> dict:
    """dMesh-style record of a DMesh (with its optode when attached), 0-based."""
    import scipy.sparse as sp
    rp = mesh.fem.rowptr.cpu().numpy()
    cl = mesh.fem.col.cpu().numpy()
    n = mesh.nn
    K = sp.csr_matrix((mesh.K.cpu().numpy(), cl, rp), shape=(n, n))
    M = sp.csr_matrix((mesh.M.cpu().numpy(), cl, rp), shape=(n, n))
    node, elem = mesh.node_host, mesh.elem_host
    a = node[elem[:, 1]] - node[elem[:, 0]]
    b = node[elem[:, 2]] - node[elem[:, 0]]
    c = node[elem[:, 3]] - node[elem[:, 0]]
    vol = np.abs(np.einsum("ij,ij->i", np.cross(a, b), c)) / 6.0
    rec = dict(node=node, elem=elem, vol=vol, face=mesh.face_host, bnd=mesh.bnd_host.astype(np.float64),
               nr=float(mesh.nr), c=float(mesh.c), mua=mesh.mua.cpu().numpy(), musp=mesh.musp.cpu().numpy(),
               kappa=(1.0 / (3.0 * (mesh.mua + mesh.musp))).cpu().numpy(), K=sp.triu(K).tocsc(),
               M=sp.triu(M).tocsc())
    o = mesh.optode
    if o is not None:
        orec = {}
        for f in _OPTODE_FIELDS:
            v = getattr(o, f, None)
            if v is None:
                continue
            if hasattr(v, "cpu"):
                v = v.cpu().numpy()
            orec[f] = v
        rec["optode"] = orec
    return rec


def _to_matlab(rec: dict) -> dict:
    out = {}
    for k, v in rec.items():
        if isinstance(v, dict):
            out[k] = _to_matlab(v)
        elif k in _ONE_BASED:
            out[k] = np.asarray(v, dtype=np.float64) + 1
        elif k in _BARY:
            b = np.array(v, dtype=np.float64, copy=True)
            b[:, 0] += 1
            out[k] = b
        else:
            out[k] = v
    return out


def _from_matlab(rec: dict) -> dict:
    out = {}
    for k, v in rec.items():
        if isinstance(v, dict):
            out[k] = _from_matlab(v)
        elif k in _ONE_BASED:
            out[k] = np.asarray(v).astype(np.int64) - 1
        elif k in _BARY:
            b = np.array(v, dtype=np.float64, copy=True)
            b[:, 0] -= 1
            out[k] = b
        else:
            out[k] = v
    return out


def save_mat(path, rec: dict) -> None:
    """MATLAB v5 .mat with dMesh property names (and an `optode` struct), 1-based indices."""
    import scipy.io
    scipy.io.savemat(str(path), _to_matlab(rec), do_compression=True, oned_as="column")


def load_mat(path) -> dict:
    """Record from save_mat (or from MATLAB's save of the same field names), 0-based."""
    import scipy.io
    raw = scipy.io.loadmat(str(path), squeeze_me=True, struct_as_record=False)

    def conv(v):
        if hasattr(v, "_fieldnames"):
            return {f: conv(getattr(v, f)) for f in v._fieldnames}
        return v

    rec = {k: conv(v) for k, v in raw.items() if not k.startswith("__")}
    for k in ("node",):
        if k in rec:
            rec[k] = np.atleast_2d(rec[k])
    for k in ("elem", "face"):
        if k in rec:
            rec[k] = np.atleast_2d(rec[k])
    if "optode" in rec:
        for k in ("s_bary", "d_bary", "link", "s_positions", "d_positions", "s_dirs", "d_dirs"):
            if k in rec["optode"]:
                rec["optode"][k] = np.atleast_2d(rec["optode"][k])
    return _from_matlab(rec)


def save_npz(path, rec: dict) -> None:
    """The same record as .npz (flat keys, `optode.<field>` for the optode; sparse K, M as CSC parts)."""
    import scipy.sparse as sp
    flat = {}
    for k, v in _to_matlab(rec).items():
        if isinstance(v, dict):
            for f, x in v.items():
                flat[f"optode.{f}"] = np.asarray(x)
        elif sp.issparse(v):
            v = v.tocsc()
            flat[f"{k}.data"], flat[f"{k}.indices"], flat[f"{k}.indptr"] = v.data, v.indices, v.indptr
            flat[f"{k}.shape"] = np.asarray(v.shape)
        else:
            flat[k] = np.asarray(v)
    np.savez_compressed(str(path), **flat)


def load_npz(path) -> dict:
    import scipy.sparse as sp
    z = np.load(str(path), allow_pickle=False)
    rec, opt = {}, {}
    for k in z.files:
        if k.startswith("optode."):
            opt[k[7:]] = z[k]
        elif k.endswith(".data"):
            base = k[:-5]
            rec[base] = sp.csc_matrix((z[k], z[base + ".indices"], z[base + ".indptr"]),
                                      shape=tuple(z[base + ".shape"]))
        elif k.endswith((".indices", ".indptr", ".shape")):
            continue
        else:
            v = z[k]
            rec[k] = v.item() if v.ndim == 0 else v
    if opt:
        rec["optode"] = {k: (v.item() if v.ndim == 0 else v) for k, v in opt.items()}
    return _from_matlab(rec)


def dmesh_from_record(rec: dict):
    """DMesh (and its optode, as recorded: no re-snapping) from a record."""
    import torch
    from .dmesh import DMesh
    from .optode import DOptode
    mesh = DMesh(rec["node"], np.asarray(rec["elem"]), float(rec["nr"]),
                 np.stack([np.asarray(rec["mua"], float), np.asarray(rec["musp"], float)], axis=1))
    if "optode" in rec:
        o = DOptode.__new__(DOptode)
        for k, v in rec["optode"].items():
            setattr(o, k, v)
        o.link = np.asarray(o.link, dtype=np.int64).reshape(-1, 2)
        o.Nf = int(o.Nf)
        o.fAxis = np.atleast_1d(np.asarray(o.fAxis, dtype=np.float64))
        o.tAxis = np.atleast_1d(np.asarray(o.tAxis, dtype=np.float64))
        o.s_fpsf = torch.as_tensor(np.atleast_1d(np.asarray(o.s_fpsf, dtype=np.complex128)), device="cuda")
        mesh.optode = o
        mesh._solver = None
    return mesh
