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
