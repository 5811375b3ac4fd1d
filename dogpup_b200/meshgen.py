"""Seeded synthetic tetrahedral meshes and optical-property fields.

These generators produce the inputs of the forward/sensitivity path: a
regular cube lattice clipped to a shape, each cube split into 6 linear
tetrahedra around its main diagonal (the conforming Kuhn split, the same
lattice family as iso2mesh ``meshgrid6``), and interior nodes jittered by a
seeded uniform offset.  Nodes are numbered either in lattice order (x
fastest, z slowest: FEM matrix bandwidth of about one lattice plane) or in
Morton (Z-curve) order of their lattice coordinates, which puts each run of
64 consecutive nodes in a compact 4x4x4 region, so a block of SpMM rows
gathers mostly from nodes that other rows of the same block also read (the
locality ``sortmesh`` aims at in the reference's meshing stack,
meshing/iso2mesh/sortmesh.m).

The reference builds its meshes with iso2mesh (``meshabox`` + ``sortmesh``,
tutorials/tut_1_meshing.m:5-7); that meshing stack is third-party and out of
scope, so the path is exercised on these structured meshes instead.
"""
from __future__ import annotations

import itertools
from dataclasses import dataclass

import numpy as np

# the 6 Kuhn tetrahedra of the unit cube: walk (0,0,0) -> (1,1,1) one axis at a time
_KUHN = []
for _perm in itertools.permutations(range(3)):
    _p = [0, 0, 0]
    _verts = [tuple(_p)]
    for _ax in _perm:
        _p[_ax] = 1
        _verts.append(tuple(_p))
    _KUHN.append(_verts)
_KUHN = np.array(_KUHN, dtype=np.int64)  # [6, 4, 3] corner offsets


@dataclass
class TetMesh:
    node: np.ndarray      # [NN, 3] float64, mm
    elem: np.ndarray      # [NE, 4] int32, 0-based node ids
    bnd: np.ndarray       # [NN] bool, node lies on the outer surface
    lattice: np.ndarray   # [NN, 3] int64 lattice coordinates of each node
    h: float              # lattice spacing (mm)
    origin: np.ndarray    # [3] lattice origin (mm)

    @property
    def nn(self) -> int:
        return int(self.node.shape[0])

    @property
    def ne(self) -> int:
        return int(self.elem.shape[0])


def boundary_nodes(elem: np.ndarray, nn: int) -> np.ndarray:
    """Nodes on faces that belong to exactly one tetrahedron."""
    faces = np.concatenate([elem[:, [0, 1, 2]], elem[:, [0, 1, 3]],
                            elem[:, [0, 2, 3]], elem[:, [1, 2, 3]]])
    faces = np.sort(faces.astype(np.int64), axis=1)
    key = (faces[:, 0] << 42) | (faces[:, 1] << 21) | faces[:, 2]
    uniq, counts = np.unique(key, return_counts=True)
    once = uniq[counts == 1]
    bnd = np.zeros(nn, dtype=bool)
    mask = (1 << 21) - 1
    bnd[(once >> 42) & mask] = True
    bnd[(once >> 21) & mask] = True
    bnd[once & mask] = True
    return bnd


def _spread_bits(v: np.ndarray) -> np.ndarray:
    """Bits 0..20 of v moved to bits 0, 3, 6, ... (3-D Morton interleave)."""
    v = v.astype(np.uint64) & np.uint64(0x1FFFFF)
    for shift, mask in ((32, 0x1F00000000FFFF), (16, 0x1F0000FF0000FF), (8, 0x100F00F00F00F00F),
                        (4, 0x10C30C30C30C30C3), (2, 0x1249249249249249)):
        v = (v | (v << np.uint64(shift))) & np.uint64(mask)
    return v


def morton_order(lat: np.ndarray) -> np.ndarray:
    """Permutation sorting lattice coordinates [N, 3] (each < 2^21) along the Z-curve."""
    key = _spread_bits(lat[:, 0]) | (_spread_bits(lat[:, 1]) << np.uint64(1)) | (_spread_bits(lat[:, 2]) << np.uint64(2))
    return np.argsort(key, kind="stable")


def lattice_mesh(inside, lo, hi, h, jitter=0.0, seed=0, order="morton") -> TetMesh:
    """Cube lattice of spacing ``h`` over the box [lo, hi], keeping cubes whose
    centre satisfies ``inside(xyz) -> bool``; 6 tets per kept cube.

    Interior nodes are moved by an independent uniform offset in
    [-jitter, jitter] per coordinate drawn from ``numpy.random.default_rng(seed)``
    in lattice order, so both node orders ("lattice", "morton") give the same
    geometry.
    """
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    n = np.maximum(np.ceil((hi - lo) / h).astype(np.int64), 1)  # cubes per axis
    nxn, nyn, nzn = n + 1                                        # nodes per axis
    ci, cj, ck = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    cubes = np.stack([ci.ravel(), cj.ravel(), ck.ravel()], axis=1)
    centres = lo + (cubes + 0.5) * h
    cubes = cubes[inside(centres)]
    if cubes.shape[0] == 0:
        raise ValueError("shape contains no lattice cube")
    # corners of every tet of every kept cube, as lattice coordinates
    corners = cubes[:, None, None, :] + _KUHN[None, :, :, :]          # [C, 6, 4, 3]
    lin = corners[..., 0] + nxn * (corners[..., 1] + nyn * corners[..., 2])
    lin = lin.reshape(-1, 4)
    used, inv = np.unique(lin, return_inverse=True)                    # lattice order
    elem = inv.reshape(-1, 4).astype(np.int64)
    lat = np.stack([used % nxn, (used // nxn) % nyn, used // (nxn * nyn)], axis=1)
    node = lo + lat * h
    # positive orientation for every tet
    a = node[elem[:, 1]] - node[elem[:, 0]]
    b = node[elem[:, 2]] - node[elem[:, 0]]
    c = node[elem[:, 3]] - node[elem[:, 0]]
    neg = np.einsum("ij,ij->i", np.cross(a, b), c) < 0
    elem[neg] = elem[neg][:, [0, 2, 1, 3]]
    bnd = boundary_nodes(elem, node.shape[0])
    if jitter > 0:
        rng = np.random.default_rng(seed)
        d = rng.uniform(-jitter, jitter, size=node.shape)
        d[bnd] = 0.0
        node = node + d
    if order == "morton":
        perm = morton_order(lat)
        new_id = np.empty_like(perm)
        new_id[perm] = np.arange(perm.shape[0])
        node, bnd, lat, elem = node[perm], bnd[perm], lat[perm], new_id[elem]
    elif order != "lattice":
        raise ValueError("order must be 'lattice' or 'morton'")
    return TetMesh(node=node, elem=elem.astype(np.int32), bnd=bnd, lattice=lat, h=float(h), origin=lo)


def cylinder_mesh(radius, height, h, jitter=0.0, seed=0, centre=(0.0, 0.0, 0.0), order="morton") -> TetMesh:
    """Cylinder with its axis along z, base at ``centre[2]``."""
    cx, cy, cz = centre

    def inside(p):
        return (p[:, 0] - cx) ** 2 + (p[:, 1] - cy) ** 2 <= radius ** 2

    lo = (cx - radius, cy - radius, cz)
    hi = (cx + radius, cy + radius, cz + height)
    return lattice_mesh(inside, lo, hi, h, jitter, seed, order)


def ellipsoid_mesh(axes, h, jitter=0.0, seed=0, centre=(0.0, 0.0, 0.0), order="morton") -> TetMesh:
    """Ellipsoid with full axis lengths ``axes`` (mm) along x, y, z."""
    a = np.asarray(axes, dtype=np.float64) / 2.0
    c = np.asarray(centre, dtype=np.float64)

    def inside(p):
        return (((p - c) / a) ** 2).sum(axis=1) <= 1.0

    return lattice_mesh(inside, c - a, c + a, h, jitter, seed, order)


def box_mesh(size, h, jitter=0.0, seed=0, order="morton") -> TetMesh:
    return lattice_mesh(lambda p: np.ones(p.shape[0], dtype=bool), (0, 0, 0), size, h, jitter, seed, order)


def smooth_random_field(mesh: TetMesh, corr_mm: float, seed: int) -> np.ndarray:
    """Zero-mean, unit-variance Gaussian random field sampled at the nodes.

    White noise on the node lattice is smoothed with a Gaussian kernel of
    standard deviation ``corr_mm`` (periodic FFT convolution on a padded box)
    and normalised to unit standard deviation over the nodes.
    """
    lat = mesh.lattice - mesh.lattice.min(axis=0)
    pad = int(np.ceil(3 * corr_mm / mesh.h))
    shape = tuple(int(v) for v in (lat.max(axis=0) + 1 + 2 * pad))
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal(shape)
    k = [np.fft.fftfreq(s) for s in shape]
    kx, ky, kz = np.meshgrid(*k, indexing="ij")
    sig = corr_mm / mesh.h
    kern = np.exp(-2.0 * (np.pi * sig) ** 2 * (kx ** 2 + ky ** 2 + kz ** 2))
    field = np.real(np.fft.ifftn(np.fft.fftn(noise) * kern))
    vals = field[lat[:, 0] + pad, lat[:, 1] + pad, lat[:, 2] + pad]
    vals = vals - vals.mean()
    sd = vals.std()
    return vals / sd if sd > 0 else vals


def ring_positions(n, radius_xy, z, centre_xy=(0.0, 0.0), phase=0.0, axes_xy=None):
    """``n`` points equally spaced in angle on a horizontal ring (circle or ellipse)."""
    th = phase + 2 * np.pi * np.arange(n) / n
    if axes_xy is None:
        ax = ay = radius_xy
    else:
        ax, ay = axes_xy
    x = centre_xy[0] + ax * np.cos(th)
    y = centre_xy[1] + ay * np.sin(th)
    return np.stack([x, y, np.full(n, float(z))], axis=1)
