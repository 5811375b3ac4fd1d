"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Each builder returns a dict with the mesh (node, elem), nodal optical
properties, refractive index, optode positions / links and the time axis.
No dataset is involved: meshes come from ``meshgen`` (lattice clipped to the
shape, 6 tets per cube, interior nodes jittered) and every random quantity is
drawn from ``numpy.random.default_rng(seed)``.
"""
from __future__ import annotations

import numpy as np

from . import meshgen


def gaussian_pulse(t, fwhm=250e-12, delay_sd=6.0):
    """Source pulse shape of tutorials/tut_2_fluence_and_sensitivity.m:17-23."""
    sd = fwhm / (2 * np.sqrt(2 * np.log(2)))
    return np.exp(-((t - delay_sd * sd) ** 2) / (2 * sd ** 2))


def time_axis(period_s=10e-9, dt=50e-12):
    """t = 0:dt:T; the Fourier period is t(end) (dOptode.m:57), so df = 1/T."""
    n = int(round(period_s / dt))
    return np.arange(n + 1) * dt


def ring(n, centre, semi_axes_xy, z, phase=0.0):
    return meshgen.ring_positions(n, None, z, centre_xy=centre[:2], phase=phase, axes_xy=semi_axes_xy)


def all_pairs(ns, nd):
    s, d = np.meshgrid(np.arange(ns), np.arange(nd), indexing="ij")
    return np.stack([s.ravel(), d.ravel()], axis=1)


def cylinder_fwd(seed=1, h=1.5, ns=16, nd=16, nf=32, order="morton"):
    """Plain FP64 forward, small: cylinder r=30 h=60 mm at 1.5 mm, 16+16 optodes on the mid ring, 32 harmonics."""
    m = meshgen.cylinder_mesh(30.0, 60.0, h, jitter=0.2, seed=seed, order=order)
    c = np.array([0.0, 0.0, 30.0])
    src = ring(ns, c, (30.0, 30.0), 30.0)
    det = ring(nd, c, (30.0, 30.0), 30.0, phase=np.pi / nd)
    return dict(name=f"cylinder r30 h60 @{h}mm", mesh=m, mua=np.full(m.nn, 0.01), musp=np.full(m.nn, 1.0),
                nr=1.4, src=src, det=det, link=all_pairs(ns, nd), t=time_axis(10e-9), nf=nf)


def ellipsoid_fwd(seed=1, axes=(90.0, 75.0, 70.0), h=1.2, ns=64, nd=64, nf=128, grf_corr_mm=8.0, order="morton"):
    """Batched mixed forward: ellipsoid head phantom, mua = 0.01 (1 + 0.2 GRF), 64 sources x 128 harmonics."""
    m = meshgen.ellipsoid_mesh(axes, h, jitter=0.2, seed=seed, order=order)
    grf = meshgen.smooth_random_field(m, grf_corr_mm, seed + 100)
    mua = 0.01 * (1.0 + 0.2 * grf)
    a = np.asarray(axes) / 2
    src, det = [], []
    rings = 4
    per = ns // rings
    for q, zf in enumerate(np.linspace(-0.45, 0.45, rings)):
        z = zf * a[2]
        scale = np.sqrt(max(1 - zf ** 2, 0.05))
        src.append(ring(per, np.zeros(3), (a[0] * scale, a[1] * scale), z))
        det.append(ring(nd // rings, np.zeros(3), (a[0] * scale, a[1] * scale), z, phase=np.pi / per))
    src, det = np.concatenate(src), np.concatenate(det)
    return dict(name=f"ellipsoid {axes[0]:g}x{axes[1]:g}x{axes[2]:g} @{h}mm", mesh=m, mua=mua,
                musp=np.full(m.nn, 1.0), nr=1.4, src=src, det=det, link=all_pairs(len(src), len(det)),
                t=time_axis(10e-9), nf=nf)


def small_fwd(seed=1, ns=8, nd=8, nf=8, order="morton"):
    """A few-thousand-node cylinder for smoke tests."""
    m = meshgen.cylinder_mesh(10.0, 16.0, 1.5, jitter=0.2, seed=seed, order=order)
    c = np.array([0.0, 0.0, 8.0])
    src = ring(ns, c, (10.0, 10.0), 8.0)
    det = ring(nd, c, (10.0, 10.0), 8.0, phase=np.pi / nd)
    return dict(name="cylinder r10 h16 @1.5mm", mesh=m, mua=np.full(m.nn, 0.01), musp=np.full(m.nn, 1.0), nr=1.4,
                src=src, det=det, link=all_pairs(ns, nd), t=time_axis(10e-9), nf=nf)


def build_dmesh(w):
    """DMesh + DOptode for a workload dict (device assembly, snapped optodes)."""
    from .dmesh import DMesh
    from .optode import DOptode
    m = w["mesh"]
    mesh = DMesh(m.node, m.elem, w["nr"], np.stack([w["mua"], w["musp"]], axis=1))
    t = w["t"]
    opt = DOptode(w["src"], w["det"], w["link"], 1e3, gaussian_pulse(t), t, w["nf"])
    mesh.add_optode(opt)
    return mesh
