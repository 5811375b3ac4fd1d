"""Float64 restatement of the Fourier-series transforms.

``td2fc`` (DOGPUP/td2fc.m:1-39), ``fc2td`` (DOGPUP/fc2td.m:1-39) and
``fc2tg`` (DOGPUP/fc2tg.m:1-40), with the time/frequency axis on the last
dimension (``dim=-1``) instead of a MATLAB ``dim`` argument.
"""
from __future__ import annotations

import numpy as np


def td2fc(fun_td, f, t):
    """c_k = dt/P * sum_t exp(-i f_k t) x(t), P = t(end), td2fc.m:26-32."""
    t = np.asarray(t, dtype=np.float64)
    f = np.asarray(f, dtype=np.float64)
    dt = t[1] - t[0]
    P = t[-1]
    T = np.exp(-1j * f[:, None] * t[None, :])          # [NF, NT]
    return dt * (np.asarray(fun_td) @ T.T) / P


def fc2td(fun_fc, f, t):
    """x(t) = 2 Re sum_k exp(i f_k t) c~_k with c~_0 = c_0/2, fc2td.m:24-31."""
    c = np.array(fun_fc, dtype=np.complex128, copy=True)
    c[..., 0] = c[..., 0] / 2
    T = np.exp(1j * np.asarray(f)[None, :] * np.asarray(t)[:, None])   # [NT, NF]
    return 2.0 * np.real(c @ T.T)


def fc2tg(fun_fc, gate_fc, f, nt):
    """y[g] = Nt * 2 Re sum_k conj(gate_fc[g,k]) c~_k, c~_0 = c_0/2, fc2tg.m:25-32."""
    c = np.array(fun_fc, dtype=np.complex128, copy=True)
    c[..., 0] = c[..., 0] / 2
    G = np.conj(np.asarray(gate_fc))                   # [NG, NF]
    return nt * 2.0 * np.real(c @ G.T)


def gaussian_tpsf(t, fwhm, delay_sd=6.0):
    """Source pulse of tutorials/tut_2_fluence_and_sensitivity.m:17-23."""
    sd = fwhm / (2 * np.sqrt(2 * np.log(2)))
    return np.exp(-((t - delay_sd * sd) ** 2) / (2 * sd ** 2))
