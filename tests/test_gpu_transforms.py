"""Device Fourier-series transforms against the oracle (oracle/transforms.py).

td2fc (DOGPUP/td2fc.m:26-32: c_k = dt/t(end) * sum_t exp(-i f_k t) x(t)),
fc2td (DOGPUP/fc2td.m:24-31: c_0 halved, x(t) = 2 Re sum_k exp(i f_k t) c_k)
and fc2tg (DOGPUP/fc2tg.m:25-32: c_0 halved, y_g = Nt * 2 Re sum_k conj(gate_gk) c_k)
on odd sizes, with the reference's conventions: the Fourier period is t(end)
(not Nt * dt), the rectangle rule runs over every sample including both ends,
and the first coefficient is halved whatever its frequency.  Also the source
spectrum of the optode constructor (dOptode.m:66-73: the TPSF scaled to the
average power, then td2fc).  Tolerance: 1e-12 relative to the output's
largest magnitude (FP64 throughout; the device forms the angles f_k * t as the
oracle does and differs only in summation order).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


def _axes(nt, nf, dt=50e-12):
    t = np.arange(nt) * dt                      # t = 0:dt:T, T = t(end) (dOptode.m:55-59)
    f = np.arange(nf) * 2 * np.pi / t[-1]
    return t, f


@pytest.mark.parametrize("nr,nt,nf", [(1, 2, 1), (7, 201, 33), (13, 97, 48), (3, 1001, 129)])
def test_td2fc_against_oracle(nr, nt, nf):
    import torch
    from dogpup_b200 import api
    from oracle.transforms import td2fc
    rng = np.random.default_rng(nr * 1000 + nt)
    t, f = _axes(nt, nf)
    x = rng.standard_normal((nr, nt)) + 0.5
    c = api.td2fc(torch.as_tensor(x, device="cuda"), torch.as_tensor(f), torch.as_tensor(t)).cpu().numpy()
    c0 = td2fc(x, f, t)
    assert c.shape == (nr, nf)
    assert _rel(c, c0) < TOL


@pytest.mark.parametrize("nr,nf,nt", [(1, 1, 2), (5, 33, 201), (11, 64, 77), (2, 129, 1001)])
def test_fc2td_against_oracle(nr, nf, nt):
    import torch
    from dogpup_b200 import api
    from oracle.transforms import fc2td
    rng = np.random.default_rng(nr * 31 + nf)
    t, f = _axes(nt, nf)
    c = rng.standard_normal((nr, nf)) + 1j * rng.standard_normal((nr, nf))
    x = api.fc2td(torch.as_tensor(c, device="cuda"), torch.as_tensor(f), torch.as_tensor(t)).cpu().numpy()
    x0 = fc2td(c, f, t)
    assert x.shape == (nr, nt)
    assert _rel(x, x0) < TOL


@pytest.mark.parametrize("nr,nf,ng", [(1, 1, 1), (9, 33, 10), (4, 64, 20), (17, 31, 3)])
def test_fc2tg_against_oracle(nr, nf, ng):
    import torch
    from dogpup_b200 import api
    from oracle.transforms import fc2tg, td2fc
    rng = np.random.default_rng(nr + 7 * nf + ng)
    nt = 201
    t, f = _axes(nt, nf)
    sd = 500e-12 / (2 * np.sqrt(2 * np.log(2)))
    gates = np.stack([np.exp(-(t - (0.5e-9 + 0.5e-9 * g)) ** 2 / (2 * sd ** 2)) for g in range(ng)])
    gfc = td2fc(gates, f, t)                    # [NG, NF] (the device td2fc is pinned above)
    c = rng.standard_normal((nr, nf)) + 1j * rng.standard_normal((nr, nf))
    y = api.fc2tg(torch.as_tensor(c, device="cuda"), torch.as_tensor(gfc, device="cuda"), nt).cpu().numpy()
    y0 = fc2tg(c, gfc, f, nt)
    assert y.shape == (nr, ng)
    assert _rel(y, y0) < TOL


def test_first_coefficient_halved_at_any_frequency():
    """fc2td / fc2tg halve the first coefficient even when the frequency axis does not start
    at 0 (fc2td.m:24, fc2tg.m:25 index the first entry, not the DC term)."""
    import torch
    from dogpup_b200 import api
    from oracle.transforms import fc2td, fc2tg
    t = np.arange(101) * 100e-12
    f = (np.arange(16) + 3) * 2 * np.pi / t[-1]
    c = np.zeros((1, 16), complex)
    c[0, 0] = 2.0
    x = api.fc2td(torch.as_tensor(c, device="cuda"), torch.as_tensor(f), torch.as_tensor(t)).cpu().numpy()
    assert _rel(x, fc2td(c, f, t)) < TOL
    assert np.allclose(x[0], 2 * np.cos(f[0] * t))          # 2 Re(c_0/2 e^{i f_0 t})
    g = np.ones((2, 16), complex)
    y = api.fc2tg(torch.as_tensor(c, device="cuda"), torch.as_tensor(g, device="cuda"), 101).cpu().numpy()
    assert _rel(y, fc2tg(c, g, f, 101)) < TOL
    assert np.allclose(y, 101 * 2 * 1.0)


def test_band_limited_round_trip():
    """fc2td(td2fc(x)) on a signal made of the harmonics themselves, through the device on
    both legs, equals the oracle's round trip (which is not the identity under the
    T = t(end) rectangle rule); and td2fc of fc2td's output returns the coefficients the
    oracle's second leg returns."""
    import torch
    from dogpup_b200 import api
    from oracle.transforms import fc2td, td2fc
    nt, nf = 401, 24
    t, f = _axes(nt, nf)
    rng = np.random.default_rng(4)
    a = rng.standard_normal(nf) + 1j * rng.standard_normal(nf)
    x = 2 * np.real(np.exp(1j * f[None, :] * t[:, None]) @ a)[None, :]
    T, F = torch.as_tensor(t), torch.as_tensor(f)
    c_d = api.td2fc(torch.as_tensor(x, device="cuda"), F, T)
    x_d = api.fc2td(c_d, F, T).cpu().numpy()
    x_o = fc2td(td2fc(x, f, t), f, t)
    assert _rel(x_d, x_o) < TOL
    c2 = api.td2fc(torch.as_tensor(x_d, device="cuda"), F, T).cpu().numpy()
    assert _rel(c2, td2fc(x_o, f, t)) < TOL


def test_source_spectrum_of_the_optode_constructor():
    """DOptode.s_fpsf = td2fc(tpsf * avgPow / mean(tpsf)) (dOptode.m:66-73), from the device
    td2fc, against the oracle's td2fc of the same scaled TPSF; fAxis and df as the
    reference sets them (:57-60)."""
    from dogpup_b200.optode import DOptode
    from dogpup_b200.workloads import gaussian_pulse, time_axis
    from oracle.transforms import td2fc
    t = time_axis(10e-9)
    tpsf = gaussian_pulse(t)
    for nf, avg in ((32, 1e3), (7, 2.5)):
        o = DOptode(np.zeros((1, 3)), np.zeros((1, 3)), [[0, 0]], avg, tpsf, t, nf)
        fAxis = np.arange(nf) * (2 * np.pi / t[-1])                  # (0:Nf-1) .* w0, w0 = 2 pi / T
        assert np.allclose(o.fAxis, fAxis, rtol=1e-15, atol=0) and abs(o.df - (fAxis[1] - fAxis[0])) <= 1e-15 * o.df
        scaled = tpsf * (avg / tpsf.mean())
        assert np.abs(o.s_tpsf - scaled).max() <= 1e-15 * np.abs(scaled).max()
        ref = td2fc(scaled[None, :], o.fAxis, t)[0]
        assert _rel(o.s_fpsf.cpu().numpy(), ref) < TOL
        assert abs(ref[0].real - avg * t[1] * len(t) / t[-1]) < 1e-9 * avg   # c_0 = dt/T sum = avgPow * Nt dt / T
