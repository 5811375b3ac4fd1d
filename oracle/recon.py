"""Float64 restatement of the weighted LM loop, DOGPUP/reconstruction/wghtd_LM_recon.m:25-168,
for the unweighted case without target spots (w = 1, :77-81).

Test infrastructure (never imported by the package).  The model is a callback, so a
test can script the data and Jacobian each iteration sees -- e.g. to make the error
rise twice in a row and exercise the step-back branch (:108-116) twice, where the
cached Jacobian is reused exactly as it was cached (normalised by the G of its own
iteration) and only the update is rescaled by the new G.
"""
from __future__ import annotations

import numpy as np

from .jacobian import tik_inv


def lm_loop(model, mua0, m2g, g2m, dm, incl, lam1, max_iter=10):
    """model(count) -> (data_c [NMeas] in x(:) order, J [NMeas, NV]) for the model at the
    current mua; dm = log(measured data)[incl] (:29-30); m2g [NV, NN], g2m [NN, NV] (in-mesh
    voxels only); lam1 = lam(1) as passed to wghtd_LM_recon.  Returns a dict with err,
    err_perc, err_del, lam, mua (after every applied update), iterations and exit."""
    k = 10 ** 0.25                                                  # :40
    lam = lam1 * k                                                  # :41
    count = 0
    mua = np.array(mua0, dtype=np.float64, copy=True)
    h = dict(err=[], err_perc=[], err_del=[], lam=[], mua=[])
    d_mu = y_prev = J_prev = None
    while True:
        data_c, J = model(count)                                    # :58
        data_c = np.log(np.asarray(data_c))[incl]                   # :62-63
        J = np.asarray(J)[incl]                                     # :64-65
        y = dm - data_c                                             # :67
        h["err"].append(float(np.linalg.norm(y)))                   # :85
        h["err_perc"].append(h["err"][-1] / float(np.linalg.norm(dm)) * 100)   # :86
        if count > 0:
            h["err_del"].append(h["err_perc"][-1] - h["err_perc"][-2])         # :89
        if count > 1 and h["err_del"][-1] < 0 and (abs(h["err_del"][-1]) < 0.12 or h["err_perc"][-1] < 1.5):
            h["exit"] = "converged"                                 # :94-96
            break
        count += 1
        if count == 1 or h["err_del"][-1] < 0:                      # :103-107
            G = m2g @ mua
            J = J * G[None, :]
            lam = lam / k
        else:                                                       # :108-116
            G = m2g @ (mua - d_mu)
            y = y_prev
            J = J_prev
            lam = lam * k
        if lam < h["err"][-1]:                                      # :118-120
            lam = h["err"][-1]
        h["lam"].append(lam)
        update = tik_inv(J, lam, y)                                 # :128
        x = G * update                                              # :133
        d_mu = g2m @ x                                              # :134
        if np.isnan(d_mu).any():                                    # :136-141
            h["exit"] = "nan_update"
            break
        new_mu = mua + d_mu                                         # :143
        if (new_mu < 0).any():                                      # :147-152
            h["exit"] = "negative_mua"
            break
        mua = new_mu                                                # :155
        h["mua"].append(mua.copy())
        if count > max_iter - 1:                                    # :159-162
            h["exit"] = "max_iter"
            break
        y_prev = y                                                  # :165-166
        J_prev = J
    h["iterations"] = count
    return h
