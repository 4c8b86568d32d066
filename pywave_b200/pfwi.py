"""``pfwi`` and ``fillpar`` with the reference's signatures (pywave/pfwi.py:5, :262).

Modes 1 (modelling), 2 (FWI) and 4 (passive modelling and least-squares
time-reversal source inversion through lstric; passive FWI with known
sources through pfwic) run on the GPU engine; mode 3 (RTM) does nothing,
as in the reference (pfwi.py:114-119).  As in the reference only ``par`` is
read:
the keyword arguments after ``mode`` are accepted and ignored
(pfwi.py:29-61).
"""
from __future__ import annotations

import numpy as np

from .pfwicfun import forward_modeling_ac, fwic, lstric, pfwic  # noqa: F401

_KEYS = ["nz", "nx", "dz", "dx", "oz", "ox", "nt", "dt", "ot", "inv", "ns", "ds", "os", "sz",
         "nb", "coef", "f0", "acqui_type", "interval", "niter"]


def pararray(par):
    """The 20-float parameter array pfwi.py builds (pfwi.py:40-61)."""
    return np.array([par[k] for k in _KEYS], dtype=np.float32)


def pfwi(vel, q, wav, src, data=None, mode=1, media=1, inv=0, verb=1, nb=60, coef=0.005, acq=1,
         ss=[0, 0.2, 1], f0=10, waterz=-30, niter=30, conv_e=0.01, par=None):
    """Acoustic modelling (mode 1), FWI (mode 2) or passive modelling /
    source inversion (mode 4).  Returns ``(data, vinv, grad, src, mwt)``
    like pywave.pfwi."""
    par = fillpar(par)
    if mode == 1:
        v = np.asarray(vel).flatten(order="F").astype(np.float32)
        qq = np.asarray(q).flatten(order="F").astype(np.float32)
        w = np.asarray(wav).flatten(order="F").astype(np.float32)
        d = forward_modeling_ac(v, qq, w, pararray(par))
        d = d.reshape(par["nt"], par["nx"], par["ns"], order="F")
        return d, [], [], [], []
    if mode == 2:
        v = np.asarray(vel).flatten(order="F").astype(np.float32)
        qq = np.asarray(q).flatten(order="F").astype(np.float32)
        w = np.asarray(wav).flatten(order="F").astype(np.float32)
        d = np.asarray(data).flatten(order="F").astype(np.float32)
        vinv = fwic(v, qq, w, d, pararray(par))
        vinv = vinv.reshape(par["nz"], par["nx"], par["niter"], order="F")
        return data, vinv, None, None, None
    if mode == 3:
        return data, None, None, src, None
    if mode == 4:
        return _mode4(vel, q, wav, src, data, par)
    print("Wrong mode")
    return 0


def _mode4(vel, q, wav, src, data, par):
    """pfwi.py:121-251: passive modelling (inv False) or source inversion
    (inv True, onlysrc True) through lstric; passive FWI (inv True, onlysrc
    False) through pfwic."""
    v = np.asarray(vel).flatten(order="F").astype(np.float32)
    qq = np.asarray(q).flatten(order="F").astype(np.float32)
    w = np.asarray(wav).flatten(order="F").astype(np.float32)
    if par["inv"] and not par["onlysrc"]:
        # pfwi.py:167-210: pfwic on the data followed by the sources; the
        # wrapper returns the flattened data in the data slot
        par["inv"] = 1
        d = np.asarray(data).flatten(order="F").astype(np.float32)
        s = np.asarray(src).flatten(order="F").astype(np.float32)
        vinv = pfwic(v, qq, w, np.concatenate([d, s]), pararray(par))
        vinv = vinv.reshape(par["nz"], par["nx"], par["niter"], order="F")
        if par["onlyvel"]:
            return d, vinv, None, None, None
        # the reference's wrapper leaves grad and mwt unbound here (pfwi.py:205-210)
        return d, vinv, None, src, None
    if par["inv"]:
        par["inv"] = 1
        d = np.asarray(data).flatten(order="F").astype(np.float32)
        s = lstric(v, qq, w, d, pararray(par))
        s = s.reshape(par["nz"], par["nx"], par["nt"], par["ns"], order="F")
        return [], None, None, s, []
    s = np.asarray(src).flatten(order="F").astype(np.float32)
    d = lstric(v, qq, w, s, pararray(par))
    d = d.reshape(par["nt"], par["nx"], par["ns"], order="F")
    return d, [], [], [], []


def fillpar(par):
    """Fill blank keywords with the reference's defaults (pywave/pfwi.py:262-301)."""
    kw = {
        "f0": 10, "nb": 100, "coef": 0.003, "acqui_type": 1, "interval": 1, "ns": 1, "ds": 0.2,
        "os": 0.0, "sz": 5, "nx": 100, "nz": 100, "nr": par["nx"], "dr": par["dx"],
        "r0": par["ox"], "fhi": 0.5 / par["dt"], "flo": 0, "onlysrc": True, "onlyvel": False,
        "inv": False, "niter": 10,
    }
    kw.update(par)
    return kw
