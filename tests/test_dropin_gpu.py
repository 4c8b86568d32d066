"""The drop-in claim, tested: the reference's own, unmodified Python wrappers
(pywave/afd2d.py:73, afd3d.py:77, pfwi.py:70,111) call their extension
modules `afdcfun` / `pfwicfun` with positional arguments that
tests/golden/make_golden.py recorded while running them against the
compiled reference.  Each recorded call is replayed here through
pywave_b200.afdcfun / pywave_b200.pfwicfun (the modules a maintainer aliases
into sys.modules) and must return what the reference's
module returned: bit-identical where no wavelet table is involved, within
the closed-form Ricker table's 1e-5 (rel-L2) for afd forward modelling, and
within the FP32/FP64 inner-product difference for fwic.  GPU only."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _calls(golden):
    z = golden("dropin_calls")
    out = []
    for i in range(int(z["ncalls"])):
        args = []
        for j in range(int(z[f"c{i}_nargs"])):
            a = z[f"c{i}_a{j}"]
            args.append(a.item() if a.ndim == 0 else a)
        out.append(dict(name=str(z[f"c{i}_name"]), args=args, digest=str(z[f"c{i}_out_digest"]),
                        shape=tuple(z[f"c{i}_out_shape"]), dec=z[f"c{i}_out_dec"]))
    return out


def _digest(a):
    import os
    import sys
    from conftest import ROOT
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import models
    return models.digest(a)


def _replay(c):
    from pywave_b200 import afdcfun, pfwicfun
    mod = afdcfun if c["name"] in ("afd2dc", "afd3dc") else pfwicfun
    out = np.asarray(getattr(mod, c["name"])(*c["args"]))
    assert out.shape == c["shape"], (c["name"], out.shape, c["shape"])
    return out


def test_recorded_calls_cover_every_module_function(golden):
    names = [c["name"] for c in _calls(golden)]
    assert names == ["afd2dc", "afd2dc", "afd3dc", "afd3dc", "forward_modeling_ac", "fwic"]


@pytest.mark.parametrize("k", [1, 3, 4])
def test_replay_bit_exact(golden, cuda_lib, k):
    """afd2dc / afd3dc time reversal and forward_modeling_ac: identical."""
    c = _calls(golden)[k]
    out = _replay(c)
    assert np.array_equal(out.reshape(-1)[::97], c["dec"])
    assert _digest(out) == c["digest"]


@pytest.mark.parametrize("k,fixture", [(0, "afd2d_fwd"), (2, "afd3d_fwd")])
def test_replay_afd_forward(golden, cuda_lib, k, fixture):
    """afd forward modelling with the Ricker table built from f, t, A: the
    reference's flat output [traces, snapshots] to 1e-5."""
    c = _calls(golden)[k]
    g = golden(fixture)
    ref = np.concatenate([g["traces"].flatten(order="F"), g["snaps"].flatten(order="F")])
    assert _digest(ref) == c["digest"]  # the golden is this call's output
    out = _replay(c)
    assert rel_l2(out, ref) < 1e-5


def test_replay_fwic(golden, cuda_lib):
    """fwic, two L-BFGS iterations: each model within 1e-3 (rel-L2) of the
    reference's (FP64 inner products here, float in the reference)."""
    c = _calls(golden)[5]
    g = golden("pfwi")
    out = _replay(c)
    nz, nx = g["vtrue"].shape
    vinv = out.reshape(nz, nx, -1, order="F")
    ref = g["vinv"]
    for it in range(ref.shape[2]):
        if np.any(ref[:, :, it]):
            assert rel_l2(vinv[:, :, it], ref[:, :, it]) < 1e-3
