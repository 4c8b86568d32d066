"""Visco-acoustic pfwi (forward_modeling, gradient_v) on the GPU through the
C ABI, against the reference's own outputs (tests/golden/visco.npz, produced
through oracle/ref_driver.c since the reference's Python glue cannot reach
this path, pfwi.c:864)."""
import sys

import numpy as np
import pytest

from conftest import GOLDEN, rel_l2

sys.path.insert(0, GOLDEN)
import models as M  # noqa: E402

pytestmark = pytest.mark.gpu


def test_visco_forward_bit_exact(golden, cuda_lib):
    """Every shot's traces identical to the reference's forward_modeling."""
    from pywave_b200 import fwi
    g = golden("visco")
    vt, _, q, wav = M.visco_case()
    d = fwi.forward_visco(vt, q, wav, M.VISCO)
    assert d.shape == g["data"].shape
    print(f"visco forward: rel-L2 vs reference {rel_l2(d, g['data']):.2e}")
    assert np.array_equal(d.view(np.uint32), g["data"].view(np.uint32))


def test_visco_gradient_bit_exact(golden, oracle, cuda_lib):
    """gradient_v after the first-call scaling and rect 1 / 3 smoothing
    identical to the reference's; misfit to the reference's float sum to
    1e-4 (FP64 here)."""
    from pywave_b200 import fwi
    g = golden("visco")
    _, vs, q, wav = M.visco_case()
    raw, J = fwi.gradient_visco(vs, q, wav, g["data"], M.VISCO)
    for rect in (1, 3):
        pp, _ = fwi.postprocess(raw, rect=rect)
        assert np.array_equal(pp, g["grad_rect%d" % rect]), rect
    assert abs(J - float(g["fcost"])) <= 1e-4 * abs(J)


def test_visco_differs_from_acoustic(golden, cuda_lib):
    """The memory variable does something: the visco traces differ from the
    acoustic ones by the attenuation (a few percent here), and a very large
    q reproduces the acoustic traces closely."""
    from pywave_b200 import fwi
    vt, _, q, wav = M.visco_case()
    dv = fwi.forward_visco(vt, q, wav, M.VISCO)
    import pywave_b200 as pw
    da = pw.pfwi(vt, np.ones_like(q), wav, None, mode=1, par=dict(M.VISCO))[0]
    dq = fwi.forward_visco(vt, np.full_like(q, 1e6), wav, M.VISCO)
    print(f"visco vs acoustic {rel_l2(dv, da):.3e}; q=1e6 vs acoustic {rel_l2(dq, da):.3e}")
    assert rel_l2(dv, da) > 1e-2
    assert rel_l2(dq, da) < 1e-3
