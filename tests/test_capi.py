"""The C-ABI library builds, loads without a GPU and exports every entry point
include/pywave_b200.h declares.  No compute calls here (CPU only)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared():
    src = open(os.path.join(ROOT, "include", "pywave_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pw_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_header_symbols():
    from pywave_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    names = declared()
    assert "pw_afd" in names and "pw_pfwi_gradient" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from pywave_b200 import _lib
    assert set(declared()) <= set(_lib.exported_symbols())


def test_version_and_error_strings():
    from pywave_b200 import _lib
    L = _lib.lib()
    assert b"sm_100a" in L.pw_version()
    assert isinstance(L.pw_last_error(), bytes)


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    from pywave_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.lib()


def test_residual_weights_host_entry_matches_reference(golden):
    """pw_residual_weights (host code, no device) against the reference's
    residual_weighting in both branches, and the default whole-record window
    fwic uses."""
    import sys
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import models as M
    from pywave_b200 import fwi
    g = golden("butter")
    nt, nr, wtn1, wtn2, woffn1, woffn2 = M.WEIGHT_CASE
    for oreo in (0, 1):
        w = fwi.residual_weights(nt, nr, wtn1, wtn2, woffn1, woffn2, oreo=bool(oreo))
        assert np.array_equal(w, g["w_oreo%d" % oreo]), oreo
    from oracle import oracle as O
    assert np.array_equal(fwi.residual_weights(80, 30), O.residual_weights(80, 30))
