"""The C-ABI library: builds, loads without a GPU, exports every entry
point include/rism3d_b200.h declares, and fails loudly (no CPU fallback)
when no device is present."""
import os
import re

import pytest

from conftest import ROOT, has_gpu


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "rism3d_b200.h")).read()
    return sorted(set(re.findall(r"\b(rism3d_[a-z_0-9]+)\s*\(", txt)))


def test_header_declares_reference_interface():
    syms = declared_symbols()
    for s in ("rism3d_initialize", "rism3d_iterate", "rism3d_output", "rism3d_create",
              "rism3d_solve", "rism3d_grad", "rism3d_grad_precision", "rism3d_solve_batch", "rism3d_destroy"):
        assert s in syms


def test_library_exports_every_declared_symbol():
    import rism3d_b200 as R
    L = R.lib()
    for s in declared_symbols():
        assert hasattr(L, s), s


def test_shape_validation_before_device():
    import rism3d_b200 as R
    with pytest.raises(R.RismError) as e:
        R.Solver((50, 64, 64), (32, 32, 32))
    assert e.value.code == R.UNSUPPORTED_SHAPE


@pytest.mark.skipif(has_gpu(), reason="checks the no-device error path")
def test_no_device_is_an_error_not_a_fallback():
    import rism3d_b200 as R
    with pytest.raises(R.RismError) as e:
        R.Solver((64, 64, 64), (32, 32, 32))
    assert e.value.code == R.NO_DEVICE
