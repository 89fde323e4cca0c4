"""The byte models bench.py reports its rooflines with: the per-pass
algorithmic bytes of the solver's passes and the minimal fused pipeline
N (31 V s + 5 s_lr + 4) (540 B per point in FP64 and 292 B with FP32 bulk
and FP64 long-range grids at V = 2; 9.06 GB per 256^3 FP64 iteration)."""
import importlib.util
import os

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_fused_pipeline_bytes():
    b = _bench()
    n = 256 ** 3
    assert b.fused_pipeline_bytes_per_iter(n, 2, 8) == 540 * n
    assert b.fused_pipeline_bytes_per_iter(n, 2, 4, 8) == 292 * n
    assert abs(b.fused_pipeline_bytes_per_iter(n, 2, 8) / 1e9 - 9.06) < 0.01


def test_pass_bytes_per_point():
    b = _bench()
    fp32, fp64 = b.iter_bytes_per_point(2, 4), b.iter_bytes_per_point(2, 8)
    assert (fp32["pass_a"], fp32["pass_k"], fp32["pass_r"]) == (72, 24, 40)
    assert (fp64["pass_a"], fp64["pass_k"], fp64["pass_r"]) == (144, 40, 80)
