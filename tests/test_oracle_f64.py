"""The oracle's f64 build (oracle/liboracle_f64.so, -DORACLE_F64): the same
restatement with its arithmetic in double, used for converged reference
images free of f32 rounding. On the same noise keys it takes the same paths
as the f32 build except where a decision sits within f32 rounding of its
threshold, so the two images agree closely but not exactly."""
import numpy as np

from oracle.binding import OracleTracer
from stargaze_b200 import workloads as W


def render(f64: bool) -> np.ndarray:
    wl = W.rings_1080p(64, 36, 16)
    t = OracleTracer((wl.width, wl.height), W.render_options(wl, 16), threads=4, f64=f64)
    W.upload_workload(t, wl)
    while t.samples() < 16:
        t.encode(wl.frame)
    return t.read_pixels()[:, :3].astype(np.float64)


def test_f64_oracle_matches_f32_to_rounding():
    a, b = render(False), render(True)
    assert np.isfinite(b).all() and (b >= 0.0).all()
    rel = np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum())
    assert 0.0 < rel < 1e-3, rel
