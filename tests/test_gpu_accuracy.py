"""Accuracy gate: the GPU's final field within 0.01 px RMS of the FP64 oracle (every correlation
step in f64) on the benchmark's kind of input: a 12-bit particle pair with a vortex, shear and
spurious particle clusters, every window size the GPU supports in a schedule."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("windows,overlap,deform", [([128, 64, 32, 16], 0.75, False), ([64, 32, 16], 0.5, True),
                                                    ([96, 48, 24, 12], 0.5, False), ([64, 32, 16, 8], 0.5, False)])
def test_final_field_within_0p01_px_rms_of_fp64(windows, overlap, deform):
    import piv_b200 as P
    from piv_b200 import synthetic as S
    h = w = 512
    f = S.vortex_shear_field(h, w, vmax=8.0, shear=0.01)
    g = P.Grid.new(h, w, windows[-1], overlap)
    rng = np.random.default_rng(1)
    k = rng.choice(len(g), len(g) // 50, replace=False)
    cells = np.stack([g.x0 + (k % g.nx) * g.step, g.y0 + (k // g.nx) * g.step], 1)
    a, b = S.baseline_pair(h, w, 9, f, ppp=0.05, dmin=2.0, dmax=4.0, bits=12, outlier_cells=cells,
                           outlier_window=windows[-1])
    an = P.PivAnalyzer(P.PivConfig(windows=windows, overlap=overlap, final_iterations=1, deform=deform))
    r = an.analyze(an.prepare(a, P.RAW), an.prepare(b, P.RAW))
    fa, fb = O.u16_to_f32(a), O.u16_to_f32(b)
    ref, _, _ = O.analyze(O.OracleConfig(windows, overlap, 1, deform=int(deform)), fa, fb, mode=O.FP64)
    ok = (ref["flags"] == 0) & (r.field.flags == 0)
    d = np.hypot(r.field.dx[ok] - ref["dx"][ok], r.field.dy[ok] - ref["dy"][ok])
    assert ok.mean() > 0.9
    assert np.sqrt(np.mean(d * d)) <= 0.01, np.sqrt(np.mean(d * d))
    assert np.mean(ref["flags"] == r.field.flags) > 0.99
