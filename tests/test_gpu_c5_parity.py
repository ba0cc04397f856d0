"""The benchmark's full-size pair against the FP32 oracle, stage by stage, in the manner of the
reference's own cross-implementation test (swift/Tests/PIVKitTests/RustParityGPUTests.swift:39-64),
which checks every pass given the other implementation's inputs.

Workload: 4096 x 4096 u16 (12-bit) particle pair with a vortex plus shear and spurious particle
clusters in 2 % of the final-pass cells, 128 -> 64 -> 32 -> 16 px windows at 75 % overlap
(15,625 / 64,009 / 259,081 / 1,042,441 cells), FP32 plain path.

Per pass, given the GPU's previous validated field:
- placement (multipass.rs:204-231): origins bit for bit;
- correlation of the GPU's origins (correlate.rs:99-303): NO_SIGNAL decisions identical, integer
  peak indices identical, sub-pixel displacement within 1e-3 px everywhere and 1e-4 px for all but
  1e-4 of the cells;
- validation of the GPU's raw field (validate.rs:51-170): flags and values bit for bit.
The final field is also compared with the FP64 oracle (every correlation step in f64), and the
split-precision tensor-core tiers must find the FP32 path's integer peaks on the same origins.
"""
import numpy as np
import pytest

from conftest import same_floats
from oracle import oracle as O

pytestmark = pytest.mark.gpu

WINDOWS = [128, 64, 32, 16]
OVERLAP = 0.75
CELLS = [15625, 64009, 259081, 1042441]


@pytest.fixture(scope="module")
def c5():
    import bench
    import piv_b200 as P
    a, b = bench.make_inputs(bench.WORKLOADS["c5"])
    assert a.shape == (4096, 4096) and a.dtype == np.uint16
    an = P.PivAnalyzer(P.PivConfig(windows=WINDOWS, overlap=OVERLAP, final_iterations=1))
    fa, fb = an.prepare(a, P.RAW), an.prepare(b, P.RAW)
    ia, ib = O.u16_to_f32(a), O.u16_to_f32(b)
    result, traces = an.analyze_traced(fa, fb)
    return dict(a=a, b=b, ia=ia, ib=ib, an=an, fa=fa, fb=fb, result=result, traces=traces)


@pytest.fixture(scope="module")
def fp64_final(c5):
    ref, _, _ = O.analyze(O.OracleConfig(tuple(WINDOWS), OVERLAP, 1), c5["ia"], c5["ib"], mode=O.FP64)
    return ref


def _integer_peaks(d, origins):
    """round(displacement - (b - a)): the integer correlation-peak index of each cell."""
    return np.round(np.r_[d[0] - (origins[:, 2] - origins[:, 0]), d[1] - (origins[:, 3] - origins[:, 1])])


def _ambiguous(d, origins):
    """Cells whose sub-pixel offset sits within 1e-3 of +-0.5, where the integer index is a tie."""
    off = np.r_[d[0] - (origins[:, 2] - origins[:, 0]), d[1] - (origins[:, 3] - origins[:, 1])]
    return np.abs(np.abs(off - np.round(off)) - 0.5) < 1e-3


def test_c5_prepared_frames_are_the_reference_decoding(c5):
    # u16 -> f32 as v / 65535 (decode.rs:227-234), bit for bit
    assert np.array_equal(c5["fa"].image.view(np.uint32), c5["ia"].view(np.uint32))
    assert np.array_equal(c5["fb"].image.view(np.uint32), c5["ib"].view(np.uint32))


def test_c5_every_pass_matches_the_fp32_oracle(c5):
    h, w = c5["a"].shape
    ia, ib = c5["ia"], c5["ib"]
    prev = None
    report = []
    for i, t in enumerate(c5["traces"]):
        g = t.raw.grid
        assert g.window == WINDOWS[i] and len(g) == CELLS[i]
        og = O.grid(h, w, g.window, OVERLAP)
        if prev is None:
            o = O.place(og, h, w)
        else:
            o = O.place(og, h, w, O.grid(h, w, prev.grid.window, OVERLAP), prev.dx, prev.dy)
        assert np.array_equal(t.origins.view(np.uint32), o.view(np.uint32)), f"pass {i}: origins"
        dx, dy, ppr, fl = O.correlate_pass(ia, ib, ia, ib, g.window, t.origins)
        assert np.array_equal(t.raw.flags.ravel(), fl), f"pass {i}: NO_SIGNAL decisions"
        fin = np.isfinite(dx)
        assert np.array_equal(fin, np.isfinite(t.raw.dx.ravel()))
        oo = t.origins[fin]
        gd = (t.raw.dx.ravel()[fin], t.raw.dy.ravel()[fin])
        od = (dx[fin], dy[fin])
        gi, oi = _integer_peaks(gd, oo), _integer_peaks(od, oo)
        amb = _ambiguous(od, oo)
        mismatch = int(np.count_nonzero((gi != oi) & ~amb))
        err = np.abs(np.r_[gd[0] - od[0], gd[1] - od[1]])
        rel_ppr = np.abs(t.raw.peak_ratio.ravel()[fin] / ppr[fin] - 1)
        report.append(dict(window=g.window, cells=len(g), no_signal=int(np.count_nonzero(fl & O.NO_SIGNAL)),
                           peak_mismatch=mismatch, ambiguous=int(np.count_nonzero(amb)), max_px=float(err.max()),
                           p9999_px=float(np.quantile(err, 0.9999)), rms_px=float(np.sqrt(np.mean(err ** 2))),
                           max_ppr_rel=float(rel_ppr.max())))
        print("c5 pass vs FP32 oracle:", report[-1])
        assert mismatch == 0, f"pass {i}: {mismatch} integer peak indices differ"
        assert err.max() <= 1e-3, report[-1]
        assert np.mean(err > 1e-4) <= 1e-4, report[-1]
        vdx, vdy, vfl, _ = O.validate(t.raw.dx, t.raw.dy, t.raw.peak_ratio, t.raw.flags, 1.3, 2.0, 0.1, True,
                                      WINDOWS[0] / 2.0)
        assert np.array_equal(vfl, t.validated.flags), f"pass {i}: validated flags"
        assert same_floats(vdx, t.validated.dx) and same_floats(vdy, t.validated.dy), f"pass {i}: validated values"
        prev = t.validated
    # the spurious clusters make outliers that the final validation catches and replaces
    final = c5["traces"][-1].validated
    assert np.count_nonzero(final.flags & O.REPLACED) > 1e-3 * CELLS[-1]


def test_c5_final_field_against_the_fp64_oracle(c5, fp64_final):
    ref = fp64_final
    f = c5["result"].field
    ok = (ref["flags"] == 0) & (f.flags == 0)
    d = np.hypot(f.dx[ok] - ref["dx"][ok], f.dy[ok] - ref["dy"][ok])
    rms, mx = float(np.sqrt(np.mean(d * d))), float(d.max())
    agree = float(np.mean(ref["flags"] == f.flags))
    print(f"c5 final field vs FP64 oracle: rms {rms:.3e} px, max {mx:.3e} px, flag agreement {agree:.6f}")
    assert ok.mean() > 0.95
    assert rms <= 1e-3 and agree >= 0.9999


@pytest.mark.parametrize("precision", ["bf16x3", "fp16x3"])
def test_c5_tensor_core_tiers_find_the_fp32_peaks(c5, fp64_final, precision):
    """On the FP32 path's own origins, every pass of the split-precision tier gives the same
    NO_SIGNAL decisions and integer peaks; its whole analysis stays within 0.01 px RMS of the FP64
    oracle's."""
    import piv_b200 as P
    an = P.PivAnalyzer(P.PivConfig(windows=WINDOWS, overlap=OVERLAP, final_iterations=1, precision=precision))
    fa, fb = an.prepare(c5["a"], P.RAW), an.prepare(c5["b"], P.RAW)
    for i, t in enumerate(c5["traces"]):
        n = t.raw.grid.window
        dx, dy, ppr, fl = an.correlate_origins(fa, fb, n, t.origins)
        assert np.array_equal(fl, t.raw.flags.ravel()), f"{precision} pass {i}"
        fin = np.isfinite(t.raw.dx.ravel())
        oo = t.origins[fin]
        ref = (t.raw.dx.ravel()[fin], t.raw.dy.ravel()[fin])
        mine = (dx[fin], dy[fin])
        amb = _ambiguous(ref, oo) | _ambiguous(mine, oo)
        mismatch = int(np.count_nonzero((_integer_peaks(mine, oo) != _integer_peaks(ref, oo)) & ~amb))
        err = np.abs(np.r_[mine[0] - ref[0], mine[1] - ref[1]])
        print(f"c5 {precision} pass {i} ({n} px, {'tensor cores' if 'tensor' in an.variant(n) else 'FP32'}) vs FP32: "
              f"peak mismatches {mismatch}, rms {np.sqrt(np.mean(err ** 2)):.3e} px, max {err.max():.3e} px")
        assert mismatch == 0, f"{precision} pass {i}: {mismatch} integer peaks differ from the FP32 path"
        assert np.sqrt(np.mean(err ** 2)) <= 1e-3
    r = an.analyze(fa, fb)
    ref = fp64_final
    ok = (ref["flags"] == 0) & (r.field.flags == 0)
    d = np.hypot(r.field.dx[ok] - ref["dx"][ok], r.field.dy[ok] - ref["dy"][ok])
    print(f"c5 {precision} final field vs FP64 oracle: rms {np.sqrt(np.mean(d * d)):.3e} px, max {d.max():.3e} px")
    assert np.sqrt(np.mean(d * d)) <= 0.01
