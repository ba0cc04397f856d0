"""The CUDA path against the reference's golden fixtures and the CPU oracle, through the C ABI.

Mirrors the reference's own cross-implementation tests:
  swift/Tests/PIVKitTests/RustParityGPUTests.swift:39-64   per pass, given Rust's predictor:
      origins identical, raw peaks within 1e-4 px, PPR rel. error < 1e-5, flags identical
  RustParityGPUTests.swift:68-89                          placement and validation bit for bit
  RustParityGPUTests.swift:105-123                        final field RMS < 1e-4 px, flags identical
  PreprocessParityTests.swift:29-61                       prepared images within 1e-4 x max|v|;
                                                          raw frames -> final field within 1e-3 px
"""
import numpy as np
import pytest

from conftest import same_floats
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _analyzer(g):
    import piv_b200 as P
    m, v = g.piv["mask"], g.val
    cfg = P.PivConfig(windows=list(g.piv["windows"]), overlap=g.piv["overlap"],
                      final_iterations=g.piv["final_iterations"], mask=P.MaskConfig(m["min_mean"], m["min_std"]),
                      validation=P.ValidationConfig(v["ppr_threshold"], v["median_threshold"], v["median_eps"],
                                                    v["replace"]))
    return P.PivAnalyzer(cfg)


def _frames(an, g):
    fa = an.frame(g.h, g.w).set_prepared(g.prepared_a, g.base_a)
    fb = an.frame(g.h, g.w).set_prepared(g.prepared_b, g.base_b)
    return fa, fb


def test_placement_matches_reference_exactly(golden):
    import piv_b200 as P
    g = golden
    an = _analyzer(g)
    pred = None
    for i, p in enumerate(g.passes):
        gr = P.Grid.new(g.h, g.w, p["grid"]["window"], g.piv["overlap"])
        o = an.place_windows(g.h, g.w, gr, pred)
        assert np.array_equal(o.view(np.uint32), p["origins"].view(np.uint32)), f"{g.name} pass {i}"
        pred = P.VectorField(gr, p["dx"], p["dy"], p["ppr"], p["flags"])


def test_raw_peaks_match_reference_pass_by_pass(golden):
    g = golden
    an = _analyzer(g)
    fa, fb = _frames(an, g)
    for i, p in enumerate(g.passes):
        dx, dy, ppr, fl = an.correlate_origins(fa, fb, p["grid"]["window"], p["origins"])
        assert np.array_equal(fl, p["raw_flags"].ravel()), f"{g.name} pass {i}: flags"
        fin = np.isfinite(p["raw_dx"].ravel())
        rdx, rdy, rppr = p["raw_dx"].ravel()[fin], p["raw_dy"].ravel()[fin], p["raw_ppr"].ravel()[fin]
        worst = np.abs(np.r_[dx[fin] - rdx, dy[fin] - rdy]).max(initial=0.0)
        assert worst < 1e-4, f"{g.name} pass {i} (n={p['grid']['window']}): worst |dd| {worst}"
        rel = np.abs(ppr[fin] / rppr - 1).max(initial=0.0)
        assert rel < 1e-5, f"{g.name} pass {i}: worst PPR rel {rel}"
        o = p["origins"][fin]
        assert np.array_equal(np.round(dx[fin] - (o[:, 2] - o[:, 0])), np.round(rdx - (o[:, 2] - o[:, 0])))
        assert np.array_equal(np.round(dy[fin] - (o[:, 3] - o[:, 1])), np.round(rdy - (o[:, 3] - o[:, 1])))


def test_validation_matches_reference_exactly(golden):
    g = golden
    an = _analyzer(g)
    for i, p in enumerate(g.passes):
        dx, dy, fl, _ = an.validate_field(p["raw_dx"], p["raw_dy"], p["raw_ppr"], p["raw_flags"])
        assert np.array_equal(fl, p["flags"]), f"{g.name} pass {i}: flags"
        assert same_floats(dx, p["dx"]) and same_floats(dy, p["dy"]), f"{g.name} pass {i}: values"


def test_final_field_matches_reference(golden):
    g = golden
    an = _analyzer(g)
    fa, fb = _frames(an, g)
    r = an.analyze(fa, fb)
    ref = g.passes[-1]
    assert np.array_equal(r.field.flags, ref["flags"]), g.name
    ok = np.isfinite(ref["dx"]) & np.isfinite(r.field.dx)
    rms = float(np.sqrt(np.mean((r.field.dx[ok] - ref["dx"][ok]) ** 2 + (r.field.dy[ok] - ref["dy"][ok]) ** 2)))
    assert rms < 1e-4, f"{g.name}: RMS {rms}"
    assert r.summary.as_dict() == g.meta["summary"]


def test_traced_run_is_consistent(golden):
    g = golden
    an = _analyzer(g)
    fa, fb = _frames(an, g)
    r, traces = an.analyze_traced(fa, fb)
    assert len(traces) == len(g.passes)
    plain = an.analyze(fa, fb)
    assert np.array_equal(plain.field.flags, r.field.flags)
    assert same_floats(plain.field.dx, r.field.dx) and same_floats(plain.field.dy, r.field.dy)
    for i, (t, p) in enumerate(zip(traces, g.passes)):
        assert np.array_equal(t.origins.view(np.uint32), p["origins"].view(np.uint32)) or i > 0
        assert np.array_equal(t.raw.flags, p["raw_flags"])


def test_prepared_images_match_reference(golden):
    import piv_b200 as P
    g = golden
    an = _analyzer(g)
    pre = P.PreprocessConfig(g.pre["smooth_sigma"], g.pre["normalize_radius"], g.pre["normalize_eps"])
    for raw, ref in ((g.frame_a, g.prepared_a), (g.frame_b, g.prepared_b)):
        img = an.prepare(raw, pre, g.background).image
        scale = max(float(np.abs(ref).max()), 1.0)
        worst = float(np.abs(img - ref).max())
        assert worst <= 1e-4 * scale, f"{g.name}: worst |d| {worst}"
        exact = float(np.mean(img.view(np.uint32) == ref.view(np.uint32)))
        assert exact > 0.999, f"{g.name}: only {exact:.6f} of pixels bit-exact"


def test_raw_frames_to_field_match_reference(golden):
    import piv_b200 as P
    g = golden
    an = _analyzer(g)
    pre = P.PreprocessConfig(g.pre["smooth_sigma"], g.pre["normalize_radius"], g.pre["normalize_eps"])
    fa = an.prepare(g.frame_a, pre, g.background)
    fb = an.prepare(g.frame_b, pre, g.background)
    r = an.analyze(fa, fb)
    ref = g.passes[-1]
    assert np.array_equal(r.field.flags, ref["flags"]), g.name
    fin = np.isfinite(ref["dx"])
    worst = float(np.abs(np.r_[r.field.dx[fin] - ref["dx"][fin], r.field.dy[fin] - ref["dy"][fin]]).max(initial=0))
    assert worst < 1e-3, f"{g.name}: worst |dd| {worst}"


def _stage_check(an, traces, a, b, windows, overlap=0.5, min_mean=0.0, min_std=0.0):
    """Every pass of a GPU trace against the oracle stage run on the GPU's own inputs: placement
    from the GPU's previous validated field (bit-exact), correlation of the GPU's origins (peak
    indices and NO_SIGNAL exact, sub-pixel within 1e-4 px), validation of the GPU's raw field
    (bit-exact)."""
    h, w = a.shape
    prev = None
    for i, t in enumerate(traces):
        g = t.raw.grid
        og = O.grid(h, w, g.window, overlap)
        if prev is None:
            o = O.place(og, h, w)
        else:
            o = O.place(og, h, w, O.grid(h, w, prev.grid.window, overlap), prev.dx, prev.dy)
        assert np.array_equal(t.origins.view(np.uint32), o.view(np.uint32)), f"{windows} pass {i}: origins"
        dx, dy, ppr, fl = O.correlate_pass(a, b, a, b, g.window, t.origins, min_mean, min_std)
        assert np.array_equal(t.raw.flags.ravel(), fl), f"{windows} pass {i}: NO_SIGNAL decisions"
        fin = np.isfinite(dx)
        gd = np.r_[t.raw.dx.ravel()[fin], t.raw.dy.ravel()[fin]]
        od = np.r_[dx[fin], dy[fin]]
        err = np.abs(gd - od).max(initial=0)
        assert err < 1e-4, f"{windows} pass {i}: worst |dd| {err}"
        oo = np.r_[t.origins[fin, 2] - t.origins[fin, 0], t.origins[fin, 3] - t.origins[fin, 1]]
        agree = np.mean(np.round(gd - oo) == np.round(od - oo))
        assert agree == 1.0, f"{windows} pass {i}: peak index agreement {agree}"
        vdx, vdy, vfl, _ = O.validate(t.raw.dx, t.raw.dy, t.raw.peak_ratio, t.raw.flags, 1.3, 2.0, 0.1, True,
                                      windows[0] / 2.0)
        assert np.array_equal(vfl, t.validated.flags), f"{windows} pass {i}: validated flags"
        assert same_floats(vdx, t.validated.dx) and same_floats(vdy, t.validated.dy), f"{windows} pass {i}: values"
        prev = t.validated


def test_matches_oracle_on_synthetic_particles():
    """GPU vs the CPU oracle, stage by stage, on seeded synthetic pairs at every supported size."""
    import piv_b200 as P
    from piv_b200 import synthetic as S
    for windows, h in (([32, 16], 256), ([64, 32, 16], 320), ([128, 64], 384), ([48, 24, 12], 240), ([96, 48], 288),
                       ([16, 8], 128)):
        a, b = S.particle_pair(h, h, 11, 0.05, 0.75, lambda x, y: (2.3 + 0.01 * y, -1.7 + 0.005 * x))
        an = P.PivAnalyzer(P.PivConfig(windows=windows, final_iterations=2))
        fa, fb = an.prepare(a, P.RAW), an.prepare(b, P.RAW)
        _, traces = an.analyze_traced(fa, fb)
        _stage_check(an, traces, a, b, windows)


def test_128px_peaks_in_every_quadrant_and_at_the_wrap():
    """The 128 px window (one window per group, its real inverse as half-size stages) against the
    oracle on window pairs whose offsets put the correlation peak in every quadrant of the plane,
    next to the +-N/2 wrap, on the self-conjugate row and column (ky or kx in {0, N/2} carry the
    packed lines) and at fractional positions: peak indices exact, sub-pixel within 1e-4 px, PPR
    within 1e-5 relative."""
    import piv_b200 as P
    from piv_b200 import synthetic as S
    n = 128
    a, _ = S.particle_pair(448, 448, 31, 0.06, 0.9, lambda x, y: (0.0, 0.0))
    a = S.add_noise(a, 0.01, 5)
    offsets = [(0.0, 0.0), (9.0, -13.0), (-21.0, 17.0), (40.0, 40.0), (-40.0, -40.0), (55.0, -3.0), (-3.0, 55.0),
               (-58.0, 0.0), (0.0, -58.0), (61.0, 61.0), (-61.0, 60.0), (62.5, -0.25), (-0.75, 62.5),
               (31.3, -47.6), (-12.2, 5.7), (64.0, 0.0), (0.0, -64.0)]
    origins = []
    for i, (ox, oy) in enumerate(offsets):
        ax, ay = 80.0 + 17.0 * (i % 5), 80.0 + 23.0 * (i // 5)
        origins.append((ax, ay, ax + ox, ay + oy))
    origins = np.array(origins, np.float32)
    an = P.PivAnalyzer(P.PivConfig(windows=[n]))
    fa, fb = an.prepare(a, P.RAW), an.prepare(a, P.RAW)
    dx, dy, ppr, fl = an.correlate_origins(fa, fb, n, origins)
    odx, ody, oppr, ofl = O.correlate_pass(a, a, a, a, n, origins)
    assert np.array_equal(fl, ofl)
    assert np.all(fl == 0)
    err = np.abs(np.r_[dx - odx, dy - ody]).max()
    assert err < 1e-4, err
    off = np.r_[origins[:, 2] - origins[:, 0], origins[:, 3] - origins[:, 1]]
    assert np.array_equal(np.round(np.r_[dx, dy] - off), np.round(np.r_[odx, ody] - off))
    assert np.abs(ppr / oppr - 1).max() < 1e-5
    # the same frame on both sides: every vector is the zero displacement up to the sub-pixel fit,
    # modulo N (a peak at index N/2 reads as -N/2, correlate.rs:283-290, so an offset of -64
    # gives -128)
    d = np.r_[dx, dy]
    assert np.abs((d + n / 2) % n - n / 2).max() < 0.5
    assert d[len(offsets) - 1 + len(offsets)] == pytest.approx(-128.0, abs=0.5)


def test_autotuned_variants_give_identical_results():
    """Launch-geometry autotuning never changes results: variants differ only in geometry."""
    import piv_b200 as P
    from piv_b200 import synthetic as S
    a, b = S.particle_pair(384, 384, 21, 0.05, 0.75, lambda x, y: (3.1 + 0.01 * y, -2.2))
    for windows in ([128, 64, 32, 16], [96, 48, 24, 12], [64, 32, 16, 8]):
        an = P.PivAnalyzer(P.PivConfig(windows=windows, overlap=0.75, final_iterations=1))
        fa, fb = an.prepare(a, P.RAW), an.prepare(b, P.RAW)
        r0, t0 = an.analyze_traced(fa, fb)
        chosen = an.autotune(fa, fb)
        assert set(chosen) == set(windows)
        r1, t1 = an.analyze_traced(fa, fb)
        for x, y in zip(t0, t1):
            assert np.array_equal(x.raw.flags, y.raw.flags)
            assert same_floats(x.raw.dx, y.raw.dx) and same_floats(x.raw.dy, y.raw.dy)
            assert same_floats(x.raw.peak_ratio, y.raw.peak_ratio)


def test_every_launch_variant_gives_identical_results():
    """Each FP32 launch variant of each window size (groups per CTA, register cap, sampler) gives
    the bit-identical field: the variants share the FFT decomposition and every rounding."""
    import piv_b200 as P
    from piv_b200 import synthetic as S
    a, b = S.particle_pair(288, 288, 23, 0.05, 0.75, lambda x, y: (3.1 + 0.01 * y, -2.2 + 0.003 * x))
    for windows in ([128, 64, 32, 16], [96, 48, 24, 12], [64, 32, 16, 8]):
        an = P.PivAnalyzer(P.PivConfig(windows=windows, overlap=0.75, final_iterations=1))
        fa, fb = an.prepare(a, P.RAW), an.prepare(b, P.RAW)
        _, ref = an.analyze_traced(fa, fb)
        counts = {n: P.PivAnalyzer.num_variants(n) for n in windows}
        for k in range(1, max(counts.values())):
            for n in windows:
                an.set_variant(n, min(k, counts[n] - 1))
            _, got = an.analyze_traced(fa, fb)
            for x, y in zip(ref, got):
                assert np.array_equal(x.raw.flags, y.raw.flags), (windows, k)
                assert same_floats(x.raw.dx, y.raw.dx) and same_floats(x.raw.dy, y.raw.dy), (windows, k)
                assert same_floats(x.raw.peak_ratio, y.raw.peak_ratio), (windows, k)


def test_validation_with_signed_zero_and_repeated_values_matches_oracle():
    """Median test and replacement on fields full of ties (values drawn from a few, with -0.0
    and +0.0 both present) agree with the oracle bit for bit: the GPU's register sorting network
    and the oracle's sort both order as f32::total_cmp."""
    import piv_b200 as P
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    pool = np.array([-0.0, 0.0, 0.5, -0.5, 1.0, 3.0, -7.0], np.float32)
    an = P.PivAnalyzer(P.PivConfig(windows=[64, 32]))
    for trial in range(4):
        ny, nx = 37, 53
        dx = rng.choice(pool, (ny, nx)).astype(np.float32)
        dy = rng.choice(pool, (ny, nx)).astype(np.float32)
        ppr = rng.choice(np.array([1.0, 2.0, 9.0], np.float32), (ny, nx)).astype(np.float32)
        fl = (rng.random((ny, nx)) < 0.05).astype(np.uint8)  # a few NO_SIGNAL cells
        dx[fl == 1] = np.nan
        dy[fl == 1] = np.nan
        gx, gy, gf, _ = an.validate_field(dx, dy, ppr, fl)
        ox, oy, of, _ = O.validate(dx, dy, ppr, fl, max_displacement=32.0)
        def same_bits(a, b):  # bit patterns, with any NaN equal to any NaN
            return bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))))
        assert np.array_equal(gf, of), trial
        assert np.any(np.signbit(ox[ox == 0])) and np.any(~np.signbit(ox[ox == 0]))
        assert same_bits(gx, ox) and same_bits(gy, oy), trial


def test_single_pass_u8_pair_of_the_cpu_case():
    """The reference's CPU-runnable case: a 512 x 512 u8 particle pair (0.05 ppp, diameters 2-4 px,
    peaks 120-255, noise sigma 4), uniform displacement (2.3, -1.7), one 32 px pass at 50 %
    overlap, no preprocessing, median test threshold 2 / eps 0.1, ppr 1.3. Stage by stage against
    the oracle, and the known displacement recovered."""
    import piv_b200 as P
    from piv_b200 import synthetic as S
    a, b = S.baseline_pair(512, 512, 1, lambda x, y: (2.3, -1.7), ppp=0.05, dmin=2.0, dmax=4.0, bits=8)
    assert a.dtype == np.uint8
    an = P.PivAnalyzer(P.PivConfig(windows=[32], overlap=0.5, final_iterations=1))
    fa, fb = an.prepare(a, P.RAW), an.prepare(b, P.RAW)
    res, traces = an.analyze_traced(fa, fb)
    assert len(res.field.dx.ravel()) == 961
    _stage_check(an, traces, O.u8_to_f32(a), O.u8_to_f32(b), [32], overlap=0.5)  # decoded as the GPU decodes
    ok = res.field.flags == 0
    assert ok.mean() > 0.95
    err = np.hypot(res.field.dx[ok] - 2.3, res.field.dy[ok] + 1.7)
    assert np.sqrt(np.mean(err ** 2)) < 0.1
