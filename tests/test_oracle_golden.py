"""The CPU oracle against the reference's golden fixtures (pins the oracle before it is trusted).

Mirrors swift/Tests/PIVKitTests/RustParityCPUTests.swift:9-20 (validation bit for bit),
RustParityGPUTests.swift:39-123 (origins exact, raw peaks within 1e-4 px, PPR within 1e-5
relative, flags identical, final RMS < 1e-4 px) and PreprocessParityTests.swift:29-61 (prepared
images within 1e-4 x max|v|), applied to the C++ restatement.
"""
import numpy as np

from conftest import same_floats
from oracle import oracle as O


def test_prepared_images_match(golden):
    g = golden
    for raw, ref in ((g.frame_a, g.prepared_a), (g.frame_b, g.prepared_b)):
        img, base = O.prepare(raw, g.pre["smooth_sigma"], g.pre["normalize_radius"], g.pre["normalize_eps"], g.background)
        scale = max(float(np.abs(ref).max()), 1.0)
        assert float(np.abs(img - ref).max()) <= 1e-4 * scale


def test_placement_is_bit_exact(golden):
    g = golden
    pg = pdx = pdy = None
    for i, p in enumerate(g.passes):
        gr = O.grid(g.h, g.w, p["grid"]["window"], g.piv["overlap"])
        assert (gr.nx, gr.ny, gr.step, gr.x0, gr.y0) == tuple(p["grid"][k] for k in ("nx", "ny", "step", "x0", "y0"))
        o = O.place(gr, g.h, g.w, pg, pdx, pdy)
        assert np.array_equal(o.view(np.uint32), p["origins"].view(np.uint32)), f"pass {i}"
        pg, pdx, pdy = gr, p["dx"], p["dy"]


def test_raw_peaks_within_tolerance(golden):
    g = golden
    m = g.piv["mask"]
    for i, p in enumerate(g.passes):
        dx, dy, ppr, fl = O.correlate_pass(g.prepared_a, g.prepared_b, g.base_a, g.base_b, p["grid"]["window"],
                                           p["origins"], m["min_mean"], m["min_std"])
        assert np.array_equal(fl, p["raw_flags"].ravel()), f"pass {i}: NO_SIGNAL decisions"
        fin = np.isfinite(p["raw_dx"].ravel())
        assert np.array_equal(fin, np.isfinite(dx))
        worst = np.abs(np.r_[dx[fin] - p["raw_dx"].ravel()[fin], dy[fin] - p["raw_dy"].ravel()[fin]]).max(initial=0)
        assert worst < 1e-4, f"pass {i}: worst |dd| {worst}"
        rel = np.abs(ppr[fin] / p["raw_ppr"].ravel()[fin] - 1).max(initial=0)
        assert rel < 1e-5, f"pass {i}: worst ppr rel {rel}"
        # integer peak index = round(raw_d - (b - a)) is bit-exact
        o = p["origins"]
        ki = np.round(dx[fin] - (o[fin, 2] - o[fin, 0]))
        kr = np.round(p["raw_dx"].ravel()[fin] - (o[fin, 2] - o[fin, 0]))
        assert np.array_equal(ki, kr)


def test_validation_is_bit_exact(golden):
    g = golden
    v = g.val
    for i, p in enumerate(g.passes):
        dx, dy, fl, _ = O.validate(p["raw_dx"], p["raw_dy"], p["raw_ppr"], p["raw_flags"], v["ppr_threshold"],
                                   v["median_threshold"], v["median_eps"], v["replace"], g.max_displacement)
        assert np.array_equal(fl, p["flags"]), f"pass {i}: flags"
        assert same_floats(dx, p["dx"]) and same_floats(dy, p["dy"]), f"pass {i}: values"


def test_full_analysis_matches(golden):
    g = golden
    m, v = g.piv["mask"], g.val
    cfg = O.OracleConfig(tuple(g.piv["windows"]), g.piv["overlap"], g.piv["final_iterations"], m["min_mean"],
                         m["min_std"], v["ppr_threshold"], v["median_threshold"], v["median_eps"], v["replace"])
    fin, summary, traces = O.analyze(cfg, g.prepared_a, g.prepared_b, g.base_a, g.base_b, trace=True)
    ref = g.passes[-1]
    assert len(traces) == len(g.passes)
    assert np.array_equal(fin["flags"], ref["flags"])
    ok = np.isfinite(fin["dx"]) & np.isfinite(ref["dx"])
    rms = np.sqrt(np.mean((fin["dx"][ok] - ref["dx"][ok]) ** 2 + (fin["dy"][ok] - ref["dy"][ok]) ** 2))
    assert rms < 1e-4
    assert summary == g.meta["summary"]


def test_fp64_mode_close_to_reference(golden):
    g = golden
    m = g.piv["mask"]
    p = g.passes[-1]
    dx, dy, _, fl = O.correlate_pass(g.prepared_a, g.prepared_b, g.base_a, g.base_b, p["grid"]["window"],
                                     p["origins"], m["min_mean"], m["min_std"], mode=O.FP64)
    assert np.array_equal(fl, p["raw_flags"].ravel())
    fin = np.isfinite(dx)
    assert np.abs(dx[fin] - p["raw_dx"].ravel()[fin]).max(initial=0) < 1e-4
