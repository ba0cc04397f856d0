"""The oracle's deformed-window restatement (no counterpart in the reference, whose windows only
shift: multipass.rs:224-231). Parity of deformation is pinned against this restatement only; these
tests pin the restatement itself: it reduces to the uniform path when the predictor is zero, its
corners are the predictor's bilinear samples, and it measures a vortex better than uniform
windows."""
import numpy as np

from oracle import oracle as O


def _pair(h, seed=7, vmax=6.0, core=30.0):
    from piv_b200 import synthetic as S
    f = S.vortex_shear_field(h, h, vmax=vmax, core=core, shear=0.0)
    a, b = S.particle_pair(h, h, seed, 0.05, 0.75, f)
    return a, b, f


def test_place_deform_without_predictor_is_uniform_placement():
    g = O.grid(200, 240, 32, 0.5)
    o, c = O.place_deform(g, 200, 240)
    assert np.array_equal(o.view(np.uint32), O.place(g, 200, 240).view(np.uint32))
    assert not c.any()


def test_zero_corners_equal_uniform_windows_bit_for_bit():
    """With a zero predictor every deformed sample sits on a pixel (bilinear weights 1, 0, 0, 0),
    so the deformed path must reproduce the uniform path exactly, in both arithmetic modes."""
    a, b, _ = _pair(160)
    for n in (32, 16):
        g = O.grid(160, 160, n, 0.5)
        o, c = O.place_deform(g, 160, 160)
        for mode in (O.REF, O.FP64):
            u = O.correlate_pass(a, b, a, b, n, o, mode=mode)
            d = O.correlate_pass_deform(a, b, a, b, g, o, c, mode=mode)
            for x, y in zip(u, d):
                assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))


def test_corners_sample_the_predictor_at_the_corner_pixels():
    h = w = 256
    pg = O.grid(h, w, 64, 0.5)
    cx = pg.x0 + np.arange(pg.nx) * pg.step + 31.5
    cy = pg.y0 + np.arange(pg.ny) * pg.step + 31.5
    X, Y = np.meshgrid(cx, cy)
    pdx = (0.5 + 0.01 * X).astype(np.float32)
    pdy = (-1.0 + 0.02 * Y).astype(np.float32)
    g = O.grid(h, w, 32, 0.5)
    _, c = O.place_deform(g, h, w, pg, pdx, pdy)
    x0 = (g.x0 + (np.arange(g.nx * g.ny) % g.nx) * g.step).astype(np.float64)
    y0 = (g.y0 + (np.arange(g.nx * g.ny) // g.nx) * g.step).astype(np.float64)
    xs = [x0, x0 + 31, x0, x0 + 31]
    ys = [y0, y0, y0 + 31, y0 + 31]
    inside = (x0 >= cx[0]) & (x0 + 31 <= cx[-1]) & (y0 >= cy[0]) & (y0 + 31 <= cy[-1])
    assert inside.sum() > 10
    for j in range(4):
        np.testing.assert_allclose(c[inside, 2 * j], 0.5 + 0.01 * xs[j][inside], atol=2e-5)
        np.testing.assert_allclose(c[inside, 2 * j + 1], -1.0 + 0.02 * ys[j][inside], atol=2e-5)


def test_deformed_windows_measure_a_vortex_better():
    """On a strong vortex the deformed windows halve the RMS error against the true field at the
    final-pass window centres (FP64 oracle, 64 -> 32 -> 16 px)."""
    for h, vmax, core in ((256, 6.0, 30.0), (384, 8.0, 40.0)):
        a, b, f = _pair(h, vmax=vmax, core=core)
        err = {}
        for d in (0, 1):
            cfg = O.OracleConfig(windows=[64, 32, 16], overlap=0.5, final_iterations=2, deform=d)
            fin, _, _ = O.analyze(cfg, a, b, mode=O.FP64)
            g = O.grid(h, h, 16, 0.5)
            X, Y = np.meshgrid(g.x0 + np.arange(g.nx) * g.step + 7.5, g.y0 + np.arange(g.ny) * g.step + 7.5)
            u, v = f(X, Y)
            ok = fin["flags"] == 0
            err[d] = float(np.sqrt(np.mean((fin["dx"][ok] - u[ok]) ** 2 + (fin["dy"][ok] - v[ok]) ** 2)))
        assert err[1] < 0.6 * err[0], (h, err)


def test_deform_is_only_used_with_a_predictor():
    """A single-pass schedule has no predictor: deform on and off give the same field."""
    a, b, _ = _pair(160)
    r = [O.analyze(O.OracleConfig(windows=[32], overlap=0.5, final_iterations=1, deform=d), a, b)[0] for d in (0, 1)]
    for k in ("dx", "dy", "ppr", "flags"):
        assert np.array_equal(r[0][k].view(np.uint8), r[1][k].view(np.uint8))
