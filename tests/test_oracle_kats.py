"""The reference's own known-answer unit tests, run on the CPU oracle.

Ported from the #[cfg(test)] modules of the reference (same inputs, same assertions):
  correlate.rs:310-421, multipass.rs:319-475, validate.rs:187-248, preprocess.rs:223-270,
  grid.rs:77-105, field.rs:96-109, synthetic.rs (the generator itself is pinned to the fixtures).
"""
import numpy as np
import pytest

from oracle import oracle as O
from piv_b200 import synthetic as S


# ------------------------------------------------------------------ correlate.rs:310-421
def test_integer_shift_is_exact_for_circular_content():
    n = 32
    rng = S.Rng(7)
    a = np.array([[rng.uniform() for _ in range(n)] for _ in range(n)], np.float32)
    sx, sy = 5, n - 3
    b = np.array([[a[(y + n - sy) % n, (x + n - sx) % n] for x in range(n)] for y in range(n)], np.float32)
    dx, dy, height, ppr = O.correlate_window(a, 0, 0, b, 0, 0, n)
    assert abs(dx - 5.0) < 0.02 and abs(dy + 3.0) < 0.02
    assert abs(height - 1.0) < 1e-4
    assert ppr > 2.0


def test_subpixel_shift_of_particles():
    a, b = S.particle_pair(64, 64, 3, 0.05, 1.2, lambda x, y: (0.4, -0.3))
    dx, dy, _, _ = O.correlate_window(a, 16, 16, b, 16, 16, 32)
    assert abs(dx - 0.4) < 0.08 and abs(dy + 0.3) < 0.08


def test_isolated_particle_is_unbiased():
    a = S.render(64, 64, [31.3], [30.7], [1.5], [1.0])
    b = S.render(64, 64, [31.7], [30.45], [1.5], [1.0])
    dx, dy, _, _ = O.correlate_window(a, 0, 0, b, 0, 0, 64)
    assert abs(dx - 0.4) < 1e-3 and abs(dy + 0.25) < 1e-3


def test_fractional_origin_interpolates():
    a = np.fromfunction(lambda y, x: (x + 2 * y), (40, 40)).astype(np.float32)
    dst, _ = O.load_window(a, 3.5, 2.25, 16)
    assert abs(dst[0, 1] - dst[0, 0] - 1.0) < 1e-4 and abs(dst[1, 0] - dst[0, 0] - 2.0) < 1e-4


def test_flat_window_has_no_peak():
    a = np.full((32, 32), 0.3, np.float32)
    assert O.correlate_window(a, 0, 0, a, 0, 0, 32) is None


def test_peak_ratio_uses_local_maxima():
    n = 16
    c = np.zeros((n, n), np.float32)
    for y in range(n):
        for x in range(n):
            dy, dx = min(y, n - y), min(x, n - x)
            c[y, x] = np.exp(np.float32(-(dx * dx + dy * dy)) / np.float32(8.0))
    c[8, 8] = 0.25
    c[2, 0] += 0.05
    c[3, 0] -= 0.05
    dx, dy, _, ppr = O.find_peak(c)
    assert (dx, dy) == (0.0, 0.0)
    assert abs(ppr - 4.0) < 1e-3


# ------------------------------------------------------------------ multipass.rs:319-475
def _errors(field, grid, truth, margin, size):
    xs = np.array([grid.x0 + i * grid.step + (grid.window - 1) / 2 for i in range(grid.nx)], np.float32)
    ys = np.array([grid.y0 + i * grid.step + (grid.window - 1) / 2 for i in range(grid.ny)], np.float32)
    s, worst, n = 0.0, 0.0, 0
    for iy, y in enumerate(ys):
        for ix, x in enumerate(xs):
            if x < margin or y < margin or x > size - margin or y > size - margin:
                continue
            u, v = truth(x, y)
            e = float(np.hypot(field["dx"][iy, ix] - u, field["dy"][iy, ix] - v))
            s += e * e
            worst = max(worst, e)
            n += 1
    return (s / n) ** 0.5, worst, n


def _run(a, b, windows, **kw):
    cfg = O.OracleConfig(tuple(windows), 0.5, 1 if len(windows) == 1 else 2, **kw)
    fin, summ, _ = O.analyze(cfg, a, b)
    h, w = a.shape
    return fin, summ, O.grid(h, w, windows[-1], 0.5)


@pytest.mark.parametrize("i,uv", list(enumerate([(0.25, 0.0), (0.0, 0.5), (3.7, 0.0), (3.7, -1.3), (-2.2, 2.6)])))
def test_uniform_shifts_particles(i, uv):
    u, v = uv
    a, b = S.particle_pair(256, 256, 10 + i, 0.04, 1.2, lambda x, y: (u, v))
    fin, summ, g = _run(a, b, [64, 32])
    rms, worst, n = _errors(fin, g, lambda x, y: (u, v), 20.0, 256.0)
    assert n > 100 and rms < 0.05
    assert summ["median_outliers"] * 50 <= g.nx * g.ny


def test_uniform_shift_fog_texture_with_noise():
    u, v = 2.4, -1.7
    a, b = S.fog_pair(256, 256, 4, lambda x, y: (u, v))
    a, b = S.add_noise(a, 0.01, 1), S.add_noise(b, 0.01, 2)
    ia, ba = O.prepare(a)
    ib, bb = O.prepare(b)
    fin, _, _ = O.analyze(O.OracleConfig(), ia, ib, ba, bb)
    rms, _, _ = _errors(fin, O.grid(256, 256, 64, 0.5), lambda x, y: (u, v), 20.0, 256.0)
    assert rms < 0.1


def test_window_as_large_as_the_image():
    u, v = 1.5, -0.5
    a, b = S.particle_pair(64, 64, 3, 0.04, 1.2, lambda x, y: (u, v))
    fin, _, g = _run(a, b, [64])
    assert g.nx * g.ny == 1
    assert abs(fin["dx"][0, 0] - u) < 0.2 and abs(fin["dy"][0, 0] - v) < 0.2
    fin, _, _ = _run(a, b, [64, 64])
    assert np.isfinite(fin["dx"][0, 0])


def test_large_shift_recovered_by_multipass():
    u, v = 20.0, -6.0
    a, b = S.particle_pair(320, 320, 5, 0.04, 1.2, lambda x, y: (u, v))
    fin, _, g = _run(a, b, [64, 32])
    rms, _, _ = _errors(fin, g, lambda x, y: (u, v), 48.0, 320.0)
    assert rms < 0.1
    fin1, _, g1 = _run(a, b, [32])
    rms1, _, _ = _errors(fin1, g1, lambda x, y: (u, v), 48.0, 320.0)
    assert rms1 > 1.0


@pytest.mark.parametrize("kind", ["rotation", "shear"])
def test_rotation_and_shear(kind):
    c = 127.5
    if kind == "rotation":
        truth = lambda x, y: (-0.03 * (y - c), 0.03 * (x - c))
        seed = 6
    else:
        truth = lambda x, y: (0.025 * (y - c), 0.0)
        seed = 8
    a, b = S.particle_pair(256, 256, seed, 0.04, 1.2, lambda x, y: truth(x, y))
    fin, _, g = _run(a, b, [64, 32])
    rms, _, _ = _errors(fin, g, truth, 20.0, 256.0)
    assert rms < 0.15


def test_blank_regions_get_no_signal():
    a, b = S.particle_pair(128, 128, 9, 0.04, 1.2, lambda x, y: (1.0, 0.0))
    a[:, :64] = 0.0
    b[:, :64] = 0.0
    a, b = S.add_noise(a, 0.002, 3), S.add_noise(b, 0.002, 4)
    cfg = O.OracleConfig(min_mean=0.01, min_std=0.01)
    fin, _, _ = O.analyze(cfg, a, b)
    g = O.grid(128, 128, 64, 0.5)
    for ix in range(g.nx):
        x = g.x0 + ix * g.step + 31.5
        col = fin["flags"][:, ix]
        if x + 16.0 < 64.0:
            assert np.all(col == O.NO_SIGNAL) and np.all(np.isnan(fin["dx"][:, ix]))
        elif x - 16.0 >= 64.0:
            assert np.all((col & O.NO_SIGNAL) == 0)


def test_rejects_bad_config():
    import ctypes
    for kw in (dict(windows=()), dict(windows=(33,)), dict(overlap=1.0), dict(final_iterations=0)):
        c = O.OracleConfig(**kw).c()
        assert O.lib().orc_check_config(ctypes.byref(c)) != 0
    c = O.OracleConfig().c()
    assert O.lib().orc_check_config(ctypes.byref(c)) == 0


# ------------------------------------------------------------------ validate.rs:187-248
def _uniform_field(u, v):
    g = O.grid(160, 160, 32, 0.5)
    sh = (g.ny, g.nx)
    return (np.full(sh, u, np.float32), np.full(sh, v, np.float32), np.full(sh, 5.0, np.float32),
            np.zeros(sh, np.uint8))


def test_catches_and_replaces_injected_outliers():
    dx, dy, ppr, fl = _uniform_field(2.0, -1.0)
    flat = dx.reshape(-1)
    for i in range(flat.size):
        flat[i] += np.float32(0.05) * np.float32((i * 7 % 5) - 2.0)
    outliers = [(2, 3), (5, 5), (8, 0)]
    for iy, ix in outliers:
        dx[iy, ix], dy[iy, ix] = 9.0, 4.0
    odx, ody, ofl, s = O.validate(dx, dy, ppr, fl)
    assert s["median_outliers"] == len(outliers) and s["replaced"] == len(outliers)
    for iy, ix in outliers:
        assert ofl[iy, ix] & O.MEDIAN_OUTLIER and ofl[iy, ix] & O.REPLACED
        assert abs(odx[iy, ix] - 2.0) < 0.2 and abs(ody[iy, ix] + 1.0) < 1e-6


def test_low_peak_ratio_is_flagged_and_no_signal_untouched():
    dx, dy, ppr, fl = _uniform_field(1.0, 1.0)
    ppr[4, 4] = 1.05
    fl[0, 0] = O.NO_SIGNAL
    dx[0, 0] = dy[0, 0] = np.nan
    odx, _, ofl, s = O.validate(dx, dy, ppr, fl)
    assert (s["low_ppr"], s["no_signal"], s["median_outliers"]) == (1, 1, 0)
    assert ofl[4, 4] == O.LOW_PPR | O.REPLACED
    assert ofl[0, 0] == O.NO_SIGNAL and np.isnan(odx[0, 0])


def test_out_of_range_vectors_are_flagged_and_replaced():
    dx, dy, ppr, fl = _uniform_field(1.0, 0.5)
    dx[3, 3] = 40.0
    odx, _, ofl, s = O.validate(dx, dy, ppr, fl, max_displacement=32.0)
    assert s["out_of_range"] == 1
    assert ofl[3, 3] & O.OUT_OF_RANGE and ofl[3, 3] & O.REPLACED
    assert odx[3, 3] == 1.0


# ------------------------------------------------------------------ preprocess.rs:223-270
def test_integral_stats_match_direct():
    f = np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0], [7.0, 8.0, 10.0]], np.float32)
    m, s = O.box_stats(f, 1, 1, 2, 2)
    assert abs(m - 7.25) < 1e-6
    var = np.mean((np.array([5.0, 6.0, 8.0, 10.0], np.float32) - 7.25) ** 2)
    assert abs(s - np.sqrt(var)) < 1e-5


def test_blur_preserves_constant_and_mass():
    b = O.gaussian_blur(np.full((20, 30), 0.5, np.float32), 1.5)
    assert np.all(np.abs(b - 0.5) < 1e-6)
    d = np.zeros((21, 21), np.float32)
    d[10, 10] = 1.0
    b = O.gaussian_blur(d, 1.0)
    assert abs(b.sum() - 1.0) < 1e-5
    assert b[10, 10] > b[10, 11] > b[10, 12]


def test_normalize_removes_gradient():
    f = np.fromfunction(lambda y, x: 0.01 * x + 0.002 * y, (40, 40)).astype(np.float32)
    n = O.local_normalize(f, 5, 0.0)
    assert abs(n[20, 20]) < 1e-3


def test_background_min_and_mean():
    a = np.array([[1.0, 4.0]], np.float32)
    b = np.array([[3.0, 2.0]], np.float32)
    assert np.array_equal(O.background(np.stack([a, b]), "min"), [[1.0, 2.0]])
    assert np.array_equal(O.background(np.stack([a, b]), "mean"), [[2.0, 3.0]])


# ------------------------------------------------------------------ synthetic.rs:10-36
def test_splitmix_matches_the_restatement():
    import ctypes
    st = ctypes.c_uint64(12345)
    r = S.Rng(12345)
    for _ in range(100):
        assert O.lib().orc_splitmix_next(ctypes.byref(st)) == r.next_u64()
    r2 = S.Rng(99)
    u = r2.uniforms(1000)
    r3 = S.Rng(99)
    assert np.array_equal(u, np.array([r3.uniform() for _ in range(1000)], np.float32))


def test_percentile_clip_definition():
    codes = np.arange(1, 101, dtype=np.uint16)[::-1].copy()
    c, clip = O.percentile_clip_u16(codes, 99.0)
    assert clip == 99 and c.max() == 99
    c, clip = O.percentile_clip_u16(codes, 100.0)
    assert clip == 100


def test_replacement_median_orders_signed_zeros_as_total_cmp():
    """validate.rs:164 sorts neighbours with f32::total_cmp, which puts -0.0 before +0.0. Seven
    usable neighbours [+0, -0, +0, -0, -0, 1, 2] sort to [-0, -0, -0, +0, +0, 1, 2]: the
    replacement of the centre is the fourth, +0.0 (a stable sort that treats the zeros as equal
    would keep the input order and give -0.0)."""
    from oracle import oracle as O
    dx = np.zeros((3, 3), np.float32)
    nb = [0.0, -0.0, 0.0, -0.0, -0.0, 1.0, 2.0, 7.0]
    k = 0
    for y in range(3):
        for x in range(3):
            if (x, y) != (1, 1):
                dx[y, x] = nb[k]
                k += 1
    dx[1, 1] = 50.0
    dy = np.zeros_like(dx)
    ppr = np.full_like(dx, 5.0)
    ppr[1, 1] = 1.0   # LOW_PPR: the centre is replaced
    ppr[2, 2] = 1.0   # the neighbour holding 7.0 is not usable either
    fl = np.zeros((3, 3), np.uint8)
    odx, _, ofl, _ = O.validate(dx, dy, ppr, fl)
    assert ofl[1, 1] & 8  # REPLACED
    assert odx[1, 1] == 0.0 and not np.signbit(odx[1, 1])
