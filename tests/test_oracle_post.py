"""The oracle's post-processing restatements against the reference's own unit tests:
flowstats.rs:150-265 (vorticity sign, uniform translation, shear, cancelling vortices, holes and
edges, empty field) and smooth.rs:327-520 (temporal mean/median, gate and min_support, spatial
normalized convolution, leave-out)."""
import math

import numpy as np

from oracle import oracle as O
from piv_b200.synthetic import Rng

N, STEP = 21, 16.0


def _field(f):
    ys, xs = np.meshgrid(np.arange(N, dtype=np.float32) * STEP, np.arange(N, dtype=np.float32) * STEP, indexing="ij")
    u, v = f(xs, ys)
    u = np.broadcast_to(np.asarray(u, np.float32), (N, N)).copy()
    v = np.broadcast_to(np.asarray(v, np.float32), (N, N)).copy()
    return u, v, np.ones((N, N), bool)


def test_solid_body_rotation_counter_clockwise_on_screen_is_positive():
    om = np.float32(3.0)
    c = np.float32((N - 1) * STEP / 2.0)
    u, v, ok = _field(lambda x, y: (om * (y - c), -om * (x - c)))
    w = O.vorticity(u, v, ok, STEP)
    assert np.all(np.abs(w - 2 * om) <= 1e-4)
    s = O.flow_stats(u, v, ok, STEP)
    assert abs(s["vorticity_mean"] - 6.0) <= 1e-4 and abs(s["vorticity_abs_mean"] - 6.0) <= 1e-4
    assert s["n_vorticity"] == N * N


def test_uniform_translation():
    u, v, ok = _field(lambda x, y: (3.0, -4.0))
    s = O.flow_stats(u, v, ok, STEP)
    assert s["vorticity_mean"] == 0.0 and s["vorticity_abs_mean"] == 0.0
    assert abs(s["ke_mean"] - 12.5) <= 1e-5
    assert abs(s["ke_sum"] - 12.5 * N * N * STEP * STEP) <= 1.0
    assert s["coverage"] == 1.0


def test_shear():
    u, v, ok = _field(lambda x, y: (np.float32(0.5) * y, 0.0))
    assert abs(O.flow_stats(u, v, ok, STEP)["vorticity_mean"] - 0.5) <= 1e-5


def test_opposite_vortices_cancel_in_the_signed_mean():
    length = N * STEP
    u, v, ok = _field(lambda x, y: (0.0, np.sin(np.float32(2 * math.pi) * x / np.float32(length)) * 10.0))
    s = O.flow_stats(u, v, ok, STEP)
    assert abs(s["vorticity_mean"]) < 0.1 * s["vorticity_abs_mean"]
    assert abs(s["vorticity_abs_mean"] - 40.0 / length) <= 0.1 * 40.0 / length


def test_holes_and_edges():
    u, v, ok = _field(lambda x, y: (y * np.float32(0.1), x * np.float32(0.2)))
    ok[5, 5] = False
    w = O.vorticity(u, v, ok, STEP)
    assert np.isnan(w[5, 5])
    for p in [(4, 5), (6, 5), (5, 4), (5, 6), (0, 0), (N - 1, N - 1)]:
        assert abs(w[p] + 0.1) <= 1e-5, p
    lonely = np.zeros((N, N), bool)
    lonely[3, 3] = True
    s = O.flow_stats(u, v, lonely, STEP)
    assert s["n_vorticity"] == 0 and math.isnan(s["vorticity_mean"]) and s["n_usable"] == 1
    un = u.copy()
    un[0, 0] = np.nan
    assert O.flow_stats(un, v, ok, STEP)["n_usable"] == N * N - 2


def test_empty_field():
    u, v, _ = _field(lambda x, y: (1.0, 1.0))
    s = O.flow_stats(u, v, np.zeros((N, N), bool), STEP)
    assert math.isnan(s["ke_mean"]) and math.isnan(s["vorticity_mean"])
    assert (s["ke_sum"], s["coverage"], s["n_usable"]) == (0.0, 0.0, 0)


def test_usable_and_pair_stats_scale_to_px_per_s():
    dx = np.full((4, 5), 1.5, np.float32)
    dy = np.zeros((4, 5), np.float32)
    fl = np.zeros((4, 5), np.uint8)
    fl[0, 0] = 1        # NO_SIGNAL
    fl[0, 1] = 2        # LOW_PPR
    fl[0, 2] = 2 | 8    # LOW_PPR but REPLACED: usable
    dx[1, 1] = np.nan
    ok = O.usable(dx, fl)
    assert not ok[0, 0] and not ok[0, 1] and ok[0, 2] and not ok[1, 1] and ok.sum() == 17
    s = O.pair_stats(dx, dy, fl, 16, 0.002)
    assert s["n_usable"] == 17 and abs(s["ke_mean"] - 0.5 * 750.0 ** 2) < 1e-2


# ------------------------------------------------------------------------------------- smoothing
def _series(nt, noise):
    ny, nx = 12, 16
    t, y, x = np.meshgrid(np.arange(nt, dtype=np.float32), np.arange(ny, dtype=np.float32),
                          np.arange(nx, dtype=np.float32), indexing="ij")
    tu = (2.0 + 0.01 * t + 0.05 * y).astype(np.float32)
    tv = (-1.0 + 0.02 * x - 0.005 * t).astype(np.float32)
    rng = Rng(1)
    du = (tu + np.float32(noise) * rng.normals(tu.size).reshape(tu.shape)).astype(np.float32)
    dv = (tv + np.float32(noise) * rng.normals(tv.size).reshape(tv.shape)).astype(np.float32)
    return du, dv, tu, tv, np.ones(tu.shape, bool)


def _rms(a, b):
    m = np.isfinite(a)
    return float(np.sqrt(np.mean((a[m] - b[m]) ** 2)))


def test_temporal_mean_reduces_noise_by_sqrt_window():
    du, dv, tu, _, ok = _series(60, 0.5)
    sx, sy, sup = O.temporal(du, dv, ok, ok, False, 9, 1)
    assert _rms(sx, tu) < _rms(du, tu) / 2.5
    assert sup[30, 5, 5] == 9 and sup[0, 5, 5] == 5


def test_temporal_median_rejects_outliers_and_respects_usable():
    du, dv, tu, _, ok = _series(30, 0.0)
    du[10, 3, 3] = 50.0
    du[11, 3, 3] = -50.0
    ok[12, 3, 3] = False
    du[12, 3, 3] = 1e6
    sx, sy, sup = O.temporal(du, dv, ok, np.ones_like(ok), True, 7, 1)
    assert abs(sx[11, 3, 3] - tu[11, 3, 3]) < 0.05
    assert abs(sx[12, 3, 3] - tu[12, 3, 3]) < 0.05
    assert sup[12, 3, 3] == 6


def test_gate_and_min_support_control_output():
    du, dv, _, _, ok = _series(20, 0.1)
    gate = ok.copy()
    gate[5, 0, 0] = False
    sx, _, _ = O.temporal(du, dv, ok, gate, False, 5, 4)
    assert np.isnan(sx[5, 0, 0]) and np.isnan(sx[0, 1, 1]) and np.isfinite(sx[1, 1, 1])


def test_spatial_smooths_noise_preserves_linear_fields_and_skips_nan():
    du, dv, tu, tv, ok = _series(3, 0.0)
    ox, oy, _ = O.spatial(du, dv, ok, 1.0, 0.25)
    assert abs(ox[1, 6, 8] - tu[1, 6, 8]) < 1e-4 and abs(oy[1, 6, 8] - tv[1, 6, 8]) < 1e-4
    du[1, 6, 9] = np.nan
    ox, _, sup = O.spatial(du, dv, ok, 1.0, 0.25)
    assert np.isfinite(ox[1, 6, 8]) and sup[1, 6, 8] == 48
    nu, nv, tu, _, ok = _series(3, 0.5)
    ox, _, _ = O.spatial(nu, nv, ok, 1.5, 0.25)
    assert _rms(ox, tu) < _rms(nu, tu) / 2.0


def test_leave_out_skips_the_requested_samples():
    du, dv, _, _, ok = _series(20, 0.0)
    du[10, 4, 4] = 100.0
    du[15, 4, 4] = 100.0
    sx, _, sup = O.temporal(du, dv, ok, ok, False, 11, 1, [0, 5, -5])
    assert sx[10, 4, 4] < 3.0 and sup[10, 4, 4] == 10
    sx, _, sup = O.temporal(du, dv, ok, ok, False, 3, 1, [0, 1, -1])
    assert sup[10, 4, 4] == 2 and np.isfinite(sx[10, 4, 4])
    du, dv, _, _, ok = _series(1, 0.0)
    du[0, 6, 7] = 100.0
    ox, _, _ = O.spatial(du, dv, ok, 1.5, 0.0, 1)
    assert ox[0, 6, 8] < 3.0
    ox, _, _ = O.spatial(du, dv, ok, 0.5, 0.0, 1)
    assert np.all(np.isnan(ox))
