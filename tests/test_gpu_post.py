"""Post-processing kernels against the oracle: flow statistics (vorticity field bit-exact, counts
exact, f64-summed means to f32 rounding), temporal and spatial smoothing bit-exact (same f32
operation order, no FMA)."""
import numpy as np
import pytest

from conftest import same_floats
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda")


def _analysed_field():
    import piv_b200 as P
    from piv_b200 import synthetic as S
    h = 384
    f = S.vortex_shear_field(h, h, vmax=6.0, shear=0.01)
    a, b = S.baseline_pair(h, h, 5, f, ppp=0.05, dmin=2.0, dmax=4.0, bits=12)
    an = P.PivAnalyzer(P.PivConfig(windows=[64, 32, 16], overlap=0.5, final_iterations=1))
    r = an.analyze(an.prepare(a, P.RAW), an.prepare(b, P.RAW))
    return r.field


def _close(g, o):
    for k in ("n_usable", "n_vorticity"):
        assert getattr(g, k) == o[k], k
    for k in ("vorticity_mean", "vorticity_abs_mean", "ke_mean", "ke_sum", "coverage"):
        a, b = getattr(g, k), o[k]
        assert (np.isnan(a) and np.isnan(b)) or abs(a - b) <= 1e-6 * max(abs(b), 1e-30), (k, a, b)


def test_flow_stats_of_an_analysed_field():
    import torch

    from piv_b200 import post
    fld = _analysed_field()
    fl = fld.flags.copy()
    fl[3, 3] |= 2          # a rejected vector
    fl[4, 4] = 2 | 8       # a replaced one (usable)
    d = [_dev(x) for x in (fld.dx, fld.dy, fl)]
    w = torch.empty(fld.dx.shape, device="cuda")
    g = post.flow_stats(*d, fld.grid.step, 0.002, vorticity=w)
    torch.cuda.synchronize()
    o = O.pair_stats(fld.dx, fld.dy, fl, fld.grid.step, 0.002)
    _close(g, o)
    k = np.float32(1 / 0.002)
    ok = O.usable(fld.dx, fl)
    ow = O.vorticity(fld.dx * k, fld.dy * k, ok, np.float32(fld.grid.step))
    assert same_floats(w.cpu().numpy(), ow)


@pytest.mark.parametrize("case", ["rotation", "translation", "holes", "empty"])
def test_flow_stats_reference_cases(case):
    from piv_b200 import post
    n, step = 21, 16
    ys, xs = np.meshgrid(np.arange(n, dtype=np.float32) * step, np.arange(n, dtype=np.float32) * step, indexing="ij")
    fl = np.zeros((n, n), np.uint8)
    if case == "rotation":
        c = np.float32((n - 1) * step / 2)
        u, v = 3 * (ys - c), -3 * (xs - c)
    elif case == "translation":
        u, v = np.full((n, n), 3.0, np.float32), np.full((n, n), -4.0, np.float32)
    elif case == "holes":
        u, v = ys * np.float32(0.1), xs * np.float32(0.2)
        fl[5, 5] = 1
        u = u.copy()
        u[5, 5] = np.nan
    else:
        u, v = np.ones((n, n), np.float32), np.ones((n, n), np.float32)
        fl[:] = 1
    u, v = u.astype(np.float32), v.astype(np.float32)
    g = post.flow_stats(_dev(u), _dev(v), _dev(fl), step, 1.0)
    _close(g, O.pair_stats(u, v, fl, step, 1.0))
    if case == "rotation":
        assert abs(g.vorticity_mean - 6.0) <= 1e-4


def _series(nt, ny, nx, seed):
    rng = np.random.default_rng(seed)
    dx = (2 + rng.normal(0, 0.5, (nt, ny, nx))).astype(np.float32)
    dy = (-1 + rng.normal(0, 0.5, (nt, ny, nx))).astype(np.float32)
    ok = rng.random((nt, ny, nx)) > 0.1
    gate = rng.random((nt, ny, nx)) > 0.05
    dx[~ok & (rng.random((nt, ny, nx)) > 0.5)] = np.nan
    return dx, dy, ok, gate


@pytest.mark.parametrize("median,window,min_support,leave_out", [(False, 9, 1, ()), (True, 7, 1, ()),
                                                                 (False, 5, 4, ()), (False, 11, 1, (0, 5, -5)),
                                                                 (True, 3, 1, (0, 1, -1))])
def test_temporal_matches_oracle(median, window, min_support, leave_out):
    import torch

    from piv_b200 import post
    dx, dy, ok, gate = _series(40, 12, 16, window)
    ox, oy, osup = O.temporal(dx, dy, ok, gate, median, window, min_support, list(leave_out))
    d = [_dev(x) for x in (dx, dy, ok.astype(np.uint8), gate.astype(np.uint8))]
    gx, gy = torch.empty_like(d[0]), torch.empty_like(d[1])
    gs = torch.empty(dx.shape, dtype=torch.int16, device="cuda")
    post.temporal_smooth(*d, gx, gy, gs, "median" if median else "mean", window, min_support, leave_out)
    torch.cuda.synchronize()
    assert same_floats(gx.cpu().numpy(), ox) and same_floats(gy.cpu().numpy(), oy)
    assert np.array_equal(gs.cpu().numpy().view(np.uint16), osup)


@pytest.mark.parametrize("sigma,min_weight,leave_out", [(1.0, 0.25, None), (1.5, 0.25, None), (1.5, 0.0, 1),
                                                        (0.5, 0.0, 1), (3.0, 0.5, 2)])
def test_spatial_matches_oracle(sigma, min_weight, leave_out):
    import torch

    from piv_b200 import post
    dx, dy, _, gate = _series(3, 24, 20, 7)
    ox, oy, osup = O.spatial(dx, dy, gate, sigma, min_weight, leave_out)
    d = [_dev(x) for x in (dx, dy, gate.astype(np.uint8))]
    gx, gy = torch.empty_like(d[0]), torch.empty_like(d[1])
    gs = torch.empty(dx.shape, dtype=torch.int16, device="cuda")
    post.spatial_smooth(*d, gx, gy, gs, sigma, min_weight, leave_out)
    torch.cuda.synchronize()
    assert same_floats(gx.cpu().numpy(), ox) and same_floats(gy.cpu().numpy(), oy)
    assert np.array_equal(gs.cpu().numpy().view(np.uint16), osup)
