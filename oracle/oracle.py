"""ctypes wrapper of the CPU oracle (oracle/piv_oracle.cpp) — TEST INFRASTRUCTURE ONLY.

A restatement of the reference's `piv-core` algorithms used to check the CUDA path. Only the
tests, the smoke check and the benchmark's CPU-baseline leg import this module; the product
package (piv_b200) never does.
"""
import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import build_oracle

REF, FP64 = 0, 1
NO_SIGNAL, LOW_PPR, MEDIAN_OUTLIER, REPLACED, OUT_OF_RANGE = 1, 2, 4, 8, 16

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_u16p = np.ctypeslib.ndpointer(dtype=np.uint16, flags="C_CONTIGUOUS")
_i64 = ctypes.c_int64


class OrcGrid(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("window", "step", "nx", "ny", "x0", "y0")]


class OrcSummary(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in ("no_signal", "low_ppr", "median_outliers", "out_of_range", "replaced")]

    def as_dict(self):
        return {n: getattr(self, n) for n, _ in self._fields_}


class OrcConfig(ctypes.Structure):
    _fields_ = [
        ("windows", ctypes.POINTER(ctypes.c_int32)),
        ("n_windows", ctypes.c_int32),
        ("overlap", ctypes.c_float),
        ("final_iterations", ctypes.c_int32),
        ("min_mean", ctypes.c_float),
        ("min_std", ctypes.c_float),
        ("ppr_threshold", ctypes.c_float),
        ("median_threshold", ctypes.c_float),
        ("median_eps", ctypes.c_float),
        ("replace", ctypes.c_int32),
        ("deform", ctypes.c_int32),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.OUT
        if not os.path.exists(path):
            path = build_oracle.build()
        L = ctypes.CDLL(path)
        L.orc_grid.argtypes = [_i64, _i64, _i64, ctypes.c_float, ctypes.POINTER(OrcGrid)]
        L.orc_grid.restype = ctypes.c_int
        L.orc_u16_to_f32.argtypes = [_u16p, _i64, _f32p]
        L.orc_u8_to_f32.argtypes = [_u8p, _i64, _f32p]
        L.orc_percentile_clip_u16.argtypes = [_u16p, _i64, ctypes.c_double]
        L.orc_percentile_clip_u16.restype = ctypes.c_int64
        L.orc_background.argtypes = [_f32p, _i64, _i64, ctypes.c_int, _f32p]
        L.orc_prepare.argtypes = [_f32p, ctypes.c_void_p, _i64, _i64, ctypes.c_float, _i64, ctypes.c_float, _f32p, ctypes.c_void_p]
        L.orc_gaussian_blur.argtypes = [_f32p, _i64, _i64, ctypes.c_float, _f32p]
        L.orc_local_normalize.argtypes = [_f32p, _i64, _i64, _i64, ctypes.c_float, _f32p]
        L.orc_box_stats.argtypes = [_f32p, _i64, _i64, _i64, _i64, _i64, _i64, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
        L.orc_place.argtypes = [ctypes.POINTER(OrcGrid), _i64, _i64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, _f32p]
        L.orc_correlate_pass.argtypes = [_f32p, _f32p, _f32p, _f32p, _i64, _i64, _i64, _i64, _f32p, ctypes.c_float,
                                         ctypes.c_float, ctypes.c_int, ctypes.c_int, _f32p, _f32p, _f32p, _u8p]
        L.orc_correlate_window.argtypes = [_f32p, _i64, _i64, ctypes.c_float, ctypes.c_float, _f32p, _i64, _i64,
                                           ctypes.c_float, ctypes.c_float, _i64, ctypes.c_int, _f32p]
        L.orc_correlate_window.restype = ctypes.c_int
        L.orc_correlation_plane.argtypes = L.orc_correlate_window.argtypes
        L.orc_correlation_plane.restype = ctypes.c_int
        L.orc_load_window.argtypes = [_f32p, _i64, _i64, ctypes.c_float, ctypes.c_float, _i64, _f32p]
        L.orc_load_window.restype = ctypes.c_double
        L.orc_find_peak.argtypes = [_f32p, _i64, _f32p]
        L.orc_validate.argtypes = [_f32p, _f32p, _f32p, _u8p, _i64, _i64, ctypes.c_float, ctypes.c_float,
                                   ctypes.c_float, ctypes.c_int, ctypes.c_float, ctypes.POINTER(OrcSummary)]
        L.orc_check_config.argtypes = [ctypes.POINTER(OrcConfig)]
        L.orc_num_passes.argtypes = [ctypes.POINTER(OrcConfig)]
        vp = ctypes.c_void_p
        L.orc_analyze.argtypes = [ctypes.POINTER(OrcConfig), _f32p, _f32p, _f32p, _f32p, _i64, _i64, ctypes.c_int,
                                  ctypes.c_int, _f32p, _f32p, _f32p, _u8p, ctypes.POINTER(OrcSummary)] + [vp] * 9
        L.orc_analyze.restype = ctypes.c_int
        L.orc_place_deform.argtypes = [ctypes.POINTER(OrcGrid), _i64, _i64, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, _f32p, _f32p]
        L.orc_correlate_pass_deform.argtypes = [_f32p, _f32p, _f32p, _f32p, _i64, _i64, ctypes.POINTER(OrcGrid), _f32p,
                                                _f32p, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int, _f32p,
                                                _f32p, _f32p, _u8p]
        L.orc_usable.argtypes = [_f32p, _u8p, _i64, _u8p]
        L.orc_vorticity.argtypes = [_f32p, _f32p, _u8p, _i64, _i64, ctypes.c_float, _f32p]
        L.orc_flow_stats.argtypes = [_f32p, _f32p, _u8p, _i64, _i64, ctypes.c_float, ctypes.POINTER(OrcFlowStats)]
        L.orc_pair_stats.argtypes = [_f32p, _f32p, _u8p, _i64, _i64, _i64, ctypes.c_double, ctypes.POINTER(OrcFlowStats)]
        L.orc_temporal.argtypes = [_f32p, _f32p, _u8p, _u8p, _i64, _i64, _i64, ctypes.c_int32, ctypes.c_int32,
                                   ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, _f32p, _f32p, ctypes.c_void_p]
        L.orc_spatial.argtypes = [_f32p, _f32p, _u8p, _i64, _i64, _i64, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                  _f32p, _f32p, ctypes.c_void_p]
        L.orc_splitmix_next.argtypes = [ctypes.POINTER(ctypes.c_uint64)]
        L.orc_splitmix_next.restype = ctypes.c_uint64
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def grid(h, w, window, overlap):
    g = OrcGrid()
    st = lib().orc_grid(h, w, window, ctypes.c_float(overlap), ctypes.byref(g))
    if st:
        raise ValueError(f"grid error {st}")
    return g


def u16_to_f32(codes):
    codes = np.ascontiguousarray(codes, dtype=np.uint16)
    out = np.empty(codes.shape, np.float32)
    lib().orc_u16_to_f32(codes.ravel(), codes.size, out.reshape(-1))
    return out


def u8_to_f32(codes):
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    out = np.empty(codes.shape, np.float32)
    lib().orc_u8_to_f32(codes.ravel(), codes.size, out.reshape(-1))
    return out


def percentile_clip_u16(codes, percentile):
    c = np.array(codes, dtype=np.uint16, order="C", copy=True)
    clip = lib().orc_percentile_clip_u16(c.reshape(-1), c.size, percentile)
    return c, clip


def background(frames, mode="min"):
    frames = _f(frames)
    out = np.empty(frames.shape[1:], np.float32)
    lib().orc_background(frames.reshape(-1), frames.shape[0], out.size, 0 if mode == "min" else 1, out.reshape(-1))
    return out


def prepare(raw, smooth_sigma=1.0, normalize_radius=4, normalize_eps=0.02, background=None):
    """PreparedFrame::new (preprocess.rs:138-158). Returns (image, base)."""
    raw = _f(raw)
    h, w = raw.shape
    img = np.empty_like(raw)
    base = np.empty_like(raw)
    bg = None if background is None else _f(background)
    lib().orc_prepare(raw, _ptr(bg), h, w, smooth_sigma, normalize_radius, normalize_eps, img, _ptr(base))
    return img, base


def gaussian_blur(src, sigma):
    src = _f(src)
    out = np.empty_like(src)
    lib().orc_gaussian_blur(src, src.shape[0], src.shape[1], sigma, out)
    return out


def local_normalize(src, radius, eps):
    src = _f(src)
    out = np.empty_like(src)
    lib().orc_local_normalize(src, src.shape[0], src.shape[1], radius, eps, out)
    return out


def box_stats(frame, x, y, bw, bh):
    frame = _f(frame)
    m, s = ctypes.c_float(), ctypes.c_float()
    lib().orc_box_stats(frame, frame.shape[0], frame.shape[1], x, y, bw, bh, ctypes.byref(m), ctypes.byref(s))
    return m.value, s.value


def place(g, h, w, pgrid=None, pdx=None, pdy=None):
    out = np.empty((g.ny * g.nx, 4), np.float32)
    pdx = None if pdx is None else _f(pdx)
    pdy = None if pdy is None else _f(pdy)
    lib().orc_place(ctypes.byref(g), h, w, ctypes.byref(pgrid) if pgrid is not None else None, _ptr(pdx), _ptr(pdy), out)
    return out


def correlate_pass(image_a, image_b, base_a, base_b, n, origins, min_mean=0.0, min_std=0.0, mode=REF, nthreads=0):
    image_a, image_b, base_a, base_b = map(_f, (image_a, image_b, base_a, base_b))
    origins = _f(origins)
    cells = origins.shape[0]
    dx, dy, ppr = (np.empty(cells, np.float32) for _ in range(3))
    flags = np.empty(cells, np.uint8)
    h, w = image_a.shape
    lib().orc_correlate_pass(image_a, image_b, base_a, base_b, h, w, n, cells, origins, min_mean, min_std, mode,
                             nthreads, dx, dy, ppr, flags)
    return dx, dy, ppr, flags


def place_deform(g, h, w, pgrid=None, pdx=None, pdy=None):
    """Origins and the predictor at each window's four corner pixels (deformed windows)."""
    out = np.empty((g.ny * g.nx, 4), np.float32)
    corners = np.empty((g.ny * g.nx, 8), np.float32)
    pdx = None if pdx is None else _f(pdx)
    pdy = None if pdy is None else _f(pdy)
    lib().orc_place_deform(ctypes.byref(g), h, w, ctypes.byref(pgrid) if pgrid is not None else None, _ptr(pdx),
                           _ptr(pdy), out, corners)
    return out, corners


def correlate_pass_deform(image_a, image_b, base_a, base_b, g, origins, corners, min_mean=0.0, min_std=0.0, mode=REF,
                          nthreads=0):
    image_a, image_b, base_a, base_b = map(_f, (image_a, image_b, base_a, base_b))
    origins, corners = _f(origins), _f(corners)
    cells = g.nx * g.ny
    dx, dy, ppr = (np.empty(cells, np.float32) for _ in range(3))
    flags = np.empty(cells, np.uint8)
    h, w = image_a.shape
    lib().orc_correlate_pass_deform(image_a, image_b, base_a, base_b, h, w, ctypes.byref(g), origins, corners, min_mean,
                                    min_std, mode, nthreads, dx, dy, ppr, flags)
    return dx, dy, ppr, flags


def correlate_window(a, ax, ay, b, bx, by, n, mode=REF):
    a, b = _f(a), _f(b)
    pk = np.empty(4, np.float32)
    ok = lib().orc_correlate_window(a, a.shape[0], a.shape[1], ax, ay, b, b.shape[0], b.shape[1], bx, by, n, mode, pk)
    return tuple(float(v) for v in pk) if ok else None


def correlation_plane(a, ax, ay, b, bx, by, n, mode=REF):
    a, b = _f(a), _f(b)
    pl = np.empty((n, n), np.float32)
    ok = lib().orc_correlation_plane(a, a.shape[0], a.shape[1], ax, ay, b, b.shape[0], b.shape[1], bx, by, n, mode, pl)
    return pl if ok else None


def load_window(img, x, y, n):
    img = _f(img)
    dst = np.empty((n, n), np.float32)
    e = lib().orc_load_window(img, img.shape[0], img.shape[1], x, y, n, dst)
    return dst, e


def find_peak(corr):
    corr = _f(corr)
    pk = np.empty(4, np.float32)
    lib().orc_find_peak(corr, corr.shape[0], pk)
    return tuple(float(v) for v in pk)


def validate(dx, dy, ppr, flags, ppr_threshold=1.3, median_threshold=2.0, median_eps=0.1, replace=True,
             max_displacement=float("inf")):
    dx, dy, ppr = (np.array(a, dtype=np.float32, order="C", copy=True) for a in (dx, dy, ppr))
    flags = np.array(flags, dtype=np.uint8, order="C", copy=True)
    ny, nx = dx.shape
    s = OrcSummary()
    lib().orc_validate(dx, dy, ppr, flags, ny, nx, ppr_threshold, median_threshold, median_eps, int(bool(replace)),
                       max_displacement, ctypes.byref(s))
    return dx, dy, flags, s.as_dict()


@dataclass
class OracleConfig:
    windows: tuple = (96, 64)
    overlap: float = 0.5
    final_iterations: int = 2
    min_mean: float = 0.0
    min_std: float = 0.0
    ppr_threshold: float = 1.3
    median_threshold: float = 2.0
    median_eps: float = 0.1
    replace: bool = True
    deform: bool = False

    def c(self):
        self._w = (ctypes.c_int32 * len(self.windows))(*self.windows)
        return OrcConfig(self._w, len(self.windows), self.overlap, self.final_iterations, self.min_mean,
                         self.min_std, self.ppr_threshold, self.median_threshold, self.median_eps,
                         int(bool(self.replace)), int(bool(self.deform)))

    def passes(self):
        return list(self.windows) + [self.windows[-1]] * (self.final_iterations - 1)


def analyze(cfg: OracleConfig, image_a, image_b, base_a=None, base_b=None, mode=REF, nthreads=0, trace=False):
    """PivAnalyzer::analyze_traced (multipass.rs:142-192) on prepared images.

    base_* default to the images (no preprocessing). Returns (final, summary, traces)."""
    image_a, image_b = _f(image_a), _f(image_b)
    base_a = image_a if base_a is None else _f(base_a)
    base_b = image_b if base_b is None else _f(base_b)
    h, w = image_a.shape
    grids = [grid(h, w, n, cfg.overlap) for n in cfg.passes()]
    g = grids[-1]
    fdx, fdy, fppr = (np.empty((g.ny, g.nx), np.float32) for _ in range(3))
    ffl = np.empty((g.ny, g.nx), np.uint8)
    s = OrcSummary()
    tot = sum(x.nx * x.ny for x in grids)
    tr = None
    if trace:
        tr = dict(origins=np.empty((tot, 4), np.float32), raw_dx=np.empty(tot, np.float32),
                  raw_dy=np.empty(tot, np.float32), raw_ppr=np.empty(tot, np.float32), raw_flags=np.empty(tot, np.uint8),
                  dx=np.empty(tot, np.float32), dy=np.empty(tot, np.float32), ppr=np.empty(tot, np.float32),
                  flags=np.empty(tot, np.uint8))
    keys = ["origins", "raw_dx", "raw_dy", "raw_ppr", "raw_flags", "dx", "dy", "ppr", "flags"]
    ptrs = [_ptr(tr[k]) if tr else None for k in keys]
    cc = cfg.c()
    st = lib().orc_analyze(ctypes.byref(cc), image_a, image_b, base_a, base_b, h, w, mode, nthreads, fdx, fdy, fppr,
                           ffl, ctypes.byref(s), *ptrs)
    if st:
        raise ValueError(f"oracle analyze error {st}")
    traces = []
    if tr:
        off = 0
        for gr in grids:
            c = gr.nx * gr.ny
            sl = slice(off, off + c)
            sh = (gr.ny, gr.nx)
            traces.append(dict(grid=gr, origins=tr["origins"][sl], raw_dx=tr["raw_dx"][sl].reshape(sh),
                               raw_dy=tr["raw_dy"][sl].reshape(sh), raw_ppr=tr["raw_ppr"][sl].reshape(sh),
                               raw_flags=tr["raw_flags"][sl].reshape(sh), dx=tr["dx"][sl].reshape(sh),
                               dy=tr["dy"][sl].reshape(sh), ppr=tr["ppr"][sl].reshape(sh),
                               flags=tr["flags"][sl].reshape(sh)))
            off += c
    return dict(dx=fdx, dy=fdy, ppr=fppr, flags=ffl), s.as_dict(), traces


# --------------------------------------------------------------------------------- post-processing
class OrcFlowStats(ctypes.Structure):
    _fields_ = [("vorticity_mean", ctypes.c_float), ("vorticity_abs_mean", ctypes.c_float), ("ke_mean", ctypes.c_float),
                ("ke_sum", ctypes.c_float), ("coverage", ctypes.c_float), ("n_usable", ctypes.c_int64),
                ("n_vorticity", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _b(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


def usable(dx, flags):
    dx, flags = _f(dx), _b(flags)
    out = np.empty(dx.shape, np.uint8)
    lib().orc_usable(dx.ravel(), flags.ravel(), dx.size, out.reshape(-1))
    return out.astype(bool)


def vorticity(u, v, ok, step):
    u, v = _f(u), _f(v)
    out = np.empty(u.shape, np.float32)
    lib().orc_vorticity(u, v, _b(ok), u.shape[0], u.shape[1], step, out)
    return out


def flow_stats(u, v, ok, step):
    u, v = _f(u), _f(v)
    s = OrcFlowStats()
    lib().orc_flow_stats(u, v, _b(ok), u.shape[0], u.shape[1], step, ctypes.byref(s))
    return s.as_dict()


def pair_stats(dx, dy, flags, step, dt_s):
    dx, dy = _f(dx), _f(dy)
    s = OrcFlowStats()
    lib().orc_pair_stats(dx, dy, _b(flags), dx.shape[0], dx.shape[1], int(step), float(dt_s), ctypes.byref(s))
    return s.as_dict()


def temporal(dx, dy, ok, gate, median, window, min_support, leave_out=()):
    dx, dy = _f(dx), _f(dy)
    nt, ny, nx = dx.shape
    lo = np.ascontiguousarray(leave_out, np.int32)
    ox, oy = np.empty_like(dx), np.empty_like(dy)
    sup = np.empty(dx.shape, np.uint16)
    lib().orc_temporal(dx, dy, _b(ok), _b(gate), nt, ny, nx, int(bool(median)), int(window), int(min_support),
                       _ptr(lo) if lo.size else None, int(lo.size), ox, oy, _ptr(sup))
    return ox, oy, sup


def spatial(dx, dy, gate, sigma, min_weight, leave_out=None):
    dx, dy = _f(dx), _f(dy)
    nt, ny, nx = dx.shape
    ox, oy = np.empty_like(dx), np.empty_like(dy)
    sup = np.empty(dx.shape, np.uint16)
    lib().orc_spatial(dx, dy, _b(gate), nt, ny, nx, float(sigma), float(min_weight),
                      -1 if leave_out is None else int(leave_out), ox, oy, _ptr(sup))
    return ox, oy, sup
