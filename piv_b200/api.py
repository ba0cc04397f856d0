"""Host-side mirror of the reference's `piv-core` interface over the CUDA path.

Names, argument meaning, defaults and errors follow the reference:
  PivConfig / MaskConfig        rust/crates/piv-core/src/multipass.rs:20-63
  ValidationConfig              rust/crates/piv-core/src/validate.rs:7-37
  PreprocessConfig              rust/crates/piv-core/src/preprocess.rs:5-29
  Grid                          rust/crates/piv-core/src/grid.rs:5-75
  VectorField, flags            rust/crates/piv-core/src/field.rs:5-95
  PivError                      rust/crates/piv-core/src/error.rs:4-19
  PivAnalyzer::{new, output_grid, analyze, analyze_traced}  multipass.rs:91-150
  PreparedFrame::new            preprocess.rs:138-158

Every computation runs in libpivb200.so on the GPU; this module only marshals arguments.
"""
import ctypes
from dataclasses import dataclass, field as dc_field
from typing import List, Optional, Tuple

import numpy as np

from . import _lib


# --------------------------------------------------------------------------------- errors
class PivError(Exception):
    """PivError (error.rs:4-19)."""


class ConfigError(PivError):
    pass


class ShapeMismatchError(PivError):
    pass


class ImageTooSmallError(PivError):
    pass


class CudaError(PivError):
    pass


class UnsupportedError(PivError):
    pass


class CancelledError(PivError):
    """The serving form's request was cancelled (no counterpart in the reference)."""


class TimeoutError(PivError):  # noqa: A001 - the library's status, not the builtin
    """A bounded wait of the serving form ran out; the request is still pending."""


def _check(status):
    if status == _lib.PIV_OK:
        return
    msg = _lib.last_error()
    cls = {
        _lib.PIV_ERR_CONFIG: ConfigError,
        _lib.PIV_ERR_SHAPE_MISMATCH: ShapeMismatchError,
        _lib.PIV_ERR_IMAGE_TOO_SMALL: ImageTooSmallError,
        _lib.PIV_ERR_CUDA: CudaError,
        _lib.PIV_ERR_UNSUPPORTED: UnsupportedError,
        _lib.PIV_ERR_CANCELLED: CancelledError,
        _lib.PIV_ERR_TIMEOUT: TimeoutError,
    }.get(status, PivError)
    raise cls(msg)


# --------------------------------------------------------------------------------- flags
class flags:  # noqa: N801 - mirrors the reference's `flags` module (field.rs:6-20)
    NO_SIGNAL = 1 << 0
    LOW_PPR = 1 << 1
    MEDIAN_OUTLIER = 1 << 2
    REPLACED = 1 << 3
    OUT_OF_RANGE = 1 << 4
    INVALID = NO_SIGNAL | LOW_PPR | MEDIAN_OUTLIER | OUT_OF_RANGE


# --------------------------------------------------------------------------------- configs
@dataclass
class MaskConfig:
    min_mean: float = 0.0
    min_std: float = 0.0


@dataclass
class ValidationConfig:
    ppr_threshold: float = 1.3
    median_threshold: float = 2.0
    median_eps: float = 0.1
    replace: bool = True


_PRECISIONS = {"fp32": 0, "bf16x3": 1, "fp16x3": 2}


@dataclass
class PivConfig:
    windows: List[int] = dc_field(default_factory=lambda: [96, 64])
    overlap: float = 0.5
    final_iterations: int = 2
    mask: MaskConfig = dc_field(default_factory=MaskConfig)
    validation: ValidationConfig = dc_field(default_factory=ValidationConfig)
    # False: windows shift uniformly (the reference). True: from the second pass on, each window
    # is deformed by the bilinear blend of the predictor at its four corner pixels.
    deform: bool = False
    # "fp32": FFTs on the FP32 cores (the reference's precision). "bf16x3" / "fp16x3": DFTs on the
    # tensor cores with operands split into two BF16 / FP16 halves (window sizes 16 and 32,
    # uniform windows).
    precision: str = "fp32"

    def passes(self):
        return list(self.windows) + [self.windows[-1]] * (self.final_iterations - 1)

    def _c(self, device=-1):
        w = (ctypes.c_int32 * max(len(self.windows), 1))(*[int(x) for x in self.windows])
        c = _lib.PivConfigC(w, len(self.windows), float(self.overlap), int(self.final_iterations),
                            float(self.mask.min_mean), float(self.mask.min_std),
                            float(self.validation.ppr_threshold), float(self.validation.median_threshold),
                            float(self.validation.median_eps), int(bool(self.validation.replace)), int(device),
                            int(bool(self.deform)), _PRECISIONS.get(self.precision, -1))
        c._keep = w
        return c


@dataclass
class PreprocessConfig:
    """PreprocessConfig (preprocess.rs:5-29) plus `clip_percentile` (0 = off; an addition)."""
    smooth_sigma: float = 1.0
    normalize_radius: int = 4
    normalize_eps: float = 0.02
    clip_percentile: float = 0.0

    def _c(self):
        return _lib.PivPreprocessC(float(self.smooth_sigma), int(self.normalize_radius), float(self.normalize_eps),
                                   float(self.clip_percentile))


RAW = PreprocessConfig(smooth_sigma=0.0, normalize_radius=0, normalize_eps=0.0)


# --------------------------------------------------------------------------------- grid / field
@dataclass(frozen=True)
class Grid:
    window: int
    step: int
    nx: int
    ny: int
    x0: int
    y0: int

    @staticmethod
    def new(height, width, window, overlap) -> "Grid":
        g = _lib.PivGridC()
        _check(_lib.load().piv_grid(int(height), int(width), int(window), float(overlap), ctypes.byref(g)))
        return Grid._from_c(g)

    @staticmethod
    def _from_c(g):
        return Grid(g.window, g.step, g.nx, g.ny, g.x0, g.y0)

    def _c(self):
        return _lib.PivGridC(self.window, self.step, self.nx, self.ny, self.x0, self.y0)

    def __len__(self):
        return self.nx * self.ny

    def window_origin(self, ix, iy):
        return self.x0 + ix * self.step, self.y0 + iy * self.step

    def center_x(self, ix):
        return np.float32(self.x0 + ix * self.step) + (np.float32(self.window) - np.float32(1)) / np.float32(2)

    def center_y(self, iy):
        return np.float32(self.y0 + iy * self.step) + (np.float32(self.window) - np.float32(1)) / np.float32(2)

    def xs(self):
        return np.array([self.center_x(i) for i in range(self.nx)], np.float32)

    def ys(self):
        return np.array([self.center_y(i) for i in range(self.ny)], np.float32)


@dataclass
class VectorField:
    """VectorField (field.rs:26-45): [ny, nx] arrays, NaN where NO_SIGNAL."""
    grid: Grid
    dx: np.ndarray
    dy: np.ndarray
    peak_ratio: np.ndarray
    flags: np.ndarray

    def valid_count(self):
        return int(np.count_nonzero((self.flags & flags.INVALID) == 0))


@dataclass
class ValidationSummary:
    no_signal: int = 0
    low_ppr: int = 0
    median_outliers: int = 0
    out_of_range: int = 0
    replaced: int = 0

    @staticmethod
    def _from_c(s):
        return ValidationSummary(s.no_signal, s.low_ppr, s.median_outliers, s.out_of_range, s.replaced)

    def as_dict(self):
        return dict(no_signal=self.no_signal, low_ppr=self.low_ppr, median_outliers=self.median_outliers,
                    out_of_range=self.out_of_range, replaced=self.replaced)


@dataclass
class PairResult:
    field: VectorField
    summary: ValidationSummary


@dataclass
class PassTrace:
    """PassTrace (multipass.rs:72-81)."""
    origins: np.ndarray
    raw: VectorField
    validated: VectorField


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _dtype_code(a):
    if a.dtype == np.uint8:
        return _lib.PIV_DTYPE_U8
    if a.dtype == np.uint16:
        return _lib.PIV_DTYPE_U16
    if a.dtype == np.float32:
        return _lib.PIV_DTYPE_F32
    raise PivError(f"unsupported sample type {a.dtype}")


# --------------------------------------------------------------------------------- frames
class PreparedFrame:
    """A device-resident prepared frame (PreparedFrame, preprocess.rs:127-158)."""

    def __init__(self, analyzer: "PivAnalyzer", height: int, width: int):
        self.analyzer = analyzer
        self.height, self.width = int(height), int(width)
        h = ctypes.c_void_p()
        _check(_lib.load().piv_frame_create(analyzer._h, self.height, self.width, ctypes.byref(h)))
        self._h = h
        self._keep = None

    @staticmethod
    def new(raw, cfg: PreprocessConfig = None, background=None, analyzer: "PivAnalyzer" = None) -> "PreparedFrame":
        """PreparedFrame::new(raw, cfg, background) from host samples (u8, u16 or f32 in 0..1)."""
        if analyzer is None:
            raise PivError("a PreparedFrame lives on an analyzer's device: pass analyzer=")
        raw = np.ascontiguousarray(raw)
        f = PreparedFrame(analyzer, raw.shape[0], raw.shape[1])
        f.prepare(raw, cfg, background)
        return f

    def prepare(self, raw, cfg: PreprocessConfig = None, background=None):
        cfg = PreprocessConfig() if cfg is None else cfg
        raw = np.ascontiguousarray(raw)
        if raw.shape != (self.height, self.width):
            raise ShapeMismatchError(f"frame shape {raw.shape} vs {(self.height, self.width)}")
        bg = None if background is None else np.ascontiguousarray(background, dtype=np.float32)
        pc = cfg._c()
        _check(_lib.load().piv_frame_prepare(self.analyzer._h, self._h, _ptr(raw), _dtype_code(raw), ctypes.byref(pc),
                                             _ptr(bg)))
        self._keep = (raw, bg)  # host buffers stay alive until the next blocking call
        self.analyzer.sync()
        self._keep = None
        return self

    def prepare_device(self, raw_ptr: int, dtype: int, cfg: PreprocessConfig = None, background_ptr: Optional[int] = None):
        """Asynchronous preparation from device memory (e.g. a torch CUDA tensor's data_ptr())."""
        cfg = PreprocessConfig() if cfg is None else cfg
        pc = cfg._c()
        _check(_lib.load().piv_frame_prepare_device(self.analyzer._h, self._h, ctypes.c_void_p(raw_ptr), int(dtype),
                                                    ctypes.byref(pc),
                                                    None if background_ptr is None else ctypes.c_void_p(background_ptr)))
        return self

    def set_prepared(self, image, base=None):
        image = np.ascontiguousarray(image, dtype=np.float32)
        base = None if base is None else np.ascontiguousarray(base, dtype=np.float32)
        _check(_lib.load().piv_frame_set_prepared(self.analyzer._h, self._h, _ptr(image), _ptr(base)))
        return self

    def set_prepared_tables(self, image, sum_table, sumsq_table):
        """The reference's own PreparedFrame (preprocess.rs:127-135): the conditioned image and
        its IntegralImage tables ((H+1) x (W+1) f64, preprocess.rs:84-103)."""
        image = np.ascontiguousarray(image, dtype=np.float32)
        t1 = np.ascontiguousarray(sum_table, dtype=np.float64)
        t2 = np.ascontiguousarray(sumsq_table, dtype=np.float64)
        shape = (self.height + 1, self.width + 1)
        if image.shape != (self.height, self.width) or t1.shape != shape or t2.shape != shape:
            raise ShapeMismatchError(f"image {image.shape} and tables {t1.shape}, {t2.shape} for a "
                                     f"{(self.height, self.width)} frame")
        _check(_lib.load().piv_frame_set_prepared_tables(self.analyzer._h, self._h, _ptr(image), _ptr(t1), _ptr(t2)))
        return self

    @property
    def image(self) -> np.ndarray:
        out = np.empty((self.height, self.width), np.float32)
        _check(_lib.load().piv_frame_download(self.analyzer._h, self._h, _ptr(out)))
        return out

    def dim(self):
        return self.height, self.width

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().piv_frame_destroy(self._h)
            self._h = None
        self.analyzer = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------------- analyzer
class PivAnalyzer:
    """PivAnalyzer (multipass.rs:83-150) running every stage on one GPU."""

    def __init__(self, cfg: PivConfig = None, device: int = -1):
        self.cfg = PivConfig() if cfg is None else cfg
        c = self.cfg._c(device)
        h = ctypes.c_void_p()
        _check(_lib.load().piv_analyzer_create(ctypes.byref(c), ctypes.byref(h)))
        self._h = h

    @staticmethod
    def new(cfg: PivConfig) -> "PivAnalyzer":
        return PivAnalyzer(cfg)

    @staticmethod
    def check_config(cfg: PivConfig):
        c = cfg._c()
        _check(_lib.load().piv_check_config(ctypes.byref(c)))

    def config(self):
        return self.cfg

    def num_passes(self):
        return _lib.load().piv_num_passes(self._h)

    def output_grid(self, height, width) -> Grid:
        g = _lib.PivGridC()
        _check(_lib.load().piv_output_grid(self._h, int(height), int(width), ctypes.byref(g)))
        return Grid._from_c(g)

    def pass_grid(self, height, width, p) -> Grid:
        g = _lib.PivGridC()
        _check(_lib.load().piv_pass_grid(self._h, int(height), int(width), int(p), ctypes.byref(g)))
        return Grid._from_c(g)

    def sync(self):
        _check(_lib.load().piv_analyzer_sync(self._h))

    def set_stream(self, stream_ptr: Optional[int]):
        _check(_lib.load().piv_analyzer_set_stream(self._h, None if not stream_ptr else ctypes.c_void_p(stream_ptr)))

    def launches(self) -> int:
        return int(_lib.load().piv_analyzer_launches(self._h))

    def prepare(self, raw, cfg: PreprocessConfig = None, background=None) -> PreparedFrame:
        return PreparedFrame.new(raw, cfg, background, analyzer=self)

    def frame(self, height, width) -> PreparedFrame:
        return PreparedFrame(self, height, width)

    def analyze(self, a: PreparedFrame, b: PreparedFrame) -> PairResult:
        """Displacement field from frame `a` to frame `b`, in pixels (multipass.rs:136-138)."""
        g = self.output_grid(a.height, a.width) if a.dim() == b.dim() else None
        if g is None:
            raise ShapeMismatchError(f"frames have different shapes: {a.dim()} vs {b.dim()}")
        dx, dy, ppr = (np.empty((g.ny, g.nx), np.float32) for _ in range(3))
        fl = np.empty((g.ny, g.nx), np.uint8)
        s = _lib.PivSummaryC()
        _check(_lib.load().piv_analyze(self._h, a._h, b._h, _ptr(dx), _ptr(dy), _ptr(ppr), _ptr(fl), ctypes.byref(s)))
        return PairResult(VectorField(g, dx, dy, ppr, fl), ValidationSummary._from_c(s))

    def analyze_device(self, a: PreparedFrame, b: PreparedFrame, dx_ptr, dy_ptr, ppr_ptr, flags_ptr, summary_ptr=None):
        """Final field into device buffers (addresses), asynchronous on the analyzer's stream."""
        vp = ctypes.c_void_p
        _check(_lib.load().piv_analyze_device(self._h, a._h, b._h, vp(dx_ptr), vp(dy_ptr), vp(ppr_ptr), vp(flags_ptr),
                                              None if summary_ptr is None else vp(summary_ptr)))

    def analyze_traced(self, a: PreparedFrame, b: PreparedFrame) -> Tuple[PairResult, List[PassTrace]]:
        """Like analyze, but also returns what each pass did (multipass.rs:142-150)."""
        if a.dim() != b.dim():
            raise ShapeMismatchError(f"frames have different shapes: {a.dim()} vs {b.dim()}")
        grids = [self.pass_grid(a.height, a.width, p) for p in range(self.num_passes())]
        tot = sum(len(g) for g in grids)
        arr = dict(origins=np.empty((tot, 4), np.float32), raw_dx=np.empty(tot, np.float32),
                   raw_dy=np.empty(tot, np.float32), raw_peak_ratio=np.empty(tot, np.float32),
                   raw_flags=np.empty(tot, np.uint8), dx=np.empty(tot, np.float32), dy=np.empty(tot, np.float32),
                   peak_ratio=np.empty(tot, np.float32), flags=np.empty(tot, np.uint8))
        tr = _lib.PivTraceC(*[arr[k].ctypes.data for k in ("origins", "raw_dx", "raw_dy", "raw_peak_ratio", "raw_flags",
                                                           "dx", "dy", "peak_ratio", "flags")])
        s = _lib.PivSummaryC()
        _check(_lib.load().piv_analyze_traced(self._h, a._h, b._h, ctypes.byref(tr), ctypes.byref(s)))
        traces, off = [], 0
        for g in grids:
            c = len(g)
            sl, sh = slice(off, off + c), (g.ny, g.nx)
            raw = VectorField(g, arr["raw_dx"][sl].reshape(sh), arr["raw_dy"][sl].reshape(sh),
                              arr["raw_peak_ratio"][sl].reshape(sh), arr["raw_flags"][sl].reshape(sh))
            val = VectorField(g, arr["dx"][sl].reshape(sh), arr["dy"][sl].reshape(sh),
                              arr["peak_ratio"][sl].reshape(sh), arr["flags"][sl].reshape(sh))
            traces.append(PassTrace(arr["origins"][sl], raw, val))
            off += c
        return PairResult(traces[-1].validated, ValidationSummary._from_c(s)), traces

    # ------------------------------------------------------------------ stage hooks
    def place_windows(self, height, width, grid: Grid, predictor: Optional[VectorField] = None) -> np.ndarray:
        out = np.empty((len(grid), 4), np.float32)
        gc = grid._c()
        if predictor is None:
            _check(_lib.load().piv_place_windows(self._h, int(height), int(width), ctypes.byref(gc), None, None, None,
                                                 _ptr(out)))
        else:
            pg = predictor.grid._c()
            pdx = np.ascontiguousarray(predictor.dx, np.float32)
            pdy = np.ascontiguousarray(predictor.dy, np.float32)
            _check(_lib.load().piv_place_windows(self._h, int(height), int(width), ctypes.byref(gc), ctypes.byref(pg),
                                                 _ptr(pdx), _ptr(pdy), _ptr(out)))
        return out

    def correlate_origins(self, a: PreparedFrame, b: PreparedFrame, window: int, origins):
        origins = np.ascontiguousarray(origins, np.float32).reshape(-1, 4)
        c = origins.shape[0]
        dx, dy, ppr = (np.empty(c, np.float32) for _ in range(3))
        fl = np.empty(c, np.uint8)
        _check(_lib.load().piv_correlate_origins(self._h, a._h, b._h, int(window), _ptr(origins), c, _ptr(dx), _ptr(dy),
                                                 _ptr(ppr), _ptr(fl)))
        return dx, dy, ppr, fl

    def place_windows_deform(self, height, width, grid: Grid, predictor: Optional[VectorField] = None):
        """Origins [cells, 4] and the predictor at each window's corner pixels [cells, 8]
        (dx00, dy00, dx10, dy10, dx01, dy01, dx11, dy11)."""
        out = np.empty((len(grid), 4), np.float32)
        corners = np.empty((len(grid), 8), np.float32)
        gc = grid._c()
        if predictor is None:
            _check(_lib.load().piv_place_windows_deform(self._h, int(height), int(width), ctypes.byref(gc), None, None,
                                                        None, _ptr(out), _ptr(corners)))
        else:
            pg = predictor.grid._c()
            pdx = np.ascontiguousarray(predictor.dx, np.float32)
            pdy = np.ascontiguousarray(predictor.dy, np.float32)
            _check(_lib.load().piv_place_windows_deform(self._h, int(height), int(width), ctypes.byref(gc),
                                                        ctypes.byref(pg), _ptr(pdx), _ptr(pdy), _ptr(out),
                                                        _ptr(corners)))
        return out, corners

    def correlate_deform(self, a: PreparedFrame, b: PreparedFrame, grid: Grid, origins, corners):
        """Raw field of the deformed windows of `grid` (mask on `origins`): dx, dy, ppr, flags."""
        origins = np.ascontiguousarray(origins, np.float32).reshape(-1, 4)
        corners = np.ascontiguousarray(corners, np.float32).reshape(-1, 8)
        c = len(grid)
        if origins.shape[0] != c or corners.shape[0] != c:
            raise PivError("origins and corners need one row per grid cell")
        dx, dy, ppr = (np.empty(c, np.float32) for _ in range(3))
        fl = np.empty(c, np.uint8)
        gc = grid._c()
        _check(_lib.load().piv_correlate_deform(self._h, a._h, b._h, ctypes.byref(gc), _ptr(origins), _ptr(corners),
                                                _ptr(dx), _ptr(dy), _ptr(ppr), _ptr(fl)))
        return dx, dy, ppr, fl

    def validate_field(self, dx, dy, peak_ratio, fl):
        dx, dy, ppr = (np.ascontiguousarray(x, np.float32) for x in (dx, dy, peak_ratio))
        fl = np.ascontiguousarray(fl, np.uint8)
        ny, nx = dx.shape
        ox, oy = np.empty_like(dx), np.empty_like(dy)
        of = np.empty_like(fl)
        s = _lib.PivSummaryC()
        _check(_lib.load().piv_validate_field(self._h, ny, nx, _ptr(dx), _ptr(dy), _ptr(ppr), _ptr(fl), _ptr(ox),
                                              _ptr(oy), _ptr(of), ctypes.byref(s)))
        return ox, oy, of, ValidationSummary._from_c(s)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().piv_analyzer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _profile_methods():
    def set_profiling(self, enable=True):
        _check(_lib.load().piv_analyzer_set_profiling(self._h, int(bool(enable))))

    def profile(self, p):
        """(summed correlation-kernel ms, launches) of pass `p` since the last read."""
        ms, n = ctypes.c_double(), ctypes.c_int64()
        _check(_lib.load().piv_analyzer_profile(self._h, int(p), ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def autotune(self, a, b):
        """Times every launch variant of each pass's window size on this pair and keeps the
        fastest (results are identical across variants)."""
        _check(_lib.load().piv_analyzer_autotune(self._h, a._h, b._h))
        return {n: self.variant(n) for n in sorted(set(self.cfg.passes()))}

    def variant(self, window):
        buf = ctypes.create_string_buffer(64)
        _check(_lib.load().piv_analyzer_variant(self._h, int(window), buf, 64))
        return buf.value.decode()

    def set_variant(self, window, v):
        """Pins FP32 launch variant `v` (0 .. num_variants(window) - 1) for `window`."""
        _check(_lib.load().piv_analyzer_set_variant(self._h, int(window), int(v)))

    def num_variants(window):
        return int(_lib.load().piv_num_variants(int(window)))

    PivAnalyzer.set_profiling = set_profiling
    PivAnalyzer.profile = profile
    PivAnalyzer.autotune = autotune
    PivAnalyzer.variant = variant
    PivAnalyzer.set_variant = set_variant
    PivAnalyzer.num_variants = staticmethod(num_variants)


_profile_methods()


class PivBatch:
    """The batching form: a fixed set of frames (sequential pairs (i, i+1), or independent pairs
    (2k, 2k+1)) analysed by one CUDA graph replay per run. Results are those of
    PivAnalyzer.analyze on each pair."""

    def __init__(self, analyzer: PivAnalyzer, height, width, pairs, sequential=True, dtype=np.uint16,
                 cfg: PreprocessConfig = None):
        cfg = RAW if cfg is None else cfg
        self.height, self.width, self.pairs, self.sequential = int(height), int(width), int(pairs), bool(sequential)
        self.dtype = np.dtype(dtype)
        self.nframes = pairs + 1 if sequential else 2 * pairs
        self.grid = analyzer.output_grid(height, width)
        h = ctypes.c_void_p()
        pc = cfg._c()
        _check(_lib.load().piv_batch_create(analyzer._h, self.height, self.width, self.pairs, int(self.sequential),
                                            _dtype_code(np.empty(0, self.dtype)), ctypes.byref(pc), ctypes.byref(h)))
        self._h = h

    def input_device(self) -> int:
        return int(_lib.load().piv_batch_input_device(self._h))

    def run(self):
        _check(_lib.load().piv_batch_run(self._h))

    def sync(self):
        _check(_lib.load().piv_batch_sync(self._h))

    def kernels(self) -> int:
        return int(_lib.load().piv_batch_kernels(self._h))

    def stream(self) -> int:
        """The batch's CUDA stream handle (for torch.cuda.ExternalStream)."""
        return int(_lib.load().piv_batch_stream(self._h))

    def set_background(self, background_ptr: Optional[int]):
        """Device background image (height*width f32) subtracted from every frame of the batch;
        None for none. It must stay alive while the batch uses it."""
        _check(_lib.load().piv_batch_set_background(self._h, ctypes.c_void_p(background_ptr) if background_ptr else None))

    def set_stream(self, stream):
        """Run this batch's kernels on `stream` (a cudaStream_t handle; None: its own stream).
        Batches sharing a stream replay one after another while their host copies overlap."""
        _check(_lib.load().piv_batch_set_stream(self._h, ctypes.c_void_p(stream) if stream else None))

    def outputs_device(self):
        ptrs = [ctypes.c_void_p() for _ in range(5)]
        _check(_lib.load().piv_batch_outputs_device(self._h, *[ctypes.byref(p) for p in ptrs]))
        return [p.value for p in ptrs]

    def run_host(self, frames):
        """frames: [nframes, H, W] samples. Returns a list of PairResult, one per pair."""
        frames = np.ascontiguousarray(frames, dtype=self.dtype)
        if frames.shape != (self.nframes, self.height, self.width):
            raise ShapeMismatchError(f"expected {(self.nframes, self.height, self.width)}, got {frames.shape}")
        g = self.grid
        sh = (self.pairs, g.ny, g.nx)
        dx, dy, ppr = (np.empty(sh, np.float32) for _ in range(3))
        fl = np.empty(sh, np.uint8)
        sums = (_lib.PivSummaryC * self.pairs)()
        _check(_lib.load().piv_batch_run_host(self._h, _ptr(frames), _ptr(dx), _ptr(dy), _ptr(ppr), _ptr(fl), sums))
        return [PairResult(VectorField(g, dx[k], dy[k], ppr[k], fl[k]), ValidationSummary._from_c(sums[k]))
                for k in range(self.pairs)]

    def submit_host(self, frames, out=None):
        """run_host without waiting; collect with wait_host(). `frames` and the outputs should be
        pinned; they are kept alive until the wait."""
        frames = np.ascontiguousarray(frames, dtype=self.dtype)
        if frames.shape != (self.nframes, self.height, self.width):
            raise ShapeMismatchError(f"expected {(self.nframes, self.height, self.width)}, got {frames.shape}")
        g = self.grid
        sh = (self.pairs, g.ny, g.nx)
        if out is None:
            out = (np.empty(sh, np.float32), np.empty(sh, np.float32), np.empty(sh, np.float32), np.empty(sh, np.uint8))
        _check(_lib.load().piv_batch_submit_host(self._h, _ptr(frames), *[_ptr(x) for x in out]))
        self._inflight = (frames, out)

    def wait_host(self):
        frames, out = self._inflight
        self._inflight = None
        sums = (_lib.PivSummaryC * self.pairs)()
        _check(_lib.load().piv_batch_wait_host(self._h, sums))
        dx, dy, ppr, fl = out
        return [PairResult(VectorField(self.grid, dx[k], dy[k], ppr[k], fl[k]), ValidationSummary._from_c(sums[k]))
                for k in range(self.pairs)]

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().piv_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PivPipeline:
    """Pipelined pairs of one size: submit() queues a pair of host frames and returns a ticket at
    once; `depth` slots (each with its own workspace; uploads, kernels and downloads on three
    shared streams) overlap one pair's copies with the others' kernels. wait(ticket) returns the PairResult, equal to PivAnalyzer.analyze of that pair.
    Frames should be pinned host memory for the uploads to be asynchronous."""

    def __init__(self, analyzer: PivAnalyzer, height, width, dtype=np.uint16, cfg: PreprocessConfig = None, depth=2):
        cfg = RAW if cfg is None else cfg
        self.height, self.width, self.dtype = int(height), int(width), np.dtype(dtype)
        self.grid = analyzer.output_grid(height, width)
        h = ctypes.c_void_p()
        pc = cfg._c()
        _check(_lib.load().piv_pipeline_create(analyzer._h, self.height, self.width, _dtype_code(np.empty(0, self.dtype)),
                                               ctypes.byref(pc), int(depth), ctypes.byref(h)))
        self._h = h
        self._pending = {}

    def submit(self, a, b, out=None):
        a = np.ascontiguousarray(a, self.dtype)
        b = np.ascontiguousarray(b, self.dtype)
        if a.shape != (self.height, self.width) or b.shape != a.shape:
            raise ShapeMismatchError(f"expected {(self.height, self.width)}, got {a.shape} and {b.shape}")
        g = self.grid
        if out is None:
            out = (np.empty((g.ny, g.nx), np.float32), np.empty((g.ny, g.nx), np.float32),
                   np.empty((g.ny, g.nx), np.float32), np.empty((g.ny, g.nx), np.uint8))
        t = ctypes.c_uint64()
        _check(_lib.load().piv_pipeline_submit(self._h, _ptr(a), _ptr(b), *[_ptr(x) for x in out], ctypes.byref(t)))
        self._pending[t.value] = (a, b, out)  # keep the buffers alive until the pair is collected
        return t.value

    def set_background(self, background_ptr: Optional[int]):
        """Device background image (height*width f32, e.g. a torch CUDA tensor's data_ptr())
        subtracted from every frame submitted from now on; None for none. It must stay alive
        while pairs use it."""
        _check(_lib.load().piv_pipeline_set_background(self._h, ctypes.c_void_p(background_ptr) if background_ptr else None))

    def wait(self, ticket):
        a, b, out = self._pending.pop(ticket)
        s = _lib.PivSummaryC()
        _check(_lib.load().piv_pipeline_wait(self._h, ctypes.c_uint64(ticket), ctypes.byref(s)))
        return PairResult(VectorField(self.grid, *out), ValidationSummary._from_c(s))

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().piv_pipeline_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PivServer:
    """The serving form: continuous batching of frame pairs of any size and window schedule on one
    GPU under a device-memory budget. submit() returns a ticket at once; wait(ticket) returns the
    PairResult and the request's latency in milliseconds."""

    def __init__(self, memory_budget_bytes=60 << 30, max_in_flight=64, device=-1):
        h = ctypes.c_void_p()
        c = _lib.PivServerConfigC(int(device), int(memory_budget_bytes), int(max_in_flight))
        _check(_lib.load().piv_server_create(ctypes.byref(c), ctypes.byref(h)))
        self._h = h
        self._pending = {}

    def submit(self, a, b, cfg: PivConfig = None, pre: PreprocessConfig = None, out=None):
        """Queues the pair (a, b) of host samples (u8/u16/f32, pinned memory recommended). `out`
        optionally gives the four result arrays (dx, dy, peak_ratio, flags) to fill."""
        cfg = PivConfig() if cfg is None else cfg
        pre = RAW if pre is None else pre
        a = np.ascontiguousarray(a)
        b = np.ascontiguousarray(b)
        if a.shape != b.shape or a.dtype != b.dtype:
            raise ShapeMismatchError(f"frames differ: {a.shape} {a.dtype} vs {b.shape} {b.dtype}")
        h, w = a.shape
        g = Grid.new(h, w, cfg.windows[-1], cfg.overlap)
        if out is None:
            out = (np.empty((g.ny, g.nx), np.float32), np.empty((g.ny, g.nx), np.float32),
                   np.empty((g.ny, g.nx), np.float32), np.empty((g.ny, g.nx), np.uint8))
        cc = cfg._c()
        q = _lib.PivRequestC(cc, pre._c(), _dtype_code(a), h, w, a.ctypes.data, b.ctypes.data, out[0].ctypes.data,
                             out[1].ctypes.data, out[2].ctypes.data, out[3].ctypes.data)
        rid = ctypes.c_uint64()
        _check(_lib.load().piv_server_submit(self._h, ctypes.byref(q), ctypes.byref(rid)))
        self._pending[rid.value] = (a, b, out, g, cc)
        return rid.value

    def wait(self, ticket, timeout_ms: Optional[float] = None):
        """(PairResult, latency ms) of the request. With timeout_ms, raises TimeoutError if it is
        not done by then (the ticket stays valid); raises CancelledError for a cancelled one."""
        s = _lib.PivSummaryC()
        lat = ctypes.c_double()
        if timeout_ms is None:
            st = _lib.load().piv_server_wait(self._h, ctypes.c_uint64(ticket), ctypes.byref(s), ctypes.byref(lat))
        else:
            st = _lib.load().piv_server_wait_timeout(self._h, ctypes.c_uint64(ticket), float(timeout_ms),
                                                     ctypes.byref(s), ctypes.byref(lat))
            if st == _lib.PIV_ERR_TIMEOUT:
                _check(st)
        # the request is finished (or failed): its host buffers may go
        a, b, out, g, cc = self._pending.pop(ticket)
        _check(st)
        return PairResult(VectorField(g, out[0], out[1], out[2], out[3]), ValidationSummary._from_c(s)), lat.value

    def cancel(self, ticket):
        """Cancels a request: a queued one at once, an admitted one at the next step boundary.
        Its wait then raises CancelledError; a request already finishing keeps its result."""
        _check(_lib.load().piv_server_cancel(self._h, ctypes.c_uint64(ticket)))

    def fail_next_allocations(self, count: int):
        """Host-side fault injection: the next `count` admissions fail as out-of-memory."""
        _check(_lib.load().piv_server_fail_next_allocations(self._h, int(count)))

    def set_fused(self, fused: bool):
        """One fused correlation launch per step for the FP32 windows of 8-64 px (default), or one
        launch per window size and kind."""
        _check(_lib.load().piv_server_set_fused(self._h, int(bool(fused))))

    def set_manual(self, manual: bool):
        """Manual stepping: admission and steps happen only when advance() grants them."""
        _check(_lib.load().piv_server_set_manual(self._h, int(bool(manual))))

    def advance(self, steps: int = 1, timeout_ms: float = 60000.0):
        """Grants `steps` scheduler steps and waits until they have been taken."""
        _check(_lib.load().piv_server_advance(self._h, int(steps), float(timeout_ms)))

    def reserve(self, nbytes: int) -> int:
        """Grows the server's memory pool by nbytes ahead of time (blocking), so that admissions
        under load are served from memory the pool already holds instead of waiting on the
        driver to map more. Returns the bytes the pool holds afterwards (nbytes = 0: only that)."""
        held = ctypes.c_int64()
        _check(_lib.load().piv_server_reserve(self._h, int(nbytes), ctypes.byref(held)))
        return int(held.value)

    def stats(self):
        s = _lib.PivServerStatsC()
        _check(_lib.load().piv_server_stats(self._h, ctypes.byref(s)))
        return {n: getattr(s, n) for n, _ in s._fields_}

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().piv_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
