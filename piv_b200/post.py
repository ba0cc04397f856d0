"""Post-processing of validated fields on the GPU: flow statistics of a pair and the temporal /
spatial smoothing filters of a pair series (flowstats.rs, flow.rs, smooth.rs).

Arrays are DEVICE arrays: anything with `data_ptr()` (a torch CUDA tensor) or a raw device
address. Shapes follow the reference: one field [ny, nx], a series [nt, ny, nx].
"""
import ctypes
from dataclasses import dataclass

from . import _lib
from .api import _check

__all__ = ["FlowStats", "flow_stats", "temporal_smooth", "spatial_smooth"]


def _p(a):
    if a is None:
        return None
    return ctypes.c_void_p(a.data_ptr() if hasattr(a, "data_ptr") else int(a))


@dataclass
class FlowStats:
    """FlowStats (flowstats.rs:10-25)."""
    vorticity_mean: float
    vorticity_abs_mean: float
    ke_mean: float
    ke_sum: float
    coverage: float
    n_usable: int
    n_vorticity: int


def flow_stats(dx, dy, flags, step, dt_s, vorticity=None, stream=None):
    """Statistics of one pair in px/s units (flow.rs:20-36); `vorticity` optionally receives the
    vorticity field."""
    ny, nx = dx.shape
    s = _lib.PivFlowStatsC()
    _check(_lib.load().piv_flow_stats_device(ny, nx, int(step), float(dt_s), _p(dx), _p(dy), _p(flags), _p(vorticity),
                                             ctypes.byref(s), _p(stream)))
    return FlowStats(s.vorticity_mean, s.vorticity_abs_mean, s.ke_mean, s.ke_sum, s.coverage, s.n_usable,
                     s.n_vorticity)


def temporal_smooth(dx, dy, usable, gate, out_dx, out_dy, support, kernel="mean", window=5, min_support=1,
                    leave_out=(), stream=None):
    """temporal (smooth.rs:44-128) into out_dx, out_dy, support (all [nt, ny, nx])."""
    nt, ny, nx = dx.shape
    lo = (ctypes.c_int32 * max(len(leave_out), 1))(*[int(v) for v in leave_out])
    _check(_lib.load().piv_temporal_smooth_device(nt, ny, nx, _p(dx), _p(dy), _p(usable), _p(gate),
                                                  int(kernel == "median"), int(window), int(min_support), lo,
                                                  len(leave_out), _p(out_dx), _p(out_dy), _p(support), _p(stream)))


def spatial_smooth(dx, dy, gate, out_dx, out_dy, support, sigma=1.0, min_weight=0.25, leave_out=None, stream=None):
    """spatial (smooth.rs:130-207) into out_dx, out_dy, support (all [nt, ny, nx])."""
    nt, ny, nx = dx.shape
    _check(_lib.load().piv_spatial_smooth_device(nt, ny, nx, _p(dx), _p(dy), _p(gate), float(sigma), float(min_weight),
                                                 -1 if leave_out is None else int(leave_out), _p(out_dx), _p(out_dy),
                                                 _p(support), _p(stream)))
