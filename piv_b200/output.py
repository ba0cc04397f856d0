"""Per-pair NPZ output with the reference's layout and field names (piv-io/src/write.rs:113-165):
one compressed `pair_AAAAAA_BBBBBB.npz` per frame pair plus `run.json` in a directory.

Arrays of one pair file:
    x, y             window centres in full-frame pixels (grid.rs:60-70 plus the ROI offset)
    dx, dy           displacement, px                  [ny, nx] f32
    u, v             velocity, px/s (dx / dt)          [ny, nx] f32
    u_mps, v_mps     velocity, m/s (only with a scale) [ny, nx] f32
    peak_ratio       [ny, nx] f32
    flags            [ny, nx] u8 (bits of validate.rs:13-19)
    frames           [frame_a, frame_b] u64
    t                pair midpoint time, s (0-d f64)
The arithmetic of the derived arrays follows write.rs:74-90 in f32: u = dx * f32(1 / dt_s),
u_mps = u * f32(m_per_px).
"""
import json
import os

import numpy as np

__all__ = ["NpzWriter", "grid_coords", "derive"]


def grid_coords(grid, roi=None):
    """Window centres (x along the columns, y along the rows) in full-frame pixels: the grid's
    centres plus the ROI offset (write.rs:64-71)."""
    ox = np.float32(roi[0] if roi else 0)
    oy = np.float32(roi[1] if roi else 0)
    return grid.xs() + ox, grid.ys() + oy


def derive(field, dt_s, m_per_px=None):
    """u, v (px/s) and, with a scale, u_mps, v_mps (m/s) as write.rs:80-90 computes them."""
    inv_dt = np.float32(1.0 / float(dt_s))
    u = (np.asarray(field.dx, np.float32) * inv_dt).astype(np.float32)
    v = (np.asarray(field.dy, np.float32) * inv_dt).astype(np.float32)
    phys = None
    if m_per_px is not None:
        k = np.float32(m_per_px)
        phys = ((u * k).astype(np.float32), (v * k).astype(np.float32))
    return u, v, phys


class NpzWriter:
    """NpzWriter (write.rs:113-165). `meta` is the run's metadata (written as run.json); it must
    hold `dt_s`, and may hold `roi` ({"x", "y", ...}) and `scale` ({"m_per_px": ...})."""

    def __init__(self, directory, meta):
        if "dt_s" not in meta or not float(meta["dt_s"]) > 0:
            raise ValueError("run metadata needs a positive dt_s")
        self.dir = str(directory)
        self.meta = dict(meta)
        os.makedirs(self.dir, exist_ok=True)
        with open(os.path.join(self.dir, "run.json"), "w") as f:
            json.dump(self.meta, f, indent=2, default=_jsonable)
        roi = self.meta.get("roi")
        self._roi = (int(roi["x"]), int(roi["y"])) if roi else None
        scale = self.meta.get("scale")
        self._m_per_px = float(scale["m_per_px"]) if scale else None

    def path(self, frame_a, frame_b):
        return os.path.join(self.dir, f"pair_{int(frame_a):06d}_{int(frame_b):06d}.npz")

    def write(self, frame_a, frame_b, time_s, field):
        x, y = grid_coords(field.grid, self._roi)
        u, v, phys = derive(field, self.meta["dt_s"], self._m_per_px)
        arrays = {"x": x, "y": y, "dx": np.asarray(field.dx, np.float32), "dy": np.asarray(field.dy, np.float32),
                  "u": u, "v": v}
        if phys is not None:
            arrays["u_mps"], arrays["v_mps"] = phys
        arrays["peak_ratio"] = np.asarray(field.peak_ratio, np.float32)
        arrays["flags"] = np.asarray(field.flags, np.uint8)
        arrays["frames"] = np.array([frame_a, frame_b], np.uint64)
        arrays["t"] = np.array(float(time_s), np.float64)
        p = self.path(frame_a, frame_b)
        np.savez_compressed(p, **arrays)
        return p

    def finish(self):
        pass


def _jsonable(o):
    if hasattr(o, "__dict__"):
        return o.__dict__
    if isinstance(o, (np.integer, np.floating)):
        return o.item()
    return str(o)
