"""Synthetic particle-image pairs with known displacement (test and benchmark inputs; never timed).

Restates the reference's generator (rust/crates/piv-core/src/synthetic.rs):
  SplitMix64 RNG                 synthetic.rs:10-36
  analytic Gaussian-blob render  synthetic.rs:48-62   (sub-pixel motion is rendered exactly)
  midpoint displacement          synthetic.rs:66-82   (3 fixed-point iterations)
  particles / fog / noise        synthetic.rs:85-144
and adds the benchmark workloads of this project (u8/u16 quantised particle pairs with vortex,
shear and outlier clusters). Rendering sums blob contributions with np.bincount (float64, then
rounded to float32), so frames agree with the reference's sequential f32 sums to rounding only.
"""
import math

import numpy as np

_MASK = (1 << 64) - 1


class Rng:
    """SplitMix64 (synthetic.rs:10-36)."""

    def __init__(self, seed):
        self.s = seed & _MASK

    def next_u64(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & _MASK
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
        return z ^ (z >> 31)

    def uniform(self):
        return np.float32(self.next_u64() >> 40) / np.float32(1 << 24)

    def uniforms(self, n):
        """n successive uniform() draws, vectorised (same sequence as n calls)."""
        k = np.arange(1, n + 1, dtype=np.uint64)
        with np.errstate(over="ignore"):
            s = np.uint64(self.s) + k * np.uint64(0x9E3779B97F4A7C15)
            z = s
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
        self.s = int(s[-1]) if n else self.s
        return (z >> np.uint64(40)).astype(np.float32) / np.float32(1 << 24)

    def normal(self):
        u1 = max(self.uniform(), np.float32(1e-7))
        u2 = self.uniform()
        return np.float32(math.sqrt(-2.0 * math.log(u1)) * math.cos(2 * math.pi * u2))

    def normals(self, n):
        u = self.uniforms(2 * n).reshape(n, 2)
        u1 = np.maximum(u[:, 0], np.float32(1e-7))
        return (np.sqrt(-2.0 * np.log(u1)) * np.cos(np.float32(2 * math.pi) * u[:, 1])).astype(np.float32)


def round_half_away(v):
    return np.where(v >= 0, np.floor(v + 0.5), np.ceil(v - 0.5))


def render(h, w, x, y, sigma, amp, chunk=1 << 16):
    """Renders Gaussian blobs additively into an h x w float32 frame (synthetic.rs:48-62)."""
    out = np.zeros(h * w, np.float64)
    x, y, sigma, amp = (np.asarray(a, np.float32) for a in (x, y, sigma, amp))
    for s in range(0, len(x), chunk):
        bx, by, bs, ba = x[s:s + chunk], y[s:s + chunk], sigma[s:s + chunk], amp[s:s + chunk]
        r = np.ceil(np.float32(3.5) * bs).astype(np.int64)
        rmax = int(r.max()) if len(r) else 0
        cx = round_half_away(bx).astype(np.int64)
        cy = round_half_away(by).astype(np.int64)
        k = np.float32(1.0) / (np.float32(2.0) * bs * bs)
        off = np.arange(-rmax, rmax + 1)
        oy, ox = np.meshgrid(off, off, indexing="ij")
        oy, ox = oy.ravel(), ox.ravel()
        yy = cy[:, None] + oy[None, :]
        xx = cx[:, None] + ox[None, :]
        m = ((np.abs(oy)[None, :] <= r[:, None]) & (np.abs(ox)[None, :] <= r[:, None]) & (yy >= 0) & (yy < h)
             & (xx >= 0) & (xx < w))
        dx = xx.astype(np.float32) - bx[:, None]
        dy = yy.astype(np.float32) - by[:, None]
        v = ba[:, None] * np.exp(-(dx * dx + dy * dy) * k[:, None])
        out += np.bincount((yy * w + xx)[m], weights=v[m], minlength=h * w)
    return out.astype(np.float32).reshape(h, w)


def displace(x, y, field):
    """Moves blobs by field at the midpoint (synthetic.rs:66-82)."""
    x = np.asarray(x, np.float32)
    y = np.asarray(y, np.float32)
    dx, dy = field(x, y)
    for _ in range(3):
        dx, dy = field(x + dx / np.float32(2), y + dy / np.float32(2))
    return (x + np.asarray(dx, np.float32)).astype(np.float32), (y + np.asarray(dy, np.float32)).astype(np.float32)


def particles(h, w, seed, density, sigma):
    """Random particles (synthetic.rs:85-97): returns x, y, sigma, amp arrays."""
    rng = Rng(seed)
    margin = np.float32(20.0)
    area = (np.float32(h) + 2 * margin) * (np.float32(w) + 2 * margin)
    n = int(np.float32(density) * area)
    u = rng.uniforms(4 * n).reshape(n, 4)
    x = u[:, 0] * (np.float32(w) + 2 * margin) - margin
    y = u[:, 1] * (np.float32(h) + 2 * margin) - margin
    s = np.float32(sigma) * (np.float32(0.8) + np.float32(0.4) * u[:, 2])
    a = np.float32(0.3) + np.float32(0.7) * u[:, 3]
    return x, y, s, a


def _field_fn(field):
    def f(x, y):
        r = field(x, y)
        return np.broadcast_to(np.asarray(r[0], np.float32), x.shape), np.broadcast_to(np.asarray(r[1], np.float32), x.shape)
    return f


def particle_pair(h, w, seed, density, sigma, field):
    """Particle image pair with displacement `field(x, y) -> (u, v)` (synthetic.rs:129-137)."""
    x, y, s, a = particles(h, w, seed, density, sigma)
    xb, yb = displace(x, y, _field_fn(field))
    return render(h, w, x, y, s, a), render(h, w, xb, yb, s, a)


def fog(h, w, seed):
    """Fog-like texture (synthetic.rs:100-112)."""
    rng = Rng(seed)
    margin = np.float32(30.0)
    area = (np.float32(h) + 2 * margin) * (np.float32(w) + 2 * margin)
    n = int(area / np.float32(40.0))
    u = rng.uniforms(4 * n).reshape(n, 4)
    x = u[:, 0] * (np.float32(w) + 2 * margin) - margin
    y = u[:, 1] * (np.float32(h) + 2 * margin) - margin
    s = np.float32(2.0) + np.float32(4.0) * u[:, 2]
    a = np.float32(0.05) + np.float32(0.1) * u[:, 3]
    return x, y, s, a


def fog_pair(h, w, seed, field):
    x, y, s, a = fog(h, w, seed)
    xb, yb = displace(x, y, _field_fn(field))
    return render(h, w, x, y, s, a), render(h, w, xb, yb, s, a)


def add_noise(frame, sigma, seed):
    """Zero-mean Gaussian noise (synthetic.rs:140-144)."""
    rng = Rng(seed)
    return (frame + np.float32(sigma) * rng.normals(frame.size).reshape(frame.shape)).astype(np.float32)


# ----------------------------------------------------------------------------------------------
# Benchmark workloads (seeded; quantised to the stated bit depth by rounding and clamping)
# ----------------------------------------------------------------------------------------------
def quantise(frame, maxcode, dtype):
    return np.clip(np.rint(frame), 0, maxcode).astype(dtype)


def _blobs(h, w, rng_seed, ppp, dmin, dmax, amin, amax, margin=20.0):
    rng = Rng(rng_seed)
    area = (h + 2 * margin) * (w + 2 * margin)
    n = int(ppp * area)
    u = rng.uniforms(4 * n).reshape(n, 4).astype(np.float64)
    x = (u[:, 0] * (w + 2 * margin) - margin).astype(np.float32)
    y = (u[:, 1] * (h + 2 * margin) - margin).astype(np.float32)
    d = dmin + (dmax - dmin) * u[:, 2]
    s = (d / 4.0).astype(np.float32)  # d is the e^-2 diameter: sigma = d / 4
    a = (amin + (amax - amin) * u[:, 3]).astype(np.float32)
    return x, y, s, a


def vortex_shear_field(h, w, vmax=10.0, core=None, shear=0.01):
    """Lamb-Oseen-type vortex u_theta ~ (1 - exp(-r^2/rc^2))/r scaled to `vmax` px, plus shear."""
    cx, cy = (w - 1) / 2.0, (h - 1) / 2.0
    rc = core if core is not None else min(h, w) / 10.0
    peak = (1.0 - math.exp(-1.2564312086261696)) / (1.1209 * rc)  # max of (1-e^-(r/rc)^2)/r at r ~ 1.1209 rc
    amp = vmax / peak

    def f(x, y):
        x = np.asarray(x, np.float64)
        y = np.asarray(y, np.float64)
        rx, ry = x - cx, y - cy
        r2 = rx * rx + ry * ry
        with np.errstate(divide="ignore", invalid="ignore"):
            g = np.where(r2 > 0, amp * (1.0 - np.exp(-r2 / (rc * rc))) / r2, 0.0)
        return (-ry * g + shear * ry).astype(np.float32), (rx * g).astype(np.float32)
    return f


def baseline_pair(h, w, seed, field, ppp=0.05, dmin=2.0, dmax=4.0, bits=12, noise=None, amin=None, amax=None,
                  outlier_cells=None, outlier_window=16):
    """A quantised particle pair: u8 when bits == 8, else u16 with `bits` significant bits.

    Peak intensities are uniform over [amin, amax] of the full scale (default 120/255 .. 1), noise
    is Gaussian with sigma 4/255 of full scale by default. `outlier_cells` (list of (x0, y0))
    paints a cluster of spurious particles into frame B only, inside a window of that size."""
    full = (1 << bits) - 1
    amin = (120.0 / 255.0) if amin is None else amin
    amax = 1.0 if amax is None else amax
    noise = (4.0 / 255.0) if noise is None else noise
    x, y, s, a = _blobs(h, w, seed, ppp, dmin, dmax, amin * full, amax * full)
    xb, yb = displace(x, y, field)
    fa = render(h, w, x, y, s, a)
    fb = render(h, w, xb, yb, s, a)
    if outlier_cells is not None and len(outlier_cells):
        rng = Rng(seed ^ 0x5EED)
        oc = np.asarray(outlier_cells, np.float32)
        k = 6
        u = rng.uniforms(4 * k * len(oc)).reshape(len(oc), k, 4)
        ox = (oc[:, :1] + u[:, :, 0] * outlier_window).ravel()
        oy = (oc[:, 1:2] + u[:, :, 1] * outlier_window).ravel()
        osg = (np.float32(0.5) + np.float32(0.5) * u[:, :, 2]).ravel()
        oa = (np.float32(amax * full) * (np.float32(0.6) + np.float32(0.4) * u[:, :, 3])).ravel()
        fb = fb + render(h, w, ox, oy, osg, oa)
    if noise > 0:
        fa = add_noise(fa, noise * full, seed + 1)
        fb = add_noise(fb, noise * full, seed + 2)
    dt = np.uint8 if bits == 8 else np.uint16
    return quantise(fa, full, dt), quantise(fb, full, dt)
