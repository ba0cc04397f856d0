"""The allocation-free validation entry point against the ordinary one.

piv_validate_field_noalloc exists for callers that cannot call cudaMalloc once running
(deadline-bound acquisition loops, where an allocation call can stall the device, and processes
whose device memory is already held by another allocator). It keeps its scratch in a fixed
device array inside the library, so this test checks, through the C ABI, that two calls in a row
on different fields give exactly what piv_validate_field gives (validation is bit-exact, so the
tolerance is zero), that the results also equal the reference's own validated golden field and
the oracle's validation of the synthetic field, that a field larger than the fixed scratch is
refused (also when its sizes would overflow a product), and that outputs overlapping inputs are
refused.

This file is named to be collected last, so a failure here comes after every other test ran.
"""
import ctypes

import numpy as np
import pytest

from conftest import Golden, same_floats

pytestmark = pytest.mark.gpu


def _noalloc(lib, torch, dx, dy, ppr, fl, max_disp, cfg):
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (dx, dy, ppr, fl)]
    ox, oy = torch.empty_like(t[0]), torch.empty_like(t[1])
    of = torch.empty_like(t[3])
    ny, nx = dx.shape
    v = cfg.validation
    stream = torch.cuda.current_stream(dev)
    st = lib.piv_validate_field_noalloc(ny, nx, *[ctypes.c_void_p(x.data_ptr()) for x in t], max_disp,
                                        v.ppr_threshold, v.median_threshold, v.median_eps, int(v.replace),
                                        ctypes.c_void_p(ox.data_ptr()), ctypes.c_void_p(oy.data_ptr()),
                                        ctypes.c_void_p(of.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
    assert st == 0, lib.piv_last_error()
    torch.cuda.synchronize(dev)
    return ox.cpu().numpy(), oy.cpu().numpy(), of.cpu().numpy()


def _synthetic_field(ny, nx, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:ny, 0:nx].astype(np.float32)
    dx = (2.0 + 0.01 * yy + 0.05 * rng.standard_normal((ny, nx))).astype(np.float32)
    dy = (-1.0 + 0.005 * xx + 0.05 * rng.standard_normal((ny, nx))).astype(np.float32)
    ppr = (1.0 + 4.0 * rng.random((ny, nx))).astype(np.float32)
    fl = np.zeros((ny, nx), np.uint8)
    k = rng.choice(ny * nx, ny * nx // 50, replace=False)
    dx.ravel()[k[: len(k) // 2]] += 9.0
    dy.ravel()[k[len(k) // 2:]] -= 30.0
    ns = rng.choice(ny * nx, ny * nx // 100, replace=False)
    fl.ravel()[ns] = 1
    dx.ravel()[ns] = np.nan
    dy.ravel()[ns] = np.nan
    ppr.ravel()[ns] = 0.0
    return dx, dy, ppr, fl


def test_noalloc_validation_matches_validate_field_on_two_calls():
    import torch

    import piv_b200 as P
    from oracle import oracle as O
    lib = P.load_library()
    cfg = P.PivConfig(windows=[64, 32])
    an = P.PivAnalyzer(cfg, device=0)
    g = Golden("particles_rotation")
    assert g.max_displacement == 32.0
    p = g.passes[-1]
    fields = [(p["raw_dx"], p["raw_dy"], p["raw_ppr"], p["raw_flags"]), _synthetic_field(1021, 1021, 7)]
    for call, (dx, dy, ppr, fl) in enumerate(fields):
        rx, ry, rf, _ = an.validate_field(dx, dy, ppr, fl)
        nx_, ny_, nf_ = _noalloc(lib, torch, dx, dy, ppr, fl, 32.0, cfg)
        assert np.array_equal(nf_, rf), f"call {call}: flags"
        assert same_floats(nx_, rx) and same_floats(ny_, ry), f"call {call}: values"
        assert np.count_nonzero(rf & P.flags.REPLACED) > 0
        if call == 0:
            # the reference's own validation of its raw field (validate.rs:51-130, written by Rust)
            assert np.array_equal(nf_, p["flags"]), "flags vs the golden validated field"
            assert same_floats(nx_, p["dx"]) and same_floats(ny_, p["dy"]), "values vs the golden validated field"
        else:
            ox, oy, of, _ = O.validate(dx, dy, ppr, fl, max_displacement=32.0)
            assert np.array_equal(nf_, of), "flags vs the oracle"
            assert same_floats(nx_, ox) and same_floats(ny_, oy), "values vs the oracle"


def test_noalloc_validation_rejects_fields_above_its_fixed_scratch():
    import torch

    import piv_b200 as P
    lib = P.load_library()
    buf = torch.zeros(16, device="cuda:0", dtype=torch.float32)
    p = ctypes.c_void_p(buf.data_ptr())
    q = ctypes.c_void_p(buf.data_ptr() + 32)
    for ny, nx in ((2048, 2048), (1 << 32, 1 << 32), (1 << 62, 4)):
        st = lib.piv_validate_field_noalloc(ny, nx, p, p, p, p, 32.0, 1.3, 2.0, 0.1, 1, q, q, q, None)
        assert st == 6, (ny, nx)  # PIV_ERR_UNSUPPORTED
        assert "exceeds" in lib.piv_last_error().decode()


def test_noalloc_validation_rejects_outputs_that_overlap_inputs():
    import torch

    import piv_b200 as P
    lib = P.load_library()
    n = 64
    buf = torch.zeros(16 * n, device="cuda:0", dtype=torch.float32)
    ptr = [ctypes.c_void_p(buf.data_ptr() + 4 * n * k) for k in range(16)]
    ins = ptr[:4]
    # in place (out_dx == dx), a partial overlap, and two outputs on one buffer
    for outs in ((ptr[0], ptr[5], ptr[6]), (ctypes.c_void_p(buf.data_ptr() + 4 * n * 3 + 4), ptr[5], ptr[6]),
                 (ptr[5], ptr[5], ptr[6])):
        st = lib.piv_validate_field_noalloc(8, 8, *ins, 32.0, 1.3, 2.0, 0.1, 1, *outs, None)
        assert st == 7, outs  # PIV_ERR_ARGUMENT
        assert "overlap" in lib.piv_last_error().decode()
    st = lib.piv_validate_field_noalloc(8, 8, *ins, 32.0, 1.3, 2.0, 0.1, 1, ptr[5], ptr[6], ptr[7], None)
    assert st == 0, lib.piv_last_error()
    torch.cuda.synchronize()
