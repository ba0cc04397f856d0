"""The C-ABI library loads, exports every symbol include/piv_b200.h declares, and its host-only
entry points (grid, config check) follow the reference (grid.rs:77-105, multipass.rs:478-507).
No GPU is needed for these."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _declared():
    with open(os.path.join(ROOT, "include", "piv_b200.h")) as f:
        src = f.read()
    return sorted(set(re.findall(r"\b(piv_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from piv_b200 import _lib
    L = ctypes.CDLL(_lib.LIB_PATH)
    declared = _declared()
    assert declared, "no declarations found"
    missing = [s for s in declared if not hasattr(L, s)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == declared


def test_abi_version():
    import piv_b200 as P
    assert P.load_library().piv_abi_version() == 1


def test_grid_matches_reference_examples():
    import piv_b200 as P
    g = P.Grid.new(1080, 1920, 32, 0.5)
    assert g.step == 16 and (g.nx, g.ny) == (119, 66) and (g.x0, g.y0) == (0, 4)
    assert g.center_x(0) == np.float32(15.5)
    g = P.Grid.new(64, 64, 32, 0.0)
    assert (g.nx, g.ny, g.step, g.x0) == (2, 2, 32, 0)
    assert list(g.xs()) == [15.5, 47.5]
    for args in ((16, 64, 32, 0.5), (64, 64, 32, 1.0), (64, 64, 32, -0.1)):
        with pytest.raises(P.PivError):
            P.Grid.new(*args)


def test_grid_counts_of_the_benchmark_configs():
    import piv_b200 as P
    assert len(P.Grid.new(4096, 4096, 16, 0.75)) == 1021 * 1021
    assert len(P.Grid.new(4096, 4096, 32, 0.75)) == 259081
    assert len(P.Grid.new(1024, 1024, 16, 0.5)) == 16129


def test_grid_matches_oracle():
    import piv_b200 as P
    from oracle import oracle as O
    rng = np.random.default_rng(0)
    for _ in range(200):
        h, w = int(rng.integers(8, 600)), int(rng.integers(8, 600))
        n = int(rng.choice([8, 12, 16, 24, 32, 48, 64]))
        ov = float(rng.choice([0.0, 0.25, 0.5, 0.75, 0.6, 0.9]))
        if n > min(h, w):
            continue
        g, o = P.Grid.new(h, w, n, ov), O.grid(h, w, n, ov)
        assert (g.step, g.nx, g.ny, g.x0, g.y0) == (o.step, o.nx, o.ny, o.x0, o.y0)


def test_rejects_bad_config():
    import piv_b200 as P
    for cfg in (P.PivConfig(windows=[]), P.PivConfig(windows=[33]), P.PivConfig(overlap=1.0),
                P.PivConfig(final_iterations=0), P.PivConfig(windows=[6])):
        with pytest.raises(P.ConfigError):
            P.PivAnalyzer.check_config(cfg)
    # valid for the reference, not supported by the GPU path: a distinct error
    with pytest.raises(P.UnsupportedError):
        P.PivAnalyzer.check_config(P.PivConfig(windows=[40]))
    P.PivAnalyzer.check_config(P.PivConfig())


def test_header_is_plain_c():
    """The boundary is a C ABI: the header compiles as strict C99 (and as C++) with no warnings."""
    import os
    import shutil
    import subprocess
    import tempfile
    cc = shutil.which("gcc")
    if cc is None:
        import pytest
        pytest.skip("no C compiler")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "h.c")
        with open(src, "w") as f:
            f.write('#include "piv_b200.h"\nint main(void) { return PIV_OK; }\n')
        for cmd in ([cc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only"],
                    [shutil.which("g++") or "g++", "-std=c++17", "-Wall", "-Werror", "-fsyntax-only", "-x", "c++"]):
            r = subprocess.run(cmd + ["-I", os.path.join(root, "include"), src], capture_output=True, text=True)
            assert r.returncode == 0, r.stderr
