"""CPU-only checks of the C ABI library and the host-side logic (no GPU calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "wust_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(wust_[a-z0-9_]+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    from waveforminversionust_b200 import _lib
    lib = _lib.load()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.EXPORTED)


def test_status_ids_match_reference_identifiers():
    from waveforminversionust_b200 import _lib
    lib = _lib.load()
    for code, name in _lib.STATUS_NAMES.items():
        assert lib.wust_status_id(code).decode() == name
    major, minor, patch = C.c_int(), C.c_int(), C.c_int()
    assert lib.wust_version(C.byref(major), C.byref(minor), C.byref(patch)) == 0


def test_header_is_plain_c():
    """The boundary header compiles as C (no C++ or torch types)."""
    import shutil
    import subprocess
    import tempfile
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("gcc absent")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        with open(src, "w") as f:
            f.write('#include "wust_b200.h"\nint main(void){ wust_solver_options o; (void)o; return 0; }\n')
        subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", os.path.dirname(HEADER), src],
                       check=True)


def test_solver_options_struct_matches_header():
    """ctypes layout of wust_solver_options equals the C layout."""
    import shutil
    import subprocess
    import tempfile
    from waveforminversionust_b200._lib import SolverOptions
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("gcc absent")
    fields = [f[0] for f in SolverOptions._fields_]
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "t.c")
        body = "".join(f'printf("%zu ", offsetof(wust_solver_options, {n}));' for n in fields)
        with open(src, "w") as f:
            f.write('#include <stdio.h>\n#include <stddef.h>\n#include "wust_b200.h"\n'
                    f'int main(void){{ {body} printf("%zu", sizeof(wust_solver_options)); return 0; }}\n')
        exe = os.path.join(d, "t")
        subprocess.run([gcc, "-I", os.path.dirname(HEADER), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    offs = [int(v) for v in out[:-1]]
    assert offs == [getattr(SolverOptions, n).offset for n in fields]
    assert int(out[-1]) == C.sizeof(SolverOptions)


def test_package_ncg_rules_match_oracle():
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import ncg
    rng = np.random.default_rng(0)
    for _ in range(20):
        g, z, pz, pd = (rng.standard_normal(12) for _ in range(4))
        z = np.abs(z) * np.sign(g)           # preconditioned gradient with g.z >= 0
        pgz = float(abs(rng.standard_normal()))
        same = bool(rng.integers(0, 2))
        a = ncg.ncg_direction(g, z, pz, pgz, pd, same)
        b = o.ncg_direction(g, z, pz, pgz, pd, same)
        # same rules; dot-product summation order may differ in the last ulp
        assert np.allclose(a[0], b[0], rtol=1e-13, atol=0)
        assert abs(a[1] - b[1]) <= 1e-13 * max(1.0, abs(b[1])) and abs(a[2] - b[2]) <= 1e-13 * abs(b[2])
    mask = rng.integers(0, 2, (9, 7)).astype(bool)
    c = 1500 + 10 * rng.standard_normal((9, 7))
    d = rng.standard_normal((9, 7)) * 1e-5
    cfg = dict(max_update_mps=12.0, bounds_mps=(1300.0, 1800.0), step_damping=.25, update_mask=mask)
    assert np.array_equal(ncg.project_slowness_update(c, d, 0.7, cfg),
                          o.project_slowness_update(c, d, 0.7, 12.0, (1300.0, 1800.0), .25, mask))
    x = np.arange(-15, 16) * 1e-3
    img = rng.standard_normal((31, 31))
    assert np.allclose(ncg.ringing_removal_filt(x, x, img, 1500, 1e5, .5, 4),
                       o.ringing_removal_filt(x, x, img, 1500, 1e5, .5, 4), rtol=0, atol=1e-12)
    assert ncg.linearized_step_length(-2.0, 4.0) == 0.5


def test_synthetic_geometry_follows_wust_geometry():
    from oracle import helmholtz_fp64 as o
    from waveforminversionust_b200 import synthetic
    for p in (synthetic.config1(), synthetic.small()):
        xy = synthetic.ring(p.rx_index.size, 35e-3 if p.name == "config1" else 0.38 * 48 * 0.5e-3)
        assert np.array_equal(p.rx_index, o.snap(xy, p.x_m, p.y_m))
        ny, nx = p.shape
        iy = (p.tx_index - 1) % ny
        ix = (p.tx_index - 1) // ny
        assert np.all((iy > 0) & (iy < ny - 1) & (ix > 0) & (ix < nx - 1))
    p = synthetic.config2()
    assert p.shape == (552, 552) and p.tx_index.size == 256 and p.rx_index.size == 256


def test_package_without_library_fails_loudly(tmp_path, monkeypatch):
    """No CPU fallback: a missing shared library is an import-time error."""
    from waveforminversionust_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(ImportError):
        _lib.load()


def test_mex_gateways_compile_against_api_declarations():
    """The MEX gateways compile as C99 against the library header and the
    declarations of the MATLAB MEX API (the MEX runtime stand-in's headers)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if not gcc:
        pytest.skip("gcc absent")
    here = os.path.dirname(os.path.abspath(__file__))
    mex_dir = os.path.join(os.path.dirname(here), "waveforminversionust_b200", "mex")
    shim = os.path.join(os.path.dirname(here), "oracle", "mexshim")
    for name in sorted(f for f in os.listdir(mex_dir) if f.endswith(".c")):
        subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-I", shim,
                        "-I", os.path.dirname(HEADER), os.path.join(mex_dir, name)], check=True)
