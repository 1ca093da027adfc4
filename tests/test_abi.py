"""The C-ABI library loads and exports every symbol include/rcwa_b200.h
declares (CPU only: no compute call is made)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rcwa_b200.h")


def _declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b(rcwa_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from rcwa_b200 import build as B
    if not os.path.exists(B.LIB_PATH):
        B.build()
    return ctypes.CDLL(B.LIB_PATH)


def test_header_declares_entry_points():
    names = _declared()
    for must in ("rcwa_solve", "rcwa_solve_sweep", "rcwa_convmat", "rcwa_eig", "rcwa_lu_solve",
                 "rcwa_redheffer", "rcwa_smatrix_layer", "rcwa_efficiencies"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in _declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from rcwa_b200 import lib as L
    assert set(_declared()) <= set(L.declared_symbols()) | set(getattr(L, "EXTRA_SYMBOLS", []))


def test_last_error_without_gpu(lib):
    lib.rcwa_last_error.restype = ctypes.c_char_p
    assert isinstance(lib.rcwa_last_error(), bytes)
    lib.rcwa_version.restype = ctypes.c_int
    assert lib.rcwa_version() >= 10000


def test_cpp_host_api_compiles_and_links(lib, tmp_path):
    """The C++ host API (reference names on the C ABI) and its demo build
    against the header and link against the library (nothing is run)."""
    import shutil
    import subprocess
    from rcwa_b200 import build as B
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    demo = os.path.join(ROOT, "rcwa-cuda_b200", "host", "demo_main.cpp")
    cmd = [gxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"), demo,
           "-L", os.path.dirname(B.LIB_PATH), "-lrcwa_b200", "-L/usr/local/cuda/lib64", "-lcudart",
           "-o", str(tmp_path / "demo")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_gemm_table_choices_without_gpu(lib, tmp_path):
    """Kernel-table entries 0, 1, 2, 3 (DMMA via cp.async, CUDA cores, DMMA
    via TMA, DMMA via cp.async on 32 x 64 tiles) and -1 are accepted,
    anything else is rejected; the tuner's table loader applies the same
    rule."""
    import json
    from rcwa_b200 import lib as L
    from rcwa_b200 import tune
    ok = (ctypes.c_int * 25)(*([2] * 12 + [0] * 6 + [1] * 3 + [3] * 3 + [-1]))
    assert lib.rcwa_set_gemm_table(ok) == L.RCWA_OK
    bad = (ctypes.c_int * 25)(*([0] * 24 + [4]))
    assert lib.rcwa_set_gemm_table(bad) == L.RCWA_ERR_INVALID
    assert lib.rcwa_set_gemm_table(None) == L.RCWA_OK
    p = tmp_path / "t.json"
    p.write_text(json.dumps({"choice": [2] * 25}))
    assert tune.load_table(str(p)) == [2] * 25
    p.write_text(json.dumps({"choice": [4] * 25}))
    assert tune.load_table(str(p)) is None
    assert tune.load_table(tune.TABLE_PATH) is not None
