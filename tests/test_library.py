"""Host-side checks of the C-ABI library (no GPU needed)."""
import os
import re
import subprocess

import pytest

import kc_cuda_b200 as K
from kc_cuda_b200 import solver

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "kt.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(kt_[a-z_0-9]+)\s*\(", src)))


def test_header_declares_entry_points():
    names = header_functions()
    assert "kt_solve" in names and "kt_load_tsv" in names and len(names) >= 18


def test_library_exports_every_declared_symbol():
    L = K.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", solver.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (kt_\w+)", out))
    for name in header_functions():
        assert name in exported, name
        assert getattr(L, name) is not None


def test_python_signatures_cover_header():
    assert {n for n, _, _ in solver.SIGNATURES} == set(header_functions())


def test_status_strings():
    L = K.lib()
    assert L.kt_status_string(0) == b"ok"
    assert L.kt_status_string(4) == b"malformed input"


def test_cli_usage_without_gpu():
    exe = os.path.join(ROOT, "kc_cuda_b200", "kt_solve")
    p = subprocess.run([exe], capture_output=True, text=True)
    assert p.returncode == 1 and p.stderr.strip() == "Usage: -f [data_file_path]"
    p = subprocess.run([exe, "-x", "file"], capture_output=True, text=True)
    assert p.returncode == 1


def test_no_cpu_fallback_without_device():
    import ctypes
    if os.environ.get("CUDA_VISIBLE_DEVICES") is None:
        pytest.skip("only meaningful where no device is visible")
    h = ctypes.c_void_p()
    s = K.lib().kt_init(0, 0, ctypes.byref(h))
    assert s != 0


def test_every_option_is_documented():
    """Each name in the library's option table (kt_set_option) is described in
    the header's option list."""
    src = open(os.path.join(ROOT, "kc_cuda_b200", "csrc", "api.cu")).read()
    table = src[src.index("option_slot(kt::Options& o"):]
    table = table[: table.index("};")]
    names = re.findall(r'\{"([a-z_0-9]+)", &o\.', table)
    assert len(names) > 20
    header = open(os.path.join(ROOT, "include", "kt.h")).read()
    missing = [n for n in names if not re.search(r"\*\s+" + n + r" \(", header)]
    assert not missing, missing
