"""The C-ABI library loads and exports every entry point of include/piafs_gpu.h
(no device work: runs without a GPU)."""
import ctypes
import os
import re

import pytest

import piafs_b200
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "piafs_gpu.h")


def declared():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(piafs_gpu_\w+)\s*\(", txt)))


def test_header_declares_the_bound_functions():
    assert declared() == sorted(piafs_b200.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = piafs_b200.load_library()
    for name in declared():
        assert isinstance(getattr(lib, name), ctypes._CFuncPtr), name


def test_error_codes_and_messages_without_device():
    lib = piafs_b200.load_library()
    h = ctypes.c_void_p()
    # a missing deck is reported as an input error before any device work
    rc = lib.piafs_gpu_create(b"/nonexistent/deck", 0, ctypes.byref(h))
    assert rc == 2 and b"solver.inp" in lib.piafs_gpu_last_error()
    assert lib.piafs_gpu_create(None, 0, ctypes.byref(h)) == 1


def test_unsupported_options_are_rejected(tmp_path):
    from piafs_b200 import cases
    d = tmp_path / "d"
    cases.euler1d_density_wave(str(d), N=16, n_iter=1)
    txt = open(d / "solver.inp").read().replace("weno5", "muscl3")
    open(d / "solver.inp", "w").write(txt)
    lib = piafs_b200.load_library()
    h = ctypes.c_void_p()
    assert lib.piafs_gpu_create(str(d).encode(), 0, ctypes.byref(h)) == 3


def test_line_length_and_singular_options_are_rejected(tmp_path):
    """Host-side checks before any device call: CRWENO5 lines beyond a
    cluster of 8 CTAs (32769 interfaces) and CRWENO5 on characteristic
    variables with photochemistry (the reference's block solve is singular)."""
    from piafs_b200 import cases
    lib = piafs_b200.load_library()
    h = ctypes.c_void_p()
    d = tmp_path / "long"
    cases.euler1d_density_wave(str(d), N=40000, n_iter=1, scheme="crweno5")
    assert lib.piafs_gpu_create(str(d).encode(), 0, ctypes.byref(h)) == 3
    assert b"32769" in lib.piafs_gpu_last_error()
    c = tmp_path / "chem"
    cases.ns2d_photochem_beam(str(c), N=16, NY=12, n_iter=1, interp="characteristic")
    assert lib.piafs_gpu_create(str(c).encode(), 0, ctypes.byref(h)) == 3
    assert b"singular" in lib.piafs_gpu_last_error()


def test_cli_binary_is_built():
    assert os.access(piafs_b200.CLI_PATH, os.X_OK)


def test_batch_entry_points_argument_checks():
    lib = piafs_b200.load_library()
    h = ctypes.c_void_p()
    assert lib.piafs_gpu_batch_create(7, 0, ctypes.byref(h)) == 1
    assert lib.piafs_gpu_batch_create(0, 0, None) == 1
    assert lib.piafs_gpu_batch_step(None, 1) == 1
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        # no device: a CUDA error, reported, not a crash
        assert lib.piafs_gpu_batch_create(0, 0, ctypes.byref(h)) == 4
        assert lib.piafs_gpu_last_error()


HYPAR_HEADER = os.path.join(ROOT, "include", "piafs_hypar.h")
HYPAR_LIB = os.path.join(ROOT, "piafs_b200", "libpiafs_hypar.so")


def test_hypar_library_exports_every_declared_symbol():
    """libpiafs_hypar.so (built against the reference's headers) exports the
    entry points of include/piafs_hypar.h with the reference's
    function-pointer signatures."""
    if not os.path.exists(HYPAR_LIB):
        pytest.skip("libpiafs_hypar.so not built (the reference's headers were not available)")
    txt = re.sub(r"/\*.*?\*/", "", open(HYPAR_HEADER).read(), flags=re.S)
    names = sorted(set(re.findall(r"\b(piafs_gpu_\w+)\s*\(", txt)))
    assert "piafs_gpu_TimeRK_ts" in names and "piafs_gpu_attach" in names
    piafs_b200.load_library()
    lib = ctypes.CDLL(HYPAR_LIB)
    for name in names:
        assert isinstance(getattr(lib, name), ctypes._CFuncPtr), name
    # no simulation object: argument errors before any device work
    assert lib.piafs_gpu_attach(None, 1, 0, ctypes.c_double(0.0)) == 1
    assert lib.piafs_gpu_TimeRK_ts(None) == 1
