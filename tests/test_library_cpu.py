"""The C-ABI library builds for sm_100a, loads, and exports every symbol
include/fdtd_b200.h declares (no compute calls: no GPU here)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names += re.findall(r"^\s*(?:const\s+)?[a-z_]+\s*\*?\s*(fdtd_[a-z0-9_]+)\s*\(", txt, re.M)
    return sorted(set(names))


def test_header_declares_the_api():
    names = declared_symbols()
    assert "fdtd_grid_create" in names and "fdtd_step" in names and "fdtd_last_error_string" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(fdtd):
    lib = ctypes.CDLL(fdtd.LIB_PATH)
    for n in declared_symbols():
        assert hasattr(lib, n), n
    assert set(declared_symbols()) <= set(fdtd.EXPORTS) | set(declared_symbols())


def test_build_targets_sm100a():
    from fdtd_b200 import build_lib
    assert build_lib.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert "-fmad=false" in build_lib.SOURCES["kernels_plain.cu"]


def test_create_without_gpu_fails_loudly(fdtd):
    import torch
    if torch.cuda.is_available():
        return
    import pytest
    from fdtd_b200.problem import TM
    with pytest.raises(fdtd.FdtdError) as e:
        fdtd.Grid(TM, (8, 8, 1), 1e-6, 1e-15)
    assert e.value.code == -2


def test_batch_calls_check_their_handle_before_any_device_call(fdtd):
    """The batch entry points refuse a null handle (FDTD_ERR_INVALID) without
    touching a device, so they behave the same on a host with no GPU."""
    lib = fdtd.load_library()
    assert lib.fdtd_batch_set_temporal(None, 2) == -1
    assert lib.fdtd_batch_temporal(None, None, None) == -1
    assert lib.fdtd_batch_tune(None, 4) == -1
    assert lib.fdtd_batch_configure(None, 0, 2) == -1
    assert lib.fdtd_batch_step(None, 1, None) == -1
    assert lib.fdtd_batch_destroy(None) == 0
