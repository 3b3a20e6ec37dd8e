"""CPU-side checks of the C ABI library: it builds for sm_100a, loads, exports
every symbol include/pico_gpu.h declares, and reports errors through status
codes (no compute calls: this container has no GPU)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def header_symbols():
    text = (ROOT / "include" / "pico_gpu.h").read_text()
    return sorted(set(re.findall(r"\b(pico_gpu_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from pico_b200 import abi

    lib = abi.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
        assert s in abi.SIGNATURES, f"{s} missing from the Python binding"


def test_abi_version():
    from pico_b200 import abi

    assert abi.load().pico_gpu_abi_version() == 1


def test_built_for_sm100a():
    from pico_b200 import build

    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_FLAGS)


def _has_gpu():
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device error path")
def test_init_without_device_reports_status():
    from pico_b200 import abi

    lib = abi.load()
    h = C.c_void_p()
    s = lib.pico_gpu_init(0, None, C.byref(h))
    assert s == 8  # PICO_ERR_NO_DEVICE
    assert b"no CUDA device" in lib.pico_gpu_last_error()
    assert not h.value


def test_null_arguments_are_rejected():
    from pico_b200 import abi

    lib = abi.load()
    assert lib.pico_gpu_init(0, None, None) == 1
    root = (C.c_uint32 * 8)()
    assert lib.pico_gpu_commit(None, 0, None, 0, 1, 0, None, root) == 1
    assert lib.pico_gpu_release(None, None) == 0  # releasing nothing is fine
    assert lib.pico_gpu_lde_shape(None, 0, None, None) == 1


def test_host_field_helpers_roundtrip():
    from pico_b200 import fields as F

    for f in (0, 1):
        x = F.uniform(f, 1000, 3)
        assert (x < F.P[f]).all()
        assert (F.from_monty(f, F.to_monty(f, x)) == x).all()
        assert F.monty(f, 1) == (1 << 32) % F.P[f]


def test_device_generator_matches_host():
    torch = pytest.importorskip("torch")
    from pico_b200 import fields as F

    for f in (0, 1):
        a = F.random_matrix(f, 9, 5, 42)
        b = F.random_matrix_torch(f, 9, 5, 42, "cpu").numpy().view(np.uint32)
        assert (a == b).all()
