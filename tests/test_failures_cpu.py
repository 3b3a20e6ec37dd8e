"""Failure detection on the host, without a device: malformed descriptors are
refused with a status code before anything touches the GPU (the reference
panics on misuse instead, vm/src/instances/machine/riscv.rs:106-110).

pico_gpu_commit_bytes plans a commit exactly as pico_gpu_commit and
pico_gpu_submit_commit do, so its validation is theirs; the allocation-free
LDE checks its arguments and its scratch limit before its first CUDA call.
"""
import ctypes as C

import numpy as np
import pytest

from pico_b200 import abi
from pico_b200 import fields as F


def descriptors(shapes, flags=0):
    bufs = [np.zeros((1 << lh, w), dtype=np.uint32) for lh, w in shapes]
    mats = (abi.Matrix * max(len(shapes), 1))()
    for k, ((lh, w), b) in enumerate(zip(shapes, bufs)):
        mats[k].values = b.ctypes.data
        mats[k].log_height = lh
        mats[k].width = w
        mats[k].shift = F.lde_shift(0)
        mats[k].flags = flags
    return mats, bufs


def commit_bytes(field, mats, n, b, flags=0):
    lib = abi.load()
    res, scr = C.c_uint64(), C.c_uint64()
    s = lib.pico_gpu_commit_bytes(field, mats, n, b, flags, C.byref(res), C.byref(scr))
    return s, res.value, scr.value


def test_commit_bytes_of_a_valid_commit():
    mats, _ = descriptors([(10, 5), (8, 3), (12, 0)])
    s, res, scr = commit_bytes(0, mats, 3, 1)
    assert s == abi.PICO_OK
    # resident: the three LDEs (2^11 x 5, 2^9 x 3, 2^13 x 0) and the digest layers of 2^13 leaves
    assert res >= 4 * ((5 << 11) + (3 << 9)) + 32 * ((2 << 13) - 1)
    assert scr > 0


@pytest.mark.parametrize("case", ["null_values", "too_tall", "flags", "blowup", "field", "none", "two_adicity"])
def test_malformed_descriptors_are_refused(case):
    mats, _ = descriptors([(10, 5), (6, 2)])
    field, n, b = 0, 2, 1
    want = abi.PICO_ERR_INVALID_ARG
    if case == "null_values":
        mats[1].values = None
    elif case == "too_tall":
        mats[0].log_height = 31
    elif case == "flags":
        mats[0].flags = 0x80
    elif case == "blowup":
        b = 17  # coset power tables are indexed in 32 bits up to log_blowup 16
    elif case == "field":
        field = 5
    elif case == "none":
        n = 0
    elif case == "two_adicity":
        mats[0].log_height = 23
        b = 2  # 2^25 LDE rows exceed KoalaBear's two-adicity 24
    s, _, _ = commit_bytes(field, mats, n, b)
    assert s == want, abi.load().pico_gpu_last_error()
    assert abi.load().pico_gpu_last_error()


def test_unsupported_lde_height_is_refused():
    mats, _ = descriptors([(3, 2)])
    mats[0].log_height = 25  # BabyBear admits 2^25 rows, but LDE inputs stop at 2^24
    s, _, _ = commit_bytes(1, mats, 1, 1)
    assert s == abi.PICO_ERR_UNSUPPORTED


def test_noalloc_refuses_bad_arguments_before_touching_the_device():
    lib = abi.load()
    buf = np.zeros(64, dtype=np.uint32)
    p = buf.ctypes.data
    assert lib.pico_gpu_coset_lde_batch_noalloc(3, p, 4, 2, 1, 1, p, None) == abi.PICO_ERR_INVALID_ARG  # field
    assert lib.pico_gpu_coset_lde_batch_noalloc(0, None, 4, 2, 1, 1, p, None) == abi.PICO_ERR_INVALID_ARG  # input
    assert lib.pico_gpu_coset_lde_batch_noalloc(0, p, 4, 2, 17, 1, p, None) == abi.PICO_ERR_INVALID_ARG  # blowup
    assert lib.pico_gpu_coset_lde_batch_noalloc(0, p, 23, 2, 2, 1, p, None) == abi.PICO_ERR_INVALID_ARG  # 2^25 rows
    # 2^20 x 64 at blowup 4 needs far more than the static scratch
    assert lib.pico_gpu_coset_lde_batch_noalloc(0, p, 20, 64, 2, 1, p, None) == abi.PICO_ERR_INVALID_ARG
    assert b"static scratch" in lib.pico_gpu_last_error()


def test_serving_calls_refuse_null_handles():
    lib = abi.load()
    root = (C.c_uint32 * 8)()
    assert lib.pico_gpu_poll(None, None) == abi.PICO_ERR_INVALID_ARG
    assert lib.pico_gpu_wait(None, None, 0, None, root) == abi.PICO_ERR_INVALID_ARG
    assert lib.pico_gpu_cancel(None, None) == abi.PICO_ERR_INVALID_ARG
    assert lib.pico_gpu_request_times(None, None, None) == abi.PICO_ERR_INVALID_ARG
    h = C.c_void_p()
    mats, _ = descriptors([(4, 2)])
    assert lib.pico_gpu_submit_commit(None, 0, mats, 1, 1, 0, C.byref(h)) == abi.PICO_ERR_INVALID_ARG
