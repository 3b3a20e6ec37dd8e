"""The host DuplexChallenger behind pico_gpu_pcs_open, through the C ABI
(pico_gpu_challenger_observe / _sample), against the oracle's challenger
(vm/src/compiler/recursion/circuit/challenger.rs:89-106, 223-234 restated).
No device is needed: the library loads and runs these on the CPU.  The scalar,
AVX2 and AVX-512 forms of the host permutation are compared with one another
in child processes (the form is chosen once per process)."""
import ctypes as C
import json
import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
P = {0: 0x7F000001, 1: 0x78000001}


def _lib():
    from pico_b200 import abi

    return abi, abi.load()


def _script(field: int, seed: int) -> list:
    """A transcript of observe and sample steps of varied lengths, covering
    partial rate blocks, samples after observes and runs of samples."""
    rng = np.random.default_rng(seed)
    steps = []
    for _ in range(40):
        if rng.random() < 0.6:
            n = int(rng.integers(0, 21))
            steps.append(("o", rng.integers(0, P[field], size=n, dtype=np.uint64).astype(np.uint32)))
        else:
            steps.append(("s", int(rng.integers(1, 12))))
    return steps


def _run_abi(field: int, steps) -> tuple:
    abi, lib = _lib()
    ch = abi.Challenger()
    out = []
    for kind, arg in steps:
        if kind == "o":
            vals = np.ascontiguousarray(arg, dtype=np.uint32)
            abi.check(lib.pico_gpu_challenger_observe(field, C.byref(ch), vals.ctypes.data, len(vals)))
        else:
            buf = np.zeros(arg, dtype=np.uint32)
            abi.check(lib.pico_gpu_challenger_sample(field, C.byref(ch), buf.ctypes.data, arg))
            out.extend(int(v) for v in buf)
    return out, list(ch.sponge)


def _run_oracle(orc, field: int, steps) -> tuple:
    ch = orc.new_challenger()
    out = []
    for kind, arg in steps:
        if kind == "o":
            for v in arg:
                orc.challenger_observe(field, ch, int(v))
        else:
            out.extend(int(orc.challenger_sample(field, ch)) for _ in range(arg))
    return out, list(ch.sponge)


@pytest.mark.parametrize("field", [0, 1])
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_host_challenger_matches_oracle(orc, field, seed):
    steps = _script(field, seed)
    assert _run_abi(field, steps) == _run_oracle(orc, field, steps)


def test_host_challenger_edge_values(orc):
    # 0 and p - 1 in every position of several rate blocks
    for field in (0, 1):
        vals = np.array([0, P[field] - 1] * 20, dtype=np.uint32)
        steps = [("o", vals), ("s", 9), ("o", vals[:3]), ("s", 1)]
        assert _run_abi(field, steps) == _run_oracle(orc, field, steps)


_CHILD = r"""
import json, sys
sys.path.insert(0, sys.argv[1])
import numpy as np
from tests.test_host_challenger import _script, _run_abi
res = {f: _run_abi(f, _script(f, 7)) for f in (0, 1)}
print(json.dumps(res))
"""


def _child(level: str) -> dict:
    env = dict(os.environ, PICO_HOST_SIMD=level)
    r = subprocess.run([sys.executable, "-c", _CHILD, str(ROOT)], env=env, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_host_permutation_forms_agree():
    """Scalar, AVX2 (where the CPU has it) and AVX-512 (where it has it) give
    the same transcript; on a CPU without a form the cap falls back, so the
    comparison still holds."""
    scalar = _child("0")
    assert _child("2") == scalar
    assert _child("3") == scalar


def test_host_challenger_rejects_bad_arguments():
    abi, lib = _lib()
    ch = abi.Challenger()
    v = np.zeros(4, dtype=np.uint32)
    assert lib.pico_gpu_challenger_observe(7, C.byref(ch), v.ctypes.data, 4) == abi.PICO_ERR_INVALID_ARG
    assert lib.pico_gpu_challenger_sample(0, None, v.ctypes.data, 4) == abi.PICO_ERR_INVALID_ARG
    assert lib.pico_gpu_challenger_observe(0, C.byref(ch), None, 4) == abi.PICO_ERR_INVALID_ARG
    ch.in_len = 9  # not a state the challenger can be in
    assert lib.pico_gpu_challenger_sample(0, C.byref(ch), v.ctypes.data, 4) == abi.PICO_ERR_INVALID_ARG
    ch.in_len = 0
    assert lib.pico_gpu_challenger_observe(0, C.byref(ch), None, 0) == abi.PICO_OK
