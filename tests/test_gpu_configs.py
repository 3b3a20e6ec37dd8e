"""Parity at the benchmarked sizes.

* The roots of the benchmark configurations (single-kb-2^16x64,
  uneven-kb-2^30, recursion-bb-48) and the FRI commit phase of fri-kb-2^23
  (roots, betas and final values for both stopping rules), committed by the
  CUDA path at full size from the benchmarks' own seeded inputs, against the
  values the CPU oracle computed once (tests/golden/config_roots.json, made by
  tests/golden/make_config_golden.py).  The batched and plain forms, device
  and host inputs, and default and autotuned LDE splits all have to give the
  golden root.
* The coset LDE of tall matrices (2^18 .. 2^22 rows, both fields) against the
  oracle, bit-exactly, for every four-step split the library accepts at each
  height, so that every sub-transform length of the three-pass kernels runs.

Integer field arithmetic: every comparison is bit-exact.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from pico_b200 import PicoError, Radix2DitParallel, TwoAdicDomain, TwoAdicFriPcs
from pico_b200 import fields as F

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden" / "config_roots.json"
COMMIT_CONFIGS = ["single-kb-2^16x64", "uneven-kb-2^30", "recursion-bb-48"]


@pytest.fixture(scope="module")
def config_golden():
    return json.loads(GOLDEN.read_text())


def device_traces(cfg, dev):
    f = F.field_id(cfg["field"])
    return [F.random_matrix_torch(f, lh, w, s, dev) for (lh, w), s in zip(cfg["shapes"], cfg["seeds"])]


def commit_root(gpu, cfg, traces, plain=False):
    f = F.field_id(cfg["field"])
    pcs = TwoAdicFriPcs(gpu, f, cfg["log_blowup"])
    doms = [TwoAdicDomain(lh) for lh, _ in cfg["shapes"]]
    root, _ = pcs.commit(list(zip(doms, traces)), plain=plain, keep=False)
    return root.tolist()


@pytest.mark.parametrize("name", COMMIT_CONFIGS)
def test_config_root_matches_golden(gpu, config_golden, name):
    import torch

    cfg = config_golden[name]
    f = F.field_id(cfg["field"])
    dev = torch.device("cuda", 0)
    traces = device_traces(cfg, dev)
    heights = [lh for lh, _ in cfg["shapes"]]
    saved = {l: gpu.lde_split(f, l) for l in range(12, 25)}
    try:
        assert commit_root(gpu, cfg, traces) == cfg["root"], "batched form, default splits"
        assert commit_root(gpu, cfg, traces, plain=True) == cfg["root"], "plain form"
        # the splits and block size the benchmark runs with
        gpu.autotune(f, max(12, min(heights)), max(12, max(heights)))
        assert commit_root(gpu, cfg, traces) == cfg["root"], "batched form, autotuned"
        # host inputs: the end-to-end path (copies and resumable row sponges)
        host = [t.cpu().numpy().view(np.uint32) for t in traces]
        del traces
        torch.cuda.empty_cache()
        assert commit_root(gpu, cfg, host) == cfg["root"], "host inputs"
    finally:
        for l, n1 in saved.items():
            gpu.lde_split(f, l, n1)


def test_fri_config_matches_golden(gpu, config_golden):
    import torch

    cfg = config_golden["fri-kb-2^23"]
    f, b = cfg["field"], cfg["log_blowup"]
    dev = torch.device("cuda", 0)
    base = F.random_matrix_torch(f, cfg["log_height"], cfg["width"], cfg["seed"], dev)
    cw = torch.empty((1 << (cfg["log_height"] + b), 4), dtype=torch.int32, device=dev)
    Radix2DitParallel(gpu, f).coset_lde_batch_bitrev(base, b, F.lde_shift(f), out=cw)
    pcs = TwoAdicFriPcs(gpu, f, b)
    for mode in ("final_1", "final_16"):
        want = cfg[mode]
        res = pcs.fri_commit_phase(cw, log_final_len=want["log_final_len"])
        assert res.roots.tolist() == want["roots"], mode
        assert res.betas.tolist() == want["betas"], mode
        assert res.final_poly.tolist() == want["final"], mode


# ---------------------------------------------------------------- tall LDEs
TALL = [(18, 3), (19, 3), (20, 2), (21, 2), (22, 1)]


def valid_splits(logn):
    return [n1 for n1 in range(6, 13) if 6 <= logn - n1 <= 12]


@pytest.mark.parametrize("f,b", [(0, 1), (1, 2)])
@pytest.mark.parametrize("logn,w", TALL)
def test_tall_lde_every_split(gpu, orc, f, b, logn, w):
    """Every split the library accepts at 2^18 .. 2^22 rows (sub-transform
    lengths 2^6 .. 2^12 in all three passes) gives the oracle's LDE."""
    m = orc.random_matrix(f, logn, w, 7100 + 31 * logn + f)
    shift = F.lde_shift(f)
    want = orc.coset_lde(f, m, b, shift)
    default = gpu.lde_split(f, logn)
    dft = Radix2DitParallel(gpu, f)
    try:
        for n1 in valid_splits(logn):
            assert gpu.lde_split(f, logn, n1) == n1
            got = dft.coset_lde_batch_bitrev(m, b, shift)
            assert (got == want).all(), (logn, n1)
    finally:
        gpu.lde_split(f, logn, default)


@pytest.mark.parametrize("f", [0, 1])
def test_wide_lde_2_20_every_split(gpu, orc, f):
    """2^20 x 70: tiles of several column groups per sub-transform, every split."""
    logn, w, b = 20, 70, 1
    m = orc.random_matrix(f, logn, w, 7300 + f)
    shift = F.lde_shift(f)
    want = orc.coset_lde(f, m, b, shift)
    default = gpu.lde_split(f, logn)
    dft = Radix2DitParallel(gpu, f)
    try:
        for n1 in valid_splits(logn):
            gpu.lde_split(f, logn, n1)
            got = dft.coset_lde_batch_bitrev(m, b, shift)
            assert (got == want).all(), n1
    finally:
        gpu.lde_split(f, logn, default)


@pytest.mark.parametrize("f,logn,b", [(0, 23, 1), (1, 24, 2)])
def test_lde_at_maximum_height(gpu, orc, f, logn, b):
    """The tallest LDEs each field allows: KoalaBear 2^23 rows at blowup 2
    (2^24 = its two-adicity), BabyBear 2^24 rows (the library's limit) at
    blowup 4, one column, at the default split and at the most unbalanced
    accepted one."""
    m = orc.random_matrix(f, logn, 1, 7400 + f)
    shift = F.lde_shift(f)
    want = orc.coset_lde(f, m, b, shift)
    default = gpu.lde_split(f, logn)
    dft = Radix2DitParallel(gpu, f)
    try:
        for n1 in (default, valid_splits(logn)[0]):
            gpu.lde_split(f, logn, n1)
            got = dft.coset_lde_batch_bitrev(m, b, shift)
            assert (got == want).all(), n1
    finally:
        gpu.lde_split(f, logn, default)
    if f == 0:  # one more doubling passes the two-adicity
        with pytest.raises(PicoError):
            dft.coset_lde_batch_bitrev(m, b + 1, shift)
