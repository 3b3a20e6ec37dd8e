"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Integer field arithmetic: every comparison is bit-exact.  The shapes here are
small and medium (heights up to 2^17 for whole-LDE comparisons, 2^19 inside
commits); every LDE, digest layer and root is compared in full with the
oracle.  The benchmarked sizes (full-size roots, FRI at 2^23, LDEs of 2^18 ..
2^22 rows at every split) are in test_gpu_configs.py.
"""
import numpy as np
import pytest

from pico_b200 import (CommitServer, GpuContext, MerkleTreeMmcs, PicoError, Poseidon2, Radix2DitParallel,
                       TwoAdicDomain, TwoAdicFriPcs)
from pico_b200 import abi
from pico_b200 import fields as F

pytestmark = pytest.mark.gpu
FIELDS = [0, 1]


def _torch():
    import torch

    return torch


def to_dev(a):
    torch = _torch()
    return torch.from_numpy(a.view(np.int32)).cuda()


# ---------------------------------------------------------------- Poseidon2
@pytest.mark.parametrize("f", FIELDS)
def test_permute_kat_and_random(gpu, orc, golden, f):
    name = F.NAMES[f]
    zero = np.zeros((1, 16), dtype=np.uint32)
    Poseidon2(gpu, f).permute(zero)
    assert F.from_monty(f, zero[0]).tolist() == golden["kat"][name]["output"]
    st = F.to_monty(f, F.uniform(f, 16 * 1000, 5)).reshape(1000, 16)
    want = orc.permute(f, st)
    got = st.copy()
    Poseidon2(gpu, f).permute(got)
    assert (got == want).all()
    d = to_dev(st.copy())
    Poseidon2(gpu, f).permute(d)
    assert (d.cpu().numpy().view(np.uint32) == want).all()
    # the four-lane form, with a state count that leaves a partial warp
    for n in (1000, 7, 1):
        got = st[:n].copy()
        Poseidon2(gpu, f).permute(got, four_lanes=True)
        assert (got == want[:n]).all(), n


# ---------------------------------------------------------------- coset LDE
LDE_SHAPES = [(0, 3, 1), (1, 1, 1), (3, 2, 2), (4, 3, 2), (7, 9, 1), (10, 8, 1), (11, 13, 1), (11, 1, 3),
              (12, 5, 1), (12, 8, 2), (13, 8, 1), (14, 33, 1), (15, 2, 2), (16, 3, 1), (17, 12, 1)]


@pytest.mark.parametrize("f", FIELDS)
@pytest.mark.parametrize("logn,w,b", LDE_SHAPES)
def test_coset_lde(gpu, orc, f, logn, w, b):
    m = F.random_matrix(f, logn, w, 300 + logn * 7 + w)
    shift = F.lde_shift(f)
    want = orc.coset_lde(f, m, b, shift)
    got = Radix2DitParallel(gpu, f).coset_lde_batch_bitrev(m, b, shift)
    assert got.shape == want.shape
    assert (got == want).all()


@pytest.mark.parametrize("f", FIELDS)
def test_coset_lde_arbitrary_shift_and_natural_order(gpu, orc, f):
    m = F.random_matrix(f, 9, 6, 17)
    shift = F.to_monty(f, [123456789])[0]
    want = orc.coset_lde(f, m, 2, int(shift), bitrev=False)
    got = Radix2DitParallel(gpu, f).coset_lde_batch(m, 2, int(shift))
    assert (got == want).all()


def test_coset_lde_device_buffers(gpu, orc):
    torch = _torch()
    f = 0
    m = F.random_matrix(f, 13, 16, 8)
    out = torch.empty((1 << 14, 16), dtype=torch.int32, device="cuda")
    Radix2DitParallel(gpu, f).coset_lde_batch_bitrev(to_dev(m), 1, F.lde_shift(f), out=out)
    assert (out.cpu().numpy().view(np.uint32) == orc.coset_lde(f, m, 1, F.lde_shift(f))).all()


# ---------------------------------------------------------------- commits
def commit_both(gpu, orc, f, shapes, b, seed0, plain=False, device=False):
    mats = [F.random_matrix(f, lh, w, seed0 + i) for i, (lh, w) in enumerate(shapes)]
    want_root, want_ldes, want_layers = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b, want_ldes=True,
                                                       want_layers=True)
    pcs = TwoAdicFriPcs(gpu, f, b)
    ins = [to_dev(m) for m in mats] if device else mats
    root, pd = pcs.commit([(pcs.natural_domain_for_degree(m.shape[0]), m) for m in ins], plain=plain)
    return mats, root, pd, want_root, want_ldes, want_layers


@pytest.mark.parametrize("f", FIELDS)
@pytest.mark.parametrize("plain", [False, True])
def test_commit_golden_shapes(gpu, orc, golden, f, plain):
    pc = golden["vectors"][F.NAMES[f]]["pcs_commit"]
    mats = [F.random_matrix(f, lh, w, s) for lh, w, s in pc["shapes"]]
    pcs = TwoAdicFriPcs(gpu, f, pc["log_blowup"])
    root, pd = pcs.commit([(TwoAdicDomain(m.shape[0].bit_length() - 1), m) for m in mats], plain=plain)
    assert root.tolist() == pc["root"]
    pd.release()


@pytest.mark.parametrize("f", FIELDS)
def test_commit_single_matrix_config1(gpu, orc, f):
    """One 2^16 x 64 trace, log_blowup 1: the plain single-matrix commit."""
    mats, root, pd, want_root, want_ldes, want_layers = commit_both(gpu, orc, f, [(16, 64)], 1, 1)
    assert root.tolist() == want_root.tolist()
    assert (pd.lde(0) == want_ldes[0]).all()
    assert (pd.digest_layer(0) == want_layers[: 1 << 17]).all()


@pytest.mark.parametrize("f", FIELDS)
@pytest.mark.parametrize("b", [1, 2])
def test_commit_uneven_batch(gpu, orc, f, b):
    rng = np.random.default_rng(7 + f + b)
    shapes = [(int(rng.integers(4, 15)), int(rng.integers(1, 120))) for _ in range(24)]
    shapes += [(14, 8), (14, 3), (9, 400), (0, 5)]
    for plain in (False, True):
        mats, root, pd, want_root, want_ldes, want_layers = commit_both(gpu, orc, f, shapes, b, 500, plain=plain)
        assert root.tolist() == want_root.tolist()
        for i in range(len(mats)):
            assert (pd.lde(i) == want_ldes[i]).all()
        log_max = max(s[0] for s in shapes) + b
        off = 0
        for lvl in range(log_max + 1):
            n = 1 << (log_max - lvl)
            assert (pd.digest_layer(lvl) == want_layers[off:off + n]).all()
            off += n
        pd.release()


@pytest.mark.parametrize("f", FIELDS)
def test_lde_every_split_bit_exact(gpu, orc, f):
    """Every four-step split the autotuner may choose gives the same LDE."""
    for logn, w in ((12, 5), (13, 3), (14, 9)):
        m = F.random_matrix(f, logn, w, 40 + logn)
        want = orc.coset_lde(f, m, 1, F.lde_shift(f))
        default = gpu.lde_split(f, logn)
        try:
            for n1 in range(6, 13):
                if not 6 <= logn - n1 <= 12:
                    with pytest.raises(PicoError):
                        gpu.lde_split(f, logn, n1)
                    continue
                assert gpu.lde_split(f, logn, n1) == n1
                got = Radix2DitParallel(gpu, f).coset_lde_batch_bitrev(m, 1, F.lde_shift(f))
                assert (got == want).all(), (logn, n1)
        finally:
            gpu.lde_split(f, logn, default)


@pytest.mark.parametrize("f", FIELDS)
def test_autotune_keeps_parity(gpu, orc, f):
    rep = gpu.autotune(f, 12, 15)
    assert set(rep) >= {12, 13, 14, 15, "hash_block"}
    for l in range(12, 16):
        assert rep[l]["log_n1"] in rep[l]["ms"]
    shapes = [(15, 7), (13, 20), (12, 3), (9, 11)]
    mats, root, pd, want_root, want_ldes, _ = commit_both(gpu, orc, f, shapes, 1, 800 + f)
    assert root.tolist() == want_root.tolist()
    for i in range(len(mats)):
        assert (pd.lde(i) == want_ldes[i]).all()
    pd.release()


@pytest.mark.parametrize("f", FIELDS)
@pytest.mark.parametrize("packed_max", ["0", str(1 << 40)])
def test_commit_allocation_forms(gpu, orc, f, packed_max, monkeypatch):
    """A commit's buffers are two blocks (commits up to PICO_PACKED_COMMIT_BYTES)
    or one allocation each: both forms give the oracle's LDEs, layers and root,
    with host and with device inputs."""
    monkeypatch.setenv("PICO_PACKED_COMMIT_BYTES", packed_max)
    shapes = [(9, 30), (5, 3), (9, 1), (7, 64), (0, 2), (7, 5), (3, 0)]
    for device in (False, True):
        mats, root, pd, want_root, want_ldes, want_layers = commit_both(gpu, orc, f, shapes, 2, 1100 + f,
                                                                        device=device)
        assert root.tolist() == want_root.tolist()
        for i in range(len(mats)):
            assert (pd.lde(i) == want_ldes[i]).all()
        off = 0
        for lvl in range(pd.log_max_height + 1):
            got = pd.digest_layer(lvl)
            assert (got == want_layers[off:off + got.shape[0]]).all()
            off += got.shape[0]
        pd.release()


@pytest.mark.parametrize("f", FIELDS)
def test_commit_many_height_groups(gpu, orc, f):
    """Twenty height groups: the batched form hashes the shorter groups' rows
    in launches of at most 16 groups, so this commit needs two; root and every
    layer must match the oracle."""
    shapes = [(h, 1 + (h * 7) % 5) for h in range(19, -1, -1)]
    mats, root, pd, want_root, want_ldes, want_layers = commit_both(gpu, orc, f, shapes, 1, 1300 + f, device=True)
    assert root.tolist() == want_root.tolist()
    off = 0
    for lvl in range(pd.log_max_height + 1):
        got = pd.digest_layer(lvl)
        assert (got == want_layers[off:off + got.shape[0]]).all()
        off += got.shape[0]
    pd.release()


@pytest.mark.parametrize("f", FIELDS)
def test_commit_chained_sponge_odd_widths(gpu, orc, f):
    """Host inputs: a height group of many matrices is hashed matrix by matrix
    (resumable sponge); widths 1..17 put the matrix boundaries at every rate
    position.  Root and every layer must match the oracle, and the device-input
    (one-pass) commit of the same matrices."""
    shapes = [(6, w) for w in (1, 2, 3, 4, 5, 6, 7, 8, 9, 15, 17)] + [(4, 3), (4, 11), (2, 1)]
    for plain in (False, True):
        mats, root, pd, want_root, want_ldes, want_layers = commit_both(gpu, orc, f, shapes, 1, 700 + f, plain=plain)
        assert root.tolist() == want_root.tolist()
        for lvl in range(pd.log_max_height + 1):
            got = pd.digest_layer(lvl)
            off = sum(1 << (pd.log_max_height - l) for l in range(lvl))
            assert (got == want_layers[off:off + got.shape[0]]).all()
        pd.release()
    mats, root_dev, pd, want_root, _, _ = commit_both(gpu, orc, f, shapes, 1, 700 + f, device=True)
    assert root_dev.tolist() == want_root.tolist()
    pd.release()


def test_commit_device_inputs_and_rows(gpu, orc):
    f = 0
    shapes = [(12, 20), (10, 7), (12, 9)]
    mats, root, pd, want_root, want_ldes, _ = commit_both(gpu, orc, f, shapes, 1, 900, device=True)
    assert root.tolist() == want_root.tolist()
    assert (pd.lde_rows(1, 100, 300) == want_ldes[1][100:300]).all()
    torch = _torch()
    out = torch.empty((50, 20), dtype=torch.int32, device="cuda")
    pd.lde_rows(0, 7, 57, out=out)
    assert (out.cpu().numpy().view(np.uint32) == want_ldes[0][7:57]).all()


def verify_batch(orc, f, root, heights, index, opened, path):
    """MMCS opening check restated from the verifier (fri.rs:389-436)."""
    order = sorted(range(len(heights)), key=lambda i: -heights[i])
    log_max = heights[order[0]].bit_length() - 1
    cur_h = heights[order[0]]
    k = 0
    elems = []
    while k < len(order) and heights[order[k]] == cur_h:
        elems.append(opened[order[k]])
        k += 1
    node = orc.hash_elems(f, np.concatenate(elems) if elems else np.zeros(0, np.uint32))
    for lvl in range(log_max):
        bit = (index >> lvl) & 1
        sib = path[lvl]
        node = orc.compress(f, sib, node) if bit else orc.compress(f, node, sib)
        cur_h //= 2
        elems = []
        while k < len(order) and heights[order[k]] == cur_h:
            elems.append(opened[order[k]])
            k += 1
        if elems:
            node = orc.compress(f, node, orc.hash_elems(f, np.concatenate(elems)))
    return node.tolist() == list(root)


@pytest.mark.parametrize("f", FIELDS)
def test_open_batch_verifies(gpu, orc, f):
    shapes = [(10, 5), (8, 3), (10, 2), (6, 11)]
    mats, root, pd, want_root, want_ldes, _ = commit_both(gpu, orc, f, shapes, 1, 40)
    assert root.tolist() == want_root.tolist()
    mmcs = MerkleTreeMmcs(gpu, f)
    heights = [pd.lde_shape(i)[0] for i in range(len(mats))]
    for index in (0, 1, 777, (1 << 11) - 1):
        rows, path = mmcs.open_batch(index, pd)
        for i, r in enumerate(rows):
            assert (r == want_ldes[i][index >> (11 - heights[i].bit_length() + 1)]).all()
        assert verify_batch(orc, f, root, heights, index, rows, path)


@pytest.mark.parametrize("f", FIELDS)
def test_mmcs_commit_prebuilt_matrices(gpu, orc, f):
    mats = [F.random_matrix(f, 9, 3, 1), F.random_matrix(f, 7, 10, 2), F.random_matrix(f, 9, 16, 3)]
    want = orc.mmcs_commit(f, mats)
    root, pd = MerkleTreeMmcs(gpu, f).commit(mats)
    assert root.tolist() == want.tolist()
    root2, _ = MerkleTreeMmcs(gpu, f).commit([to_dev(m) for m in mats])
    assert root2.tolist() == want.tolist()


def test_invalid_shapes_are_reported(gpu):
    import ctypes as C

    from pico_b200 import abi

    pcs = TwoAdicFriPcs(gpu, 0, 1)
    with pytest.raises(ValueError):  # trace height differs from its domain
        pcs.commit([(TwoAdicDomain(4), np.zeros((10, 2), np.uint32))])
    m = np.zeros((16, 2), dtype=np.uint32)
    mats = (abi.Matrix * 1)()
    mats[0].values = m.ctypes.data
    mats[0].log_height = 23
    mats[0].width = 2
    root = (C.c_uint32 * 8)()
    # 2^23 rows with blowup 4 exceeds KoalaBear's two-adicity 24
    with pytest.raises(PicoError):
        abi.check(gpu.lib.pico_gpu_commit(gpu.handle, 0, mats, 1, 2, 0, None, root))
    # BabyBear admits 2^25 x 2, but LDE inputs above 2^24 rows are refused
    # before any buffer is touched
    mats[0].log_height = 25
    with pytest.raises(PicoError) as e:
        abi.check(gpu.lib.pico_gpu_commit(gpu.handle, 1, mats, 1, 1, 0, None, root))
    assert e.value.status == abi.PICO_ERR_UNSUPPORTED


# ---------------------------------------------------------------- FRI
def ef4_codeword(f, log_trace, b, seed):
    base = F.random_matrix(f, log_trace, 4, seed)
    import oracle.cpu as o

    return o.coset_lde(f, base, b, F.lde_shift(f))


@pytest.mark.parametrize("f", FIELDS)
@pytest.mark.parametrize("log_trace,b", [(5, 1), (10, 1), (9, 2), (14, 1)])
def test_fri_commit_phase_challenger(gpu, orc, f, log_trace, b):
    cw = ef4_codeword(f, log_trace, b, 60 + log_trace)
    roots, betas, final, ch = orc.fri_commit_phase(f, cw, b)
    res = TwoAdicFriPcs(gpu, f, b).fri_commit_phase(cw)
    assert res.rounds == log_trace
    assert (res.roots == roots).all()
    assert (res.betas == betas).all()
    assert (res.final_poly[0] == final[0]).all()


@pytest.mark.parametrize("f", FIELDS)
def test_fri_commit_phase_explicit_betas_and_early_stop(gpu, orc, f):
    b = 1
    cw = ef4_codeword(f, 11, b, 70)
    betas = F.to_monty(f, F.uniform(f, 4 * 11, 71)).reshape(11, 4)
    roots, _, final, _ = orc.fri_commit_phase(f, cw, b, 0, betas=betas)
    res = TwoAdicFriPcs(gpu, f, b).fri_commit_phase(cw, betas=betas)
    assert (res.roots == roots).all() and (res.final_poly[0] == final[0]).all()
    roots4, betas4, final4, _ = orc.fri_commit_phase(f, cw, b, 4)
    res4 = TwoAdicFriPcs(gpu, f, b).fri_commit_phase(cw, log_final_len=4, keep=True)
    assert (res4.roots == roots4).all() and (res4.betas == betas4).all()
    assert (res4.final_poly == final4).all()
    assert (res4.data.layer(0) == cw).all()
    res4.data.release()


def test_fri_rejects_high_degree_codeword(gpu):
    cw = F.to_monty(0, F.uniform(0, 4 * 64, 3)).reshape(64, 4)  # random: not low degree
    with pytest.raises(PicoError):
        TwoAdicFriPcs(gpu, 0, 1).fri_commit_phase(cw)


# ---------------------------------------------------------------- serving
def test_serving_results_match_alone(gpu, orc):
    """Each request's root is the same when run alone and in a concurrent mix."""
    server = CommitServer(gpu)
    rng = np.random.default_rng(3)
    reqs = []
    for k in range(12):
        f = int(rng.random() < 0.3)
        b = int(rng.integers(1, 3))
        shapes = [(int(rng.integers(3, 13)), int(rng.integers(1, 64))) for _ in range(int(rng.integers(1, 6)))]
        mats = [F.random_matrix(f, lh, w, 1000 * k + i) for i, (lh, w) in enumerate(shapes)]
        reqs.append((f, b, mats, server.submit(f, mats, b)))
    for f, b, mats, r in reqs:
        root, pd = r.wait(timeout_ms=60000)
        alone, _ = TwoAdicFriPcs(gpu, f, b).commit([(TwoAdicDomain(m.shape[0].bit_length() - 1), m) for m in mats],
                                                   keep=False)
        want, _, _ = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b)
        assert root.tolist() == alone.tolist() == want.tolist()
        q, run = r.times()
        assert q >= 0 and run > 0
        pd.release()
        r.free()
    assert gpu.memory()[0] == 0


# ------------------------------------------- extension traces, domain reads
@pytest.mark.parametrize("f", FIELDS)
def test_extension_trace_commits_as_its_flattening(gpu, orc, f):
    """A permutation trace of EF4 elements (prover.rs:404-415) commits as
    flatten_to_base makes it: each element's c0..c3 in place, 4w base columns."""
    pcs = TwoAdicFriPcs(gpu, f, 1)
    ext = [F.random_matrix(f, lh, 4 * w, 700 + lh).reshape(1 << lh, w, 4) for lh, w in ((6, 3), (4, 5), (6, 1))]
    flat = [np.ascontiguousarray(e.reshape(e.shape[0], -1)) for e in ext]
    doms = [pcs.natural_domain_for_degree(e.shape[0]) for e in ext]
    root_ext, pd = pcs.commit(list(zip(doms, ext)))
    root_flat, _ = pcs.commit(list(zip(doms, flat)), keep=False)
    want, _, _ = orc.pcs_commit(f, flat, [F.lde_shift(f)] * len(flat), 1)
    assert (root_ext == want).all() and (root_flat == want).all()
    assert pd.lde_shape(0) == (128, 12)


@pytest.mark.parametrize("f", FIELDS)
@pytest.mark.parametrize("log_n,b,extra", [(5, 1, 1), (5, 1, 0), (6, 2, 1), (6, 2, 2), (4, 2, -1), (0, 1, 1)])
def test_evaluations_on_domain(gpu, orc, f, log_n, b, extra):
    """get_evaluations_on_domain(g * H_(2^(log_n + extra))): natural-order
    evaluations, i.e. the natural-order coset LDE at stride 2^(b - extra)."""
    pcs = TwoAdicFriPcs(gpu, f, b)
    t = F.random_matrix(f, log_n, 3, 900 + log_n)
    _, pd = pcs.commit([(pcs.natural_domain_for_degree(1 << log_n), t)])
    ld = log_n + extra
    got = pd.evaluations_on_domain(0, ld)
    nat = orc.coset_lde(f, t, b, F.lde_shift(f), bitrev=False)
    assert np.array_equal(got, nat[:: 1 << (log_n + b - ld)])
    torch = _torch()
    dev = torch.zeros((1 << ld, 3), dtype=torch.int32, device="cuda")
    pd.evaluations_on_domain(0, ld, out=dev)
    assert np.array_equal(dev.cpu().numpy().view(np.uint32), got)
    with pytest.raises(PicoError):
        pd.evaluations_on_domain(0, log_n + b + 1)


def test_grouped_requests_match_alone(orc, tmp_path, monkeypatch):
    """Continuous batching: with max_group > 1, device-input requests queued
    behind a running one are admitted together and share their LDE and
    row-hashing launches; every root is the one the request gets alone (and
    the oracle's), across mixed blowups, heights, width-0 matrices and both
    fields (which never share a group)."""
    import json

    torch = _torch()
    log = tmp_path / "metrics.jsonl"
    monkeypatch.setenv("PICO_METRICS_LOG", str(log))
    ctx = GpuContext(0, n_streams=2, max_inflight=1, max_group=8)
    try:
        server = CommitServer(ctx)
        rng = np.random.default_rng(17)
        big = torch.from_numpy(F.random_matrix(0, 18, 64, 77).view(np.int32)).cuda()
        reqs = [(0, 2, [big], server.submit(0, [big], 2))]  # runs while the others queue
        for k in range(14):
            f = 1 if k in (4, 9) else 0
            b = int(rng.integers(1, 3))
            shapes = [(int(rng.integers(3, 14)), int(rng.integers(0, 40))) for _ in range(int(rng.integers(1, 7)))]
            mats = [torch.from_numpy(F.random_matrix(f, lh, w, 2000 * k + i).view(np.int32)).cuda()
                    for i, (lh, w) in enumerate(shapes)]
            reqs.append((f, b, mats, server.submit(f, mats, b)))
        for f, b, mats, r in reqs:
            root, pd = r.wait(timeout_ms=120000)
            host = [m.cpu().numpy().view(np.uint32) for m in mats]
            alone, _ = TwoAdicFriPcs(ctx, f, b).commit(
                [(TwoAdicDomain(m.shape[0].bit_length() - 1), m) for m in host], keep=False)
            assert root.tolist() == alone.tolist()
            if len(host) > 1 or host[0].shape[0] < (1 << 18):
                want, _, _ = orc.pcs_commit(f, host, [F.lde_shift(f)] * len(host), b)
                assert root.tolist() == want.tolist()
            # the prover data of a grouped member reads back like any commit's
            k = int(np.argmax([m.shape[0] * m.shape[1] for m in host]))
            if host[k].shape[1]:
                lde = pd.lde_rows(k, 0, 4)
                assert lde.shape == (4, host[k].shape[1])
            pd.release()
            r.free()
        assert ctx.memory()[0] == 0
    finally:
        ctx.close()
    groups = [json.loads(l)["group"] for l in log.read_text().splitlines() if json.loads(l)["kind"] == "request"]
    assert len(groups) == 15 and max(groups) > 1


@pytest.mark.parametrize("f,b,k", [(0, 1, 1), (1, 2, 2), (0, 2, 1), (1, 1, 0)])
def test_row_split_commit(gpu, orc, f, b, k):
    """pico_gpu_commit_shard: shard s of 2^k holds rows [s N / 2^k, (s+1) N / 2^k)
    of every committed LDE (both LDE forms, heights 2^0 .. 2^14) and its
    root is the full tree's node s at depth k; merkle_top over the shard
    roots is the commitment root.  More shards than coset blocks is refused."""
    from pico_b200.pcs import merkle_top

    shapes = [(14, 3), (12, 2), (9, 5), (6, 1), (0, 2)]
    mats = [F.random_matrix(f, lh, w, 9100 + 17 * i + f) for i, (lh, w) in enumerate(shapes)]
    pcs = TwoAdicFriPcs(gpu, f, b)
    doms = [pcs.natural_domain_for_degree(m.shape[0]) for m in mats]
    full, pd_full = pcs.commit(list(zip(doms, mats)))
    want, ldes, layers = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b, want_ldes=True, want_layers=True)
    assert full.tolist() == want.tolist()
    depth_k = layers[len(layers) - (2 << k) + 1: len(layers) - (1 << k) + 1]
    subs = []
    for s in range(1 << k):
        sub, pd = pcs.commit_shard(list(zip(doms, mats)), k, s)
        assert sub.tolist() == depth_k[s].tolist(), s
        if k:  # a shard holds a slice of the rows: calls that need all of them refuse it
            with pytest.raises(PicoError) as e:
                pd.evaluations_on_domain(0, shapes[0][0])
            assert e.value.status == abi.PICO_ERR_UNSUPPORTED
        for i, l in enumerate(ldes):
            rows = l.shape[0] >> k
            assert pd.lde_shape(i) == (rows, l.shape[1])
            if l.shape[1]:
                assert np.array_equal(pd.lde_rows(i), l[s * rows:(s + 1) * rows]), (s, i)
        pd.release()
        subs.append(sub)
    assert merkle_top(f, np.stack(subs)).tolist() == want.tolist()
    pd_full.release()
    with pytest.raises(PicoError):
        pcs.commit_shard(list(zip(doms, mats)), b + 1, 0, keep=False)
    with pytest.raises(PicoError) as e:  # a shard index past the last shard
        pcs.commit_shard(list(zip(doms, mats)), k, 1 << k, keep=False)
    assert e.value.status == abi.PICO_ERR_INVALID_ARG
    assert gpu.memory()[0] == 0


def test_row_split_commit_device_inputs_at_2_20(gpu, orc):
    """Two shards of a 2^20-row commit from device inputs (three-pass LDE at
    the autotuner's default split): shard roots and the combined root."""
    from pico_b200.pcs import merkle_top

    torch = _torch()
    f, b = 0, 1
    host = [F.random_matrix(f, 20, 4, 9200), F.random_matrix(f, 17, 3, 9201)]
    dev = [torch.from_numpy(m.view(np.int32)).cuda() for m in host]
    pcs = TwoAdicFriPcs(gpu, f, b)
    doms = [pcs.natural_domain_for_degree(m.shape[0]) for m in host]
    want, _, _ = orc.pcs_commit(f, host, [F.lde_shift(f)] * 2, b)
    subs = [pcs.commit_shard(list(zip(doms, dev)), 1, s, keep=False)[0] for s in range(2)]
    assert merkle_top(f, np.stack(subs)).tolist() == want.tolist()


def test_commit_sharded_over_a_one_rank_group(orc, tmp_path):
    """pico_b200.sharded.commit_sharded on a one-rank gloo group (this GPU is
    shard 0 of 1): the product path end to end, all-gather included."""
    import socket

    import torch.distributed as dist

    from pico_b200.sharded import commit_sharded

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    ctx = GpuContext(0)
    try:
        f, b = 1, 2
        mats = [F.random_matrix(f, lh, w, 9300 + lh) for lh, w in ((12, 6), (10, 3))]
        pcs = TwoAdicFriPcs(ctx, f, b)
        root, pd, sub = commit_sharded(pcs, [(TwoAdicDomain(m.shape[0].bit_length() - 1), m) for m in mats])
        want, _, _ = orc.pcs_commit(f, mats, [F.lde_shift(f)] * 2, b)
        assert root.tolist() == sub.tolist() == want.tolist()
        pd.release()
    finally:
        ctx.close()
        dist.destroy_process_group()


@pytest.mark.parametrize("dev_in", [False, True])
@pytest.mark.parametrize("plain", [False, True])
def test_commit_with_more_matrices_per_height_than_one_launch(gpu, orc, dev_in, plain):
    """70 matrices of one height (more than the 64 segments one row-hashing
    launch concatenates) plus a shorter group: that height's rows are absorbed
    matrix by matrix through the resumable sponge, bit-exact with the oracle;
    served, such a request runs alone."""
    f, b = 0, 1
    shapes = [(6, 1 + i % 3) for i in range(70)] + [(4, 2), (6, 0)]
    mats = [F.random_matrix(f, lh, w, 9500 + i) for i, (lh, w) in enumerate(shapes)]
    want, _, _ = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b)
    inputs = mats
    if dev_in:
        torch = _torch()
        inputs = [torch.from_numpy(m.view(np.int32)).cuda() for m in mats]
    pcs = TwoAdicFriPcs(gpu, f, b)
    root, _ = pcs.commit([(TwoAdicDomain(lh), m) for (lh, _), m in zip(shapes, inputs)], plain=plain, keep=False)
    assert root.tolist() == want.tolist()
    if not plain:
        req = CommitServer(gpu).submit(f, inputs, b)
        got, _ = req.wait(timeout_ms=60_000, keep=False)
        req.free()
        assert got.tolist() == want.tolist()
    assert gpu.memory()[0] == 0


@pytest.mark.parametrize("f", FIELDS)
def test_row_split_commit_with_extension_traces(gpu, orc, f):
    """A permutation trace of EF4 elements in a row-split commit: each shard
    holds its rows of the flattened (4w-column) LDE, and the shard roots
    combine to the root of the flattened commit."""
    from pico_b200.pcs import merkle_top

    b, k = 2, 2
    ext = F.random_matrix(f, 9, 12, 9600 + f).reshape(1 << 9, 3, 4)
    base = F.random_matrix(f, 10, 5, 9610 + f)
    pcs = TwoAdicFriPcs(gpu, f, b)
    items = [(pcs.natural_domain_for_degree(1 << 10), base), (pcs.natural_domain_for_degree(1 << 9), ext)]
    flat = [base, np.ascontiguousarray(ext.reshape(1 << 9, 12))]
    want, _, _ = orc.pcs_commit(f, flat, [F.lde_shift(f)] * 2, b)
    subs = [pcs.commit_shard(items, k, s, keep=False)[0] for s in range(1 << k)]
    assert merkle_top(f, np.stack(subs)).tolist() == want.tolist()


@pytest.mark.parametrize("f,k,lf", [(0, 1, 0), (1, 2, 0), (0, 2, 4), (1, 3, 2)])
def test_fri_row_split_matches_one_device(gpu, orc, f, k, lf):
    """The FRI commit phase split by rows over 2^k shards (every shard on this
    GPU in turn, as 2^k ranks would run them side by side): roots, betas,
    final polynomial and the challenger afterwards equal the one-device
    phase's and the oracle's."""
    from pico_b200.pcs import new_challenger
    from pico_b200.sharded import fri_commit_phase_split

    cw = orc.coset_lde(f, F.random_matrix(f, 13, 4, 9700 + f), 1, F.lde_shift(f))  # 2^14 EF4 rows
    pcs = TwoAdicFriPcs(gpu, f, 1)
    roots, betas, final, ch = fri_commit_phase_split(pcs, cw, k, log_final_len=lf, min_log_rows=4)
    want_r, want_b, want_f, want_ch = orc.fri_commit_phase(f, cw, 1, lf)
    assert np.array_equal(roots, want_r) and np.array_equal(betas, want_b)
    assert np.array_equal(final, want_f)
    one_ch = new_challenger()
    one = pcs.fri_commit_phase(cw, log_final_len=lf, challenger=one_ch)
    assert np.array_equal(one.roots, roots) and np.array_equal(one.betas, betas)
    assert bytes(one_ch) == bytes(ch)
    assert gpu.memory()[0] == 0


def test_fri_sharded_over_a_one_rank_group(orc):
    """fri_commit_phase_sharded through a one-rank gloo group (its gathers
    included): the one shard folds on the device until 2^4 rows remain."""
    import socket

    import torch.distributed as dist

    from pico_b200.sharded import fri_commit_phase_sharded

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    ctx = GpuContext(0)
    try:
        f = 0
        cw = orc.coset_lde(f, F.random_matrix(f, 11, 4, 9750), 1, F.lde_shift(f))
        roots, betas, final, _ = fri_commit_phase_sharded(TwoAdicFriPcs(ctx, f, 1), cw, 12, min_log_rows=4)
        want_r, want_b, want_f, _ = orc.fri_commit_phase(f, cw, 1, 0)
        assert np.array_equal(roots, want_r) and np.array_equal(betas, want_b) and np.array_equal(final, want_f)
    finally:
        ctx.close()
        dist.destroy_process_group()


@pytest.mark.parametrize("f,b,k", [(0, 1, 1), (1, 2, 2)])
def test_row_split_open_batch(gpu, f, b, k):
    """Mmcs::open_batch of a row-split commit: the owning shard's open_batch at
    the index's row within the shard, plus merkle_top_path over the shard
    roots, equals open_batch on the whole commit (rows and path)."""
    from pico_b200.pcs import merkle_top_path

    shapes = [(11, 3), (9, 5), (11, 2), (4, 1)]
    mats = [F.random_matrix(f, lh, w, 9800 + 5 * i + f) for i, (lh, w) in enumerate(shapes)]
    pcs = TwoAdicFriPcs(gpu, f, b)
    items = [(pcs.natural_domain_for_degree(m.shape[0]), m) for m in mats]
    _, full = pcs.commit(items)
    shards = [pcs.commit_shard(items, k, s) for s in range(1 << k)]
    roots = np.stack([r for r, _ in shards])
    mmcs = MerkleTreeMmcs(gpu, f)
    log_max = 11 + b
    rng = np.random.default_rng(3)
    for index in list(rng.integers(0, 1 << log_max, size=12)) + [0, (1 << log_max) - 1]:
        index = int(index)
        s, local = index >> (log_max - k), index & ((1 << (log_max - k)) - 1)
        rows, path = mmcs.open_batch(local, shards[s][1])
        want_rows, want_path = mmcs.open_batch(index, full)
        assert all(np.array_equal(a, w) for a, w in zip(rows, want_rows))
        assert np.array_equal(np.concatenate([path, merkle_top_path(f, roots, s)]), want_path)
    for _, pd in shards:
        pd.release()
    full.release()
