"""Parity of the PCS opening (TwoAdicFriPcs::open) on the GPU with the oracle.

Bit-exact: opened values, reduced openings, commit-phase roots and betas, the
final element, the proof-of-work witness, query indices and query records.
Every GPU proof is also run through the oracle's restatement of the Pico
verifier (vm/src/compiler/recursion/circuit/fri.rs:77-436), which is how the
larger shapes are checked.
"""
import copy

import numpy as np
import pytest

from pico_b200 import PicoError, TwoAdicFriPcs, abi
from pico_b200 import fields as F

pytestmark = pytest.mark.gpu


def rand_ef(f, rng):
    return F.to_monty(f, rng.integers(0, F.P[f], size=4, dtype=np.uint64).astype(np.uint32))


def new_oracle_challenger(orc, f, observed):
    """A prover challenger that has already observed some transcript."""
    ch = orc.new_challenger()
    for v in observed:
        orc.challenger_observe(f, ch, int(F.monty(f, v)))
    return ch


def challenger_state(ch):
    return (list(ch.sponge), list(ch.in_buf)[: ch.in_len], list(ch.out_buf)[: ch.out_len])


def to_gpu_challenger(ch):
    out = abi.Challenger()
    if ch is not None:
        for name in ("sponge", "in_buf", "out_buf"):
            getattr(out, name)[:] = list(getattr(ch, name))
        out.in_len, out.out_len = ch.in_len, ch.out_len
    return out


def setup(gpu, orc, f, b, shapes, points_fn, seed, oracle=True):
    """Commit every batch on the GPU (resident) and, for the oracle, on the CPU."""
    pcs = TwoAdicFriPcs(gpu, f, b)
    rounds, obatches = [], []
    for bi, shp in enumerate(shapes):
        mats = [F.random_matrix(f, logn, w, seed + 31 * bi + 7 * m) for m, (logn, w) in enumerate(shp)]
        root, pd = pcs.commit([(pcs.natural_domain_for_degree(1 << logn), t) for (logn, _), t in zip(shp, mats)])
        pts = [points_fn(bi, m, logn) for m, (logn, _) in enumerate(shp)]
        rounds.append((pd, pts))
        if oracle:
            oroot, ldes, layers = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b, want_ldes=True,
                                                  want_layers=True)
            assert (oroot == root).all()
            obatches.append({"ldes": ldes, "points": pts, "layers": layers, "root": root})
        else:
            obatches.append({"shapes": [pd.lde_shape(i) for i in range(len(shp))], "points": pts, "root": root})
    return pcs, rounds, obatches


def check_proof(orc, f, b, obatches, nq, pow_bits, pr, ch0):
    rc, idx = orc.verify_open(f, obatches, b, nq, pow_bits, pr, challenger=copy.deepcopy(ch0))
    assert rc == 0
    assert (idx == pr["indices"]).all()


SHAPES = {
    # mixed heights, a low coset above one block (2^12 rows), narrow and wide (> 256 and > 512 columns) matrices
    "mixed": [[(6, 4), (3, 3), (6, 1), (2, 6)], [(12, 3), (5, 300), (4, 600), (3, 513)], [(7, 2)], [(1, 2), (4, 1)]],
    "single": [[(9, 17)]],
}


def points_mixed(rng, f):
    zeta = rand_ef(f, rng)
    nxt = {k: rand_ef(f, rng) for k in range(32)}

    def fn(bi, m, logn):
        k = (bi + m) % 4
        if k == 0:
            return np.stack([zeta, nxt[logn]])
        if k == 1:
            return np.stack([zeta])
        if k == 2:
            return np.zeros((0, 4), np.uint32)
        return np.stack([nxt[1], zeta, nxt[1]])

    return fn


@pytest.mark.parametrize("f,b", [(0, 1), (1, 1), (0, 2), (1, 3)])
def test_pcs_open_parity(gpu, orc, f, b):
    rng = np.random.default_rng(50 + 10 * f + b)
    pcs, rounds, obatches = setup(gpu, orc, f, b, SHAPES["mixed"], points_mixed(rng, f), 900 + f)
    nq, pow_bits = 9, 8
    ch0 = new_oracle_challenger(orc, f, [11, 12, 13])
    want = orc.pcs_open(f, obatches, b, nq, pow_bits, challenger=copy.deepcopy(ch0))
    ch = to_gpu_challenger(ch0)
    got = pcs.open(rounds, ch, num_queries=nq, proof_of_work_bits=pow_bits)
    for k in ("values", "roots", "betas", "final", "indices", "queries"):
        assert np.array_equal(got[k], want[k]), k
    assert got["pow_witness"] == want["pow_witness"]
    # the challenger leaves in the state the oracle's does
    assert challenger_state(ch) == challenger_state(want["challenger"])
    check_proof(orc, f, b, obatches, nq, pow_bits, got, ch0)
    st = got["stats"]
    assert st["rounds"] == len(got["roots"]) and st["launches"] > 0


@pytest.mark.parametrize("f", [0, 1])
def test_open_values_and_reduced_openings(gpu, orc, f):
    rng = np.random.default_rng(70 + f)
    b = 1
    pcs, rounds, obatches = setup(gpu, orc, f, b, SHAPES["mixed"], points_mixed(rng, f), 1200 + f)
    vals = pcs.open_values(rounds)
    want = np.concatenate([orc.open_values(f, ob, b) for ob in obatches])
    assert np.array_equal(vals, want)
    alpha = rand_ef(f, rng)
    for h in (13, 7, 6, 3, 2):
        got = pcs.reduced_opening(rounds, vals, alpha, h)
        assert np.array_equal(got, orc.reduce_openings(f, obatches, vals, alpha, h)), h


def test_many_points_one_height(gpu, orc):
    """Six distinct points at one height: the reduction runs in two launches of
    at most four points, the second adding to the first."""
    f, b = 0, 1
    rng = np.random.default_rng(3)
    zs = [rand_ef(f, rng) for _ in range(6)]
    shapes = [[(5, 3), (5, 2), (5, 4)]]
    pts = {0: np.stack(zs[:3]), 1: np.stack(zs[3:5]), 2: np.stack([zs[5], zs[0]])}
    pcs, rounds, obatches = setup(gpu, orc, f, b, shapes, lambda bi, m, logn: pts[m], 1500)
    vals = pcs.open_values(rounds)
    alpha = rand_ef(f, rng)
    assert np.array_equal(pcs.reduced_opening(rounds, vals, alpha, 6),
                          orc.reduce_openings(f, obatches, vals, alpha, 6))
    ch0 = new_oracle_challenger(orc, f, [])
    got = pcs.open(rounds, to_gpu_challenger(ch0), num_queries=5, proof_of_work_bits=4)
    want = orc.pcs_open(f, obatches, b, 5, 4, challenger=copy.deepcopy(ch0))
    assert np.array_equal(got["queries"], want["queries"]) and np.array_equal(got["roots"], want["roots"])


def test_pcs_open_pico_shape_pow16(gpu, orc):
    """Pico's configuration (log_blowup 1, 84 queries, 16 proof-of-work bits) on a
    prover-like round structure: traces at (zeta, zeta * w_n), quotient chunks at zeta."""
    f, b = 0, 1
    rng = np.random.default_rng(16)
    zeta = rand_ef(f, rng)

    def next_point(logn):
        w = F.to_monty(f, np.array([F.two_adic_generator(f, logn), 0, 0, 0], np.uint32))
        return orc.ext_mul(f, zeta, w)

    main = [(10, 20), (8, 7), (10, 3), (6, 11)]
    quot = [(10, 4), (10, 4), (8, 4)]
    shapes = [main, main, quot]

    def pts(bi, m, logn):
        if bi == 2:
            return np.stack([zeta])
        return np.stack([zeta, next_point(logn)])

    pcs, rounds, obatches = setup(gpu, orc, f, b, shapes, pts, 1600)
    ch0 = new_oracle_challenger(orc, f, [1, 2, 3, 4, 5, 6, 7])
    got = pcs.open(rounds, to_gpu_challenger(ch0), num_queries=84, proof_of_work_bits=16)
    want = orc.pcs_open(f, obatches, b, 84, 16, challenger=copy.deepcopy(ch0))
    for k in ("values", "roots", "final", "indices", "queries"):
        assert np.array_equal(got[k], want[k]), k
    assert got["pow_witness"] == want["pow_witness"]


@pytest.mark.parametrize("f", [0, 1])
def test_pcs_open_large_verifies(gpu, orc, f):
    """2^20-row traces (LDE 2^21): the proof the GPU produces passes the
    restated verifier (the oracle prover is not run at this size)."""
    b = 1
    rng = np.random.default_rng(20 + f)
    fn = points_mixed(rng, f)
    shapes = [[(20, 8), (16, 40), (20, 3)], [(18, 300), (12, 5)], [(20, 4)]]
    pcs, rounds, obatches = setup(gpu, orc, f, b, shapes, fn, 2000 + f, oracle=False)
    ch0 = new_oracle_challenger(orc, f, [9])
    got = pcs.open(rounds, to_gpu_challenger(ch0), num_queries=20, proof_of_work_bits=10)
    check_proof(orc, f, b, obatches, 20, 10, got, ch0)
    # opened values of one matrix against the oracle on its own LDE
    pd = rounds[1][0]
    ob = {"ldes": [pd.lde(1)], "points": [rounds[1][1][1]]}
    n1 = len(rounds[0][1][0]) * 8 + len(rounds[0][1][1]) * 40 + len(rounds[0][1][2]) * 3 \
        + len(rounds[1][1][0]) * 300
    k = len(rounds[1][1][1]) * 5
    assert np.array_equal(got["values"][n1:n1 + k], orc.open_values(f, ob, b))


def test_wrong_claim_is_rejected(gpu, orc):
    """A point on the committed coset (z = g, where 1/(z - x_0) does not exist;
    Plonky3 fails on that inversion) is rejected by every opening call."""
    f, b = 1, 1
    rng = np.random.default_rng(8)
    pcs = TwoAdicFriPcs(gpu, f, b)
    t = F.random_matrix(f, 5, 3, 77)
    _, pd = pcs.commit([(pcs.natural_domain_for_degree(32), t)])
    # z = g (the first committed x): the inverse denominator of row 0 is 1/0
    g = F.to_monty(f, np.array([F.GENERATOR[f], 0, 0, 0], np.uint32))
    with pytest.raises(PicoError, match="coset"):
        pcs.open([(pd, [np.stack([g])])], to_gpu_challenger(new_oracle_challenger(orc, f, [])),
                 num_queries=2, proof_of_work_bits=2)
    with pytest.raises(PicoError, match="coset"):
        pcs.open_values([(pd, [np.stack([g])])])
    # another point of the coset: g * w_64^5
    x = F.to_monty(f, np.array([F.GENERATOR[f] * pow(F.two_adic_generator(f, 6), 5, F.P[f]) % F.P[f], 0, 0, 0],
                               np.uint32))
    with pytest.raises(PicoError, match="coset"):
        pcs.open_values([(pd, [np.stack([x])])])


def test_open_rejects_bad_arguments(gpu):
    f = 0
    pcs = TwoAdicFriPcs(gpu, f, 1)
    _, pd = pcs.commit([(pcs.natural_domain_for_degree(16), F.random_matrix(f, 4, 2, 1))])
    with pytest.raises(ValueError):
        pcs.open([(pd, [])], to_gpu_challenger(None))
    with pytest.raises(PicoError):
        pcs.open([(pd, [np.zeros((0, 4), np.uint32)])], to_gpu_challenger(None), num_queries=1,
                 proof_of_work_bits=30)


def test_concurrent_commits_and_openings(gpu, orc):
    """The ABI is thread-safe (the prover commits from rayon workers): four host
    threads each commit and open their own batch at once on one context; every
    result equals the same work done one call at a time."""
    import threading

    f, b = 0, 1
    jobs = []
    for t in range(4):
        rng = np.random.default_rng(300 + t)
        shapes = [[(10 - t, 5 + t), (8, 3), (9 - (t % 2), 17)]]
        jobs.append((shapes, points_mixed(rng, f), 4000 + 10 * t))

    def run(shapes, fn, seed):
        pcs, rounds, _ = setup(gpu, orc, f, b, shapes, fn, seed, oracle=False)
        got = pcs.open(rounds, to_gpu_challenger(None), num_queries=6, proof_of_work_bits=6)
        return rounds[0][0].root.copy(), got

    want = [run(*j) for j in jobs]
    got = [None] * len(jobs)
    errors = []

    def worker(k):
        try:
            got[k] = run(*jobs[k])
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(jobs))]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    for (r1, p1), (r2, p2) in zip(want, got):
        assert np.array_equal(r1, r2)
        for key in ("values", "roots", "final", "indices", "queries"):
            assert np.array_equal(p1[key], p2[key]), key
