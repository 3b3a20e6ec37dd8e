"""CPU tests of the opening oracle (TwoAdicFriPcs::open restated).

Pins: opened values against interpolation + evaluation done here in plain
Python integers; reduced openings against a direct per-row restatement of
fri.rs:150-238; whole proofs against the restated Pico verifier
(vm/src/compiler/recursion/circuit/fri.rs:77-436), including rejection of
tampered proofs.
"""
import numpy as np
import pytest

W_EXT = {0: 3, 1: 11}


class EF:
    """Degree-4 binomial extension in canonical integers (test-side arithmetic)."""

    def __init__(self, field, p):
        self.f, self.p, self.w = field, p, W_EXT[field]

    def mul(self, a, b):
        p, w = self.p, self.w
        acc = [0] * 7
        for i in range(4):
            for j in range(4):
                acc[i + j] += a[i] * b[j]
        return [(acc[k] + (w * acc[k + 4] if k < 3 else 0)) % p for k in range(4)]

    def add(self, a, b):
        return [(x + y) % self.p for x, y in zip(a, b)]

    def sub(self, a, b):
        return [(x - y) % self.p for x, y in zip(a, b)]

    def scale(self, a, s):
        return [(x * s) % self.p for x in a]

    def pow(self, a, e):
        r, b = [1, 0, 0, 0], list(a)
        while e:
            if e & 1:
                r = self.mul(r, b)
            b = self.mul(b, b)
            e >>= 1
        return r

    def inv(self, a):
        # a^(p^4 - 2): Fermat in the extension (independent of the oracle's norm method)
        return self.pow(a, self.p ** 4 - 2)


def canon(orc, field, a):
    lib = orc.load()
    return [lib.orc_from_monty(field, int(v)) for v in np.asarray(a).ravel()]


def monty(orc, field, a):
    lib = orc.load()
    return np.array([lib.orc_to_monty(field, int(v)) for v in a], dtype=np.uint32)


def rand_mat(rng, p, logn, w):
    # raw values < p are valid Monty representatives
    return rng.integers(0, p, size=(1 << logn, w), dtype=np.uint64).astype(np.uint32)


def rand_ef(rng, p):
    return rng.integers(0, p, size=4, dtype=np.uint64).astype(np.uint32)


def bitrev(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


@pytest.mark.parametrize("field", [0, 1])
def test_ext_inv(orc, field):
    lib = orc.load()
    p = lib.orc_prime(field)
    rng = np.random.default_rng(10 + field)
    one = monty(orc, field, [1, 0, 0, 0])
    for _ in range(20):
        a = rand_ef(rng, p)
        if not a.any():
            continue
        assert np.array_equal(orc.ext_mul(field, a, orc.ext_inv(field, a)), one)
    # an element of the base field and one with a zero constant term
    for a in ([5, 0, 0, 0], [0, 7, 0, 0], [0, 0, 0, 9]):
        am = monty(orc, field, a)
        assert np.array_equal(orc.ext_mul(field, am, orc.ext_inv(field, am)), one)


@pytest.mark.parametrize("field,logn,w,b", [(0, 4, 3, 1), (1, 5, 2, 2), (0, 3, 1, 3), (1, 1, 4, 1)])
def test_open_values_match_polynomial_evaluation(orc, field, logn, w, b):
    """p(z) from the committed low coset equals interpolation over H_n followed by
    evaluation at z (coefficients by an O(n^2) inverse DFT, Horner in EF4)."""
    lib = orc.load()
    p = lib.orc_prime(field)
    E = EF(field, p)
    rng = np.random.default_rng(100 * field + logn)
    trace = rand_mat(rng, p, logn, w)
    g = lib.orc_to_monty(field, lib.orc_generator(field))
    lde = orc.coset_lde(field, trace, b, g)
    zs = [rand_ef(rng, p) for _ in range(2)]
    vals = orc.open_values(field, {"ldes": [lde], "points": [np.stack(zs)]}, b)
    n = 1 << logn
    wn = lib.orc_two_adic_generator(field, logn)
    wn_inv = pow(wn, p - 2, p)
    n_inv = pow(n, p - 2, p)
    T = [canon(orc, field, trace[k]) for k in range(n)]
    for zi, z in enumerate(zs):
        zc = canon(orc, field, z)
        for j in range(w):
            coeffs = [n_inv * sum(T[k][j] * pow(wn_inv, (i * k) % n, p) for k in range(n)) % p for i in range(n)]
            acc = [0, 0, 0, 0]
            for cf in reversed(coeffs):
                acc = E.add(E.mul(acc, zc), [cf, 0, 0, 0])
            assert canon(orc, field, vals[zi * w + j]) == acc, (zi, j)


def test_reduce_openings_direct(orc):
    """Reduced opening of the tallest height against the per-row formula
    ro[i] = sum over (matrix, point) of alpha^off * sum_j alpha^j (p_j(z) - M_ij) / (z - x_i)."""
    field = 1
    lib = orc.load()
    p = lib.orc_prime(field)
    E = EF(field, p)
    rng = np.random.default_rng(7)
    b = 1
    g = lib.orc_to_monty(field, lib.orc_generator(field))
    mats = [rand_mat(rng, p, 3, 3), rand_mat(rng, p, 3, 2), rand_mat(rng, p, 2, 2)]
    _, ldes, layers = orc.pcs_commit(field, mats, [g] * 3, b, want_ldes=True, want_layers=True)
    z1, z2 = rand_ef(rng, p), rand_ef(rng, p)
    pts = [np.stack([z1, z2]), np.stack([z2]), np.stack([z1])]
    batch = {"ldes": ldes, "points": pts}
    vals = orc.open_values(field, batch, b)
    alpha = rand_ef(rng, p)
    h = 4
    ro = orc.reduce_openings(field, [batch], vals, alpha, h)
    a = canon(orc, field, alpha)
    N = 1 << h
    wh = lib.orc_two_adic_generator(field, h)
    gc = lib.orc_generator(field)
    expect = [[0, 0, 0, 0] for _ in range(N)]
    off = 0
    vpos = 0
    for m, P in enumerate(pts):
        w = ldes[m].shape[1]
        for z in P:
            ys = [canon(orc, field, vals[vpos + j]) for j in range(w)]
            vpos += w
            if ldes[m].shape[0] != N:
                continue
            zc = canon(orc, field, z)
            for i in range(N):
                x = gc * pow(wh, bitrev(i, h), p) % p
                row = canon(orc, field, ldes[m][i])
                acc = [0, 0, 0, 0]
                for j in range(w):
                    t = E.sub(ys[j], [row[j], 0, 0, 0])
                    acc = E.add(acc, E.mul(E.pow(a, off + j), t))
                expect[i] = E.add(expect[i], E.mul(acc, E.inv(E.sub(zc, [x, 0, 0, 0]))))
            off += w
    got = [canon(orc, field, ro[i]) for i in range(N)]
    assert got == expect


def make_batches(orc, field, rng, shapes, b, points_fn):
    lib = orc.load()
    p = lib.orc_prime(field)
    g = lib.orc_to_monty(field, lib.orc_generator(field))
    out = []
    for bi, shp in enumerate(shapes):
        mats = [rand_mat(rng, p, logn, w) for logn, w in shp]
        root, ldes, layers = orc.pcs_commit(field, mats, [g] * len(mats), b, want_ldes=True, want_layers=True)
        pts = [points_fn(bi, m, logn) for m, (logn, _) in enumerate(shp)]
        out.append({"ldes": ldes, "points": pts, "layers": layers, "root": root})
    return out


@pytest.mark.parametrize("field,b", [(0, 1), (1, 1), (0, 2), (1, 3)])
def test_open_proof_verifies(orc, field, b):
    lib = orc.load()
    p = lib.orc_prime(field)
    rng = np.random.default_rng(1000 + 10 * field + b)
    zeta = rand_ef(rng, p)
    extra = {k: rand_ef(rng, p) for k in range(8)}

    def points(bi, m, logn):
        # zeta and a per-height "next" point for most matrices; one point, none, a repeat
        k = (bi + m) % 4
        if k == 0:
            return np.stack([zeta, extra[logn % 8]])
        if k == 1:
            return np.stack([zeta])
        if k == 2:
            return np.zeros((0, 4), np.uint32)
        return np.stack([extra[1], zeta, extra[1]])

    shapes = [[(5, 4), (3, 3), (5, 1), (2, 6)], [(4, 2), (4, 5)], [(6, 3)], [(1, 2), (3, 1)]]
    batches = make_batches(orc, field, rng, shapes, b, points)
    nq, pow_bits = 7, 6
    ch0 = orc.new_challenger()
    for v in range(5):
        orc.challenger_observe(field, ch0, v)  # prior transcript
    import copy
    pr = orc.pcs_open(field, batches, b, nq, pow_bits, challenger=copy.deepcopy(ch0))
    rc, idx = orc.verify_open(field, batches, b, nq, pow_bits, pr, challenger=copy.deepcopy(ch0))
    assert rc == 0
    assert np.array_equal(idx, pr["indices"])
    assert len(pr["roots"]) == 6  # LDE height 2^(6+b) folded down to 2^b
    assert pr["queries"].shape[1] == orc.open_query_words(batches, b)
    # tampering is caught by the check it breaks
    bad = dict(pr, queries=pr["queries"].copy())
    bad["queries"][0, 0] ^= 1
    assert orc.verify_open(field, batches, b, nq, pow_bits, bad, challenger=copy.deepcopy(ch0))[0] == 11
    bad = dict(pr, queries=pr["queries"].copy())
    bad["queries"][1, -1] ^= 1  # last digest of the last commit-phase path
    assert orc.verify_open(field, batches, b, nq, pow_bits, bad, challenger=copy.deepcopy(ch0))[0] == 13
    bad = dict(pr, final=pr["final"].copy())
    bad["final"][0] ^= 1
    assert orc.verify_open(field, batches, b, nq, pow_bits, bad, challenger=copy.deepcopy(ch0))[0] != 0


def test_open_wrong_value_fails(orc):
    """A wrong opened value changes the transcript and breaks the reduced
    openings: with the witness re-ground the proof still fails the fold check."""
    field, b = 0, 1
    lib = orc.load()
    p = lib.orc_prime(field)
    rng = np.random.default_rng(5)
    zeta = rand_ef(rng, p)
    batches = make_batches(orc, field, rng, [[(4, 3), (3, 2)]], b, lambda bi, m, logn: np.stack([zeta]))
    vals = orc.open_values(field, {"ldes": batches[0]["ldes"], "points": batches[0]["points"]}, b)
    vals[0, 0] ^= 1
    # the prover cannot produce a low-degree codeword for a wrong claim; the
    # verifier on the honest proof with a wrong value rejects
    pr = orc.pcs_open(field, batches, b, 4, 4)
    bad = dict(pr, values=vals)
    assert orc.verify_open(field, batches, b, 4, 4, bad)[0] != 0


def test_grind_is_smallest(orc):
    import copy

    field = 1
    lib = orc.load()
    rng = np.random.default_rng(9)
    p = lib.orc_prime(field)
    zeta = rand_ef(rng, p)
    batches = make_batches(orc, field, rng, [[(3, 2)]], 1, lambda bi, m, logn: np.stack([zeta]))
    pr = orc.pcs_open(field, batches, 1, 1, 5)
    w = lib.orc_from_monty(field, pr["pow_witness"])
    # rebuild the challenger state at the grind: replay the transcript
    ch = orc.new_challenger()
    for v in pr["values"].ravel():
        orc.challenger_observe(field, ch, int(v))
    for _ in range(4):
        orc.challenger_sample(field, ch)
    for r in pr["roots"]:
        for v in r:
            orc.challenger_observe(field, ch, int(v))
        for _ in range(4):
            orc.challenger_sample(field, ch)
    for v in pr["final"]:
        orc.challenger_observe(field, ch, int(v))
    for cand in range(w + 1):
        t = copy.deepcopy(ch)
        orc.challenger_observe(field, t, lib.orc_to_monty(field, cand))
        ok = lib.orc_from_monty(field, orc.challenger_sample(field, t)) & 31 == 0
        assert ok == (cand == w)
