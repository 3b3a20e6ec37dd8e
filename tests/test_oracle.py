"""CPU tests of the oracle: pinned to the reference's known answers, then
checked for internal consistency against independent Python restatements."""
import numpy as np
import pytest

from pico_b200 import fields as F

FIELDS = [(0, "koalabear"), (1, "babybear")]


@pytest.mark.parametrize("f,name", FIELDS)
def test_poseidon2_kat(orc, golden, f, name):
    kat = golden["kat"][name]
    got = orc.permute_canonical(f, np.array(kat["input"], dtype=np.uint32))
    assert got.tolist() == kat["output"]


@pytest.mark.parametrize("f,name", FIELDS)
def test_two_adic_generator(golden, orc, f, name):
    S = F.TWO_ADICITY[f]
    p = F.P[f]
    w = golden["two_adic"][name]["max_root"]
    assert w == orc.load().orc_two_adic_generator(f, S)
    assert pow(w, 1 << S, p) == 1 and pow(w, 1 << (S - 1), p) == p - 1


@pytest.mark.parametrize("f,name", FIELDS)
def test_golden_vectors(orc, golden, f, name):
    v = golden["vectors"][name]
    assert orc.permute(f, np.array(v["permute"]["in"], dtype=np.uint32)).tolist() == v["permute"]["out"]
    for h in v["hash"]:
        x = F.to_monty(f, F.uniform(f, h["len"], h["seed"])) if h["len"] else np.zeros(0, np.uint32)
        assert orc.hash_elems(f, x).tolist() == h["digest"]
    import hashlib

    for c in v["coset_lde"]:
        m = F.random_matrix(f, c["log_n"], c["width"], c["seed"])
        out = orc.coset_lde(f, m, c["log_blowup"], F.lde_shift(f))
        assert hashlib.sha256(out.tobytes()).hexdigest() == c["sha256"]
    pc = v["pcs_commit"]
    mats = [F.random_matrix(f, lh, w, s) for lh, w, s in pc["shapes"]]
    root, _, _ = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), pc["log_blowup"])
    assert root.tolist() == pc["root"]


def _bitrev(i, bits):
    return int(format(i, f"0{bits}b")[::-1], 2) if bits else 0


@pytest.mark.parametrize("f,_", FIELDS)
@pytest.mark.parametrize("logn,w,b", [(0, 2, 1), (1, 1, 1), (3, 2, 1), (4, 3, 2), (5, 1, 3)])
def test_lde_matches_direct_evaluation(orc, f, _, logn, w, b):
    """Row i of the committed LDE equals f(shift * w_N^rev(i)) (fri.rs:155-171),
    evaluated here by interpolation in plain Python integers."""
    p = F.P[f]
    n, N = 1 << logn, 1 << (logn + b)
    m = F.random_matrix(f, logn, w, 1000 + logn)
    shift = F.lde_shift(f)  # Monty(GENERATOR)
    out = F.from_monty(f, orc.coset_lde(f, m, b, shift))
    evals = F.from_monty(f, m).astype(object)
    wn = F.two_adic_generator(f, logn)
    wN = F.two_adic_generator(f, logn + b)
    ninv = pow(n, p - 2, p)
    g = F.GENERATOR[f]
    for c in range(w):
        coef = [sum(int(evals[j, c]) * pow(wn, (-i * j) % n, p) for j in range(n)) * ninv % p for i in range(n)]
        for i in range(N):
            x = g * pow(wN, _bitrev(i, logn + b), p) % p
            val = sum(coef[k] * pow(x, k, p) for k in range(n)) % p
            assert int(out[i, c]) == val


@pytest.mark.parametrize("f,_", FIELDS)
def test_sponge_and_compress_semantics(orc, f, _):
    """PaddingFreeSponge overwrite mode and TruncatedPermutation (hash.rs:40-52, 89-94)."""
    x = F.to_monty(f, F.uniform(f, 11, 5))
    s = np.zeros(16, dtype=np.uint32)
    s[:8] = x[:8]
    s = orc.permute(f, s)
    s[:3] = x[8:11]
    s = orc.permute(f, s)
    assert orc.hash_elems(f, x).tolist() == s[:8].tolist()
    assert orc.hash_elems(f, np.zeros(0, np.uint32)).tolist() == [0] * 8
    l, r = x[:8], F.to_monty(f, F.uniform(f, 8, 6))
    st = orc.permute(f, np.concatenate([l, r]))
    assert orc.compress(f, l, r).tolist() == st[:8].tolist()


@pytest.mark.parametrize("f,_", FIELDS)
def test_mmcs_mixed_heights_restated(orc, f, _):
    """Mixed-height MMCS restated from the verifier (fri.rs:389-436): tallest
    rows hashed as leaves; a level whose length equals a matrix height gets
    node = compress(compress(l, r), hash(rows))."""
    mats = [F.random_matrix(f, 3, 3, 1), F.random_matrix(f, 1, 2, 2), F.random_matrix(f, 3, 4, 3),
            F.random_matrix(f, 2, 5, 4)]
    root = orc.mmcs_commit(f, mats)
    order = sorted(range(len(mats)), key=lambda i: -mats[i].shape[0])
    by_h = {}
    for i in order:
        by_h.setdefault(mats[i].shape[0], []).append(i)
    H = mats[order[0]].shape[0]
    layer = [orc.hash_elems(f, np.concatenate([mats[i][r] for i in by_h[H]])) for r in range(H)]
    h = H
    while h > 1:
        h //= 2
        nxt = []
        for r in range(h):
            d = orc.compress(f, layer[2 * r], layer[2 * r + 1])
            if h in by_h:
                d = orc.compress(f, d, orc.hash_elems(f, np.concatenate([mats[i][r] for i in by_h[h]])))
            nxt.append(d)
        layer = nxt
    assert root.tolist() == layer[0].tolist()


@pytest.mark.parametrize("f,_", FIELDS)
def test_challenger_semantics(orc, f, _):
    """observe clears the output buffer and duplexes at 8 inputs; sample pops
    from the end after duplexing pending input (challenger.rs:89-115,202-237)."""
    ch = orc.new_challenger()
    vals = F.to_monty(f, F.uniform(f, 10, 9))
    for v in vals:
        orc.challenger_observe(f, ch, int(v))
    s = np.zeros(16, dtype=np.uint32)
    s[:8] = vals[:8]
    s = orc.permute(f, s)
    s[:2] = vals[8:10]
    s = orc.permute(f, s)
    got = [orc.challenger_sample(f, ch) for _ in range(3)]
    assert got == [int(s[7]), int(s[6]), int(s[5])]


@pytest.mark.parametrize("f,_", FIELDS)
def test_fri_fold_matches_verifier_formula(orc, f, _):
    """One fold restated as the verifier computes it, e0 + (beta - x0)(e1 - e0)/(x1 - x0)
    with x1 = -x0 and x0 = w^rev(r) (fri.rs:345-377), with explicit betas."""
    p = F.P[f]
    W = 3 if f == 0 else 11
    base = F.random_matrix(f, 3, 4, 77)
    cw = orc.coset_lde(f, base, 1, F.lde_shift(f))  # 16 EF4 elements
    betas = F.to_monty(f, F.uniform(f, 4 * 3, 78)).reshape(3, 4)
    roots, _, final, _ = orc.fri_commit_phase(f, cw, 1, 0, betas=betas)
    assert roots.shape == (3, 8)

    def emul(a, b):
        acc = [0] * 7
        for i in range(4):
            for j in range(4):
                acc[i + j] += a[i] * b[j]
        return [(acc[k] + (W * acc[k + 4] if k + 4 < 7 else 0)) % p for k in range(4)]

    cur = [list(map(int, r)) for r in F.from_monty(f, cw)]
    for rnd in range(3):
        L = len(cur)
        beta = [int(v) for v in F.from_monty(f, betas[rnd])]
        g = F.two_adic_generator(f, L.bit_length() - 1)
        nxt = []
        for r in range(L // 2):
            x0 = pow(g, _bitrev(r, L.bit_length() - 2), p)
            e0, e1 = cur[2 * r], cur[2 * r + 1]
            inv = pow((p - 2 * x0) % p, p - 2, p)  # 1 / (x1 - x0)
            num = [(b - (x0 if k == 0 else 0)) % p for k, b in enumerate(beta)]
            d = [(e1[k] - e0[k]) * inv % p for k in range(4)]
            t = emul(num, d)
            nxt.append([(e0[k] + t[k]) % p for k in range(4)])
        cur = nxt
    assert F.from_monty(f, final[0]).tolist() == cur[0] == cur[1]


@pytest.mark.parametrize("f,_", FIELDS)
def test_fri_final_poly_coefficients(orc, f, _):
    """Early stop (log_final_len > 0): the remaining codeword interpolates to a
    polynomial with at most 2^log_final_len coefficients."""
    base = F.random_matrix(f, 6, 4, 90)
    cw = orc.coset_lde(f, base, 1, F.lde_shift(f))
    r0, b0, f0, _ = orc.fri_commit_phase(f, cw, 1, 0)
    r2, b2, f2, _ = orc.fri_commit_phase(f, cw, 1, 2)
    assert f2.shape == (4, 4)
    # the first rounds coincide with the full run
    assert (r2 == r0[: len(r2)]).all() and (b2 == b0[: len(b2)]).all()
