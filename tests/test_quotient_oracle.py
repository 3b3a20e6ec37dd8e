"""The oracle's compute_quotient_values and the constraint-program builder,
pinned on the CPU by the property the quotient exists for: for a trace that
satisfies its AIR, sum_k alpha^k C_k(x) / Z_H(x) is a polynomial of degree
below (D - 1) n (D the constraint degree), so its values on the quotient
domain interpolate to a low-degree polynomial; a trace that breaks one
constraint does not.  Interpolation here is plain Python integer arithmetic,
independent of the oracle's transforms."""
import numpy as np
import pytest

from oracle import cpu as orc
from pico_b200 import fields as F
from pico_b200.quotient import MAX_BASE_REGS, ConstraintBuilder

FIELDS = [0, 1]


def fibonacci_air(b: ConstraintBuilder):
    """Two columns (x, y): x_0 = pub0, y_0 = pub1, next.x = y, next.y = x + y,
    y_{n-1} = pub2."""
    x, y = b.main(0), b.main(1)
    xn, yn = b.main(0, True), b.main(1, True)
    b.when_first_row().assert_eq(x, b.public(0))
    b.when_first_row().assert_eq(y, b.public(1))
    b.when_transition().assert_eq(xn, y)
    b.when_transition().assert_eq(yn, x + y)
    b.when_last_row().assert_eq(y, b.public(2))


def fib_trace(f, logn, a=1, c=1):
    p = F.P[f]
    n = 1 << logn
    rows = [(a % p, c % p)]
    for _ in range(n - 1):
        x, y = rows[-1]
        rows.append((y, (x + y) % p))
    t = np.array(rows, dtype=np.uint64)
    return F.to_monty(f, t).reshape(n, 2), [F.monty(f, a), F.monty(f, c), F.monty(f, int(rows[-1][1]))]


def interpolate_degree(f, log_q, vals_monty):
    """Largest j with a nonzero coefficient of the polynomial taking the given
    values at GENERATOR * w_Q^i (natural order), per extension coordinate."""
    p = F.P[f]
    Q = 1 << log_q
    w = F.two_adic_generator(f, log_q)
    g = F.GENERATOR[f]
    winv, ginv, qinv = pow(w, p - 2, p), pow(g, p - 2, p), pow(Q, p - 2, p)
    y = [[F.unmonty(f, int(v)) for v in vals_monty[:, k]] for k in range(4)]
    deg = -1
    for j in range(Q):
        wj = pow(winv, j, p)
        s = [0, 0, 0, 0]
        t = 1
        for i in range(Q):
            for k in range(4):
                s[k] += y[k][i] * t
            t = t * wj % p
        if any(v % p for v in s):
            deg = j
    return deg


@pytest.mark.parametrize("f", FIELDS)
def test_fibonacci_quotient_is_low_degree_only_for_a_valid_trace(f):
    logn, log_qd = 4, 1
    b = ConstraintBuilder()
    fibonacci_air(b)
    prog = b.program(f)
    trace, pub = fib_trace(f, logn)
    alpha = F.to_monty(f, [5, 7, 11, 13])
    q = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, trace, log_qd), public_values=pub,
                            alpha=alpha)
    assert interpolate_degree(f, logn + log_qd, q) < (1 << logn)  # D = 2: degree < n
    bad = trace.copy()
    bad[5, 1] = F.to_monty(f, [12345])[0]
    qb = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, bad, log_qd), public_values=pub,
                             alpha=alpha)
    assert interpolate_degree(f, logn + log_qd, qb) >= (1 << logn)
    wrong_pub = list(pub)
    wrong_pub[2] = F.monty(f, 3)
    qp = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, trace, log_qd),
                             public_values=wrong_pub, alpha=alpha)
    assert interpolate_degree(f, logn + log_qd, qp) >= (1 << logn)


@pytest.mark.parametrize("f", FIELDS)
def test_extension_constraint_with_permutation_columns(f):
    """A degree-3 constraint mixing a permutation (extension) column, a
    challenge and main columns, satisfied by construction:
    perm_next - perm = ch * x * y  on transitions.  The quotient has degree
    below 2n; breaking one permutation value raises it."""
    p = F.P[f]
    logn, log_qd = 3, 2
    n = 1 << logn
    rng = np.random.default_rng(3 + f)
    xy = rng.integers(0, p, size=(n, 2), dtype=np.uint64)
    ch = [int(v) for v in rng.integers(0, p, size=4)]
    acc = [0, 0, 0, 0]
    perm = []
    for r in range(n):
        perm.append(list(acc))
        prod = int(xy[r, 0]) * int(xy[r, 1]) % p
        acc = [(acc[k] + ch[k] * prod) % p for k in range(4)]
    perm_m = F.to_monty(f, np.array(perm, dtype=np.uint64)).reshape(n, 1, 4)
    main_m = F.to_monty(f, xy).reshape(n, 2)
    b = ConstraintBuilder()
    z, zn = b.permutation(0), b.permutation(0, True)
    b.when_transition().assert_zero(zn - z - b.challenge(0) * (b.main(0) * b.main(1)))
    prog = b.program(f)
    chal = F.to_monty(f, ch).reshape(1, 4)
    alpha = F.to_monty(f, [2, 3, 5, 7])
    q = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, main_m, log_qd),
                            perm_q=orc.on_quotient_domain(f, perm_m, log_qd), perm_challenges=chal, alpha=alpha)
    assert interpolate_degree(f, logn + log_qd, q) < 2 * n
    perm_bad = perm_m.copy()
    perm_bad[3, 0, 2] ^= 1
    qb = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, main_m, log_qd),
                             perm_q=orc.on_quotient_domain(f, perm_bad, log_qd), perm_challenges=chal, alpha=alpha)
    assert interpolate_degree(f, logn + log_qd, qb) >= 2 * n


def test_builder_reuses_registers_and_rejects_oversized_programs():
    b = ConstraintBuilder()
    acc = b.main(0)
    for k in range(1, 300):  # a long chain needs only a few live registers
        acc = acc * b.main(k % 7) + b.const(k)
    b.assert_zero(acc)
    prog = b.program(0)
    assert prog[:, 1].max() < 8
    b2 = ConstraintBuilder()
    live = [b2.main(k) for k in range(MAX_BASE_REGS + 1)]  # all live at once
    b2.assert_zero(sum(live[1:], live[0]))
    with pytest.raises(ValueError):
        b2.program(0)


def test_oracle_rejects_malformed_programs():
    trace = np.zeros((8, 2), dtype=np.uint32)
    alpha = np.zeros(4, dtype=np.uint32)
    for bad in ([1, 0, 5, 0], [9, 70, 0, 0], [3, 0, 0, 0], [99, 0, 0, 0], [5, 0, 0, 0]):
        with pytest.raises(RuntimeError):
            orc.quotient_values(0, 2, 1, np.array([bad], np.uint32), orc.on_quotient_domain(0, trace[:4], 1),
                                alpha=alpha)


def test_opcodes_agree_across_header_builder_and_oracle():
    import re
    from pathlib import Path

    from pico_b200.quotient import OPS

    root = Path(__file__).resolve().parents[1]
    header = (root / "include" / "pico_gpu.h").read_text()
    oracle_h = (root / "oracle" / "oracle.h").read_text()
    for name, v in OPS.items():
        m = re.search(rf"PICO_Q_{name} = (\d+)", header)
        o = re.search(rf"ORC_Q_{name} = (\d+)", oracle_h)
        assert m and int(m.group(1)) == v, name
        assert o and int(o.group(1)) == v, name


def test_quotient_chunk_domains_are_the_split_domains():
    """split_domains of GENERATOR * <w_Q> into D chunks: chunk j is
    GENERATOR * w_Q^j * <w_n>, and its LDE shift GENERATOR / shift is w_Q^-j
    (Monty form), the shift its chunk of PICO_QUOTIENT_CHUNKS output commits with."""
    from pico_b200 import fields as F
    from pico_b200.quotient import quotient_chunk_domains

    for f in (0, 1):
        p = F.P[f]
        for log_n, log_qd in ((5, 1), (8, 2), (3, 3)):
            wq = F.two_adic_generator(f, log_n + log_qd)
            doms = quotient_chunk_domains(f, log_n, log_qd)
            assert len(doms) == 1 << log_qd
            for j, d in enumerate(doms):
                assert d.log_n == log_n
                assert d.shift == F.GENERATOR[f] * pow(wq, j, p) % p
                assert F.lde_shift(f, d.shift) == F.monty(f, pow(wq, (p - 1 - j) % (p - 1), p))
