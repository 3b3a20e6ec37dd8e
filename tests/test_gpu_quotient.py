"""compute_quotient_values on the GPU (pico_gpu_quotient_values) against the
oracle, bit-exactly: the GPU reads the resident committed LDEs (bit-reversed
rows, local and next row of each quotient-domain point); the oracle gets
the traces' evaluations on the quotient domain from its own coset LDE in
natural order, so the row mapping is checked too.  Programs: a Fibonacci
AIR (first-row, transition, last-row constraints with public values), a
permutation-column constraint with challenges and cumulative sums, and
random straight-line programs over all opcodes, with a preprocessed trace
from a separate commit."""
import numpy as np
import pytest

from pico_b200 import PicoError, TwoAdicDomain, TwoAdicFriPcs
from pico_b200 import fields as F
from pico_b200.quotient import OPS, ConstraintBuilder, compute_quotient_values

pytestmark = pytest.mark.gpu
FIELDS = [0, 1]


def commit(gpu, f, b, mats):
    pcs = TwoAdicFriPcs(gpu, f, b)
    return pcs.commit([(TwoAdicDomain(m.shape[0].bit_length() - 1), m) for m in mats])[1]


def rand_ext(f, n, seed):
    return F.to_monty(f, F.uniform(f, 4 * n, seed)).reshape(n, 4)


@pytest.mark.parametrize("f", FIELDS)
@pytest.mark.parametrize("logn,log_qd,b", [(6, 1, 1), (10, 1, 2), (9, 2, 2), (14, 1, 1)])
def test_fibonacci_quotient_matches_oracle(gpu, orc, f, logn, log_qd, b):
    bld = ConstraintBuilder()
    x, y = bld.main(0), bld.main(1)
    bld.when_first_row().assert_eq(x, bld.public(0))
    bld.when_first_row().assert_eq(y, bld.public(1))
    bld.when_transition().assert_eq(bld.main(0, True), y)
    bld.when_transition().assert_eq(bld.main(1, True), x + y)
    bld.when_last_row().assert_eq(y, bld.public(2))
    prog = bld.program(f)
    # a random trace: the quotient need not be low-degree for bit-exactness
    main = F.random_matrix(f, logn, 3, 8100 + logn)
    pub = F.to_monty(f, [1, 1, 12345])
    alpha = rand_ext(f, 1, 8200 + f)[0]
    pd = commit(gpu, f, b, [main])
    want = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, main, log_qd), public_values=pub,
                               alpha=alpha)
    got = compute_quotient_values(gpu, prog, logn, log_qd, (pd, 0), public_values=pub, alpha=alpha)
    assert (got == want).all()
    pd.release()


@pytest.mark.parametrize("f", FIELDS)
def test_permutation_constraint_matches_oracle(gpu, orc, f):
    logn, log_qd, b = 9, 2, 2
    n = 1 << logn
    main = F.random_matrix(f, logn, 5, 8300)
    perm = rand_ext(f, n * 3, 8301).reshape(n, 3, 4)
    bld = ConstraintBuilder()
    z, zn = bld.permutation(1), bld.permutation(1, True)
    ch0, ch1 = bld.challenge(0), bld.challenge(1)
    denom = ch0 + bld.main(2) * ch1 + bld.main(4)
    bld.when_transition().assert_zero((zn - z) * denom - bld.main(3))
    bld.when_first_row().assert_zero(bld.permutation(0) - bld.regional_cumulative_sum())
    bld.when_last_row().assert_zero(bld.permutation(2, True) * bld.global_cumulative_sum(3) - bld.main(0))
    prog = bld.program(f)
    chal = rand_ext(f, 2, 8302)
    reg = rand_ext(f, 1, 8303)[0]
    glob = F.to_monty(f, F.uniform(f, 14, 8304))
    alpha = rand_ext(f, 1, 8305)[0]
    pd_main = commit(gpu, f, b, [main])
    pcs = TwoAdicFriPcs(gpu, f, b)
    _, pd_perm = pcs.commit([(TwoAdicDomain(logn), perm)])  # (n, w, 4): committed as its base flattening
    want = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, main, log_qd),
                               perm_q=orc.on_quotient_domain(f, perm, log_qd), perm_challenges=chal,
                               regional_sum=reg, global_sum=glob, alpha=alpha)
    got = compute_quotient_values(gpu, prog, logn, log_qd, (pd_main, 0), permutation=(pd_perm, 0),
                                  perm_challenges=chal, regional_sum=reg, global_sum=glob, alpha=alpha)
    assert (got == want).all()


def random_program(f, rng, main_w, prep_w, perm_w, n_pub, n_chal, steps=120):
    bld = ConstraintBuilder()
    pool_b = [bld.main(int(rng.integers(main_w)), bool(rng.integers(2))) for _ in range(4)]
    pool_e = [bld.challenge(0)]
    for _ in range(steps):
        r = rng.integers(12)
        if r == 0:
            pool_b.append(bld.main(int(rng.integers(main_w)), bool(rng.integers(2))))
        elif r == 1:
            pool_b.append(bld.preprocessed(int(rng.integers(prep_w)), bool(rng.integers(2))))
        elif r == 2:
            pool_e.append(bld.permutation(int(rng.integers(perm_w)), bool(rng.integers(2))))
        elif r == 3:
            pool_b.append([bld.is_first_row, bld.is_last_row, bld.is_transition][int(rng.integers(3))]())
        elif r == 4:
            pool_b.append(bld.const(int(rng.integers(F.P[f]))) if rng.integers(2) else bld.public(int(rng.integers(n_pub))))
        elif r == 5:
            pool_e.append(bld.challenge(int(rng.integers(n_chal))) if rng.integers(2) else bld.regional_cumulative_sum())
        elif r == 6:
            pool_b.append(bld.global_cumulative_sum(int(rng.integers(14))))
        elif r in (7, 8):
            a, c = pool_b[int(rng.integers(len(pool_b)))], pool_b[int(rng.integers(len(pool_b)))]
            pool_b.append([a + c, a - c, a * c][int(rng.integers(3))])
        elif r == 9:
            a, c = pool_e[int(rng.integers(len(pool_e)))], pool_e[int(rng.integers(len(pool_e)))]
            pool_e.append([a + c, a - c, a * c][int(rng.integers(3))])
        elif r == 10:
            a, c = pool_e[int(rng.integers(len(pool_e)))], pool_b[int(rng.integers(len(pool_b)))]
            pool_e.append([a * c, a + c, c - a][int(rng.integers(3))])
        else:
            if rng.integers(2):
                bld.assert_zero(pool_b[int(rng.integers(len(pool_b)))])
            else:
                bld.assert_zero(pool_e[int(rng.integers(len(pool_e)))])
        # keep the live sets small enough for the register files
        pool_b, pool_e = pool_b[-24:], pool_e[-6:]
    bld.assert_zero(pool_e[-1])
    return bld.program(f)


@pytest.mark.parametrize("f", FIELDS)
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_random_programs_match_oracle(gpu, orc, f, seed):
    rng = np.random.default_rng(8400 + 10 * seed + f)
    logn, log_qd, b = 8, 1 + seed % 2, 2
    n = 1 << logn
    main_w, prep_w, perm_w, n_pub, n_chal = 7, 3, 2, 4, 3
    prog = random_program(f, rng, main_w, prep_w, perm_w, n_pub, n_chal)
    main = F.random_matrix(f, logn, main_w, 8500 + seed)
    prep = F.random_matrix(f, logn, prep_w, 8600 + seed)
    perm = rand_ext(f, n * perm_w, 8700 + seed).reshape(n, perm_w, 4)
    pub = F.to_monty(f, F.uniform(f, n_pub, 8800 + seed))
    chal = rand_ext(f, n_chal, 8900 + seed)
    reg = rand_ext(f, 1, 9000 + seed)[0]
    glob = F.to_monty(f, F.uniform(f, 14, 9100 + seed))
    alpha = rand_ext(f, 1, 9200 + seed)[0]
    pcs = TwoAdicFriPcs(gpu, f, b)
    _, pd_main = pcs.commit([(TwoAdicDomain(logn), main), (TwoAdicDomain(logn), perm)])  # main and perm: one commit
    _, pd_prep = pcs.commit([(TwoAdicDomain(logn), prep)])
    want = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, main, log_qd),
                               prep_q=orc.on_quotient_domain(f, prep, log_qd),
                               perm_q=orc.on_quotient_domain(f, perm, log_qd), public_values=pub,
                               perm_challenges=chal, regional_sum=reg, global_sum=glob, alpha=alpha)
    got = compute_quotient_values(gpu, prog, logn, log_qd, (pd_main, 0), preprocessed=(pd_prep, 0),
                                  permutation=(pd_main, 1), public_values=pub, perm_challenges=chal,
                                  regional_sum=reg, global_sum=glob, alpha=alpha)
    assert (got == want).all()


def test_device_output_and_refusals(gpu, orc):
    import torch

    f, logn, log_qd = 0, 7, 1
    bld = ConstraintBuilder()
    bld.when_transition().assert_eq(bld.main(0, True), bld.main(1))
    prog = bld.program(f)
    main = F.random_matrix(f, logn, 2, 9300)
    alpha = rand_ext(f, 1, 9301)[0]
    pd = commit(gpu, f, 1, [main])
    want = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, main, log_qd), alpha=alpha)
    out = torch.empty((1 << (logn + log_qd), 4), dtype=torch.int32, device="cuda")
    compute_quotient_values(gpu, prog, logn, log_qd, (pd, 0), alpha=alpha, out=out)
    assert (out.cpu().numpy().view(np.uint32) == want).all()
    with pytest.raises(PicoError):  # quotient domain taller than the committed LDE (blowup 1)
        compute_quotient_values(gpu, prog, logn, 2, (pd, 0), alpha=alpha)
    k = int(np.nonzero(prog[:, 0] == OPS["MAIN"])[0][0])
    bad = prog.copy()
    bad[k, 2] = 5  # main column beyond the width
    with pytest.raises(PicoError):
        compute_quotient_values(gpu, bad, logn, log_qd, (pd, 0), alpha=alpha)
    bad = prog.copy()
    bad[k, 1] = 64  # base register beyond the register file
    with pytest.raises(PicoError):
        compute_quotient_values(gpu, bad, logn, log_qd, (pd, 0), alpha=alpha)
    pd.release()


@pytest.mark.parametrize("f", FIELDS)
@pytest.mark.parametrize("log_qd", [1, 2])
def test_quotient_chunks_commit_as_the_prover_does(gpu, orc, f, log_qd):
    """PICO_QUOTIENT_CHUNKS: chunk j holds points j, j + D, ... (split_evals);
    committed on their split domains (prover.rs:513-538), the root is the
    oracle's commit of the same chunks with shifts GENERATOR / (GENERATOR w_Q^j)."""
    from pico_b200.quotient import commit_quotient_chunks, quotient_chunk_domains

    logn, b = 8, log_qd
    bld = ConstraintBuilder()
    x, y = bld.main(0), bld.main(1)
    bld.when_transition().assert_eq(bld.main(0, True), y)
    bld.when_transition().assert_eq(bld.main(1, True), x * y)
    prog = bld.program(f)
    main = F.random_matrix(f, logn, 2, 8700 + f)
    alpha = rand_ext(f, 1, 8710 + f)[0]
    pd = commit(gpu, f, b, [main])
    nat = compute_quotient_values(gpu, prog, logn, log_qd, (pd, 0), alpha=alpha)
    ch = compute_quotient_values(gpu, prog, logn, log_qd, (pd, 0), alpha=alpha, chunks=True)
    D = 1 << log_qd
    assert ch.shape == (D, 1 << logn, 4)
    for j in range(D):
        assert (ch[j] == nat[j::D]).all()
    pcs = TwoAdicFriPcs(gpu, f, b)
    root, qpd = commit_quotient_chunks(pcs, [ch[j] for j in range(D)], logn, log_qd)
    doms = quotient_chunk_domains(f, logn, log_qd)
    want, _, _ = orc.pcs_commit(f, [np.ascontiguousarray(ch[j]) for j in range(D)],
                                [F.lde_shift(f, d.shift) for d in doms], b)
    assert root.tolist() == want.tolist()
    qpd.release()
    pd.release()
