"""Failure detection on the GPU path, injected on the host (nothing here
faults, traps or hangs a GPU).  The reference prover panics on these
conditions (vm/src/instances/machine/riscv.rs:106-110); this library reports
them as status codes and keeps the context usable:

* a device allocation that fails part-way through a commit (injected with
  pico_gpu_test_fail_allocations) returns PICO_ERR_OUT_OF_MEMORY, gives back
  every reserved byte and leaves the next commit bit-exact;
* a request that does not fit the HBM budget next to a resident commit stays
  queued: poll says not ready, wait with a timeout returns PICO_ERR_TIMEOUT,
  cancel makes it PICO_ERR_CANCELLED, and releasing the resident commit
  admits the next one;
* requests larger than the whole budget, and synchronous commits larger than
  what is left of it, are refused with PICO_ERR_OUT_OF_MEMORY.
"""
import numpy as np
import pytest

from pico_b200 import CommitServer, GpuContext, PicoError, TwoAdicDomain, TwoAdicFriPcs, abi
from pico_b200 import fields as F

pytestmark = pytest.mark.gpu


def mats_of(f, shapes, seed):
    return [F.random_matrix(f, lh, w, seed + i) for i, (lh, w) in enumerate(shapes)]


def doms(mats):
    return [TwoAdicDomain(m.shape[0].bit_length() - 1) for m in mats]


@pytest.mark.parametrize("packed", ["0", str(1 << 40)])
def test_allocation_failure_returns_budget_and_recovers(gpu, orc, packed, monkeypatch):
    """Every allocation position of a commit fails once in turn."""
    monkeypatch.setenv("PICO_PACKED_COMMIT_BYTES", packed)
    f = 0
    shapes = [(13, 9), (12, 5), (13, 3), (9, 17), (12, 2)]
    mats = mats_of(f, shapes, 2100)
    want = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), 1)[0]
    pcs = TwoAdicFriPcs(gpu, f, 1)
    lib = abi.load()
    reserved0 = gpu.memory()[0]
    failed = 0
    try:
        for after in range(40):
            lib.pico_gpu_test_fail_allocations(after)
            try:
                root, pd = pcs.commit(list(zip(doms(mats), mats)))
            except PicoError as e:
                assert e.status == abi.PICO_ERR_OUT_OF_MEMORY
                assert "injected" in str(e)
                assert gpu.memory()[0] == reserved0  # nothing of the failed commit stays reserved
                failed += 1
                continue
            # this commit made fewer allocations than `after`: injection is still armed
            lib.pico_gpu_test_fail_allocations(-1)
            assert root.tolist() == want.tolist()
            pd.release()
            break
    finally:
        lib.pico_gpu_test_fail_allocations(-1)
    assert failed >= 2
    root, pd = pcs.commit(list(zip(doms(mats), mats)))
    assert root.tolist() == want.tolist()
    pd.release()
    assert gpu.memory()[0] == reserved0


def test_admission_queue_timeout_cancel_and_release(orc):
    f = 0
    small = mats_of(f, [(10, 8), (9, 4)], 2200)
    big = mats_of(f, [(14, 32), (13, 16)], 2300)
    pcs_probe = TwoAdicFriPcs(None, f, 1)
    res_small, scr_small = pcs_probe.commit_bytes(list(zip(doms(small), small)))
    res_big, scr_big = pcs_probe.commit_bytes(list(zip(doms(big), big)))
    # the big request fits the budget alone, but not next to the small one's resident commit
    budget = res_small + res_big + scr_big - 1
    assert res_small + scr_small <= budget
    want_small = orc.pcs_commit(f, small, [F.lde_shift(f)] * 2, 1)[0]
    want_big = orc.pcs_commit(f, big, [F.lde_shift(f)] * 2, 1)[0]
    with GpuContext(0, hbm_budget_bytes=budget, n_streams=2) as ctx:
        server = CommitServer(ctx)
        r1 = server.submit(f, small, 1)
        root1, pd1 = r1.wait(keep=True)
        assert root1.tolist() == want_small.tolist()
        assert ctx.memory()[0] == res_small
        r2 = server.submit(f, big, 1)
        assert not r2.poll()  # queued: not admitted while pd1 holds its budget
        for timeout_ms in (0, 50):
            with pytest.raises(PicoError) as e:
                r2.wait(timeout_ms=timeout_ms)
            assert e.value.status == abi.PICO_ERR_TIMEOUT
        r2.cancel()
        with pytest.raises(PicoError) as e:
            r2.poll()
        assert e.value.status == abi.PICO_ERR_CANCELLED
        with pytest.raises(PicoError) as e:
            r2.wait()
        assert e.value.status == abi.PICO_ERR_CANCELLED
        r2.free()
        # a synchronous commit that does not fit what is left is refused at once
        with pytest.raises(PicoError) as e:
            TwoAdicFriPcs(ctx, f, 1).commit(list(zip(doms(big), big)))
        assert e.value.status == abi.PICO_ERR_OUT_OF_MEMORY
        # releasing the resident commit admits the next request
        r3 = server.submit(f, big, 1)
        assert not r3.poll()
        pd1.release()
        root3, pd3 = r3.wait(timeout_ms=60_000, keep=True)
        assert root3.tolist() == want_big.tolist()
        with pytest.raises(PicoError) as e:  # a cancelled request cannot be cancelled twice
            r3.cancel()
        assert e.value.status == abi.PICO_ERR_NOT_READY
        pd3.release()
        r1.free()
        r3.free()
        assert ctx.memory()[0] == 0
        # a request larger than the whole budget is refused at submission
        huge = mats_of(f, [(15, 64)], 2400)
        with pytest.raises(PicoError) as e:
            server.submit(f, huge, 2)
        assert e.value.status == abi.PICO_ERR_OUT_OF_MEMORY


def test_context_stays_usable_after_refused_calls(gpu, orc):
    """Malformed descriptors on a live context are refused before any launch,
    and the next valid commit is bit-exact."""
    import ctypes as C

    lib = abi.load()
    m = F.random_matrix(0, 8, 3, 2500)
    mats = (abi.Matrix * 1)()
    mats[0].values = m.ctypes.data
    mats[0].log_height = 8
    mats[0].width = 3
    mats[0].shift = F.lde_shift(0)
    root = (C.c_uint32 * 8)()
    for field, b, patch in ((0, 17, None), (5, 1, None), (0, 1, ("flags", 0x40)), (0, 1, ("values", None))):
        if patch:
            setattr(mats[0], *patch)
        assert lib.pico_gpu_commit(gpu.handle, field, mats, 1, b, 0, None, root) == abi.PICO_ERR_INVALID_ARG
        mats[0].flags = 0
        mats[0].values = m.ctypes.data
    assert lib.pico_gpu_coset_lde_batch(gpu.handle, 0, m.ctypes.data, 8, 3, 17, 1, None, 0) != abi.PICO_OK
    want = orc.pcs_commit(0, [m], [F.lde_shift(0)], 1)[0]
    got, _ = TwoAdicFriPcs(gpu, 0, 1).commit([(TwoAdicDomain(8), m)], keep=False)
    assert got.tolist() == want.tolist()


def test_reserve_pool_grows_the_pool_and_reports_failures(gpu):
    """pico_gpu_reserve_pool: the pool holds at least what was asked, the
    budget accounting is untouched, and an allocation failure on the way is
    reported as PICO_ERR_OUT_OF_MEMORY with the context still usable."""
    lib = abi.load()
    before = gpu.reserve_pool(0)
    after = gpu.reserve_pool(before + (256 << 20))
    assert after >= before + (256 << 20)
    assert gpu.memory()[0] == 0
    lib.pico_gpu_test_fail_allocations(0)
    try:
        with pytest.raises(PicoError) as e:
            gpu.reserve_pool(after + (64 << 20))
        assert e.value.status == abi.PICO_ERR_OUT_OF_MEMORY
    finally:
        lib.pico_gpu_test_fail_allocations(-1)
    assert gpu.reserve_pool(0) >= after


def test_grouped_requests_survive_an_allocation_failure(orc):
    """An allocation that fails while device-input requests are admitted as a
    group: every request either finishes with its oracle root or reports
    PICO_ERR_OUT_OF_MEMORY, every reserved byte comes back, and the next
    group is bit-exact.  (Which request meets the failure depends on timing;
    the outcome rules do not.)"""
    import time

    import torch

    lib = abi.load()
    f, b = 0, 1
    big = torch.from_numpy(F.random_matrix(f, 22, 64, 2600).view(np.int32)).cuda()
    small = [mats_of(f, [(9 + i, 5), (7, 3)], 2610 + 10 * i) for i in range(4)]
    want = [orc.pcs_commit(f, m, [F.lde_shift(f)] * 2, b)[0] for m in small]
    dev = [[torch.from_numpy(x.view(np.int32)).cuda() for x in m] for m in small]
    with GpuContext(0, n_streams=2, max_inflight=1, max_group=8) as ctx:
        server = CommitServer(ctx)
        first = server.submit(f, [big], b)  # holds the only slot while the others queue
        time.sleep(0.05)
        lib.pico_gpu_test_fail_allocations(0)
        try:
            reqs = [server.submit(f, d, b) for d in dev]
            failed = 0
            try:
                first.wait(timeout_ms=120_000, keep=False)
            except PicoError as e:
                assert e.status == abi.PICO_ERR_OUT_OF_MEMORY
                failed += 1
            for r, w in zip(reqs, want):
                try:
                    root, _ = r.wait(timeout_ms=120_000, keep=False)
                    assert root.tolist() == w.tolist()
                except PicoError as e:
                    assert e.status == abi.PICO_ERR_OUT_OF_MEMORY
                    failed += 1
                r.free()
            assert failed >= 1  # the one injected failure reached a request (a group fails whole)
        finally:
            lib.pico_gpu_test_fail_allocations(-1)
        first.free()
        assert ctx.memory()[0] == 0
        # the same requests again, after the injection: all bit-exact
        first = server.submit(f, [big], b)
        reqs = [server.submit(f, d, b) for d in dev]
        first.wait(timeout_ms=120_000, keep=False)
        for r, w in zip(reqs, want):
            root, _ = r.wait(timeout_ms=120_000, keep=False)
            assert root.tolist() == w.tolist()
            r.free()
        first.free()
        assert ctx.memory()[0] == 0
