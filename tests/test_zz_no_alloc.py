"""The allocation-free LDE entry point (pico_gpu_coset_lde_batch_noalloc).

Some callers cannot let the library allocate device memory: a prover that has
reserved all of HBM for its own arena, or a latency-bound loop that cannot
afford cudaMalloc/cudaFree's device-wide synchronisation.  This entry point
takes its scratch from a fixed array inside the library.  The test calls it
through the C ABI twice in a row (the second call finds the first call's data
in the shared scratch) and compares each result bit-exactly with the
allocating entry point, pico_gpu_coset_lde_batch, after checking with
pico_gpu_noalloc_status that no kernel skipped an access.  This file sorts last so a
run that stops at the first failure has already run every other test.
"""
import numpy as np
import pytest

from pico_b200 import PicoError, Radix2DitParallel, abi
from pico_b200 import fields as F

pytestmark = pytest.mark.gpu

# (field, log_n, width, log_blowup): three-pass shapes that fit the 8 Mi-word
# scratch, and a one-pass shape.
CASES = [(0, 16, 24, 1), (1, 13, 7, 2), (0, 10, 33, 1)]


def test_noalloc_lde_matches_allocating_entry_point(gpu):
    import torch

    lib = abi.load()
    stream = torch.cuda.current_stream()
    for f, log_n, w, b in CASES:
        m = F.random_matrix(f, log_n, w, 4242 + log_n)
        shift = F.lde_shift(f)
        want = Radix2DitParallel(gpu, f).coset_lde_batch_bitrev(m, b, shift)
        din = torch.from_numpy(m.view(np.int32)).cuda()
        for _ in range(2):
            dout = torch.full(((1 << (log_n + b)), w), -1, dtype=torch.int32, device="cuda")
            abi.check(lib.pico_gpu_coset_lde_batch_noalloc(f, din.data_ptr(), log_n, w, b, shift, dout.data_ptr(),
                                                           stream.cuda_stream))
            # waits for the stream and reports any skipped out-of-range access
            abi.check(lib.pico_gpu_noalloc_status(stream.cuda_stream))
            assert (dout.cpu().numpy().view(np.uint32) == want).all()


def test_noalloc_rejects_sizes_beyond_its_scratch(gpu):
    import torch

    lib = abi.load()
    din = torch.zeros(16, dtype=torch.int32, device="cuda")
    # 2^20 x 64 with blowup 2 needs 2^26 * 5 words, far beyond the 8 Mi-word scratch;
    # the size check rejects it before anything is launched.
    with pytest.raises(PicoError, match="static scratch"):
        abi.check(lib.pico_gpu_coset_lde_batch_noalloc(0, din.data_ptr(), 20, 64, 2, F.lde_shift(0),
                                                       din.data_ptr(), torch.cuda.current_stream().cuda_stream))
