"""B200-native trace commitment for the Pico STARK prover.

The hot path of the reference prover's `pcs.commit` -- batched coset LDE over
KoalaBear / BabyBear, Poseidon2-16 Merkle commitment with mixed-height
injection, and the FRI commit-phase fold -- as sm_100a CUDA kernels behind the
C ABI in include/pico_gpu.h (libpico_gpu.so, built in-tree by build.py).
This package is the host-side mirror of the prover's trait surface.
"""
from . import abi, fields
from .abi import PicoError
from .pcs import (
    CommitRequest,
    CommitServer,
    FriCommitResult,
    GpuContext,
    MerkleTreeMmcs,
    Poseidon2,
    ProverData,
    Radix2DitParallel,
    TwoAdicDomain,
    TwoAdicFriPcs,
    new_challenger,
)

__all__ = [
    "abi",
    "fields",
    "PicoError",
    "GpuContext",
    "TwoAdicFriPcs",
    "TwoAdicDomain",
    "MerkleTreeMmcs",
    "Radix2DitParallel",
    "Poseidon2",
    "ProverData",
    "FriCommitResult",
    "CommitServer",
    "CommitRequest",
    "new_challenger",
]
