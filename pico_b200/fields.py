"""Host-side field constants, Montgomery conversions and the seeded input
generator used for synthetic traces.

KoalaBear p = 2^31 - 2^24 + 1, BabyBear p = 2^31 - 2^27 + 1; elements are
stored as x * 2^32 mod p (Plonky3 MontyField31).  GENERATOR is the coset
generator of vm/src/compiler/recursion/ir/utils.rs:13-19.
"""
from __future__ import annotations

import numpy as np

KOALABEAR = 0
BABYBEAR = 1

P = {KOALABEAR: 0x7F000001, BABYBEAR: 0x78000001}
TWO_ADICITY = {KOALABEAR: 24, BABYBEAR: 27}
GENERATOR = {KOALABEAR: 3, BABYBEAR: 31}
NAMES = {KOALABEAR: "koalabear", BABYBEAR: "babybear"}


def field_id(field) -> int:
    if isinstance(field, str):
        return {"koalabear": KOALABEAR, "kb": KOALABEAR, "babybear": BABYBEAR, "bb": BABYBEAR}[field.lower()]
    return int(field)


def to_monty(field, x):
    p = P[field_id(field)]
    a = np.asarray(x, dtype=np.uint64) % np.uint64(p)
    return ((a << np.uint64(32)) % np.uint64(p)).astype(np.uint32)


def from_monty(field, x):
    p = P[field_id(field)]
    rinv = pow(2**32 % p, p - 2, p)
    a = np.asarray(x, dtype=np.uint64) % np.uint64(p)
    return ((a * np.uint64(rinv)) % np.uint64(p)).astype(np.uint32)


def monty(field, v: int) -> int:
    p = P[field_id(field)]
    return ((v % p) << 32) % p


def unmonty(field, v: int) -> int:
    p = P[field_id(field)]
    return (v * pow(2**32 % p, p - 2, p)) % p


def inv(field, v: int) -> int:
    p = P[field_id(field)]
    return pow(v % p, p - 2, p)


def two_adic_generator(field, bits: int) -> int:
    """Canonical w with order 2^bits: GENERATOR^((p-1) / 2^bits)."""
    f = field_id(field)
    if bits > TWO_ADICITY[f]:
        raise ValueError("bits exceeds two-adicity")
    p = P[f]
    return pow(GENERATOR[f], (p - 1) >> bits, p)


def lde_shift(field, domain_shift_canonical: int = 1) -> int:
    """Monty-form LDE shift GENERATOR / domain.shift (TwoAdicFriPcs::commit)."""
    f = field_id(field)
    p = P[f]
    return monty(f, GENERATOR[f] * inv(f, domain_shift_canonical) % p)


_MASK64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n outputs of SplitMix64 starting from `seed` (vectorised, wrapping)."""
    with np.errstate(over="ignore"):
        gamma = np.uint64(0x9E3779B97F4A7C15)
        idx = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + idx * gamma
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(field, n: int, seed: int) -> np.ndarray:
    """n canonical elements uniform in [0, p): 31-bit SplitMix64 draws,
    rejection-sampled against p (deterministic for a given seed)."""
    p = P[field_id(field)]
    out = np.empty(0, dtype=np.uint32)
    start = 0
    while out.size < n:
        want = (n - out.size) * 17 // 16 + 64
        z = splitmix64(seed + start * 0x9E3779B97F4A7C15, want)
        v = (z >> np.uint64(33)).astype(np.uint32)
        out = np.concatenate([out, v[v < p]])
        start += want
    return out[:n]


def random_matrix(field, log_height: int, width: int, seed: int) -> np.ndarray:
    """Seeded (2^log_height, width) matrix of Monty-form elements."""
    vals = uniform(field, (1 << log_height) * width, seed)
    return to_monty(field, vals).reshape(1 << log_height, width)


def _lsr(z, k: int):
    """Logical right shift of int64 tensors holding u64 bit patterns."""
    import torch

    return (z >> k) & ((1 << (64 - k)) - 1)


def splitmix64_torch(seed: int, n: int, device):
    """SplitMix64 as in splitmix64(), computed with torch int64 (wrapping)."""
    import torch

    def s64(v: int) -> int:  # u64 constant as a signed int64
        v &= 0xFFFFFFFFFFFFFFFF
        return v - (1 << 64) if v >= 1 << 63 else v

    idx = torch.arange(1, n + 1, dtype=torch.int64, device=device)
    z = s64(seed) + idx * s64(0x9E3779B97F4A7C15)
    z = (z ^ _lsr(z, 30)) * s64(0xBF58476D1CE4E5B9)
    z = (z ^ _lsr(z, 27)) * s64(0x94D049BB133111EB)
    return z ^ _lsr(z, 31)


def uniform_torch(field, n: int, seed: int, device, chunk: int = 1 << 26):
    """Same stream as uniform(), generated on `device` (int32 tensor holding u32)."""
    import torch

    p = P[field_id(field)]
    parts, have, start = [], 0, 0
    while have < n:
        want = min((n - have) * 17 // 16 + 64, chunk)
        z = splitmix64_torch(seed + start * 0x9E3779B97F4A7C15, want, device)
        v = _lsr(z, 33)
        v = v[v < p]
        parts.append(v)
        have += v.numel()
        start += want
    return torch.cat(parts)[:n]


def random_matrix_torch(field, log_height: int, width: int, seed: int, device):
    """Device twin of random_matrix(): Monty-form int32 tensor (u32 bit patterns)."""
    import torch

    p = P[field_id(field)]
    v = uniform_torch(field, (1 << log_height) * width, seed, device)
    m = (v << 32) % p
    return m.to(torch.int32).reshape(1 << log_height, width)
