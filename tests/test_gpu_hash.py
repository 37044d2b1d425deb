"""GPU hash cores (SHA-256, SHA-512, Keccak SHAKE128/256) through the batched
core_hash entry point (hash.c:29-65) against hashlib, across block and rate
boundaries and unaligned message offsets."""
import hashlib

import numpy as np
import pytest

LENS = [0, 1, 3, 4, 5, 31, 32, 55, 56, 63, 64, 65, 96, 111, 112, 119, 127, 128, 129, 135, 136, 137,
        167, 168, 169, 255, 256, 1000, 4096, 4099]

FAMILIES = [
    (0, 32, lambda m, n: hashlib.sha256(m).digest()),
    (0, 24, lambda m, n: hashlib.sha256(m).digest()[:24]),
    (0, 64, lambda m, n: hashlib.sha512(m).digest()),
    (1, 32, lambda m, n: hashlib.shake_128(m).digest(n)),
    (2, 24, lambda m, n: hashlib.shake_256(m).digest(n)),
    (2, 32, lambda m, n: hashlib.shake_256(m).digest(n)),
    (2, 64, lambda m, n: hashlib.shake_256(m).digest(n)),
]


@pytest.mark.gpu
@pytest.mark.parametrize("func,n,ref", FAMILIES)
def test_core_hash_vs_hashlib(xb, func, n, ref):
    rng = np.random.default_rng(func * 100 + n)
    msgs = [rng.bytes(L) for L in LENS]
    # odd leading pad shifts every message off 4-byte alignment
    got = xb.core_hash_batch(func, n, [b"x" * 3] + msgs)[1:]
    for L, m, g in zip(LENS, msgs, got):
        assert g == ref(m, n), (func, n, L)
