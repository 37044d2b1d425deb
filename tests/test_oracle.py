"""The CPU oracle against the hash standards and the reference's own
outputs (golden fixtures made from the reference C path)."""
import hashlib
import os

import numpy as np
import pytest


@pytest.mark.parametrize("n", [0, 1, 31, 55, 56, 63, 64, 65, 111, 112, 127, 128, 135, 136, 167, 168, 169, 500])
def test_hash_primitives_vs_hashlib(oracle, n):
    m = np.random.default_rng(n).bytes(n)
    assert oracle.sha256(m) == hashlib.sha256(m).digest()
    assert oracle.sha512(m) == hashlib.sha512(m).digest()
    for ol in (10, 24, 32, 64, 300):
        assert oracle.shake128(m, ol) == hashlib.shake_128(m).digest(ol)
        assert oracle.shake256(m, ol) == hashlib.shake_256(m).digest(ol)


def test_reference_vectors(oracle, golden):
    """All 21 lines of the reference's test/vectors.c output (WOTS+, XMSS and
    XMSS^MT over every hash family) reproduced by the oracle."""
    assert oracle.vectors_lines() == golden("vectors.txt")


def test_config1_keypair_and_signatures(oracle, golden):
    g = golden("config1.json")
    p = oracle.params(1)
    seed = bytes.fromhex(g["seed"])
    nodes = oracle.tree_nodes(p, seed[:32], seed[64:], 0, 0, os.cpu_count())
    pk = nodes[-32:] + seed[64:]
    assert "00000001" + pk.hex() == g["pk"]
    sk = bytes.fromhex(g["sk"])[4:]
    for i, (m, sm) in enumerate(zip(g["msgs"], g["sms"])):
        r, sk, got = oracle.sign(p, sk, bytes.fromhex(m), trees=nodes)
        assert r == 0 and got.hex() == sm, i
        assert "00000001" + sk.hex() == g["sk_after"][i]
        assert oracle.sign_open(p, got, pk)[0] == 0
        bad = bytearray(got)
        bad[-1] ^= 1
        assert oracle.sign_open(p, bytes(bad), pk)[0] == -1


def test_mt_small_every_family(oracle, golden):
    for k in golden("mt_small.json"):
        p = oracle.params(k["oid"], True)
        pk, sk = oracle.seed_keypair(p, bytes.fromhex(k["seed"]))
        assert pk.hex() == k["pk"] and sk.hex() == k["sk"], k["oid"]
        for s in k["sigs"]:
            skx = s["idx"].to_bytes(p.index_bytes, "big") + sk[p.index_bytes:]
            r, _, sm = oracle.sign(p, skx, bytes.fromhex(s["m"]))
            assert r == 0 and sm.hex() == s["sm"], (k["oid"], s["idx"])
            assert oracle.sign_open(p, sm, pk) == (0, bytes.fromhex(s["m"]))


def test_exhaustion_quirk(oracle):
    """xmss_core.c:212-231: index 2^h-1 signs with a wiped key, then -2."""
    p = oracle.params(0x02, True)  # XMSSMT-SHA2_20/4_256, tree height 5
    seed = np.random.default_rng(7).bytes(3 * p.n)
    pk, sk = oracle.seed_keypair(p, seed)
    last = (1 << p.full_height) - 1
    sk = last.to_bytes(p.index_bytes, "big") + sk[p.index_bytes:]
    r, sk2, sm = oracle.sign(p, sk, b"abc")
    assert r == 0
    assert sk2[:p.index_bytes] == (last + 1).to_bytes(p.index_bytes, "big")
    assert sk2[p.index_bytes:] == bytes(p.sk_bytes - p.index_bytes)
    assert sm[:p.index_bytes] == b"\xff" * p.index_bytes
    assert oracle.sign_open(p, sm, pk)[0] == -1
    r, sk3, _ = oracle.sign(p, sk2, b"abc")
    assert r == -2 and sk3[:p.index_bytes] == b"\xff" * p.index_bytes


def test_oracle_against_compiled_reference(oracle):
    """When the reference C path was compiled here (oracle/_ref), random
    keygen / sign / verify cases agree byte for byte."""
    from oracle import REF_PATH, RefLib

    if not os.path.exists(REF_PATH):
        pytest.skip("reference build oracle/_ref not present")
    ref = RefLib()
    rng = np.random.default_rng(11)
    for oid, mt in ((0x02, True), (0x0A, True), (0x12, True), (0x22, True), (0x2A, True), (0x32, True)):
        p, rp = oracle.params(oid, mt), ref.params(oid, mt)
        assert p.as_dict() == rp.as_dict()
        seed = rng.bytes(3 * p.n)
        assert oracle.seed_keypair(p, seed) == ref.seed_keypair(rp, seed)
        pk, sk = oracle.seed_keypair(p, seed)
        idx = int(rng.integers(0, 1 << p.full_height))
        skx = idx.to_bytes(p.index_bytes, "big") + sk[p.index_bytes:]
        m = rng.bytes(int(rng.integers(0, 200)))
        a, b = oracle.sign(p, skx, m), ref.sign(rp, skx, m)
        assert a == b
        bad = bytearray(a[2])
        bad[int(rng.integers(0, len(bad)))] ^= 1 << int(rng.integers(0, 8))
        assert oracle.sign_open(p, bytes(bad), pk) == ref.sign_open(rp, bytes(bad), pk)
