"""Byte-exact pins of the workload parameter sets that the other tests reach
only through verify statuses:

* the batched-keygen workload (8 x XMSS-SHA2_16_256 + 1 x XMSS-SHA2_20_256
  from seeded seeds): every public and secret key equal to the golden keys
  made by the reference's own C path (h = 16) and the threaded oracle
  (h = 20) from the same seeds (tests/golden/keygen_config3.json);
* XMSS^MT 20/2 and 40/4 batched signing (xmss_b200_sign_batch) of runs of
  consecutive indices that cross subtree boundaries of the bottom layer (and,
  for 40/4, of the layer above), messages log-uniform in 32 B..64 KB: every
  signature and every advanced sk equal to the oracle's
  (xmss_core.c:183-273, sign with treehash per layer; the oracle signs from
  node arrays it builds on all host cores, same bytes).
"""
import os
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_keygen_workload_keys_match_golden(xb, golden):
    doc = golden("keygen_config3.json")
    by_oid = {}
    for k in doc["keys"]:
        by_oid.setdefault(k["oid"], []).append(k)
    assert sorted((o, len(v)) for o, v in by_oid.items()) == [(0x02, 8), (0x03, 1)]
    for oid, keys in by_oid.items():
        p = xb.parse_oid(oid)
        seeds = np.stack([np.frombuffer(bytes.fromhex(k["seed"]), np.uint8) for k in keys])
        pks, sks = xb.keypair_batch(oid, False, seeds)
        for k, pk, sk in zip(keys, pks, sks):
            seed = bytes.fromhex(k["seed"])
            want_pk = bytes.fromhex(k["pk"])
            assert pk[4:].tobytes() == want_pk, (oid, k["seed"][:16])
            # sk = idx 0 || SK_SEED || SK_PRF || root || PUB_SEED (xmss_core.c:150-158)
            ib, n = p.index_bytes, p.n
            assert sk[4:].tobytes() == bytes(ib) + seed[:2 * n] + want_pk[:n] + seed[2 * n:]


@pytest.mark.parametrize("name", ["XMSS-SHA2_10_256", "XMSS-SHA2_10_192", "XMSS-SHA2_10_512", "XMSS-SHAKE_10_256",
                                  "XMSS-SHAKE256_10_192", "XMSS-SHAKE_10_512", "XMSSMT-SHA2_20/4_256"])
def test_in_cta_subtrees_match_oracle(xb, oracle, name):
    """Subtrees built as in-CTA subtrees of height 5, 6 and 7 (one thread per
    leaf, streaming L-tree, lower Merkle levels in shared memory; WOTS
    lengths 51, 67 and 131) give the keys and signatures of the
    one-thread-per-chain form and of the oracle."""
    mt = name.startswith("XMSSMT")
    oid = xb.xmssmt_str_to_oid(name) if mt else xb.xmss_str_to_oid(name)
    p, po = xb.parse_oid(oid, mt), oracle.params(oid, mt)
    rng = np.random.default_rng(zlib.crc32(name.encode()) + 1)
    seeds = np.frombuffer(rng.bytes(3 * 3 * p.n), np.uint8).reshape(3, -1)
    # the oracle's public key of the first seed (top-layer tree on all cores)
    s0 = seeds[0].tobytes()
    top = oracle.tree_nodes(po, s0[:p.n], s0[2 * p.n:], p.d - 1, 0, os.cpu_count() or 1)
    saved = xb.tree_tuning_get(oid, mt)
    try:
        xb.tree_tuning_set(oid, mt, 0, 0)
        want_pk, want_sk = xb.keypair_batch(oid, mt, seeds)
        assert want_pk[0, 4:].tobytes() == top[-p.n:] + s0[2 * p.n:]
        idx = int(rng.integers(0, (1 << p.full_height) - 1))
        msg = rng.bytes(int(rng.integers(0, 3000)))
        row = want_sk[:1].copy()
        row[0, 4:4 + p.index_bytes] = np.frombuffer(idx.to_bytes(p.index_bytes, "big"), np.uint8)
        ret, want_sm = xb.sign_batch(mt, row.copy(), [msg])
        assert ret[0] == 0
        for k in (5, 6, 7):
            xb.tree_tuning_set(oid, mt, k, 0)
            assert xb.tree_tuning_get(oid, mt)["chains_per_warp"] == 32 * p.wots_len
            pk, sk = xb.keypair_batch(oid, mt, seeds)
            assert (pk == want_pk).all() and (sk == want_sk).all(), (name, k)
            ret, sm = xb.sign_batch(mt, row.copy(), [msg])
            assert ret[0] == 0 and sm == want_sm, (name, k)
        # the signature itself against the oracle
        sk = row[0, 4:].tobytes()
        ib, n, th = p.index_bytes, p.n, p.tree_height
        trees = b"".join(oracle.tree_nodes(po, sk[ib:ib + n], sk[ib + 3 * n:ib + 4 * n], layer,
                                           idx >> (th * (layer + 1)) if th * (layer + 1) < 64 else 0,
                                           os.cpu_count() or 1) for layer in range(p.d))
        assert oracle.sign(po, sk, msg, trees=trees)[2] == want_sm[0]
    finally:
        xb.tree_tuning_set(oid, mt, saved["subtree_height"], saved["min_leaves"])


def test_in_cta_subtrees_keygen_workload_golden(xb, golden):
    """The h = 16 and h = 20 golden keys again with the in-CTA form forced."""
    doc = golden("keygen_config3.json")
    for oid in (0x02, 0x03):
        keys = [k for k in doc["keys"] if k["oid"] == oid][:2]
        seeds = np.stack([np.frombuffer(bytes.fromhex(k["seed"]), np.uint8) for k in keys])
        saved = xb.tree_tuning_get(oid, False)
        try:
            xb.tree_tuning_set(oid, False, 7, 0)
            pks, _ = xb.keypair_batch(oid, False, seeds)
        finally:
            xb.tree_tuning_set(oid, False, saved["subtree_height"], saved["min_leaves"])
        assert [pk[4:].tobytes().hex() for pk in pks] == [k["pk"] for k in keys]


def test_bench_workload_same_bytes_from_gpu_and_oracle(xb):
    """bench.py's two arms build the verify workload independently: the GPU
    arm with this library, the reference arm with the CPU oracle.  Both
    must give the same bytes (keys, signed messages with their corruptions,
    expected statuses), including signatures at the wiped last index."""
    import bench

    count, keys = 64, 3
    p = xb.parse_oid(bench.OID)
    rank = next(r for r in range(500)
                if (bench._workload_draws(np.random.default_rng(bench.SEED + r), p.n, p.full_height, count,
                                          keys)[2] == 1023).any())
    g = bench.make_workload(xb, rank, count=count, keys=keys)
    c = bench.make_workload_cpu(rank, count=count, keys=keys)
    assert (g["pks"] == c["pks"]).all()
    assert g["sms"] == c["sms"]
    assert (g["expect"] == c["expect"]).all() and (g["expect"] == -1).any()
    assert (xb.sign_open_batch(False, g["buf"], g["off"], g["len"], g["pks"], g["keyix"]) == g["expect"]).all()


def _oracle_trees(oracle, po, sk, idx, cache):
    """Concatenated node arrays of the subtrees that signing at idx uses,
    one per layer, built by the oracle on all host cores (cached)."""
    ib, n, th = po.index_bytes, po.n, po.tree_height
    out = []
    for layer in range(po.d):
        tree = idx >> (th * (layer + 1)) if th * (layer + 1) < 64 else 0
        key = (layer, tree)
        if key not in cache:
            cache[key] = oracle.tree_nodes(po, sk[ib:ib + n], sk[ib + 3 * n:ib + 4 * n], layer, tree,
                                           os.cpu_count() or 1)
        out.append(cache[key])
    return b"".join(out)


@pytest.mark.parametrize("name,start,count", [
    ("XMSSMT-SHA2_20/2_256", 7 * 1024 - 40, 80),            # one bottom-subtree boundary
    ("XMSSMT-SHA2_40/4_256", (5 << 20) - 40, 80),           # bottom and second-layer boundaries
])
def test_mt_batched_sign_consecutive_indices(xb, oracle, name, start, count):
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    oid = xb.xmssmt_str_to_oid(name)
    p, po = xb.parse_oid(oid, True), oracle.params(oid, True)
    seed = rng.bytes(3 * p.n)
    pks, sks = xb.keypair_batch(oid, True, np.frombuffer(seed, np.uint8)[None, :])
    # the public key from the oracle's top-layer tree (layer d-1, tree 0)
    top = oracle.tree_nodes(po, seed[:p.n], seed[2 * p.n:], p.d - 1, 0, os.cpu_count() or 1)
    assert pks[0, 4:].tobytes() == top[-p.n:] + seed[2 * p.n:]
    sk0 = sks[0, 4:].tobytes()
    mlen = np.exp(rng.uniform(np.log(32), np.log(65536), count)).astype(int)
    msgs = [rng.bytes(int(L)) for L in mlen]
    ib = p.index_bytes
    rows = np.repeat(sks[:1], count, axis=0)
    for i in range(count):
        rows[i, 4:4 + ib] = np.frombuffer((start + i).to_bytes(ib, "big"), np.uint8)
    ret, sms = xb.sign_batch(True, rows, msgs)
    assert (ret == 0).all()
    cache = {}
    for i in range(count):
        sk = (start + i).to_bytes(ib, "big") + sk0[ib:]
        ro, sk_after, smo = oracle.sign(po, sk, msgs[i], trees=_oracle_trees(oracle, po, sk, start + i, cache))
        assert ro == 0 and sms[i] == smo, (name, start + i)
        assert rows[i, 4:].tobytes() == sk_after, (name, start + i)  # index advanced in place
    # the layers that change across the run were really crossed
    assert len({k for k in cache if k[0] == 0}) == 2
    if p.d == 4:
        assert len({k for k in cache if k[0] == 1}) == 2
    # and the batch verifies, with corruptions rejected as the oracle rejects them
    sms = [bytearray(s) for s in sms]
    expect = np.zeros(count, np.int32)
    for i in range(0, count, 9):
        sms[i][int(rng.integers(0, len(sms[i])))] ^= 1 << int(rng.integers(0, 8))
        expect[i] = oracle.sign_open(po, bytes(sms[i]), pks[0, 4:].tobytes())[0]
    buf, off, ln = xb.pack([bytes(s) for s in sms], align=16)
    st = xb.sign_open_batch(True, buf, off, ln, pks, np.zeros(count, np.uint32))
    assert (st == expect).all()
