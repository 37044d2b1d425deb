"""XMSS / XMSS^MT on the GPU through the C-ABI, byte for byte against the
reference's own outputs (golden fixtures) and the CPU oracle."""
import hashlib
import os
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def h10(b):
    return hashlib.shake_128(b).hexdigest(10)


def test_config1_plain_api(xb, golden):
    """Config 1: keypair from a seeded 96-byte seed, 16 signatures of 32-byte
    messages at indices 0..15 through xmss_sign, each verified through
    xmss_sign_open; pk, sk and every signature byte-identical to the
    reference C path."""
    g = golden("config1.json")
    p = xb.parse_oid(1)
    r, pk, sk = xb.xmssmt_core_seed_keypair(p, bytes.fromhex(g["seed"]))
    assert r == 0
    assert "00000001" + pk.hex() == g["pk"]
    assert "00000001" + sk.hex() == g["sk"]
    sk = bytes.fromhex(g["sk"])
    pkf = bytes.fromhex(g["pk"])
    for i, m in enumerate(g["msgs"]):
        m = bytes.fromhex(m)
        r, sk, sm = xb.xmss_sign(sk, m)
        assert r == 0
        assert sm.hex() == g["sms"][i], i
        assert sk.hex() == g["sk_after"][i]
        assert xb.xmss_sign_open(sm, pkf) == (0, m)
        bad = bytearray(sm)
        bad[-1] ^= 1  # flip the last message bit (test/xmss.c:233-242)
        assert xb.xmss_sign_open(bytes(bad), pkf) == (-1, b"")


def test_invalid_signature_every_hash(xb, golden):
    """One bit per n-byte hash of the signature, index included
    (test/xmss.c:244-261, XMSS_TEST_INVALIDSIG), must reject: checked as one
    batch."""
    g = golden("config1.json")
    pk = np.frombuffer(bytes.fromhex(g["pk"]), np.uint8)[None, :]
    sm = bytes.fromhex(g["sms"][3])
    mlen = 32
    variants = []
    for j in range(0, len(sm) - mlen, 32):
        b = bytearray(sm)
        b[j] ^= 1
        variants.append(bytes(b))
    variants.append(sm)
    buf, off, ln = xb.pack(variants)
    st = xb.sign_open_batch(False, buf, off, ln, pk, np.zeros(len(variants), np.uint32))
    assert (st[:-1] == -1).all() and st[-1] == 0


def test_mt_small_every_family(xb, golden):
    """XMSS^MT 20/4 keys of all seven hash families: keygen, signature at a
    given index and verify equal the reference's bytes."""
    for k in golden("mt_small.json"):
        p = xb.parse_oid(k["oid"], True)
        r, pk, sk = xb.xmssmt_core_seed_keypair(p, bytes.fromhex(k["seed"]))
        assert r == 0 and pk.hex() == k["pk"] and sk.hex() == k["sk"], k["oid"]
        for s in k["sigs"]:
            skx = s["idx"].to_bytes(p.index_bytes, "big") + sk[p.index_bytes:]
            r, sk2, sm = xb.xmssmt_core_sign(p, skx, bytes.fromhex(s["m"]))
            assert r == 0 and sm.hex() == s["sm"], (k["oid"], s["idx"])
            assert xb.xmssmt_core_sign_open(p, sm, pk) == (0, bytes.fromhex(s["m"]))


def test_reference_vectors_xmss_lines(xb, golden):
    """The XMSS and XMSS^MT lines of the reference's test/vectors.c
    (seed[i] = i, signature of {37} at index 2^(h-1)) over every family."""
    want = [l for l in golden("vectors.txt") if not l.startswith("WOTS")]
    got = []
    for mt, oids in ((True, range(2, 57, 8)), (False, range(1, 0x15 + 1, 3))):
        for oid in oids:
            p = xb.parse_oid(oid, mt)
            seed = bytes(i & 0xFF for i in range(3 * p.n))
            r, pk, sk = xb.xmssmt_core_seed_keypair(p, seed)
            assert r == 0
            sk = (1 << (p.full_height - 1)).to_bytes(p.index_bytes, "big") + sk[p.index_bytes:]
            r, _, sm = xb.xmssmt_core_sign(p, sk, bytes([37]))
            assert r == 0
            got.append(f"{'XMSSMT' if mt else 'XMSS'} {oid} {h10(pk)} {h10(sm[:p.sig_bytes])}")
    assert got == want


def test_batch_verify_matches_oracle(xb, oracle):
    """A mixed batch: several keys, uneven message lengths (0 B..5 KB),
    random bit flips anywhere in sig || message; accept bitmap == oracle."""
    rng = np.random.default_rng(5)
    p = xb.parse_oid(0x01, True)  # XMSSMT-SHA2_20/2_256: two layers of height 10
    po = oracle.params(0x01, True)
    seeds = np.frombuffer(rng.bytes(3 * 32 * 3), np.uint8).reshape(3, 96)
    pks, sks = xb.keypair_batch(0x01, True, seeds)
    sms, keyix, flips = [], [], []
    for i in range(24):
        k = i % 3
        idx = int(rng.integers(0, 1 << 20))
        sk = bytes(sks[k, :4]) + idx.to_bytes(p.index_bytes, "big") + bytes(sks[k, 4 + p.index_bytes:])
        m = rng.bytes(int(rng.integers(0, 5000)))
        r, _, sm = xb.xmssmt_sign(sk, m)
        assert r == 0
        sm = bytearray(sm)
        if i % 4 == 1:
            pos = int(rng.integers(0, len(sm)))
            sm[pos] ^= 1 << int(rng.integers(0, 8))
        sms.append(bytes(sm))
        keyix.append(k)
    buf, off, ln = xb.pack(sms)
    st = xb.sign_open_batch(True, buf, off, ln, pks, np.array(keyix, np.uint32))
    want = [oracle.sign_open(po, sm, bytes(pks[k, 4:]))[0] for sm, k in zip(sms, keyix)]
    assert list(st) == want
    assert sum(1 for w in want if w == -1) >= 5


def test_exhaustion_quirk_matches_oracle(xb, oracle):
    """xmss_core.c:212-231 at the last index: the wiped key still signs
    (byte-identical garbage signature), then -2; the sk bytes follow."""
    p = xb.parse_oid(0x02, True)
    po = oracle.params(0x02, True)
    seed = np.random.default_rng(7).bytes(3 * p.n)
    r, pk, sk = xb.xmssmt_core_seed_keypair(p, seed)
    last = (1 << p.full_height) - 1
    sk = last.to_bytes(p.index_bytes, "big") + sk[p.index_bytes:]
    a = xb.xmssmt_core_sign(p, sk, b"abc")
    b = oracle.sign(po, sk, b"abc")
    assert a == b and a[0] == 0
    a2 = xb.xmssmt_core_sign(p, a[1], b"abc")
    b2 = oracle.sign(po, b[1], b"abc")
    assert a2[0] == -2 and a2[:2] == b2[:2]
    assert a2[2][p.sig_bytes:] == b"abc"


def test_determinism_and_empty_message(xb):
    """Same sk copy signs the same bytes twice (test/xmss_determinism.c);
    empty messages sign and verify; short sm is rejected."""
    p = xb.parse_oid(0x02, True)
    r, pk, sk = xb.xmssmt_core_seed_keypair(p, bytes(range(96)))
    a = xb.xmssmt_core_sign(p, sk, b"")
    b = xb.xmssmt_core_sign(p, sk, b"")
    assert a == b and a[0] == 0 and len(a[2]) == p.sig_bytes
    assert xb.xmssmt_core_sign_open(p, a[2], pk) == (0, b"")
    assert xb.xmssmt_core_sign_open(p, a[2][:-1], pk)[0] == -1


def test_sign_batch_shares_subtrees(xb, oracle):
    """Batched signing of consecutive indices of one key (and copies of
    another) equals one-by-one signing by the oracle."""
    p = xb.parse_oid(0x02, True)
    po = oracle.params(0x02, True)
    rng = np.random.default_rng(9)
    seeds = np.frombuffer(rng.bytes(2 * 96), np.uint8).reshape(2, 96)
    pks, sks = xb.keypair_batch(0x02, True, seeds)
    rows, msgs = [], []
    for i in range(12):
        k = i % 2
        idx = 30 + i
        rows.append(np.concatenate([sks[k, :4], np.frombuffer(idx.to_bytes(p.index_bytes, "big"), np.uint8),
                                    sks[k, 4 + p.index_bytes:]]))
        msgs.append(rng.bytes(int(rng.integers(1, 300))))
    sk_arr = np.stack(rows)
    want = [oracle.sign(po, bytes(r[4:]), m) for r, m in zip(sk_arr, msgs)]
    ret, sms = xb.sign_batch(True, sk_arr, msgs)
    for i, (w, sm) in enumerate(zip(want, sms)):
        assert ret[i] == 0 and sm == w[2] and bytes(sk_arr[i, 4:]) == w[1], i


def test_sign_batch_long_messages_match_oracle(xb, oracle):
    """XMSS-SHA2_10_256 batch signing with the benchmark's message-length
    distribution (log-uniform 32 B..4 KB, unaligned lengths) equals the
    oracle's signatures, and the batch verify accepts them all."""
    rng = np.random.default_rng(21)
    p, po = xb.parse_oid(1), oracle.params(1)
    seeds = np.frombuffer(rng.bytes(2 * 96), np.uint8).reshape(2, 96)
    pks, sks = xb.keypair_batch(1, False, seeds)
    trees = [oracle.tree_nodes(po, bytes(s[:32]), bytes(s[64:]), 0, 0, os.cpu_count()) for s in seeds]
    for k in range(2):
        assert bytes(pks[k, 4:36]) == trees[k][-32:]
    count = 40
    keyix = rng.integers(0, 2, count)
    idx = rng.integers(0, 1024, count)
    mlen = np.exp(rng.uniform(np.log(32), np.log(4096), count)).astype(int)
    msgs = [rng.bytes(int(L)) for L in mlen]
    rows = np.array(sks[keyix])
    for i in range(count):
        rows[i, 4:8] = np.frombuffer(int(idx[i]).to_bytes(4, "big"), np.uint8)
    want = [oracle.sign(po, bytes(rows[i, 4:]), msgs[i], trees=trees[keyix[i]]) for i in range(count)]
    ret, sms = xb.sign_batch(False, rows.copy(), msgs)
    for i in range(count):
        assert ret[i] == 0 and sms[i] == want[i][2], (i, int(mlen[i]), int(idx[i]))
    buf, off, ln = xb.pack(sms, align=16)
    st = xb.sign_open_batch(False, buf, off, ln, pks, keyix.astype(np.uint32))
    assert (st == 0).all()


def test_large_batch_two_group_path(xb, oracle):
    """Batches of 1024+ signatures are verified as a short-H_msg and a
    long-H_msg group on two streams; the accept bitmap must still be exact
    (corruptions anywhere, the last-index quirk) and agree with the oracle."""
    rng = np.random.default_rng(41)
    p, po = xb.parse_oid(1), oracle.params(1)
    count, keys = 1100, 4
    seeds = np.frombuffer(rng.bytes(keys * 96), np.uint8).reshape(keys, 96)
    pks, sks = xb.keypair_batch(1, False, seeds)
    keyix = rng.integers(0, keys, count).astype(np.uint32)
    idx = rng.integers(0, 1024, count)
    idx[:3] = 1023
    mlen = np.exp(rng.uniform(np.log(1), np.log(4096), count)).astype(int)
    msgs = [rng.bytes(int(L)) for L in mlen]
    rows = np.array(sks[keyix])
    for i in range(count):
        rows[i, 4:8] = np.frombuffer(int(idx[i]).to_bytes(4, "big"), np.uint8)
    ret, sms = xb.sign_batch(False, rows, msgs)
    assert (ret == 0).all()
    expect = np.where(idx == 1023, -1, 0)
    sms = [bytearray(s) for s in sms]
    for i in range(5, count, 9):
        sms[i][int(rng.integers(0, len(sms[i])))] ^= 1 << int(rng.integers(0, 8))
        expect[i] = -1
    sms = [bytes(s) for s in sms]
    buf, off, ln = xb.pack(sms, align=8)
    st = xb.sign_open_batch(False, buf, off, ln, pks, keyix)
    assert (st == expect).all()
    for i in rng.choice(count, 40, replace=False):
        assert oracle.sign_open(po, sms[i], bytes(pks[keyix[i], 4:]))[0] == st[i]


def test_hmsg_block_edges_every_family(xb, oracle, golden):
    """H_msg streams prefix || M block by block (prefix blocks unrolled, body
    blocks prefetched and funnel-shifted, bounded tail).  For every hash
    family, message lengths around each block, rate and padding edge up to
    70 KB, signed at unaligned message offsets (XMSS^MT 20/4: 3 index bytes),
    must equal the oracle's signatures, and verify - with the message
    starting at any byte offset - must accept them and reject a bit flip at
    the start, middle or end of the message."""
    lengths = [0, 1, 2, 3, 5, 31, 63, 64, 65, 100, 127, 128, 129, 135, 136, 137, 167, 168, 169, 200, 255, 256,
               257, 300, 1000, 1023, 4099, 70001]
    rng = np.random.default_rng(77)
    for k in golden("mt_small.json"):
        p, po = xb.parse_oid(k["oid"], True), oracle.params(k["oid"], True)
        pk, sk = bytes.fromhex(k["pk"]), bytes.fromhex(k["sk"])
        oidb = k["oid"].to_bytes(4, "big")
        msgs = [rng.bytes(L) for L in lengths]
        idx = rng.integers(0, (1 << 20) - 1, len(msgs))
        rows = np.zeros((len(msgs), 4 + len(sk)), np.uint8)
        for i in range(len(msgs)):
            rows[i] = np.frombuffer(oidb + int(idx[i]).to_bytes(p.index_bytes, "big") + sk[p.index_bytes:], np.uint8)
        ret, sms = xb.sign_batch(True, rows.copy(), msgs)
        for i, m in enumerate(msgs):
            want = oracle.sign(po, bytes(rows[i, 4:]), m)[2]
            assert ret[i] == 0 and sms[i] == want, (k["oid"], len(m))
        variants, expect = [], []
        for sm, m in zip(sms, msgs):
            variants.append(sm)
            expect.append(0)
            for pos in (0, len(m) // 2, len(m) - 1) if m else ():
                b = bytearray(sm)
                b[p.sig_bytes + pos] ^= 1 << int(rng.integers(0, 8))
                variants.append(bytes(b))
                expect.append(-1)
        # byte offsets 0, 1, 2, 3, ... mod 4 for the signed messages
        pad = [rng.bytes(int(rng.integers(0, 4))) for _ in variants]
        buf, off, ln = xb.pack([q + v for q, v in zip(pad, variants)])
        off = off + np.array([len(q) for q in pad], np.uint64)
        ln = ln - np.array([len(q) for q in pad], np.uint64)
        pkarr = np.frombuffer(oidb + pk, np.uint8)[None, :]
        st = xb.sign_open_batch(True, buf, off, ln, pkarr, np.zeros(len(variants), np.uint32))
        assert list(st) == expect, k["oid"]


@pytest.mark.parametrize("name", ["XMSSMT-SHA2_40/8_256", "XMSSMT-SHA2_60/6_256", "XMSSMT-SHA2_60/12_256",
                                  "XMSSMT-SHAKE_20/4_512", "XMSSMT-SHA2_20/4_192",
                                  "XMSSMT-SHAKE256_60/12_192"])
def test_remaining_mt_heights(xb, oracle, name):
    """XMSS^MT heights and hash widths beyond the fixtures (8 and 12 layers,
    60-bit indices above 2^32, SHAKE256 with n = 64, SHA-256/192): keypair,
    signatures at seeded indices and verify equal the oracle's."""
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    oid = xb.xmssmt_str_to_oid(name)
    p, po = xb.parse_oid(oid, True), oracle.params(oid, True)
    seed = rng.bytes(3 * p.n)
    r, pk, sk = xb.xmssmt_core_seed_keypair(p, seed)
    pk_o, sk_o = oracle.seed_keypair(po, seed)
    assert r == 0 and pk == pk_o and sk == sk_o
    top = (1 << p.full_height) - 1
    for idx in (int(rng.integers(0, min(top, 1 << 31))), int(rng.integers(0, min(top, 1 << 62)))):
        m = rng.bytes(int(rng.integers(0, 500)))
        skx = idx.to_bytes(p.index_bytes, "big") + sk[p.index_bytes:]
        r, sk2, sm = xb.xmssmt_core_sign(p, skx, m)
        # the oracle signs from its own threaded node arrays of each layer's subtree
        ib, n, th = p.index_bytes, p.n, p.tree_height
        trees = b"".join(oracle.tree_nodes(po, sk[ib:ib + n], sk[ib + 3 * n:ib + 4 * n], layer,
                                           idx >> (th * (layer + 1)) if th * (layer + 1) < 64 else 0,
                                           os.cpu_count()) for layer in range(p.d))
        ro, sk2o, smo = oracle.sign(po, skx, m, trees=trees)
        assert r == ro == 0 and sm == smo and sk2 == sk2o, (name, idx)
        assert xb.xmssmt_core_sign_open(p, sm, pk) == (0, m)
        bad = bytearray(sm)
        bad[int(rng.integers(0, len(bad)))] ^= 1
        assert xb.xmssmt_core_sign_open(p, bytes(bad), pk)[0] == -1


def test_sign_open_batch_async_two_streams(xb, oracle):
    """The pipelined host-buffer verify (xmss_b200_sign_open_batch_async)
    gives the blocking call's statuses, with calls in flight on two streams
    at once over the same pinned inputs, including the split path of large
    batches."""
    import torch

    rng = np.random.default_rng(61)
    keys, count = 3, 1500
    seeds = np.frombuffer(rng.bytes(keys * 96), np.uint8).reshape(keys, 96)
    pks, sks = xb.keypair_batch(1, False, seeds)
    keyix = rng.integers(0, keys, count).astype(np.uint32)
    rows = np.array(sks[keyix])
    idx = rng.integers(0, 1024, count)
    for i in range(count):
        rows[i, 4:8] = np.frombuffer(int(idx[i]).to_bytes(4, "big"), np.uint8)
    msgs = [rng.bytes(int(L)) for L in np.exp(rng.uniform(0, np.log(5000), count)).astype(int)]
    ret, sms = xb.sign_batch(False, rows, msgs)
    sms = [bytearray(s) for s in sms]
    for i in range(0, count, 7):
        sms[i][int(rng.integers(0, len(sms[i])))] ^= 1
    buf, off, ln = xb.pack([bytes(s) for s in sms], align=16)
    want = xb.sign_open_batch(False, buf, off, ln, pks, keyix)
    assert (want[::7] == -1).sum() >= count // 7 - 3
    h_sm = torch.from_numpy(buf).pin_memory().numpy()
    outs = [torch.full((count,), 7, dtype=torch.int32).pin_memory().numpy() for _ in range(4)]
    streams = [torch.cuda.Stream() for _ in range(2)]
    sub = slice(0, 300)
    for i, o in enumerate(outs):
        if i < 2:
            xb.sign_open_batch_async(False, h_sm, off, ln, pks, keyix, o, streams[i % 2].cuda_stream)
        else:  # a small batch (no split) on the same streams
            xb.sign_open_batch_async(False, h_sm, np.ascontiguousarray(off[sub]), np.ascontiguousarray(ln[sub]),
                                     pks, np.ascontiguousarray(keyix[sub]), o, streams[i % 2].cuda_stream)
    torch.cuda.synchronize()
    assert (outs[0] == want).all() and (outs[1] == want).all()
    assert (outs[2][:300] == want[:300]).all() and (outs[3][:300] == want[:300]).all()

    # Calls queued ahead: a call waits only until the previous call on its
    # stream has copied its inputs, so several batches per stream are in
    # flight at once; small and large batches alternate, so a stream's
    # buffers grow while its earlier calls are still queued, and the host
    # arrays are rewritten between calls (they are read before a call
    # returns).
    plan = [slice(700, 1000), slice(0, count), slice(100, 250), slice(0, count), slice(1200, 1500), slice(0, count)]
    outs = [torch.full((count,), 7, dtype=torch.int32).pin_memory().numpy() for _ in range(2 * len(plan))]
    streams = [torch.cuda.Stream() for _ in range(2)]
    h_off, h_len, h_kix = off.copy(), ln.copy(), keyix.copy()
    for i, o in enumerate(outs):
        s = plan[i % len(plan)]
        n = s.stop - s.start
        h_off[:n], h_len[:n], h_kix[:n] = off[s], ln[s], keyix[s]
        xb.sign_open_batch_async(False, h_sm, np.ascontiguousarray(h_off[:n]), np.ascontiguousarray(h_len[:n]),
                                 pks, np.ascontiguousarray(h_kix[:n]), o, streams[i % 2].cuda_stream)
        h_off[:] = 0  # reuse of the host arrays after the call returned
    torch.cuda.synchronize()
    for i, o in enumerate(outs):
        s = plan[i % len(plan)]
        n = s.stop - s.start
        assert (o[:n] == want[s]).all(), i
        assert (o[n:] == 7).all(), i


@pytest.mark.parametrize("count", [300, 1100])
def test_verify_graph_replays(xb, count):
    """A verify captured in a CUDA graph (xmss_b200_verify_graph_*) gives the
    statuses of the plain device call, and replays read the buffers' current
    contents (refilled with other signatures between launches); 1,100
    signatures take the two-stream split inside the graph."""
    import torch

    rng = np.random.default_rng(83 + count)
    keys = 4
    seeds = np.frombuffer(rng.bytes(keys * 96), np.uint8).reshape(keys, 96)
    pks, sks = xb.keypair_batch(1, False, seeds)
    batches = []
    for _ in range(2):
        keyix = rng.integers(0, keys, count).astype(np.uint32)
        rows = np.array(sks[keyix])
        idx = rng.integers(0, 1023, count)
        for i in range(count):
            rows[i, 4:8] = np.frombuffer(int(idx[i]).to_bytes(4, "big"), np.uint8)
        msgs = [rng.bytes(int(L)) for L in np.exp(rng.uniform(0, np.log(3000), count)).astype(int)]
        _, sms = xb.sign_batch(False, rows, msgs)
        sms = [bytearray(s) for s in sms]
        for i in range(int(rng.integers(0, 5)), count, 5):
            sms[i][int(rng.integers(0, len(sms[i])))] ^= 1
        buf, off, ln = xb.pack([bytes(s) for s in sms], align=16)
        want = xb.sign_open_batch(False, buf, off, ln, pks, keyix)
        batches.append((buf, off, ln, keyix, want))
    cap = max(len(b[0]) for b in batches)
    dev = torch.device("cuda", 0)
    d_sm = torch.zeros(cap, dtype=torch.uint8, device=dev)
    d_off = torch.zeros(count, dtype=torch.int64, device=dev)
    d_len = torch.zeros(count, dtype=torch.int64, device=dev)
    d_kix = torch.zeros(count, dtype=torch.int32, device=dev)
    d_pk = torch.from_numpy(np.ascontiguousarray(pks[:, 4:])).to(dev)
    d_st = torch.full((count,), 7, dtype=torch.int32, device=dev)

    def load(b):
        buf, off, ln, keyix, _ = b
        d_sm[:len(buf)].copy_(torch.from_numpy(buf))
        d_off.copy_(torch.from_numpy(off.astype(np.int64)))
        d_len.copy_(torch.from_numpy(ln.astype(np.int64)))
        d_kix.copy_(torch.from_numpy(keyix.astype(np.int32)))
        torch.cuda.synchronize()

    load(batches[0])
    g = xb.VerifyGraph(1, False, count, d_sm.data_ptr(), d_off.data_ptr(), d_len.data_ptr(), d_pk.data_ptr(), keys,
                       d_kix.data_ptr(), d_st.data_ptr())
    for rep in range(3):
        b = batches[rep % 2]
        load(b)
        d_st.fill_(7)
        g.launch(torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert (d_st.cpu().numpy() == b[4]).all(), rep
    g.close()


def test_verify_graphs_concurrent_on_streams(xb):
    """Verify graphs own their scratch, so several of them, each over its
    own batch, replay concurrently on several streams (the pipelined form of
    the benchmark): every replay's statuses equal the blocking call's for its
    batch, including split (1,100-signature) and unsplit batches in flight
    together, each graph replayed twice with nothing in between."""
    import torch

    rng = np.random.default_rng(97)
    keys = 3
    seeds = np.frombuffer(rng.bytes(keys * 96), np.uint8).reshape(keys, 96)
    pks, sks = xb.keypair_batch(1, False, seeds)
    dev = torch.device("cuda", 0)
    d_pk = torch.from_numpy(np.ascontiguousarray(pks[:, 4:])).to(dev)
    items = []
    for count in (1100, 300, 1100, 64):
        keyix = rng.integers(0, keys, count).astype(np.uint32)
        rows = np.array(sks[keyix])
        idx = rng.integers(0, 1023, count)
        for i in range(count):
            rows[i, 4:8] = np.frombuffer(int(idx[i]).to_bytes(4, "big"), np.uint8)
        msgs = [rng.bytes(int(L)) for L in np.exp(rng.uniform(0, np.log(4000), count)).astype(int)]
        _, sms = xb.sign_batch(False, rows, msgs)
        sms = [bytearray(s) for s in sms]
        for i in range(int(rng.integers(0, 4)), count, 4):
            sms[i][int(rng.integers(0, len(sms[i])))] ^= 1
        buf, off, ln = xb.pack([bytes(s) for s in sms], align=16)
        want = xb.sign_open_batch(False, buf, off, ln, pks, keyix)
        d = dict(sm=torch.from_numpy(buf).to(dev), off=torch.from_numpy(off.astype(np.int64)).to(dev),
                 ln=torch.from_numpy(ln.astype(np.int64)).to(dev), kix=torch.from_numpy(keyix.astype(np.int32)).to(dev),
                 st=torch.full((count,), 7, dtype=torch.int32, device=dev), want=want, count=count)
        d["g"] = xb.VerifyGraph(1, False, count, d["sm"].data_ptr(), d["off"].data_ptr(), d["ln"].data_ptr(),
                                d_pk.data_ptr(), keys, d["kix"].data_ptr(), d["st"].data_ptr())
        items.append(d)
    streams = [torch.cuda.Stream() for _ in range(len(items))]
    torch.cuda.synchronize()
    for rep in range(2):
        for d in items:
            d["st"].fill_(7)
        torch.cuda.synchronize()
        for d, s in zip(items, streams):
            d["g"].launch(s.cuda_stream)
            d["g"].launch(s.cuda_stream)
        torch.cuda.synchronize()
        for k, d in enumerate(items):
            assert (d["st"].cpu().numpy() == d["want"]).all(), (rep, k)
    for d in items:
        d["g"].close()


def test_results_do_not_depend_on_launch_shape(xb, golden):
    """Every tunable shape (CTA sizes 32 / 64 / 128, split on or off at any
    H_msg boundary) gives the same accept bitmap and the same keys; the
    autotuner runs, checks its candidates and leaves a valid shape."""
    rng = np.random.default_rng(97)
    keys, count = 3, 1200
    seeds = np.frombuffer(rng.bytes(keys * 96), np.uint8).reshape(keys, 96)
    base = xb.tuning_get(0, 32)
    pks, sks = xb.keypair_batch(1, False, seeds)
    keyix = rng.integers(0, keys, count).astype(np.uint32)
    rows = np.array(sks[keyix])
    idx = rng.integers(0, 1023, count)
    for i in range(count):
        rows[i, 4:8] = np.frombuffer(int(idx[i]).to_bytes(4, "big"), np.uint8)
    msgs = [rng.bytes(int(L)) for L in np.exp(rng.uniform(0, np.log(4000), count)).astype(int)]
    _, sms = xb.sign_batch(False, rows.copy(), msgs)
    sms = [bytearray(s) for s in sms]
    for i in range(0, count, 6):
        sms[i][int(rng.integers(0, len(sms[i])))] ^= 1
    buf, off, ln = xb.pack([bytes(s) for s in sms], align=16)
    want = xb.sign_open_batch(False, buf, off, ln, pks, keyix)
    try:
        for shape in (dict(base, verify_chain_block=32, level_block=32, keygen_chain_block=32),
                      dict(base, verify_chain_block=64, level_block=128, keygen_chain_block=64, split_min=1,
                           short_hmsg_blocks=8),
                      dict(base, split_min=1 << 30)):
            xb.tuning_set(0, 32, shape)
            assert (xb.sign_open_batch(False, buf, off, ln, pks, keyix) == want).all(), shape
            pk2, sk2 = xb.keypair_batch(1, False, seeds)
            assert (pk2 == pks).all() and (sk2 == sks).all(), shape
            _, sms2 = xb.sign_batch(False, rows.copy()[:20], msgs[:20])
            r, _, sm0 = xb.xmss_sign(bytes(rows[0]), msgs[0])
            assert sms2[0] == sm0
        best, report = xb.autotune(1, False, 512)
        assert best["verify_chain_block"] in (32, 64, 128) and len(report["trials"]) >= 10
        assert xb.tuning_get(0, 32) == best
    finally:
        xb.tuning_set(0, 32, base)
