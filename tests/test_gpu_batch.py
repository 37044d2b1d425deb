"""Mixed batches (xmss_b200_batch_*): keygen, sign and verify groups of
several parameter sets (XMSS-SHA2_10_256, XMSSMT-SHA2_20/4_256 and
XMSS-SHAKE_10_256: two hash families, XMSS and XMSS^MT) captured in ONE CUDA
graph and run by a single launch.  Every key, signature, advanced secret key,
return code and verify status equals the oracle's (xmss_core.c:134-161
keygen, :183-273 sign, xmss_commons.c:120-215 verify), including the
reference's index bookkeeping at the end of a key (index 2^h - 1 signs with a
wiped key, later indices return -2).
"""
import os
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SETS = [("XMSS-SHA2_10_256", False), ("XMSSMT-SHA2_20/4_256", True), ("XMSS-SHAKE_10_256", False)]


def _oid(xb, name, mt):
    return xb.xmssmt_str_to_oid(name) if mt else xb.xmss_str_to_oid(name)


def _oracle_trees(oracle, po, sk, idx, cache):
    ib, n, th = po.index_bytes, po.n, po.tree_height
    out = []
    for layer in range(po.d):
        tree = idx >> (th * (layer + 1)) if th * (layer + 1) < 64 else 0
        key = (sk[ib:ib + n], sk[ib + 3 * n:ib + 4 * n], layer, tree)
        if key not in cache:
            cache[key] = oracle.tree_nodes(po, key[0], key[1], layer, tree, os.cpu_count() or 1)
        out.append(cache[key])
    return b"".join(out)


def _dev(torch, a):
    return torch.from_numpy(np.array(a, copy=True)).cuda()


def _keygen_expect(oracle, po, seed):
    """pk (root || PUB_SEED) and sk (idx 0 || SK_SEED || SK_PRF || root ||
    PUB_SEED) of xmssmt_core_seed_keypair, root from the oracle's top tree."""
    n = po.n
    root = oracle.tree_nodes(po, seed[:n], seed[2 * n:], po.d - 1, 0, os.cpu_count() or 1)[-n:]
    return root + seed[2 * n:], bytes(po.index_bytes) + seed[:2 * n] + root + seed[2 * n:]


@pytest.mark.parametrize("persistent", [False, True])
def test_mixed_batch_one_graph_matches_oracle(xb, oracle, persistent):
    """persistent: the same batch as one persistent launch per hash family
    (xmss_b200_batch_create_persistent: keygen, sign and verify tasks of
    every set of the family in one device work queue)."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(zlib.crc32(b"mixed batch"))
    groups, checks, keep = [], [], []
    for si, (name, mt) in enumerate(SETS):
        oid = _oid(xb, name, mt)
        p, po = xb.parse_oid(oid, mt), oracle.params(oid, mt)
        n = p.n
        # keygen group: fresh seeds
        kseeds = np.frombuffer(rng.bytes(3 * 3 * n), np.uint8).reshape(3, 3 * n)
        d_seeds, d_pk = _dev(torch, kseeds), torch.zeros((3, 2 * n), dtype=torch.uint8, device="cuda")
        d_sk = torch.zeros((3, p.sk_bytes), dtype=torch.uint8, device="cuda")
        keep += [d_seeds, d_pk, d_sk]
        groups.append(dict(kind=xb.KEYGEN, oid=oid, mt=int(mt), count=3, d_seeds=d_seeds.data_ptr(),
                           d_pk=d_pk.data_ptr(), d_sk=d_sk.data_ptr()))
        checks.append(("keygen", po, kseeds, d_pk, d_sk))
        # keys the sign and verify groups use (host keygen of this library)
        seeds = np.frombuffer(rng.bytes(2 * 3 * n), np.uint8).reshape(2, 3 * n)
        pks, sks = xb.keypair_batch(oid, mt, seeds)
        # sign group: random indices, messages 0..3000 B, and for the first
        # set the last index (wiped key) and one past it (-2)
        count = 12
        keyix = rng.integers(0, 2, count)
        last = (1 << p.full_height) - 1
        idx = [int(x) for x in rng.integers(0, last, count)]
        if si == 0:
            idx[3], idx[7] = last, last + 1
        rows = np.array(sks[keyix])
        for i in range(count):
            rows[i, 4:4 + p.index_bytes] = np.frombuffer(idx[i].to_bytes(p.index_bytes, "big"), np.uint8)
        before = rows.copy()
        msgs = [rng.bytes(int(L)) for L in rng.integers(0, 3000, count)]
        off = np.zeros(count, np.uint64)
        pos = 0
        for i, m in enumerate(msgs):
            off[i] = pos
            pos += (p.sig_bytes + len(m) + 15) & ~15
        smbuf = np.zeros(pos, np.uint8)
        for i, m in enumerate(msgs):
            smbuf[int(off[i]) + p.sig_bytes:int(off[i]) + p.sig_bytes + len(m)] = np.frombuffer(m, np.uint8)
        d_sm, d_off = _dev(torch, smbuf), _dev(torch, off.astype(np.int64))
        d_len = _dev(torch, np.array([len(m) for m in msgs], np.int64))
        keep += [d_sm, d_off, d_len]
        groups.append(dict(kind=xb.SIGN, oid=oid, mt=int(mt), count=count, sk=rows, d_sm=d_sm.data_ptr(),
                           d_sm_off=d_off.data_ptr(), d_len=d_len.data_ptr()))
        checks.append(("sign", po, before, rows, msgs, off, d_sm, len(groups) - 1))
        # verify group: signatures from the host batch sign, 1 in 4 corrupted
        vcount = 16
        vkey = rng.integers(0, 2, vcount).astype(np.uint32)
        vrows = np.array(sks[vkey])
        for i in range(vcount):
            vrows[i, 4:4 + p.index_bytes] = np.frombuffer(
                int(rng.integers(0, last)).to_bytes(p.index_bytes, "big"), np.uint8)
        vmsgs = [rng.bytes(int(L)) for L in rng.integers(1, 2000, vcount)]
        ret, sms = xb.sign_batch(mt, vrows, vmsgs)
        assert (np.asarray(ret) == 0).all()
        sms = [bytearray(s) for s in sms]
        for i in range(0, vcount, 4):
            sms[i][int(rng.integers(0, len(sms[i])))] ^= 1 << int(rng.integers(0, 8))
        sms = [bytes(s) for s in sms]
        buf, voff, vlen = xb.pack(sms, align=16)
        d_vsm, d_voff, d_vlen = _dev(torch, buf), _dev(torch, voff.astype(np.int64)), _dev(torch, vlen.astype(np.int64))
        d_vpk = _dev(torch, np.ascontiguousarray(pks[:, 4:]))
        d_vix = _dev(torch, vkey.astype(np.int32))
        d_st = torch.full((vcount,), 99, dtype=torch.int32, device="cuda")
        keep += [d_vsm, d_voff, d_vlen, d_vpk, d_vix, d_st]
        groups.append(dict(kind=xb.VERIFY, oid=oid, mt=int(mt), count=vcount, d_sm=d_vsm.data_ptr(),
                           d_sm_off=d_voff.data_ptr(), d_len=d_vlen.data_ptr(), d_pk=d_vpk.data_ptr(), npk=2,
                           d_pk_index=d_vix.data_ptr(), d_status=d_st.data_ptr()))
        want = [oracle.sign_open(po, s, bytes(pks[k, 4:]))[0] for s, k in zip(sms, vkey)]
        checks.append(("verify", po, want, d_st))
    torch.cuda.synchronize()
    b = xb.Batch(groups, persistent=persistent)
    # create signed nothing into the caller's buffers
    for c in checks:
        if c[0] == "sign":
            sm = c[6].cpu().numpy()
            for i in range(len(c[4])):
                assert not sm[int(c[5][i]):int(c[5][i]) + c[1].sig_bytes].any()
    stream = torch.cuda.Stream()
    assert b.launch(stream.cuda_stream) == 0
    torch.cuda.synchronize()
    for c in checks:
        if c[0] == "keygen":
            _, po, seeds, d_pk, d_sk = c
            got_pk, got_sk = d_pk.cpu().numpy(), d_sk.cpu().numpy()
            for k in range(len(seeds)):
                pk, sk = _keygen_expect(oracle, po, seeds[k].tobytes())
                assert got_pk[k].tobytes() == pk and got_sk[k].tobytes() == sk, (po.d, k)
        elif c[0] == "sign":
            _, po, before, rows, msgs, off, d_sm, gi = c
            sm = d_sm.cpu().numpy()
            cache = {}
            for i, m in enumerate(msgs):
                sk0 = before[i, 4:].tobytes()
                i0 = int.from_bytes(sk0[:po.index_bytes], "big")
                trees = _oracle_trees(oracle, po, sk0, i0, cache) if i0 < (1 << po.full_height) - 1 else None
                r, sk1, want = oracle.sign(po, sk0, m, trees=trees)
                assert b.ret[gi][i] == r, (po.d, i)
                assert rows[i, 4:].tobytes() == sk1, (po.d, i)
                if r == 0:
                    o = int(off[i])
                    assert sm[o:o + len(want)].tobytes() == want, (po.d, i, i0)
        else:
            _, po, want, d_st = c
            assert d_st.cpu().numpy().tolist() == want, po.d
    # the signing indices are used: a second launch runs nothing
    assert b.launch(stream.cuda_stream) == -2
    b.close()


@pytest.mark.parametrize("persistent", [False, True])
def test_keygen_verify_batch_relaunches(xb, oracle, persistent):
    """A batch without sign groups replays: refilled buffers give new results
    at each launch (keygen from new seeds, verify statuses rewritten)."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(7)
    oid_mt = xb.xmssmt_str_to_oid("XMSSMT-SHA2_20/4_256")
    p_mt, po_mt = xb.parse_oid(oid_mt, True), oracle.params(oid_mt, True)
    n = p_mt.n
    d_seeds = torch.zeros((4, 3 * n), dtype=torch.uint8, device="cuda")
    d_pk = torch.zeros((4, 2 * n), dtype=torch.uint8, device="cuda")
    d_sk = torch.zeros((4, p_mt.sk_bytes), dtype=torch.uint8, device="cuda")
    # verify group: XMSS-SHA2_10_256 signatures, valid
    p = xb.parse_oid(1)
    pks, sks = xb.keypair_batch(1, False, np.frombuffer(rng.bytes(96), np.uint8).reshape(1, 96))
    rows = np.repeat(sks, 8, axis=0)
    ret, sms = xb.sign_batch(False, rows, [rng.bytes(100 + i) for i in range(8)])
    buf, off, ln = xb.pack(sms, align=16)
    d_sm = _dev(torch, buf)
    d_off, d_len = _dev(torch, off.astype(np.int64)), _dev(torch, ln.astype(np.int64))
    d_vpk, d_ix = _dev(torch, np.ascontiguousarray(pks[:, 4:])), torch.zeros(8, dtype=torch.int32, device="cuda")
    d_st = torch.full((8,), 99, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    b = xb.Batch([dict(kind=xb.KEYGEN, oid=oid_mt, mt=1, count=4, d_seeds=d_seeds.data_ptr(), d_pk=d_pk.data_ptr(),
                       d_sk=d_sk.data_ptr()),
                  dict(kind=xb.VERIFY, oid=1, mt=0, count=8, d_sm=d_sm.data_ptr(), d_sm_off=d_off.data_ptr(),
                       d_len=d_len.data_ptr(), d_pk=d_vpk.data_ptr(), npk=1, d_pk_index=d_ix.data_ptr(),
                       d_status=d_st.data_ptr())], persistent=persistent)
    for rep in range(2):
        seeds = np.frombuffer(rng.bytes(4 * 3 * n), np.uint8).reshape(4, 3 * n)
        d_seeds.copy_(torch.from_numpy(seeds.copy()))
        d_st.fill_(99)
        flip = rep == 1  # the second launch sees signature 5 corrupted
        if flip:
            d_sm[int(off[5]) + 40] ^= 1
        torch.cuda.synchronize()
        assert b.launch(0) == 0
        torch.cuda.synchronize()
        for k in range(4):
            pk, sk = _keygen_expect(oracle, po_mt, seeds[k].tobytes())
            assert d_pk[k].cpu().numpy().tobytes() == pk and d_sk[k].cpu().numpy().tobytes() == sk, (rep, k)
        want = [0] * 8
        if flip:
            want[5] = -1
        assert d_st.cpu().numpy().tolist() == want, rep
    b.close()
