"""The serving loop (xmss_b200_server_*) on the GPU: signatures byte-identical
to the reference's (golden fixtures) and the oracle's, every one-time index
issued exactly once under concurrent submitters, each result the same alone
and inside a mixed stream, exhaustion, subtree-cache eviction."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def key_at(sk: bytes, index: int, index_bytes: int) -> bytes:
    """OID-prefixed sk with its index field set to `index`."""
    return sk[:4] + index.to_bytes(index_bytes, "big") + sk[4 + index_bytes:]


def test_serve_config1_byte_exact(xb, golden):
    """Config 1's 16 reference signatures (indices 0..15) come back from the
    server byte for byte, in submission order, and the exported sk equals the
    reference's sk after the 16th signature."""
    g = golden("config1.json")
    p = xb.parse_oid(1)
    with xb.Server() as srv:
        kid = srv.add_key(bytes.fromhex(g["sk"]))
        tags = [srv.submit_sign(kid, bytes.fromhex(m), p.sig_bytes) for m in g["msgs"]]
        res = srv.wait(tags)
        for i, t in enumerate(tags):
            assert res[t]["ret"] == 0 and res[t]["index"] == i
            assert res[t]["sm"].hex() == g["sms"][i], i
        assert srv.export_sk(kid).hex() == g["sk_after"][-1]
        # verify requests of the same signatures, one flipped
        pk = bytes.fromhex(g["pk"])
        sms = [bytes.fromhex(s) for s in g["sms"]]
        bad = bytearray(sms[5])
        bad[100] ^= 0x10
        vt = [srv.submit_verify(s, pk) for s in sms] + [srv.submit_verify(bytes(bad), pk),
                                                        srv.submit_verify(sms[0][:100], pk)]
        vr = srv.wait(vt)
        assert [vr[t]["ret"] for t in vt] == [0] * 16 + [-1, -1]
        st = srv.stats()
        assert st["completed"] == 34 and st["trees_built"] == 1


def test_serve_admission_refuses_what_never_fits(xb, golden):
    """Admission by free device memory: with a reserve larger than any GPU's
    memory no batch fits, so the dispatcher halves each batch down to single
    requests and refuses those with -3 (the deferrals are counted), before
    any one-time index is taken: the key exports unchanged.  The free-memory
    figure comes from the monitor thread; the dispatcher's own query, made
    only when that figure says no, refuses too."""
    g = golden("config1.json")
    p = xb.parse_oid(1)
    sk = bytes.fromhex(g["sk"])
    with xb.Server(mem_reserve_bytes=1 << 60) as srv:
        kid = srv.add_key(sk)
        pk = bytes.fromhex(g["pk"])
        sms = [bytes.fromhex(s) for s in g["sms"][:4]]
        tags = [srv.submit_verify(s, pk) for s in sms] + [srv.submit_sign(kid, bytes.fromhex(m), p.sig_bytes)
                                                          for m in g["msgs"][:3]]
        res = srv.wait(tags)
        assert [res[t]["ret"] for t in tags] == [-3] * len(tags)
        assert srv.stats()["deferred_for_memory"] >= len(tags)
        assert srv.export_sk(kid) == sk
    with xb.Server() as srv:  # the same requests with the default reserve
        kid = srv.add_key(sk)
        tags = [srv.submit_verify(s, pk) for s in sms] + [srv.submit_sign(kid, bytes.fromhex(m), p.sig_bytes)
                                                          for m in g["msgs"][:3]]
        res = srv.wait(tags)
        assert [res[t]["ret"] for t in tags] == [0] * len(tags)
        assert [res[t]["sm"].hex() for t in tags[4:]] == g["sms"][:3]


def test_serve_every_family_mt(xb, golden):
    """The reference's XMSS^MT 20/4 signatures of all seven hash families at
    seeded indices, signed by the server from keys resumed at those indices
    (each signature needs four cached subtrees)."""
    doc = golden("mt_small.json")
    with xb.Server(slots=2) as srv:
        tags, want = [], {}
        for e in doc:
            p = xb.parse_oid(e["oid"], True)
            sk = e["oid"].to_bytes(4, "big") + bytes.fromhex(e["sk"])
            for s in e["sigs"]:
                kid = srv.add_key(key_at(sk, s["idx"], p.index_bytes), mt=True)
                t = srv.submit_sign(kid, bytes.fromhex(s["m"]), p.sig_bytes)
                tags.append(t)
                want[t] = s["sm"]
        res = srv.wait(tags)
        for t in tags:
            assert res[t]["ret"] == 0
            assert res[t]["sm"].hex() == want[t]
        # and verified by the server against the OID-prefixed pk
        vt = {}
        for e in doc:
            pk = e["oid"].to_bytes(4, "big") + bytes.fromhex(e["pk"])
            for s in e["sigs"]:
                vt[srv.submit_verify(bytes.fromhex(s["sm"]), pk, mt=True)] = 0
        vr = srv.wait(list(vt))
        assert all(vr[t]["ret"] == 0 for t in vt)


def test_serve_index_exactly_once(xb, oracle):
    """Four threads submit 1,200 signs over three keys at once: each key's
    completions carry indices 0..n-1 exactly once, the index bytes of each
    signature equal the reported index, every signature verifies, and the
    exported sk resumes after the last one."""
    rng = np.random.default_rng(7)
    p = xb.parse_oid(1)
    keys = []
    for _ in range(3):
        pk, sk = oracle.api_seed_keypair(1, False, rng.bytes(96))
        keys.append((pk, sk))
    with xb.Server(max_batch=128, slots=4) as srv:
        kids = [srv.add_key(sk) for _, sk in keys]
        lock = threading.Lock()
        tags = []

        def submitter(seed):
            r = np.random.default_rng(seed)
            mine = []
            for _ in range(300):
                k = int(r.integers(0, 3))
                m = r.bytes(int(r.integers(1, 600)))
                with lock:  # the binding's tag counter is shared
                    t = srv.submit_sign(kids[k], m, p.sig_bytes)
                mine.append((t, k, m))
            with lock:
                tags.extend(mine)

        ths = [threading.Thread(target=submitter, args=(s,)) for s in range(4)]
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        res = srv.wait([t for t, _, _ in tags])
        per_key = {k: [] for k in range(3)}
        sms, pks = [], []
        for t, k, m in tags:
            d = res[t]
            assert d["ret"] == 0
            assert int.from_bytes(d["sm"][:4], "big") == d["index"]
            assert d["sm"][p.sig_bytes:] == m
            per_key[k].append(d["index"])
            sms.append(d["sm"])
            pks.append(k)
        for k, idx in per_key.items():
            assert sorted(idx) == list(range(len(idx))), k
            exported = srv.export_sk(kids[k])
            assert exported == key_at(keys[k][1], len(idx), p.index_bytes)
    buf, off, ln = xb.pack(sms)
    pkarr = np.stack([np.frombuffer(keys[k][0], np.uint8) for k in range(3)])
    st = xb.sign_open_batch(False, buf, off, ln, pkarr, np.array(pks, np.uint32))
    assert (st == 0).all()


def _run_requests(xb, sk_a, msgs_a, verify_items, extra=None):
    """Runs sign requests on key A plus verify requests, optionally inside
    extra traffic; returns (signatures of A, verify results)."""
    p = xb.parse_oid(1)
    with xb.Server(max_batch=256, slots=3) as srv:
        ka = srv.add_key(sk_a)
        noise = []
        if extra:
            kb = [srv.add_key(sk) for sk in extra["sks"]]
        ta, tv = [], []
        for i, m in enumerate(msgs_a):
            if extra:
                for j, m2 in enumerate(extra["msgs"][i]):
                    noise.append(srv.submit_sign(kb[j % len(kb)], m2, p.sig_bytes))
                for sm, pk in extra["verify"][i]:
                    noise.append(srv.submit_verify(sm, pk))
            ta.append(srv.submit_sign(ka, m, p.sig_bytes))
            sm, pk = verify_items[i]
            tv.append(srv.submit_verify(sm, pk))
        res = srv.wait(ta + tv + noise)
    return [res[t]["sm"] for t in ta], [res[t]["ret"] for t in tv]


def test_serve_alone_equals_mixed(xb, oracle, golden):
    """Each request's result is the same when it is served alone and when it
    is served inside a stream of other keys' signs and verifies (the integer
    path has no tolerance: bytes and codes must be equal)."""
    g = golden("config1.json")
    rng = np.random.default_rng(11)
    pk_a = bytes.fromhex(g["pk"])
    sk_a = bytes.fromhex(g["sk"])
    msgs_a = [rng.bytes(int(rng.integers(0, 3000))) for _ in range(12)]
    sms = [bytes.fromhex(s) for s in g["sms"]]
    verify_items = []
    for i in range(12):
        sm = bytearray(sms[i])
        if i % 3 == 2:
            sm[int(rng.integers(0, len(sm)))] ^= 1 << int(rng.integers(0, 8))
        verify_items.append((bytes(sm), pk_a))
    others = [oracle.api_seed_keypair(1, False, rng.bytes(96)) for _ in range(4)]
    extra = {"sks": [sk for _, sk in others],
             "msgs": [[rng.bytes(int(rng.integers(0, 5000))) for _ in range(6)] for _ in range(12)],
             "verify": [[(sms[int(rng.integers(0, 16))], pk_a) for _ in range(10)] for _ in range(12)]}
    alone = _run_requests(xb, sk_a, msgs_a, verify_items)
    mixed = _run_requests(xb, sk_a, msgs_a, verify_items, extra)
    assert alone == mixed
    assert alone[1] == [0 if i % 3 != 2 else -1 for i in range(12)]
    # and the signatures are the oracle's
    p = oracle.params(1)
    sk = sk_a[4:]
    for i, m in enumerate(msgs_a[:3]):
        r, sk, sm = oracle.sign(p, sk, m)
        assert r == 0 and sm == alone[0][i]


def test_serve_exhaustion(xb, oracle, golden):
    """A key resumed at index 2^h - 2 signs once (the oracle's bytes), then
    every request completes with -2; the exported sk stops at 2^h - 1 and
    the reference's wiped-key signature at 2^h - 1 is never issued."""
    g = golden("config1.json")
    p = xb.parse_oid(1)
    sk = key_at(bytes.fromhex(g["sk"]), 1022, p.index_bytes)
    m = b"last one-time key"
    with xb.Server() as srv:
        kid = srv.add_key(sk)
        tags = [srv.submit_sign(kid, m, p.sig_bytes) for _ in range(3)]
        res = srv.wait(tags)
        assert [res[t]["ret"] for t in tags] == [0, -2, -2]
        assert res[tags[0]]["index"] == 1022
        assert srv.export_sk(kid) == key_at(sk, 1023, p.index_bytes)
    r, _, want = oracle.sign(oracle.params(1), sk[4:], m)
    assert r == 0 and res[tags[0]]["sm"] == want
    assert xb.xmss_sign_open(want, bytes.fromhex(g["pk"])) == (0, m)


def test_serve_eviction_and_warm(xb, oracle):
    """A subtree pool that holds two h=10 subtrees serves five keys in turn
    (every switch evicts one); warm requests prebuild without taking an
    index; all signatures verify and indices stay consecutive per key."""
    rng = np.random.default_rng(3)
    p = xb.parse_oid(1)
    tree_bytes = ((2 << 10) - 1) * 32
    keys = [oracle.api_seed_keypair(1, False, rng.bytes(96)) for _ in range(5)]
    with xb.Server(max_batch=4, slots=1, tree_pool_bytes=2 * ((tree_bytes + 255) // 256 * 256)) as srv:
        kids = [srv.add_key(sk) for _, sk in keys]
        w = srv.wait([srv.submit_warm(kids[0])])
        assert list(w.values())[0]["ret"] == 0
        assert srv.export_sk(kids[0]) == keys[0][1]  # warm takes no index
        order = [k for _ in range(3) for k in range(5)]
        tags = [(srv.submit_sign(kids[k], bytes([k, i]), p.sig_bytes), k) for i, k in enumerate(order)]
        res = srv.wait([t for t, _ in tags])
        st = srv.stats()
        assert st["trees_evicted"] > 0
    seen = {k: [] for k in range(5)}
    for t, k in tags:
        d = res[t]
        assert d["ret"] == 0
        seen[k].append(d["index"])
        assert xb.xmss_sign_open(d["sm"], keys[k][0])[0] == 0
    assert all(v == [0, 1, 2] for v in seen.values())


def test_serve_replay_mixed_params(xb, oracle):
    """A timed trace over five parameter sets (S10, S16 resumed, S512,
    SHAKE K10, XMSS^MT 20/2) through xmss_b200_server_replay: every sign
    verifies under its key and every verify result is the expected one."""
    rng = np.random.default_rng(5)
    names = [("XMSS-SHA2_10_256", False), ("XMSS-SHA2_10_512", False), ("XMSS-SHAKE_10_256", False),
             ("XMSSMT-SHA2_20/2_256", True), ("XMSS-SHA2_16_256", False)]
    keys = []
    for name, mt in names:
        oid = xb.xmssmt_str_to_oid(name) if mt else xb.xmss_str_to_oid(name)
        p = xb.parse_oid(oid, mt)
        if p.full_height == 16:  # h=16 keygen on the GPU (the oracle would take minutes)
            seeds = np.frombuffer(rng.bytes(3 * p.n), np.uint8)[None, :]
            pk, sk = xb.keypair_batch(oid, mt, seeds)
            pk, sk = bytes(pk[0]), bytes(sk[0])
        else:
            pk, sk = oracle.api_seed_keypair(oid, mt, rng.bytes(3 * p.n))
        keys.append((name, mt, p, pk, sk))
    with xb.Server(max_batch=64, slots=4) as srv:
        kids = [srv.add_key(sk, mt) for _, mt, _, _, sk in keys]
        n = 300
        kinds = rng.random(n) < 0.3
        which = rng.integers(0, len(keys), n)
        # verify requests use earlier signatures of the same keys
        pool = {}
        for k, (_, mt, p, pk, _) in enumerate(keys):
            m = rng.bytes(200)
            t = srv.submit_sign(kids[k], m, p.sig_bytes)
            pool[k] = srv.wait([t])[t]["sm"]
        trace = np.zeros(n, xb.TRACE_DTYPE)
        keep = []
        expect = []
        t_us = np.cumsum(rng.exponential(50.0, n))
        for i in range(n):
            k = int(which[i])
            _, mt, p, pk, _ = keys[k]
            trace[i]["t_us"] = t_us[i]
            if kinds[i]:
                m = np.frombuffer(rng.bytes(int(np.exp(rng.uniform(np.log(32), np.log(65536))))), np.uint8).copy()
                out = np.zeros(p.sig_bytes + len(m), np.uint8)
                ln = np.zeros(1, np.uint64)
                keep += [m, out, ln]
                trace[i]["kind"] = 0
                trace[i]["key_id"] = kids[k]
                trace[i]["in_ptr"] = m.ctypes.data
                trace[i]["inlen"] = len(m)
                trace[i]["sm_ptr"] = out.ctypes.data
                trace[i]["smlen_ptr"] = ln.ctypes.data
                expect.append(("sign", k, m, out, ln))
            else:
                sm = bytearray(pool[k])
                bad = bool(rng.random() < 0.2)
                if bad:
                    sm[int(rng.integers(0, p.sig_bytes))] ^= 1
                sm = np.frombuffer(bytes(sm), np.uint8).copy()
                pkb = np.frombuffer(pk, np.uint8).copy()
                keep += [sm, pkb]
                trace[i]["kind"] = 1
                trace[i]["mt"] = int(mt)
                trace[i]["in_ptr"] = sm.ctypes.data
                trace[i]["inlen"] = len(sm)
                trace[i]["pk_ptr"] = pkb.ctypes.data
                expect.append(("verify", k, bad, None, None))
        ret, lat, idx, elapsed = srv.replay(trace)
        assert elapsed > 0 and (lat > 0).all()
    for i, e in enumerate(expect):
        if e[0] == "verify":
            assert ret[i] == (-1 if e[2] else 0), i
        else:
            _, k, m, out, ln = e
            name, mt, p, pk, _ = keys[k]
            assert ret[i] == 0, (i, name)
            sm = bytes(out[:int(ln[0])])
            f = xb.xmssmt_sign_open if mt else xb.xmss_sign_open
            assert f(sm, pk) == (0, bytes(m)), (i, name)
