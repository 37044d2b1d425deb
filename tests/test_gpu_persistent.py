"""xmss_b200_sign_open_device_persistent: the whole verify of a batch as one
persistent launch fed by a device work queue.  Its statuses must be those of
the multi-launch device entry point, which the other tests pin to the
oracle and to the reference (xmss_commons.c:136-215): every hash family,
XMSS and XMSS^MT up to 12 layers, partial groups of 32, corruptions
anywhere in sig || message, too-short signed messages, the last-index
quirk, and the same buffers verified twice (the launch's counters restart)."""
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _signed_batch(xb, name, count, keys=3, max_mlen=3000, seed=None):
    """Signed messages of `name` under `keys` seeded keys; every 5th one
    gets a bit flip and one is cut below sig_bytes.  Returns the packed
    buffers, the public keys, the key index per message and the expected
    statuses."""
    mt = name.startswith("XMSSMT")
    oid = xb.xmssmt_str_to_oid(name) if mt else xb.xmss_str_to_oid(name)
    p = xb.parse_oid(oid, mt)
    rng = np.random.default_rng(zlib.crc32(name.encode()) if seed is None else seed)
    seeds = np.frombuffer(rng.bytes(keys * 3 * p.n), np.uint8).reshape(keys, 3 * p.n)
    pks, sks = xb.keypair_batch(oid, mt, seeds)
    keyix = rng.integers(0, keys, count).astype(np.uint32)
    top = (1 << p.full_height) - 1
    idx = rng.integers(0, min(top, 1 << 62), count)  # below 2^h - 1: every signature valid
    mlen = np.exp(rng.uniform(0, np.log(max_mlen), count)).astype(int) - 1
    msgs = [rng.bytes(int(L)) for L in mlen]
    rows = np.array(sks[keyix])
    ib = p.index_bytes
    for i in range(count):
        rows[i, 4:4 + ib] = np.frombuffer(int(idx[i]).to_bytes(ib, "big"), np.uint8)
    ret, sms = xb.sign_batch(mt, rows, msgs)
    assert (ret == 0).all()
    expect = np.zeros(count, np.int32)
    sms = [bytearray(s) for s in sms]
    for i in range(1, count, 5):
        sms[i][int(rng.integers(0, len(sms[i])))] ^= 1 << int(rng.integers(0, 8))
        expect[i] = -1
    if count > 3:
        sms[3] = sms[3][:p.sig_bytes - 1]
        expect[3] = -1
    buf, off, ln = xb.pack([bytes(s) for s in sms], align=4)
    return oid, mt, buf, off, ln, pks, keyix, expect


def _device_statuses(xb, torch, entry, oid, mt, buf, off, ln, pks, keyix, calls=1):
    dev = torch.device("cuda", 0)
    d_sm = torch.from_numpy(buf).to(dev)
    d_off = torch.from_numpy(off.astype(np.int64)).to(dev)
    d_len = torch.from_numpy(ln.astype(np.int64)).to(dev)
    d_pk = torch.from_numpy(np.ascontiguousarray(pks[:, 4:])).to(dev)
    d_kix = torch.from_numpy(keyix.astype(np.int32)).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    out = []
    for _ in range(calls):
        st = torch.full((len(off),), 7, dtype=torch.int32, device=dev)
        entry(oid, mt, len(off), d_sm.data_ptr(), d_off.data_ptr(), d_len.data_ptr(), d_pk.data_ptr(),
              pks.shape[0], d_kix.data_ptr(), st.data_ptr(), stream)
        torch.cuda.synchronize()
        out.append(st.cpu().numpy())
    return out


@pytest.mark.parametrize("name,count", [
    ("XMSS-SHA2_10_256", 1),
    ("XMSS-SHA2_10_256", 33),
    ("XMSS-SHA2_10_256", 250),
    ("XMSS-SHA2_10_256", 1100),
    ("XMSSMT-SHA2_20/2_256", 1030),
    ("XMSS-SHA2_10_512", 70),
    ("XMSS-SHAKE_10_256", 70),
    ("XMSS-SHAKE_10_512", 40),
    ("XMSS-SHA2_10_192", 70),
    ("XMSS-SHAKE256_10_192", 40),
    ("XMSSMT-SHA2_20/2_256", 100),
    ("XMSSMT-SHA2_20/4_256", 70),
    ("XMSSMT-SHA2_60/12_256", 40),
    ("XMSSMT-SHAKE_20/4_512", 40),
])
def test_persistent_matches_device_entry_point(xb, name, count):
    torch = pytest.importorskip("torch")
    oid, mt, buf, off, ln, pks, keyix, expect = _signed_batch(xb, name, count)
    (want,) = _device_statuses(xb, torch, xb.sign_open_device, oid, mt, buf, off, ln, pks, keyix)
    assert (want == expect).all()
    got = _device_statuses(xb, torch, xb.sign_open_device_persistent, oid, mt, buf, off, ln, pks, keyix, calls=2)
    for g in got:
        assert (g == want).all(), (name, np.nonzero(g != want)[0][:10])


def test_persistent_large_batch_last_index(xb):
    """1,100 XMSS-SHA2_10_256 signatures with messages up to 4 KB (groups of
    32 whose H_msg lengths differ), some at the wiped last index 1023."""
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(77)
    count, keys = 1100, 5
    seeds = np.frombuffer(rng.bytes(keys * 96), np.uint8).reshape(keys, 96)
    pks, sks = xb.keypair_batch(1, False, seeds)
    keyix = rng.integers(0, keys, count).astype(np.uint32)
    idx = rng.integers(0, 1024, count)
    idx[::97] = 1023
    mlen = np.exp(rng.uniform(np.log(32), np.log(4096), count)).astype(int)
    msgs = [rng.bytes(int(L)) for L in mlen]
    rows = np.array(sks[keyix])
    for i in range(count):
        rows[i, 4:8] = np.frombuffer(int(idx[i]).to_bytes(4, "big"), np.uint8)
    ret, sms = xb.sign_batch(False, rows, msgs)
    assert (ret == 0).all()
    expect = np.where(idx == 1023, -1, 0).astype(np.int32)
    sms = [bytearray(s) for s in sms]
    for i in range(4, count, 10):
        sms[i][int(rng.integers(0, len(sms[i])))] ^= 1 << int(rng.integers(0, 8))
        expect[i] = -1
    buf, off, ln = xb.pack([bytes(s) for s in sms], align=8)
    got = _device_statuses(xb, torch, xb.sign_open_device_persistent, 1, False, buf, off, ln, pks, keyix, calls=2)
    for g in got:
        assert (g == expect).all()


def test_persistent_multi_mixed_sets(xb):
    """xmss_b200_sign_open_device_persistent_multi: batches of five parameter
    sets (four SHA-256 n = 32 sets in one persistent launch, XMSS-SHAKE_10_256
    in a second launch on a forked stream) give every batch the statuses its
    own multi-launch verify gives, twice in a row (counters restart), and a
    set of nine SHA-256 batches (more than one launch of a family) as well."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    names = ["XMSS-SHA2_10_256", "XMSSMT-SHA2_20/2_256", "XMSSMT-SHA2_20/4_256", "XMSSMT-SHA2_40/4_256",
             "XMSS-SHAKE_10_256"]
    batches = [_signed_batch(xb, nm, c, seed=100 + i) for i, (nm, c) in enumerate(zip(names, (90, 70, 40, 33, 50)))]
    keep, jobs, want = [], [], []
    for oid, mt, buf, off, ln, pks, keyix, expect in batches:
        d = dict(d_sm=torch.from_numpy(buf).to(dev), d_sm_off=torch.from_numpy(off.astype(np.int64)).to(dev),
                 d_smlen=torch.from_numpy(ln.astype(np.int64)).to(dev),
                 d_pk=torch.from_numpy(np.ascontiguousarray(pks[:, 4:])).to(dev),
                 d_pk_index=torch.from_numpy(keyix.astype(np.int32)).to(dev),
                 d_status=torch.full((len(off),), 7, dtype=torch.int32, device=dev))
        keep.append(d)
        jobs.append(dict(oid=oid, mt=int(mt), count=len(off), npk=len(pks),
                         **{k: v.data_ptr() for k, v in d.items()}))
        ref = _device_statuses(xb, torch, xb.sign_open_device, oid, mt, buf, off, ln, pks, keyix)[0]
        assert (ref == expect).all()
        want.append(ref)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for _ in range(2):
        for d in keep:
            d["d_status"].fill_(7)
        xb.sign_open_device_persistent_multi(jobs, stream)
        torch.cuda.synchronize()
        for d, w, nm in zip(keep, want, names):
            assert (d["d_status"].cpu().numpy() == w).all(), nm
    # nine batches of one family (two launches of it), each with its own statuses
    st9 = [torch.full((jobs[i % 4]["count"],), 7, dtype=torch.int32, device=dev) for i in range(9)]
    jobs9 = [dict(jobs[i % 4], d_status=st9[i].data_ptr()) for i in range(9)]
    xb.sign_open_device_persistent_multi(jobs9, stream)
    torch.cuda.synchronize()
    for i in range(9):
        assert (st9[i].cpu().numpy() == want[i % 4]).all(), (i, names[i % 4])
