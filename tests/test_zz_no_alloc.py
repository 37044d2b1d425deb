"""xmss_b200_sign_open_device_noalloc: the verify entry point for callers
that cannot allocate device memory while they verify (tight latency paths,
fixed device-memory budgets).  It must give exactly the statuses of the
regular device entry point, call after call, from its fixed scratch array.

This file is collected last so that a failure here cannot stop the rest of
a run that stops at the first failure."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(xb, count=96, keys=3, seed=31):
    """Signed messages (some corrupted, one at the exhausting last index)."""
    rng = np.random.default_rng(seed)
    p = xb.parse_oid(1)
    seeds = np.frombuffer(rng.bytes(keys * 96), np.uint8).reshape(keys, 96)
    pks, sks = xb.keypair_batch(1, False, seeds)
    keyix = rng.integers(0, keys, count).astype(np.uint32)
    idx = rng.integers(0, 1024, count)
    idx[5] = 1023
    mlen = np.exp(rng.uniform(np.log(1), np.log(3000), count)).astype(int)
    msgs = [rng.bytes(int(L)) for L in mlen]
    rows = np.array(sks[keyix])
    for i in range(count):
        rows[i, 4:8] = np.frombuffer(int(idx[i]).to_bytes(4, "big"), np.uint8)
    ret, sms = xb.sign_batch(False, rows, msgs)
    assert (ret == 0).all()
    sms = [bytearray(s) for s in sms]
    for i in range(0, count, 7):
        sms[i][int(rng.integers(0, len(sms[i])))] ^= 4
    buf, off, ln = xb.pack([bytes(s) for s in sms], align=4)
    return buf, off, ln, pks, keyix


def test_noalloc_matches_device_entry_point_twice(xb):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    buf, off, ln, pks, keyix = _batch(xb)
    count, npk = len(off), pks.shape[0]
    d_sm = torch.from_numpy(buf).to(dev)
    d_off = torch.from_numpy(off.astype(np.int64)).to(dev)
    d_len = torch.from_numpy(ln.astype(np.int64)).to(dev)
    d_pk = torch.from_numpy(np.ascontiguousarray(pks[:, 4:])).to(dev)
    d_kix = torch.from_numpy(keyix.astype(np.int32)).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    ptrs = (d_sm.data_ptr(), d_off.data_ptr(), d_len.data_ptr(), d_pk.data_ptr(), npk, d_kix.data_ptr())

    ref = torch.full((count,), 7, dtype=torch.int32, device=dev)
    xb.sign_open_device(1, False, count, *ptrs, ref.data_ptr(), stream)
    torch.cuda.synchronize()
    want = ref.cpu().numpy()
    assert (want == -1).sum() >= count // 7 and (want == 0).sum() > count // 2
    # the host entry point agrees with the device one
    assert (xb.sign_open_batch(False, buf, off, ln, pks, keyix) == want).all()

    for call in range(2):
        got = torch.full((count,), 7, dtype=torch.int32, device=dev)
        r = xb.sign_open_device_noalloc(1, False, count, *ptrs, got.data_ptr(), stream)
        torch.cuda.synchronize()
        assert r == 0, xb.last_error()
        assert (got.cpu().numpy() == want).all(), f"call {call}"


def test_noalloc_xmssmt_batch_matches_oracle_without_allocating(xb, oracle):
    """An XMSS^MT batch (four layers, so the per-layer bucket counters of
    layers 1..3 in the fixed array are used too): statuses equal the
    oracle's, on two calls in a row, and the second call changes the free
    device memory by nothing."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    oid, mt, count, keys = 0x02, True, 64, 2  # XMSSMT-SHA2_20/4_256
    rng = np.random.default_rng(47)
    p, po = xb.parse_oid(oid, mt), oracle.params(oid, mt)
    seeds = np.frombuffer(rng.bytes(keys * 3 * p.n), np.uint8).reshape(keys, -1)
    pks, sks = xb.keypair_batch(oid, mt, seeds)
    keyix = rng.integers(0, keys, count).astype(np.uint32)
    idx = rng.integers(0, (1 << p.full_height) - 1, count)
    idx[7] = (1 << p.full_height) - 1  # the last index signs with a wiped key: must reject
    msgs = [rng.bytes(int(L)) for L in np.exp(rng.uniform(np.log(8), np.log(3000), count)).astype(int)]
    rows = np.array(sks[keyix])
    for i in range(count):
        rows[i, 4:4 + p.index_bytes] = np.frombuffer(int(idx[i]).to_bytes(p.index_bytes, "big"), np.uint8)
    ret, sms = xb.sign_batch(mt, rows, msgs)
    assert (ret == 0).all()
    sms = [bytearray(s) for s in sms]
    for i in range(0, count, 5):
        sms[i][int(rng.integers(0, len(sms[i])))] ^= 1 << int(rng.integers(0, 8))
    sms = [bytes(s) for s in sms]
    want = np.array([oracle.sign_open(po, sms[i], pks[keyix[i], 4:].tobytes())[0] for i in range(count)], np.int32)
    assert (want == -1).sum() >= count // 5 and (want == 0).sum() > count // 2
    buf, off, ln = xb.pack(sms, align=4)
    d_sm = torch.from_numpy(buf).to(dev)
    d_off = torch.from_numpy(off.astype(np.int64)).to(dev)
    d_len = torch.from_numpy(ln.astype(np.int64)).to(dev)
    d_pk = torch.from_numpy(np.ascontiguousarray(pks[:, 4:])).to(dev)
    d_kix = torch.from_numpy(keyix.astype(np.int32)).to(dev)
    outs = [torch.full((count,), 7, dtype=torch.int32, device=dev) for _ in range(2)]
    stream = torch.cuda.current_stream(dev).cuda_stream
    free = []
    for call in range(2):
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info(dev)[0])
        r = xb.sign_open_device_noalloc(oid, mt, count, d_sm.data_ptr(), d_off.data_ptr(), d_len.data_ptr(),
                                        d_pk.data_ptr(), keys, d_kix.data_ptr(), outs[call].data_ptr(), stream)
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info(dev)[0])
        assert r == 0, xb.last_error()
        assert (outs[call].cpu().numpy() == want).all(), f"call {call}"
    assert free[3] == free[2], "the second call changed the free device memory"


def test_noalloc_rejects_a_batch_beyond_its_array(xb):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    count = 2000  # about 22 MB of scratch for XMSS-SHA2_10_256 > 8 MiB
    # inputs sized for the whole batch (empty signed messages), so nothing
    # could be read out of bounds even if the call went ahead
    sm = torch.zeros(4096, dtype=torch.uint8, device=dev)
    off = torch.zeros(count, dtype=torch.int64, device=dev)
    ln = torch.zeros(count, dtype=torch.int64, device=dev)
    pk = torch.zeros(64, dtype=torch.uint8, device=dev)
    kix = torch.zeros(count, dtype=torch.int32, device=dev)
    st = torch.zeros(count, dtype=torch.int32, device=dev)
    r = xb.sign_open_device_noalloc(1, False, count, sm.data_ptr(), off.data_ptr(), ln.data_ptr(), pk.data_ptr(), 1,
                                    kix.data_ptr(), st.data_ptr(), 0)
    assert r == -1
    assert "scratch" in xb.last_error()
