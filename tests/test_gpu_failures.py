"""Failure paths of the device entry points, made without a GPU fault:

* a signature whose key index lies outside the caller's key table is
  rejected (-1) on the device by every device-pointer verify (multi-launch,
  persistent, CUDA graph, allocation-free), and nothing of it is read; the
  host forms reject such a batch before any launch (-1);
* a persistent launch whose dependency waits are bounded below what a long
  H_msg takes ends with -3 in every status (the waits run out, the launch
  returns, the context stays usable), and with the default bound the same
  batch verifies.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(xb, count, keys=3, seed=11, long_len=0):
    rng = np.random.default_rng(seed)
    seeds = np.frombuffer(rng.bytes(keys * 96), np.uint8).reshape(keys, 96)
    pks, sks = xb.keypair_batch(1, False, seeds)
    keyix = rng.integers(0, keys, count).astype(np.uint32)
    idx = rng.integers(0, 1023, count)
    msgs = [rng.bytes(int(L)) for L in np.exp(rng.uniform(np.log(32), np.log(2000), count)).astype(int)]
    if long_len:
        msgs[0] = rng.bytes(long_len)
    rows = np.array(sks[keyix])
    for i in range(count):
        rows[i, 4:8] = np.frombuffer(int(idx[i]).to_bytes(4, "big"), np.uint8)
    ret, sms = xb.sign_batch(False, rows, msgs)
    assert (ret == 0).all()
    buf, off, ln = xb.pack(sms, align=16)
    return buf, off, ln, pks, keyix


def _device(torch, buf, off, ln, pks, keyix):
    dev = torch.device("cuda", 0)
    return dict(sm=torch.from_numpy(buf).to(dev), off=torch.from_numpy(off.astype(np.int64)).to(dev),
                len=torch.from_numpy(ln.astype(np.int64)).to(dev),
                pk=torch.from_numpy(np.ascontiguousarray(pks[:, 4:])).to(dev),
                kix=torch.from_numpy(keyix.astype(np.int64).astype(np.uint32).view(np.int32)).to(dev),
                count=len(off), npk=pks.shape[0])


def _run(xb, torch, entry, d):
    st = torch.full((d["count"],), 7, dtype=torch.int32, device=d["sm"].device)
    stream = torch.cuda.current_stream(d["sm"].device).cuda_stream
    r = entry(1, False, d["count"], d["sm"].data_ptr(), d["off"].data_ptr(), d["len"].data_ptr(),
              d["pk"].data_ptr(), d["npk"], d["kix"].data_ptr(), st.data_ptr(), stream)
    torch.cuda.synchronize()
    assert r in (None, 0), xb.last_error()
    return st.cpu().numpy()


def _graph(xb, torch, d):
    st = torch.full((d["count"],), 7, dtype=torch.int32, device=d["sm"].device)
    g = xb.VerifyGraph(1, False, d["count"], d["sm"].data_ptr(), d["off"].data_ptr(), d["len"].data_ptr(),
                       d["pk"].data_ptr(), d["npk"], d["kix"].data_ptr(), st.data_ptr())
    st.fill_(7)
    g.launch(torch.cuda.current_stream(d["sm"].device).cuda_stream)
    torch.cuda.synchronize()
    g.close()
    return st.cpu().numpy()


@pytest.mark.parametrize("count", [40, 1500])  # one sequence, and the two-group split of large batches
def test_key_index_out_of_range_rejected_on_device(xb, count):
    torch = pytest.importorskip("torch")
    buf, off, ln, pks, keyix = _batch(xb, count)
    good = _device(torch, buf, off, ln, pks, keyix)
    want = _run(xb, torch, xb.sign_open_device, good)
    assert (want == 0).all()
    bad_ix = keyix.copy()
    bad = {2: pks.shape[0], 5: 0xFFFFFFFF, count - 1: pks.shape[0] + 1000}
    for i, v in bad.items():
        bad_ix[i] = v
    d = _device(torch, buf, off, ln, pks, bad_ix)
    expect = want.copy()
    for i in bad:
        expect[i] = -1
    entries = {"device": lambda: _run(xb, torch, xb.sign_open_device, d),
               "persistent": lambda: _run(xb, torch, xb.sign_open_device_persistent, d),
               "graph": lambda: _graph(xb, torch, d)}
    if count <= 500:  # the allocation-free form's fixed scratch holds ~760 of these
        entries["noalloc"] = lambda: _run(xb, torch, xb.sign_open_device_noalloc, d)
    for name, fn in entries.items():
        got = fn()
        assert (got == expect).all(), (name, np.nonzero(got != expect)[0][:10])
    # the host form refuses the batch before launching anything
    with pytest.raises(ValueError):
        xb.sign_open_batch(False, buf, off, ln, pks, bad_ix)


def test_persistent_wait_bound_runs_out(xb):
    torch = pytest.importorskip("torch")
    # one 4 MB message: its H_msg is ~65,000 dependent compressions (about
    # 0.1 s), far longer than the 20 us bound; its group's chain tasks wait
    # for it and run out, so the launch fails as a whole
    buf, off, ln, pks, keyix = _batch(xb, 32, long_len=4 << 20)
    d = _device(torch, buf, off, ln, pks, keyix)
    try:
        xb.set_wait_bound(20_000)
        got = _run(xb, torch, xb.sign_open_device_persistent, d)
        assert (got == -3).all(), got
    finally:
        xb.set_wait_bound(0)
    # default bound: the same launch completes and every signature verifies
    assert (_run(xb, torch, xb.sign_open_device_persistent, d) == 0).all()
    assert (_run(xb, torch, xb.sign_open_device, d) == 0).all()
