"""BDS ("fast") secret keys: export (xmss_b200_sk_to_bds) must give, byte for
byte, the sk the reference's own fast build (xmss_core_fast.c, compiled from
its sources into oracle/_ref/libxmssref_fast.so) holds after the same number
of signatures, and import must give back the plain key."""
import ctypes as C
import os

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_FAST = os.path.join(ROOT, "oracle", "_ref", "libxmssref_fast.so")


class FastRef:
    """The reference's fast build through ctypes (zero-initialised buffers:
    the fields its keygen leaves unset read as zero, as the export writes
    them)."""

    def __init__(self, xb):
        self.xb = xb
        self.lib = C.CDLL(REF_FAST)
        P = C.POINTER(xb.XmssParams)
        self.lib.xmss_parse_oid.argtypes = self.lib.xmssmt_parse_oid.argtypes = [P, C.c_uint32]
        for f in ("xmss_core_keypair", "xmssmt_core_keypair"):
            getattr(self.lib, f).argtypes = [P, C.c_void_p, C.c_void_p]
        for f in ("xmss_core_sign", "xmssmt_core_sign"):
            getattr(self.lib, f).argtypes = [P, C.c_void_p, C.c_void_p, C.POINTER(C.c_ulonglong), C.c_void_p,
                                             C.c_ulonglong]
        self.lib.ref_randombytes_seed.argtypes = [C.c_uint64]

    def params(self, oid, mt):
        p = self.xb.XmssParams()
        assert (self.lib.xmssmt_parse_oid if mt else self.lib.xmss_parse_oid)(C.byref(p), oid) == 0
        return p

    def keypair(self, p, mt):
        pk, sk = (C.c_uint8 * p.pk_bytes)(), (C.c_uint8 * p.sk_bytes)()
        assert (self.lib.xmssmt_core_keypair if mt else self.lib.xmss_core_keypair)(C.byref(p), pk, sk) == 0
        return bytes(pk), bytes(sk)

    def sign(self, p, mt, sk, m):
        skb = (C.c_uint8 * len(sk)).from_buffer_copy(sk)
        sm = (C.c_uint8 * (p.sig_bytes + len(m)))()
        smlen = C.c_ulonglong()
        mb = (C.c_uint8 * max(1, len(m))).from_buffer_copy(m or b"\0")
        r = (self.lib.xmssmt_core_sign if mt else self.lib.xmss_core_sign)(C.byref(p), skb, sm, C.byref(smlen), mb,
                                                                          len(m))
        return r, bytes(skb), bytes(sm)[:smlen.value]


@pytest.fixture(scope="module")
def fast(xb):
    if not os.path.exists(REF_FAST):
        pytest.skip("reference fast build missing (oracle/Makefile ref)")
    return FastRef(xb)


@pytest.mark.parametrize("name,mt,last,checks", [
    ("XMSS-SHA2_10_256", False, 300, {0, 1, 2, 3, 4, 5, 6, 7, 8, 15, 16, 17, 31, 32, 63, 64, 100, 255, 256, 300}),
    ("XMSSMT-SHA2_20/4_256", True, 200, {0, 1, 2, 3, 30, 31, 32, 33, 63, 64, 65, 100, 127, 128, 129, 200}),
    ("XMSSMT-SHA2_20/2_256", True, 1100, {0, 1, 511, 1022, 1023, 1024, 1025, 1100}),
])
def test_bds_export_matches_reference_fast_build(xb, fast, name, mt, last, checks):
    oid = xb.xmssmt_str_to_oid(name) if mt else xb.xmss_str_to_oid(name)
    pf = fast.params(oid, mt)
    assert pf.sk_bytes == xb.bds_sk_bytes(oid, mt)
    fast.lib.ref_randombytes_seed(0x5EED + oid)
    pk, fsk = fast.keypair(pf, mt)
    oidb = oid.to_bytes(4, "big")
    p = xb.parse_oid(oid, mt)
    sign = xb.xmssmt_sign if mt else xb.xmss_sign
    for k in range(last + 1):
        m = bytes([k & 0xFF]) * (k % 50)
        if k in checks:
            bds = oidb + fsk
            plain = xb.sk_from_bds(mt, bds)
            assert int.from_bytes(plain[4:4 + p.index_bytes], "big") == k
            assert plain[4 + p.index_bytes:] == fsk[p.index_bytes:p.index_bytes + 4 * p.n]
            assert xb.sk_to_bds(mt, plain) == bds, (name, k)
            # the plain path signs index k with the same bytes
            r, _, sm_plain = sign(plain, m)
            r2, fsk, sm = fast.sign(pf, mt, fsk, m)
            assert r == r2 == 0 and sm == sm_plain, (name, k)
        else:
            r, fsk, sm = fast.sign(pf, mt, fsk, m)
            assert r == 0
