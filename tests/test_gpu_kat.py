"""h = 20 known-answer keys: the zero-seed public keys embedded in the
reference's GPU key headers (cuxmss/gpu/*_key.h), for XMSS h=20 and XMSS^MT
40/2 and 60/3 (tree height 20) over SHA-256 n=32/24 and SHAKE256 n=32/24.
Each is a full 2^20-leaf tree build on the GPU."""
import pytest

pytestmark = pytest.mark.gpu


def test_h20_zero_seed_public_keys(xb, golden):
    for k in golden("kat_h20.json"):
        p = xb.parse_oid(k["oid"], k["mt"])
        assert p.tree_height == 20
        r, pk, _ = xb.xmssmt_core_seed_keypair(p, bytes(3 * p.n))
        assert r == 0
        assert pk.hex() == k["pk"], (k["source"], k["condition"])
