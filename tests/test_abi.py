"""The C-ABI library on the CPU: it loads, exports every function that
include/*.h declares, and its host-side parameter tables match the oracle's
restatement of params.c for all 77 OIDs.  No GPU compute is called."""
import ctypes as C

import pytest


def test_exports_every_declared_function(xb):
    declared = xb.header_functions()
    assert len(declared) >= 30
    missing = [f for f in declared if not hasattr(xb.lib, f)]
    assert not missing, missing


@pytest.mark.parametrize("mt,count", [(False, 21), (True, 56)])
def test_params_tables_match_oracle(xb, oracle, mt, count):
    for oid in range(1, count + 1):
        assert xb.parse_oid(oid, mt).as_dict() == oracle.params(oid, mt).as_dict(), oid
    for bad in (0, count + 1, 0xFFFFFFFF):
        with pytest.raises(ValueError):
            xb.parse_oid(bad, mt)


def test_names_round_trip(xb, oracle):
    names = ["XMSS-SHA2_10_256", "XMSS-SHAKE_10_256", "XMSS-SHA2_10_512", "XMSS-SHAKE256_20_192",
             "XMSSMT-SHA2_20/2_256", "XMSSMT-SHA2_40/4_256", "XMSSMT-SHAKE256_60/12_192", "XMSSMT-SHAKE_40/8_512"]
    for n in names:
        oid, mt = oracle.str_to_oid(n)
        assert (xb.xmssmt_str_to_oid(n) if mt else xb.xmss_str_to_oid(n)) == oid
    with pytest.raises(ValueError):
        xb.xmss_str_to_oid("XMSS-SHA2_12_256")


def test_initialize_params_rejects_bad_w(xb):
    p = xb.parse_oid(1)
    p.wots_w = 8
    assert xb.lib.xmss_xmssmt_initialize_params(C.byref(p)) == -1
    p.wots_w = 16
    assert xb.lib.xmss_xmssmt_initialize_params(C.byref(p)) == 0
    assert xb.lib.xmss_xmssmt_core_sk_bytes(C.byref(p)) == 132


def test_every_family_supported(xb):
    for func, n in ((0, 24), (0, 32), (0, 64), (1, 32), (2, 24), (2, 32), (2, 64)):
        assert xb.lib.xmss_b200_supported(func, n) == 1
    assert xb.lib.xmss_b200_supported(1, 64) == 0


def test_unknown_oid_rejected_before_gpu(xb):
    """OID parsing happens on the host: unknown OIDs return -1 like xmss.c."""
    r, _, _ = xb.xmss_keypair(0x99)
    assert r == -1


def test_binding_argtypes_match_headers(xb):
    """Every binding that sets argtypes passes as many arguments as the
    header declares (a miscount only shows when the GPU call is made)."""
    import os
    import re

    decls = {}
    for f in sorted(os.listdir(xb.INCLUDE_DIR)):
        if f.endswith(".h"):
            text = re.sub(r"/\*.*?\*/", "", open(os.path.join(xb.INCLUDE_DIR, f)).read(), flags=re.S)
            for name, args in re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\(([^;{()]*(?:\([^()]*\)[^;{()]*)*)\)\s*;",
                                         text):
                args = re.sub(r"\([^()]*\)", "P", args).strip()  # function-pointer groups
                decls[name] = 0 if args in ("", "void") else args.count(",") + 1
    checked = 0
    for name, nargs in decls.items():
        fn = getattr(xb.lib, name, None)
        if fn is not None and fn.argtypes is not None:
            assert len(fn.argtypes) == nargs, (name, len(fn.argtypes), nargs)
            checked += 1
    assert checked >= 25


def test_tuning_table_without_gpu(xb):
    """Launch shapes are host state: readable and settable without a GPU,
    validated (CTA sizes 32, 64, 128), one entry per hash family."""
    for f, n in xb.FAMILIES:
        t = xb.tuning_get(f, n)
        assert t["verify_chain_block"] in (32, 64, 128) and t["split_min"] >= 1
    old = xb.tuning_get(0, 32)
    try:
        xb.tuning_set(0, 32, dict(old, level_block=64))
        assert xb.tuning_get(0, 32)["level_block"] == 64
        assert xb.tuning_get(0, 24)["level_block"] == xb.tuning_get(0, 24)["level_block"]
        for bad in (dict(old, verify_chain_block=256), dict(old, level_block=100), dict(old, split_min=0)):
            with pytest.raises(ValueError):
                xb.tuning_set(0, 32, bad)
        with pytest.raises(ValueError):
            xb.tuning_set(1, 64, old)  # no SHAKE128 n = 64 family
    finally:
        xb.tuning_set(0, 32, old)
