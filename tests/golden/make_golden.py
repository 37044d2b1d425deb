"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference sources (default
/root/reference/cuxmss, override with XMSS_REF_DIR):

    make -C oracle ref && python tests/golden/make_golden.py

Outputs (all small, committed):
  vectors.txt   stdout of the reference's test/vectors.c built by oracle/Makefile
                (SHAKE128 digests of WOTS+/XMSS/XMSS^MT keys and signatures for
                every hash family, cuxmss/test/vectors.c:29-124)
  kat_h20.json  zero-seed h=20 public keys embedded in the reference's GPU key
                headers (cuxmss/gpu/sha256_key.h, sha256_192_key.h,
                shake256_key.h, shake256_192_key.h), read as text
  config1.json  XMSS-SHA2_10_256 keypair from a seeded 96-byte seed and 16
                signatures of 32-byte messages at indices 0..15, all computed by
                the reference C path (xmssmt_core_seed_keypair / xmssmt_core_sign)
  mt_small.json one XMSS^MT 20/4 key per hash family and signatures at seeded
                indices, computed by the reference C path
"""
from __future__ import annotations

import json
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle import RefLib  # noqa: E402

REF_DIR = os.environ.get("XMSS_REF_DIR", "/root/reference/cuxmss")

# (header, #if condition fields) -> (mt, oid).  Each header holds three keys in
# order: XMSS h=20, XMSS^MT 40/2 (tree height 20), XMSS^MT 60/3 (tree height 20).
KAT_HEADERS = {
    "sha256_key.h": [(False, 0x03), (True, 0x03), (True, 0x06)],
    "sha256_192_key.h": [(False, 0x0F), (True, 0x23), (True, 0x26)],
    "shake256_key.h": [(False, 0x12), (True, 0x2B), (True, 0x2E)],
    "shake256_192_key.h": [(False, 0x15), (True, 0x33), (True, 0x36)],
}


def make_vectors() -> None:
    exe = os.path.join(ROOT, "oracle", "_ref", "vectors")
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    with open(os.path.join(HERE, "vectors.txt"), "w") as f:
        f.write(out)


def make_kat() -> None:
    kats = []
    for name, ids in KAT_HEADERS.items():
        text = open(os.path.join(REF_DIR, "gpu", name)).read()
        conds = re.findall(r"#(?:el)?if (FULL_HEIGHT == \d+ && TREE_HEIGHT == \d+ && N == \d+ && FUNC == \w+)", text)
        pks = re.findall(r"public_pk\[\]\s*=\s*\{([^}]*)\}", text)
        assert len(pks) == 3 and len(conds) == 3, name
        for (mt, oid), cond, body in zip(ids, conds, pks):
            pk = bytes(int(x, 16) for x in re.findall(r"0x([0-9a-fA-F]{2})", body))
            kats.append({"source": f"cuxmss/gpu/{name}", "condition": cond, "mt": mt, "oid": oid,
                         "seed": "00" * (3 * (len(pk) // 2)), "pk": pk.hex()})
    with open(os.path.join(HERE, "kat_h20.json"), "w") as f:
        json.dump(kats, f, indent=1)


def make_config1(ref: RefLib) -> None:
    rng = np.random.default_rng(20260101)
    p = ref.params(0x01, False)
    seed = rng.bytes(3 * p.n)
    msgs = [rng.bytes(32) for _ in range(16)]
    pk, sk0 = ref.seed_keypair(p, seed)

    def one(i):
        sk = i.to_bytes(p.index_bytes, "big") + sk0[p.index_bytes:]
        r, sk_after, sm = ref.sign(p, sk, msgs[i])
        assert r == 0
        return sk_after, sm

    with ThreadPoolExecutor(os.cpu_count() or 4) as ex:
        res = list(ex.map(one, range(16)))
    for sk_after, sm in res:
        assert ref.sign_open(p, sm, pk)[0] == 0
    doc = {"oid": 1, "mt": False, "name": "XMSS-SHA2_10_256", "seed": seed.hex(),
           "pk": "00000001" + pk.hex(), "sk": "00000001" + sk0.hex(),
           "msgs": [m.hex() for m in msgs], "sms": [sm.hex() for _, sm in res],
           "sk_after": ["00000001" + s.hex() for s, _ in res]}
    with open(os.path.join(HERE, "config1.json"), "w") as f:
        json.dump(doc, f, indent=1)


def make_mt_small(ref: RefLib) -> None:
    rng = np.random.default_rng(20260202)
    out = []
    for oid in (0x02, 0x0A, 0x12, 0x1A, 0x22, 0x2A, 0x32):  # every family, 20/4
        p = ref.params(oid, True)
        seed = rng.bytes(3 * p.n)
        pk, sk0 = ref.seed_keypair(p, seed)
        sigs = []
        for _ in range(3):
            idx = int(rng.integers(0, 1 << p.full_height))
            mlen = int(rng.integers(0, 300))
            m = rng.bytes(mlen)
            sk = idx.to_bytes(p.index_bytes, "big") + sk0[p.index_bytes:]
            r, _, sm = ref.sign(p, sk, m)
            assert r == 0 and ref.sign_open(p, sm, pk)[0] == 0
            sigs.append({"idx": idx, "m": m.hex(), "sm": sm.hex()})
        out.append({"oid": oid, "mt": True, "seed": seed.hex(), "pk": pk.hex(), "sk": sk0.hex(),
                    "sigs": sigs})
    with open(os.path.join(HERE, "mt_small.json"), "w") as f:
        json.dump(out, f, indent=1)


def main() -> None:
    ref = RefLib()
    make_vectors()
    make_kat()
    make_mt_small(ref)
    make_config1(ref)


if __name__ == "__main__":
    main()
