"""ctypes bindings for the CPU oracle (TEST INFRASTRUCTURE ONLY).

`Oracle` wraps oracle/liboracle.so, the plain-C restatement of the reference
CU-XMSS CPU path.  `RefLib` wraps oracle/_ref/libxmssref.so, the reference's
own C sources compiled here by `make -C oracle ref` (present only where the
reference sources were available at build time).

Only tests/, the smoke check and bench.py's CPU-baseline leg import this
module; the CUDA library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libxmssref.so")


class Params(C.Structure):
    """Same layout as xmss_params (cuxmss/params.h:15-33)."""

    _fields_ = [
        ("func", C.c_uint),
        ("n", C.c_uint),
        ("padding_len", C.c_uint),
        ("wots_w", C.c_uint),
        ("wots_log_w", C.c_uint),
        ("wots_len1", C.c_uint),
        ("wots_len2", C.c_uint),
        ("wots_len", C.c_uint),
        ("wots_sig_bytes", C.c_uint),
        ("full_height", C.c_uint),
        ("tree_height", C.c_uint),
        ("d", C.c_uint),
        ("index_bytes", C.c_uint),
        ("sig_bytes", C.c_uint),
        ("pk_bytes", C.c_uint),
        ("sk_bytes", C.c_ulonglong),
        ("bds_k", C.c_uint),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and the reference build when its sources exist)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "liboracle.so"], check=True, stdout=out)
    # skipped by the Makefile where the reference sources are absent
    subprocess.run(["make", "-C", HERE, "ref"], check=True, stdout=out)


def _buf(b: bytes | bytearray | int):
    if isinstance(b, int):
        return (C.c_uint8 * max(b, 1))()
    return (C.c_uint8 * max(len(b), 1)).from_buffer_copy(bytes(b) or b"\0")


def _addr(a):
    return (C.c_uint32 * 8)(*a)


class Oracle:
    """The plain-C restatement (oracle/xmss_oracle.c)."""

    def __init__(self, path: str = LIB_PATH):
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        L = self.lib
        u8p = C.POINTER(C.c_uint8)
        L.xo_parse_oid.argtypes = [C.POINTER(Params), C.c_uint32, C.c_int]
        L.xo_str_to_oid.argtypes = [C.POINTER(C.c_uint32), C.c_char_p, C.c_int]
        for f in ("xo_sha256", "xo_sha512"):
            getattr(L, f).argtypes = [u8p, u8p, C.c_size_t]
        for f in ("xo_shake128", "xo_shake256"):
            getattr(L, f).argtypes = [u8p, C.c_size_t, u8p, C.c_size_t]
        L.xo_seed_keypair.argtypes = [C.POINTER(Params), u8p, u8p, u8p]
        L.xo_sign.argtypes = [C.POINTER(Params), u8p, u8p, C.POINTER(C.c_ulonglong), u8p, C.c_ulonglong]
        L.xo_sign_with_trees.argtypes = [C.POINTER(Params), u8p, u8p, C.POINTER(C.c_ulonglong),
                                         u8p, C.c_ulonglong, u8p]
        L.xo_sign_open.argtypes = [C.POINTER(Params), u8p, C.POINTER(C.c_ulonglong), u8p,
                                   C.c_ulonglong, u8p]
        L.xo_tree_nodes.argtypes = [C.POINTER(Params), u8p, u8p, u8p, C.c_uint32, C.c_uint64, C.c_int]
        L.xo_leaves.argtypes = [C.POINTER(Params), u8p, u8p, u8p, C.c_uint32, C.c_uint64,
                                C.c_uint32, C.c_uint32, C.c_int]
        L.xo_wots_pkgen.argtypes = [C.POINTER(Params), u8p, u8p, u8p, C.POINTER(C.c_uint32)]
        L.xo_wots_sign.argtypes = [C.POINTER(Params), u8p, u8p, u8p, u8p, C.POINTER(C.c_uint32)]
        L.xo_wots_pk_from_sig.argtypes = [C.POINTER(Params), u8p, u8p, u8p, u8p, C.POINTER(C.c_uint32)]
        L.xo_gen_leaf_wots.argtypes = [C.POINTER(Params), u8p, u8p, u8p, C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_uint32)]
        L.xo_thash_f.argtypes = [C.POINTER(Params), u8p, u8p, u8p, C.POINTER(C.c_uint32)]
        L.xo_thash_h.argtypes = [C.POINTER(Params), u8p, u8p, u8p, C.POINTER(C.c_uint32)]
        L.xo_prf.argtypes = [C.POINTER(Params), u8p, u8p, u8p]
        L.xo_prf_keygen.argtypes = [C.POINTER(Params), u8p, u8p, u8p]
        L.xo_hash_message.argtypes = [C.POINTER(Params), u8p, u8p, u8p, C.c_ulonglong, u8p, C.c_ulonglong]
        L.xo_chain_lengths.argtypes = [C.POINTER(Params), C.POINTER(C.c_int), u8p]
        L.xo_verify_chain_steps.argtypes = [C.POINTER(Params), u8p]
        L.xo_api_seed_keypair.argtypes = [u8p, u8p, C.c_uint32, C.c_int, u8p]
        L.xo_api_sign.argtypes = [u8p, u8p, C.POINTER(C.c_ulonglong), u8p, C.c_ulonglong, C.c_int]
        L.xo_api_sign_open.argtypes = [u8p, C.POINTER(C.c_ulonglong), u8p, C.c_ulonglong, u8p, C.c_int]

    # -- parameters -------------------------------------------------------
    def params(self, oid: int, mt: bool = False) -> Params:
        p = Params()
        if self.lib.xo_parse_oid(C.byref(p), oid, int(mt)):
            raise ValueError(f"unknown {'XMSSMT' if mt else 'XMSS'} OID {oid:#x}")
        return p

    def str_to_oid(self, name: str) -> tuple[int, bool]:
        mt = name.startswith("XMSSMT")
        o = C.c_uint32()
        if self.lib.xo_str_to_oid(C.byref(o), name.encode(), int(mt)):
            raise ValueError(name)
        return o.value, mt

    # -- hashes -----------------------------------------------------------
    def sha256(self, m: bytes) -> bytes:
        o = _buf(32)
        self.lib.xo_sha256(o, _buf(m), len(m))
        return bytes(o)

    def sha512(self, m: bytes) -> bytes:
        o = _buf(64)
        self.lib.xo_sha512(o, _buf(m), len(m))
        return bytes(o)

    def shake128(self, m: bytes, outlen: int) -> bytes:
        o = _buf(outlen)
        self.lib.xo_shake128(o, outlen, _buf(m), len(m))
        return bytes(o)[:outlen]

    def shake256(self, m: bytes, outlen: int) -> bytes:
        o = _buf(outlen)
        self.lib.xo_shake256(o, outlen, _buf(m), len(m))
        return bytes(o)[:outlen]

    # -- tweakable hashes -------------------------------------------------
    def thash_f(self, p: Params, x: bytes, pub_seed: bytes, addr) -> bytes:
        o = _buf(p.n)
        self.lib.xo_thash_f(C.byref(p), o, _buf(x), _buf(pub_seed), _addr(addr))
        return bytes(o)[: p.n]

    def thash_h(self, p: Params, lr: bytes, pub_seed: bytes, addr) -> bytes:
        o = _buf(p.n)
        self.lib.xo_thash_h(C.byref(p), o, _buf(lr), _buf(pub_seed), _addr(addr))
        return bytes(o)[: p.n]

    def prf(self, p: Params, in32: bytes, key: bytes) -> bytes:
        o = _buf(p.n)
        self.lib.xo_prf(C.byref(p), o, _buf(in32), _buf(key))
        return bytes(o)[: p.n]

    def prf_keygen(self, p: Params, inp: bytes, key: bytes) -> bytes:
        o = _buf(p.n)
        self.lib.xo_prf_keygen(C.byref(p), o, _buf(inp), _buf(key))
        return bytes(o)[: p.n]

    def hash_message(self, p: Params, R: bytes, root: bytes, idx: int, m: bytes) -> bytes:
        o = _buf(p.n)
        self.lib.xo_hash_message(C.byref(p), o, _buf(R), _buf(root), idx, _buf(m), len(m))
        return bytes(o)[: p.n]

    def chain_lengths(self, p: Params, msg: bytes) -> list[int]:
        arr = (C.c_int * p.wots_len)()
        self.lib.xo_chain_lengths(C.byref(p), arr, _buf(msg))
        return list(arr)

    def verify_chain_steps(self, p: Params, msg: bytes) -> int:
        return self.lib.xo_verify_chain_steps(C.byref(p), _buf(msg))

    # -- WOTS / leaves ----------------------------------------------------
    def wots_pkgen(self, p: Params, seed: bytes, pub_seed: bytes, addr) -> bytes:
        o = _buf(p.wots_sig_bytes)
        self.lib.xo_wots_pkgen(C.byref(p), o, _buf(seed), _buf(pub_seed), _addr(addr))
        return bytes(o)

    def wots_sign(self, p: Params, msg: bytes, seed: bytes, pub_seed: bytes, addr) -> bytes:
        o = _buf(p.wots_sig_bytes)
        self.lib.xo_wots_sign(C.byref(p), o, _buf(msg), _buf(seed), _buf(pub_seed), _addr(addr))
        return bytes(o)

    def wots_pk_from_sig(self, p: Params, sig: bytes, msg: bytes, pub_seed: bytes, addr) -> bytes:
        o = _buf(p.wots_sig_bytes)
        self.lib.xo_wots_pk_from_sig(C.byref(p), o, _buf(sig), _buf(msg), _buf(pub_seed), _addr(addr))
        return bytes(o)

    def gen_leaf_wots(self, p: Params, sk_seed: bytes, pub_seed: bytes, ltree_addr, ots_addr) -> bytes:
        o = _buf(p.n)
        self.lib.xo_gen_leaf_wots(C.byref(p), o, _buf(sk_seed), _buf(pub_seed),
                                  _addr(ltree_addr), _addr(ots_addr))
        return bytes(o)[: p.n]

    def leaves(self, p: Params, sk_seed: bytes, pub_seed: bytes, layer: int, tree: int,
               first: int, count: int, nthreads: int = 1) -> bytes:
        o = _buf(count * p.n)
        self.lib.xo_leaves(C.byref(p), o, _buf(sk_seed), _buf(pub_seed), layer, tree,
                           first, count, nthreads)
        return bytes(o)

    def tree_nodes(self, p: Params, sk_seed: bytes, pub_seed: bytes, layer: int, tree: int,
                   nthreads: int = 1) -> bytes:
        total = ((2 << p.tree_height) - 1) * p.n
        o = _buf(total)
        if self.lib.xo_tree_nodes(C.byref(p), o, _buf(sk_seed), _buf(pub_seed), layer, tree, nthreads):
            raise RuntimeError("xo_tree_nodes failed")
        return bytes(o)

    # -- core keygen / sign / verify (no OID prefix) ----------------------
    def seed_keypair(self, p: Params, seed: bytes) -> tuple[bytes, bytes]:
        pk, sk = _buf(p.pk_bytes), _buf(p.sk_bytes)
        self.lib.xo_seed_keypair(C.byref(p), pk, sk, _buf(seed))
        return bytes(pk), bytes(sk)

    def sign(self, p: Params, sk: bytes, m: bytes, trees: bytes | None = None) -> tuple[int, bytes, bytes]:
        skb = _buf(sk)
        sm = _buf(p.sig_bytes + len(m))
        smlen = C.c_ulonglong()
        if trees is None:
            r = self.lib.xo_sign(C.byref(p), skb, sm, C.byref(smlen), _buf(m), len(m))
        else:
            r = self.lib.xo_sign_with_trees(C.byref(p), skb, sm, C.byref(smlen), _buf(m), len(m),
                                            _buf(trees))
        return r, bytes(skb)[: len(sk)], bytes(sm)[: smlen.value]

    def sign_open(self, p: Params, sm: bytes, pk: bytes) -> tuple[int, bytes]:
        m = _buf(len(sm))
        mlen = C.c_ulonglong()
        r = self.lib.xo_sign_open(C.byref(p), m, C.byref(mlen), _buf(sm), len(sm), _buf(pk))
        return r, bytes(m)[: mlen.value]

    # -- OID-prefixed API (xmss.c) ----------------------------------------
    def api_seed_keypair(self, oid: int, mt: bool, seed: bytes) -> tuple[bytes, bytes]:
        p = self.params(oid, mt)
        pk, sk = _buf(p.pk_bytes + 4), _buf(p.sk_bytes + 4)
        if self.lib.xo_api_seed_keypair(pk, sk, oid, int(mt), _buf(seed)):
            raise ValueError(oid)
        return bytes(pk), bytes(sk)

    def api_sign_open(self, sm: bytes, pk: bytes, mt: bool) -> tuple[int, bytes]:
        m = _buf(len(sm))
        mlen = C.c_ulonglong()
        r = self.lib.xo_api_sign_open(m, C.byref(mlen), _buf(sm), len(sm), _buf(pk), int(mt))
        return r, bytes(m)[: mlen.value]

    # -- reference test/vectors.c flow, restated ----------------------------
    def vectors_lines(self, nthreads: int | None = None) -> list[str]:
        """The lines test/vectors.c prints (cuxmss/test/vectors.c:29-124).

        Single-tree sets are signed from a node array built on `nthreads`
        host threads (same bytes as the treehash path, much faster)."""
        nthreads = nthreads or os.cpu_count() or 1
        lines = []

        def h10(b: bytes) -> str:
            return self.shake128(b, 10).hex()

        for oid in range(1, 0x15 + 1, 3):
            p = self.params(oid, False)
            a1 = [(500000000 * i) & 0xFFFFFFFF for i in range(8)]
            a2 = [(400000000 * i) & 0xFFFFFFFF for i in range(8)]
            m = bytes((3 * i) & 0xFF for i in range(p.n))
            pub = bytes((2 * i) & 0xFF for i in range(p.n))
            sks = bytes(i & 0xFF for i in range(p.n))
            pk = self.wots_pkgen(p, sks, pub, a1)
            sig = self.wots_sign(p, m, sks, pub, a1)
            leaf = self.gen_leaf_wots(p, sks, pub, a1, a2)
            lines.append(f"WOTS+ {oid} {h10(pk)} {h10(sig)} {h10(leaf)}")
        for mt, oids in ((True, range(2, 57, 8)), (False, range(1, 0x15 + 1, 3))):
            for oid in oids:
                p = self.params(oid, mt)
                seed = bytes(i & 0xFF for i in range(3 * p.n))
                idx = (1 << (p.full_height - 1)).to_bytes(p.index_bytes, "big")
                if p.d == 1:
                    nodes = self.tree_nodes(p, seed[:p.n], seed[2 * p.n:], 0, 0, nthreads)
                    pk = nodes[-p.n:] + seed[2 * p.n:]
                    sk = idx + seed[:2 * p.n] + pk
                    _, _, sm = self.sign(p, sk, bytes([37]), trees=nodes)
                else:
                    pk, sk = self.seed_keypair(p, seed)
                    sk = idx + sk[p.index_bytes:]
                    _, _, sm = self.sign(p, sk, bytes([37]))
                lines.append(f"{'XMSSMT' if mt else 'XMSS'} {oid} {h10(pk)} {h10(sm[:p.sig_bytes])}")
        return lines


class RefLib:
    """The reference's own C path compiled into oracle/_ref (present only when
    the reference sources were available when the repository was built)."""

    def __init__(self, path: str = REF_PATH):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)
        L = self.lib
        u8p = C.POINTER(C.c_uint8)
        L.xmss_parse_oid.argtypes = [C.POINTER(Params), C.c_uint32]
        L.xmssmt_parse_oid.argtypes = [C.POINTER(Params), C.c_uint32]
        L.xmssmt_core_seed_keypair.argtypes = [C.POINTER(Params), u8p, u8p, u8p]
        L.xmssmt_core_sign.argtypes = [C.POINTER(Params), u8p, u8p, C.POINTER(C.c_ulonglong), u8p,
                                       C.c_ulonglong]
        L.xmssmt_core_sign_open.argtypes = [C.POINTER(Params), u8p, C.POINTER(C.c_ulonglong), u8p,
                                            C.c_ulonglong, u8p]
        L.xmss_sign_open.argtypes = [u8p, C.POINTER(C.c_ulonglong), u8p, C.c_ulonglong, u8p]
        L.xmssmt_sign_open.argtypes = [u8p, C.POINTER(C.c_ulonglong), u8p, C.c_ulonglong, u8p]
        L.gen_leaf_wots.argtypes = [C.POINTER(Params), u8p, u8p, u8p, C.POINTER(C.c_uint32),
                                    C.POINTER(C.c_uint32)]
        L.ref_randombytes_seed.argtypes = [C.c_uint64]

    def params(self, oid: int, mt: bool = False) -> Params:
        p = Params()
        f = self.lib.xmssmt_parse_oid if mt else self.lib.xmss_parse_oid
        if f(C.byref(p), oid):
            raise ValueError(oid)
        return p

    def seed_keypair(self, p: Params, seed: bytes) -> tuple[bytes, bytes]:
        pk, sk = _buf(p.pk_bytes), _buf(p.sk_bytes)
        self.lib.xmssmt_core_seed_keypair(C.byref(p), pk, sk, _buf(seed))
        return bytes(pk), bytes(sk)

    def sign(self, p: Params, sk: bytes, m: bytes) -> tuple[int, bytes, bytes]:
        skb = _buf(sk)
        sm = _buf(p.sig_bytes + len(m))
        smlen = C.c_ulonglong()
        r = self.lib.xmssmt_core_sign(C.byref(p), skb, sm, C.byref(smlen), _buf(m), len(m))
        return r, bytes(skb)[: len(sk)], bytes(sm)[: smlen.value]

    def sign_open(self, p: Params, sm: bytes, pk: bytes) -> tuple[int, bytes]:
        m = _buf(len(sm))
        mlen = C.c_ulonglong()
        r = self.lib.xmssmt_core_sign_open(C.byref(p), m, C.byref(mlen), _buf(sm), len(sm), _buf(pk))
        return r, bytes(m)[: mlen.value]

    def gen_leaf_wots(self, p: Params, sk_seed: bytes, pub_seed: bytes, ltree_addr, ots_addr) -> bytes:
        o = _buf(p.n)
        self.lib.gen_leaf_wots(C.byref(p), o, _buf(sk_seed), _buf(pub_seed), _addr(ltree_addr),
                               _addr(ots_addr))
        return bytes(o)[: p.n]


@dataclass
class Sizes:
    n: int
    sig_bytes: int
    pk_bytes: int
    sk_bytes: int
