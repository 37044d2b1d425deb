"""Python bindings of libxmss_b200.so, the sm_100a XMSS / XMSS^MT library.

The functions mirror the reference's C API (cuxmss/xmss.h, xmss_core.h,
params.h) with Python return values instead of output pointers:

    xmss_keypair(oid)                 -> (ret, pk, sk)
    xmss_sign(sk, m)                  -> (ret, sk_updated, sm)
    xmss_sign_open(sm, pk)            -> (ret, m)
    xmssmt_* likewise; xmssmt_core_seed_keypair(params, seed) -> (ret, pk, sk)

plus the batch / device entry points of include/xmss_b200.h.  Every call
runs on the GPU; importing this module fails loudly when the shared library
has not been built (python -c "import __graft_entry__ as g; g.build()").
"""
from __future__ import annotations

import ctypes as C
import os
import re
from typing import Sequence

import numpy as np

# 32 hardware work queues for the serving loop's streams (read by the CUDA
# runtime when the process creates its first context; an existing setting wins)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

HERE = os.path.dirname(os.path.abspath(__file__))
# XMSS_B200_LIB selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("XMSS_B200_LIB") or os.path.join(HERE, "libxmss_b200.so")
INCLUDE_DIR = os.path.join(os.path.dirname(os.path.dirname(HERE)), "include")

XMSS_SHA2, XMSS_SHAKE128, XMSS_SHAKE256 = 0, 1, 2
XMSS_OID_LEN = 4
GPU_FAILURE = -3


class XmssParams(C.Structure):
    """xmss_params (include/params.h; cuxmss/params.h:15-33)."""

    _fields_ = [
        ("func", C.c_uint), ("n", C.c_uint), ("padding_len", C.c_uint), ("wots_w", C.c_uint),
        ("wots_log_w", C.c_uint), ("wots_len1", C.c_uint), ("wots_len2", C.c_uint),
        ("wots_len", C.c_uint), ("wots_sig_bytes", C.c_uint), ("full_height", C.c_uint),
        ("tree_height", C.c_uint), ("d", C.c_uint), ("index_bytes", C.c_uint),
        ("sig_bytes", C.c_uint), ("pk_bytes", C.c_uint), ("sk_bytes", C.c_ulonglong),
        ("bds_k", C.c_uint),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Work(C.Structure):
    _fields_ = [("hmsg_blocks", C.c_ulonglong), ("f_calls", C.c_ulonglong), ("h_calls", C.c_ulonglong)]


class GpuError(RuntimeError):
    pass


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C cu-xmss_b200` "
                          "(or __graft_entry__.build()); there is no CPU fallback")
    return C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL | os.RTLD_NOW)


lib = _load()
_u8p = C.POINTER(C.c_uint8)
_u64p = C.POINTER(C.c_uint64)
_ullp = C.POINTER(C.c_ulonglong)
_u32p = C.POINTER(C.c_uint32)
_intp = C.POINTER(C.c_int)

lib.xmss_str_to_oid.argtypes = [_u32p, C.c_char_p]
lib.xmssmt_str_to_oid.argtypes = [_u32p, C.c_char_p]
lib.xmss_parse_oid.argtypes = [C.POINTER(XmssParams), C.c_uint32]
lib.xmssmt_parse_oid.argtypes = [C.POINTER(XmssParams), C.c_uint32]
lib.xmss_xmssmt_initialize_params.argtypes = [C.POINTER(XmssParams)]
lib.xmss_xmssmt_core_sk_bytes.argtypes = [C.POINTER(XmssParams)]
lib.xmss_xmssmt_core_sk_bytes.restype = C.c_ulonglong
for _f in ("xmss_keypair", "xmssmt_keypair"):
    getattr(lib, _f).argtypes = [_u8p, _u8p, C.c_uint32]
for _f in ("xmss_sign", "xmssmt_sign"):
    getattr(lib, _f).argtypes = [_u8p, _u8p, _ullp, _u8p, C.c_ulonglong]
for _f in ("xmss_sign_open", "xmssmt_sign_open"):
    getattr(lib, _f).argtypes = [_u8p, _ullp, _u8p, C.c_ulonglong, _u8p]
lib.xmssmt_core_seed_keypair.argtypes = [C.POINTER(XmssParams), _u8p, _u8p, _u8p]
for _f in ("xmss_core_keypair", "xmssmt_core_keypair"):
    getattr(lib, _f).argtypes = [C.POINTER(XmssParams), _u8p, _u8p]
for _f in ("xmss_core_sign", "xmssmt_core_sign"):
    getattr(lib, _f).argtypes = [C.POINTER(XmssParams), _u8p, _u8p, _ullp, _u8p, C.c_ulonglong]
for _f in ("xmss_core_sign_open", "xmssmt_core_sign_open"):
    getattr(lib, _f).argtypes = [C.POINTER(XmssParams), _u8p, _ullp, _u8p, C.c_ulonglong, _u8p]
lib.xmss_b200_init.argtypes = [C.c_int]
lib.xmss_b200_last_error.restype = C.c_char_p
_RNG = C.CFUNCTYPE(None, _u8p, C.c_ulonglong)
lib.xmss_b200_set_randombytes.argtypes = [_RNG]
lib.xmss_b200_supported.argtypes = [C.c_uint, C.c_uint]
lib.xmss_b200_keypair_batch.argtypes = [C.c_uint32, C.c_int, C.c_uint32, _u8p, _u8p, _u8p]
lib.xmss_b200_keypair_device.argtypes = [C.c_uint32, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]
lib.xmss_b200_sign_open_batch.argtypes = [C.c_int, C.c_uint32, _u8p, _u64p, _u64p, _u8p, C.c_uint32,
                                          _u32p, _intp]
lib.xmss_b200_sign_open_device.argtypes = [C.c_uint32, C.c_int, C.c_uint32, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p,
                                           C.c_void_p]
lib.xmss_b200_sign_open_batch_async.argtypes = [C.c_int, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
lib.xmss_b200_bds_sk_bytes.argtypes = [C.c_uint32, C.c_int]
lib.xmss_b200_bds_sk_bytes.restype = C.c_ulonglong
lib.xmss_b200_sk_from_bds.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
lib.xmss_b200_sk_to_bds.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
lib.xmss_b200_verify_graph_create.argtypes = [C.c_uint32, C.c_int, C.c_uint32] + [C.c_void_p] * 4 + [
    C.c_uint32, C.c_void_p, C.c_void_p, C.POINTER(C.c_void_p)]
lib.xmss_b200_verify_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
lib.xmss_b200_verify_graph_destroy.argtypes = [C.c_void_p]
lib.xmss_b200_verify_graph_destroy.restype = None


class Tuning(C.Structure):
    """xmss_b200_tuning (include/xmss_b200.h)."""

    _fields_ = [(k, C.c_uint32) for k in ("verify_chain_block", "keygen_chain_block", "level_block", "split_min",
                                          "short_hmsg_blocks", "prep_split")]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


lib.xmss_b200_tuning_get.argtypes = [C.c_uint, C.c_uint, C.POINTER(Tuning)]
lib.xmss_b200_tuning_set.argtypes = [C.c_uint, C.c_uint, C.POINTER(Tuning)]
lib.xmss_b200_autotune.argtypes = [C.c_uint32, C.c_int, C.c_uint32, C.POINTER(Tuning), C.c_char_p, C.c_size_t]
lib.xmss_b200_sign_batch.argtypes = [C.c_int, C.c_uint32, _u8p, _u8p, _u64p, _u64p, _u8p, _u64p,
                                     _u64p, _intp]
lib.xmss_b200_core_hash_batch.argtypes = [C.c_uint, C.c_uint, C.c_uint32, _u8p, _u64p, _u64p, _u8p]
lib.xmss_b200_last_verify_work.argtypes = [C.POINTER(Work)]
lib.xmss_b200_sign_open_device_noalloc.argtypes = lib.xmss_b200_sign_open_device.argtypes
lib.xmss_b200_sign_open_device_persistent.argtypes = lib.xmss_b200_sign_open_device.argtypes
lib.xmss_b200_set_wait_bound.argtypes = [C.c_ulonglong]
lib.xmss_b200_profile.argtypes = [C.c_int]
lib.xmss_b200_phase_ms.argtypes = [C.POINTER(C.c_double)]
lib.xmss_b200_rate_probe.argtypes = [C.c_int, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p]


class ServerConfig(C.Structure):
    """xmss_b200_server_config (include/xmss_b200.h)."""

    _fields_ = [("max_batch", C.c_uint32), ("slots", C.c_uint32), ("window_us", C.c_uint32),
                ("reserved0", C.c_uint32), ("tree_pool_bytes", C.c_uint64), ("mem_reserve_bytes", C.c_uint64)]


class Completion(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("ret", C.c_int32), ("kind", C.c_uint32), ("index", C.c_uint64),
                ("latency_us", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "batches", "sign_groups", "verify_groups",
                                          "largest_batch", "deferred_for_memory", "trees_built", "tree_hits",
                                          "trees_evicted")] + [
        ("launch_us", C.c_double), ("finish_us", C.c_double), ("batch_us", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchTrace(C.Structure):
    """xmss_b200_batch_trace (include/xmss_b200.h)."""

    _fields_ = [("seq", C.c_uint64), ("requests", C.c_uint32), ("plans", C.c_uint32), ("slow_kind", C.c_uint32),
                ("slow_oid", C.c_uint32), ("queue_us", C.c_double), ("launch_us", C.c_double),
                ("gpu_us", C.c_double), ("lane_us", C.c_double), ("done_us", C.c_double),
                ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64), ("start_skew_us", C.c_double),
                ("join_us", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


# xmss_b200_trace_item as a numpy record (same layout as the C struct)
TRACE_DTYPE = np.dtype([("t_us", "<f8"), ("kind", "<u4"), ("key_id", "<u4"), ("mt", "<i4"), ("reserved0", "<u4"),
                        ("in_ptr", "<u8"), ("inlen", "<u8"), ("sm_ptr", "<u8"), ("smlen_ptr", "<u8"),
                        ("pk_ptr", "<u8")])
assert TRACE_DTYPE.itemsize == 64

_srvp = C.c_void_p
lib.xmss_b200_server_create.argtypes = [C.POINTER(ServerConfig), C.POINTER(_srvp)]
lib.xmss_b200_server_destroy.argtypes = [_srvp]
lib.xmss_b200_server_destroy.restype = None
lib.xmss_b200_server_add_key.argtypes = [_srvp, C.c_int, C.c_void_p, _u32p]
lib.xmss_b200_server_export_sk.argtypes = [_srvp, C.c_uint32, C.c_void_p]
lib.xmss_b200_server_submit_sign.argtypes = [_srvp, C.c_uint32, C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                                             C.c_uint64]
lib.xmss_b200_server_submit_verify.argtypes = [_srvp, C.c_int, C.c_void_p, C.c_uint64, C.c_void_p, C.c_uint64]
lib.xmss_b200_server_submit_warm.argtypes = [_srvp, C.c_uint32, C.c_uint64]
lib.xmss_b200_server_poll.argtypes = [_srvp, C.POINTER(Completion), C.c_uint32, C.c_uint32]
lib.xmss_b200_server_stats_get.argtypes = [_srvp, C.POINTER(ServerStats)]
lib.xmss_b200_server_trace.argtypes = [_srvp, C.POINTER(BatchTrace), C.c_uint32]
lib.xmss_b200_server_replay.argtypes = [_srvp, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.POINTER(C.c_double)]

PHASES = ("prep", "chains", "ltree", "root", "tree")


def header_functions() -> list[str]:
    """Names of every function declared in include/*.h."""
    names = []
    for f in sorted(os.listdir(INCLUDE_DIR)):
        if f.endswith(".h"):
            text = re.sub(r"/\*.*?\*/", "", open(os.path.join(INCLUDE_DIR, f)).read(), flags=re.S)
            names += re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if n not in ("if", "while", "for", "return", "sizeof")))


def _buf(b, size: int | None = None):
    if isinstance(b, int):
        return (C.c_uint8 * max(b, 1))()
    b = bytes(b)
    n = max(len(b) if size is None else size, 1)
    out = (C.c_uint8 * n)()
    C.memmove(out, b, len(b))
    return out


def _np_ptr(a: np.ndarray, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))


def last_error() -> str:
    return lib.xmss_b200_last_error().decode()


def _check(ret: int, what: str) -> int:
    if ret == GPU_FAILURE:
        raise GpuError(f"{what}: {last_error()}")
    return ret


# -- params.h ----------------------------------------------------------------

def xmss_str_to_oid(name: str) -> int:
    o = C.c_uint32()
    if lib.xmss_str_to_oid(C.byref(o), name.encode()):
        raise ValueError(name)
    return o.value


def xmssmt_str_to_oid(name: str) -> int:
    o = C.c_uint32()
    if lib.xmssmt_str_to_oid(C.byref(o), name.encode()):
        raise ValueError(name)
    return o.value


def parse_oid(oid: int, mt: bool = False) -> XmssParams:
    p = XmssParams()
    f = lib.xmssmt_parse_oid if mt else lib.xmss_parse_oid
    if f(C.byref(p), oid):
        raise ValueError(f"unknown {'XMSSMT' if mt else 'XMSS'} OID {oid:#x}")
    return p


def params_by_name(name: str) -> tuple[int, bool, XmssParams]:
    mt = name.startswith("XMSSMT")
    oid = xmssmt_str_to_oid(name) if mt else xmss_str_to_oid(name)
    return oid, mt, parse_oid(oid, mt)


# -- device / randomness ---------------------------------------------------

def init(device: int = 0) -> None:
    _check(lib.xmss_b200_init(device), "xmss_b200_init")


_rng_keepalive = None


def set_randombytes(fn) -> None:
    """fn(nbytes) -> bytes; None restores /dev/urandom."""
    global _rng_keepalive
    if fn is None:
        _rng_keepalive = None
        lib.xmss_b200_set_randombytes(_RNG())
        return

    def cb(x, n):
        b = fn(n)
        C.memmove(x, b, n)

    _rng_keepalive = _RNG(cb)
    lib.xmss_b200_set_randombytes(_rng_keepalive)


# -- xmss.h / xmss_core.h ----------------------------------------------------

def _keypair(oid: int, mt: bool):
    try:
        p = parse_oid(oid, mt)
        pkb, skb = XMSS_OID_LEN + p.pk_bytes, XMSS_OID_LEN + p.sk_bytes
    except ValueError:  # the library answers -1 itself
        pkb, skb = XMSS_OID_LEN + 128, XMSS_OID_LEN + 8 + 256
    pk, sk = _buf(pkb), _buf(skb)
    r = _check((lib.xmssmt_keypair if mt else lib.xmss_keypair)(pk, sk, oid), "keypair")
    return r, bytes(pk), bytes(sk)


def xmss_keypair(oid: int):
    return _keypair(oid, False)


def xmssmt_keypair(oid: int):
    return _keypair(oid, True)


def _sign(sk: bytes, m: bytes, mt: bool):
    oid = int.from_bytes(sk[:4], "big")
    try:
        p = parse_oid(oid, mt)
        cap = p.sig_bytes + len(m)
    except ValueError:
        cap = len(m) + 1
    skb = _buf(sk)
    sm = _buf(cap)
    smlen = C.c_ulonglong()
    r = _check((lib.xmssmt_sign if mt else lib.xmss_sign)(skb, sm, C.byref(smlen), _buf(m), len(m)), "sign")
    return r, bytes(skb)[: len(sk)], bytes(sm)[: smlen.value]


def xmss_sign(sk: bytes, m: bytes):
    return _sign(sk, m, False)


def xmssmt_sign(sk: bytes, m: bytes):
    return _sign(sk, m, True)


def _sign_open(sm: bytes, pk: bytes, mt: bool):
    m = _buf(len(sm) + 1)
    mlen = C.c_ulonglong()
    r = _check((lib.xmssmt_sign_open if mt else lib.xmss_sign_open)(m, C.byref(mlen), _buf(sm), len(sm),
                                                                    _buf(pk)), "sign_open")
    return r, bytes(m)[: mlen.value]


def xmss_sign_open(sm: bytes, pk: bytes):
    return _sign_open(sm, pk, False)


def xmssmt_sign_open(sm: bytes, pk: bytes):
    return _sign_open(sm, pk, True)


def xmssmt_core_seed_keypair(p: XmssParams, seed: bytes):
    pk, sk = _buf(p.pk_bytes), _buf(p.sk_bytes)
    r = _check(lib.xmssmt_core_seed_keypair(C.byref(p), pk, sk, _buf(seed)), "seed_keypair")
    return r, bytes(pk), bytes(sk)


def xmssmt_core_sign(p: XmssParams, sk: bytes, m: bytes):
    skb = _buf(sk)
    sm = _buf(p.sig_bytes + len(m))
    smlen = C.c_ulonglong()
    r = _check(lib.xmssmt_core_sign(C.byref(p), skb, sm, C.byref(smlen), _buf(m), len(m)), "core_sign")
    return r, bytes(skb)[: len(sk)], bytes(sm)[: smlen.value]


def xmssmt_core_sign_open(p: XmssParams, sm: bytes, pk: bytes):
    m = _buf(len(sm) + 1)
    mlen = C.c_ulonglong()
    r = _check(lib.xmssmt_core_sign_open(C.byref(p), m, C.byref(mlen), _buf(sm), len(sm), _buf(pk)),
               "core_sign_open")
    return r, bytes(m)[: mlen.value]


# -- xmss_b200.h batch API ---------------------------------------------------

def keypair_batch(oid: int, mt: bool, seeds: np.ndarray):
    """seeds: uint8 [count, 3n] -> (pk [count, 4+2n], sk [count, 4+sk_bytes])."""
    p = parse_oid(oid, mt)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint8)
    count = seeds.shape[0]
    pk = np.zeros((count, XMSS_OID_LEN + p.pk_bytes), np.uint8)
    sk = np.zeros((count, XMSS_OID_LEN + p.sk_bytes), np.uint8)
    r = _check(lib.xmss_b200_keypair_batch(oid, int(mt), count, _np_ptr(seeds, C.c_uint8), _np_ptr(pk, C.c_uint8),
                                           _np_ptr(sk, C.c_uint8)), "keypair_batch")
    if r:
        raise ValueError(f"keypair_batch returned {r}")
    return pk, sk


def pack(chunks: Sequence[bytes], align: int = 1):
    """Concatenates byte strings; returns (buffer uint8, offsets u64, lengths u64)."""
    offs, lens, pos = [], [], 0
    for c in chunks:
        offs.append(pos)
        lens.append(len(c))
        pos += (len(c) + align - 1) // align * align
    buf = np.zeros(max(pos, 1), np.uint8)
    for o, c in zip(offs, chunks):
        buf[o:o + len(c)] = np.frombuffer(bytes(c), np.uint8)
    return buf, np.array(offs, np.uint64), np.array(lens, np.uint64)


def sign_open_batch(mt: bool, sm: np.ndarray, sm_off: np.ndarray, smlen: np.ndarray, pk: np.ndarray,
                    pk_index: np.ndarray | None = None) -> np.ndarray:
    """Batched xmss[mt]_sign_open; returns int32 status per signed message."""
    sm = np.ascontiguousarray(sm, np.uint8)
    sm_off = np.ascontiguousarray(sm_off, np.uint64)
    smlen = np.ascontiguousarray(smlen, np.uint64)
    pk = np.ascontiguousarray(pk, np.uint8)
    count = len(sm_off)
    status = np.full(count, -7, np.int32)
    idxp = None
    if pk_index is not None:
        pk_index = np.ascontiguousarray(pk_index, np.uint32)
        idxp = _np_ptr(pk_index, C.c_uint32)
    r = _check(lib.xmss_b200_sign_open_batch(int(mt), count, _np_ptr(sm, C.c_uint8), _np_ptr(sm_off, C.c_uint64),
                                             _np_ptr(smlen, C.c_uint64), _np_ptr(pk, C.c_uint8), pk.shape[0],
                                             idxp, _np_ptr(status, C.c_int)), "sign_open_batch")
    if r:
        raise ValueError(f"sign_open_batch returned {r}: {last_error()}")
    return status


def sign_open_batch_async(mt: bool, sm: np.ndarray, sm_off: np.ndarray, smlen: np.ndarray, pk: np.ndarray,
                          pk_index: np.ndarray, status: np.ndarray, stream: int) -> None:
    """xmss_b200_sign_open_batch_async: enqueue on `stream` and return.  sm
    and status should be pinned (e.g. torch pin_memory) and stay alive and
    untouched until the stream has passed the call."""
    for a, t in ((sm, np.uint8), (sm_off, np.uint64), (smlen, np.uint64), (pk, np.uint8), (pk_index, np.uint32),
                 (status, np.int32)):
        if a.dtype != t or not a.flags.c_contiguous:
            raise TypeError("sign_open_batch_async wants contiguous arrays of the documented dtypes")
    r = _check(lib.xmss_b200_sign_open_batch_async(int(mt), len(sm_off), sm.ctypes.data, sm_off.ctypes.data,
                                                   smlen.ctypes.data, pk.ctypes.data, pk.shape[0],
                                                   pk_index.ctypes.data, status.ctypes.data, stream),
               "sign_open_batch_async")
    if r:
        raise ValueError(f"sign_open_batch_async returned {r}: {last_error()}")


def sign_batch(mt: bool, sk: np.ndarray, msgs: Sequence[bytes]):
    """Batched xmss[mt]_sign.  sk: uint8 [count, 4+sk_bytes], updated in place.
    Returns (ret int32 [count], list of sm bytes)."""
    sk = np.ascontiguousarray(sk, np.uint8)
    count = sk.shape[0]
    oid = int.from_bytes(bytes(sk[0, :4]), "big")
    p = parse_oid(oid, mt)
    mbuf, moff, mlen = pack(msgs)
    sm_sizes = [p.sig_bytes + len(m) for m in msgs]
    smbuf, smoff, _ = pack([b"\0" * s for s in sm_sizes])
    smlen = np.zeros(count, np.uint64)
    ret = np.zeros(count, np.int32)
    r = _check(lib.xmss_b200_sign_batch(int(mt), count, _np_ptr(sk, C.c_uint8), _np_ptr(mbuf, C.c_uint8),
                                        _np_ptr(moff, C.c_uint64), _np_ptr(mlen, C.c_uint64),
                                        _np_ptr(smbuf, C.c_uint8), _np_ptr(smoff, C.c_uint64),
                                        _np_ptr(smlen, C.c_uint64), _np_ptr(ret, C.c_int)), "sign_batch")
    if r:
        raise ValueError(f"sign_batch returned {r}: {last_error()}")
    sms = [bytes(smbuf[int(o):int(o) + int(l)]) for o, l in zip(smoff, smlen)]
    return ret, sms


def sign_batch_packed(mt: bool, sk: np.ndarray, mbuf: np.ndarray, moff: np.ndarray, mlen: np.ndarray,
                      smbuf: np.ndarray, smoff: np.ndarray, smlen: np.ndarray, ret: np.ndarray) -> None:
    """xmss_b200_sign_batch on arrays the caller packed (contiguous uint8 /
    uint64 / int32, nothing copied): sk [count, 4+sk_bytes] is advanced in
    place, sm i lands at smbuf[smoff[i]:smoff[i]+smlen[i]]."""
    for a, t in ((sk, np.uint8), (mbuf, np.uint8), (moff, np.uint64), (mlen, np.uint64), (smbuf, np.uint8),
                 (smoff, np.uint64), (smlen, np.uint64), (ret, np.int32)):
        if a.dtype != t or not a.flags.c_contiguous:
            raise TypeError("sign_batch_packed wants contiguous arrays of the documented dtypes")
    r = _check(lib.xmss_b200_sign_batch(int(mt), sk.shape[0], _np_ptr(sk, C.c_uint8), _np_ptr(mbuf, C.c_uint8),
                                        _np_ptr(moff, C.c_uint64), _np_ptr(mlen, C.c_uint64),
                                        _np_ptr(smbuf, C.c_uint8), _np_ptr(smoff, C.c_uint64),
                                        _np_ptr(smlen, C.c_uint64), _np_ptr(ret, C.c_int)), "sign_batch")
    if r:
        raise ValueError(f"sign_batch returned {r}: {last_error()}")


def bds_sk_bytes(oid: int, mt: bool) -> int:
    """Size of the reference's BDS ("fast") sk without the OID."""
    return int(lib.xmss_b200_bds_sk_bytes(oid, int(mt)))


def sk_from_bds(mt: bool, bds_sk: bytes) -> bytes:
    """The plain OID-prefixed sk inside a BDS sk (xmss_b200_sk_from_bds)."""
    oid = int.from_bytes(bytes(bds_sk[:4]), "big")
    out = _buf(XMSS_OID_LEN + parse_oid(oid, mt).sk_bytes)
    r = lib.xmss_b200_sk_from_bds(int(mt), _buf(bds_sk), out)
    if r:
        raise ValueError(f"sk_from_bds returned {r}")
    return bytes(out)


def sk_to_bds(mt: bool, sk: bytes) -> bytes:
    """The BDS sk the reference's fast build holds at this sk's index
    (xmss_b200_sk_to_bds)."""
    oid = int.from_bytes(bytes(sk[:4]), "big")
    out = _buf(XMSS_OID_LEN + bds_sk_bytes(oid, mt))
    r = _check(lib.xmss_b200_sk_to_bds(int(mt), _buf(sk), out), "sk_to_bds")
    if r:
        raise ValueError(f"sk_to_bds returned {r}: {last_error()}")
    return bytes(out)


def core_hash_batch(func: int, n: int, msgs: Sequence[bytes]) -> list[bytes]:
    buf, off, ln = pack(msgs)
    out = np.zeros((len(msgs), n), np.uint8)
    r = _check(lib.xmss_b200_core_hash_batch(func, n, len(msgs), _np_ptr(buf, C.c_uint8), _np_ptr(off, C.c_uint64),
                                             _np_ptr(ln, C.c_uint64), _np_ptr(out, C.c_uint8)), "core_hash_batch")
    if r:
        raise ValueError(f"core_hash_batch returned {r}")
    return [bytes(row) for row in out]


def profile(enable: bool) -> None:
    _check(lib.xmss_b200_profile(int(enable)), "profile")


def phase_ms() -> dict:
    a = (C.c_double * 5)()
    _check(lib.xmss_b200_phase_ms(a), "phase_ms")
    return dict(zip(PHASES, list(a)))


def rate_probe(kind: int, blocks: int, iters: int, d_sink: int, stream: int = 0) -> None:
    r = _check(lib.xmss_b200_rate_probe(kind, blocks, iters, d_sink, stream), "rate_probe")
    if r:
        raise ValueError(f"rate_probe returned {r}")


def last_verify_work() -> Work:
    w = Work()
    _check(lib.xmss_b200_last_verify_work(C.byref(w)), "last_verify_work")
    return w


# -- device-pointer API (for callers that keep data in HBM, e.g. torch) -----

def sign_open_device(oid: int, mt: bool, count: int, d_sm: int, d_sm_off: int, d_smlen: int, d_pk: int, npk: int,
                     d_pk_index: int, d_status: int, stream: int = 0) -> None:
    r = _check(lib.xmss_b200_sign_open_device(oid, int(mt), count, d_sm, d_sm_off, d_smlen, d_pk, npk, d_pk_index,
                                              d_status, stream), "sign_open_device")
    if r:
        raise ValueError(f"sign_open_device returned {r}: {last_error()}")


def sign_open_device_persistent(oid: int, mt: bool, count: int, d_sm: int, d_sm_off: int, d_smlen: int, d_pk: int,
                                npk: int, d_pk_index: int, d_status: int, stream: int = 0) -> None:
    """xmss_b200_sign_open_device_persistent: sign_open_device as one
    persistent launch fed by a device work queue."""
    r = _check(lib.xmss_b200_sign_open_device_persistent(oid, int(mt), count, d_sm, d_sm_off, d_smlen, d_pk, npk,
                                                         d_pk_index, d_status, stream), "sign_open_device_persistent")
    if r:
        raise ValueError(f"sign_open_device_persistent returned {r}: {last_error()}")


class VerifyJob(C.Structure):
    """xmss_b200_verify_job (include/xmss_b200.h); d_ fields are device pointers as ints."""
    _fields_ = [("oid", C.c_uint32), ("mt", C.c_int), ("count", C.c_uint32), ("d_sm", C.c_void_p),
                ("d_sm_off", C.c_void_p), ("d_smlen", C.c_void_p), ("d_pk", C.c_void_p), ("npk", C.c_uint32),
                ("d_pk_index", C.c_void_p), ("d_status", C.c_void_p)]


lib.xmss_b200_sign_open_device_persistent_multi.argtypes = [C.POINTER(VerifyJob), C.c_uint32, C.c_void_p]


def sign_open_device_persistent_multi(jobs: Sequence[dict], stream: int = 0) -> None:
    """xmss_b200_sign_open_device_persistent_multi: batches of any parameter
    sets, one persistent launch per hash family (jobs: dicts of VerifyJob fields)."""
    arr = (VerifyJob * len(jobs))()
    for i, j in enumerate(jobs):
        for k, v in j.items():
            setattr(arr[i], k, int(v))
    r = _check(lib.xmss_b200_sign_open_device_persistent_multi(arr, len(jobs), stream),
               "sign_open_device_persistent_multi")
    if r:
        raise ValueError(f"sign_open_device_persistent_multi returned {r}: {last_error()}")


def set_wait_bound(ns: int) -> None:
    """xmss_b200_set_wait_bound: bound of one dependency wait inside later
    persistent launches, in ns (0 = the default of 8 s)."""
    r = _check(lib.xmss_b200_set_wait_bound(int(ns)), "set_wait_bound")
    if r:
        raise ValueError(f"set_wait_bound returned {r}: {last_error()}")


def sign_open_device_noalloc(oid: int, mt: bool, count: int, d_sm: int, d_sm_off: int, d_smlen: int, d_pk: int,
                             npk: int, d_pk_index: int, d_status: int, stream: int = 0) -> int:
    """xmss_b200_sign_open_device_noalloc: returns the C return code (-1 when the
    batch does not fit the fixed scratch array; see last_error())."""
    return _check(lib.xmss_b200_sign_open_device_noalloc(oid, int(mt), count, d_sm, d_sm_off, d_smlen, d_pk, npk,
                                                        d_pk_index, d_status, stream), "sign_open_device_noalloc")


def keypair_device(oid: int, mt: bool, count: int, d_seeds: int, d_pk: int, d_sk: int, stream: int = 0) -> None:
    r = _check(lib.xmss_b200_keypair_device(oid, int(mt), count, d_seeds, d_pk, d_sk, stream), "keypair_device")
    if r:
        raise ValueError(f"keypair_device returned {r}: {last_error()}")


# -- serving (xmss_b200_server_*) -------------------------------------------

class Server:
    """Request loop over device-resident keys (include/xmss_b200.h, serving).

    submit_* return a tag; completions come back from poll() / wait() as
    dicts {tag, ret, kind, index, latency_us} plus "sm" (bytes) for signs.
    Buffers handed to the library are kept alive here until their request
    completes."""

    def __init__(self, max_batch: int = 0, slots: int = 0, window_us: int = 0, tree_pool_bytes: int = 0,
                 mem_reserve_bytes: int = 0):
        cfg = ServerConfig(max_batch, slots, window_us, 0, tree_pool_bytes, mem_reserve_bytes)
        h = _srvp()
        r = _check(lib.xmss_b200_server_create(C.byref(cfg), C.byref(h)), "server_create")
        if r:
            raise ValueError(f"server_create returned {r}")
        self._h = h
        self._next_tag = 1
        self._pending: dict[int, tuple] = {}
        self._sk_len: dict[int, int] = {}

    def close(self) -> None:
        if self._h:
            lib.xmss_b200_server_destroy(self._h)
            self._h = None
            self._pending.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _tag(self) -> int:
        t = self._next_tag
        self._next_tag += 1
        return t

    def add_key(self, sk: bytes, mt: bool = False) -> int:
        key_id = C.c_uint32()
        b = _buf(sk)
        r = _check(lib.xmss_b200_server_add_key(self._h, int(mt), b, C.byref(key_id)), "server_add_key")
        if r:
            raise ValueError(f"server_add_key returned {r}: {last_error()}")
        self._sk_len[key_id.value] = len(sk)
        return key_id.value

    def export_sk(self, key_id: int) -> bytes:
        out = _buf(self._sk_len[key_id])
        r = lib.xmss_b200_server_export_sk(self._h, key_id, out)
        if r:
            raise ValueError(f"server_export_sk returned {r}")
        return bytes(out)

    def submit_sign(self, key_id: int, m: bytes, sig_bytes: int) -> int:
        tag = self._tag()
        mb = _buf(m)
        smb = _buf(sig_bytes + len(m))
        smlen = C.c_uint64()
        r = lib.xmss_b200_server_submit_sign(self._h, key_id, mb, len(m), smb, C.byref(smlen), tag)
        if r:
            raise ValueError(f"server_submit_sign returned {r}")
        self._pending[tag] = (mb, smb, smlen)
        return tag

    def submit_verify(self, sm: bytes, pk: bytes, mt: bool = False) -> int:
        tag = self._tag()
        smb = _buf(sm)
        r = lib.xmss_b200_server_submit_verify(self._h, int(mt), smb, len(sm), _buf(pk), tag)
        if r:
            raise ValueError(f"server_submit_verify returned {r}")
        self._pending[tag] = (smb,)
        return tag

    def submit_warm(self, key_id: int) -> int:
        tag = self._tag()
        r = lib.xmss_b200_server_submit_warm(self._h, key_id, tag)
        if r:
            raise ValueError(f"server_submit_warm returned {r}")
        self._pending[tag] = ()
        return tag

    def poll(self, max_items: int = 4096, wait_us: int = 0) -> list[dict]:
        arr = (Completion * max_items)()
        n = lib.xmss_b200_server_poll(self._h, arr, max_items, wait_us)
        out = []
        for c in arr[:n]:
            d = {"tag": c.tag, "ret": c.ret, "kind": c.kind, "index": c.index, "latency_us": c.latency_us}
            keep = self._pending.pop(c.tag, None)
            if c.kind == 0 and keep:
                _, smb, smlen = keep
                d["sm"] = bytes(smb)[:smlen.value] if c.ret == 0 else b""
            out.append(d)
        return out

    def wait(self, tags, timeout_s: float = 120.0) -> dict[int, dict]:
        """Polls until every tag in tags has completed; returns them by tag."""
        import time
        want = set(tags)
        got: dict[int, dict] = {}
        t_end = time.monotonic() + timeout_s
        while want - got.keys():
            if time.monotonic() > t_end:
                raise TimeoutError(f"{len(want - got.keys())} requests still pending")
            for d in self.poll(wait_us=20000):
                got[d["tag"]] = d
        return {t: got[t] for t in tags}

    def stats(self) -> dict:
        st = ServerStats()
        r = lib.xmss_b200_server_stats_get(self._h, C.byref(st))
        if r:
            raise GpuError(f"server failed: {last_error()}")
        return st.as_dict()

    def batch_trace(self, max_items: int = 4096) -> list[dict]:
        """The most recent batch records (xmss_b200_server_trace), oldest first."""
        arr = (BatchTrace * max_items)()
        n = lib.xmss_b200_server_trace(self._h, arr, max_items)
        return [arr[i].as_dict() for i in range(n)]

    def replay(self, trace: np.ndarray):
        """xmss_b200_server_replay over a TRACE_DTYPE array (pointers inside must
        stay valid).  Returns (ret int32, latency_us f64, index u64, elapsed_s)."""
        trace = np.ascontiguousarray(trace, TRACE_DTYPE)
        n = len(trace)
        ret = np.full(n, -7, np.int32)
        lat = np.zeros(n, np.float64)
        idx = np.zeros(n, np.uint64)
        el = C.c_double()
        r = lib.xmss_b200_server_replay(self._h, trace.ctypes.data, n, ret.ctypes.data, lat.ctypes.data,
                                        idx.ctypes.data, C.byref(el))
        if r:
            raise ValueError(f"server_replay returned {r}")
        return ret, lat, idx, el.value


class VerifyGraph:
    """xmss_b200_verify_graph_*: a device verify of fixed shape captured in a
    CUDA graph (device pointers as ints)."""

    def __init__(self, oid: int, mt: bool, count: int, d_sm: int, d_sm_off: int, d_smlen: int, d_pk: int, npk: int,
                 d_pk_index: int, d_status: int):
        h = C.c_void_p()
        r = _check(lib.xmss_b200_verify_graph_create(oid, int(mt), count, d_sm, d_sm_off, d_smlen, d_pk, npk,
                                                     d_pk_index, d_status, C.byref(h)), "verify_graph_create")
        if r:
            raise ValueError(f"verify_graph_create returned {r}: {last_error()}")
        self._h = h

    def launch(self, stream: int = 0) -> None:
        _check(lib.xmss_b200_verify_graph_launch(self._h, stream), "verify_graph_launch")

    def close(self) -> None:
        if self._h:
            lib.xmss_b200_verify_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


KEYGEN, SIGN, VERIFY = 1, 2, 3


class BatchGroup(C.Structure):
    """xmss_b200_batch_group: one kind and one parameter set of a mixed batch
    (d_ fields are device pointers as ints; sk / ret host buffers)."""
    _fields_ = [("kind", C.c_int), ("oid", C.c_uint32), ("mt", C.c_int), ("count", C.c_uint32),
                ("d_seeds", C.c_void_p), ("d_pk", C.c_void_p), ("d_sk", C.c_void_p), ("sk", C.c_void_p),
                ("ret", C.c_void_p), ("d_sm", C.c_void_p), ("d_sm_off", C.c_void_p), ("d_len", C.c_void_p),
                ("npk", C.c_uint32), ("d_pk_index", C.c_void_p), ("d_status", C.c_void_p)]


lib.xmss_b200_batch_create.argtypes = [C.POINTER(BatchGroup), C.c_uint32, C.POINTER(C.c_void_p)]
lib.xmss_b200_batch_create_persistent.argtypes = lib.xmss_b200_batch_create.argtypes
lib.xmss_b200_batch_launch.argtypes = [C.c_void_p, C.c_void_p]
lib.xmss_b200_batch_destroy.argtypes = [C.c_void_p]
lib.xmss_b200_batch_destroy.restype = None


class Batch:
    """xmss_b200_batch_*: keygen / sign / verify groups of any parameter sets
    captured in one CUDA graph.  groups: dicts of BatchGroup fields; a sign
    group's "sk" is a writable uint8 numpy array (count x (4 + sk_bytes)),
    advanced in place by create, and its codes land in self.ret[i]."""

    def __init__(self, groups: Sequence[dict], persistent: bool = False):
        arr = (BatchGroup * len(groups))()
        self._keep = []
        self.ret = []
        for i, g in enumerate(groups):
            g = dict(g)
            ret = None
            if g.get("kind") == SIGN:
                sk = g.pop("sk")
                assert sk.dtype == np.uint8 and sk.flags.c_contiguous and sk.flags.writeable
                ret = np.zeros(int(g["count"]), np.int32)
                g["sk"] = sk.ctypes.data
                g["ret"] = ret.ctypes.data
                self._keep += [sk, ret]
            self.ret.append(ret)
            for k, v in g.items():
                setattr(arr[i], k, v)
        h = C.c_void_p()
        create = lib.xmss_b200_batch_create_persistent if persistent else lib.xmss_b200_batch_create
        r = _check(create(arr, len(groups), C.byref(h)), "batch_create")
        if r:
            raise ValueError(f"batch_create returned {r}: {last_error()}")
        self._h = h

    def launch(self, stream: int = 0) -> int:
        """0, or -2 when a batch with sign groups is launched again."""
        return _check(lib.xmss_b200_batch_launch(self._h, stream), "batch_launch")

    def close(self) -> None:
        if self._h:
            lib.xmss_b200_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# -- launch-shape tuning ------------------------------------------------------

FAMILIES = ((XMSS_SHA2, 24), (XMSS_SHA2, 32), (XMSS_SHA2, 64), (XMSS_SHAKE128, 32), (XMSS_SHAKE256, 24),
            (XMSS_SHAKE256, 32), (XMSS_SHAKE256, 64))
TUNING_PATH = os.path.join(HERE, "tuning.json")


def tuning_get(func: int, n: int) -> dict:
    t = Tuning()
    if lib.xmss_b200_tuning_get(func, n, C.byref(t)):
        raise ValueError(f"no family ({func}, {n})")
    return t.as_dict()


def tuning_set(func: int, n: int, shape: dict) -> None:
    """Sets the knobs `shape` names; the others keep their current values."""
    cur = tuning_get(func, n)
    t = Tuning(**{k: int(shape.get(k, cur[k])) for k, _ in Tuning._fields_})
    if lib.xmss_b200_tuning_set(func, n, C.byref(t)):
        raise ValueError(f"tuning_set({func}, {n}): {last_error()}")


def autotune(oid: int, mt: bool, count: int = 4096):
    """xmss_b200_autotune: returns (chosen shape, report of every trial)."""
    import json

    best = Tuning()
    rep = C.create_string_buffer(1 << 16)
    r = _check(lib.xmss_b200_autotune(oid, int(mt), count, C.byref(best), rep, len(rep)), "autotune")
    if r:
        raise ValueError(f"autotune returned {r}: {last_error()}")
    return best.as_dict(), json.loads(rep.value.decode())


class TreeTuning(C.Structure):
    """xmss_b200_tree_tuning (include/xmss_b200.h)."""

    _fields_ = [("subtree_height", C.c_uint32), ("chains_per_warp", C.c_uint32), ("min_leaves", C.c_uint64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


lib.xmss_b200_tree_tuning_get.argtypes = [C.c_uint32, C.c_int, C.POINTER(TreeTuning)]
lib.xmss_b200_tree_tuning_set.argtypes = [C.c_uint32, C.c_int, C.POINTER(TreeTuning)]
lib.xmss_b200_autotune_tree.argtypes = [C.c_uint32, C.c_int, C.POINTER(TreeTuning), C.c_char_p, C.c_size_t]


def tree_tuning_get(oid: int, mt: bool) -> dict:
    """How the subtrees of parameter set (oid, mt) are built."""
    t = TreeTuning()
    if lib.xmss_b200_tree_tuning_get(oid, int(mt), C.byref(t)):
        raise ValueError(f"unknown parameter set ({oid:#x}, mt={mt})")
    return t.as_dict()


def tree_tuning_set(oid: int, mt: bool, subtree_height: int, min_leaves: int = 0) -> None:
    t = TreeTuning(subtree_height=subtree_height, chains_per_warp=0, min_leaves=min_leaves)
    if lib.xmss_b200_tree_tuning_set(oid, int(mt), C.byref(t)):
        raise ValueError(f"tree_tuning_set: {last_error()}")


def autotune_tree(oid: int, mt: bool):
    """xmss_b200_autotune_tree: returns (chosen shape, report of every trial)."""
    import json

    best = TreeTuning()
    rep = C.create_string_buffer(1 << 14)
    r = _check(lib.xmss_b200_autotune_tree(oid, int(mt), C.byref(best), rep, len(rep)), "autotune_tree")
    if r:
        raise ValueError(f"autotune_tree returned {r}: {last_error()}")
    return best.as_dict(), json.loads(rep.value.decode())


def save_tuning(path: str = TUNING_PATH, notes: dict | None = None, sets=()) -> None:
    """Writes the current shape of every family, and the tree shape of the
    parameter sets `sets` ((oid, mt) pairs), as a JSON table."""
    import json

    table = {"families": [{"func": f, "n": n, **tuning_get(f, n)} for f, n in FAMILIES],
             "sets": [{"oid": oid, "mt": bool(mt), **tree_tuning_get(oid, mt)} for oid, mt in sets]}
    if notes:
        table["notes"] = notes
    with open(path, "w") as fh:
        json.dump(table, fh, indent=1)


def load_tuning(path: str = TUNING_PATH) -> bool:
    """Applies a table written by save_tuning; False when there is none."""
    import json

    if not os.path.exists(path):
        return False
    table = json.load(open(path))
    for e in table["families"]:
        tuning_set(e["func"], e["n"], e)
    for e in table.get("sets", []):
        tree_tuning_set(e["oid"], e["mt"], e["subtree_height"], e["min_leaves"])
    return True


# the shapes measured on this GPU type, when a table sits next to the library
if os.environ.get("XMSS_B200_TUNING", "1") != "0":
    load_tuning(os.environ.get("XMSS_B200_TUNING_FILE", TUNING_PATH))
