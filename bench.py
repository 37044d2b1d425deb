"""Benchmark of the XMSS hot path on B200: batched XMSS-SHA2_10_256 verify.

Workload (one step): 4096 XMSS-SHA2_10_256 signed messages under 64 seeded
keys, message lengths log-uniform in 32 B..4 KB, leaf indices uniform in
[0, 1023], 10% with one random bit flipped (must reject); one verify call per
step.  Inputs are synthetic and seeded; they are produced by this library's
own batched keygen / sign (untimed) and the accept bitmap is checked.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value      verifies/s with inputs resident in HBM, CUDA events around each
           step on the launching stream, L2 flushed between steps (the input
           is 14 MB, smaller than L2), max over ranks (replicas, weak scaling)
e2e        the same through the host-buffer C-ABI (xmss_b200_sign_open_batch)
           from pinned host memory, copies included, wall clock per call
roofline   the chain kernel (the dominant kernel): algorithmic SHA-256
           compressions per launch (4 per F call, counted on the GPU) over
           its CUDA-event duration, against the measured compression rate of
           the rate probe (same SHA-256 core, all SMs busy) in the same run
secondary  XMSS-SHA2_16_256 keygen leaves/s (8 keys, 65,536 leaves each)
--impl reference   times the reference's own CPU path (oracle/_ref, compiled
           from the reference sources) on a bounded sample of the same
           workload on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "cu-xmss_b200"))

NUM_SIGS = 4096
NUM_KEYS = 64
OID = 0x01  # XMSS-SHA2_10_256
SEED = 20260303
MEASURED = os.path.join(ROOT, "MEASURED_PEAKS.json")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def make_workload(xb, rank: int = 0):
    """Seeded config: keys, signed messages (10% one-bit corrupted)."""
    rng = np.random.default_rng(SEED + rank)
    p = xb.parse_oid(OID)
    seeds = np.frombuffer(rng.bytes(NUM_KEYS * 3 * p.n), np.uint8).reshape(NUM_KEYS, 3 * p.n)
    pks, sks = xb.keypair_batch(OID, False, seeds)
    keyix = rng.integers(0, NUM_KEYS, NUM_SIGS).astype(np.uint32)
    idx = rng.integers(0, 1 << p.full_height, NUM_SIGS)
    mlen = np.exp(rng.uniform(np.log(32), np.log(4096), NUM_SIGS)).astype(np.int64)
    msgs = [rng.bytes(int(L)) for L in mlen]
    rows = np.array(sks[keyix])
    for i in range(NUM_SIGS):
        rows[i, 4:4 + p.index_bytes] = np.frombuffer(int(idx[i]).to_bytes(p.index_bytes, "big"), np.uint8)
    ret, sms = xb.sign_batch(False, rows, msgs)
    assert (ret == 0).all()
    flip = rng.choice(NUM_SIGS, NUM_SIGS // 10, replace=False)
    # Index 2^h - 1 is the reference's exhaustion case (xmss_core.c:212-231):
    # the key is wiped before signing, so that signature must reject.
    expect = np.where(idx == (1 << p.full_height) - 1, -1, 0).astype(np.int32)
    sms = [bytearray(s) for s in sms]
    for i in flip:
        pos = int(rng.integers(0, len(sms[i])))
        sms[i][pos] ^= 1 << int(rng.integers(0, 8))
        expect[i] = -1
    sms = [bytes(s) for s in sms]
    buf, off, ln = xb.pack(sms, align=16)
    return dict(p=p, pks=pks, keyix=keyix, sms=sms, buf=buf, off=off, len=ln, expect=expect,
                mean_mlen=float(mlen.mean()))


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------

class ClockSampler:
    """SM clock and clock-event reasons polled through NVML every 5 ms during
    the timed region (started before it; waits for the first sample)."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.stop = threading.Event()
        self.thread = None
        self.max_mhz = None
        self.err = None

    def _run(self):
        try:
            import pynvml as N

            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.device)
            self.max_mhz = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
            while not self.stop.is_set():
                mhz = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                try:
                    rs = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                except AttributeError:
                    rs = N.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.samples.append((float(mhz), int(rs)))
                time.sleep(0.005)
            N.nvmlShutdown()
        except Exception as ex:  # NVML missing: report unsampled
            self.err = str(ex)

    def __enter__(self):
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()
        t0 = time.time()
        while not self.samples and self.err is None and time.time() - t0 < 5:
            time.sleep(0.001)
        self.n0 = len(self.samples)
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.thread.join(timeout=5)

    def summary(self):
        s = self.samples[self.n0:] or self.samples
        if not s:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "error": self.err}
        reasons = sorted({name for _, r in s for bit, name in self.REASONS.items() if r & bit})
        return {"sm_mhz": float(np.median([m for m, _ in s])), "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(s), "source": "NVML, 5 ms"}


# ---------------------------------------------------------------------------
# replicas: every rank verifies its own batch, no data-path collective
# ---------------------------------------------------------------------------

def max_over_ranks(x: float, world: int, device) -> float:
    """The slowest rank's time (all ranks get it)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(per_rank_items: int, world: int, steps: int, seconds: float) -> float:
    """Whole-job throughput of `world` replicas (weak scaling)."""
    return per_rank_items * world * steps / seconds


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def run_ours(args, rank: int, world: int, local_rank: int):
    import torch
    import torch.distributed as dist

    import xmss_b200 as xb

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    xb.init(local_rank)
    w = make_workload(xb, rank)
    p = w["p"]
    n = p.n
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream

    # inputs resident in HBM
    d_sm = torch.from_numpy(w["buf"]).to(dev)
    d_off = torch.from_numpy(w["off"].astype(np.int64)).to(dev)
    d_len = torch.from_numpy(w["len"].astype(np.int64)).to(dev)
    d_pk = torch.from_numpy(np.ascontiguousarray(w["pks"][:, 4:])).to(dev)
    d_kix = torch.from_numpy(w["keyix"].astype(np.int32)).to(dev)
    d_status = torch.empty(NUM_SIGS, dtype=torch.int32, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=dev)  # 512 MB > 126 MB L2

    def verify_once():
        xb.sign_open_device(OID, False, NUM_SIGS, d_sm.data_ptr(), d_off.data_ptr(), d_len.data_ptr(),
                            d_pk.data_ptr(), NUM_KEYS, d_kix.data_ptr(), d_status.data_ptr(), sh)

    for _ in range(args.warmup):
        flush.zero_()
        verify_once()
    torch.cuda.synchronize()
    status = d_status.cpu().numpy()
    correct = bool((status == w["expect"]).all())
    if not correct:
        log(f"rank {rank}: accept bitmap mismatch: {(status != w['expect']).sum()} of {NUM_SIGS}")
    work = xb.last_verify_work()
    # per-verify algorithmic compressions (SHA-256 with per-key midstates)
    comp_chain = 4 * work.f_calls
    comp_total = work.hmsg_blocks + 4 * work.f_calls + 6 * work.h_calls

    # ---- timed region: value ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clocks:
        for i in range(args.steps):
            flush.zero_()
            starts[i].record(stream)
            verify_once()
            ends[i].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    t_ms = max_over_ranks(float(sum(step_ms)), world, dev)
    value = replica_rate(NUM_SIGS, world, args.steps, t_ms / 1e3)

    # ---- per-kernel timing (separate pass; profiling serialises calls) ----
    xb.profile(True)
    phases = []
    for _ in range(max(3, min(args.steps, 10))):
        flush.zero_()
        verify_once()
        phases.append(xb.phase_ms())
    xb.profile(False)
    med = {k: float(np.median([ph[k] for ph in phases])) for k in phases[0]}

    # ---- compression-rate probe (roofline denominator): the best of the
    # plain (ALU pipe) and FMA-pipe forms of the SHA-256 compression ----
    probe_blocks = 148 * 16 * 4
    iters = 2000
    sink = torch.zeros(probe_blocks * 128, dtype=torch.int32, device=dev)
    probe = {}
    for kind in (10, 11):
        xb.rate_probe(kind, probe_blocks, 50, sink.data_ptr(), sh)
        torch.cuda.synchronize()
        pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        pe0.record(stream)
        xb.rate_probe(kind, probe_blocks, iters, sink.data_ptr(), sh)
        pe1.record(stream)
        torch.cuda.synchronize()
        probe[kind] = probe_blocks * 128 * iters / (pe0.elapsed_time(pe1) / 1e3)
    probe_rate = max(probe.values())
    # latency of one dependent compression for a lone warp per SM (what the
    # serial phases, H_msg and the tree levels, are bound by)
    lat_iters = 500
    xb.rate_probe(20, 148, 10, sink.data_ptr(), sh)
    pe0.record(stream)
    xb.rate_probe(20, 148, lat_iters, sink.data_ptr(), sh)
    pe1.record(stream)
    torch.cuda.synchronize()
    lone_us = pe0.elapsed_time(pe1) * 1e3 / lat_iters

    # ---- e2e through the host-buffer C-ABI ----
    h_sm = torch.from_numpy(w["buf"]).pin_memory().numpy()
    h_off, h_len = w["off"], w["len"]
    h_pk = np.ascontiguousarray(w["pks"])
    h_kix = w["keyix"]
    for _ in range(2):
        xb.sign_open_batch(False, h_sm, h_off, h_len, h_pk, h_kix)
    e2e_t = []
    if world > 1:
        dist.barrier()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = xb.sign_open_batch(False, h_sm, h_off, h_len, h_pk, h_kix)
        e2e_t.append(time.perf_counter() - t0)
    correct = correct and bool((st == w["expect"]).all())
    e2e_s = max_over_ranks(float(sum(e2e_t)), world, dev)
    e2e_value = replica_rate(NUM_SIGS, world, args.steps, e2e_s)
    h2d = int(w["buf"].nbytes + h_off.nbytes + h_len.nbytes + NUM_KEYS * 2 * n + h_kix.nbytes)
    d2h = 4 * NUM_SIGS

    # ---- secondary: keygen leaves/s (XMSS-SHA2_16_256) ----
    sec = None
    if not args.skip_keygen:
        sec = keygen_rate(xb, torch, dev, sh)

    # ---- CPU baseline (rank 0, N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu = cpu_baseline(w, budget_s=args.cpu_seconds)

    if rank != 0:
        return None
    peaks = json.load(open(MEASURED)) if os.path.exists(MEASURED) else {}
    chain_ms = med["chains"]
    achieved = comp_chain / (chain_ms / 1e3) / 1e9
    pipeline_rate = comp_total / (t_ms / args.steps / 1e3) / 1e9 if world == 1 else None
    traffic = read_traffic()
    out = {
        "metric": "XMSS-SHA2_10_256 batched verifies/s (4096 sigs, 64 keys, mlen 32B-4KB log-uniform, 10% bit-flipped)",
        "value": value,
        "unit": "verifies/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32",
        "data": "synthetic (seeded keys and messages; signatures made by this library, accept bitmap checked)",
        "config": {"workload": "batched verify, XMSS-SHA2_10_256", "oid": OID, "signatures": NUM_SIGS,
                   "keys": NUM_KEYS, "mlen": "log-uniform 32..4096 B", "mean_mlen": w["mean_mlen"],
                   "bitflip_fraction": 0.1, "parallelism": f"replicas x{world}",
                   "l2": "flushed between steps (512 MB write; inputs 14 MB < 126 MB L2)"},
        "correct": correct,
        "e2e": {"value": e2e_value, "unit": "verifies/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "xmss_b200_sign_open_batch (host buffers, pinned)"},
        "gpu_launches": 11 * args.steps,
        "roofline": {"bound": "alu", "kernel": "k_verify_chains<Sha256N32>", "achieved": achieved,
                     "peak": probe_rate / 1e9, "unit": "Gcompr/s", "frac": achieved / (probe_rate / 1e9),
                     "traffic": traffic,
                     "peak_source": "measured in this run: rate probe, 4 x 148 x 16 CTAs of 128 threads x "
                                    f"{iters} SHA-256 compressions (same core as the kernels), best of the "
                                    "ALU-pipe and FMA-pipe forms",
                     "probe_gcompr_s": {"alu_form": probe[10] / 1e9, "fma_form": probe[11] / 1e9},
                     "lone_warp_us_per_compression": lone_us,
                     "work_per_launch": {"compressions": comp_chain, "f_calls": work.f_calls},
                     "phase_ms": med,
                     "pipeline_gcompr_s": pipeline_rate,
                     "pipeline_frac": (pipeline_rate / (probe_rate / 1e9)) if pipeline_rate else None,
                     "pipeline_compressions": comp_total,
                     "hbm_gbs_peak_measured": peaks.get("hbm_gbs")},
        "clocks": clocks.summary(),
    }
    if sec:
        out["secondary"] = sec
    if cpu:
        out["cpu_baseline"] = cpu
    return out


def keygen_rate(xb, torch, dev, sh):
    """Batched keygen of the survey's config 3: 8 XMSS-SHA2_16_256 keys and
    1 XMSS-SHA2_20_256 key from seeded seeds, in one timed region."""
    rng = np.random.default_rng(SEED + 16)
    jobs = []
    for oid, count in ((0x02, 8), (0x03, 1)):
        p = xb.parse_oid(oid)
        seeds = torch.from_numpy(np.frombuffer(rng.bytes(count * 3 * p.n), np.uint8).copy()).to(dev)
        d_pk = torch.empty(count * 2 * p.n, dtype=torch.uint8, device=dev)
        d_sk = torch.empty(count * p.sk_bytes, dtype=torch.uint8, device=dev)
        jobs.append((oid, count, p, seeds, d_pk, d_sk))

    def run():
        for oid, count, p, seeds, d_pk, d_sk in jobs:
            xb.keypair_device(oid, False, count, seeds.data_ptr(), d_pk.data_ptr(), d_sk.data_ptr(), sh)

    run()  # warm-up (scratch growth)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    leaves = sum(count << p.full_height for _, count, p, *_ in jobs)
    leaf_compr = 67 * 2 + 67 * 15 * 4 + 66 * 6  # PRF_keygen, 15 F per chain, L-tree
    comp = sum(count * ((leaf_compr << p.full_height) + 6 * ((1 << p.full_height) - 1)) for _, count, p, *_ in jobs)
    return {"metric": "keygen leaves/s: 8 x XMSS-SHA2_16_256 + 1 x XMSS-SHA2_20_256 (1,572,864 leaves)",
            "value": leaves / (ms / 1e3), "unit": "leaves/s", "ms": ms, "gcompr_s": comp / (ms / 1e3) / 1e9,
            "compressions": comp}


def read_traffic():
    """DRAM bytes per chain-kernel launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "verify_chains_sha256_4096sigs.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
# CPU reference / baseline
# ---------------------------------------------------------------------------

def _cpu_verifier():
    """xmss_sign_open of the reference build (oracle/_ref) when present, else
    the oracle's restatement of it."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ctypes as C

    from oracle import LIB_PATH, REF_PATH, build

    if os.path.exists(REF_PATH):
        fn = C.CDLL(REF_PATH).xmss_sign_open
        fn.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_ulonglong, C.c_void_p]
        return fn, "reference"
    if not os.path.exists(LIB_PATH):
        build()
    raw = C.CDLL(LIB_PATH).xo_api_sign_open
    raw.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_ulonglong, C.c_void_p, C.c_int]
    return (lambda m, mlen, sm, smlen, pk: raw(m, mlen, sm, smlen, pk, 0)), "port"


_CPU_STATE = {}


def _cpu_init(sms, pks):
    import ctypes as C

    fn, kind = _cpu_verifier()
    _CPU_STATE.update(fn=fn, sms=sms, pks=pks,
                      bufs=[(C.create_string_buffer(s, len(s)), C.create_string_buffer(len(s) + 8),
                             C.create_string_buffer(pk, len(pk))) for s, pk in zip(sms, pks)])


def _cpu_verify_range(rng_):
    import ctypes as C

    st = _CPU_STATE
    out = []
    for i in range(*rng_):
        smb, mb, pkb = st["bufs"][i]
        mlen = C.c_ulonglong()
        out.append(st["fn"](mb, C.byref(mlen), smb, len(st["sms"][i]), pkb))
    return out


def cpu_baseline(w, budget_s: float = 2.5, sample=None, pool=None):
    """Reference CPU verifies/s on all host cores over a bounded sample.

    One process per core (spawned): the reference hashes with OpenSSL's
    one-shot SHA256(), whose per-call algorithm lookup serialises threads of
    one process, so threads would not use the cores."""
    import multiprocessing as mp

    cores = os.cpu_count() or 1
    sel = range(len(w["sms"])) if sample is None else sample
    sms = [w["sms"][i] for i in sel]
    pks = [bytes(w["pks"][w["keyix"][i]]) for i in sel]
    expect = [int(w["expect"][i]) for i in sel]
    own = pool is None
    if own:
        pool = mp.get_context("spawn").Pool(cores, initializer=_cpu_init, initargs=(sms, pks))
    chunk = (len(sms) + cores - 1) // cores
    ranges = [(a, min(a + chunk, len(sms))) for a in range(0, len(sms), chunk)]
    pool.map(_cpu_verify_range, ranges)  # warm every worker
    done, ok, t0 = 0, True, time.perf_counter()
    try:
        while True:
            res = [r for part in pool.map(_cpu_verify_range, ranges) for r in part]
            ok = ok and res == expect
            done += len(sms)
            if time.perf_counter() - t0 >= budget_s:
                break
        dt = time.perf_counter() - t0
    finally:
        if own:
            pool.close()
            pool.join()
    kind = _cpu_verifier()[1]
    return {"value": done / dt, "unit": "verifies/s", "cores": cores, "kind": kind,
            "sample": f"{done} verifies ({len(sms)}-signature sample of the same workload, repeated) "
                      f"in {dt:.2f} s on {cores} processes", "correct": ok}


def run_reference(args, rank: int, world: int):
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    w = None
    try:
        import xmss_b200 as xb

        xb.init(0)
        w = make_workload(xb, 0)
    except Exception as ex:  # no GPU: build the sample with the CPU oracle
        log(f"workload via the CPU oracle ({ex})")
        w = make_workload_cpu()
    import multiprocessing as mp

    rng = np.random.default_rng(SEED + 99)
    sample = rng.choice(len(w["sms"]), min(512, len(w["sms"])), replace=False)
    sms = [w["sms"][i] for i in sample]
    pks = [bytes(w["pks"][w["keyix"][i]]) for i in sample]
    cores = os.cpu_count() or 1
    vals = []
    with mp.get_context("spawn").Pool(cores, initializer=_cpu_init, initargs=(sms, pks)) as pool:
        for _ in range(args.warmup):
            cpu_baseline(w, budget_s=0.0, sample=sample, pool=pool)
        for _ in range(args.steps):
            vals.append(cpu_baseline(w, budget_s=0.0, sample=sample, pool=pool))
    value = float(np.mean([v["value"] for v in vals]))
    cores = vals[0]["cores"]
    return {
        "metric": "XMSS-SHA2_10_256 batched verifies/s (4096 sigs, 64 keys, mlen 32B-4KB log-uniform, 10% bit-flipped)",
        "value": value, "unit": "verifies/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * len(sample) / value, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded)", "impl": "reference",
        "config": {"workload": "batched verify, XMSS-SHA2_10_256", "oid": OID, "signatures": NUM_SIGS,
                   "keys": NUM_KEYS, "mlen": "log-uniform 32..4096 B", "bitflip_fraction": 0.1,
                   "parallelism": "host threads"},
        "correct": all(v["correct"] for v in vals),
        "cpu_baseline": {"value": value, "unit": "verifies/s", "cores": cores, "kind": vals[0]["kind"],
                         "sample": f"each step verifies the same 512-signature sample of the workload on {cores} threads"},
        "e2e": {"value": value, "unit": "verifies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def make_workload_cpu(count: int = 512, keys: int = 8):
    """A sample of the same workload shape built with the CPU oracle (no-GPU
    hosts only; fewer keys so the trees build in seconds)."""
    from oracle import Oracle

    o = Oracle()
    rng = np.random.default_rng(SEED)
    p = o.params(OID)
    seeds = [rng.bytes(3 * p.n) for _ in range(keys)]
    keyix = rng.integers(0, keys, count).astype(np.uint32)
    idx = rng.integers(0, 1 << p.full_height, count)
    mlen = np.exp(rng.uniform(np.log(32), np.log(4096), count)).astype(np.int64)
    trees, pks = [], np.zeros((keys, 4 + 2 * p.n), np.uint8)
    for k, s in enumerate(seeds):
        trees.append(o.tree_nodes(p, s[:32], s[64:], 0, 0, os.cpu_count()))
        pks[k] = np.frombuffer(b"\0\0\0\x01" + trees[k][-32:] + s[64:], np.uint8)
    sms, expect = [], np.zeros(count, np.int32)
    for i in range(count):
        k = int(keyix[i])
        s = seeds[k]
        sk = int(idx[i]).to_bytes(4, "big") + s[:64] + trees[k][-32:] + s[64:]
        sm = bytearray(o.sign(p, sk, rng.bytes(int(mlen[i])), trees=trees[k])[2])
        if i % 10 == 0:
            sm[int(rng.integers(0, len(sm)))] ^= 1 << int(rng.integers(0, 8))
            expect[i] = -1
        sms.append(bytes(sm))
    return dict(p=p, pks=pks, keyix=keyix, sms=sms, expect=expect, mean_mlen=float(mlen.mean()))


# ---------------------------------------------------------------------------

MIX_SETS = (("XMSSMT-SHA2_20/2_256", 0x01, True), ("XMSSMT-SHA2_40/4_256", 0x04, True),
            ("XMSS-SHA2_10_512", 0x04, False), ("XMSS-SHAKE_10_256", 0x07, False))


def run_mix(args):
    """Config 4: per parameter set one seeded key, 2,048 signatures at
    consecutive indices over messages log-uniform in 32 B..64 KB (batched
    sign through the host C-ABI), then a batched verify of all of them."""
    import torch

    import xmss_b200 as xb

    xb.init(0)
    rng = np.random.default_rng(SEED + 4)
    out = {"workload": "mix", "sets": []}
    for name, oid, mt in MIX_SETS:
        p = xb.parse_oid(oid, mt)
        count = 2048
        # consecutive indices per key; a key of height 10 has 1,023 usable ones
        cap = min((1 << p.full_height) - 1, count)
        nkeys = -(-count // cap)
        seeds = np.frombuffer(rng.bytes(nkeys * 3 * p.n), np.uint8).reshape(nkeys, -1)
        pks, sks = xb.keypair_batch(oid, mt, seeds)
        start = 0 if cap < count else int(rng.integers(0, (1 << min(p.full_height, 40)) - count))
        mlen = np.exp(rng.uniform(np.log(32), np.log(65536), count)).astype(np.int64)
        msgs = [rng.bytes(int(L)) for L in mlen]
        kix = (np.arange(count) // cap).astype(np.uint32)
        rows = np.array(sks[kix])
        for i in range(count):
            rows[i, 4:4 + p.index_bytes] = np.frombuffer((start + i % cap).to_bytes(p.index_bytes, "big"),
                                                         np.uint8)
        xb.sign_batch(mt, rows.copy()[:64], msgs[:64])  # warm-up
        t0 = time.perf_counter()
        ret, sms = xb.sign_batch(mt, rows, msgs)
        t_sign = time.perf_counter() - t0
        buf, off, ln = xb.pack(sms, align=16)
        xb.sign_open_batch(mt, buf, off, ln, pks, kix)  # warm-up
        t0 = time.perf_counter()
        st = xb.sign_open_batch(mt, buf, off, ln, pks, kix)
        t_ver = time.perf_counter() - t0
        w = xb.last_verify_work()
        out["sets"].append({"set": name, "keys": nkeys, "signs": count, "signs_per_s": count / t_sign,
                            "verifies_per_s": count / t_ver, "sign_s": t_sign, "verify_s": t_ver,
                            "mean_mlen": float(mlen.mean()), "all_signed": bool((ret == 0).all()),
                            "all_verified": bool((st == 0).all()),
                            "verify_work": {"hmsg_blocks": w.hmsg_blocks, "f_calls": w.f_calls,
                                            "h_calls": w.h_calls}})
        log(out["sets"][-1])
    return out


def run_plain(args):
    """Config 1 and the per-call baseline: XMSS-SHA2_10_256 keypair from a
    seeded seed, then 16 x (xmss_sign, xmss_sign_open) of 32-byte messages,
    one reference-API call at a time (each sign recomputes its subtree)."""
    import xmss_b200 as xb

    xb.init(0)
    rng = np.random.default_rng(SEED + 1)
    p = xb.parse_oid(1)
    seed = rng.bytes(96)
    t0 = time.perf_counter()
    r, pk, sk = xb.xmssmt_core_seed_keypair(p, seed)
    t_kp = time.perf_counter() - t0
    pkf, skf = b"\0\0\0\x01" + pk, b"\0\0\0\x01" + sk
    xb.xmss_sign(skf, b"w" * 32)
    ts, tv = [], []
    for i in range(16):
        m = rng.bytes(32)
        t0 = time.perf_counter()
        r, skf, sm = xb.xmss_sign(skf, m)
        ts.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        rv, mo = xb.xmss_sign_open(sm, pkf)
        tv.append(time.perf_counter() - t0)
        assert r == 0 and rv == 0 and mo == m
    return {"workload": "plain", "keypair_ms": 1e3 * t_kp, "sign_ms_median": 1e3 * float(np.median(ts)),
            "verify_ms_median": 1e3 * float(np.median(tv)), "signs_per_s": 1 / float(np.median(ts)),
            "verifies_per_s": 1 / float(np.median(tv))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["verify", "mix", "plain"], default="verify",
                    help="verify: the headline line; mix / plain: the XMSS^MT + wide-hash and per-call configs")
    ap.add_argument("--skip-keygen", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=2.5)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        if args.impl == "reference":
            if rank != 0:
                return
        else:
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.workload == "mix":
        out = run_mix(args)
    elif args.workload == "plain":
        out = run_plain(args)
    else:
        out = run_ours(args, rank, world, local_rank)
    if out is not None:
        print(json.dumps(out), flush=True)
    if world > 1 and args.impl != "reference":
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
