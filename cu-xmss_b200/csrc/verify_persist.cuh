// Persistent verify: a whole batch of xmss(mt)_core_sign_open
// (xmss_commons.c:136-215), every layer of XMSS^MT included, in ONE launch
// whose warps take their work from device queues.
//
// Signatures are taken in groups of 32 (one per lane); a task is one warp's
// work on one group.  Two queues feed the warps:
//
// * A static ticket counter over the tasks whose inputs exist when the
//   launch starts, ordered so that each one depends only on smaller
//   tickets:
//     count    1,024 signatures: histogram of their H_msg block counts
//     ctx      32 keys: the PUB_SEED midstates
//     prefix   bucket cursors of the histogram, longest H_msg first   (count)
//     scatter  1,024 signatures: their places in that order (perm)   (prefix)
//     hmsg     one group: H_msg + base_w, then the group's chain list (scatter)
//     hpre     one group, one H node of one layer: h_pre              (ctx)
// * A ready queue of the tasks that depend on other tasks' results,
//   pushed by the task that completes their last input:
//     chain    32 entries of a group's chain list (layer l)   pushed by hmsg (l = 0)
//                                                             or root of l - 1
//     ltree    one pair index of one L-tree level of a group  pushed by the last chain
//                                                             task / h_pre task of the
//                                                             group, or the last task
//                                                             of the level below
//     root     compute_root of a group, then the next layer's
//              chain list (pushed as chain tasks) or the
//              comparison with the public root                pushed by the last task
//                                                             of the last L-tree level
//
// A warp takes the next static ticket while there are any, then claims the
// next ready-queue slot (one atomic add each) and waits for its entry, or
// leaves once every group has finished.  So no warp holds a task whose
// inputs are missing: the only waits are for a static ticket's smaller
// tickets (short), and a warp with nothing else to do waiting for the next
// push.  Work never stops while any
// remains: a task is pushed when its last input completes, and every task
// taken completes.  Each wait is bounded (PersistArgs::wait_ns of the
// global timer, 8 s unless the caller sets another bound; a warp that
// finds nothing to take for that long counts too); one that runs out sets
// an error flag, every warp leaves, and the last CTA to exit writes -3 into
// every status.
//
// With `sorted`, group g holds the signatures perm[32g .. 32g + 31]: the
// batch sorted by H_msg length, longest first, so a group's chains wait
// only for messages of about the same length; the hmsg tickets run longest
// first (the long, serial H_msg start first) and the hpre tickets shortest
// first.  Without it, groups are taken in batch order.
//
// Results are those of the multi-launch pipeline (same per-node hash calls;
// only the schedule differs).
#pragma once

#include "xmss_kernels.cuh"

namespace xb {

// Buckets of the H_msg length sort (block counts at or above the last one
// share it) and signatures per count / scatter task.
constexpr uint32_t kSortBuckets = 1024;
constexpr uint32_t kSortChunk = 1024;

// Header words of a persistent launch's state.
enum : uint32_t {
    kPhErr = 0,        // error flag
    kPhExited = 1,     // CTAs that have left the task loop
    kPhCtx = 2,        // ctx tasks done
    kPhCount = 3,      // count tasks done
    kPhPrefix = 4,     // prefix task done
    kPhScatter = 5,    // scatter tasks done
    kPhLong = 6,       // signatures with more than short_blocks H_msg blocks
    kPhFinished = 7,   // groups whose last layer is done
    kPhHead = 8,       // ready queue: next entry to take
    kPhTail = 9,       // ready queue: entries reserved
    kPhHmsgTicket = 10,  // next hmsg task
    kPhHmsgDone = 11,  // hmsg tasks done
    kPhHeadHi = 12,    // high-priority queue: next entry to take
    kPhTailHi = 13,    // high-priority queue: entries reserved
    kPersistHdrWords = 16
};

// State of one persistent launch.  Zeroed before the launch.
struct PersistArgs {
    unsigned long long* ticket;  // next static ticket
    uint32_t* hdr;               // [kPersistHdrWords], see above
    unsigned long long* rq;      // ready queue of chain tasks [rq_cap]: task word | kReady once written
    unsigned long long* rqh;     // high-priority ready queue of L-tree and root tasks [rqh_cap]
    uint32_t* ntot;              // [G*d] chain entries in the list of (group, layer)
    uint32_t* chains_done;       // [G*d] chain tasks finished
    uint32_t* gate;              // [G*d] inputs of L-tree level 0 complete: chains (1) and h_pre (1)
    uint32_t* lt_done;           // [G*d*8] L-tree level tasks finished
    uint32_t* hpre_done;         // [G] h_pre tasks finished
    uint32_t* list;              // [G][32*LEN] chain items (s*LEN + chain) of the group's current layer
    uint32_t* perm;              // [count] signatures in group order
    uint32_t* sort;              // [2 * kSortBuckets] histogram, then bucket cursors
    uint32_t* smctr;             // [kPersistSmSlots] CTAs arrived per SM
    void* ctx;                   // [npk] F::Ctx, written by the ctx tasks
    unsigned long long wait_ns;  // bound of one wait (%globaltimer ns)
    unsigned long long rq_cap;   // chain-queue entries
    unsigned long long rqh_cap;  // high-priority-queue entries
    uint32_t npk;
    uint32_t groups;
    uint32_t short_blocks;       // hash blocks of H_msg that count as long (hdr[kPhLong])
    uint32_t sorted;             // 1: groups sorted by H_msg length; 0: batch order
    uint32_t hmsg_sms;           // SMs 0 .. hmsg_sms-1 start with one CTA of hmsg tasks (0: none)
    unsigned long long* trace;   // optional [kTrKinds][4]: ~first start, last end, busy ns, tasks
};

// Task kinds of the optional trace; kTrIdle is a warp's wait for its next
// ready-queue entry.
enum : uint32_t {
    kTrCount, kTrCtx, kTrPrefix, kTrScatter, kTrHmsg, kTrHpre, kTrChain, kTrLtree, kTrRoot, kTrIdle, kTrKinds,
    kTrNone = 0xFFFFFFFFu
};

// Default bound of a single wait (ns of %globaltimer).  Inputs of a task are
// produced by tasks already running, so a legitimate wait lasts at most about
// one H_msg: 8 s is a message of several hundred MB.
constexpr unsigned long long kPersistWaitNs = 8000000000ull;

// SMs whose arrivals are counted (H_msg CTAs go to SMs below hmsg_sms).
constexpr uint32_t kPersistSmSlots = 256;

// L-tree shape (xmss_commons.c:16-49): level l reduces cnt(l) nodes into
// items(l) = ceil(cnt/2) (the odd node is carried up); its hashed pairs are
// h_pre nodes base(l) .. base(l) + cnt(l)/2 - 1.
__host__ __device__ constexpr int lt_cnt(int len, int lev)
{
    int c = len;
    for (int i = 0; i < lev; i++) c = (c + 1) / 2;
    return c;
}
__host__ __device__ constexpr int lt_items(int len, int lev) { return (lt_cnt(len, lev) + 1) / 2; }
__host__ __device__ constexpr int lt_base(int len, int lev)
{
    int c = len, b = 0;
    for (int i = 0; i < lev; i++) {
        b += c / 2;
        c = (c + 1) / 2;
    }
    return b;
}
__host__ __device__ constexpr int lt_levels(int len)
{
    int c = len, l = 0;
    while (c > 1) {
        c = (c + 1) / 2;
        l++;
    }
    return l;
}
__host__ __device__ constexpr int lt_items_total(int len)
{
    int s = 0;
    for (int l = 0; l < lt_levels(len); l++) s += lt_items(len, l);
    return s;
}
static_assert(lt_levels(131) <= 8 && lt_levels(67) == 7 && lt_items_total(67) == 71, "L-tree shape");

// Ready-queue entries a launch can push at most: per (group, layer) at most
// LEN chain tasks (chain queue), and every L-tree task and one root task
// (high-priority queue).
__host__ __device__ inline unsigned long long persist_rq_cap(uint32_t count, uint32_t d, int len)
{
    return (unsigned long long)((count + 31) / 32) * d * len;
}
__host__ __device__ inline unsigned long long persist_rqh_cap(uint32_t count, uint32_t d, int len)
{
    return (unsigned long long)((count + 31) / 32) * d * (lt_items_total(len) + 1);
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p)
{
    uint32_t x;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(x) : "l"(p) : "memory");
    return x;
}

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p)
{
    uint32_t x;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(x) : "l"(p) : "memory");
    return x;
}

__device__ __forceinline__ unsigned long long ld_acquire64(const unsigned long long* p)
{
    unsigned long long x;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(x) : "l"(p) : "memory");
    return x;
}

__device__ __forceinline__ unsigned long long ld_relaxed64(const unsigned long long* p)
{
    unsigned long long x;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(x) : "l"(p) : "memory");
    return x;
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Every lane polls until *c >= target.  Warp-uniform result: false when the
// wait ran out (the error flag is then set) or another warp failed.  Polls
// are relaxed loads followed by one acquire fence, so a waiting warp does not
// order its SM's L1 against the GPU on every poll.
__device__ __forceinline__ bool persist_wait(const uint32_t* c, uint32_t target, uint32_t* err,
                                             unsigned long long bound_ns)
{
    bool ok = true;
    if (ld_acquire(c) < target) {
        const unsigned long long t0 = global_ns();
        unsigned ns = 64;
        while (ld_relaxed(c) < target) {
            if (*(volatile uint32_t*)err) {
                ok = false;
                break;
            }
            if (global_ns() - t0 > bound_ns) {
                atomicExch(err, 1u);
                ok = false;
                break;
            }
            __nanosleep(ns);
            if (ns < 1024) ns *= 2;
        }
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
    }
    return __all_sync(0xffffffffu, ok);
}

// Publishes the warp's writes and bumps a task counter by one.
__device__ __forceinline__ void persist_signal(uint32_t* c)
{
    __threadfence();
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        __threadfence();
        atomicAdd(c, 1u);
    }
}

// Publishes the warp's writes and counts one finished task on c.  Warp-
// uniform: true for the warp that brings c to `total` (it sees every other
// finisher's writes and may push what depended on them).
__device__ __forceinline__ bool persist_finish(uint32_t* c, uint32_t total)
{
    __threadfence();
    __syncwarp();
    uint32_t last = 0;
    if ((threadIdx.x & 31) == 0) last = atomicAdd(c, 1u) + 1 == total;
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) __threadfence();
    return last != 0;
}

// Ready-queue task words: kind (bits 60-62), layer (52-59), L-tree level
// (48-51), group (24-47), index (0-23; the chain chunk c or the pair p);
// bit 63 marks a written entry.
enum : uint32_t { kTaskChain = 1, kTaskLtree = 2, kTaskRoot = 3 };
constexpr unsigned long long kReady = 1ull << 63;

__device__ __forceinline__ unsigned long long task_word(uint32_t kind, uint32_t layer, uint32_t lev, uint32_t g,
                                                        uint32_t i)
{
    return ((unsigned long long)kind << 60) | ((unsigned long long)layer << 52) | ((unsigned long long)lev << 48) |
           ((unsigned long long)g << 24) | i;
}

// Pushes n tasks (index 0 .. n-1 of `base`) onto the chain queue or, with
// hi, the high-priority queue (whole warp).
__device__ __forceinline__ void persist_push(const PersistArgs& q, unsigned long long base, uint32_t n, bool hi)
{
    if (!n) return;
    uint32_t first = 0;
    if ((threadIdx.x & 31) == 0) first = atomicAdd(&q.hdr[hi ? kPhTailHi : kPhTail], n);
    first = __shfl_sync(0xffffffffu, first, 0);
    unsigned long long* qe = hi ? q.rqh : q.rq;
    for (uint32_t i = threadIdx.x & 31; i < n; i += 32) {
        unsigned long long* e = qe + first + i;
        asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(e), "l"((base + i) | kReady) : "memory");
    }
}

// Every lane acquires a taken entry, so each one's loads see what the task's
// producers wrote before publishing it.
__device__ __forceinline__ void persist_acquire_entry(const unsigned long long* e)
{
    (void)ld_acquire64(e);
}

// Slot values of a warp: none claimed, and (high-priority queue) every slot
// already claimed by some warp.
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;
constexpr uint32_t kHiDone = 0xFFFFFFFEu;

// Claims a high-priority slot when the queue shows an entry nobody has
// claimed yet: one atomic add, never a retry loop (a compare-and-swap head
// serialised the claims of thousands of polling warps).  A warp that raced
// past the tail owns a slot whose entry comes later; every slot below
// rqh_cap gets exactly one entry, since each (group, layer) pushes all of its
// L-tree tasks and one root.  Whole warp.
__device__ __forceinline__ uint32_t persist_claim_hi(const PersistArgs& q)
{
    uint32_t slot = kNoSlot;
    if ((threadIdx.x & 31) == 0) {
        const uint32_t h = ld_relaxed(&q.hdr[kPhHeadHi]);
        if (h >= q.rqh_cap) {
            slot = kHiDone;
        } else if (h < ld_relaxed(&q.hdr[kPhTailHi])) {
            slot = atomicAdd(&q.hdr[kPhHeadHi], 1u);
            if (slot >= q.rqh_cap) slot = kHiDone;
        }
    }
    return __shfl_sync(0xffffffffu, slot, 0);
}

// Claims the next chain-queue slot (one atomic add, no retry; the warp then
// owns it until its entry arrives).  Whole warp.
__device__ __forceinline__ uint32_t persist_claim_lo(const PersistArgs& q)
{
    uint32_t slot = 0;
    if ((threadIdx.x & 31) == 0) slot = atomicAdd(&q.hdr[kPhHead], 1u);
    return __shfl_sync(0xffffffffu, slot, 0);
}

// Polls the warp's claimed slots a few times, the high-priority one first
// (relaxed loads with growing sleeps: an acquire per poll would order the
// SM's L1 against the GPU every time, evicting what the working warps read).
// Returns the task word and clears the slot it came from, or 0 when neither
// entry has arrived yet.  Whole warp.
__device__ __forceinline__ unsigned long long persist_poll(const PersistArgs& q, uint32_t& hi_slot,
                                                           uint32_t& lo_slot, int polls)
{
    unsigned long long w = 0;
    uint32_t from = 0;  // 1: high-priority slot, 2: chain slot
    if ((threadIdx.x & 31) == 0) {
        // a chain slot beyond the queue never gets an entry: the warp only
        // sleeps (and comes back for high-priority tasks, or to leave)
        unsigned ns = 128;
        for (int i = 0; i < polls; i++) {
            if (hi_slot < kHiDone && ((w = ld_relaxed64(q.rqh + hi_slot)) & kReady)) {
                from = 1;
                break;
            }
            if (lo_slot != kNoSlot && lo_slot < q.rq_cap && ((w = ld_relaxed64(q.rq + lo_slot)) & kReady)) {
                from = 2;
                break;
            }
            w = 0;
            if (i + 1 < polls) {
                __nanosleep(ns);
                ns *= 2;
            }
        }
    }
    w = __shfl_sync(0xffffffffu, w, 0);
    from = __shfl_sync(0xffffffffu, from, 0);
    if (from == 1) {
        persist_acquire_entry(q.rqh + hi_slot);
        hi_slot = kNoSlot;
    } else if (from == 2) {
        persist_acquire_entry(q.rq + lo_slot);
        lo_slot = kNoSlot;
    }
    return w;
}

// Buckets the chains of one group and layer by step count, longest first,
// into the group's list (zero-step chains go straight to the WOTS pk).
// lane: its signature s, live when it is still valid.  cnt: 32 words of
// this warp's shared memory.  Returns the chain entries (warp-uniform).
template <class F>
__device__ uint32_t persist_bucket(const VerifyArgs& v, const PersistArgs& q, uint32_t g, uint32_t layer, bool live,
                                   uint32_t s, uint32_t* cnt)
{
    const uint32_t lane = threadIdx.x & 31;
    if (lane < 16) cnt[lane] = 0;
    __syncwarp();
    const uint8_t* lens = v.lens + (uint64_t)s * F::LEN;
    uint32_t steps_sum = 0;
    if (live) {
        const uint32_t th = v.tree_height;
        const uint64_t wsb = (uint64_t)F::LEN * F::N;
        const uint8_t* sig = v.sm + v.sm_off[s] + v.index_bytes + F::N + layer * (wsb + (uint64_t)th * F::N);
#pragma unroll 1
        for (int i = 0; i < F::LEN; i++) {
            const uint32_t st = 15 - lens[i];
            steps_sum += st;
            if (st) {
                atomicAdd(&cnt[st], 1u);
            } else {
                uint32_t x[F::NW];
                F::load(x, sig + (uint64_t)i * F::N);
                F::store(v.wpk + ((uint64_t)s * F::LEN + i) * F::N, x);
            }
        }
    }
    __syncwarp();
    uint32_t b = 0;
    if (lane == 0) {
        for (int k = 15; k >= 1; k--) {
            const uint32_t c = cnt[k];
            cnt[16 + k] = b;
            b += c;
        }
        q.ntot[g * v.d + layer] = b;
    }
    b = __shfl_sync(0xffffffffu, b, 0);
    __syncwarp();
    if (live) {
        uint32_t* list = q.list + (uint64_t)g * 32 * F::LEN;
#pragma unroll 1
        for (int i = 0; i < F::LEN; i++) {
            const uint32_t st = 15 - lens[i];
            if (st) list[atomicAdd(&cnt[16 + st], 1u)] = s * F::LEN + i;
        }
    }
    const uint32_t tot = __reduce_add_sync(0xffffffffu, steps_sum);
    if (lane == 0 && v.work && tot) atomicAdd(&v.work[1], (unsigned long long)tot);
    __threadfence();
    __syncwarp();
    return b;
}

// Resident CTAs of 128 threads the register budget is set for: the
// persistent kernel holds every task's code, so without a bound the
// compiler gives the SHA-256 form 128 registers (4 CTAs per SM).  5 CTAs
// (96 registers) spill about 36 bytes, 6 (80) 300, 8 (64) 780; the SHA-512
// and SHAKE forms spill 120-536 bytes at 3 CTAs (168 registers) and none at
// 2.
template <class F>
constexpr int persist_min_ctas()
{
    return HMsgKind<F>::v == 0 ? 5 : 2;
}

// Sort bucket of a signature: longer H_msg first; signatures that are
// rejected before H_msg (too short) last.
template <class F>
__device__ __forceinline__ uint32_t persist_sort_bucket(const VerifyArgs& v, uint32_t s)
{
    const uint64_t smlen = v.smlen[s];
    if (smlen < v.sig_bytes) return kSortBuckets - 1;
    const unsigned long long b = hmsg_blocks<F>(smlen - v.sig_bytes);
    return kSortBuckets - 1 - (uint32_t)(b < kSortBuckets - 1 ? b : kSortBuckets - 1);
}

// Static tickets of one persistent verify.
__host__ __device__ inline unsigned long long persist_static_tasks(uint32_t count, uint32_t npk, uint32_t d,
                                                                   uint32_t th, int len)
{
    const unsigned long long G = (count + 31) / 32, K = (npk + 31) / 32, S = (count + kSortChunk - 1) / kSortChunk;
    const unsigned long long nh = (unsigned long long)len - 1 + th;
    return 2 * S + 1 + K + G * d * nh;
}

// F runs every task except the chains, which run FT (same family, another
// pipe mix; the key context is shared).  EXTRA CTAs per SM beyond
// persist_min_ctas trade spills for occupancy (a tuning knob,
// Tuning::persist_extra_ctas).
template <class F, class FT, int EXTRA = 0>
__global__ void __launch_bounds__(128, persist_min_ctas<F>() + EXTRA) k_verify_persist(VerifyArgs v, PersistArgs q)
{
    using Ctx = typename F::Ctx;
    using HPre = typename F::HPre;
    constexpr int LEN = F::LEN, LV = lt_levels(F::LEN);
    __shared__ uint32_t sh_cnt[4][32];
    __shared__ int sh_last;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t* cnt = sh_cnt[(threadIdx.x >> 5) & 3];
    uint32_t* err = q.hdr + kPhErr;
    Ctx* ctx = (Ctx*)q.ctx;
    const uint32_t G = q.groups, d = v.d, th = v.tree_height, count = v.count;
    const uint32_t nh = LEN - 1 + th;
    const unsigned long long K = (q.npk + 31) / 32;
    const unsigned long long S = (count + kSortChunk - 1) / kSortChunk;
    const unsigned long long n_hpre = (unsigned long long)G * d * nh;
    const unsigned long long total_static = persist_static_tasks(count, q.npk, d, th, LEN);
    uint32_t* hist = q.sort;
    uint32_t* cursor = q.sort + kSortBuckets;
    // signature of lane `lane` in group g (count: none)
    auto sig_of = [&](uint32_t g) -> uint32_t {
        const uint32_t i = g * 32 + lane;
        return i < count ? (q.sorted ? q.perm[i] : i) : count;
    };
    // the group at position `pos` of the readiness order (shortest H_msg first)
    auto group_at = [&](uint32_t pos) -> uint32_t { return q.sorted ? G - 1 - pos : pos; };
    // the list of (g, layer) is written: push its chain tasks, or, with no
    // chain to run, count the chains of (g, layer) complete at once
    auto push_chains = [&](uint32_t g, uint32_t layer, uint32_t ntot) -> bool {
        const uint32_t nct = (ntot + 31) / 32;
        if (nct) {
            persist_push(q, task_word(kTaskChain, layer, 0, g, 0), nct, false);
            return false;
        }
        return true;  // caller runs the gate
    };
    // one of the two inputs of L-tree level 0 of (g, layer) is complete: the
    // second pushes the level's tasks
    auto gate = [&](uint32_t g, uint32_t layer) {
        uint32_t second = 0;
        if (lane == 0) second = atomicAdd(&q.gate[g * d + layer], 1u) == 1;
        second = __shfl_sync(0xffffffffu, second, 0);
        if (second) {
            __threadfence();
            persist_push(q, task_word(kTaskLtree, layer, 0, g, 0), (uint32_t)lt_items(LEN, 0), true);
        }
    };

    // optional trace: the kind and start of the warp's current task, recorded
    // when the next one begins (every task ends at the top of the loop)
    uint32_t tr_kind = kTrNone;
    unsigned long long tr_t0 = 0;
    auto tr_end = [&]() {
        if (q.trace && tr_kind != kTrNone && lane == 0) {
            const unsigned long long t1 = global_ns();
            unsigned long long* r = q.trace + 4 * tr_kind;
            atomicMax(r, ~tr_t0);
            atomicMax(r + 1, t1);
            atomicAdd(r + 2, t1 - tr_t0);
            atomicAdd(r + 3, 1ull);
        }
        tr_kind = kTrNone;
    };
    auto tr_begin = [&](uint32_t k) {
        if (q.trace) {
            tr_kind = k;
            tr_t0 = global_ns();
        }
    };

    // H_msg + base_w of group g (longest first when sorted), then its
    // layer-0 chain tasks; false when a wait ran out
    auto run_hmsg = [&](uint32_t g) -> bool {
        if (!persist_wait(&q.hdr[kPhScatter], (uint32_t)S, err, q.wait_ns)) return false;
        // the chain tasks read the key contexts
        if (!persist_wait(&q.hdr[kPhCtx], (uint32_t)K, err, q.wait_ns)) return false;
        const uint32_t s = sig_of(g);
        bool live = false;
        if (s < count) {
            const uint64_t smlen = v.smlen[s];
            if (!verify_input_ok(v, s)) {  // too short, or a key index outside the table
                v.status[s] = -1;
            } else {
                const uint8_t* sm = v.sm + v.sm_off[s];
                const uint64_t idx = bytes_be(sm, (int)v.index_bytes);
                uint32_t mh[F::NW];
                if constexpr (std::is_same<typename F::Ctx, Sha256N32Ctx>::value) {
                    // the register-lean form keeps the kernel at the chains' register count
                    hmsg_sha256_n32_lean(mh, sm + v.index_bytes, v.key_root + (uint64_t)v.key[s] * v.key_stride,
                                         idx, sm + v.sig_bytes, smlen - v.sig_bytes);
                } else {
                    uint32_t R[F::NW], root[F::NW];
                    F::load(R, sm + v.index_bytes);
                    F::load(root, v.key_root + (uint64_t)v.key[s] * v.key_stride);
                    hmsg<F>(mh, R, root, idx, sm + v.sig_bytes, smlen - v.sig_bytes);
                }
                F::store(v.node + (uint64_t)s * F::N, mh);
                chain_lengths<F>(v.lens + (uint64_t)s * F::LEN, mh);
                v.idx[s] = idx;
                v.status[s] = 0;
                live = true;
                if (v.work) {
                    atomicAdd(&v.work[0], hmsg_blocks<F>(smlen - v.sig_bytes));
                    atomicAdd(&v.work[2], (unsigned long long)nh * d);
                }
            }
        }
        const uint32_t ntot = persist_bucket<F>(v, q, g, 0, live, s, cnt);
        if (push_chains(g, 0, ntot)) gate(g, 0);
        persist_signal(&q.hdr[kPhHmsgDone]);
        return true;
    };

    // Role of this CTA: on the first hmsg_sms SMs the first CTA to arrive runs
    // hmsg tasks first (one warp per SM sub-partition, so each serial H_msg
    // gets most of its sub-partition's issue slots) and the other CTAs there
    // wait until every hmsg task is done; all others start with the static
    // tickets.  Every warp also takes hmsg tickets once its static tickets run
    // out, so the launch never depends on where its CTAs land.
    __shared__ uint32_t sh_role;
    if (threadIdx.x == 0) {
        uint32_t role = 0;
        if (q.hmsg_sms) {
            uint32_t smid;
            asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
            if (smid < q.hmsg_sms && smid < kPersistSmSlots) role = atomicAdd(&q.smctr[smid], 1u) == 0 ? 1 : 2;
        }
        sh_role = role;
    }
    __syncthreads();
    bool run = true;
    if (sh_role == 1) {
        for (;;) {
            unsigned long long t = 0;
            if (lane == 0) t = atomicAdd(&q.hdr[kPhHmsgTicket], 1u);
            t = __shfl_sync(0xffffffffu, t, 0);
            if (t >= G) break;
            tr_begin(kTrHmsg);
            if (!run_hmsg((uint32_t)t)) {
                run = false;
                break;
            }
            tr_end();
        }
    } else if (sh_role == 2) {
        run = persist_wait(&q.hdr[kPhHmsgDone], G, err, q.wait_ns);
    }

    bool static_left = true, hmsg_left = true;
    uint32_t lo_slot = kNoSlot;  // chain-queue slot this warp has claimed
    uint32_t hi_slot = kNoSlot;  // high-priority slot this warp has claimed (kHiDone: none left)
    unsigned long long idle_since = 0;
    for (; run;) {
        tr_end();
        // decisions are made by lane 0 and broadcast: the warp stays converged
        if (__shfl_sync(0xffffffffu, *(volatile uint32_t*)err, 0)) break;
        // ---------------- static tickets first ----------------
        if (static_left) {
            unsigned long long t = 0;
            if (lane == 0) t = atomicAdd(q.ticket, 1ull);
            t = __shfl_sync(0xffffffffu, t, 0);
            if (t >= total_static) {
                static_left = false;
                continue;
            }
            tr_begin(t < S ? kTrCount : t < S + K ? kTrCtx : t < S + K + 1 ? kTrPrefix
                     : t < 2 * S + K + 1 ? kTrScatter : kTrHpre);
            if (t < S) {  // -------- count: H_msg length histogram of 1,024 signatures
                for (uint32_t i = lane; q.sorted && i < kSortChunk; i += 32) {
                    const uint32_t s = (uint32_t)t * kSortChunk + i;
                    if (s < count) atomicAdd(&hist[persist_sort_bucket<F>(v, s)], 1u);
                }
                persist_signal(&q.hdr[kPhCount]);
                continue;
            }
            t -= S;
            if (t < K) {  // -------- ctx: 32 keys
                const uint32_t k = (uint32_t)t * 32 + lane;
                if (k < q.npk) {
                    Ctx c;
                    F::make_ctx(c, v.key_root + (uint64_t)k * v.key_stride + F::N, nullptr, nullptr);
                    ctx[k] = c;
                }
                persist_signal(&q.hdr[kPhCtx]);
                continue;
            }
            t -= K;
            if (t == 0) {  // -------- prefix: bucket cursors (exclusive prefix sums), long signatures
                if (!persist_wait(&q.hdr[kPhCount], (uint32_t)S, err, q.wait_ns)) break;
                constexpr uint32_t per = kSortBuckets / 32;
                uint32_t sum = 0;
                for (uint32_t j = 0; j < per; j++) sum += ld_relaxed(&hist[lane * per + j]);
                uint32_t incl = sum;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                    if ((int)lane >= o) incl += y;
                }
                uint32_t run = incl - sum;
                for (uint32_t j = 0; j < per; j++) {
                    const uint32_t b = lane * per + j;
                    cursor[b] = run;
                    run += ld_relaxed(&hist[b]);
                }
                __syncwarp();
                // signatures with more than short_blocks H_msg blocks come before
                // bucket kSortBuckets - 1 - short_blocks
                const uint32_t cut =
                    kSortBuckets - 1 - (q.short_blocks < kSortBuckets - 1 ? q.short_blocks : kSortBuckets - 1);
                if (lane == cut / per) {
                    uint32_t c = incl - sum;
                    for (uint32_t b = lane * per; b < cut; b++) c += ld_relaxed(&hist[b]);
                    q.hdr[kPhLong] = c;
                }
                persist_signal(&q.hdr[kPhPrefix]);
                continue;
            }
            t -= 1;
            if (t < S) {  // -------- scatter: places of 1,024 signatures in group order
                if (!persist_wait(&q.hdr[kPhPrefix], 1u, err, q.wait_ns)) break;
                for (uint32_t i = lane; q.sorted && i < kSortChunk; i += 32) {
                    const uint32_t s = (uint32_t)t * kSortChunk + i;
                    if (s < count) q.perm[atomicAdd(&cursor[persist_sort_bucket<F>(v, s)], 1u)] = s;
                }
                persist_signal(&q.hdr[kPhScatter]);
                continue;
            }
            t -= S;
            if (t < n_hpre) {  // -------- h_pre of one H node of one layer, for a group
                const uint32_t pos = (uint32_t)(t / ((unsigned long long)d * nh));
                const uint32_t k = (uint32_t)(t - (unsigned long long)pos * d * nh);
                const uint32_t g = group_at(pos);
                if (!persist_wait(&q.hdr[kPhCtx], (uint32_t)K, err, q.wait_ns)) break;
                if (!persist_wait(&q.hdr[kPhScatter], (uint32_t)S, err, q.wait_ns)) break;
                const uint32_t s = sig_of(g);
                if (s < count) verify_hpre_item<F>(v, ctx, (uint64_t)s * d * nh + k);
                if (persist_finish(&q.hpre_done[g], d * nh))
                    for (uint32_t layer = 0; layer < d; layer++) gate(g, layer);
                continue;
            }
            continue;  // not reached: t < total_static
        }
        // ---------------- then the next ready slot (or leave) ----------------
        // ---------------- high-priority tasks first: L-tree levels and roots ----------------
        if (hi_slot == kNoSlot) hi_slot = persist_claim_hi(q);
        uint32_t no_lo = kNoSlot;
        unsigned long long w = hi_slot < kHiDone ? persist_poll(q, hi_slot, no_lo, 1) : 0;
        if (!w) {
            // ---------------- then hmsg tickets no H_msg CTA took ----------------
            if (hmsg_left) {
                unsigned long long t = 0;
                if (lane == 0) t = atomicAdd(&q.hdr[kPhHmsgTicket], 1u);
                t = __shfl_sync(0xffffffffu, t, 0);
                if (t < G) {
                    tr_begin(kTrHmsg);
                    if (!run_hmsg((uint32_t)t)) break;
                    continue;
                }
                hmsg_left = false;
            }
            // ---------------- then the warp's chain slot ----------------
            if (lo_slot == kNoSlot) lo_slot = persist_claim_lo(q);
            tr_begin(kTrIdle);
            w = persist_poll(q, hi_slot, lo_slot, 6);
            tr_end();
            if (!w) {
                // nothing yet: leave when every group is done, fail when idle too long
                uint32_t stop = 0;
                if (lane == 0) {
                    const unsigned long long now = global_ns();
                    if (ld_relaxed(&q.hdr[kPhFinished]) >= G) {
                        stop = 1;
                    } else if (!idle_since) {
                        idle_since = now;
                    } else if (now - idle_since > q.wait_ns) {
                        atomicExch(err, 1u);
                        stop = 1;
                    }
                }
                if (__shfl_sync(0xffffffffu, stop, 0)) break;
                continue;
            }
        }
        idle_since = 0;
        {
            const uint32_t kind = (uint32_t)(w >> 60) & 7, layer = (uint32_t)(w >> 52) & 0xFF;
            tr_begin(kind == kTaskChain ? kTrChain : kind == kTaskLtree ? kTrLtree : kTrRoot);
            const uint32_t lev = (uint32_t)(w >> 48) & 0xF, g = (uint32_t)(w >> 24) & 0xFFFFFF;
            const uint32_t idx = (uint32_t)w & 0xFFFFFF;
            const uint32_t gl = g * d + layer;
            uint32_t leafidx;
            uint64_t tree;
            if (kind == kTaskChain) {  // -------- 32 entries of the chain list of (g, layer)
                const uint32_t ntot = q.ntot[gl];
                const uint32_t e = idx * 32 + lane;
                if (e < ntot) {
                    const uint32_t item = q.list[(uint64_t)g * 32 * LEN + e];
                    const uint32_t s = item / LEN, chain = item - s * LEN;
                    layer_addr<F>(v.idx[s], th, layer, leafidx, tree);
                    const uint32_t start = v.lens[item];
                    const uint64_t wsb = (uint64_t)LEN * F::N;
                    const uint8_t* sig =
                        v.sm + v.sm_off[s] + v.index_bytes + F::N + layer * (wsb + (uint64_t)th * F::N);
                    uint32_t x[F::NW], a[8];
                    F::load(x, sig + (uint64_t)chain * F::N);
                    set_addr(a, layer, tree, ADDR_OTS, leafidx, chain, 0);
                    // the key context in registers: ctx is written by this launch, so
                    // the chain loop cannot read it through the read-only path, and
                    // re-reading its midstate from L1 / L2 on every F call made a
                    // lone chain warp ~3x slower than in k_verify_chains
                    const typename FT::Ctx kc = ((const typename FT::Ctx*)ctx)[v.key[s]];
                    run_chain<FT>(x, kc, a, start, 15 - start, false);
                    F::store(v.wpk + (uint64_t)item * F::N, x);
                }
                if (persist_finish(&q.chains_done[gl], (ntot + 31) / 32)) gate(g, layer);
                continue;
            }
            if (kind == kTaskLtree) {  // -------- one pair index of one L-tree level
                const uint32_t p = idx;
                const uint32_t s = sig_of(g);
                if (s < count && v.status[s] == 0) {
                    const int cin = lt_cnt(LEN, (int)lev);
                    // levels alternate between the WOTS pk buffer and the half-size one
                    const bool even = (lev & 1) == 0;
                    const uint8_t* src =
                        even ? v.wpk + (uint64_t)s * LEN * F::N : v.wpk2 + (uint64_t)s * ((LEN + 1) / 2) * F::N;
                    uint8_t* out = (cin == 2) ? v.leaf + (uint64_t)s * F::N
                                   : even     ? v.wpk2 + ((uint64_t)s * ((LEN + 1) / 2) + p) * F::N
                                              : v.wpk + ((uint64_t)s * LEN + p) * F::N;
                    uint32_t l[F::NW], o[F::NW];
                    F::load(l, src + (uint64_t)(2 * p) * F::N);
                    if (2 * (int)p + 1 < cin) {
                        uint32_t rr[F::NW];
                        F::load(rr, src + (uint64_t)(2 * p + 1) * F::N);
                        const HPre& hp =
                            ((const HPre*)v.hpre)[((uint64_t)s * d + layer) * nh + lt_base(LEN, (int)lev) + p];
                        F::h_fin(o, hp, l, rr);
                        F::store(out, o);
                    } else {
                        F::store(out, l);
                    }
                }
                if (persist_finish(&q.lt_done[gl * 8 + lev], (uint32_t)lt_items(LEN, (int)lev))) {
                    if ((int)lev + 1 < LV)
                        persist_push(q, task_word(kTaskLtree, layer, lev + 1, g, 0), (uint32_t)lt_items(LEN, lev + 1),
                                     true);
                    else
                        persist_push(q, task_word(kTaskRoot, layer, 0, g, 0), 1, true);
                }
                continue;
            }
            {  // -------- compute_root of (g, layer), then the next layer's list or the verdict
                const uint32_t s = sig_of(g);
                const bool live = s < count && v.status[s] == 0;
                bool next_live = false;
                if (live) {
                    layer_addr<F>(v.idx[s], th, layer, leafidx, tree);
                    const uint64_t wsb = (uint64_t)LEN * F::N;
                    const uint8_t* auth =
                        v.sm + v.sm_off[s] + v.index_bytes + F::N + layer * (wsb + (uint64_t)th * F::N) + wsb;
                    const HPre* hp = (const HPre*)v.hpre + ((uint64_t)s * d + layer) * nh + (LEN - 1);
                    uint32_t cur[F::NW], sib[F::NW];
                    F::load(cur, v.leaf + (uint64_t)s * F::N);
#pragma unroll 1
                    for (uint32_t i = 0; i < th; i++) {
                        F::load(sib, auth + (uint64_t)i * F::N);
                        // the node goes right when its index is odd (xmss_commons.c:61-69)
                        const bool odd = leafidx & 1;
                        uint32_t l[F::NW], rr[F::NW];
#pragma unroll
                        for (int k = 0; k < F::NW; k++) {
                            l[k] = odd ? sib[k] : cur[k];
                            rr[k] = odd ? cur[k] : sib[k];
                        }
                        F::h_fin(cur, hp[i], l, rr);
                        leafidx >>= 1;
                    }
                    if (layer + 1 < d) {
                        F::store(v.node + (uint64_t)s * F::N, cur);
                        chain_lengths<F>(v.lens + (uint64_t)s * F::LEN, cur);
                        next_live = true;
                    } else {
                        uint32_t pr[F::NW];
                        F::load(pr, v.key_root + (uint64_t)v.key[s] * v.key_stride);
                        uint32_t diff = 0;
#pragma unroll
                        for (int i = 0; i < F::NW; i++) diff |= pr[i] ^ cur[i];
                        v.status[s] = diff ? -1 : 0;
                    }
                }
                if (layer + 1 < d) {
                    const uint32_t ntot = persist_bucket<F>(v, q, g, layer + 1, next_live, s, cnt);
                    if (push_chains(g, layer + 1, ntot)) gate(g, layer + 1);
                } else {
                    persist_signal(&q.hdr[kPhFinished]);
                }
                continue;
            }
        }
    }

    // The last CTA out turns a failed launch into -3 for every signature.
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        sh_last = atomicAdd(&q.hdr[kPhExited], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (sh_last) {
        __threadfence();
        if (*(volatile uint32_t*)err)
            for (uint32_t s = threadIdx.x; s < v.count; s += blockDim.x) v.status[s] = -3;
    }
}

}  // namespace xb
