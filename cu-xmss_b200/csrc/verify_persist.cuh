// Persistent verify: a whole batch of xmss(mt)_core_sign_open
// (xmss_commons.c:136-215), every layer of XMSS^MT included, in ONE launch
// fed by a device work queue.
//
// The queue is a single 64-bit ticket counter over a task sequence that is
// ordered topologically: every task depends only on tasks with smaller
// tickets.  Signatures are taken in groups of 32 (one per lane), and each
// warp pops one ticket at a time:
//
//   count    1,024 signatures: histogram of their H_msg block counts  (no deps)
//   ctx      32 keys: the PUB_SEED midstates                         (no deps)
//   prefix   bucket offsets of the histogram, longest H_msg first      (count)
//   scatter  1,024 signatures: their places in that order (perm)       (prefix)
//   hmsg     one group: H_msg + base_w (lane = signature), then the
//            group's chains bucketed longest first into its list   (scatter)
//   hpre     one group, one H node of one layer: h_pre             (ctx)
//   per layer l:
//     chain  32 list entries of one group (entry c*32 .. c*32+31)  (list of g, l)
//     ltree  one L-tree pair index of one level for the group      (chains, h_pre /
//                                                                   level before)
//     root   compute_root of the group; then the next layer's
//            chain list, or the comparison with the public root    (last level)
//
// Group g holds the signatures perm[32g .. 32g + 31]: the batch sorted by
// H_msg length, longest first, so a group's chains wait only for messages of
// about the same length.  The hmsg tickets run in that order (the long,
// serial H_msg start first); the tasks after them run in the reverse order,
// shortest H_msg first, so that the first chain tickets find their lists
// ready.  Chain tickets are taken in two bands, like the two-stream split of
// the multi-launch pipeline: the groups whose H_msg is at most short_blocks
// hash blocks, then the longer ones; inside a band they go by list position
// c, so the longest chains of every group go first.
//
// A warp waits for a task's inputs by polling a per-group counter that the
// producing tasks increment.  Since every producer holds a smaller ticket,
// and a ticket is only taken by a running warp, the smallest unfinished
// ticket never waits: the launch always completes, whatever the residency
// of its CTAs.  No CTA-wide barrier is used inside the loop.  Each wait is
// still bounded (PersistArgs::wait_ns of the global timer, 8 s unless the
// caller sets another bound); one that runs out sets an error flag, every
// warp then leaves the loop, and the last CTA to exit writes -3 into every
// status.
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

// State of one persistent launch.  Zeroed before the launch.
struct PersistArgs {
    unsigned long long* ticket;  // next ticket
    uint32_t* hdr;               // [0] error flag, [1] CTAs exited, [2] ctx tasks done, [3] count tasks
                                 // done, [4] prefix done, [5] scatter tasks done, [6] long signatures
    uint32_t* ready;             // [G*d] chain list of (group, layer) written
    uint32_t* ntot;              // [G*d] chains in that list
    uint32_t* chains_done;       // [G*d] chain tasks finished
    uint32_t* lt_done;           // [G*d*8] L-tree level tasks finished
    uint32_t* hpre_done;         // [G] h_pre tasks finished
    uint32_t* list;              // [G][32*LEN] chain items (s*LEN + chain) of the group's current layer
    uint32_t* perm;              // [count] signatures in group order
    uint32_t* sort;              // [2 * kSortBuckets] histogram, then bucket cursors
    void* ctx;                   // [npk] F::Ctx, written by the ctx tasks
    unsigned long long wait_ns;  // bound of one dependency wait (%globaltimer ns)
    uint32_t npk;
    uint32_t groups;
    uint32_t short_blocks;       // chain band boundary: H_msg hash blocks of a short group
};

// Header words of a PersistArgs state block.
constexpr uint32_t kPersistHdrWords = 8;

// Default bound of a single dependency wait (ns of %globaltimer).  Inputs of
// a task are produced by tasks already running, so a legitimate wait lasts at
// most about one H_msg: 8 s is a message of several hundred MB.
constexpr unsigned long long kPersistWaitNs = 8000000000ull;


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

// Buckets the chains of one group and layer by step count, longest first,
// into the group's list (zero-step chains go straight to the WOTS pk), then
// publishes the list.  lane: its signature s, live when it is still valid.
// cnt: 32 words of this warp's shared memory.
template <class F>
__device__ void persist_bucket(const VerifyArgs& v, const PersistArgs& q, uint32_t g, uint32_t layer, bool live,
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
    if (lane == 0) {
        uint32_t b = 0;
        for (int k = 15; k >= 1; k--) {
            const uint32_t c = cnt[k];
            cnt[16 + k] = b;
            b += c;
        }
        q.ntot[g * v.d + layer] = b;
    }
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
    persist_signal(&q.ready[g * v.d + layer]);
}

// Resident CTAs of 128 threads the register budget is set for: the
// persistent kernel holds every task's code, so without a bound the
// compiler gives the SHA-256 form 128 registers (4 CTAs per SM).  5 CTAs
// (96 registers) spill 36 bytes, 6 (80) spill 256; the SHA-512 and SHAKE
// forms spill 120-536 bytes at 3 CTAs (168 registers) and none at 2.
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

// Tasks of one persistent verify (the ticket count of its launch).
__host__ __device__ inline unsigned long long persist_verify_tasks(uint32_t count, uint32_t npk, uint32_t d,
                                                                   uint32_t th, int len)
{
    const unsigned long long G = (count + 31) / 32, K = (npk + 31) / 32, S = (count + kSortChunk - 1) / kSortChunk;
    const unsigned long long nh = (unsigned long long)len - 1 + th;
    return 2 * S + 1 + K + G + G * d * nh + (unsigned long long)d * G * (len + lt_items_total(len) + 1);
}

// F runs every task except the chains, which run FT (same family, another
// pipe mix; the key context is shared).
template <class F, class FT>
__global__ void __launch_bounds__(128, persist_min_ctas<F>()) k_verify_persist(VerifyArgs v, PersistArgs q)
{
    using Ctx = typename F::Ctx;
    using HPre = typename F::HPre;
    constexpr int LEN = F::LEN, LV = lt_levels(F::LEN), LT = lt_items_total(F::LEN);
    __shared__ uint32_t sh_cnt[4][32];
    __shared__ int sh_last;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t* cnt = sh_cnt[(threadIdx.x >> 5) & 3];
    uint32_t* err = q.hdr;
    Ctx* ctx = (Ctx*)q.ctx;
    const uint32_t G = q.groups, d = v.d, th = v.tree_height, count = v.count;
    const uint32_t nh = LEN - 1 + th;
    const unsigned long long K = (q.npk + 31) / 32;
    const unsigned long long S = (count + kSortChunk - 1) / kSortChunk;
    const unsigned long long n_hpre = (unsigned long long)G * d * nh;
    const unsigned long long per_layer = (unsigned long long)G * (LEN + LT + 1);
    const unsigned long long total = persist_verify_tasks(count, q.npk, d, th, LEN);
    uint32_t* hist = q.sort;
    uint32_t* cursor = q.sort + kSortBuckets;
    // signature of lane `lane` in group g (count: none)
    auto sig_of = [&](uint32_t g) -> uint32_t {
        const uint32_t i = g * 32 + lane;
        return i < count ? q.perm[i] : count;
    };
    // the group at position `pos` of the readiness order (shortest H_msg first)
    auto group_at = [&](uint32_t pos) -> uint32_t { return G - 1 - pos; };

    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(q.ticket, 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total || *(volatile uint32_t*)err) break;

        if (t < S) {  // -------- count: H_msg length histogram of 1,024 signatures
            for (uint32_t i = lane; i < kSortChunk; i += 32) {
                const uint32_t s = (uint32_t)t * kSortChunk + i;
                if (s < count) atomicAdd(&hist[persist_sort_bucket<F>(v, s)], 1u);
            }
            persist_signal(&q.hdr[3]);
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
            persist_signal(&q.hdr[2]);
            continue;
        }
        t -= K;
        if (t == 0) {  // -------- prefix: bucket cursors (exclusive prefix sums), long signatures
            if (!persist_wait(&q.hdr[3], (uint32_t)S, err, q.wait_ns)) break;
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
            const uint32_t cut = kSortBuckets - 1 - (q.short_blocks < kSortBuckets - 1 ? q.short_blocks : kSortBuckets - 1);
            if (lane == cut / per) {
                uint32_t c = incl - sum;
                for (uint32_t b = lane * per; b < cut; b++) c += ld_relaxed(&hist[b]);
                q.hdr[6] = c;
            }
            persist_signal(&q.hdr[4]);
            continue;
        }
        t -= 1;
        if (t < S) {  // -------- scatter: places of 1,024 signatures in group order
            if (!persist_wait(&q.hdr[4], 1u, err, q.wait_ns)) break;
            for (uint32_t i = lane; i < kSortChunk; i += 32) {
                const uint32_t s = (uint32_t)t * kSortChunk + i;
                if (s < count) q.perm[atomicAdd(&cursor[persist_sort_bucket<F>(v, s)], 1u)] = s;
            }
            persist_signal(&q.hdr[5]);
            continue;
        }
        t -= S;
        if (t < G) {  // -------- H_msg + base_w of one group (longest first), then its layer-0 list
            const uint32_t g = (uint32_t)t;
            if (!persist_wait(&q.hdr[5], (uint32_t)S, err, q.wait_ns)) break;
            const uint32_t s = sig_of(g);
            bool live = false;
            if (s < count) {
                const uint64_t smlen = v.smlen[s];
                if (!verify_input_ok(v, s)) {  // too short, or a key index outside the table
                    v.status[s] = -1;
                } else {
                    const uint8_t* sm = v.sm + v.sm_off[s];
                    const uint64_t idx = bytes_be(sm, (int)v.index_bytes);
                    uint32_t R[F::NW], root[F::NW], mh[F::NW];
                    F::load(R, sm + v.index_bytes);
                    F::load(root, v.key_root + (uint64_t)v.key[s] * v.key_stride);
                    hmsg<F>(mh, R, root, idx, sm + v.sig_bytes, smlen - v.sig_bytes);
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
            persist_bucket<F>(v, q, g, 0, live, s, cnt);
            continue;
        }
        t -= G;
        if (t < n_hpre) {  // -------- h_pre of one H node of one layer, for a group
            const uint32_t pos = (uint32_t)(t / ((unsigned long long)d * nh));
            const uint32_t k = (uint32_t)(t - (unsigned long long)pos * d * nh);
            const uint32_t g = group_at(pos);
            if (!persist_wait(&q.hdr[2], (uint32_t)K, err, q.wait_ns)) break;
            if (!persist_wait(&q.hdr[5], (uint32_t)S, err, q.wait_ns)) break;
            const uint32_t s = sig_of(g);
            if (s < count) verify_hpre_item<F>(v, ctx, (uint64_t)s * d * nh + k);
            persist_signal(&q.hpre_done[g]);
            continue;
        }
        t -= n_hpre;
        const uint32_t layer = (uint32_t)(t / per_layer);
        unsigned long long r = t - (unsigned long long)layer * per_layer;
        uint32_t leafidx;
        uint64_t tree;
        if (r < (unsigned long long)G * LEN) {  // -------- 32 chains of a group's list
            // bands: the groups of short H_msg (positions 0 .. GS-1), then the
            // long ones; inside a band c-major, so longest chains go first
            if (!persist_wait(&q.hdr[4], 1u, err, q.wait_ns)) break;
            const uint32_t GL = min(G, (ld_relaxed(&q.hdr[6]) + 31) / 32), GS = G - GL;
            uint32_t c, pos;
            if (r < (unsigned long long)GS * LEN) {
                c = (uint32_t)(r / GS);
                pos = (uint32_t)(r - (unsigned long long)c * GS);
            } else {
                const unsigned long long r2 = r - (unsigned long long)GS * LEN;
                c = (uint32_t)(r2 / GL);
                pos = GS + (uint32_t)(r2 - (unsigned long long)c * GL);
            }
            const uint32_t g = group_at(pos);
            const uint32_t gl = g * d + layer;
            if (!persist_wait(&q.ready[gl], 1u, err, q.wait_ns)) break;
            if (layer == 0 && !persist_wait(&q.hdr[2], (uint32_t)K, err, q.wait_ns)) break;
            const uint32_t e = c * 32 + lane;
            if (e < q.ntot[gl]) {
                const uint32_t item = q.list[(uint64_t)g * 32 * LEN + e];
                const uint32_t s = item / LEN, chain = item - s * LEN;
                layer_addr<F>(v.idx[s], th, layer, leafidx, tree);
                const uint32_t start = v.lens[item];
                const uint64_t wsb = (uint64_t)LEN * F::N;
                const uint8_t* sig = v.sm + v.sm_off[s] + v.index_bytes + F::N + layer * (wsb + (uint64_t)th * F::N);
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
            persist_signal(&q.chains_done[gl]);
            continue;
        }
        r -= (unsigned long long)G * LEN;
        if (r < (unsigned long long)G * LT) {  // -------- one pair index of one L-tree level
            int lev = 0;
            while (r >= (unsigned long long)G * lt_items(LEN, lev)) {
                r -= (unsigned long long)G * lt_items(LEN, lev);
                lev++;
            }
            const uint32_t items = (uint32_t)lt_items(LEN, lev);
            const uint32_t pos = (uint32_t)(r / items), p = (uint32_t)(r - (unsigned long long)pos * items);
            const uint32_t g = group_at(pos);
            const uint32_t gl = g * d + layer;
            if (lev == 0) {
                if (!persist_wait(&q.chains_done[gl], (uint32_t)LEN, err, q.wait_ns)) break;
                if (!persist_wait(&q.hpre_done[g], d * nh, err, q.wait_ns)) break;
            } else if (!persist_wait(&q.lt_done[gl * 8 + lev - 1], (uint32_t)lt_items(LEN, lev - 1), err, q.wait_ns)) {
                break;
            }
            const uint32_t s = sig_of(g);
            if (s < count && v.status[s] == 0) {
                const int cin = lt_cnt(LEN, lev);
                // levels alternate between the WOTS pk buffer and the half-size one
                const bool even = (lev & 1) == 0;
                const uint8_t* src = even ? v.wpk + (uint64_t)s * LEN * F::N : v.wpk2 + (uint64_t)s * ((LEN + 1) / 2) * F::N;
                uint8_t* out = (cin == 2) ? v.leaf + (uint64_t)s * F::N
                               : even     ? v.wpk2 + ((uint64_t)s * ((LEN + 1) / 2) + p) * F::N
                                          : v.wpk + ((uint64_t)s * LEN + p) * F::N;
                uint32_t l[F::NW], o[F::NW];
                F::load(l, src + (uint64_t)(2 * p) * F::N);
                if (2 * (int)p + 1 < cin) {
                    uint32_t rr[F::NW];
                    F::load(rr, src + (uint64_t)(2 * p + 1) * F::N);
                    const HPre& hp = ((const HPre*)v.hpre)[((uint64_t)s * d + layer) * nh + lt_base(LEN, lev) + p];
                    F::h_fin(o, hp, l, rr);
                    F::store(out, o);
                } else {
                    F::store(out, l);
                }
            }
            persist_signal(&q.lt_done[gl * 8 + lev]);
            continue;
        }
        r -= (unsigned long long)G * LT;
        {  // -------- compute_root of a group, then the next layer's list or the verdict
            const uint32_t g = group_at((uint32_t)r), gl = g * d + layer;
            if (!persist_wait(&q.lt_done[gl * 8 + LV - 1], 1u, err, q.wait_ns)) break;
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
            if (layer + 1 < d) persist_bucket<F>(v, q, g, layer + 1, next_live, s, cnt);
            continue;
        }
    }

    // The last CTA out turns a failed launch into -3 for every signature.
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        sh_last = atomicAdd(&q.hdr[1], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (sh_last) {
        __threadfence();
        if (*(volatile uint32_t*)err)
            for (uint32_t s = threadIdx.x; s < v.count; s += blockDim.x) v.status[s] = -3;
    }
}

}  // namespace xb
