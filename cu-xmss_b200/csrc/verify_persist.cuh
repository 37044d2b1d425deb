// Persistent verify: a whole batch of xmss(mt)_core_sign_open
// (xmss_commons.c:136-215), every layer of XMSS^MT included, in ONE launch
// fed by a device work queue.
//
// The queue is a single 64-bit ticket counter over a task sequence that is
// ordered topologically: every task depends only on tasks with smaller
// tickets.  Signatures are taken in groups of 32 (one per lane), and each
// warp pops one ticket at a time:
//
//   ctx      32 keys: the PUB_SEED midstates                       (no deps)
//   hmsg     one group: H_msg + base_w (lane = signature), then the
//            group's chains bucketed longest first into its list   (no deps)
//   hpre     one group, one H node of one layer: h_pre             (ctx)
//   per layer l:
//     chain  32 list entries of one group (entry c*32 .. c*32+31),
//            tickets ordered by c so the longest chains go first  (list of g, l)
//     ltree  one L-tree pair index of one level for the group      (chains, h_pre /
//                                                                   level before)
//     root   compute_root of the group; then the next layer's
//            chain list, or the comparison with the public root    (last level)
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

#include "family_ops.h"
#include "xmss_kernels.cuh"

namespace xb {

// State of one persistent launch.  Zeroed before the launch.
struct PersistArgs {
    unsigned long long* ticket;  // next ticket
    uint32_t* hdr;               // [0] error flag, [1] CTAs exited, [2] ctx tasks done
    uint32_t* ready;             // [G*d] chain list of (group, layer) written
    uint32_t* ntot;              // [G*d] chains in that list
    uint32_t* chains_done;       // [G*d] chain tasks finished
    uint32_t* lt_done;           // [G*d*8] L-tree level tasks finished
    uint32_t* hpre_done;         // [G] h_pre tasks finished
    uint32_t* list;              // [G][32*LEN] chain items (s*LEN + chain) of the group's current layer
    void* ctx;                   // [npk] F::Ctx, written by the ctx tasks
    unsigned long long wait_ns;  // bound of one dependency wait (%globaltimer ns)
    uint32_t npk;
    uint32_t groups;
};

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

// Tickets of one batch: key contexts, H_msg groups, h_pre items, then per
// layer the chain, L-tree and root tasks.
__host__ __device__ inline unsigned long long persist_total(int len, uint32_t groups, uint32_t npk, uint32_t d,
                                                            uint32_t th)
{
    const unsigned long long G = groups, K = (npk + 31) / 32;
    const unsigned long long n_hpre = G * d * (len - 1 + th);
    return K + G + n_hpre + G * (len + lt_items_total(len) + 1) * d;
}
template <class F>
__device__ __forceinline__ unsigned long long persist_tickets(const VerifyArgs& v, const PersistArgs& q)
{
    return persist_total(F::LEN, q.groups, q.npk, v.d, v.tree_height);
}

// Runs ticket t of one batch (whole warp).  F runs every task except the
// chains, which run FT (same family, another pipe mix; the key context is
// shared).  cnt: 32 words of this warp's shared memory.  False when a
// dependency wait ran out or the batch failed.
template <class F, class FT>
__device__ __forceinline__ bool persist_step(const VerifyArgs& v, const PersistArgs& q, unsigned long long t,
                                             uint32_t* cnt)
{
    using Ctx = typename F::Ctx;
    using HPre = typename F::HPre;
    constexpr int LEN = F::LEN, LV = lt_levels(F::LEN), LT = lt_items_total(F::LEN);
    const uint32_t lane = threadIdx.x & 31;
    uint32_t* err = q.hdr;
    Ctx* ctx = (Ctx*)q.ctx;
    const uint32_t G = q.groups, d = v.d, th = v.tree_height;
    const uint32_t nh = LEN - 1 + th;
    const unsigned long long K = (q.npk + 31) / 32;
    const unsigned long long n_hpre = (unsigned long long)G * d * nh;
    const unsigned long long per_layer = (unsigned long long)G * (LEN + LT + 1);

    if (t < K) {  // -------- ctx: 32 keys
        const uint32_t k = (uint32_t)t * 32 + lane;
        if (k < q.npk) {
            Ctx c;
            F::make_ctx(c, v.key_root + (uint64_t)k * v.key_stride + F::N, nullptr, nullptr);
            ctx[k] = c;
        }
        persist_signal(&q.hdr[2]);
        return true;
    }
    t -= K;
    if (t < G) {  // -------- H_msg + base_w of one group, then its layer-0 list
        const uint32_t g = (uint32_t)t, s = g * 32 + lane;
        bool live = false;
        if (s < v.count) {
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
        return true;
    }
    t -= G;
    if (t < n_hpre) {  // -------- h_pre of one H node of one layer, for a group
        const uint32_t g = (uint32_t)(t / ((unsigned long long)d * nh));
        const uint32_t k = (uint32_t)(t - (unsigned long long)g * d * nh);
        if (!persist_wait(&q.hdr[2], (uint32_t)K, err, q.wait_ns)) return false;
        const uint32_t s = g * 32 + lane;
        if (s < v.count) verify_hpre_item<F>(v, ctx, (uint64_t)s * d * nh + k);
        persist_signal(&q.hpre_done[g]);
        return true;
    }
    t -= n_hpre;
    const uint32_t layer = (uint32_t)(t / per_layer);
    unsigned long long r = t - (unsigned long long)layer * per_layer;
    uint32_t leafidx;
    uint64_t tree;
    if (r < (unsigned long long)G * LEN) {  // -------- 32 chains of a group's list
        const uint32_t c = (uint32_t)(r / G), g = (uint32_t)(r - (unsigned long long)c * G);
        const uint32_t gl = g * d + layer;
        if (!persist_wait(&q.ready[gl], 1u, err, q.wait_ns)) return false;
        if (layer == 0 && !persist_wait(&q.hdr[2], (uint32_t)K, err, q.wait_ns)) return false;
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
        return true;
    }
    r -= (unsigned long long)G * LEN;
    if (r < (unsigned long long)G * LT) {  // -------- one pair index of one L-tree level
        int lev = 0;
        while (r >= (unsigned long long)G * lt_items(LEN, lev)) {
            r -= (unsigned long long)G * lt_items(LEN, lev);
            lev++;
        }
        const uint32_t items = (uint32_t)lt_items(LEN, lev);
        const uint32_t g = (uint32_t)(r / items), p = (uint32_t)(r - (unsigned long long)g * items);
        const uint32_t gl = g * d + layer;
        if (lev == 0) {
            if (!persist_wait(&q.chains_done[gl], (uint32_t)LEN, err, q.wait_ns)) return false;
            if (!persist_wait(&q.hpre_done[g], d * nh, err, q.wait_ns)) return false;
        } else if (!persist_wait(&q.lt_done[gl * 8 + lev - 1], (uint32_t)lt_items(LEN, lev - 1), err, q.wait_ns)) {
            return false;
        }
        const uint32_t s = g * 32 + lane;
        if (s < v.count && v.status[s] == 0) {
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
        return true;
    }
    r -= (unsigned long long)G * LT;
    {  // -------- compute_root of a group, then the next layer's list or the verdict
        const uint32_t g = (uint32_t)r, gl = g * d + layer;
        if (!persist_wait(&q.lt_done[gl * 8 + LV - 1], 1u, err, q.wait_ns)) return false;
        const uint32_t s = g * 32 + lane;
        const bool live = s < v.count && v.status[s] == 0;
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
        return true;
    }
    return true;
}

// One batch in one launch: warps pop tickets from q.ticket until the
// sequence is exhausted.
template <class F, class FT>
__global__ void __launch_bounds__(128, persist_min_ctas<F>()) k_verify_persist(const __grid_constant__ VerifyArgs v,
                                                                              const __grid_constant__ PersistArgs q)
{
    __shared__ uint32_t sh_cnt[4][32];
    __shared__ int sh_last;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t* cnt = sh_cnt[(threadIdx.x >> 5) & 3];
    uint32_t* err = q.hdr;
    const unsigned long long total = persist_tickets<F>(v, q);
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(q.ticket, 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total || *(volatile uint32_t*)err) break;
        if (!persist_step<F, FT>(v, q, t, cnt)) break;
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

// Keygen and sign batches inside a persistent launch.  Their subtrees (all
// of height h) are built by tasks of the same queue:
//   ctx     32 keys: PUB_SEED / SK_SEED / SK_PRF midstates            (no deps)
//   chain   chain c of 32 leaves (a lane each): PRF_keygen + 15 F     (ctx)
//   ltree   one pair index of one L-tree level of those 32 leaves     (chains / level below)
//   merkle  32 nodes of one level of one subtree                      (leaf groups / level below)
// then, for keygen, one task per key writing pk and sk (its tree), and for
// sign, the preparation of 32 signatures (R, H_msg, chain lengths, auth
// paths; every subtree built) and the signature chains, 32 at a time (their
// preparation).  Ticket order: ctx, chains (leaf-group major), L-tree levels,
// Merkle levels (level major), then the tail; each task waits only on
// smaller tickets.  Leaf groups never straddle subtrees: h >= 5 in every
// parameter set.

struct TreeTask {
    const TreeJob* trees;   // [ntrees]: key, layer, tree, node_off
    uint32_t ntrees, h;
    uint8_t* nodes;         // node arrays
    uint8_t* wpk;           // [ntrees << h][LEN][n] WOTS public keys
    uint8_t* wpk2;          // [ntrees << h][(LEN + 1) / 2][n] (L-tree ping-pong)
    const uint8_t* keys;    // key material rows the contexts are made from
    uint32_t key_stride, off_pub, off_sks, off_skp, nkeys;
    uint32_t* chains_done;  // [leaf groups] chain tasks finished
    uint32_t* lt_done;      // [leaf groups][8] L-tree level tasks finished
    uint32_t* lvl_done;     // [ntrees][h + 1] level 0: leaf groups done; level m: its Merkle tasks
    uint32_t* trees_done;   // subtrees complete
    uint32_t* prep_done;    // sign preparation tasks finished
    const uint8_t* seeds;   // keygen: [ntrees][3n] SK_SEED || SK_PRF || PUB_SEED
    uint8_t* pk;            // keygen: [ntrees][2n]
    uint8_t* sk;            // keygen: [ntrees][sk_bytes]
    uint32_t index_bytes, sk_bytes;
    const uint8_t* ibytes;  // sign: [count][8] the index bytes of each signature
};

struct PersistBatch {
    uint32_t kind;   // kJobVerify, kJobKeygen, kJobSign
    VerifyArgs v;    // verify
    PersistArgs q;   // hdr (error flag, CTAs out, contexts done), ctx, wait_ns: every kind
    TreeTask t;      // keygen, sign
    SignArgs g;      // sign
};

// Merkle tasks of level m (nodes of level m + 1 in groups of 32) per subtree.
__host__ __device__ inline unsigned long long merkle_chunks(uint32_t h, uint32_t m)
{
    return ((1ull << (h - m - 1)) + 31) / 32;
}

// Ticket counts of a keygen or sign batch: [0] ctx, [1] chains, [2] L-tree,
// [3] Merkle, [4] tail (keygen: one per key; sign: preparation), [5] sign
// chains.
__host__ __device__ inline void gen_counts(const PersistBatch& J, int len, unsigned long long (&c)[6])
{
    const TreeTask& t = J.t;
    const unsigned long long groups = ((unsigned long long)t.ntrees << t.h) >> 5;
    c[0] = (t.nkeys + 31) / 32;
    c[1] = groups * len;
    c[2] = groups * lt_items_total(len);
    c[3] = 0;
    for (uint32_t m = 0; m < t.h; m++) c[3] += t.ntrees * merkle_chunks(t.h, m);
    if (J.kind == kJobKeygen) {
        c[4] = t.ntrees;
        c[5] = 0;
    } else {
        c[4] = (J.g.count + 31) / 32;
        c[5] = ((unsigned long long)J.g.count * J.g.d * len + 31) / 32;
    }
}

__host__ __device__ inline unsigned long long gen_total(const PersistBatch& J, int len)
{
    unsigned long long c[6];
    gen_counts(J, len, c);
    return c[0] + c[1] + c[2] + c[3] + c[4] + c[5];
}

// The rare, register-heavy tasks of a keygen or sign batch, kept out of
// line so that the chain loop of the frequent tasks keeps its registers.
template <class F>
__device__ __noinline__ void gen_ctx_task(const TreeTask& T, typename F::Ctx* ctx, uint32_t k)
{
    if (k < T.nkeys) {
        const uint8_t* row = T.keys + (uint64_t)k * T.key_stride;
        typename F::Ctx x;
        F::make_ctx(x, row + T.off_pub, row + T.off_sks, row + T.off_skp);
        ctx[k] = x;
    }
}

template <class F>
__device__ __noinline__ void gen_sign_prep_task(const SignArgs& g, const TreeTask& T, const typename F::Ctx* ctx,
                                                uint32_t s)
{
    if (s < g.count) {
        sign_prep_one<F>(g, ctx, s);
        uint8_t* sm = g.sm + g.sm_off[s];
        for (uint32_t i = 0; i < g.index_bytes; i++) sm[i] = T.ibytes[(uint64_t)s * 8 + i];
    }
}

// Runs ticket t of a keygen or sign batch (whole warp); false when a wait
// ran out or the batch failed.
template <class F, class FT>
__device__ __forceinline__ bool gen_step(const PersistBatch& J, unsigned long long t)
{
    using Ctx = typename F::Ctx;
    constexpr int LEN = F::LEN, N = F::N;
    const TreeTask& T = J.t;
    const PersistArgs& q = J.q;
    const uint32_t lane = threadIdx.x & 31, h = T.h;
    uint32_t* err = q.hdr;
    Ctx* ctx = (Ctx*)q.ctx;
    unsigned long long c[6];
    gen_counts(J, LEN, c);
    if (t < c[0]) {  // -------- contexts of 32 keys
        gen_ctx_task<F>(T, ctx, (uint32_t)t * 32 + lane);
        persist_signal(&q.hdr[2]);
        return true;
    }
    t -= c[0];
    if (t < c[1]) {  // -------- chain c of 32 leaves: wots_pkgen's chain (PRF_keygen + 15 F)
        const uint32_t grp = (uint32_t)(t / LEN), ch = (uint32_t)(t - (unsigned long long)grp * LEN);
        if (!persist_wait(&q.hdr[2], (uint32_t)c[0], err, q.wait_ns)) return false;
        const uint64_t slot = (uint64_t)grp * 32 + lane;
        const TreeJob tj = T.trees[slot >> h];
        const uint32_t leaf = (uint32_t)(slot & ((1ull << h) - 1));
        const typename FT::Ctx kc = ((const typename FT::Ctx*)ctx)[tj.key];
        uint32_t a[8], x[F::NW];
        set_addr(a, tj.layer, tj.tree, ADDR_OTS, leaf, ch, 0);
        run_chain<FT>(x, kc, a, 0, 15, true);
        F::store(T.wpk + (slot * LEN + ch) * N, x);
        persist_signal(&T.chains_done[grp]);
        return true;
    }
    t -= c[1];
    if (t < c[2]) {  // -------- one pair index of one L-tree level of 32 leaves
        const unsigned long long groups = c[1] / LEN;
        int lev = 0;
        while (t >= groups * lt_items(LEN, lev)) {
            t -= groups * lt_items(LEN, lev);
            lev++;
        }
        const uint32_t items = (uint32_t)lt_items(LEN, lev);
        const uint32_t grp = (uint32_t)(t / items), p = (uint32_t)(t - (unsigned long long)grp * items);
        if (lev == 0) {
            if (!persist_wait(&T.chains_done[grp], (uint32_t)LEN, err, q.wait_ns)) return false;
        } else if (!persist_wait(&T.lt_done[grp * 8 + lev - 1], (uint32_t)lt_items(LEN, lev - 1), err, q.wait_ns)) {
            return false;
        }
        const uint64_t slot = (uint64_t)grp * 32 + lane;
        const uint32_t j = (uint32_t)(slot >> h);
        const TreeJob tj = T.trees[j];
        const uint32_t leaf = (uint32_t)(slot & ((1ull << h) - 1));
        const int cin = lt_cnt(LEN, lev);
        const bool even = (lev & 1) == 0;
        const uint8_t* src = even ? T.wpk + slot * LEN * N : T.wpk2 + slot * ((LEN + 1) / 2) * N;
        uint8_t* out = (cin == 2) ? T.nodes + tj.node_off + (level_offset((int)h, 0) + leaf) * N
                       : even     ? T.wpk2 + (slot * ((LEN + 1) / 2) + p) * N
                                  : T.wpk + (slot * LEN + p) * N;
        uint32_t l[F::NW], o[F::NW];
        F::load(l, src + (uint64_t)(2 * p) * N);
        if (2 * (int)p + 1 < cin) {
            uint32_t rr[F::NW], a[8];
            F::load(rr, src + (uint64_t)(2 * p + 1) * N);
            set_addr(a, tj.layer, tj.tree, ADDR_LTREE, leaf, (uint32_t)lev, p);
            F::thash_h(o, l, rr, ctx[tj.key], a);
            F::store(out, o);
        } else {
            F::store(out, l);
        }
        persist_signal(&T.lt_done[grp * 8 + lev]);
        // the leaf group's last level completes a group of its subtree's leaves
        if (cin == 2) persist_signal(&T.lvl_done[j * (h + 1)]);
        return true;
    }
    t -= c[2];
    if (t < c[3]) {  // -------- 32 nodes of Merkle level m + 1 of one subtree
        uint32_t m = 0;
        while (t >= T.ntrees * merkle_chunks(h, m)) {
            t -= T.ntrees * merkle_chunks(h, m);
            m++;
        }
        const unsigned long long per = merkle_chunks(h, m);
        const uint32_t j = (uint32_t)(t / per), ck = (uint32_t)(t - (unsigned long long)j * per);
        const uint32_t need = m == 0 ? (1u << h) / 32 : (uint32_t)merkle_chunks(h, m - 1);
        if (!persist_wait(&T.lvl_done[j * (h + 1) + m], need, err, q.wait_ns)) return false;
        const TreeJob tj = T.trees[j];
        uint8_t* base = T.nodes + tj.node_off;
        const uint32_t i = ck * 32 + lane;
        if (i < (1u << (h - m - 1))) {
            uint32_t l[F::NW], r[F::NW], o[F::NW], a[8];
            F::load(l, base + (level_offset((int)h, (int)m) + 2ull * i) * N);
            F::load(r, base + (level_offset((int)h, (int)m) + 2ull * i + 1) * N);
            set_addr(a, tj.layer, tj.tree, ADDR_HASHTREE, 0, m, i);
            F::thash_h(o, l, r, ctx[tj.key], a);
            F::store(base + (level_offset((int)h, (int)m + 1) + i) * N, o);
        }
        persist_signal(&T.lvl_done[j * (h + 1) + m + 1]);
        if (m + 1 == h) persist_signal(T.trees_done);
        return true;
    }
    t -= c[3];
    if (J.kind == kJobKeygen) {  // -------- pk and sk of key t (xmss_core.c:134-161)
        const uint32_t k = (uint32_t)t;
        if (!persist_wait(&T.lvl_done[k * (h + 1) + h], 1u, err, q.wait_ns)) return false;
        const uint8_t* seed = T.seeds + (uint64_t)k * 3 * N;
        const uint8_t* root = T.nodes + T.trees[k].node_off + level_offset((int)h, (int)h) * N;
        uint8_t* P = T.pk + (uint64_t)k * 2 * N;
        uint8_t* S = T.sk + (uint64_t)k * T.sk_bytes;
        const uint32_t ib = T.index_bytes;
        for (uint32_t i = lane; i < (uint32_t)N; i += 32) {
            P[i] = root[i];
            P[N + i] = seed[2 * N + i];
            S[ib + i] = seed[i];
            S[ib + N + i] = seed[N + i];
            S[ib + 2 * N + i] = root[i];
            S[ib + 3 * N + i] = seed[2 * N + i];
        }
        for (uint32_t i = lane; i < ib; i += 32) S[i] = 0;
        return true;
    }
    const SignArgs& g = J.g;
    if (t < c[4]) {  // -------- preparation of 32 signatures (every subtree built)
        if (!persist_wait(T.trees_done, T.ntrees, err, q.wait_ns)) return false;
        gen_sign_prep_task<F>(g, T, ctx, (uint32_t)t * 32 + lane);
        persist_signal(T.prep_done);
        return true;
    }
    t -= c[4];
    {  // -------- 32 signature chains (wots_sign, wots.c:136-154)
        if (!persist_wait(T.prep_done, (uint32_t)c[4], err, q.wait_ns)) return false;
        const uint64_t item = t * 32 + lane;
        if (item < (uint64_t)g.count * g.d * LEN) {
            const typename FT::Ctx kc = ((const typename FT::Ctx*)ctx)[g.key[item / LEN / g.d]];
            sign_chain_one<FT>(g, kc, item);
        }
        return true;
    }
}

// Batches of several parameter sets of one family (same F: LEN and n
// agree; d, h', index and signature sizes may differ) and of all three
// kinds in ONE launch over one shared ticket counter.  Each batch's ticket
// sequence is cut into phases - a verify batch's key contexts, H_msg and
// h_pre, then one phase per layer; a keygen or sign batch is one phase - and
// the shared sequence takes phase 0 of every batch, then layer 0 of every
// verify batch, then layer 1 of those that have one, and so on (segment s =
// local tickets [local0[s], local0[s] + first[s + 1] - first[s]) of batch
// job[s]).  Every batch keeps its own order and depends on nothing of the
// others, so the sequence is still topological and the launch completes
// whatever the residency, while the batches run their phases side by side.
// A batch whose dependency wait ran out (its own error flag) skips its
// remaining tickets; a verify batch then ends with -3 in its statuses, the
// others finish.
constexpr uint32_t kMaxPersistJobs = 8;
constexpr uint32_t kMaxPersistSegs = kMaxPersistJobs * 13;  // phases: 1 + up to 12 layers
struct PersistJobs {
    PersistBatch job[kMaxPersistJobs];
    unsigned long long first[kMaxPersistSegs + 1];  // first shared ticket of each segment
    unsigned long long local0[kMaxPersistSegs];     // its first ticket in its batch's sequence
    uint8_t seg_job[kMaxPersistSegs];               // its batch
    unsigned long long* ticket;  // the shared ticket counter (zeroed before the launch)
    uint32_t* exited;            // CTAs that have left the loop (zeroed before the launch)
    uint32_t njobs, nsegs;
};

// GEN: the launch holds keygen or sign batches.  Their task code raises the
// kernel's register use, so launches of verify batches only leave it out,
// and with it the SHA-256 form runs 4 CTAs per SM (128 registers, ~0.5 KB of
// spills) instead of 5 (96 registers, ~1 KB).
template <class F>
constexpr int persist_gen_min_ctas()
{
    return persist_min_ctas<F>() > 2 ? persist_min_ctas<F>() - 1 : persist_min_ctas<F>();
}

template <class F, class FT, bool GEN>
__global__ void __launch_bounds__(128, GEN ? persist_gen_min_ctas<F>() : persist_min_ctas<F>())
    k_verify_persist_multi(const __grid_constant__ PersistJobs P)
{
    __shared__ uint32_t sh_cnt[4][32];
    __shared__ int sh_last;
    const uint32_t lane = threadIdx.x & 31;
    uint32_t* cnt = sh_cnt[(threadIdx.x >> 5) & 3];
    const unsigned long long total = P.first[P.nsegs];
    uint32_t sg = 0;  // a warp's tickets only grow, so its segment only grows
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(P.ticket, 1ull);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= total) break;
        while (t >= P.first[sg + 1]) sg++;
        const PersistBatch& J = P.job[P.seg_job[sg]];
        if (*(volatile uint32_t*)J.q.hdr) continue;  // that batch failed
        const unsigned long long lt = P.local0[sg] + (t - P.first[sg]);
        if (!GEN || J.kind == kJobVerify) {
            persist_step<F, FT>(J.v, J.q, lt, cnt);
        } else if constexpr (GEN) {
            gen_step<F, FT>(J, lt);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        sh_last = atomicAdd(P.exited, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (sh_last) {
        __threadfence();
        for (uint32_t k = 0; k < P.njobs; k++)
            if (P.job[k].kind == kJobVerify && *(volatile uint32_t*)P.job[k].q.hdr)
                for (uint32_t s = threadIdx.x; s < P.job[k].v.count; s += blockDim.x) P.job[k].v.status[s] = -3;
    }
}

}  // namespace xb
