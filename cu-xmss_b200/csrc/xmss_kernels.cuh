// XMSS / XMSS^MT kernels for sm_100a, templated over a hash family F
// (families.cuh).  The hot path is split into phases with flat work lists so
// every launch has one uniform work item per thread:
//
//   keygen / tree build   chains (PRF_keygen + 15 F per chain)
//                         -> L-tree levels -> Merkle tree levels
//   verify                prep (H_msg + base_w) -> chains (len_i .. 14)
//                         -> L-tree levels -> root (compute_root, compare)
//   sign                  trees (as keygen) -> prep (R, H_msg, auth paths,
//                         base_w of every layer) -> chains (0 .. len_i - 1)
//
// Reference functions restated here (cuxmss/): wots.c:14-175 (expand_seed,
// gen_chain, base_w, checksum), xmss_commons.c:16-96 (l_tree, compute_root),
// xmss_core.c:19-86 (treehash as level-synchronous reduction),
// xmss_commons.c:136-215 (sign_open), xmss_core.c:183-273 (sign).
#pragma once

#include <cstdint>
#include <type_traits>

#include "families.cuh"

namespace xb {

enum : uint32_t { ADDR_OTS = 0, ADDR_LTREE = 1, ADDR_HASHTREE = 2 };

// One WOTS leaf slot of an L-tree launch: its address and where the leaf goes.
struct LeafRef {
    uint32_t key;
    uint32_t layer;
    uint64_t tree;
    uint32_t leaf;
    uint32_t pad;
    uint64_t out_off;  // byte offset of the finished leaf in the leaf output
};

// One Merkle subtree to build (all jobs of a launch share the same height).
struct TreeJob {
    uint32_t key;
    uint32_t layer;
    uint64_t tree;
    uint64_t node_off;  // byte offset of the node array (levels 0..h, level-major)
};

// Byte offset (in nodes) of level l inside a subtree node array of height h.
__host__ __device__ __forceinline__ uint64_t level_offset(int h, int l)
{
    return (2ull << h) - (2ull << (h - l));
}

__device__ __forceinline__ void set_addr(uint32_t (&a)[8], uint32_t layer, uint64_t tree, uint32_t type,
                                         uint32_t w4, uint32_t w5, uint32_t w6)
{
    a[0] = layer;
    a[1] = (uint32_t)(tree >> 32);
    a[2] = (uint32_t)tree;
    a[3] = type;
    a[4] = w4;
    a[5] = w5;
    a[6] = w6;
    a[7] = 0;
}

__device__ __forceinline__ uint64_t bytes_be(const uint8_t* p, int len)
{
    uint64_t r = 0;
    for (int i = 0; i < len; i++) r = (r << 8) | p[i];
    return r;
}

// base_w of the n-byte message plus the checksum digits (wots.c:60-107);
// writes the LEN chain start positions.
template <class F>
__device__ __forceinline__ void chain_lengths(uint8_t* lens, const uint32_t (&msg)[F::NW])
{
    int csum = 0;
#pragma unroll
    for (int k = 0; k < F::N; k++) {
        const uint32_t b = F::byte_at(msg, k);
        lens[2 * k] = (uint8_t)(b >> 4);
        lens[2 * k + 1] = (uint8_t)(b & 15);
        csum += 30 - (int)(b >> 4) - (int)(b & 15);
    }
    // len2 = 3 digits of csum << 4, i.e. the top 12 bits of a 16-bit value
    csum <<= 4;
    lens[F::LEN1] = (uint8_t)((csum >> 12) & 15);
    lens[F::LEN1 + 1] = (uint8_t)((csum >> 8) & 15);
    lens[F::LEN1 + 2] = (uint8_t)((csum >> 4) & 15);
}

// Per-key contexts from strided rows of PUB_SEED, SK_SEED and SK_PRF (the
// secret rows may be absent for verify-only keys).
// WOTS chain: optional PRF_keygen (expand_seed, wots.c:14-29) then F at hash
// addresses start .. start+steps-1 (gen_chain, wots.c:38-53).  Families with
// a fused chain loop (F::kHasChain) run it; others call their hashes.
template <class F, class = void>
struct HasChain : std::false_type {};
template <class F>
struct HasChain<F, std::void_t<decltype(F::kHasChain)>> : std::true_type {};

template <class F>
__device__ __forceinline__ void run_chain(uint32_t (&x)[F::NW], const typename F::Ctx& c, uint32_t (&a)[8],
                                          uint32_t start, uint32_t steps, bool keygen)
{
    if constexpr (HasChain<F>::value) {
        F::chain(x, c, a, start, steps, keygen);
    } else {
        if (keygen) F::prf_keygen(x, c, a);
#pragma unroll 1
        for (uint32_t i = start; i < start + steps; i++) {
            a[6] = i;
            F::thash_f(x, c, a);
        }
    }
}

// Per-key contexts from strided rows of PUB_SEED, SK_SEED and SK_PRF (the
// secret rows may be absent for verify-only keys).
template <class F>
__global__ void k_make_ctx(const uint8_t* __restrict__ pub, uint32_t pub_stride, const uint8_t* __restrict__ sks,
                           uint32_t sks_stride, const uint8_t* __restrict__ skp, uint32_t skp_stride,
                           uint32_t nkeys, typename F::Ctx* __restrict__ ctx)
{
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nkeys) return;
    typename F::Ctx c;
    F::make_ctx(c, pub + (size_t)k * pub_stride, sks ? sks + (size_t)k * sks_stride : nullptr,
                skp ? skp + (size_t)k * skp_stride : nullptr);
    ctx[k] = c;
}

// ---------------------------------------------------------------------------
// Tree building.
// ---------------------------------------------------------------------------

// One thread per (job, leaf, chain): PRF_keygen then the full chain (15 F),
// i.e. expand_seed + gen_chain(0, w-1) of wots_pkgen (wots.c:117-131).
// Leaf slots are numbered job-major (slot = job << h | leaf); one launch
// covers slots [slot0, slot0 + nslots) and indexes wpk / refs from slot0.
template <class F>
__global__ void __launch_bounds__(128) k_keygen_chains(const TreeJob* __restrict__ jobs, int h, uint64_t slot0,
                                                       uint64_t nslots, const typename F::Ctx* __restrict__ ctx,
                                                       uint8_t* __restrict__ wpk, LeafRef* __restrict__ refs)
{
    const uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= nslots * F::LEN) return;
    const uint64_t local = item / F::LEN;
    const uint32_t chain = (uint32_t)(item - local * F::LEN);
    const uint64_t slot = slot0 + local;
    const uint32_t j = (uint32_t)(slot >> h);
    const uint32_t leaf = (uint32_t)(slot & ((1ull << h) - 1));
    const TreeJob job = jobs[j];
    const typename F::Ctx& c = ctx[job.key];
    uint32_t a[8], x[F::NW];
    set_addr(a, job.layer, job.tree, ADDR_OTS, leaf, chain, 0);
    run_chain<F>(x, c, a, 0, 15, true);
    F::store(wpk + item * F::N, x);
    if (chain == 0) {
        LeafRef r;
        r.key = job.key;
        r.layer = job.layer;
        r.tree = job.tree;
        r.leaf = leaf;
        r.pad = 0;
        r.out_off = job.node_off + (uint64_t)leaf * F::N;
        refs[local] = r;
    }
}

// In-CTA subtrees: one thread per leaf, a CTA of 2^k threads builds a whole
// subtree of height k (wots_pkgen + l_tree + the lowest k levels of
// treehash, wots.c:117-131, xmss_commons.c:16-49, xmss_core.c:19-86).
//
// The thread computes its leaf's LEN chains in order (PRF_keygen + 15 F
// each) and reduces them as they come: a stack in shared memory holds the
// complete L-tree subtrees so far, whose sizes are the set bits of the
// chains pushed (a binary counter), so chain ch merges with the stack top
// once for every trailing one bit of ch.  After the last chain the odd
// nodes are carried up exactly as l_tree carries them (a node alone at the
// end of its level moves to the next level unhashed) and merged with the
// remaining entries.  The hashes, their addresses and their order per node
// are those of l_tree; nothing of the WOTS public key leaves the thread.
// Then the 2^k leaves are reduced level by level in shared memory, and every
// node of the subtree (levels 0..k) is written to the job's node array;
// levels k+1..h follow as k_tree_level launches across CTAs.
//
// Grid: jobs x 2^(h-k) CTAs, numbered from cta0.  Dynamic shared memory:
// subtree_smem<F>(2^k) bytes.
__host__ __device__ constexpr int bit_width_c(int x) { return x ? 1 + bit_width_c(x >> 1) : 0; }

template <class F>
__host__ __device__ constexpr size_t subtree_smem(uint32_t threads)
{
    return (size_t)(bit_width_c(F::LEN) + 1) * threads * F::N;
}

template <class F>
__global__ void __launch_bounds__(128) k_keygen_subtree(const TreeJob* __restrict__ jobs, int h, int k, uint64_t cta0,
                                                        const typename F::Ctx* __restrict__ ctx,
                                                        uint8_t* __restrict__ nodes)
{
    constexpr int LEN = F::LEN, N = F::N, D = bit_width_c(F::LEN);
    extern __shared__ __align__(16) uint8_t sh[];
    const uint32_t B = blockDim.x;  // 2^k
    const uint32_t t = threadIdx.x;
    uint8_t* stk = sh + (size_t)t * N;            // entry e at stk + e * B * N
    uint8_t* lvl = sh + (size_t)D * B * N;        // [B][N] nodes of the current level
    const uint64_t cta = cta0 + blockIdx.x;
    const int sub_bits = h - k;
    const uint32_t j = (uint32_t)(cta >> sub_bits);
    const uint64_t sub = cta & ((1ull << sub_bits) - 1);
    const TreeJob job = jobs[j];
    const uint32_t leaf = (uint32_t)((sub << k) + t);
    const typename F::Ctx& c = ctx[job.key];
    uint8_t* base = nodes + job.node_off;
    uint32_t x[F::NW], a[8];
    int sp = 0;
#pragma unroll 1
    for (uint32_t ch = 0; ch < (uint32_t)LEN; ch++) {
        set_addr(a, job.layer, job.tree, ADDR_OTS, leaf, ch, 0);
        run_chain<F>(x, c, a, 0, 15, true);
        // node (level l, index ch >> l) merges while its index is odd
#pragma unroll 1
        for (uint32_t l = 0; (ch >> l) & 1; l++) {
            uint32_t left[F::NW];
            F::load(left, stk + (size_t)(--sp) * B * N);
            set_addr(a, job.layer, job.tree, ADDR_LTREE, leaf, l, ch >> (l + 1));
            F::thash_h(x, left, x, c, a);
        }
        F::store(stk + (size_t)(sp++) * B * N, x);
    }
    // The top entry (level L, index I) covers the last 2^L chains; the
    // entries below it are the higher set bits R of LEN, lowest on top.  A
    // node below the next entry's level is the last of its level with an
    // even index: it moves up unhashed (l_tree's carry); at that level it is
    // the right sibling of the entry, and they merge.
    uint32_t L = __ffs(LEN) - 1, I = ((uint32_t)LEN >> L) - 1, R = (uint32_t)LEN & ((uint32_t)LEN - 1);
    F::load(x, stk + (size_t)(--sp) * B * N);
#pragma unroll 1
    while (R) {
        const uint32_t L2 = __ffs(R) - 1;
        I >>= (L2 - L);
        L = L2;
        uint32_t left[F::NW];
        F::load(left, stk + (size_t)(--sp) * B * N);
        set_addr(a, job.layer, job.tree, ADDR_LTREE, leaf, L, I >> 1);
        F::thash_h(x, left, x, c, a);
        L++;
        I >>= 1;
        R &= R - 1;
    }
    // x is the leaf: level 0 of the subtree, then levels 1..k in shared memory
    F::store(base + (level_offset(h, 0) + leaf) * N, x);
    F::store(lvl + (size_t)t * N, x);
    __syncthreads();
#pragma unroll 1
    for (int l = 0; l < k; l++) {
        const uint32_t cnt = B >> (l + 1);
        const uint32_t gi = (uint32_t)(sub << (k - l - 1)) + t;  // the parent's index on level l + 1
        if (t < cnt) {
            uint32_t le[F::NW], ri[F::NW];
            F::load(le, lvl + (size_t)(2 * t) * N);
            F::load(ri, lvl + (size_t)(2 * t + 1) * N);
            set_addr(a, job.layer, job.tree, ADDR_HASHTREE, 0, (uint32_t)l, gi);
            F::thash_h(x, le, ri, c, a);
        }
        __syncthreads();
        if (t < cnt) {
            F::store(lvl + (size_t)t * N, x);
            F::store(base + (level_offset(h, l + 1) + gi) * N, x);
        }
        __syncthreads();
    }
}

// One L-tree level (xmss_commons.c:16-49) for many leaf slots: item =
// (slot, pair).  Pairs hash nodes 2p, 2p+1; an odd last node is carried up.
// The final level (cnt_in == 2) writes the leaf to leaf_out + ref.out_off.
template <class F>
__global__ void __launch_bounds__(128) k_ltree_level(const LeafRef* __restrict__ refs, uint32_t nslots, int level,
                                                     int cnt_in, const uint8_t* __restrict__ src, uint32_t src_stride,
                                                     uint8_t* __restrict__ dst, uint32_t dst_stride,
                                                     uint8_t* __restrict__ leaf_out,
                                                     const typename F::Ctx* __restrict__ ctx,
                                                     const int* __restrict__ status)
{
    const int pairs = (cnt_in + 1) >> 1;
    const uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= (uint64_t)nslots * pairs) return;
    const uint32_t slot = (uint32_t)(item / pairs);
    const int p = (int)(item - (uint64_t)slot * pairs);
    if (status && status[slot] != 0) return;
    const LeafRef r = refs[slot];
    const uint8_t* s = src + ((uint64_t)slot * src_stride) * F::N;
    uint8_t* out = (cnt_in == 2) ? leaf_out + r.out_off : dst + ((uint64_t)slot * dst_stride + p) * F::N;
    uint32_t l[F::NW], rr[F::NW], o[F::NW];
    F::load(l, s + (uint64_t)(2 * p) * F::N);
    if (2 * p + 1 < cnt_in) {
        F::load(rr, s + (uint64_t)(2 * p + 1) * F::N);
        uint32_t a[8];
        set_addr(a, r.layer, r.tree, ADDR_LTREE, r.leaf, (uint32_t)level, (uint32_t)p);
        F::thash_h(o, l, rr, ctx[r.key], a);
        F::store(out, o);
    } else {
        F::store(out, l);
    }
}

// One Merkle level of many subtrees of equal height h: item = (job, node i
// of level+1) = H(child 2i, child 2i+1) with tree_height = level, tree_index
// = i (xmss_core.c:62-83).
template <class F>
__global__ void __launch_bounds__(128) k_tree_level(const TreeJob* __restrict__ jobs, uint32_t njobs, int h, int level,
                                                    uint8_t* __restrict__ nodes,
                                                    const typename F::Ctx* __restrict__ ctx)
{
    const int sh = h - level - 1;
    const uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= ((uint64_t)njobs << sh)) return;
    const uint32_t j = (uint32_t)(item >> sh);
    const uint32_t i = (uint32_t)(item & ((1ull << sh) - 1));
    const TreeJob job = jobs[j];
    uint8_t* base = nodes + job.node_off;
    uint32_t l[F::NW], r[F::NW], o[F::NW], a[8];
    F::load(l, base + (level_offset(h, level) + 2ull * i) * F::N);
    F::load(r, base + (level_offset(h, level) + 2ull * i + 1) * F::N);
    set_addr(a, job.layer, job.tree, ADDR_HASHTREE, 0, (uint32_t)level, i);
    F::thash_h(o, l, r, ctx[job.key], a);
    F::store(base + (level_offset(h, level + 1) + i) * F::N, o);
}

// ---------------------------------------------------------------------------
// Verify (xmss_commons.c:136-215).
//
// Per layer the work is: chains (wots_pk_from_sig), L-tree (66 H for n=32),
// compute_root (h H).  Every H is split into h_pre (address only) and h_fin
// (data dependent); all h_pre of all layers run in the prep launch next to
// H_msg, so the dependent L-tree / root steps are 2 compressions each.  The
// chains are bucketed by their number of F steps (15 - len_i) and run
// longest first, so each warp runs chains of equal length.
// ---------------------------------------------------------------------------
struct VerifyArgs {
    const uint8_t* sm;        // concatenated signed messages
    const uint64_t* sm_off;   // [count] byte offset of each sm
    const uint64_t* smlen;    // [count]
    const uint32_t* key;      // [count] key index, checked against npk on the device
    const uint8_t* key_root;  // public root of key k at key_root + k * key_stride
    uint32_t key_stride;
    uint32_t npk;             // keys at key_root; a signature naming key >= npk is rejected (-1)
    uint8_t* node;            // [count][N] running message / root
    uint8_t* lens;            // [count][LEN] chain start positions
    uint64_t* idx;            // [count]
    int* status;              // [count] 0 = valid so far
    uint8_t* wpk;             // [count][LEN][N]
    uint8_t* wpk2;            // [count][LEN/2 + 1][N]
    uint8_t* leaf;            // [count][N]
    LeafRef* refs;            // [count]
    void* hpre;               // [count][d][NH] F::HPre, NH = LEN - 1 + tree_height
    uint32_t* hist;           // [d][32]: chains per step count, then bucket cursors
    uint32_t* list;           // [count * LEN] chain work list, longest first
    const uint32_t* sel;      // optional: the signatures this launch sequence handles
    const uint32_t* sel_n;    // (device) number of entries in sel; sel == null: all
    unsigned long long* work; // [3] H_msg blocks, F calls, H calls (accumulated)
    uint32_t count;
    uint32_t index_bytes;
    uint32_t sig_bytes;
    uint32_t tree_height;
    uint32_t d;
};

// Hash blocks H_msg absorbs for a message of mlen bytes (prefix pl + 3n).
template <class F>
__device__ __forceinline__ unsigned long long hmsg_blocks(uint64_t mlen)
{
    const uint64_t L = (uint64_t)F::PL + 3 * F::N + mlen;
    constexpr int K = HMsgKind<F>::v;
    if constexpr (K == 0) return (L + 9 + 63) / 64;
    else if constexpr (K == 1) return (L + 17 + 127) / 128;
    else return L / (4 * K) + 1;
}

// Adds the step counts of one signature's chains to a block histogram.
template <class F>
__device__ __forceinline__ unsigned long long count_steps(const uint8_t* lens, uint32_t* sh_hist)
{
    unsigned long long s = 0;
    for (int i = 0; i < F::LEN; i++) {
        const uint32_t steps = 15 - lens[i];
        s += steps;
        atomicAdd(&sh_hist[steps], 1u);
    }
    return s;
}

__device__ __forceinline__ void flush_hist(uint32_t* sh_hist, uint32_t* hist)
{
    __syncthreads();
    if (threadIdx.x < 16 && sh_hist[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh_hist[threadIdx.x]);
}

// Signatures handled by this launch sequence: all of them, or the selection.
__device__ __forceinline__ uint32_t sel_count(const VerifyArgs& v) { return v.sel ? *v.sel_n : v.count; }

// Inputs a signature must have before anything of it is read: a signed
// message at least sig_bytes long (the reference would underflow its message
// length there, xmss_commons.c:158) and a key index inside the key table.
// Failing either rejects the signature (-1); every later step skips it.
__device__ __forceinline__ bool verify_input_ok(const VerifyArgs& v, uint32_t s)
{
    return v.smlen[s] >= v.sig_bytes && v.key[s] < v.npk;
}
__device__ __forceinline__ uint32_t sel_sig(const VerifyArgs& v, uint32_t i) { return v.sel ? v.sel[i] : i; }

template <class F>
__device__ __forceinline__ void layer_addr(uint64_t idx, uint32_t th, uint32_t layer, uint32_t& leaf, uint64_t& tree)
{
    leaf = (uint32_t)((idx >> (th * layer)) & ((1ull << th) - 1));
    tree = (th * (layer + 1) >= 64) ? 0 : idx >> (th * (layer + 1));
}

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialization starts launching as the CTAs of the kernel before it in the
// stream exit, instead of after that kernel's completion: it reads only what
// earlier launches wrote until pdl_wait(), which returns once that kernel
// has completed and its writes are visible (at once for a plain launch).
// Every thread of such a kernel calls pdl_wait() before it exits, so the
// kernel completes only after its predecessor does, and stream order holds
// for whatever comes after it.  The L-tree levels after the first and the
// root are launched this way (1.6 % per 4,096-signature batch; the scatter
// and chain launches measured no gain).  No kernel here triggers its
// dependents early (griddepcontrol.launch_dependents): dependents that
// launched at the start of the L-tree levels sat resident beside the other
// group's chains and cost 4 % per batch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// h_pre of H node `pitem` of the signatures v selects: item = (signature,
// layer, node), the nodes of a layer numbered L-tree level by level (level 0
// pairs first), then the h authentication-path levels.  Reads the index
// from the signature itself, so it runs independently of H_msg.
template <class F>
__device__ __forceinline__ void verify_hpre_item(const VerifyArgs& v, const typename F::Ctx* __restrict__ ctx,
                                                 uint64_t pitem)
{
    using HPre = typename F::HPre;
    const uint32_t nh = F::LEN - 1 + v.tree_height;
    if (pitem >= (uint64_t)sel_count(v) * v.d * nh) return;
    const uint32_t si = (uint32_t)(pitem / ((uint64_t)v.d * nh));
    const uint32_t rem = (uint32_t)(pitem - (uint64_t)si * v.d * nh);
    const uint32_t s = sel_sig(v, si);
    const uint64_t item = (uint64_t)s * v.d * nh + rem;
    const uint32_t layer = rem / nh;
    uint32_t node = rem - layer * nh;
    if (!verify_input_ok(v, s)) return;
    const uint64_t idx = bytes_be(v.sm + v.sm_off[s], (int)v.index_bytes);
    uint32_t leaf;
    uint64_t tree;
    layer_addr<F>(idx, v.tree_height, layer, leaf, tree);
    uint32_t a[8];
    if (node < F::LEN - 1) {
        // locate (level, pair) of L-tree node `node`
        int cnt = F::LEN, level = 0;
        while (node >= (uint32_t)(cnt >> 1)) {
            node -= cnt >> 1;
            cnt = (cnt + 1) >> 1;
            level++;
        }
        set_addr(a, layer, tree, ADDR_LTREE, leaf, (uint32_t)level, node);
    } else {
        const uint32_t i = node - (F::LEN - 1);
        set_addr(a, layer, tree, ADDR_HASHTREE, 0, i, leaf >> (i + 1));
    }
    HPre hp;
    F::h_pre(hp, ctx[v.key[s]], a);
    ((HPre*)v.hpre)[item] = hp;
}

// Launch = [hmsg_blocks x 64 threads: one signature each] followed by
// [pre blocks: one H node's h_pre each]; either part may be empty.  PART 1
// and 2 compile only the H_msg or only the h_pre path (the launches of a
// split batch): each gets its own register allocation and a smaller body.
template <class F, int PART = 0>
__global__ void __launch_bounds__(64) k_verify_prep(VerifyArgs v, uint32_t hmsg_blocks_n,
                                                    const typename F::Ctx* __restrict__ ctx)
{
    __shared__ uint32_t sh_hist[16];
    if (PART != 2 && (PART == 1 || blockIdx.x < hmsg_blocks_n)) {
        if (threadIdx.x < 16) sh_hist[threadIdx.x] = 0;
        __syncthreads();
        const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
        if (i < sel_count(v)) {
            const uint32_t s = sel_sig(v, i);
            const uint64_t smlen = v.smlen[s];
            if (!verify_input_ok(v, s)) {
                v.status[s] = -1;
            } else {
                const uint8_t* sm = v.sm + v.sm_off[s];
                const uint64_t idx = bytes_be(sm, (int)v.index_bytes);
                uint32_t R[F::NW], root[F::NW], mh[F::NW];
                F::load(R, sm + v.index_bytes);
                F::load(root, v.key_root + (uint64_t)v.key[s] * v.key_stride);
                hmsg<F>(mh, R, root, idx, sm + v.sig_bytes, smlen - v.sig_bytes);
                F::store(v.node + (uint64_t)s * F::N, mh);
                uint8_t* lens = v.lens + (uint64_t)s * F::LEN;
                chain_lengths<F>(lens, mh);
                v.idx[s] = idx;
                v.status[s] = 0;
                const unsigned long long steps = count_steps<F>(lens, sh_hist);
                if (v.work) {
                    atomicAdd(&v.work[0], hmsg_blocks<F>(smlen - v.sig_bytes));
                    atomicAdd(&v.work[1], steps);
                    atomicAdd(&v.work[2], (unsigned long long)(F::LEN - 1 + v.tree_height) * v.d);
                }
            }
        }
        flush_hist(sh_hist, v.hist);
        return;
    }
    if constexpr (PART != 1)
        verify_hpre_item<F>(v, ctx, (uint64_t)(blockIdx.x - hmsg_blocks_n) * blockDim.x + threadIdx.x);
}

// The H_msg part of k_verify_prep with one WARP per signature, for the
// families with a warp-parallel permutation (kWarpHmsg: SHAKE).  H_msg is a
// serial chain of permutations, so a batch's prep lasts as long as its
// longest message; spread over a warp the chain runs about four times
// faster.  Two signatures per 64-thread block; same outputs as the thread
// form (digest, chain lengths, index, status, step histogram, work).  As in
// k_verify_prep, blocks from hmsg_blocks_n on compute h_pre items instead.
template <class F>
__global__ void __launch_bounds__(64) k_verify_hmsg_warp(VerifyArgs v, uint32_t hmsg_blocks_n,
                                                         const typename F::Ctx* __restrict__ ctx)
{
    if (blockIdx.x >= hmsg_blocks_n) {
        verify_hpre_item<F>(v, ctx, (uint64_t)(blockIdx.x - hmsg_blocks_n) * blockDim.x + threadIdx.x);
        return;
    }
    __shared__ uint32_t sh_hist[16];
    if (threadIdx.x < 16) sh_hist[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t i = blockIdx.x * 2 + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (i < sel_count(v)) {
        const uint32_t s = sel_sig(v, i);
        const uint64_t smlen = v.smlen[s];
        if (!verify_input_ok(v, s)) {
            if (lane == 0) v.status[s] = -1;
        } else {
            const uint8_t* sm = v.sm + v.sm_off[s];
            const uint64_t idx = bytes_be(sm, (int)v.index_bytes);
            uint32_t R[F::NW], root[F::NW], mh[F::NW];
            F::load(R, sm + v.index_bytes);
            F::load(root, v.key_root + (uint64_t)v.key[s] * v.key_stride);
            hmsg_warp<F>(mh, R, root, idx, sm + v.sig_bytes, smlen - v.sig_bytes);
            if (lane == 0) {
                F::store(v.node + (uint64_t)s * F::N, mh);
                uint8_t* lens = v.lens + (uint64_t)s * F::LEN;
                chain_lengths<F>(lens, mh);
                v.idx[s] = idx;
                v.status[s] = 0;
                const unsigned long long steps = count_steps<F>(lens, sh_hist);
                if (v.work) {
                    atomicAdd(&v.work[0], hmsg_blocks<F>(smlen - v.sig_bytes));
                    atomicAdd(&v.work[1], steps);
                    atomicAdd(&v.work[2], (unsigned long long)(F::LEN - 1 + v.tree_height) * v.d);
                }
            }
        }
    }
    flush_hist(sh_hist, v.hist);
}

// Splits the signatures into a short-H_msg group (at most `blocks_max` hash
// blocks) and a long one, so the long messages' serial H_msg runs on its own
// stream while the short group's chains keep the GPU busy.
template <class F>
__global__ void k_verify_partition(VerifyArgs v, uint32_t blocks_max, uint32_t* sel_short, uint32_t* sel_long,
                                   uint32_t* n2)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= v.count) return;
    const uint64_t smlen = v.smlen[s];
    const bool lng = smlen >= v.sig_bytes && hmsg_blocks<F>(smlen - v.sig_bytes) > blocks_max;
    if (lng) {
        sel_long[atomicAdd(&n2[1], 1u)] = s;
    } else {
        sel_short[atomicAdd(&n2[0], 1u)] = s;
    }
}

// Buckets the chains of one layer by step count (longest first) into
// v.list; zero-step chains are copied straight to the WOTS pk.  Also writes
// the L-tree address of every signature.
template <class F>
__global__ void __launch_bounds__(256) k_verify_scatter(VerifyArgs v, uint32_t layer)
{
    __shared__ uint32_t sh_cnt[16], sh_base[16];
    uint32_t* hist = v.hist + 32 * layer;
    if (threadIdx.x < 16) sh_cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t it = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = it < (uint64_t)sel_count(v) * F::LEN;
    const uint32_t si = in ? (uint32_t)(it / F::LEN) : 0;
    const uint32_t chain = in ? (uint32_t)(it - (uint64_t)si * F::LEN) : 0;
    const uint32_t s = in ? sel_sig(v, si) : 0;
    const uint64_t item = (uint64_t)s * F::LEN + chain;
    const bool live = in && v.status[s] == 0;
    uint32_t steps = 0, local = 0;
    if (live) {
        steps = 15 - v.lens[item];
        if (steps) local = atomicAdd(&sh_cnt[steps], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 16) {
        const uint32_t k = threadIdx.x;
        uint32_t base = 0;
        for (uint32_t j = k + 1; j < 16; j++) base += hist[j];  // longer chains first
        sh_base[k] = sh_cnt[k] ? base + atomicAdd(&hist[16 + k], sh_cnt[k]) : 0;
    }
    __syncthreads();
    if (!live) return;
    const uint32_t th = v.tree_height;
    const uint64_t wsb = (uint64_t)F::LEN * F::N;
    if (steps) {
        v.list[sh_base[steps] + local] = (uint32_t)item;
    } else {
        const uint8_t* sig = v.sm + v.sm_off[s] + v.index_bytes + F::N + layer * (wsb + (uint64_t)th * F::N);
        uint32_t x[F::NW];
        F::load(x, sig + (uint64_t)chain * F::N);
        F::store(v.wpk + item * F::N, x);
    }
    if (chain == 0) {
        LeafRef r;
        layer_addr<F>(v.idx[s], th, layer, r.leaf, r.tree);
        r.key = v.key[s];
        r.layer = layer;
        r.pad = 0;
        r.out_off = (uint64_t)s * F::N;
        v.refs[s] = r;
    }
}

// One thread per listed chain: gen_chain(len_i, w-1-len_i) of
// wots_pk_from_sig (wots.c:161-175).
template <class F>
__global__ void __launch_bounds__(128) k_verify_chains(VerifyArgs v, uint32_t layer,
                                                       const typename F::Ctx* __restrict__ ctx)
{
    const uint32_t* hist = v.hist + 32 * layer;
    uint32_t total = 0;
#pragma unroll
    for (int k = 1; k < 16; k++) total += hist[k];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) return;
    const uint32_t item = v.list[t];
    const uint32_t s = item / F::LEN;
    const uint32_t chain = item - s * F::LEN;
    uint32_t leaf;
    uint64_t tree;
    layer_addr<F>(v.idx[s], v.tree_height, layer, leaf, tree);
    const uint32_t start = v.lens[item];
    const uint64_t wsb = (uint64_t)F::LEN * F::N;
    const uint8_t* sig =
        v.sm + v.sm_off[s] + v.index_bytes + F::N + layer * (wsb + (uint64_t)v.tree_height * F::N);
    uint32_t x[F::NW], a[8];
    F::load(x, sig + (uint64_t)chain * F::N);
    set_addr(a, layer, tree, ADDR_OTS, leaf, chain, 0);
    run_chain<F>(x, ctx[v.key[s]], a, start, 15 - start, false);
    F::store(v.wpk + (uint64_t)item * F::N, x);
}

// One L-tree level of one layer with precomputed h_pre: item = (sig, pair).
// Levels after the first are launched as dependents of the level before
// (programmatic serialization): the selection, status and h_pre loads run
// before pdl_wait(), the previous level's nodes after it.
template <class F>
__global__ void __launch_bounds__(128) k_verify_ltree(VerifyArgs v, uint32_t layer, int cnt_in, uint32_t node_base,
                                                      const uint8_t* __restrict__ src, uint32_t src_stride,
                                                      uint8_t* __restrict__ dst, uint32_t dst_stride)
{
    using HPre = typename F::HPre;
    const int pairs = (cnt_in + 1) >> 1;
    const uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    bool live = item < (uint64_t)sel_count(v) * pairs;
    uint32_t s = 0;
    int p = 0;
    if (live) {
        const uint32_t si = (uint32_t)(item / pairs);
        p = (int)(item - (uint64_t)si * pairs);
        s = sel_sig(v, si);
        live = v.status[s] == 0;
    }
    const bool pair = live && 2 * p + 1 < cnt_in;
    HPre hp;
    if (pair) {
        const uint32_t nh = F::LEN - 1 + v.tree_height;
        hp = ((const HPre*)v.hpre)[((uint64_t)s * v.d + layer) * nh + node_base + p];
    }
    pdl_wait();
    if (!live) return;
    const uint8_t* sp = src + ((uint64_t)s * src_stride) * F::N;
    uint8_t* out = (cnt_in == 2) ? v.leaf + (uint64_t)s * F::N : dst + ((uint64_t)s * dst_stride + p) * F::N;
    uint32_t l[F::NW], r[F::NW], o[F::NW];
    F::load(l, sp + (uint64_t)(2 * p) * F::N);
    if (pair) {
        F::load(r, sp + (uint64_t)(2 * p + 1) * F::N);
        F::h_fin(o, hp, l, r);
        F::store(out, o);
    } else {
        F::store(out, l);
    }
}

// The whole L-tree of one layer (xmss_commons.c:16-49) for a signature per
// warp: its LEN WOTS public-key values go to shared memory, the lanes hash
// the pairs of a level (h_fin with the precomputed h_pre), the odd node is
// carried up, and the level's nodes stay in shared memory for the next; the
// last level writes the leaf.  Same nodes, order and outputs as LEN - 1
// launches of k_verify_ltree, in one launch: for latency-bound batches (a
// warp instruction costs one issue slot however few lanes are active, so
// where many warps compete for the ALU the per-level kernels are cheaper).
template <class F>
__global__ void __launch_bounds__(64) k_verify_ltree_warp(VerifyArgs v, uint32_t layer)
{
    using HPre = typename F::HPre;
    constexpr int L0 = F::LEN, L1 = (F::LEN + 1) / 2;
    __shared__ __align__(16) uint8_t sh[2][(L0 + L1) * F::N];
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31;
    if (w >= sel_count(v)) return;
    const uint32_t s = sel_sig(v, w);
    if (v.status[s] != 0) return;
    uint8_t* a = sh[threadIdx.x >> 5];
    uint8_t* b = a + L0 * F::N;
    // level 0 from the chain outputs (N is a multiple of 8)
    const uint2* g = (const uint2*)(v.wpk + (uint64_t)s * L0 * F::N);
    for (int i = lane; i < L0 * F::N / 8; i += 32) ((uint2*)a)[i] = g[i];
    __syncwarp();
    const uint32_t nh = F::LEN - 1 + v.tree_height;
    const HPre* hp = (const HPre*)v.hpre + ((uint64_t)s * v.d + layer) * nh;
    int cnt = L0;
    uint32_t base = 0;
    while (cnt > 1) {
        const int pairs = (cnt + 1) >> 1;
        for (int p = lane; p < pairs; p += 32) {
            uint32_t l[F::NW], o[F::NW];
            F::load(l, a + (uint64_t)(2 * p) * F::N);
            if (2 * p + 1 < cnt) {
                uint32_t r[F::NW];
                F::load(r, a + (uint64_t)(2 * p + 1) * F::N);
                F::h_fin(o, hp[base + p], l, r);
            } else {
#pragma unroll
                for (int i = 0; i < F::NW; i++) o[i] = l[i];
            }
            F::store(cnt == 2 ? v.leaf + (uint64_t)s * F::N : b + (uint64_t)p * F::N, o);
        }
        __syncwarp();
        base += cnt >> 1;
        cnt = pairs;
        uint8_t* t = a;
        a = b;
        b = t;
    }
}

// compute_root (xmss_commons.c:54-96) for one layer with precomputed h_pre;
// then either the next layer's chain lengths or the comparison with the
// public root (xmss_commons.c:204-209).
template <class F>
__global__ void __launch_bounds__(64) k_verify_root(VerifyArgs v, uint32_t layer)
{
    using HPre = typename F::HPre;
    __shared__ uint32_t sh_hist[16];
    if (threadIdx.x < 16) sh_hist[threadIdx.x] = 0;
    __syncthreads();
    // before pdl_wait(): the selection, status, index, authentication path
    // and h_pre (earlier launches); after it: the leaf (the launch before)
    const uint32_t si = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t s = si < sel_count(v) ? sel_sig(v, si) : 0;
    const bool live = si < sel_count(v) && v.status[s] == 0;
    const uint32_t th = v.tree_height;
    uint32_t leafidx = 0;
    uint64_t tree = 0;
    const uint8_t* auth = nullptr;
    const HPre* hp = nullptr;
    uint32_t cur[F::NW], sib[F::NW], nsib[F::NW];
    HPre h, hnext;
    if (live) {
        layer_addr<F>(v.idx[s], th, layer, leafidx, tree);
        const uint64_t wsb = (uint64_t)F::LEN * F::N;
        auth = v.sm + v.sm_off[s] + v.index_bytes + F::N + layer * (wsb + (uint64_t)th * F::N) + wsb;
        const uint32_t nh = F::LEN - 1 + th;
        hp = (const HPre*)v.hpre + ((uint64_t)s * v.d + layer) * nh + (F::LEN - 1);
        F::load(sib, auth);
        h = hp[0];
    }
    pdl_wait();
    if (live) {
        F::load(cur, v.leaf + (uint64_t)s * F::N);
#pragma unroll 1
        for (uint32_t i = 0; i < th; i++) {
            // fetch the next level's operands while this level hashes
            if (i + 1 < th) {
                hnext = hp[i + 1];
                F::load(nsib, auth + (uint64_t)(i + 1) * F::N);
            }
            // the node goes right when its index is odd (xmss_commons.c:61-69);
            // select operands instead of branching so a warp runs one path
            const bool odd = leafidx & 1;
            uint32_t l[F::NW], r[F::NW];
#pragma unroll
            for (int k = 0; k < F::NW; k++) {
                l[k] = odd ? sib[k] : cur[k];
                r[k] = odd ? cur[k] : sib[k];
            }
            F::h_fin(cur, h, l, r);
            leafidx >>= 1;
            h = hnext;
#pragma unroll
            for (int k = 0; k < F::NW; k++) sib[k] = nsib[k];
        }
        if (layer + 1 < v.d) {
            F::store(v.node + (uint64_t)s * F::N, cur);
            uint8_t* lens = v.lens + (uint64_t)s * F::LEN;
            chain_lengths<F>(lens, cur);
            const unsigned long long st = count_steps<F>(lens, sh_hist);
            if (v.work) atomicAdd(&v.work[1], st);
        } else {
            uint32_t pr[F::NW];
            F::load(pr, v.key_root + (uint64_t)v.key[s] * v.key_stride);
            uint32_t diff = 0;
#pragma unroll
            for (int i = 0; i < F::NW; i++) diff |= pr[i] ^ cur[i];
            v.status[s] = diff ? -1 : 0;
        }
    }
    if (layer + 1 < v.d) flush_hist(sh_hist, v.hist + 32 * (layer + 1));
}


// ---------------------------------------------------------------------------
// Sign (xmss_core.c:183-273) given built subtrees.
// ---------------------------------------------------------------------------
struct SignArgs {
    uint8_t* sm;              // concatenated output buffers; M at sm + sig_bytes unless msg is set
    const uint64_t* sm_off;   // [count]
    const uint64_t* mlen;     // [count]
    const uint8_t* msg;       // optional: message i at msg + msg_off[i] (signatures then stand alone)
    const uint64_t* msg_off;  // [count]
    const uint64_t* idx;      // [count] one-time index of each signature
    const uint32_t* key;      // [count]
    const uint8_t* key_root;  // public root of key k at key_root + k * key_stride
    uint32_t key_stride;
    const uint64_t* tree_off; // [count][d] byte offset of each layer's subtree node array
    const uint8_t* nodes;     // subtree node arrays
    uint8_t* lens;            // [count][d][LEN]
    uint32_t count;
    uint32_t index_bytes;
    uint32_t sig_bytes;
    uint32_t tree_height;
    uint32_t d;
};

// One thread per signature: R, H_msg, every layer's chain lengths (layer 0
// signs the message digest, layer i signs the root of layer i-1) and the
// authentication paths copied out of the subtree node arrays.
// HMSG_DONE: R and layer 0's chain lengths were written by k_sign_hmsg_warp.
template <class F, bool HMSG_DONE = false>
__device__ __forceinline__ void sign_prep_one(const SignArgs& g, const typename F::Ctx* __restrict__ ctx, uint32_t s)
{
    uint8_t* sm = g.sm + g.sm_off[s];
    const uint64_t idx = g.idx[s];
    const uint32_t th = g.tree_height;
    uint32_t mh[F::NW];
    if constexpr (!HMSG_DONE) {
        const typename F::Ctx& c = ctx[g.key[s]];
        uint32_t R[F::NW], root[F::NW];
        F::prf_r(R, c, idx);
        F::store(sm + g.index_bytes, R);
        F::load(root, g.key_root + (uint64_t)g.key[s] * g.key_stride);
        hmsg<F>(mh, R, root, idx, g.msg ? g.msg + g.msg_off[s] : sm + g.sig_bytes, g.mlen[s]);
    }
    const uint64_t wsb = (uint64_t)F::LEN * F::N;
    for (uint32_t layer = 0; layer < g.d; layer++) {
        const uint8_t* tn = g.nodes + g.tree_off[(uint64_t)s * g.d + layer];
        const uint32_t leaf = (uint32_t)((idx >> (th * layer)) & ((1ull << th) - 1));
        if (layer == 0) {
            if constexpr (!HMSG_DONE) chain_lengths<F>(g.lens + ((uint64_t)s * g.d) * F::LEN, mh);
        } else {
            uint32_t r[F::NW];
            const uint8_t* prev = g.nodes + g.tree_off[(uint64_t)s * g.d + layer - 1];
            F::load(r, prev + level_offset((int)th, (int)th) * F::N);
            chain_lengths<F>(g.lens + ((uint64_t)s * g.d + layer) * F::LEN, r);
        }
        uint8_t* auth = sm + g.index_bytes + F::N + layer * (wsb + (uint64_t)th * F::N) + wsb;
        for (uint32_t l = 0; l < th; l++) {
            uint32_t v[F::NW];
            F::load(v, tn + (level_offset((int)th, (int)l) + ((leaf >> l) ^ 1)) * F::N);
            F::store(auth + (uint64_t)l * F::N, v);
        }
    }
}

template <class F, bool HMSG_DONE = false>
__global__ void k_sign_prep(SignArgs g, const typename F::Ctx* __restrict__ ctx)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < g.count) sign_prep_one<F, HMSG_DONE>(g, ctx, s);
}

// R and H_msg of each signature with one thread per signature (the
// families without a warp-parallel H_msg), writing R into the signature and
// layer 0's chain lengths; k_sign_prep<F, true> does the rest.  It reads
// only the key contexts, the key roots and the message, so it can run
// beside the subtree builds.
template <class F>
__global__ void k_sign_hmsg(SignArgs g, const typename F::Ctx* __restrict__ ctx)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.count) return;
    uint8_t* sm = g.sm + g.sm_off[s];
    const uint64_t idx = g.idx[s];
    uint32_t R[F::NW], root[F::NW], mh[F::NW];
    F::prf_r(R, ctx[g.key[s]], idx);
    F::store(sm + g.index_bytes, R);
    F::load(root, g.key_root + (uint64_t)g.key[s] * g.key_stride);
    hmsg<F>(mh, R, root, idx, g.msg ? g.msg + g.msg_off[s] : sm + g.sig_bytes, g.mlen[s]);
    chain_lengths<F>(g.lens + ((uint64_t)s * g.d) * F::LEN, mh);
}

// R and H_msg of each signature with one WARP per signature (kWarpHmsg
// families: the warp-parallel permutation), writing R into the signature and
// layer 0's chain lengths; k_sign_prep<F, true> does the rest.  Two
// signatures per 64-thread block.
template <class F>
__global__ void __launch_bounds__(64) k_sign_hmsg_warp(SignArgs g, const typename F::Ctx* __restrict__ ctx)
{
    const uint32_t s = blockIdx.x * 2 + (threadIdx.x >> 5);
    const uint32_t lane = threadIdx.x & 31;
    if (s >= g.count) return;
    uint8_t* sm = g.sm + g.sm_off[s];
    const uint64_t idx = g.idx[s];
    uint32_t R[F::NW], root[F::NW], mh[F::NW];
    F::prf_r(R, ctx[g.key[s]], idx);
    F::load(root, g.key_root + (uint64_t)g.key[s] * g.key_stride);
    hmsg_warp<F>(mh, R, root, idx, g.msg ? g.msg + g.msg_off[s] : sm + g.sig_bytes, g.mlen[s]);
    if (lane == 0) {
        F::store(sm + g.index_bytes, R);
        chain_lengths<F>(g.lens + ((uint64_t)s * g.d) * F::LEN, mh);
    }
}

// One thread per (signature, layer, chain): PRF_keygen then gen_chain(0,
// len_i) of wots_sign (wots.c:136-154).
template <class F>
__device__ __forceinline__ void sign_chain_one(const SignArgs& g, const typename F::Ctx& c, uint64_t item)
{
    const uint64_t sl = item / F::LEN;
    const uint32_t chain = (uint32_t)(item - sl * F::LEN);
    const uint32_t s = (uint32_t)(sl / g.d);
    const uint32_t layer = (uint32_t)(sl - (uint64_t)s * g.d);
    const uint64_t idx = g.idx[s];
    const uint32_t th = g.tree_height;
    const uint32_t leaf = (uint32_t)((idx >> (th * layer)) & ((1ull << th) - 1));
    const uint64_t tree = (th * (layer + 1) >= 64) ? 0 : idx >> (th * (layer + 1));
    const uint32_t steps = g.lens[item];
    uint32_t x[F::NW], a[8];
    set_addr(a, layer, tree, ADDR_OTS, leaf, chain, 0);
    run_chain<F>(x, c, a, 0, steps, true);
    const uint64_t wsb = (uint64_t)F::LEN * F::N;
    uint8_t* sig = g.sm + g.sm_off[s] + g.index_bytes + F::N + layer * (wsb + (uint64_t)th * F::N);
    F::store(sig + (uint64_t)chain * F::N, x);
}

template <class F>
__global__ void __launch_bounds__(128) k_sign_chains(SignArgs g, const typename F::Ctx* __restrict__ ctx)
{
    const uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= (uint64_t)g.count * g.d * F::LEN) return;
    sign_chain_one<F>(g, ctx[g.key[item / F::LEN / g.d]], item);
}

// ---------------------------------------------------------------------------
// Batched core_hash (hash.c:29-65) with a WOTS-style single-message stream:
// digest of M under the family's hash (SHA-256 [truncated], SHA-512,
// SHAKE128/256 with n output bytes).  Used to check the hash cores.
// ---------------------------------------------------------------------------
template <class F>
__global__ void k_core_hash(const uint8_t* __restrict__ msgs, const uint64_t* __restrict__ off,
                            const uint64_t* __restrict__ len, uint32_t count, uint8_t* __restrict__ out)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    const uint8_t* m = msgs + off[s];
    const uint64_t L = len[s];
    uint32_t o[F::NW];
    constexpr int K = HMsgKind<F>::v;
    if constexpr (K == 0) {
        const uint64_t nb = (L + 9 + 63) / 64;
        uint32_t st[8];
        sha256_iv(st);
        for (uint64_t b = 0; b < nb; b++) {
            uint32_t w[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const uint64_t p = 64 * b + 4 * j;
                uint32_t le = (p < L) ? fetch4_le(m, L, p) : 0;
                if (p <= L && L < p + 4) le |= 0x80u << (8 * (L - p));
                w[j] = bswap32(le);
            }
            if (b == nb - 1) {
                w[14] = (uint32_t)((L * 8) >> 32);
                w[15] = (uint32_t)(L * 8);
            }
            sha256_compress(st, w);
        }
#pragma unroll
        for (int i = 0; i < F::NW; i++) o[i] = st[i];
    } else if constexpr (K == 1) {
        const uint64_t nb = (L + 17 + 127) / 128;
        uint64_t st[8];
        sha512_iv(st);
        for (uint64_t b = 0; b < nb; b++) {
            uint64_t w[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                uint32_t hl[2];
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const uint64_t p = 128 * b + 8 * j + 4 * q;
                    uint32_t le = (p < L) ? fetch4_le(m, L, p) : 0;
                    if (p <= L && L < p + 4) le |= 0x80u << (8 * (L - p));
                    hl[q] = bswap32(le);
                }
                w[j] = join64(hl[0], hl[1]);
            }
            if (b == nb - 1) {
                w[14] = 0;
                w[15] = L * 8;
            }
            sha512_compress(st, w);
        }
#pragma unroll
        for (int i = 0; i < 8; i++) {
            if (2 * i < F::NW) o[2 * i] = (uint32_t)(st[i] >> 32);
            if (2 * i + 1 < F::NW) o[2 * i + 1] = (uint32_t)st[i];
        }
    } else {
        const uint64_t RB = 4 * K;
        const uint64_t nb = L / RB + 1;
        uint64_t A[25];
#pragma unroll
        for (int i = 0; i < 25; i++) A[i] = 0;
        for (uint64_t b = 0; b < nb; b++) {
#pragma unroll
            for (int i = 0; i < K / 2; i++) {
                uint32_t hl[2];
#pragma unroll
                for (int q = 0; q < 2; q++) {
                    const uint64_t p = RB * b + 8 * i + 4 * q;
                    uint32_t le = (p < L) ? fetch4_le(m, L, p) : 0;
                    if (p <= L && L < p + 4) le ^= 0x1Fu << (8 * (L - p));
                    hl[q] = le;
                }
                if (b == nb - 1 && 2 * i + 1 == K - 1) hl[1] ^= 0x80000000u;
                A[i] ^= ((uint64_t)hl[1] << 32) | hl[0];
            }
            keccak_f1600(A);
        }
#pragma unroll
        for (int i = 0; i < F::NW; i++) o[i] = (i & 1) ? (uint32_t)(A[i / 2] >> 32) : (uint32_t)A[i / 2];
    }
    F::store(out + (uint64_t)s * F::N, o);
}

}  // namespace xb
