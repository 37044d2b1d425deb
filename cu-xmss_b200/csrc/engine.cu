// Host engine of libxmss_b200 (see engine.h).
#include "engine.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <tuple>

#include "verify_persist.cuh"
#include "xmss_kernels.cuh"

namespace xb {

// Scratch budget of one chain launch when building trees: WOTS public keys
// of at most this many bytes are live at once (2 GiB; HBM is 180 GB, this
// keeps room for many concurrent tree node arrays).
constexpr uint64_t kChainScratchBytes = 2ull << 30;

DevBuf::~DevBuf()
{
    if (p_) cudaFree(p_);
}

void* DevBuf::get(size_t bytes)
{
    if (bytes == 0) bytes = 1;
    if (bytes > cap_) {
        size_t cap = std::max(bytes, cap_ + cap_ / 2);
        cap = (cap + 4095) & ~(size_t)4095;
        if (ordered_) {
            // stream-ordered: work already queued on order_ keeps the old
            // block until it has run; nothing else waits
            if (p_) XB_CUDA(cudaFreeAsync(p_, order_));
            p_ = nullptr;
            cap_ = 0;
            XB_CUDA(cudaMallocAsync(&p_, cap, order_));
        } else {
            if (p_) {
                XB_CUDA(cudaDeviceSynchronize());
                XB_CUDA(cudaFree(p_));
                p_ = nullptr;
                cap_ = 0;
            }
            XB_CUDA(cudaMalloc(&p_, cap));
        }
        cap_ = cap;
    }
    return p_;
}

void SplitStreams::create()
{
    // Equal priorities: giving the latency-bound phases (or one group) a
    // higher stream priority measured 7-14 % slower per batch.
    XB_CUDA(cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking));
    XB_CUDA(cudaStreamCreateWithFlags(&pre, cudaStreamNonBlocking));
    XB_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
    XB_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    XB_CUDA(cudaEventCreateWithFlags(&pre_done, cudaEventDisableTiming));
}

void SplitStreams::destroy()
{
    for (cudaStream_t* s : {&aux, &pre})
        if (*s) cudaStreamDestroy(*s), *s = nullptr;
    for (cudaEvent_t* e : {&fork, &join, &pre_done})
        if (*e) cudaEventDestroy(*e), *e = nullptr;
}

void Workspace::order_on(cudaStream_t st)
{
    for (DevBuf* b : {&ctx, &jobs, &refs, &wpk, &wpk2, &nodes, &keys, &node, &lens, &idx, &leaf, &hpre, &hist, &list,
                      &list2, &aux, &work, &pstate})
        b->order_on(st);
}

PinnedBuf::~PinnedBuf()
{
    if (p_) cudaFreeHost(p_);
    for (void* q : retired_) cudaFreeHost(q);
}

void* PinnedBuf::get(size_t bytes)
{
    if (bytes == 0) bytes = 1;
    if (bytes > cap_) {
        if (keep_old_) {
            // the owner guarantees no copy uses the old block when it grows;
            // it is kept (not freed: cudaFreeHost may wait for the device)
            size_t cap = std::max(bytes, 2 * cap_);
            cap = (cap + 4095) & ~(size_t)4095;
            if (p_) retired_.push_back(p_);
            p_ = nullptr;
            cap_ = 0;
            XB_CUDA(cudaMallocHost(&p_, cap));
            cap_ = cap;
            return p_;
        }
        size_t cap = std::max(bytes, cap_ + cap_ / 2);
        cap = (cap + 4095) & ~(size_t)4095;
        if (p_) {
            XB_CUDA(cudaDeviceSynchronize());
            XB_CUDA(cudaFreeHost(p_));
            p_ = nullptr;
            cap_ = 0;
        }
        XB_CUDA(cudaMallocHost(&p_, cap));
        cap_ = cap;
    }
    return p_;
}

// ---------------------------------------------------------------------------

const FamilyOps* family_ops(unsigned func, unsigned n)
{
    switch (func) {
        case XMSS_SHA2:
            if (n == 32) return &kOpsSha256N32;
            if (n == 24) return &kOpsSha256N24;
            if (n == 64) return &kOpsSha512N64;
            return nullptr;
        case XMSS_SHAKE128:
            return n == 32 ? &kOpsShake128N32 : nullptr;
        case XMSS_SHAKE256:
            if (n == 24) return &kOpsShake256N24;
            if (n == 32) return &kOpsShake256N32;
            if (n == 64) return &kOpsShake256N64;
            return nullptr;
        default:
            return nullptr;
    }
}

const FamilyOps* ops_for(const xmss_params& p)
{
    const FamilyOps* o = family_ops(p.func, p.n);
    if (!o || p.wots_w != 16) throw std::invalid_argument("parameter set has no GPU implementation");
    return o;
}

Engine& Engine::get()
{
    static std::mutex m;
    static Engine* e = nullptr;
    std::lock_guard<std::mutex> g(m);
    if (!e) {
        // The server runs up to ~30 streams at once; with the runtime's
        // default of 8 hardware work queues unrelated streams share a queue
        // and wait behind each other's kernels.  Effective only when this is
        // the process's first CUDA call; a caller's own setting wins.
        setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
        int dev = 0;
        const char* env = getenv("XMSS_B200_DEVICE");
        if (env) {
            dev = atoi(env);
        } else if (cudaGetDevice(&dev) != cudaSuccess) {
            dev = 0;
        }
        e = new Engine(dev);  // lives until exit
    }
    return *e;
}

Engine::Engine(int device) : device_(device)
{
    int n = 0;
    XB_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) throw CudaFailure("no CUDA device " + std::to_string(device));
    XB_CUDA(cudaSetDevice(device));
    XB_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    XB_CUDA(cudaEventCreateWithFlags(&done_, cudaEventDisableTiming));
    split_.create();
    work_ = s_work_.as<unsigned long long>(4);
    XB_CUDA(cudaMemset(work_, 0, 4 * sizeof(unsigned long long)));
}

Engine::~Engine() = default;

void Engine::begin(cudaStream_t st)
{
    XB_CUDA(cudaSetDevice(device_));
    if (have_done_) XB_CUDA(cudaStreamWaitEvent(st, done_, 0));
    if (profiling) {
        XB_CUDA(cudaEventSynchronize(done_));
        for (auto& m : marks_) {
            free_events_.push_back(m.a);
            free_events_.push_back(m.b);
        }
        marks_.clear();
    }
}

cudaEvent_t Engine::event()
{
    if (!free_events_.empty()) {
        cudaEvent_t e = free_events_.back();
        free_events_.pop_back();
        return e;
    }
    cudaEvent_t e;
    XB_CUDA(cudaEventCreate(&e));
    return e;
}

void Engine::mark(int phase, bool start, cudaStream_t st, bool on)
{
    if (!profiling || !on) return;
    if (start) {
        marks_.push_back(Mark{phase, event(), nullptr});
        XB_CUDA(cudaEventRecord(marks_.back().a, st));
    } else {
        marks_.back().b = event();
        XB_CUDA(cudaEventRecord(marks_.back().b, st));
    }
}

void Engine::phase_ms(double out[kPhases])
{
    for (int i = 0; i < kPhases; i++) out[i] = 0;
    XB_CUDA(cudaSetDevice(device_));
    if (have_done_) XB_CUDA(cudaEventSynchronize(done_));
    for (auto& m : marks_) {
        if (!m.b) continue;
        float ms = 0;
        XB_CUDA(cudaEventElapsedTime(&ms, m.a, m.b));
        out[m.phase] += ms;
    }
}

void Engine::end(cudaStream_t st)
{
    XB_CUDA(cudaGetLastError());
    XB_CUDA(cudaEventRecord(done_, st));
    have_done_ = true;
}

// ---------------------------------------------------------------------------
// Small byte-moving kernels (family independent).
// ---------------------------------------------------------------------------

// pk = root || PUB_SEED; sk = 0^ib || SK_SEED || SK_PRF || root || PUB_SEED
// (xmss_core.c:134-161) from seeds (SK_SEED || SK_PRF || PUB_SEED) and roots.
__global__ void k_keypair_finish(const uint8_t* __restrict__ seeds, const uint8_t* __restrict__ nodes,
                                 uint64_t tree_bytes, uint64_t root_off, uint32_t n, uint32_t ib,
                                 uint32_t sk_bytes, uint32_t count, uint8_t* __restrict__ pk, uint8_t* __restrict__ sk)
{
    const uint32_t k = blockIdx.x;
    if (k >= count) return;
    const uint8_t* seed = seeds + (uint64_t)k * 3 * n;
    const uint8_t* root = nodes + (uint64_t)k * tree_bytes + root_off;
    uint8_t* P = pk + (uint64_t)k * 2 * n;
    uint8_t* S = sk + (uint64_t)k * sk_bytes;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        P[i] = root[i];
        P[n + i] = seed[2 * n + i];
        S[ib + i] = seed[i];
        S[ib + n + i] = seed[n + i];
        S[ib + 2 * n + i] = root[i];
        S[ib + 3 * n + i] = seed[2 * n + i];
    }
    for (uint32_t i = threadIdx.x; i < ib; i += blockDim.x) S[i] = 0;
}

// ---------------------------------------------------------------------------
// Pipelines.
// ---------------------------------------------------------------------------

static void run_ltree(const FamilyOps* ops, const LeafRef* refs, uint32_t nslots, uint8_t* wpk, uint8_t* wpk2,
                      uint8_t* leaf_out, const void* ctx, const int* status, cudaStream_t st)
{
    int cnt = (int)ops->len, level = 0;
    uint8_t *src = wpk, *dst = wpk2;
    uint32_t sstr = ops->len, dstr = (ops->len + 1) / 2;
    while (cnt > 1) {
        ops->ltree_level(refs, nslots, level, cnt, src, sstr, dst, dstr, leaf_out, ctx, status, st);
        cnt = (cnt + 1) / 2;
        std::swap(src, dst);
        std::swap(sstr, dstr);
        level++;
    }
}

void Engine::build_trees(const FamilyOps* ops, const TreeJob* d_jobs, uint32_t njobs, int h, uint8_t* d_nodes,
                         const void* d_ctx, cudaStream_t st, Workspace& w, int subtree_k)
{
    const bool on = &w == &ws_;  // server workspaces record no marks
    if (subtree_k >= 5 && subtree_k <= 7 && subtree_k <= h) {
        // levels 0..k in one launch of in-CTA subtrees, the rest across CTAs
        mark(kChains, true, st, on);
        ops->keygen_subtree(d_jobs, njobs, h, subtree_k, d_ctx, d_nodes, st);
        mark(kChains, false, st, on);
        mark(kTree, true, st, on);
        for (int level = subtree_k; level < h; level++) ops->tree_level(d_jobs, njobs, h, level, d_nodes, d_ctx, st);
        mark(kTree, false, st, on);
        return;
    }
    const uint64_t total = (uint64_t)njobs << h;
    const uint64_t per_slot = (uint64_t)ops->len * ops->n;
    const uint64_t cap = std::max<uint64_t>(1, std::min<uint64_t>(total, kChainScratchBytes / per_slot));
    uint8_t* wpk = w.wpk.as<uint8_t>(cap * per_slot);
    uint8_t* wpk2 = w.wpk2.as<uint8_t>(cap * ((ops->len + 1) / 2) * ops->n);
    LeafRef* refs = w.refs.as<LeafRef>(cap);
    for (uint64_t s0 = 0; s0 < total; s0 += cap) {
        const uint64_t ns = std::min(cap, total - s0);
        mark(kChains, true, st, on);
        ops->keygen_chains(d_jobs, h, s0, ns, d_ctx, wpk, refs, st);
        mark(kChains, false, st, on);
        mark(kLtree, true, st, on);
        run_ltree(ops, refs, (uint32_t)ns, wpk, wpk2, d_nodes, d_ctx, nullptr, st);
        mark(kLtree, false, st, on);
    }
    mark(kTree, true, st, on);
    for (int level = 0; level < h; level++) ops->tree_level(d_jobs, njobs, h, level, d_nodes, d_ctx, st);
    mark(kTree, false, st, on);
}

void Engine::keypair(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* d_seeds,
                     uint8_t* d_pk, uint8_t* d_sk, cudaStream_t st, Workspace& w, bool wait)
{
    if (!count) return;
    const uint32_t n = p.n, th = p.tree_height;
    void* ctx = w.ctx.get((size_t)count * ops->ctx_bytes);
    ops->make_ctx(d_seeds + 2 * n, 3 * n, d_seeds, 3 * n, d_seeds + n, 3 * n, count, ctx, st);
    const uint64_t tree_bytes = ((2ull << th) - 1) * n;
    TreeJob* hj = w.h_jobs.as<TreeJob>(count);
    for (uint32_t k = 0; k < count; k++) hj[k] = TreeJob{k, p.d - 1, 0, (uint64_t)k * tree_bytes};
    TreeJob* dj = w.jobs.as<TreeJob>(count);
    XB_CUDA(cudaMemcpyAsync(dj, hj, count * sizeof(TreeJob), cudaMemcpyHostToDevice, st));
    uint8_t* nodes = w.nodes.as<uint8_t>(count * tree_bytes);
    build_trees(ops, dj, count, (int)th, nodes, ctx, st, w, subtree_k(p, count));
    k_keypair_finish<<<count, 64, 0, st>>>(d_seeds, nodes, tree_bytes, level_offset((int)th, (int)th) * n, n,
                                          p.index_bytes, (uint32_t)p.sk_bytes, count, d_pk, d_sk);
    // the host job list is reused by the next call only after this one's
    // copy has been consumed
    if (wait) XB_CUDA(cudaStreamSynchronize(st));
}

// One launch sequence of verify (prep, then per layer: bucket, chains, L-tree,
// root) over the signatures v selects, on stream st.  With hpre_ready the
// caller has launched the prep's parts itself: the H_msg part ahead on st,
// the h_pre part elsewhere, ending at that event, which the first L-tree
// waits for.
void Engine::verify_sequence(const FamilyOps* ops, const xmss_params& p, const VerifyArgs& v, const void* ctx,
                             cudaStream_t st, bool on, bool fused_ltree, cudaEvent_t hpre_ready)
{
    const uint32_t len = ops->len;
    if (!hpre_ready) {
        mark(kPrep, true, st, on);
        ops->verify_prep(v, ctx, st);
        mark(kPrep, false, st, on);
    }
    for (uint32_t layer = 0; layer < p.d; layer++) {
        mark(kChains, true, st, on);
        ops->verify_scatter(v, layer, st);
        ops->verify_chains(v, layer, ctx, st);
        mark(kChains, false, st, on);
        if (layer == 0 && hpre_ready) XB_CUDA(cudaStreamWaitEvent(st, hpre_ready, 0));
        mark(kLtree, true, st, on);
        if (fused_ltree) {
            ops->verify_ltree_warp(v, layer, st);
        } else {
            int cnt = (int)len;
            uint32_t node_base = 0;
            uint8_t *src = v.wpk, *dst = v.wpk2;
            uint32_t sstr = len, dstr = (len + 1) / 2;
            while (cnt > 1) {
                ops->verify_ltree(v, layer, cnt, node_base, src, sstr, dst, dstr, st);
                node_base += cnt / 2;
                cnt = (cnt + 1) / 2;
                std::swap(src, dst);
                std::swap(sstr, dstr);
            }
        }
        mark(kLtree, false, st, on);
        mark(kRoot, true, st, on);
        ops->verify_root(v, layer, st);
        mark(kRoot, false, st, on);
    }
}

void Engine::verify(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* d_sm,
                    const uint64_t* d_sm_off, const uint64_t* d_smlen, const uint8_t* d_pk, uint32_t npk,
                    const uint32_t* d_pk_index, int* d_status, cudaStream_t st, Workspace& w, bool allow_split)
{
    // the engine's own calls report their work through xmss_b200_last_verify_work;
    // other workspaces (server slots) count into their own buffer and record no marks
    const bool own = &w == &ws_;
    unsigned long long* work = own ? work_ : w.work.as<unsigned long long>(4);
    XB_CUDA(cudaMemsetAsync(work, 0, 3 * sizeof(unsigned long long), st));
    if (!count) return;
    const uint32_t n = p.n, len = ops->len, nh = len - 1 + p.tree_height;
    void* ctx = w.ctx.get((size_t)npk * ops->ctx_bytes);
    ops->make_ctx(d_pk + n, 2 * n, nullptr, 0, nullptr, 0, npk, ctx, st);
    VerifyArgs v;
    v.sm = d_sm;
    v.sm_off = d_sm_off;
    v.smlen = d_smlen;
    v.key = d_pk_index;
    v.key_root = d_pk;
    v.key_stride = 2 * n;
    v.npk = npk;
    v.node = w.node.as<uint8_t>((size_t)count * n);
    v.lens = w.lens.as<uint8_t>((size_t)count * len);
    v.idx = w.idx.as<uint64_t>(count);
    v.status = d_status;
    v.wpk = w.wpk.as<uint8_t>((size_t)count * len * n);
    v.wpk2 = w.wpk2.as<uint8_t>((size_t)count * ((len + 1) / 2) * n);
    v.leaf = w.leaf.as<uint8_t>((size_t)count * n);
    v.refs = w.refs.as<LeafRef>(count);
    v.hpre = w.hpre.get((size_t)count * p.d * nh * ops->hpre_bytes);
    uint32_t* hist = w.hist.as<uint32_t>(2 * 32 * p.d + 2);  // two groups + 2 group sizes
    uint32_t* list = w.list.as<uint32_t>((size_t)count * len + 2 * (size_t)count);
    v.hist = hist;
    v.list = list;
    v.sel = nullptr;
    v.sel_n = nullptr;
    v.work = work;
    v.count = count;
    v.index_bytes = p.index_bytes;
    v.sig_bytes = p.sig_bytes;
    v.tree_height = p.tree_height;
    v.d = p.d;
    XB_CUDA(cudaMemsetAsync(hist, 0, (2 * 32 * p.d + 2) * sizeof(uint32_t), st));
    // Large batches run as two groups on two streams: signatures whose
    // H_msg is short start their chains at once while the long messages are
    // still being hashed (H_msg is a serial chain of compressions).  The
    // profiling pass keeps one sequence so each kernel's time is its own.
    SplitStreams* ss = own ? &split_ : w.split;
    const Tuning& tn = tuning_for(ops->func, ops->n);
    if (!allow_split || count < tn.split_min || profiling || !ss) {
        verify_sequence(ops, p, v, ctx, st, own, count < kFusedLtreeBelow);
        return;
    }
    uint32_t* n2 = hist + 2 * 32 * p.d;
    uint32_t* sel_short = list + (size_t)count * len;
    uint32_t* sel_long = sel_short + count;
    ops->verify_partition(v, tn.short_hmsg_blocks, sel_short, sel_long, n2, st);
    VerifyArgs a = v, b = v;
    a.sel = sel_short;
    a.sel_n = n2;
    b.sel = sel_long;
    b.sel_n = n2 + 1;
    b.hist = hist + 32 * p.d;
    b.list = w.list2.as<uint32_t>((size_t)count * len);  // each group has its own chain list
    XB_CUDA(cudaEventRecord(ss->fork, st));
    XB_CUDA(cudaStreamWaitEvent(ss->aux, ss->fork, 0));
    if (tn.prep_split) {
        // Each group's chains wait only for its own H_msg; the h_pre items
        // of both groups run as one launch on a third stream, enqueued
        // after the two H_msg launches so these get their CTAs first, and
        // only the L-trees wait for it.
        XB_CUDA(cudaStreamWaitEvent(ss->pre, ss->fork, 0));
        ops->verify_prep_part(b, ctx, ss->aux, 1);
        ops->verify_prep_part(a, ctx, st, 1);
        ops->verify_prep_part(v, ctx, ss->pre, 2);
        XB_CUDA(cudaEventRecord(ss->pre_done, ss->pre));
        verify_sequence(ops, p, b, ctx, ss->aux, own, false, ss->pre_done);
        verify_sequence(ops, p, a, ctx, st, own, false, ss->pre_done);
    } else {
        verify_sequence(ops, p, b, ctx, ss->aux, own);
        verify_sequence(ops, p, a, ctx, st, own);
    }
    XB_CUDA(cudaEventRecord(ss->join, ss->aux));
    XB_CUDA(cudaStreamWaitEvent(st, ss->join, 0));
}

namespace {

// Keys and subtrees of `count` sign requests, staged to the device.
struct SignPlan {
    const uint8_t* keys;      // nkeys rows of SK_SEED | SK_PRF | root | PUB_SEED (4n)
    const TreeJob* jobs;      // njobs distinct (key, layer, tree) subtrees
    const uint64_t* tree_off; // [count][d] node array of each request's subtree per layer
    const uint64_t* idx;      // [count]
    const uint32_t* key;      // [count] row in keys
    const uint8_t* ibytes;    // [count][8] index bytes (when given)
    uint32_t nkeys, njobs;
};

SignPlan plan_sign(const xmss_params& p, uint32_t count, const uint8_t* h_sk, const uint64_t* h_idx,
                   const uint8_t* h_ibytes, Workspace& w, cudaStream_t st)
{
    const uint32_t n = p.n, th = p.tree_height, d = p.d, ib = p.index_bytes;
    const uint64_t skb = p.sk_bytes;
    // Keys: distinct (SK_SEED, SK_PRF, root, PUB_SEED) tuples.
    std::map<std::string, uint32_t> keyidx;
    std::vector<uint32_t> req_key(count);
    std::vector<uint8_t> keymat;  // nkeys x 4n
    for (uint32_t r = 0; r < count; r++) {
        std::string k((const char*)h_sk + r * skb + ib, 4 * n);
        auto it = keyidx.find(k);
        if (it == keyidx.end()) {
            it = keyidx.emplace(k, (uint32_t)keyidx.size()).first;
            keymat.insert(keymat.end(), k.begin(), k.end());
        }
        req_key[r] = it->second;
    }
    const uint32_t nkeys = (uint32_t)keyidx.size();
    // Subtrees: distinct (key, layer, tree).
    const uint64_t tree_bytes = ((2ull << th) - 1) * n;
    std::map<std::tuple<uint32_t, uint32_t, uint64_t>, uint32_t> jobidx;
    std::vector<TreeJob> jobs;
    std::vector<uint64_t> tree_off((size_t)count * d);
    for (uint32_t r = 0; r < count; r++) {
        for (uint32_t l = 0; l < d; l++) {
            const uint32_t sh = th * (l + 1);
            const uint64_t tree = sh >= 64 ? 0 : (h_idx[r] >> sh);
            auto key = std::make_tuple(req_key[r], l, tree);
            auto it = jobidx.find(key);
            if (it == jobidx.end()) {
                it = jobidx.emplace(key, (uint32_t)jobs.size()).first;
                jobs.push_back(TreeJob{req_key[r], l, tree, (uint64_t)jobs.size() * tree_bytes});
            }
            tree_off[(size_t)r * d + l] = jobs[it->second].node_off;
        }
    }
    const uint32_t njobs = (uint32_t)jobs.size();
    // Stage everything in one pinned block and one device block.
    const size_t sz_keys = (size_t)nkeys * 4 * n, sz_jobs = njobs * sizeof(TreeJob),
                 sz_toff = tree_off.size() * sizeof(uint64_t), sz_idx = count * sizeof(uint64_t),
                 sz_key = count * sizeof(uint32_t), sz_ib = h_ibytes ? (size_t)count * 8 : 0;
    auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
    const size_t o_jobs = al(sz_keys), o_toff = o_jobs + al(sz_jobs), o_idx = o_toff + al(sz_toff),
                 o_key = o_idx + al(sz_idx), o_ib = o_key + al(sz_key), total = o_ib + al(sz_ib);
    uint8_t* hs = w.h_jobs.as<uint8_t>(total);
    memcpy(hs, keymat.data(), sz_keys);
    memcpy(hs + o_jobs, jobs.data(), sz_jobs);
    memcpy(hs + o_toff, tree_off.data(), sz_toff);
    memcpy(hs + o_idx, h_idx, sz_idx);
    memcpy(hs + o_key, req_key.data(), sz_key);
    if (sz_ib) memcpy(hs + o_ib, h_ibytes, sz_ib);
    uint8_t* ds = w.keys.as<uint8_t>(total);
    XB_CUDA(cudaMemcpyAsync(ds, hs, total, cudaMemcpyHostToDevice, st));
    return SignPlan{ds, (const TreeJob*)(ds + o_jobs), (const uint64_t*)(ds + o_toff), (const uint64_t*)(ds + o_idx),
                    (const uint32_t*)(ds + o_key), sz_ib ? ds + o_ib : nullptr, nkeys, njobs};
}

}  // namespace

void Engine::persist_setup(const PersistJob& j, Workspace& w, VerifyArgs& v, PersistArgs& q, cudaStream_t st)
{
    const FamilyOps* ops = j.ops;
    const xmss_params& p = j.p;
    const uint32_t count = j.count, npk = j.npk;
    const uint32_t n = p.n, len = ops->len, d = p.d, nh = len - 1 + p.tree_height;
    const uint32_t groups = (count + 31) / 32;
    v = VerifyArgs{};
    v.sm = j.d_sm;
    v.sm_off = j.d_sm_off;
    v.smlen = j.d_smlen;
    v.key = j.d_pk_index;
    v.key_root = j.d_pk;
    v.key_stride = 2 * n;
    v.npk = npk;
    v.node = w.node.as<uint8_t>((size_t)count * n);
    v.lens = w.lens.as<uint8_t>((size_t)count * len);
    v.idx = w.idx.as<uint64_t>(count);
    v.status = j.d_status;
    v.wpk = w.wpk.as<uint8_t>((size_t)count * len * n);
    v.wpk2 = w.wpk2.as<uint8_t>((size_t)count * ((len + 1) / 2) * n);
    v.leaf = w.leaf.as<uint8_t>((size_t)count * n);
    v.hpre = w.hpre.get((size_t)count * d * nh * ops->hpre_bytes);
    v.work = work_;
    v.count = count;
    v.index_bytes = p.index_bytes;
    v.sig_bytes = p.sig_bytes;
    v.tree_height = p.tree_height;
    v.d = d;
    // state: ticket (8 B), header, then per (group, layer) ready / ntot /
    // chains_done / 8 L-tree level counters, then per group h_pre counters
    const size_t gl = (size_t)groups * d;
    const size_t words = 4 + gl * 11 + groups;
    uint8_t* st8 = w.pstate.as<uint8_t>(8 + words * 4);
    uint32_t* u = (uint32_t*)(st8 + 8);
    q = PersistArgs{};
    q.ticket = (unsigned long long*)st8;
    q.hdr = u;
    q.ready = u + 4;
    q.ntot = q.ready + gl;
    q.chains_done = q.ntot + gl;
    q.lt_done = q.chains_done + gl;
    q.hpre_done = q.lt_done + 8 * gl;
    q.list = w.list.as<uint32_t>((size_t)groups * 32 * len);
    q.ctx = w.ctx.get((size_t)npk * ops->ctx_bytes);
    q.npk = npk;
    q.groups = groups;
    q.wait_ns = persist_wait_ns;
    XB_CUDA(cudaMemsetAsync(st8, 0, 8 + words * 4, st));
}

void Engine::verify_persistent(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* d_sm,
                               const uint64_t* d_sm_off, const uint64_t* d_smlen, const uint8_t* d_pk, uint32_t npk,
                               const uint32_t* d_pk_index, int* d_status, cudaStream_t st)
{
    XB_CUDA(cudaMemsetAsync(work_, 0, 3 * sizeof(unsigned long long), st));
    if (!count) return;
    VerifyArgs v;
    PersistArgs q;
    PersistJob j;
    j.ops = ops;
    j.p = p;
    j.count = count;
    j.d_sm = d_sm;
    j.d_sm_off = d_sm_off;
    j.d_smlen = d_smlen;
    j.d_pk = d_pk;
    j.npk = npk;
    j.d_pk_index = d_pk_index;
    j.d_status = d_status;
    persist_setup(j, ws_, v, q, st);
    ops->verify_persist(v, q, st);
    XB_CUDA(cudaGetLastError());
}

void Engine::gen_setup(const PersistJob& j, Workspace& w, PersistBatch& J, cudaStream_t st)
{
    const FamilyOps* ops = j.ops;
    const xmss_params& p = j.p;
    const uint32_t n = p.n, len = ops->len, h = p.tree_height;
    J = PersistBatch{};
    J.kind = j.kind;
    TreeTask& T = J.t;
    if (j.kind == kJobKeygen) {
        // one top-layer subtree per key (xmss_core.c:134-161)
        const uint64_t tree_bytes = ((2ull << h) - 1) * n;
        TreeJob* hj = w.h_jobs.as<TreeJob>(j.count);
        for (uint32_t k = 0; k < j.count; k++) hj[k] = TreeJob{k, p.d - 1, 0, (uint64_t)k * tree_bytes};
        TreeJob* dj = w.jobs.as<TreeJob>(j.count);
        XB_CUDA(cudaMemcpyAsync(dj, hj, j.count * sizeof(TreeJob), cudaMemcpyHostToDevice, st));
        T.trees = dj;
        T.ntrees = T.nkeys = j.count;
        T.keys = j.d_seeds;  // SK_SEED || SK_PRF || PUB_SEED
        T.key_stride = 3 * n;
        T.off_pub = 2 * n;
        T.off_sks = 0;
        T.off_skp = n;
        T.seeds = j.d_seeds;
        T.pk = j.d_pk_out;
        T.sk = j.d_sk_out;
        T.index_bytes = p.index_bytes;
        T.sk_bytes = (uint32_t)p.sk_bytes;
    } else {
        const SignPlan sp = plan_sign(p, j.count, j.h_sk, j.h_idx, j.h_ibytes, w, st);
        T.trees = sp.jobs;
        T.ntrees = sp.njobs;
        T.nkeys = sp.nkeys;
        T.keys = sp.keys;  // SK_SEED | SK_PRF | root | PUB_SEED
        T.key_stride = 4 * n;
        T.off_pub = 3 * n;
        T.off_sks = 0;
        T.off_skp = n;
        T.ibytes = sp.ibytes;
        SignArgs& g = J.g;
        g.sm = j.d_sign_sm;
        g.sm_off = j.d_sm_off;
        g.mlen = j.d_mlen;
        g.msg = nullptr;
        g.msg_off = nullptr;
        g.idx = sp.idx;
        g.key = sp.key;
        g.key_root = sp.keys + 2 * n;
        g.key_stride = 4 * n;
        g.tree_off = sp.tree_off;
        g.lens = w.lens.as<uint8_t>((size_t)j.count * p.d * len);
        g.count = j.count;
        g.index_bytes = p.index_bytes;
        g.sig_bytes = p.sig_bytes;
        g.tree_height = h;
        g.d = p.d;
    }
    T.h = h;
    const uint64_t tree_bytes = ((2ull << h) - 1) * n;
    T.nodes = w.nodes.as<uint8_t>(T.ntrees * tree_bytes);
    J.g.nodes = T.nodes;
    const uint64_t slots = (uint64_t)T.ntrees << h;
    T.wpk = w.wpk.as<uint8_t>(slots * len * n);
    T.wpk2 = w.wpk2.as<uint8_t>(slots * ((len + 1) / 2) * n);
    // state: header, per leaf group the chain and L-tree counters, per
    // subtree its level counters, subtrees done, preparation tasks done
    const size_t groups = slots >> 5;
    const size_t words = 4 + groups * 9 + (size_t)T.ntrees * (h + 1) + 2;
    uint32_t* u = w.pstate.as<uint32_t>(words);
    J.q.hdr = u;
    T.chains_done = u + 4;
    T.lt_done = T.chains_done + groups;
    T.lvl_done = T.lt_done + 8 * groups;
    T.trees_done = T.lvl_done + (size_t)T.ntrees * (h + 1);
    T.prep_done = T.trees_done + 1;
    J.q.ctx = w.ctx.get((size_t)T.nkeys * ops->ctx_bytes);
    J.q.wait_ns = persist_wait_ns;
    XB_CUDA(cudaMemsetAsync(u, 0, words * 4, st));
}

void Engine::persistent_multi(const std::vector<PersistJob>& jobs, cudaStream_t st, PersistScratch& scratch)
{
    XB_CUDA(cudaMemsetAsync(work_, 0, 3 * sizeof(unsigned long long), st));
    // launches: the batches of one family, at most kMaxPersistJobs each
    std::vector<std::vector<size_t>> launches;
    std::map<const FamilyOps*, size_t> open;
    for (size_t i = 0; i < jobs.size(); i++) {
        if (!jobs[i].count) continue;
        auto it = open.find(jobs[i].ops);
        if (it == open.end() || launches[it->second].size() == kMaxPersistJobs) {
            open[jobs[i].ops] = launches.size();
            launches.emplace_back();
        }
        launches[open[jobs[i].ops]].push_back(i);
    }
    if (launches.empty()) return;
    while (scratch.ws.size() < jobs.size()) scratch.ws.emplace_back(new Workspace());
    while (pstreams_.size() + 1 < launches.size()) {
        cudaStream_t s;
        cudaEvent_t e;
        XB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        XB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        pstreams_.push_back(s);
        pjoin_.push_back(e);
    }
    if (!pfork_) XB_CUDA(cudaEventCreateWithFlags(&pfork_, cudaEventDisableTiming));
    // a ticket counter and an exit counter per launch, zeroed before the fork
    unsigned long long* ctr = scratch.ctr.as<unsigned long long>(2 * launches.size());
    XB_CUDA(cudaMemsetAsync(ctr, 0, 2 * launches.size() * sizeof(unsigned long long), st));
    XB_CUDA(cudaEventRecord(pfork_, st));
    for (size_t l = 0; l < launches.size(); l++) {
        cudaStream_t s = l == 0 ? st : pstreams_[l - 1];
        if (l) XB_CUDA(cudaStreamWaitEvent(s, pfork_, 0));
        PersistJobs P{};
        P.njobs = (uint32_t)launches[l].size();
        P.ticket = ctr + 2 * l;
        P.exited = (uint32_t*)(ctr + 2 * l + 1);
        uint32_t phases = 1;
        for (uint32_t k = 0; k < P.njobs; k++) {
            const size_t i = launches[l][k];
            PersistBatch& J = P.job[k];
            if (jobs[i].kind == kJobVerify) {
                J = PersistBatch{};
                J.kind = kJobVerify;
                persist_setup(jobs[i], *scratch.ws[i], J.v, J.q, s);
                phases = std::max(phases, 1 + J.v.d);
            } else {
                gen_setup(jobs[i], *scratch.ws[i], J, s);
            }
        }
        // segments: phase 0 of every batch (a verify batch's contexts, H_msg
        // and h_pre; a whole keygen or sign batch), then each layer of every
        // verify batch that has it
        P.nsegs = 0;
        P.first[0] = 0;
        for (uint32_t ph = 0; ph < phases; ph++) {
            for (uint32_t k = 0; k < P.njobs; k++) {
                const PersistBatch& J = P.job[k];
                const unsigned long long len = jobs[launches[l][k]].ops->len;
                unsigned long long a = 0, cnt = 0;
                if (J.kind != kJobVerify) {
                    if (ph) continue;
                    cnt = gen_total(J, (int)len);
                } else {
                    const VerifyArgs& v = J.v;
                    const PersistArgs& q = J.q;
                    if (ph > v.d) continue;
                    const unsigned long long G = q.groups, K = (q.npk + 31) / 32;
                    const unsigned long long head = K + G + G * v.d * (len - 1 + v.tree_height);
                    const unsigned long long per_layer = G * (len + lt_items_total((int)len) + 1);
                    a = ph == 0 ? 0 : head + (ph - 1) * per_layer;
                    cnt = ph == 0 ? head : per_layer;
                }
                P.seg_job[P.nsegs] = (uint8_t)k;
                P.local0[P.nsegs] = a;
                P.first[P.nsegs + 1] = P.first[P.nsegs] + cnt;
                P.nsegs++;
            }
        }
        jobs[launches[l][0]].ops->verify_persist_multi(P, s);
        XB_CUDA(cudaGetLastError());
        if (l) {
            XB_CUDA(cudaEventRecord(pjoin_[l - 1], s));
            XB_CUDA(cudaStreamWaitEvent(st, pjoin_[l - 1], 0));
        }
    }
}

void Engine::last_verify_work(unsigned long long out[3])
{
    XB_CUDA(cudaSetDevice(device_));
    if (have_done_) XB_CUDA(cudaEventSynchronize(done_));
    XB_CUDA(cudaMemcpy(out, work_, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
}


void Engine::sign(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* h_sk,
                  const uint64_t* h_idx, uint8_t* d_sm, const uint64_t* d_sm_off, const uint64_t* d_mlen,
                  cudaStream_t st, Workspace& w, bool wait)
{
    if (!count) return;
    const uint32_t n = p.n, th = p.tree_height, d = p.d;
    const SignPlan sp = plan_sign(p, count, h_sk, h_idx, nullptr, w, st);
    void* ctx = w.ctx.get((size_t)sp.nkeys * ops->ctx_bytes);
    // key material rows: SK_SEED | SK_PRF | root | PUB_SEED
    ops->make_ctx(sp.keys + 3 * n, 4 * n, sp.keys, 4 * n, sp.keys + n, 4 * n, sp.nkeys, ctx, st);
    const uint64_t tree_bytes = ((2ull << th) - 1) * n;
    uint8_t* nodes = w.nodes.as<uint8_t>(sp.njobs * tree_bytes);
    SignArgs g;
    g.sm = d_sm;
    g.sm_off = d_sm_off;
    g.mlen = d_mlen;
    g.msg = nullptr;  // messages follow the signatures in d_sm
    g.msg_off = nullptr;
    g.idx = sp.idx;
    g.key = sp.key;
    g.key_root = sp.keys + 2 * n;
    g.key_stride = 4 * n;
    g.tree_off = sp.tree_off;
    g.nodes = nodes;
    g.lens = w.lens.as<uint8_t>((size_t)count * d * ops->len);
    g.count = count;
    g.index_bytes = p.index_bytes;
    g.sig_bytes = p.sig_bytes;
    g.tree_height = th;
    g.d = d;
    // R and H_msg read only the key contexts and the messages: they run on
    // a second stream beside the subtree builds (a 64 KB message is ~1,000
    // compressions in a row), and the rest of the preparation waits for both.
    // The profiling pass keeps one sequence so each kernel's time is its own.
    SplitStreams* ss = &w == &ws_ ? &split_ : w.split;
    if (ss && !profiling) {
        XB_CUDA(cudaEventRecord(ss->fork, st));
        XB_CUDA(cudaStreamWaitEvent(ss->aux, ss->fork, 0));
        ops->sign_hmsg(g, ctx, ss->aux);
        XB_CUDA(cudaEventRecord(ss->join, ss->aux));
        build_trees(ops, sp.jobs, sp.njobs, (int)th, nodes, ctx, st, w, subtree_k(p, sp.njobs));
        XB_CUDA(cudaStreamWaitEvent(st, ss->join, 0));
        ops->sign_prep_rest(g, ctx, st);
    } else {
        build_trees(ops, sp.jobs, sp.njobs, (int)th, nodes, ctx, st, w, subtree_k(p, sp.njobs));
        mark(kRoot, true, st);
        ops->sign_prep(g, ctx, st);
        mark(kRoot, false, st);
    }
    mark(kChains, true, st);
    ops->sign_chains(g, ctx, st);
    mark(kChains, false, st);
    if (wait) XB_CUDA(cudaStreamSynchronize(st));  // staging buffers are reused by the next call
}

void Engine::core_hash(const FamilyOps* ops, uint32_t count, const uint8_t* d_in, const uint64_t* d_off,
                       const uint64_t* d_len, uint8_t* d_out, cudaStream_t st)
{
    ops->core_hash(d_in, d_off, d_len, count, d_out, st);
}

}  // namespace xb
