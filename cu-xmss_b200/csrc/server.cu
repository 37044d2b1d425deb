// Serving loop of libxmss_b200 (the xmss_b200_server_* entry points):
// sign / verify requests admitted as they arrive, batched continuously onto
// the GPU, over keys whose state lives in device memory.
//
// Threads.  Callers queue requests (mu).  One dispatcher thread owns the
// batch slots: whenever a slot is free it takes what is queued, plans it on
// the host and launches it on the slot's stream, then goes back to the queue
// while that batch runs, so several batches overlap on the device.  Planning
// and launching, and reaping finished slots, hold launch_mu, which add_key
// also takes before it touches the key tables.  A monitor thread reads the
// device's free memory for admission every 20 ms.
//
// Signing with resident keys.  The reference recomputes the whole subtree
// for every signature (treehash, xmss_core.c:253-270).  Here each subtree a
// signature needs is built once into a pooled device cache (LRU eviction of
// subtrees no in-flight batch uses), and a signature is R, H_msg and each
// layer's WOTS signature plus an authentication path copied from the cache:
// the bytes xmssmt_core_sign writes.
//
// One-time indices.  Each resident key has a u64 counter in device memory.
// A slot's batch reserves n consecutive indices per key with one atomicAdd,
// on a single index stream shared by all slots, in launch order; batches
// are launched in queue order, so a key's requests get its indices in
// submission order.  The host keeps a mirror of each counter to plan the
// subtrees; the device result is compared with the plan and any difference
// fails the batch.  The reference's last index 2^h - 1 (signed after the key
// is wiped, xmss_core.c:212-231) is never issued: -2 from there on.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/params.h"
#include "../../include/xmss_b200.h"
#include "engine.h"
#include "xmss_kernels.cuh"

namespace xb {
void set_last_error(const std::string& msg);  // api.cu
}

namespace {

using Clock = std::chrono::steady_clock;

// ---------------------------------------------------------------------------
// Index kernels.
// ---------------------------------------------------------------------------

// Group g (one key of one batch) takes n[g] consecutive indices of the
// counter at address counter_addr[g].
__global__ void k_serve_reserve(const uint64_t* __restrict__ counter_addr, const uint32_t* __restrict__ n,
                                uint32_t groups, unsigned long long* __restrict__ base)
{
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g < groups) base[g] = atomicAdd((unsigned long long*)counter_addr[g], (unsigned long long)n[g]);
}

// Index of request r = its group's base + its rank in the group; any
// difference from the host's plan is flagged.
__global__ void k_serve_index(const unsigned long long* __restrict__ base, const uint32_t* __restrict__ group,
                              const uint32_t* __restrict__ rank, const uint64_t* __restrict__ planned,
                              uint32_t count, uint64_t* __restrict__ idx, int* __restrict__ mismatch)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= count) return;
    const uint64_t i = base[group[r]] + rank[r];
    idx[r] = i;
    if (i != planned[r]) atomicExch(mismatch, 1);
}

uint64_t be_read(const uint8_t* p, unsigned len)
{
    uint64_t r = 0;
    for (unsigned i = 0; i < len; i++) r = (r << 8) | p[i];
    return r;
}

void be_write(uint8_t* p, unsigned len, uint64_t v)
{
    for (int i = (int)len - 1; i >= 0; i--) {
        p[i] = (uint8_t)(v & 0xff);
        v >>= 8;
    }
}

constexpr size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }
constexpr size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

bool parse(int mt, uint32_t oid, xmss_params* p)
{
    return (mt ? xmssmt_parse_oid(p, oid) : xmss_parse_oid(p, oid)) == 0;
}

// ---------------------------------------------------------------------------
// Server state.
// ---------------------------------------------------------------------------

// Keys of one parameter set: device rows indexed by the key's row.
struct KeyTable {
    xmss_params p{};
    const xb::FamilyOps* ops = nullptr;
    uint32_t count = 0, cap = 0;
    xb::DevBuf ctx;       // cap x ctx_bytes
    xb::DevBuf mat;       // cap x 4n: SK_SEED | SK_PRF | root | PUB_SEED
    xb::DevBuf counters;  // cap x u64: next one-time index
};

struct Key {
    uint32_t oid = 0;
    int mt = 0;
    xmss_params p{};
    KeyTable* table = nullptr;
    uint32_t row = 0;
    uint64_t next = 0;   // host mirror of the device counter
    uint64_t limit = 0;  // first index refused (2^h - 1)
    std::vector<uint8_t> mat;
};

struct TreeEntry {
    uint64_t off = 0, cap = 0;    // region of the pool
    cudaEvent_t ready = nullptr;  // recorded on the building stream after the build
    bool settled = false;         // the build has completed
    uint64_t last_use = 0;
    uint64_t pinned_batch = 0;  // last batch that pinned it
    int pins = 0;               // in-flight batches using it
};
using TreeId = std::tuple<uint32_t, uint32_t, uint64_t>;  // key, layer, tree

struct Request {
    uint64_t tag = 0;
    uint32_t kind = 0;  // 0 sign, 1 verify, 2 warm
    uint32_t key_id = 0;
    int mt = 0;
    uint32_t oid = 0;
    xmss_params p{};
    const uint8_t* in = nullptr;  // sign: message; verify: signed message
    uint64_t inlen = 0;
    uint8_t* sm_out = nullptr;  // sign
    uint64_t* smlen_out = nullptr;
    std::vector<uint8_t> pk;  // verify: root || PUB_SEED
    Clock::time_point t0;
    int ret = 0;
    uint64_t idx = 0;      // sign: planned index
    uint64_t out_off = 0;  // staging offset of its result
    bool deferred = false;  // its subtrees did not fit the pool this time
};

// One stream of a slot with its own scratch: the plans of a batch (one per
// operation and parameter set) run side by side on the slot's lanes.
struct Lane {
    cudaStream_t st = nullptr;
    cudaEvent_t start = nullptr, done = nullptr;  // timing events
    xb::Workspace w;
    uint32_t kind = 0, oid = 0;  // plan of the current batch
};

struct Slot {
    cudaStream_t st = nullptr;  // copies in and out; joins the lanes
    cudaEvent_t done = nullptr, staged = nullptr, reserved = nullptr;
    std::vector<std::unique_ptr<Lane>> lanes;
    xb::PinnedBuf stage;
    xb::DevBuf dev;
    bool busy = false;
    size_t admitted = 0;      // largest estimate this slot has grown to
    int* mismatch = nullptr;  // host copy, in stage
    bool any_sign = false;
    std::vector<std::unique_ptr<Request>> reqs;
    std::vector<TreeId> pinned, built;
    Clock::time_point launched;
    size_t lanes_used = 0;
    xmss_b200_batch_trace trace{};  // filled at launch, completed at finish
};

// One (operation, parameter set) group of a batch.
struct Plan {
    uint32_t kind = 0;  // 0 sign (warm requests ride along), 1 verify
    uint32_t oid = 0;
    xmss_params p{};
    const xb::FamilyOps* ops = nullptr;
    KeyTable* table = nullptr;
    std::vector<Request*> reqs;  // launched requests (sign: signing ones)
    std::vector<Request*> warm;
    // sign
    std::vector<xb::TreeJob> jobs;
    std::vector<TreeId> job_ids;
    std::vector<TreeId> used;  // every subtree its requests read
    std::vector<uint64_t> tree_off;  // [c][d]
    std::vector<uint32_t> grp, rank;
    // verify: distinct public keys
    std::vector<uint8_t> pks;
    std::vector<uint32_t> pkx;
    // staging offsets
    size_t o_in = 0, o_off = 0, o_len = 0, o_key = 0, o_soff = 0, o_plan = 0, o_grp = 0, o_rank = 0, o_toff = 0,
           o_jobs = 0, o_pk = 0, o_out = 0, o_idx = 0;
};

enum class Launch { kLaunched, kNothing, kDeferred };

// Lanes per slot.  With 4 slots, slots x (lanes + 1) + 1 streams stay
// within the 32 hardware work queues of the device; the default 8 slots
// share queues and still measured the lower p99 (more batches start at
// once, so requests wait less for a free slot).
constexpr size_t kMaxLanes = 6;

// Estimated critical path of a plan in microseconds on an idle GPU: the
// fixed pipeline depth of its family (chains, L-tree and root levels per
// layer) plus its longest H_msg, a serial chain of compressions
// (lone-thread latency per block: SHA-256 ~1.8, SHA-512 ~6.8, Keccak ~6.2).
double plan_cost_us(uint32_t kind, const xmss_params& p, uint64_t max_inlen)
{
    const bool sha2 = p.func == XMSS_SHA2;
    const double per_block = sha2 ? (p.n == 64 ? 6.8 : 1.8) : 6.2;
    const double block = sha2 ? (p.n == 64 ? 128.0 : 64.0) : (p.n == 32 && p.func == XMSS_SHAKE128 ? 168.0 : 136.0);
    const double depth = (sha2 ? (p.n == 64 ? 900.0 : 220.0) : 800.0) * (kind == 1 ? 1.3 : 1.0) * p.d;
    return depth + per_block * ((double)max_inlen / block + 2);
}

// Host threads that share the byte copies of a batch (requests into the
// pinned staging block, results out of it): one thread copies ~10 GB/s,
// less than a full batch of 64 KB messages needs.
class CopyPool {
   public:
    explicit CopyPool(unsigned n)
    {
        for (unsigned i = 0; i < n; i++) threads_.emplace_back([this] { work(); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    // fn(i) for every i in [0, count), on the pool and the calling thread.
    template <class Fn>
    void run(size_t count, Fn&& fn)
    {
        if (count < 64 || threads_.empty()) {
            for (size_t i = 0; i < count; i++) fn(i);
            return;
        }
        std::function<void(size_t)> f(fn);
        {
            std::lock_guard<std::mutex> g(mu_);
            fn_ = &f;
            count_ = count;
            next_ = 0;
            busy_ = (unsigned)threads_.size();
            gen_++;
        }
        cv_.notify_all();
        drain();
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return busy_ == 0; });
        fn_ = nullptr;
    }

   private:
    void drain()
    {
        for (;;) {
            const size_t i = next_.fetch_add(8);
            if (i >= count_) return;
            for (size_t j = i; j < std::min(count_, i + 8); j++) (*fn_)(j);
        }
    }
    void work()
    {
        uint64_t seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            drain();
            std::lock_guard<std::mutex> g(mu_);
            if (--busy_ == 0) done_cv_.notify_all();
        }
    }
    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(size_t)>* fn_ = nullptr;
    std::atomic<size_t> next_{0};
    size_t count_ = 0;
    unsigned busy_ = 0;
    uint64_t gen_ = 0;
    bool stop_ = false;
};

}  // namespace

struct xmss_b200_server {
    xmss_b200_server_config cfg{};
    xb::Engine* engine = nullptr;
    int device = 0;
    cudaStream_t index_stream = nullptr;

    std::mutex mu;  // queue, completions, keys vector, stats
    std::condition_variable cv, done_cv;
    std::deque<std::unique_ptr<Request>> queue;
    std::deque<xmss_b200_completion> done;
    xmss_b200_server_stats stats{};
    std::string fatal;
    bool stop = false;

    std::mutex launch_mu;  // key state, tree cache, slots (taken before mu)
    std::vector<std::unique_ptr<Key>> keys;
    std::map<std::pair<int, uint32_t>, std::unique_ptr<KeyTable>> tables;
    std::map<TreeId, TreeEntry> trees;
    xb::DevBuf pool;
    uint64_t pool_top = 0;
    std::vector<std::pair<uint64_t, uint64_t>> holes;  // free pool regions (off, cap)
    uint64_t use_clock = 0, batch_seq = 0;
    uint64_t trees_built = 0, tree_hits = 0, trees_evicted = 0;
    std::deque<xmss_b200_batch_trace> traces;  // guarded by mu
    std::vector<std::unique_ptr<Slot>> slots;
    std::unique_ptr<CopyPool> copies;
    std::thread thread;
    // Free device memory for admission, read by the monitor thread: on B200
    // a cudaMemGetInfo call took 4-90 ms at times while batches were in
    // flight, which on the dispatcher thread stalled every request behind it.
    std::atomic<uint64_t> free_bytes{0};
    std::atomic<uint64_t> admitted_since{0};  // growth admitted since the last reading
    std::thread monitor;
    std::condition_variable monitor_cv;  // wakes the monitor at stop
    void watch_memory();

    void run();
    Launch launch(Slot& s, std::vector<std::unique_ptr<Request>>& reqs,
                  std::vector<std::unique_ptr<Request>>& deferred);
    void finish(Slot& s);
    void complete_locked(Request& r);
    bool pool_alloc(uint64_t bytes, uint64_t& off, uint64_t& cap);
    TreeEntry* tree_for(uint32_t key_id, uint32_t layer, uint64_t tree, Plan& pl, Slot& s);
    void release(Slot& s);
};

void xmss_b200_server::complete_locked(Request& r)
{
    xmss_b200_completion c{};
    c.tag = r.tag;
    c.ret = r.ret;
    c.kind = r.kind;
    c.index = r.kind == 0 ? r.idx : 0;
    c.latency_us = std::chrono::duration<double, std::micro>(Clock::now() - r.t0).count();
    done.push_back(c);
    stats.completed++;
}

// A pool region of at least `bytes`: a free hole, fresh pool space, or the
// region of the least recently used subtree that no in-flight batch uses.
bool xmss_b200_server::pool_alloc(uint64_t bytes, uint64_t& off, uint64_t& cap)
{
    bytes = al256(bytes);
    size_t best = holes.size();
    for (size_t i = 0; i < holes.size(); i++)
        if (holes[i].second >= bytes && (best == holes.size() || holes[i].second < holes[best].second)) best = i;
    if (best < holes.size()) {
        off = holes[best].first;
        cap = holes[best].second;
        holes.erase(holes.begin() + best);
        return true;
    }
    if (pool_top + bytes <= cfg.tree_pool_bytes) {
        off = pool_top;
        cap = bytes;
        pool_top += bytes;
        return true;
    }
    auto victim = trees.end();
    for (auto it = trees.begin(); it != trees.end(); ++it) {
        const TreeEntry& e = it->second;
        if (e.pins || !e.settled || e.cap < bytes) continue;
        if (victim == trees.end() || e.last_use < victim->second.last_use) victim = it;
    }
    if (victim == trees.end()) return false;
    off = victim->second.off;
    cap = victim->second.cap;
    cudaEventDestroy(victim->second.ready);
    trees.erase(victim);
    trees_evicted++;
    return true;
}

// The cached subtree (key, layer, tree), pinned for slot s's batch; a
// missing one is allocated and queued for building in plan pl.
TreeEntry* xmss_b200_server::tree_for(uint32_t key_id, uint32_t layer, uint64_t tree, Plan& pl, Slot& s)
{
    const TreeId id{key_id, layer, tree};
    auto it = trees.find(id);
    if (it == trees.end()) {
        const Key& k = *keys[key_id];
        uint64_t off = 0, cap = 0;
        if (!pool_alloc(((2ull << k.p.tree_height) - 1) * k.p.n, off, cap)) return nullptr;
        TreeEntry e;
        e.off = off;
        e.cap = cap;
        if (cudaEventCreateWithFlags(&e.ready, cudaEventDisableTiming) != cudaSuccess) {
            holes.emplace_back(off, cap);
            return nullptr;
        }
        it = trees.emplace(id, e).first;
        pl.jobs.push_back(xb::TreeJob{k.row, layer, tree, off});
        pl.job_ids.push_back(id);
        s.built.push_back(id);
        trees_built++;
    } else if (it->second.pinned_batch != batch_seq) {
        tree_hits++;
    }
    TreeEntry& e = it->second;
    if (std::find(pl.used.begin(), pl.used.end(), id) == pl.used.end()) pl.used.push_back(id);
    e.last_use = ++use_clock;
    if (e.pinned_batch != batch_seq) {
        e.pinned_batch = batch_seq;
        e.pins++;
        s.pinned.push_back(id);
    }
    return &e;
}

// Drops slot s's pins; subtrees it built are complete once it is done.
void xmss_b200_server::release(Slot& s)
{
    for (const TreeId& id : s.pinned) {
        auto it = trees.find(id);
        if (it != trees.end()) it->second.pins--;
    }
    for (const TreeId& id : s.built) {
        auto it = trees.find(id);
        if (it != trees.end()) it->second.settled = true;
    }
    s.pinned.clear();
    s.built.clear();
}

// Plans, stages and launches `reqs` on slot s; on kLaunched the slot owns
// them.  Requests refused while planning keep their code in ret; requests
// that must wait for pool space move to `deferred`.
Launch xmss_b200_server::launch(Slot& s, std::vector<std::unique_ptr<Request>>& reqs,
                                std::vector<std::unique_ptr<Request>>& deferred)
{
    using namespace xb;
    // ---- admission: only growth of this slot's buffers needs new memory ----
    size_t est = 0, tree_scratch = 0;
    {
        std::map<uint32_t, bool> sign_keys;
        for (auto& rp : reqs) {
            const Request& r = *rp;
            const xmss_params& p = r.p;
            const size_t chains = (size_t)p.d * p.wots_len * p.n;
            est += 160 + 16 * p.d + al16(r.inlen) + al16(p.sig_bytes) + 4 * chains + 2 * p.n;
            if (r.kind != 1 && !sign_keys[r.key_id]) {
                sign_keys[r.key_id] = true;
                tree_scratch += ((size_t)p.d << p.tree_height) * p.wots_len * p.n * 3 / 2;
            }
        }
        est += std::min<size_t>(tree_scratch, 3ull << 30);
    }
    if (est > s.admitted) {
        // against the monitor's last reading less the growth admitted since;
        // only when that says no is the device asked again, here
        const uint64_t need = est - s.admitted + cfg.mem_reserve_bytes;
        const uint64_t since = admitted_since.load();
        uint64_t freeb = free_bytes.load();
        freeb = freeb > since ? freeb - since : 0;
        if (freeb < need) {
            size_t f = 0, totalb = 0;
            XB_CUDA(cudaMemGetInfo(&f, &totalb));
            free_bytes = f;
            admitted_since = 0;
            freeb = f;
        }
        if (freeb < need) {
            std::lock_guard<std::mutex> g(mu);
            stats.deferred_for_memory++;
            return Launch::kDeferred;
        }
        admitted_since += est - s.admitted;
    }
    batch_seq++;

    // ---- plan: group by (operation, mt, oid), take indices, pick subtrees ----
    std::map<std::tuple<uint32_t, int, uint32_t>, Plan> plans;
    for (auto& rp : reqs) {
        Request& r = *rp;
        r.deferred = false;
        Plan& pl = plans[{r.kind == 1 ? 1u : 0u, r.mt, r.oid}];
        if (!pl.ops) {
            pl.kind = r.kind == 1 ? 1 : 0;
            pl.oid = r.oid;
            pl.p = r.p;
            pl.ops = family_ops(r.p.func, r.p.n);
            if (pl.kind == 0) pl.table = keys[r.key_id]->table;
        }
        if (!pl.ops) {
            r.ret = -1;
            continue;
        }
        if (r.kind == 1) {
            if (r.inlen < r.p.sig_bytes) {
                r.ret = -1;
                continue;
            }
            pl.reqs.push_back(&r);
        } else if (r.kind == 2) {
            pl.warm.push_back(&r);
        } else {
            Key& k = *keys[r.key_id];
            if (k.next >= k.limit) {
                r.ret = -2;
                continue;
            }
            r.idx = k.next++;
            pl.reqs.push_back(&r);
        }
    }
    // subtrees of each sign plan.  When the pool cannot take a request's
    // subtrees (the rest is pinned by batches in flight) that request and
    // the plan's later ones wait for the next batch: their indices are given
    // back, so each key's indices still follow submission order.
    for (auto& kv : plans) {
        Plan& pl = kv.second;
        if (pl.kind != 0) continue;
        const uint32_t d = pl.p.d, th = pl.p.tree_height;
        auto need = [&](uint32_t key_id, uint64_t idx, uint64_t* toff) {
            for (uint32_t l = 0; l < d; l++) {
                const uint32_t sh = th * (l + 1);
                TreeEntry* e = tree_for(key_id, l, sh >= 64 ? 0 : idx >> sh, pl, s);
                if (!e) return false;
                if (toff) toff[l] = e->off;
            }
            return true;
        };
        pl.tree_off.resize(pl.reqs.size() * d);
        size_t fit = 0;
        while (fit < pl.reqs.size() && need(pl.reqs[fit]->key_id, pl.reqs[fit]->idx, &pl.tree_off[fit * d])) fit++;
        bool warm_ok = fit == pl.reqs.size();
        if (!warm_ok) {
            std::map<uint32_t, uint64_t> first;
            for (size_t j = fit; j < pl.reqs.size(); j++) {
                Request* r = pl.reqs[j];
                auto f = first.find(r->key_id);
                if (f == first.end() || r->idx < f->second) first[r->key_id] = r->idx;
                r->deferred = true;
            }
            for (auto& f : first) keys[f.first]->next = f.second;
            pl.reqs.resize(fit);
            pl.tree_off.resize(fit * d);
        }
        for (Request* r : pl.warm) {
            const Key& k = *keys[r->key_id];
            if (!warm_ok || (k.next < k.limit && !need(r->key_id, k.next, nullptr))) {
                warm_ok = false;
                r->deferred = true;
            }
        }
    }
    {
        std::vector<std::unique_ptr<Request>> keep;
        for (auto& rp : reqs) (rp->deferred ? deferred : keep).push_back(std::move(rp));
        reqs.swap(keep);
    }
    bool work = false;
    for (auto& kv : plans) work |= !kv.second.reqs.empty() || !kv.second.jobs.empty();
    if (!work) return Launch::kNothing;

    // ---- staging layout: inputs first (one H2D), outputs after (one D2H) ----
    size_t top = 0;
    auto take = [&](size_t bytes) {
        const size_t o = top;
        top += al256(bytes);
        return o;
    };
    uint32_t G = 0;  // sign key groups across plans
    for (auto& kv : plans) {
        Plan& pl = kv.second;
        const size_t c = pl.reqs.size();
        size_t in_bytes = 0;
        for (Request* r : pl.reqs) in_bytes += al16(r->inlen);
        pl.o_in = take(in_bytes);
        pl.o_off = take(c * 8);
        pl.o_len = take(c * 8);
        pl.o_key = take(c * 4);
        if (pl.kind == 0) {
            pl.o_soff = take(c * 8);
            pl.o_plan = take(c * 8);
            pl.o_grp = take(c * 4);
            pl.o_rank = take(c * 4);
            pl.o_toff = take(c * pl.p.d * 8);
            pl.o_jobs = take(pl.jobs.size() * sizeof(TreeJob));
            std::map<uint32_t, uint32_t> gi;
            std::vector<uint32_t> cnt;
            pl.grp.resize(c);
            pl.rank.resize(c);
            for (size_t j = 0; j < c; j++) {
                auto it = gi.find(pl.reqs[j]->key_id);
                if (it == gi.end()) {
                    it = gi.emplace(pl.reqs[j]->key_id, (uint32_t)cnt.size()).first;
                    cnt.push_back(0);
                }
                pl.grp[j] = G + it->second;
                pl.rank[j] = cnt[it->second]++;
            }
            G += (uint32_t)cnt.size();
        } else {
            std::map<std::string, uint32_t> distinct;
            pl.pkx.resize(c);
            for (size_t j = 0; j < c; j++) {
                std::string key((const char*)pl.reqs[j]->pk.data(), pl.reqs[j]->pk.size());
                auto it = distinct.find(key);
                if (it == distinct.end()) {
                    it = distinct.emplace(key, (uint32_t)distinct.size()).first;
                    pl.pks.insert(pl.pks.end(), key.begin(), key.end());
                }
                pl.pkx[j] = it->second;
            }
            pl.o_pk = take(pl.pks.size());
        }
    }
    const size_t o_gctr = take((size_t)G * 8), o_gn = take((size_t)G * 4);
    const size_t in_end = top;
    const size_t o_base = take((size_t)G * 8);
    const size_t out_begin = top;
    const size_t o_mismatch = take(sizeof(int));
    for (auto& kv : plans) {
        Plan& pl = kv.second;
        const size_t c = pl.reqs.size();
        if (pl.kind == 0) {
            pl.o_out = take(c * al16(pl.p.sig_bytes));
            pl.o_idx = take(c * 8);
        } else {
            pl.o_out = take(c * 4);
        }
    }
    const size_t total = top;

    // ---- stage ----
    uint8_t* h = s.stage.as<uint8_t>(total);
    uint8_t* d = s.dev.as<uint8_t>(total);
    uint64_t* gctr = (uint64_t*)(h + o_gctr);
    uint32_t* gn = (uint32_t*)(h + o_gn);
    for (uint32_t g = 0; g < G; g++) gn[g] = 0;
    for (auto& kv : plans) {
        Plan& pl = kv.second;
        const size_t c = pl.reqs.size();
        uint64_t* off = (uint64_t*)(h + pl.o_off);
        uint64_t* len = (uint64_t*)(h + pl.o_len);
        uint32_t* key = (uint32_t*)(h + pl.o_key);
        size_t in = 0;
        for (size_t j = 0; j < c; j++) {
            Request& r = *pl.reqs[j];
            off[j] = in;
            len[j] = r.inlen;
            in += al16(r.inlen);
        }
        copies->run(c, [&](size_t j) {
            if (len[j]) memcpy(h + pl.o_in + off[j], pl.reqs[j]->in, len[j]);
        });
        if (pl.kind == 1) {
            memcpy(key, pl.pkx.data(), c * 4);
            memcpy(h + pl.o_pk, pl.pks.data(), pl.pks.size());
            for (size_t j = 0; j < c; j++) pl.reqs[j]->out_off = pl.o_out + 4 * j;
            continue;
        }
        uint64_t* soff = (uint64_t*)(h + pl.o_soff);
        uint64_t* plan = (uint64_t*)(h + pl.o_plan);
        const size_t sb = al16(pl.p.sig_bytes);
        for (size_t j = 0; j < c; j++) {
            Request& r = *pl.reqs[j];
            const Key& k = *keys[r.key_id];
            key[j] = k.row;
            soff[j] = j * sb;
            plan[j] = r.idx;
            r.out_off = pl.o_out + j * sb;
            const uint32_t g = pl.grp[j];
            gctr[g] = (uint64_t)(uintptr_t)(pl.table->counters.as<unsigned long long>(0) + k.row);
            gn[g]++;
        }
        memcpy(h + pl.o_grp, pl.grp.data(), c * 4);
        memcpy(h + pl.o_rank, pl.rank.data(), c * 4);
        memcpy(h + pl.o_toff, pl.tree_off.data(), pl.tree_off.size() * 8);
        memcpy(h + pl.o_jobs, pl.jobs.data(), pl.jobs.size() * sizeof(TreeJob));
    }
    int* mismatch_dev = (int*)(d + o_mismatch);
    s.mismatch = (int*)(h + o_mismatch);
    XB_CUDA(cudaMemcpyAsync(d, h, in_end, cudaMemcpyHostToDevice, s.st));
    XB_CUDA(cudaMemsetAsync(mismatch_dev, 0, sizeof(int), s.st));

    // ---- launch: the index reservation of all sign plans on the index
    // stream, then each plan on its own lane (its new subtrees first, each
    // published by its event), joined back into the slot's stream ----
    XB_CUDA(cudaEventRecord(s.staged, s.st));
    if (G) {
        XB_CUDA(cudaStreamWaitEvent(index_stream, s.staged, 0));
        k_serve_reserve<<<(G + 127) / 128, 128, 0, index_stream>>>((const uint64_t*)(d + o_gctr),
                                                                    (const uint32_t*)(d + o_gn), G,
                                                                    (unsigned long long*)(d + o_base));
        XB_CUDA(cudaEventRecord(s.reserved, index_stream));
    }
    uint64_t groups_sign = 0, groups_verify = 0;
    // plans onto lanes, longest first onto the least loaded lane (a lane
    // runs its plans one after the other)
    std::vector<std::pair<double, Plan*>> order;
    for (auto& kv : plans) {
        Plan& pl = kv.second;
        if (pl.reqs.empty() && pl.jobs.empty()) continue;
        uint64_t longest = 0;
        for (Request* r : pl.reqs) longest = std::max(longest, r->inlen);
        double cost = plan_cost_us(pl.kind, pl.p, longest);
        if (!pl.jobs.empty()) cost += 1e6;  // subtree builds: alone on a lane, first
        order.emplace_back(cost, &pl);
    }
    std::sort(order.begin(), order.end(), [](const auto& a, const auto& b) { return a.first > b.first; });
    const size_t nl = std::min(order.size(), kMaxLanes);
    while (s.lanes.size() < nl) {  // lanes are made at create; a fallback only
        auto ln = std::make_unique<Lane>();
        XB_CUDA(cudaStreamCreateWithFlags(&ln->st, cudaStreamNonBlocking));
        XB_CUDA(cudaEventCreate(&ln->start));
        XB_CUDA(cudaEventCreate(&ln->done));
        ln->w.order_on(ln->st);
        s.lanes.push_back(std::move(ln));
    }
    std::vector<double> load(nl, 0.0);
    std::vector<std::vector<Plan*>> lane_plans(nl);
    for (auto& [cost, pl] : order) {
        const size_t i = std::min_element(load.begin(), load.end()) - load.begin();
        load[i] += cost;
        lane_plans[i].push_back(pl);
    }
    for (size_t li = 0; li < nl; li++) {
        Lane& L = *s.lanes[li];
        XB_CUDA(cudaStreamWaitEvent(L.st, s.staged, 0));
        XB_CUDA(cudaEventRecord(L.start, L.st));
        L.kind = lane_plans[li].front()->kind;
        L.oid = lane_plans[li].front()->oid;
        for (Plan* plp : lane_plans[li]) {
            Plan& pl = *plp;
            const uint32_t c = (uint32_t)pl.reqs.size();
            const xmss_params& p = pl.p;
            if (pl.kind == 1) {
                engine->verify(pl.ops, p, c, d + pl.o_in, (const uint64_t*)(d + pl.o_off), (const uint64_t*)(d + pl.o_len),
                               d + pl.o_pk, (uint32_t)(pl.pks.size() / (2 * p.n)), (const uint32_t*)(d + pl.o_key),
                               (int*)(d + pl.o_out), L.st, L.w, false);
                groups_verify++;
            } else {
                if (!pl.jobs.empty()) {
                    engine->build_trees(pl.ops, (const TreeJob*)(d + pl.o_jobs), (uint32_t)pl.jobs.size(),
                                        (int)p.tree_height, pool.as<uint8_t>(0), pl.table->ctx.as<uint8_t>(0), L.st, L.w,
                                        xb::Engine::subtree_k(p, (uint32_t)pl.jobs.size()));
                    for (const TreeId& id : pl.job_ids) XB_CUDA(cudaEventRecord(trees[id].ready, L.st));
                }
                for (const TreeId& id : pl.used) {  // subtrees other slots are still building
                    const TreeEntry& e = trees[id];
                    if (!e.settled && std::find(pl.job_ids.begin(), pl.job_ids.end(), id) == pl.job_ids.end())
                        XB_CUDA(cudaStreamWaitEvent(L.st, e.ready, 0));
                }
                if (c) {
                    XB_CUDA(cudaStreamWaitEvent(L.st, s.reserved, 0));
                    uint64_t* d_idx = (uint64_t*)(d + pl.o_idx);
                    k_serve_index<<<(c + 127) / 128, 128, 0, L.st>>>(
                        (const unsigned long long*)(d + o_base), (const uint32_t*)(d + pl.o_grp),
                        (const uint32_t*)(d + pl.o_rank), (const uint64_t*)(d + pl.o_plan), c, d_idx, mismatch_dev);
                    SignArgs g{};
                    g.sm = d + pl.o_out;
                    g.sm_off = (const uint64_t*)(d + pl.o_soff);
                    g.mlen = (const uint64_t*)(d + pl.o_len);
                    g.msg = d + pl.o_in;
                    g.msg_off = (const uint64_t*)(d + pl.o_off);
                    g.idx = d_idx;
                    g.key = (const uint32_t*)(d + pl.o_key);
                    g.key_root = pl.table->mat.as<uint8_t>(0) + 2 * p.n;
                    g.key_stride = 4 * p.n;
                    g.tree_off = (const uint64_t*)(d + pl.o_toff);
                    g.nodes = pool.as<uint8_t>(0);
                    g.lens = L.w.lens.as<uint8_t>((size_t)c * p.d * pl.ops->len);
                    g.count = c;
                    g.index_bytes = p.index_bytes;
                    g.sig_bytes = p.sig_bytes;
                    g.tree_height = p.tree_height;
                    g.d = p.d;
                    pl.ops->sign_prep(g, pl.table->ctx.as<uint8_t>(0), L.st);
                    pl.ops->sign_chains(g, pl.table->ctx.as<uint8_t>(0), L.st);
                    groups_sign++;
                }
            }
        }
        XB_CUDA(cudaEventRecord(L.done, L.st));
        XB_CUDA(cudaStreamWaitEvent(s.st, L.done, 0));
    }
    XB_CUDA(cudaMemcpyAsync(h + out_begin, d + out_begin, total - out_begin, cudaMemcpyDeviceToHost, s.st));
    XB_CUDA(cudaGetLastError());
    XB_CUDA(cudaEventRecord(s.done, s.st));
    s.admitted = std::max(s.admitted, est);
    s.any_sign = G != 0;
    s.launched = Clock::now();
    s.lanes_used = nl;
    s.trace = xmss_b200_batch_trace{};
    s.trace.seq = batch_seq;
    s.trace.requests = (uint32_t)reqs.size();
    s.trace.plans = (uint32_t)nl;
    s.trace.h2d_bytes = in_end;
    s.trace.d2h_bytes = total - out_begin;
    Clock::time_point oldest = s.launched;
    for (auto& rp : reqs) oldest = std::min(oldest, rp->t0);
    s.trace.queue_us = std::chrono::duration<double, std::micro>(s.launched - oldest).count();
    s.reqs = std::move(reqs);
    s.busy = true;
    std::lock_guard<std::mutex> lk(mu);
    stats.batches++;
    stats.sign_groups += groups_sign;
    stats.verify_groups += groups_verify;
    stats.largest_batch = std::max<uint64_t>(stats.largest_batch, s.reqs.size());
    return Launch::kLaunched;
}

// Copies a finished slot's results out and completes its requests.
void xmss_b200_server::finish(Slot& s)
{
    const Clock::time_point t0 = Clock::now();
    const uint8_t* h = s.stage.as<uint8_t>(1);
    const bool mismatch = s.any_sign && *s.mismatch != 0;
    copies->run(s.reqs.size(), [&](size_t i) {
        Request& r = *s.reqs[i];
        if (r.ret != 0) return;  // refused while planning
        if (r.kind == 1) {
            r.ret = *(const int*)(h + r.out_off) == 0 ? 0 : -1;
        } else if (r.kind == 0) {
            if (mismatch) {
                r.ret = -3;
                return;
            }
            const xmss_params& p = r.p;
            if (r.inlen) memmove(r.sm_out + p.sig_bytes, r.in, r.inlen);  // sm = sig || m (xmss_core.c:200-201)
            memcpy(r.sm_out, h + r.out_off, p.sig_bytes);
            be_write(r.sm_out, p.index_bytes, r.idx);  // index bytes (xmss_core.c:233)
            if (r.smlen_out) *r.smlen_out = p.sig_bytes + r.inlen;
        }
    });
    release(s);
    s.busy = false;
    xmss_b200_batch_trace& tr = s.trace;
    tr.done_us = std::chrono::duration<double, std::micro>(t0 - s.launched).count();
    float ms = 0;
    if (cudaEventElapsedTime(&ms, s.staged, s.done) == cudaSuccess) tr.gpu_us = 1e3 * ms;
    double last_end = 0;
    for (size_t i = 0; i < s.lanes_used; i++) {
        const Lane& L = *s.lanes[i];
        if (cudaEventElapsedTime(&ms, L.start, L.done) == cudaSuccess && 1e3 * ms > tr.lane_us) {
            tr.lane_us = 1e3 * ms;
            tr.slow_kind = L.kind;
            tr.slow_oid = L.oid;
        }
        if (cudaEventElapsedTime(&ms, s.staged, L.start) == cudaSuccess) tr.start_skew_us = std::max(tr.start_skew_us, 1e3 * ms);
        if (cudaEventElapsedTime(&ms, s.staged, L.done) == cudaSuccess) last_end = std::max(last_end, 1e3 * (double)ms);
    }
    tr.join_us = tr.gpu_us - last_end;
    cudaGetLastError();  // clear a not-ready / invalid-handle status of the queries above
    std::lock_guard<std::mutex> lk(mu);
    traces.push_back(tr);
    if (traces.size() > 4096) traces.pop_front();
    stats.batch_us += std::chrono::duration<double, std::micro>(t0 - s.launched).count();
    stats.finish_us += std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
    if (mismatch) fatal = "xmss_b200_server: device index counter differs from the plan";
    for (auto& rp : s.reqs) complete_locked(*rp);
    s.reqs.clear();
    done_cv.notify_all();
}

// Reads the device's free memory every 20 ms until the server stops.
void xmss_b200_server::watch_memory()
{
    cudaSetDevice(device);
    std::unique_lock<std::mutex> lk(mu);
    while (!stop) {
        lk.unlock();
        size_t f = 0, t = 0;
        const uint64_t since = admitted_since.load();
        if (cudaMemGetInfo(&f, &t) == cudaSuccess) {
            free_bytes = f;
            admitted_since -= std::min<uint64_t>(since, admitted_since.load());
        }
        lk.lock();
        monitor_cv.wait_for(lk, std::chrono::milliseconds(20), [this] { return stop; });
    }
}

void xmss_b200_server::run()
{
    cudaSetDevice(device);
    size_t limit = cfg.max_batch;
    for (;;) {
        bool any_busy = false;
        Slot* free_slot = nullptr;
        {
            std::lock_guard<std::mutex> lk(launch_mu);
            for (auto& sp : slots) {
                if (sp->busy && cudaEventQuery(sp->done) == cudaSuccess) finish(*sp);
                any_busy |= sp->busy;
                if (!sp->busy && !free_slot) free_slot = sp.get();
            }
        }
        std::vector<std::unique_ptr<Request>> take;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (!free_slot || queue.empty()) {
                if (stop && queue.empty() && !any_busy) return;
                cv.wait_for(lk, std::chrono::microseconds(any_busy ? 10 : 2000));
                continue;
            }
            if (cfg.window_us && queue.size() < limit && !stop) {
                const auto due = queue.front()->t0 + std::chrono::microseconds(cfg.window_us);
                if (Clock::now() < due) {
                    cv.wait_until(lk, std::min(due, Clock::now() + std::chrono::microseconds(any_busy ? 10 : 2000)));
                    continue;
                }
            }
            while (!queue.empty() && take.size() < limit) {
                take.push_back(std::move(queue.front()));
                queue.pop_front();
            }
        }
        Launch res = Launch::kNothing;
        std::vector<std::unique_ptr<Request>> wait_pool;
        try {
            std::lock_guard<std::mutex> lk(launch_mu);
            const Clock::time_point t0 = Clock::now();
            res = launch(*free_slot, take, wait_pool);
            {
                const double us = std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
                free_slot->trace.launch_us = us;
                std::lock_guard<std::mutex> g(mu);
                stats.launch_us += us;
            }
            if (res == Launch::kNothing) {  // refused while planning, or warm and cached
                release(*free_slot);
                std::lock_guard<std::mutex> g(mu);
                for (auto& r : take) complete_locked(*r);
                done_cv.notify_all();
            }
        } catch (const std::exception& ex) {
            std::lock_guard<std::mutex> lk(launch_mu);
            release(*free_slot);
            free_slot->busy = false;
            auto& rs = free_slot->reqs.empty() ? take : free_slot->reqs;
            std::lock_guard<std::mutex> g(mu);
            fatal = ex.what();
            for (auto* v : {&rs, &wait_pool})
                for (auto& r : *v) {
                    if (!r) continue;
                    r->ret = -3;
                    complete_locked(*r);
                }
            free_slot->reqs.clear();
            done_cv.notify_all();
            continue;
        }
        if (!wait_pool.empty()) {
            std::lock_guard<std::mutex> g(mu);
            bool others = false;
            for (auto& sp : slots) others |= sp->busy;
            if (!others && res != Launch::kLaunched) {
                // nothing in flight will release pool space: these cannot fit
                for (auto& r : wait_pool) {
                    r->ret = -3;
                    complete_locked(*r);
                }
                done_cv.notify_all();
            } else {
                for (auto it = wait_pool.rbegin(); it != wait_pool.rend(); ++it) queue.push_front(std::move(*it));
            }
        }
        if (res == Launch::kDeferred) {
            std::lock_guard<std::mutex> g(mu);
            if (take.size() > 1) {  // retry with half the batch
                limit = std::max<size_t>(1, take.size() / 2);
                for (auto it = take.rbegin(); it != take.rend(); ++it) queue.push_front(std::move(*it));
            } else {  // a single request does not fit: refuse it
                take[0]->ret = -3;
                complete_locked(*take[0]);
                done_cv.notify_all();
            }
        } else if (limit < cfg.max_batch) {
            limit = std::min<size_t>(cfg.max_batch, 2 * limit);
        }
    }
}

// ===========================================================================
// C-ABI
// ===========================================================================

namespace {

int fail(const char* where, const std::exception& ex)
{
    xb::set_last_error(std::string(where) + ": " + ex.what());
    return -3;
}

void enqueue(xmss_b200_server* srv, std::unique_ptr<Request> r)
{
    std::lock_guard<std::mutex> g(srv->mu);
    srv->queue.push_back(std::move(r));
    srv->stats.submitted++;
    srv->cv.notify_one();
}

// Request on a resident key (sign, warm); nullptr for an unknown key.
std::unique_ptr<Request> key_request(xmss_b200_server* srv, uint32_t key_id, uint32_t kind)
{
    std::lock_guard<std::mutex> g(srv->mu);
    if (key_id >= srv->keys.size()) return nullptr;
    const Key& k = *srv->keys[key_id];
    auto r = std::make_unique<Request>();
    r->kind = kind;
    r->key_id = key_id;
    r->mt = k.mt;
    r->oid = k.oid;
    r->p = k.p;
    return r;
}

std::unique_ptr<Request> verify_request(int mt, const uint8_t* sm, uint64_t smlen, const uint8_t* pk)
{
    auto r = std::make_unique<Request>();
    r->kind = 1;
    r->mt = mt;
    r->oid = (uint32_t)be_read(pk, XMSS_OID_LEN);
    if (!parse(mt, r->oid, &r->p) || (!sm && smlen)) return nullptr;
    r->pk.assign(pk + XMSS_OID_LEN, pk + XMSS_OID_LEN + 2 * r->p.n);
    r->in = sm;
    r->inlen = smlen;
    return r;
}

}  // namespace

extern "C" int xmss_b200_server_create(const xmss_b200_server_config* cfg, xmss_b200_server** out)
{
    try {
        auto srv = std::make_unique<xmss_b200_server>();
        xmss_b200_server_config c{};
        c.max_batch = 4096;
        c.slots = 8;  // p99 at 100k requests/s: 8.9 ms with 8, 10.2 ms with 4 (B200)
        c.tree_pool_bytes = 1ull << 30;
        c.mem_reserve_bytes = 1ull << 30;
        if (cfg) {
            if (cfg->max_batch) c.max_batch = cfg->max_batch;
            if (cfg->slots) c.slots = cfg->slots;
            c.window_us = cfg->window_us;
            if (cfg->tree_pool_bytes) c.tree_pool_bytes = cfg->tree_pool_bytes;
            if (cfg->mem_reserve_bytes) c.mem_reserve_bytes = cfg->mem_reserve_bytes;
        }
        srv->cfg = c;
        srv->engine = &xb::Engine::get();
        srv->device = srv->engine->device();
        XB_CUDA(cudaSetDevice(srv->device));
        XB_CUDA(cudaStreamCreateWithFlags(&srv->index_stream, cudaStreamNonBlocking));
        srv->pool.get(c.tree_pool_bytes);
        // slot scratch grows stream-ordered from the device's default pool;
        // blocks freed there stay cached for the next growth
        cudaMemPool_t mp;
        XB_CUDA(cudaDeviceGetDefaultMemPool(&mp, srv->device));
        uint64_t keep = ~0ull;
        XB_CUDA(cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &keep));
        for (uint32_t i = 0; i < c.slots; i++) {
            auto s = std::make_unique<Slot>();
            XB_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
            XB_CUDA(cudaEventCreate(&s->done));
            XB_CUDA(cudaEventCreate(&s->staged));
            XB_CUDA(cudaEventCreateWithFlags(&s->reserved, cudaEventDisableTiming));
            s->dev.order_on(s->st);
            // staging for a full batch of long messages up front: growing
            // pinned memory later takes tens of milliseconds of page pinning
            const size_t stage = std::min<size_t>((size_t)c.max_batch << 16, 256ull << 20);
            s->stage.keep_old_blocks();
            s->stage.get(stage);
            s->dev.get(stage);
            // every lane up front: creating streams and events while batches
            // run took 8-34 ms of the dispatcher's time on B200
            while (s->lanes.size() < kMaxLanes) {
                auto ln = std::make_unique<Lane>();
                XB_CUDA(cudaStreamCreateWithFlags(&ln->st, cudaStreamNonBlocking));
                XB_CUDA(cudaEventCreate(&ln->start));
                XB_CUDA(cudaEventCreate(&ln->done));
                ln->w.order_on(ln->st);
                s->lanes.push_back(std::move(ln));
            }
            srv->slots.push_back(std::move(s));
        }
        for (auto& sp : srv->slots) XB_CUDA(cudaStreamSynchronize(sp->st));
        srv->copies = std::make_unique<CopyPool>(
            std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 4)));
        {
            size_t f = 0, t = 0;
            XB_CUDA(cudaMemGetInfo(&f, &t));
            srv->free_bytes = f;
        }
        xmss_b200_server* p = srv.release();
        p->thread = std::thread([p] { p->run(); });
        p->monitor = std::thread([p] { p->watch_memory(); });
        *out = p;
        return 0;
    } catch (const std::exception& ex) {
        return fail("xmss_b200_server_create", ex);
    }
}

extern "C" void xmss_b200_server_destroy(xmss_b200_server* srv)
{
    if (!srv) return;
    {
        std::lock_guard<std::mutex> g(srv->mu);
        srv->stop = true;
    }
    srv->cv.notify_all();
    srv->monitor_cv.notify_all();
    if (srv->thread.joinable()) srv->thread.join();
    if (srv->monitor.joinable()) srv->monitor.join();
    cudaSetDevice(srv->device);
    for (auto& s : srv->slots) {
        for (auto& ln : s->lanes) {
            cudaStreamSynchronize(ln->st);
            cudaEventDestroy(ln->start);
            cudaEventDestroy(ln->done);
            cudaStreamDestroy(ln->st);
        }
        cudaEventDestroy(s->done);
        cudaEventDestroy(s->staged);
        cudaEventDestroy(s->reserved);
        cudaStreamDestroy(s->st);
    }
    cudaStreamSynchronize(srv->index_stream);
    cudaStreamDestroy(srv->index_stream);
    for (auto& kv : srv->trees) cudaEventDestroy(kv.second.ready);
    delete srv;
}

extern "C" int xmss_b200_server_add_key(xmss_b200_server* srv, int mt, const uint8_t* sk, uint32_t* key_id)
{
    auto k = std::make_unique<Key>();
    const uint32_t oid = (uint32_t)be_read(sk, XMSS_OID_LEN);
    if (!parse(mt, oid, &k->p) || !xb::family_ops(k->p.func, k->p.n)) {
        xb::set_last_error("xmss_b200_server_add_key: unknown OID");
        return -1;
    }
    const xmss_params& p = k->p;
    const xb::FamilyOps* ops = xb::family_ops(p.func, p.n);
    k->oid = oid;
    k->mt = mt;
    k->next = be_read(sk + XMSS_OID_LEN, p.index_bytes);
    k->limit = p.full_height >= 64 ? ~0ull : (1ull << p.full_height) - 1;
    k->mat.assign(sk + XMSS_OID_LEN + p.index_bytes, sk + XMSS_OID_LEN + p.index_bytes + 4 * p.n);
    try {
        std::lock_guard<std::mutex> lk(srv->launch_mu);
        XB_CUDA(cudaSetDevice(srv->device));
        // the tables may move: no batch may be using them
        for (auto& s : srv->slots)
            if (s->busy) XB_CUDA(cudaEventSynchronize(s->done));
        auto& tp = srv->tables[{mt, oid}];
        if (!tp) {
            tp = std::make_unique<KeyTable>();
            tp->p = p;
            tp->ops = ops;
        }
        KeyTable& t = *tp;
        if (t.count == t.cap) {
            const uint32_t cap = std::max<uint32_t>(16, 2 * t.cap);
            xb::DevBuf nctx, nmat, ncnt;
            nctx.get((size_t)cap * ops->ctx_bytes);
            nmat.get((size_t)cap * 4 * p.n);
            ncnt.get((size_t)cap * 8);
            if (t.count) {
                XB_CUDA(cudaMemcpy(nctx.get(1), t.ctx.get(1), (size_t)t.count * ops->ctx_bytes,
                                   cudaMemcpyDeviceToDevice));
                XB_CUDA(cudaMemcpy(nmat.get(1), t.mat.get(1), (size_t)t.count * 4 * p.n, cudaMemcpyDeviceToDevice));
                XB_CUDA(cudaMemcpy(ncnt.get(1), t.counters.get(1), (size_t)t.count * 8, cudaMemcpyDeviceToDevice));
            }
            t.ctx.swap(nctx);
            t.mat.swap(nmat);
            t.counters.swap(ncnt);
            t.cap = cap;
        }
        k->table = &t;
        k->row = t.count;
        uint8_t* dm = t.mat.as<uint8_t>(0) + (size_t)k->row * 4 * p.n;
        XB_CUDA(cudaMemcpy(dm, k->mat.data(), 4 * p.n, cudaMemcpyHostToDevice));
        const unsigned long long c0 = k->next;
        XB_CUDA(cudaMemcpy(t.counters.as<unsigned long long>(0) + k->row, &c0, 8, cudaMemcpyHostToDevice));
        // per-key hash context from the row: PUB_SEED at 3n, SK_SEED at 0, SK_PRF at n
        ops->make_ctx(dm + 3 * p.n, 4 * p.n, dm, 4 * p.n, dm + p.n, 4 * p.n, 1,
                      t.ctx.as<uint8_t>(0) + (size_t)k->row * ops->ctx_bytes, srv->index_stream);
        XB_CUDA(cudaGetLastError());
        XB_CUDA(cudaStreamSynchronize(srv->index_stream));
        t.count++;
        std::lock_guard<std::mutex> g(srv->mu);
        *key_id = (uint32_t)srv->keys.size();
        srv->keys.push_back(std::move(k));
        return 0;
    } catch (const std::exception& ex) {
        return fail("xmss_b200_server_add_key", ex);
    }
}

extern "C" int xmss_b200_server_export_sk(xmss_b200_server* srv, uint32_t key_id, uint8_t* sk)
{
    std::lock_guard<std::mutex> lk(srv->launch_mu);
    std::lock_guard<std::mutex> g(srv->mu);
    if (key_id >= srv->keys.size()) return -1;
    const Key& k = *srv->keys[key_id];
    be_write(sk, XMSS_OID_LEN, k.oid);
    be_write(sk + XMSS_OID_LEN, k.p.index_bytes, k.next);
    memcpy(sk + XMSS_OID_LEN + k.p.index_bytes, k.mat.data(), k.mat.size());
    return 0;
}

extern "C" int xmss_b200_server_submit_sign(xmss_b200_server* srv, uint32_t key_id, const uint8_t* m, uint64_t mlen,
                                            uint8_t* sm, uint64_t* smlen, uint64_t tag)
{
    auto r = key_request(srv, key_id, 0);
    if (!r || (!m && mlen) || !sm) return -1;
    r->t0 = Clock::now();
    r->tag = tag;
    r->in = m;
    r->inlen = mlen;
    r->sm_out = sm;
    r->smlen_out = smlen;
    enqueue(srv, std::move(r));
    return 0;
}

extern "C" int xmss_b200_server_submit_warm(xmss_b200_server* srv, uint32_t key_id, uint64_t tag)
{
    auto r = key_request(srv, key_id, 2);
    if (!r) return -1;
    r->t0 = Clock::now();
    r->tag = tag;
    enqueue(srv, std::move(r));
    return 0;
}

extern "C" int xmss_b200_server_submit_verify(xmss_b200_server* srv, int mt, const uint8_t* sm, uint64_t smlen,
                                              const uint8_t* pk, uint64_t tag)
{
    auto r = verify_request(mt, sm, smlen, pk);
    if (!r) return -1;
    r->t0 = Clock::now();
    r->tag = tag;
    enqueue(srv, std::move(r));
    return 0;
}

extern "C" int xmss_b200_server_poll(xmss_b200_server* srv, xmss_b200_completion* out, uint32_t max,
                                     uint32_t wait_us)
{
    std::unique_lock<std::mutex> lk(srv->mu);
    if (srv->done.empty() && wait_us)
        srv->done_cv.wait_for(lk, std::chrono::microseconds(wait_us), [&] { return !srv->done.empty(); });
    uint32_t n = 0;
    while (n < max && !srv->done.empty()) {
        out[n++] = srv->done.front();
        srv->done.pop_front();
    }
    return (int)n;
}

extern "C" int xmss_b200_server_stats_get(xmss_b200_server* srv, xmss_b200_server_stats* out)
{
    std::lock_guard<std::mutex> lk(srv->launch_mu);
    std::lock_guard<std::mutex> g(srv->mu);
    *out = srv->stats;
    out->trees_built = srv->trees_built;
    out->tree_hits = srv->tree_hits;
    out->trees_evicted = srv->trees_evicted;
    if (srv->fatal.empty()) return 0;
    xb::set_last_error(srv->fatal);
    return -3;
}

extern "C" int xmss_b200_server_replay(xmss_b200_server* srv, const xmss_b200_trace_item* items, uint32_t count,
                                       int* ret, double* latency_us, uint64_t* index, double* elapsed_s)
{
    if (!srv || (!items && count)) return -1;
    // requests are built before the clock starts; the submitter only queues
    std::vector<std::unique_ptr<Request>> reqs(count);
    for (uint32_t i = 0; i < count; i++) {
        const xmss_b200_trace_item& it = items[i];
        if ((i && it.t_us < items[i - 1].t_us) || it.kind > 1) return -1;
        if (it.kind == 0) {
            reqs[i] = key_request(srv, it.key_id, 0);
            if (!reqs[i] || !it.sm || (!it.in && it.inlen)) return -1;
            reqs[i]->in = it.in;
            reqs[i]->inlen = it.inlen;
            reqs[i]->sm_out = it.sm;
            reqs[i]->smlen_out = it.smlen;
        } else {
            if (!it.pk) return -1;
            reqs[i] = verify_request(it.mt, it.in, it.inlen, it.pk);
            if (!reqs[i]) return -1;
        }
        reqs[i]->tag = (1ull << 63) | i;  // replay tags carry the top bit
    }
    std::vector<uint8_t> seen(count, 0);
    const Clock::time_point start = Clock::now();
    std::thread submitter([&] {
        for (uint32_t i = 0; i < count; i++) {
            const auto due = start + std::chrono::duration_cast<Clock::duration>(
                                         std::chrono::duration<double, std::micro>(items[i].t_us));
            while (Clock::now() < due) {
            }
            reqs[i]->t0 = due;  // latency counts from the scheduled time
            enqueue(srv, std::move(reqs[i]));
        }
    });
    uint32_t got = 0;
    std::vector<xmss_b200_completion> buf(4096);
    Clock::time_point last = start;
    while (got < count) {
        const int n = xmss_b200_server_poll(srv, buf.data(), (uint32_t)buf.size(), 1000);
        for (int j = 0; j < n; j++) {
            const xmss_b200_completion& c = buf[j];
            if (!(c.tag >> 63)) continue;  // another caller's request
            const uint64_t i = c.tag & ~(1ull << 63);
            if (i >= count || seen[i]) continue;
            seen[i] = 1;
            got++;
            if (ret) ret[i] = c.ret;
            if (latency_us) latency_us[i] = c.latency_us;
            if (index) index[i] = c.index;
        }
        if (n > 0) last = Clock::now();
    }
    submitter.join();
    if (elapsed_s) *elapsed_s = std::chrono::duration<double>(last - start).count();
    return 0;
}

extern "C" int xmss_b200_server_trace(xmss_b200_server* srv, xmss_b200_batch_trace* out, uint32_t max)
{
    std::lock_guard<std::mutex> g(srv->mu);
    const size_t n = std::min<size_t>(max, srv->traces.size());
    for (size_t i = 0; i < n; i++) out[i] = srv->traces[srv->traces.size() - n + i];
    return (int)n;
}
