// Host engine of libxmss_b200: owns the CUDA stream, grow-only scratch
// memory and the launch sequences (pipelines) of keygen, sign and verify.
// One engine per process, bound to one device.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/params.h"
#include "family_ops.h"

namespace xb {

struct LeafRef;
struct TreeJob;
struct VerifyArgs;
struct PersistBatch;

class CudaFailure : public std::runtime_error {
   public:
    using std::runtime_error::runtime_error;
};

#define XB_CUDA(call)                                                                             \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            throw ::xb::CudaFailure(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " + \
                                    __FILE__ + ":" + std::to_string(__LINE__));                   \
    } while (0)

// Device buffer that only grows.  Growing waits for all device work.
class DevBuf {
   public:
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf();
    void* get(size_t bytes);
    template <class T>
    T* as(size_t count)
    {
        return (T*)get(count * sizeof(T));
    }
    void swap(DevBuf& o)
    {
        std::swap(p_, o.p_);
        std::swap(cap_, o.cap_);
        std::swap(order_, o.order_);
        std::swap(ordered_, o.ordered_);
    }
    // Growth becomes stream-ordered on st (cudaFreeAsync / cudaMallocAsync)
    // instead of waiting for the whole device: for buffers only st uses.
    void order_on(cudaStream_t st)
    {
        order_ = st;
        ordered_ = true;
    }

   private:
    void* p_ = nullptr;
    size_t cap_ = 0;
    cudaStream_t order_ = nullptr;
    bool ordered_ = false;
};

// Pinned host buffer that only grows.
class PinnedBuf {
   public:
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf();
    void* get(size_t bytes);
    template <class T>
    T* as(size_t count)
    {
        return (T*)get(count * sizeof(T));
    }

    // Growth doubles and keeps the old block alive (the owner guarantees
    // no copy uses it), so it never waits for the device.
    void keep_old_blocks() { keep_old_ = true; }

   private:
    void* p_ = nullptr;
    size_t cap_ = 0;
    bool keep_old_ = false;
    std::vector<void*> retired_;
};

// Second stream of a split verify batch (the long-H_msg group runs there
// while the short group runs on the caller's stream) and its fork / join;
// a third stream for the h_pre items of both groups and the event that
// ends them.
struct SplitStreams {
    cudaStream_t aux = nullptr, pre = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr, pre_done = nullptr;
    void create();
    void destroy();
};

// Scratch of one in-flight launch sequence.  The engine owns one for its
// own entry points; the server gives each of its batch slots one, so
// batches on different streams never share intermediate buffers.
struct Workspace {
    DevBuf ctx, jobs, refs, wpk, wpk2, nodes, keys, node, lens, idx, leaf, hpre, hist, list, list2, aux;
    DevBuf work;    // verify work counters of non-engine workspaces
    DevBuf pstate;  // task counters of the persistent verify
    PinnedBuf h_jobs;
    void order_on(cudaStream_t st);  // every buffer grows stream-ordered on st
    // Streams of large verify batches (two groups split by H_msg length)
    // for workspaces outside the engine; none: no split.
    SplitStreams* split = nullptr;
};

class Engine {
   public:
    static Engine& get();  // lazily created on the current device
    explicit Engine(int device);
    ~Engine();

    std::mutex mu;  // serialises host-buffer calls

    // Orders work on `st` after the previous call (scratch reuse) and records
    // the end of this call's work.
    void begin(cudaStream_t st);
    void end(cudaStream_t st);

    cudaStream_t stream() const { return stream_; }
    int device() const { return device_; }

    // -- pipelines (device pointers, asynchronous on st) ---------------------
    // Builds every subtree of `jobs` (all of height h): node arrays at
    // d_nodes + job.node_off, levels 0..h.  d_jobs is the device copy of jobs.
    // subtree_k 0: one thread per chain and a launch per level; 5..7: levels
    // 0..k as in-CTA subtrees (subtree_height_for gives it per parameter set).
    void build_trees(const FamilyOps* ops, const TreeJob* d_jobs, uint32_t njobs, int h, uint8_t* d_nodes,
                     const void* d_ctx, cudaStream_t st, Workspace& w, int subtree_k = 0);

    // The in-CTA subtree height for a build of njobs subtrees of parameter set p.
    static int subtree_k(const xmss_params& p, uint32_t njobs)
    {
        const TreeShape& s = tree_shape_for(p.func, p.n, p.full_height, p.d);
        return subtree_height_for(s, (int)p.tree_height, (uint64_t)njobs << p.tree_height);
    }

    // Verify of `count` signed messages against npk public keys (root||seed).
    void verify(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* d_sm,
                const uint64_t* d_sm_off, const uint64_t* d_smlen, const uint8_t* d_pk, uint32_t npk,
                const uint32_t* d_pk_index, int* d_status, cudaStream_t st)
    {
        verify(ops, p, count, d_sm, d_sm_off, d_smlen, d_pk, npk, d_pk_index, d_status, st, ws_, true);
    }
    // With allow_split false the batch runs as one sequence on st only.
    void verify(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* d_sm,
                const uint64_t* d_sm_off, const uint64_t* d_smlen, const uint8_t* d_pk, uint32_t npk,
                const uint32_t* d_pk_index, int* d_status, cudaStream_t st, Workspace& w, bool allow_split);

    // The same verify as one persistent launch fed by a device work queue
    // (verify_persist.cuh), on st only; same statuses, plus -3 for every
    // signature if a dependency wait ran out.
    void verify_persistent(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* d_sm,
                           const uint64_t* d_sm_off, const uint64_t* d_smlen, const uint8_t* d_pk, uint32_t npk,
                           const uint32_t* d_pk_index, int* d_status, cudaStream_t st);

    // One verify batch of the persistent form (device pointers).
    // A keygen or sign batch of the persistent form.
    struct PersistJob {
        uint32_t kind = 0;  // 0 verify, 1 keygen, 2 sign
        const FamilyOps* ops = nullptr;
        xmss_params p{};
        uint32_t count = 0;
        // verify
        const uint8_t* d_sm = nullptr;
        const uint64_t* d_sm_off = nullptr;
        const uint64_t* d_smlen = nullptr;
        const uint8_t* d_pk = nullptr;
        uint32_t npk = 0;
        const uint32_t* d_pk_index = nullptr;
        int* d_status = nullptr;
        // keygen: seeds (count x 3n) -> pk (count x 2n), sk (count x sk_bytes)
        const uint8_t* d_seeds = nullptr;
        uint8_t* d_pk_out = nullptr;
        uint8_t* d_sk_out = nullptr;
        // sign: per item the key as it signs (sk without OID, after the index
        // bookkeeping), the index and the index bytes of the signature (8 per
        // item), host memory read at setup; d_sm / d_sm_off / d_mlen as Engine::sign
        const uint8_t* h_sk = nullptr;
        const uint64_t* h_idx = nullptr;
        const uint8_t* h_ibytes = nullptr;
        uint8_t* d_sign_sm = nullptr;
        const uint64_t* d_mlen = nullptr;
    };
    // Scratch of persistent multi-batch launches: a workspace per batch and
    // the launches' ticket / exit counters (the engine keeps one for its own
    // calls; a captured graph keeps its own).
    struct PersistScratch {
        std::vector<std::unique_ptr<Workspace>> ws;
        DevBuf ctr;
    };
    // Batches of any parameter sets and kinds: one persistent launch per hash
    // family (up to 8 batches each), the families' launches on streams forked
    // from st and joined back into it.
    void verify_persistent_multi(const std::vector<PersistJob>& jobs, cudaStream_t st)
    {
        persistent_multi(jobs, st, pscratch_);
    }
    void persistent_multi(const std::vector<PersistJob>& jobs, cudaStream_t st, PersistScratch& scratch);

    // Key generation from seeds (count x 3n) into pk (count x 2n) and sk
    // (count x sk_bytes), no OID prefix.
    void keypair(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* d_seeds, uint8_t* d_pk,
                 uint8_t* d_sk, cudaStream_t st)
    {
        keypair(ops, p, count, d_seeds, d_pk, d_sk, st, ws_);
    }
    // wait false: returns without waiting for st (the caller keeps w's
    // pinned job list unchanged until the work has run; graph capture).
    void keypair(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* d_seeds, uint8_t* d_pk,
                 uint8_t* d_sk, cudaStream_t st, Workspace& w, bool wait = true);

    // Signing given per-request key material.  h_sk: count x sk_bytes (no
    // OID), already reflecting the reference's exhaustion handling; h_idx:
    // the index each request signs with.  d_sm: output buffers with the
    // message already at sm_off + sig_bytes.
    void sign(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* h_sk,
              const uint64_t* h_idx, uint8_t* d_sm, const uint64_t* d_sm_off, const uint64_t* d_mlen,
              cudaStream_t st)
    {
        sign(ops, p, count, h_sk, h_idx, d_sm, d_sm_off, d_mlen, st, ws_);
    }
    // wait as for keypair.
    void sign(const FamilyOps* ops, const xmss_params& p, uint32_t count, const uint8_t* h_sk,
              const uint64_t* h_idx, uint8_t* d_sm, const uint64_t* d_sm_off, const uint64_t* d_mlen,
              cudaStream_t st, Workspace& w, bool wait = true);

    void core_hash(const FamilyOps* ops, uint32_t count, const uint8_t* d_in, const uint64_t* d_off,
                   const uint64_t* d_len, uint8_t* d_out, cudaStream_t st);

    // Verify launch sequence over the signatures v selects (all when
    // v.sel is null), on one stream.
    // fused_ltree: the whole L-tree in one warp-per-signature launch (for
    // groups whose L-tree runs with the GPU otherwise idle) instead of one
    // launch per level.
    void verify_sequence(const FamilyOps* ops, const xmss_params& p, const VerifyArgs& v, const void* ctx,
                         cudaStream_t st, bool marks = true, bool fused_ltree = false,
                         cudaEvent_t hpre_ready = nullptr);
    // Single-sequence batches below this size are latency-bound: fused
    // L-tree (measured: it lowers serving latency at light load; for larger
    // batches, and for the tail group of a split batch, it cost throughput).
    static constexpr uint32_t kFusedLtreeBelow = 256;
    // Batches of at least Tuning::split_min signatures are verified as two
    // groups split at Tuning::short_hmsg_blocks hash blocks of H_msg.

    // Bound of one dependency wait inside a persistent launch, in ns of the
    // GPU's global timer (xmss_b200_set_wait_bound).  A wait that runs out
    // ends the launch with -3 for every item instead of waiting on.
    static constexpr unsigned long long kDefaultWaitNs = 8000000000ull;
    unsigned long long persist_wait_ns = kDefaultWaitNs;

    // Work counters of the last verify (see xmss_b200_last_verify_work).
    void last_verify_work(unsigned long long out[3]);

    // Phase timing (xmss_b200_profile / xmss_b200_phase_ms).
    enum Phase { kPrep = 0, kChains = 1, kLtree = 2, kRoot = 3, kTree = 4, kPhases = 5 };
    bool profiling = false;
    void mark(int phase, bool start, cudaStream_t st, bool on = true);  // no-op unless profiling and on
    void phase_ms(double out[kPhases]);

    // Scratch for host-buffer entry points (guarded by mu).
    DevBuf d_in, d_in2, d_off, d_len, d_out, d_aux, d_aux2;
    PinnedBuf h_stage, h_stage2;

   private:
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t done_ = nullptr;
    SplitStreams split_;  // streams of the engine's own split verify batches
    bool have_done_ = false;
    Workspace ws_;  // scratch of the engine's own entry points
    DevBuf s_work_;
    unsigned long long* work_ = nullptr;
    // persistent batches: arguments of one batch over workspace w, its task
    // counters zeroed on st
    void persist_setup(const PersistJob& j, Workspace& w, VerifyArgs& v, PersistArgs& q, cudaStream_t st);
    // a keygen or sign batch of a multi-batch launch
    void gen_setup(const PersistJob& j, Workspace& w, PersistBatch& J, cudaStream_t st);
    PersistScratch pscratch_;
    std::vector<cudaStream_t> pstreams_;           // launches after the first
    std::vector<cudaEvent_t> pjoin_;
    cudaEvent_t pfork_ = nullptr;
    struct Mark {
        int phase;
        cudaEvent_t a, b;
    };
    std::vector<Mark> marks_;
    std::vector<cudaEvent_t> free_events_;
    cudaEvent_t event();
};

// Engine selected by (func, n); throws when the family is not built.
const FamilyOps* ops_for(const xmss_params& p);

// rate_kernel.cu
void launch_rate(int kind, uint32_t blocks, uint32_t iters, uint32_t* sink, cudaStream_t st);

}  // namespace xb
