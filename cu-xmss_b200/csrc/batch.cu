// Mixed batches (xmss_b200_batch_*): keygen, sign and verify groups of any
// parameter sets in one CUDA graph.
//
// Each group gets a stream and a Workspace of its own and runs the launch
// sequence of its kind (Engine::keypair / Engine::sign / Engine::verify, the
// same sequences as the per-kind entry points).  Create runs every group once
// uncaptured, which sizes its scratch (sign groups write that run's output
// into a scratch copy of their buffer, wiped afterwards), then captures all
// groups between a fork and a join event of one capture stream: the graph's
// groups are independent branches, so the GPU runs them concurrently, and a
// launch is one cudaGraphLaunch.
//
// Sign groups keep the reference's index bookkeeping (xmss_core.c:209-239):
// create advances the host keys exactly as that many xmss[mt]_sign calls
// would, the graph signs at the indices taken then, and the batch launches
// at most once, so no index signs two messages.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/params.h"
#include "../../include/xmss_b200.h"
#include "engine.h"

namespace xb {
void set_last_error(const std::string& msg);                                        // api.cu
int sign_advance(const xmss_params& p, uint8_t* sk, uint64_t* idx, uint8_t* idx_bytes);  // api.cu

// Writes each signed item's index bytes (the bytes the reference copies from
// the sk, xmss_core.c: memcpy(sm, sk, index_bytes)) at the start of its
// signature.  ib: index bytes per item, 8-byte rows.
__global__ void k_put_index(uint8_t* __restrict__ sm, const uint64_t* __restrict__ sm_off,
                            const uint8_t* __restrict__ ib_rows, uint32_t ib, uint32_t count)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    uint8_t* s = sm + sm_off[i];
    for (uint32_t k = 0; k < ib; k++) s[k] = ib_rows[(uint64_t)i * 8 + k];
}
}  // namespace xb

namespace {

using xb::DevBuf;
using xb::Engine;

uint64_t be_read(const uint8_t* p, unsigned len)
{
    uint64_t r = 0;
    for (unsigned i = 0; i < len; i++) r = (r << 8) | p[i];
    return r;
}

struct Group {
    xmss_b200_batch_group g{};
    xmss_params p{};
    const xb::FamilyOps* ops = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t join = nullptr;
    xb::SplitStreams split;
    xb::Workspace w;
    // sign: the live items (not exhausted), their keys after the index
    // bookkeeping, indices and index bytes, and device copies of their
    // offsets, message lengths and index bytes
    uint32_t live = 0;
    std::vector<uint8_t> keys;
    std::vector<uint64_t> idx;
    std::vector<uint8_t> ib;  // 8 per live item
    DevBuf d_off, d_len, d_ib;
    uint64_t extent = 0;  // bytes of d_sm the live items cover

    ~Group()
    {
        if (join) cudaEventDestroy(join);
        if (st) cudaStreamDestroy(st);
        split.destroy();
    }
};

}  // namespace

struct xmss_b200_batch {
    std::vector<std::unique_ptr<Group>> groups;
    cudaStream_t capture = nullptr;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
    bool has_sign = false;
    bool launched = false;
    bool persistent = false;        // one persistent launch per family instead of the per-group sequences
    Engine::PersistScratch pscratch;  // its workspaces and counters
    ~xmss_b200_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (fork) cudaEventDestroy(fork);
        if (capture) cudaStreamDestroy(capture);
    }
};

namespace {

// Checks a group's fields; host-side set-up of sign groups (index
// bookkeeping, live items, device copies of their arrays).  Throws
// std::invalid_argument for a bad group.
void prepare(Group& G)
{
    const xmss_b200_batch_group& g = G.g;
    if ((g.mt ? xmssmt_parse_oid(&G.p, g.oid) : xmss_parse_oid(&G.p, g.oid)) != 0)
        throw std::invalid_argument("unknown OID");
    G.ops = xb::ops_for(G.p);
    const xmss_params& p = G.p;
    switch (g.kind) {
        case XMSS_B200_KEYGEN:
            if (!g.d_seeds || !g.d_pk || !g.d_sk) throw std::invalid_argument("keygen group without buffers");
            return;
        case XMSS_B200_VERIFY:
            if (!g.d_sm || !g.d_sm_off || !g.d_len || !g.d_pk || !g.npk || !g.d_pk_index || !g.d_status)
                throw std::invalid_argument("verify group without buffers");
            return;
        case XMSS_B200_SIGN:
            break;
        default:
            throw std::invalid_argument("unknown group kind");
    }
    if (!g.sk || !g.ret || !g.d_sm || !g.d_sm_off || !g.d_len) throw std::invalid_argument("sign group without buffers");
    const size_t sks = XMSS_OID_LEN + p.sk_bytes;
    for (uint32_t r = 0; r < g.count; r++)
        if ((uint32_t)be_read(g.sk + r * sks, XMSS_OID_LEN) != g.oid)
            throw std::invalid_argument("sign group: a secret key of another OID");
    std::vector<uint64_t> off(g.count), len(g.count);
    XB_CUDA(cudaMemcpy(off.data(), g.d_sm_off, g.count * 8, cudaMemcpyDeviceToHost));
    XB_CUDA(cudaMemcpy(len.data(), g.d_len, g.count * 8, cudaMemcpyDeviceToHost));
    std::vector<uint64_t> loff, llen;
    std::vector<uint8_t> ib;
    for (uint32_t r = 0; r < g.count; r++) {
        uint8_t* sk = g.sk + r * sks + XMSS_OID_LEN;
        uint64_t i = 0;
        uint8_t b[8] = {0};
        g.ret[r] = xb::sign_advance(p, sk, &i, b);
        if (g.ret[r] != 0) continue;
        G.keys.insert(G.keys.end(), sk, sk + p.sk_bytes);  // the key as the reference signs with it
        G.idx.push_back(i);
        loff.push_back(off[r]);
        llen.push_back(len[r]);
        ib.insert(ib.end(), b, b + 8);
        G.extent = std::max(G.extent, off[r] + p.sig_bytes + len[r]);
    }
    G.live = (uint32_t)G.idx.size();
    G.ib = ib;
    if (!G.live) return;
    uint64_t* d_off = G.d_off.as<uint64_t>(G.live);
    uint64_t* d_len = G.d_len.as<uint64_t>(G.live);
    uint8_t* d_ib = G.d_ib.as<uint8_t>((size_t)G.live * 8);
    XB_CUDA(cudaMemcpy(d_off, loff.data(), G.live * 8, cudaMemcpyHostToDevice));
    XB_CUDA(cudaMemcpy(d_len, llen.data(), G.live * 8, cudaMemcpyHostToDevice));
    XB_CUDA(cudaMemcpy(d_ib, ib.data(), (size_t)G.live * 8, cudaMemcpyHostToDevice));
}

// One group's launch sequence on its stream; sm_out replaces a sign group's
// output buffer (the sizing run's scratch).
void run(Engine& e, Group& G, uint8_t* sm_out)
{
    const xmss_b200_batch_group& g = G.g;
    switch (g.kind) {
        case XMSS_B200_KEYGEN:
            e.keypair(G.ops, G.p, g.count, g.d_seeds, g.d_pk, g.d_sk, G.st, G.w, false);
            break;
        case XMSS_B200_VERIFY:
            e.verify(G.ops, G.p, g.count, g.d_sm, g.d_sm_off, g.d_len, g.d_pk, g.npk, g.d_pk_index, g.d_status,
                     G.st, G.w, true);
            break;
        default: {
            if (!G.live) break;
            uint8_t* sm = sm_out ? sm_out : g.d_sm;
            const uint64_t* off = G.d_off.as<uint64_t>(G.live);
            e.sign(G.ops, G.p, G.live, G.keys.data(), G.idx.data(), sm, off, G.d_len.as<uint64_t>(G.live), G.st,
                   G.w, false);
            xb::k_put_index<<<(G.live + 127) / 128, 128, 0, G.st>>>(sm, off, G.d_ib.as<uint8_t>((size_t)G.live * 8),
                                                                   G.p.index_bytes, G.live);
            XB_CUDA(cudaGetLastError());
        }
    }
}

}  // namespace

namespace {

// The batch's groups as batches of the persistent form; sign groups write
// into sm_out (the sizing run's scratch) when given.
std::vector<Engine::PersistJob> persist_jobs(xmss_b200_batch& b, const std::vector<uint8_t*>& sm_out)
{
    std::vector<Engine::PersistJob> js;
    for (size_t i = 0; i < b.groups.size(); i++) {
        Group& G = *b.groups[i];
        const xmss_b200_batch_group& g = G.g;
        Engine::PersistJob j;
        j.ops = G.ops;
        j.p = G.p;
        j.count = g.count;
        if (g.kind == XMSS_B200_KEYGEN) {
            j.kind = xb::kJobKeygen;
            j.d_seeds = g.d_seeds;
            j.d_pk_out = g.d_pk;
            j.d_sk_out = g.d_sk;
        } else if (g.kind == XMSS_B200_VERIFY) {
            j.kind = xb::kJobVerify;
            j.d_sm = g.d_sm;
            j.d_sm_off = g.d_sm_off;
            j.d_smlen = g.d_len;
            j.d_pk = g.d_pk;
            j.npk = g.npk;
            j.d_pk_index = g.d_pk_index;
            j.d_status = g.d_status;
        } else {
            j.kind = xb::kJobSign;
            j.count = G.live;
            if (!G.live) continue;
            j.h_sk = G.keys.data();
            j.h_idx = G.idx.data();
            j.h_ibytes = G.ib.data();
            j.d_sign_sm = sm_out[i] ? sm_out[i] : g.d_sm;
            j.d_sm_off = G.d_off.as<uint64_t>(G.live);
            j.d_mlen = G.d_len.as<uint64_t>(G.live);
        }
        js.push_back(j);
    }
    return js;
}

int create(const xmss_b200_batch_group* groups, uint32_t ngroups, xmss_b200_batch** out, bool persistent);

}  // namespace

extern "C" int xmss_b200_batch_create_persistent(const xmss_b200_batch_group* groups, uint32_t ngroups,
                                                 xmss_b200_batch** out)
{
    return create(groups, ngroups, out, true);
}

extern "C" int xmss_b200_batch_create(const xmss_b200_batch_group* groups, uint32_t ngroups, xmss_b200_batch** out)
{
    return create(groups, ngroups, out, false);
}

namespace {

int create(const xmss_b200_batch_group* groups, uint32_t ngroups, xmss_b200_batch** out, bool persistent)
{
    if (!groups || !ngroups || !out) {
        xb::set_last_error("xmss_b200_batch_create: bad argument");
        return -1;
    }
    try {
        Engine& e = Engine::get();
        std::lock_guard<std::mutex> lk(e.mu);
        XB_CUDA(cudaSetDevice(e.device()));
        auto b = std::make_unique<xmss_b200_batch>();
        b->device = e.device();
        for (uint32_t i = 0; i < ngroups; i++) {
            if (!groups[i].count) continue;
            auto G = std::make_unique<Group>();
            G->g = groups[i];
            try {
                prepare(*G);
            } catch (const std::invalid_argument& ex) {
                xb::set_last_error("xmss_b200_batch_create: group " + std::to_string(i) + ": " + ex.what());
                return -1;
            }
            b->has_sign |= G->g.kind == XMSS_B200_SIGN;
            b->groups.push_back(std::move(G));
        }
        for (auto& G : b->groups) {
            XB_CUDA(cudaStreamCreateWithFlags(&G->st, cudaStreamNonBlocking));
            XB_CUDA(cudaEventCreateWithFlags(&G->join, cudaEventDisableTiming));
            G->split.create();
            G->w.split = &G->split;
        }
        XB_CUDA(cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking));
        XB_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
        const bool prof = e.profiling;
        e.profiling = false;  // the captured sequences are the production ones
        struct Restore {
            Engine& e;
            bool prof;
            ~Restore() { e.profiling = prof; }
        } restore{e, prof};
        b->persistent = persistent;
        XB_CUDA(cudaDeviceSynchronize());  // the caller's buffers are ready
        if (persistent) {
            // sizing run of the whole batch (sign groups into wiped scratch),
            // then the capture of the same launches
            std::vector<std::unique_ptr<DevBuf>> scratch;
            std::vector<uint8_t*> sm_out(b->groups.size(), nullptr);
            for (size_t i = 0; i < b->groups.size(); i++) {
                Group& G = *b->groups[i];
                if (G.g.kind != XMSS_B200_SIGN || !G.live) continue;
                scratch.emplace_back(new DevBuf());
                sm_out[i] = scratch.back()->as<uint8_t>(G.extent);
                XB_CUDA(cudaMemcpyAsync(sm_out[i], G.g.d_sm, G.extent, cudaMemcpyDeviceToDevice, b->capture));
            }
            e.persistent_multi(persist_jobs(*b, sm_out), b->capture, b->pscratch);
            for (size_t i = 0; i < b->groups.size(); i++)
                if (sm_out[i]) XB_CUDA(cudaMemsetAsync(sm_out[i], 0, b->groups[i]->extent, b->capture));
            XB_CUDA(cudaStreamSynchronize(b->capture));
            XB_CUDA(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
            try {
                e.persistent_multi(persist_jobs(*b, std::vector<uint8_t*>(b->groups.size(), nullptr)), b->capture,
                                   b->pscratch);
            } catch (...) {
                cudaGraph_t broken = nullptr;
                cudaStreamEndCapture(b->capture, &broken);
                if (broken) cudaGraphDestroy(broken);
                throw;
            }
            XB_CUDA(cudaStreamEndCapture(b->capture, &b->graph));
            XB_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
            *out = b.release();
            return 0;
        }
        // sizing run: every group once, sign groups into wiped scratch
        for (auto& G : b->groups) {
            DevBuf scratch;
            uint8_t* sm = nullptr;
            if (G->g.kind == XMSS_B200_SIGN && G->live) {
                sm = scratch.as<uint8_t>(G->extent);
                XB_CUDA(cudaMemcpyAsync(sm, G->g.d_sm, G->extent, cudaMemcpyDeviceToDevice, G->st));
            }
            run(e, *G, sm);
            if (sm) XB_CUDA(cudaMemsetAsync(sm, 0, G->extent, G->st));
            XB_CUDA(cudaStreamSynchronize(G->st));
        }
        // capture: fork from the capture stream into every group's stream, join back
        XB_CUDA(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
        try {
            XB_CUDA(cudaEventRecord(b->fork, b->capture));
            for (auto& G : b->groups) {
                XB_CUDA(cudaStreamWaitEvent(G->st, b->fork, 0));
                run(e, *G, nullptr);
                XB_CUDA(cudaEventRecord(G->join, G->st));
                XB_CUDA(cudaStreamWaitEvent(b->capture, G->join, 0));
            }
        } catch (...) {
            cudaGraph_t broken = nullptr;
            cudaStreamEndCapture(b->capture, &broken);
            if (broken) cudaGraphDestroy(broken);
            throw;
        }
        XB_CUDA(cudaStreamEndCapture(b->capture, &b->graph));
        XB_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
        *out = b.release();
        return 0;
    } catch (const std::invalid_argument& ex) {
        xb::set_last_error(std::string("xmss_b200_batch_create: ") + ex.what());
        return -1;
    } catch (const std::exception& ex) {
        xb::set_last_error(std::string("xmss_b200_batch_create: ") + ex.what());
        return -3;
    }
}

}  // namespace

extern "C" int xmss_b200_batch_launch(xmss_b200_batch* b, void* stream)
{
    if (!b) return -1;
    if (b->has_sign && b->launched) {
        xb::set_last_error("xmss_b200_batch_launch: the batch's signing indices are used (it has run once)");
        return -2;
    }
    cudaError_t err = cudaSetDevice(b->device);
    if (err == cudaSuccess) err = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    if (err != cudaSuccess) {
        xb::set_last_error(std::string("xmss_b200_batch_launch: ") + cudaGetErrorString(err));
        return -3;
    }
    b->launched = true;
    return 0;
}

extern "C" void xmss_b200_batch_destroy(xmss_b200_batch* b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();  // no launch of it may still run
    delete b;
}
