// CUDA-graph form of the device verify (xmss_b200_verify_graph_*): the
// launch sequence of one fixed-shape batch - per-key contexts, preparation,
// the optional two-group split on a second stream, chains, L-tree levels,
// roots - captured once and replayed with a single launch.
//
// The graph owns its scratch (a Workspace and split streams of its own):
// one uncaptured run sizes every buffer, so the captured sequence allocates
// nothing and always reads and writes the same device addresses.
#include <cuda_runtime.h>

#include <memory>
#include <string>

#include "../../include/params.h"
#include "../../include/xmss_b200.h"
#include "engine.h"

namespace xb {
void set_last_error(const std::string& msg);  // api.cu
}

struct xmss_b200_verify_graph {
    xb::SplitStreams split;
    xb::Workspace w;
    cudaStream_t capture = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
    ~xmss_b200_verify_graph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (capture) cudaStreamDestroy(capture);
        split.destroy();
    }
};

extern "C" int xmss_b200_verify_graph_create(uint32_t oid, int mt, uint32_t count, const uint8_t* d_sm,
                                             const uint64_t* d_sm_off, const uint64_t* d_smlen, const uint8_t* d_pk,
                                             uint32_t npk, const uint32_t* d_pk_index, int* d_status,
                                             xmss_b200_verify_graph** out)
{
    xmss_params p;
    if ((mt ? xmssmt_parse_oid(&p, oid) : xmss_parse_oid(&p, oid)) != 0 || !out || !count || !npk ||
        !d_pk_index) {
        xb::set_last_error("xmss_b200_verify_graph_create: bad argument");
        return -1;
    }
    try {
        xb::Engine& e = xb::Engine::get();
        std::lock_guard<std::mutex> lk(e.mu);
        XB_CUDA(cudaSetDevice(e.device()));
        const xb::FamilyOps* ops = xb::ops_for(p);
        auto g = std::make_unique<xmss_b200_verify_graph>();
        g->device = e.device();
        g->split.create();
        g->w.split = &g->split;
        XB_CUDA(cudaStreamCreateWithFlags(&g->capture, cudaStreamNonBlocking));
        const bool prof = e.profiling;
        e.profiling = false;  // the captured sequence is the production one
        // sizing run, then the capture of the same sequence
        e.verify(ops, p, count, d_sm, d_sm_off, d_smlen, d_pk, npk, d_pk_index, d_status, g->capture, g->w, true);
        XB_CUDA(cudaStreamSynchronize(g->capture));
        XB_CUDA(cudaStreamBeginCapture(g->capture, cudaStreamCaptureModeThreadLocal));
        try {
            e.verify(ops, p, count, d_sm, d_sm_off, d_smlen, d_pk, npk, d_pk_index, d_status, g->capture, g->w,
                     true);
        } catch (...) {
            cudaGraph_t broken = nullptr;
            cudaStreamEndCapture(g->capture, &broken);
            if (broken) cudaGraphDestroy(broken);
            e.profiling = prof;
            throw;
        }
        XB_CUDA(cudaStreamEndCapture(g->capture, &g->graph));
        e.profiling = prof;
        XB_CUDA(cudaGraphInstantiate(&g->exec, g->graph, 0));
        *out = g.release();
        return 0;
    } catch (const std::exception& ex) {
        xb::set_last_error(std::string("xmss_b200_verify_graph_create: ") + ex.what());
        return -3;
    }
}

extern "C" int xmss_b200_verify_graph_launch(xmss_b200_verify_graph* g, void* stream)
{
    if (!g) return -1;
    cudaError_t err = cudaSetDevice(g->device);
    if (err == cudaSuccess) err = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
    if (err != cudaSuccess) {
        xb::set_last_error(std::string("xmss_b200_verify_graph_launch: ") + cudaGetErrorString(err));
        return -3;
    }
    return 0;
}

extern "C" void xmss_b200_verify_graph_destroy(xmss_b200_verify_graph* g)
{
    if (!g) return;
    cudaSetDevice(g->device);
    cudaDeviceSynchronize();  // no launch of it may still run
    delete g;
}
