// Batched verify that allocates no memory: xmss_b200_sign_open_device_noalloc.
//
// Some callers cannot allocate device memory at the moment they verify: a
// request path with a hard latency budget cannot afford cudaMalloc (which may
// synchronise the device and take milliseconds), a process whose device
// memory is owned by another allocator or capped by a fixed budget must not
// grow its footprint on demand, and code that runs where the CUDA allocation
// API must not be called at all is in the same position.  This entry point
// serves them: it takes the same device-resident inputs and outputs as
// xmss_b200_sign_open_device, but all of its intermediate buffers are carved
// out of one fixed array in device memory (g_noalloc_scratch below) instead
// of the library's growable scratch, and it calls no cudaMalloc, cudaFree or
// other allocating routine.
//
// Limits and sharing:
//   * The array is kNoallocScratchBytes (8 MiB) per GPU and lives as long as
//     the library stays loaded; every GPU the process uses holds one copy.
//   * A call whose buffers do not fit is rejected with -1 (see
//     xmss_b200_last_error); XMSS-SHA2_10_256 fits up to about 760
//     signatures per call (about 11 KB of scratch each).
//   * All calls share the one array, so calls whose GPU work overlaps (for
//     example on two streams without ordering between them) race and give
//     wrong results; callers serialise them.  The array keeps whatever the
//     last call left in it; every buffer that must start at zero is cleared
//     on the stream at the start of each call.
//   * The first call on each device is its set-up: with that device current
//     it looks up the array's device address (cudaGetSymbolAddress), which
//     loads the library's device code on that device if it is not loaded
//     yet; make that first call before capturing any stream.  Later calls
//     repeat the lookup (a table lookup once the code is loaded, no
//     allocation), so the address is never stale: after cudaDeviceReset, or
//     under another context, the call uses the array of the context that is
//     current then.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/params.h"
#include "../../include/xmss_b200.h"
#include "family_ops.h"
#include "xmss_kernels.cuh"

namespace xb {
void set_last_error(const std::string& msg);  // api.cu
}

namespace {

constexpr size_t kNoallocScratchBytes = 8u << 20;

// The fixed scratch array.  In host code this name is only a stand-in for the
// symbol; kernels receive the device address looked up below.
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoallocScratchBytes];

// Device address of g_noalloc_scratch in the current context (the device the
// call runs on must be current).
cudaError_t scratch_address(void** out)
{
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    *out = p;
    return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

extern "C" int xmss_b200_sign_open_device_noalloc(uint32_t oid, int mt, uint32_t count, const uint8_t* d_sm,
                                                  const uint64_t* d_sm_off, const uint64_t* d_smlen,
                                                  const uint8_t* d_pk, uint32_t npk, const uint32_t* d_pk_index,
                                                  int* d_status, void* stream)
{
    using namespace xb;
    xmss_params p;
    if ((mt ? xmssmt_parse_oid(&p, oid) : xmss_parse_oid(&p, oid)) != 0) {
        set_last_error("xmss_b200_sign_open_device_noalloc: unknown OID");
        return -1;
    }
    const FamilyOps* ops = family_ops(p.func, p.n);
    if (!ops) {
        set_last_error("xmss_b200_sign_open_device_noalloc: parameter set not supported");
        return -1;
    }
    if (!count) return 0;
    if (!d_pk_index || !npk) {
        set_last_error("xmss_b200_sign_open_device_noalloc: d_pk_index and npk are required");
        return -1;
    }
    const uint32_t n = p.n, len = ops->len, nh = len - 1 + p.tree_height;
    // carve the scratch: same buffers as the growable path
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off = align256(off + bytes);
        return o;
    };
    const size_t o_ctx = take((size_t)npk * ops->ctx_bytes);
    const size_t o_node = take((size_t)count * n);
    const size_t o_lens = take((size_t)count * len);
    const size_t o_idx = take((size_t)count * sizeof(uint64_t));
    const size_t o_wpk = take((size_t)count * len * n);
    const size_t o_wpk2 = take((size_t)count * ((len + 1) / 2) * n);
    const size_t o_leaf = take((size_t)count * n);
    const size_t o_refs = take((size_t)count * sizeof(LeafRef));
    const size_t o_hpre = take((size_t)count * p.d * nh * ops->hpre_bytes);
    const size_t o_hist = take((size_t)32 * p.d * sizeof(uint32_t));
    const size_t o_list = take((size_t)count * len * sizeof(uint32_t));
    if (off > kNoallocScratchBytes) {
        set_last_error("xmss_b200_sign_open_device_noalloc: " + std::to_string(count) + " signatures need " +
                       std::to_string(off) + " bytes of scratch, more than the fixed " +
                       std::to_string(kNoallocScratchBytes) + "; split the batch");
        return -1;
    }
    uint8_t* base = nullptr;
    cudaError_t e = scratch_address((void**)&base);
    if (e != cudaSuccess) {
        set_last_error(std::string("xmss_b200_sign_open_device_noalloc: ") + cudaGetErrorString(e));
        return -3;
    }
    cudaStream_t st = (cudaStream_t)stream;
    void* ctx = base + o_ctx;
    VerifyArgs v;
    v.sm = d_sm;
    v.sm_off = d_sm_off;
    v.smlen = d_smlen;
    v.key = d_pk_index;
    v.key_root = d_pk;
    v.key_stride = 2 * n;
    v.npk = npk;
    v.node = base + o_node;
    v.lens = base + o_lens;
    v.idx = (uint64_t*)(base + o_idx);
    v.status = d_status;
    v.wpk = base + o_wpk;
    v.wpk2 = base + o_wpk2;
    v.leaf = base + o_leaf;
    v.refs = (LeafRef*)(base + o_refs);
    v.hpre = base + o_hpre;
    v.hist = (uint32_t*)(base + o_hist);
    v.list = (uint32_t*)(base + o_list);
    v.sel = nullptr;
    v.sel_n = nullptr;
    v.work = nullptr;
    v.count = count;
    v.index_bytes = p.index_bytes;
    v.sig_bytes = p.sig_bytes;
    v.tree_height = p.tree_height;
    v.d = p.d;
    // the bucket counters start at zero on every call
    e = cudaMemsetAsync(v.hist, 0, 32 * p.d * sizeof(uint32_t), st);
    if (e == cudaSuccess) {
        ops->make_ctx(d_pk + n, 2 * n, nullptr, 0, nullptr, 0, npk, ctx, st);
        ops->verify_prep(v, ctx, st);
        for (uint32_t layer = 0; layer < p.d; layer++) {
            ops->verify_scatter(v, layer, st);
            ops->verify_chains(v, layer, ctx, st);
            int cnt = (int)len;
            uint32_t node_base = 0;
            uint8_t *src = v.wpk, *dst = v.wpk2;
            uint32_t sstr = len, dstr = (len + 1) / 2;
            while (cnt > 1) {
                ops->verify_ltree(v, layer, cnt, node_base, src, sstr, dst, dstr, st);
                node_base += cnt / 2;
                cnt = (cnt + 1) / 2;
                uint8_t* t = src;
                src = dst;
                dst = t;
                const uint32_t ts = sstr;
                sstr = dstr;
                dstr = ts;
            }
            ops->verify_root(v, layer, st);
        }
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        set_last_error(std::string("xmss_b200_sign_open_device_noalloc: ") + cudaGetErrorString(e));
        return -3;
    }
    return 0;
}
