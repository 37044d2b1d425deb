// Launchers that bind the templated kernels of one family into a FamilyOps
// table.  Included by exactly one fam_*.cu per family.
#pragma once

#include <algorithm>

#include "family_ops.h"
#include "verify_persist.cuh"
#include "xmss_kernels.cuh"

namespace xb {

constexpr int kBlock = 128;

inline unsigned grid_for(uint64_t items, unsigned block = kBlock)
{
    return (unsigned)((items + block - 1) / block);
}

// Launch with programmatic stream serialization: the kernel starts launching
// as the CTAs of the kernel before it in the stream exit and synchronises
// with it through pdl_wait() (xmss_kernels.cuh).  A plain launch where the
// attribute is refused (same results; only the overlap is lost).
template <class... KArgs, class... Args>
inline void launch_pdl(void (*kernel)(KArgs...), unsigned grid, unsigned block, cudaStream_t st, Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, kernel, args...) != cudaSuccess) {
        (void)cudaGetLastError();
        kernel<<<grid, block, 0, st>>>(args...);
    }
}

// F runs every kernel except the chain kernels, which run FT (the same
// family with another SHA-256 pipe mix; Ctx and HPre are shared).
template <class F, class FT = F>
struct Launch {
    using Ctx = typename F::Ctx;
    static inline unsigned s_func = 0;  // set by table()
    static const Tuning& tune() { return tuning_for(s_func, (unsigned)F::N); }
    static_assert(sizeof(typename FT::Ctx) == sizeof(Ctx), "chain family must share the key context");

    static void make_ctx(const uint8_t* pub, uint32_t pub_stride, const uint8_t* sks, uint32_t sks_stride,
                         const uint8_t* skp, uint32_t skp_stride, uint32_t nkeys, void* ctx, cudaStream_t st)
    {
        if (!nkeys) return;
        k_make_ctx<F><<<grid_for(nkeys), kBlock, 0, st>>>(pub, pub_stride, sks, sks_stride, skp, skp_stride, nkeys,
                                                          (Ctx*)ctx);
    }
    static void keygen_chains(const TreeJob* jobs, int h, uint64_t slot0, uint64_t nslots, const void* ctx,
                              uint8_t* wpk, LeafRef* refs, cudaStream_t st)
    {
        const uint64_t items = nslots * F::LEN;
        if (!items) return;
        const unsigned b = tune().keygen_chain_block;
        k_keygen_chains<FT>
            <<<grid_for(items, b), b, 0, st>>>(jobs, h, slot0, nslots, (const typename FT::Ctx*)ctx, wpk, refs);
    }
    static void ltree_level(const LeafRef* refs, uint32_t nslots, int level, int cnt_in, const uint8_t* src,
                            uint32_t src_stride, uint8_t* dst, uint32_t dst_stride, uint8_t* leaf_out,
                            const void* ctx, const int* status, cudaStream_t st)
    {
        const uint64_t items = (uint64_t)nslots * ((cnt_in + 1) / 2);
        if (!items) return;
        const unsigned b = tune().level_block;
        k_ltree_level<F><<<grid_for(items, b), b, 0, st>>>(refs, nslots, level, cnt_in, src, src_stride, dst,
                                                            dst_stride, leaf_out, (const Ctx*)ctx, status);
    }
    static void tree_level(const TreeJob* jobs, uint32_t njobs, int h, int level, uint8_t* nodes, const void* ctx,
                           cudaStream_t st)
    {
        const uint64_t items = (uint64_t)njobs << (h - level - 1);
        if (!items) return;
        const unsigned b = tune().level_block;
        k_tree_level<F><<<grid_for(items, b), b, 0, st>>>(jobs, njobs, h, level, nodes, (const Ctx*)ctx);
    }
    static void keygen_subtree(const TreeJob* jobs, uint32_t njobs, int h, int k, const void* ctx, uint8_t* nodes,
                               cudaStream_t st)
    {
        if (!njobs || k < 1 || k > 7 || k > h) return;
        const unsigned b = 1u << k;
        // opt in to more than 48 KB of dynamic shared memory where the
        // widest family needs it (n = 64: 80 KB at 128 threads)
        static const bool attr = [] {
            return cudaFuncSetAttribute(k_keygen_subtree<FT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)subtree_smem<FT>(128)) == cudaSuccess;
        }();
        (void)attr;
        const uint64_t ctas = (uint64_t)njobs << (h - k);
        for (uint64_t c0 = 0; c0 < ctas; c0 += 1u << 30)
            k_keygen_subtree<FT><<<(unsigned)std::min<uint64_t>(ctas - c0, 1u << 30), b, subtree_smem<FT>(b), st>>>(
                jobs, h, k, c0, (const typename FT::Ctx*)ctx, nodes);
    }
    static void verify_partition(const VerifyArgs& v, uint32_t blocks_max, uint32_t* sel_short, uint32_t* sel_long,
                                 uint32_t* n2, cudaStream_t st)
    {
        if (!v.count) return;
        k_verify_partition<F><<<grid_for(v.count), kBlock, 0, st>>>(v, blocks_max, sel_short, sel_long, n2);
    }
    static void verify_prep(const VerifyArgs& v, const void* ctx, cudaStream_t st)
    {
        if (!v.count) return;
        const uint64_t pre = (uint64_t)v.count * v.d * (F::LEN - 1 + v.tree_height);
        if constexpr (kWarpHmsg<F>) {
            // H_msg one warp per signature, beside the h_pre blocks
            const uint32_t hw = (v.count + 1) / 2;
            k_verify_hmsg_warp<F><<<(unsigned)(hw + (pre + 63) / 64), 64, 0, st>>>(v, hw, (const Ctx*)ctx);
            return;
        }
        const uint32_t hb = (v.count + 63) / 64;
        k_verify_prep<F><<<(unsigned)(hb + (pre + 63) / 64), 64, 0, st>>>(v, hb, (const Ctx*)ctx);
    }
    static void verify_prep_part(const VerifyArgs& v, const void* ctx, cudaStream_t st, int part)
    {
        if (!v.count) return;
        if (part == 1) {
            if constexpr (kWarpHmsg<F>) {
                const uint32_t hw = (v.count + 1) / 2;
                k_verify_hmsg_warp<F><<<hw, 64, 0, st>>>(v, hw, (const Ctx*)ctx);
                return;
            }
            const uint32_t hb = (v.count + 63) / 64;
            k_verify_prep<F, 1><<<hb, 64, 0, st>>>(v, hb, (const Ctx*)ctx);
            return;
        }
        // the h_pre blocks alone (the chain kernels' pipe mix and 128-thread
        // CTAs measured slower here)
        const uint64_t pre = (uint64_t)v.count * v.d * (F::LEN - 1 + v.tree_height);
        k_verify_prep<F, 2><<<grid_for(pre, 64), 64, 0, st>>>(v, 0, (const Ctx*)ctx);
    }
    static void verify_scatter(const VerifyArgs& v, uint32_t layer, cudaStream_t st)
    {
        const uint64_t items = (uint64_t)v.count * F::LEN;
        if (!items) return;
        k_verify_scatter<F><<<(unsigned)((items + 255) / 256), 256, 0, st>>>(v, layer);
    }
    static void verify_chains(const VerifyArgs& v, uint32_t layer, const void* ctx, cudaStream_t st)
    {
        const uint64_t items = (uint64_t)v.count * F::LEN;
        if (!items) return;
        const unsigned b = tune().verify_chain_block;
        k_verify_chains<FT><<<grid_for(items, b), b, 0, st>>>(v, layer, (const typename FT::Ctx*)ctx);
    }
    static void verify_ltree(const VerifyArgs& v, uint32_t layer, int cnt_in, uint32_t node_base,
                             const uint8_t* src, uint32_t src_stride, uint8_t* dst, uint32_t dst_stride,
                             cudaStream_t st)
    {
        const uint64_t items = (uint64_t)v.count * ((cnt_in + 1) / 2);
        if (!items) return;
        const unsigned b = tune().level_block;
        // the first level follows the chains (and, in a split batch, an
        // event wait): a plain launch; later levels follow the level before
        if (cnt_in == (int)F::LEN)
            k_verify_ltree<F><<<grid_for(items, b), b, 0, st>>>(v, layer, cnt_in, node_base, src, src_stride, dst,
                                                                dst_stride);
        else
            launch_pdl(k_verify_ltree<F>, grid_for(items, b), b, st, v, layer, cnt_in, node_base, src, src_stride,
                       dst, dst_stride);
    }
    static void verify_ltree_warp(const VerifyArgs& v, uint32_t layer, cudaStream_t st)
    {
        if (!v.count) return;
        k_verify_ltree_warp<F><<<(v.count + 1) / 2, 64, 0, st>>>(v, layer);
    }
    static void verify_root(const VerifyArgs& v, uint32_t layer, cudaStream_t st)
    {
        if (!v.count) return;
        launch_pdl(k_verify_root<F>, (v.count + 63) / 64, 64, st, v, layer);
    }
    static void verify_persist(const VerifyArgs& v, const PersistArgs& q, cudaStream_t st)
    {
        if (!v.count) return;
        // as many CTAs as fit on the GPU at once: each loops over the ticket
        // sequence (more would only queue behind them; fewer leave SMs idle)
        static const unsigned grid = [] {
            int dev = 0, sms = 0, per = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_verify_persist<F, FT>, 128, 0);
            return (unsigned)(sms * (per > 0 ? per : 1));
        }();
        k_verify_persist<F, FT><<<grid, 128, 0, st>>>(v, q);
    }
    template <bool GEN>
    static unsigned persist_multi_grid()
    {
        static const unsigned grid = [] {
            int dev = 0, sms = 0, per = 0;
            cudaGetDevice(&dev);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_verify_persist_multi<F, FT, GEN>, 128, 0);
            return (unsigned)(sms * (per > 0 ? per : 1));
        }();
        return grid;
    }
    static void verify_persist_multi(const PersistJobs& P, cudaStream_t st)
    {
        if (!P.njobs) return;
        bool gen = false;
        for (uint32_t k = 0; k < P.njobs; k++) gen |= P.job[k].kind != kJobVerify;
        if (gen)
            k_verify_persist_multi<F, FT, true><<<persist_multi_grid<true>(), 128, 0, st>>>(P);
        else
            k_verify_persist_multi<F, FT, false><<<persist_multi_grid<false>(), 128, 0, st>>>(P);
    }
    static void sign_prep(const SignArgs& g, const void* ctx, cudaStream_t st)
    {
        if (!g.count) return;
        if constexpr (kWarpHmsg<F>) {
            k_sign_hmsg_warp<F><<<(g.count + 1) / 2, 64, 0, st>>>(g, (const Ctx*)ctx);
            k_sign_prep<F, true><<<(g.count + 63) / 64, 64, 0, st>>>(g, (const Ctx*)ctx);
            return;
        }
        k_sign_prep<F><<<(g.count + 63) / 64, 64, 0, st>>>(g, (const Ctx*)ctx);
    }
    // sign_prep in two parts: R, H_msg and layer 0's chain lengths (needs no
    // subtree), then the other layers' chain lengths and the authentication
    // paths (needs the subtrees)
    static void sign_hmsg(const SignArgs& g, const void* ctx, cudaStream_t st)
    {
        if (!g.count) return;
        if constexpr (kWarpHmsg<F>) {
            k_sign_hmsg_warp<F><<<(g.count + 1) / 2, 64, 0, st>>>(g, (const Ctx*)ctx);
            return;
        }
        k_sign_hmsg<F><<<(g.count + 63) / 64, 64, 0, st>>>(g, (const Ctx*)ctx);
    }
    static void sign_prep_rest(const SignArgs& g, const void* ctx, cudaStream_t st)
    {
        if (!g.count) return;
        k_sign_prep<F, true><<<(g.count + 63) / 64, 64, 0, st>>>(g, (const Ctx*)ctx);
    }
    static void sign_chains(const SignArgs& g, const void* ctx, cudaStream_t st)
    {
        const uint64_t items = (uint64_t)g.count * g.d * F::LEN;
        if (!items) return;
        const unsigned b = tune().keygen_chain_block;
        k_sign_chains<FT><<<grid_for(items, b), b, 0, st>>>(g, (const typename FT::Ctx*)ctx);
    }
    static void core_hash(const uint8_t* msgs, const uint64_t* off, const uint64_t* len, uint32_t count,
                          uint8_t* out, cudaStream_t st)
    {
        if (!count) return;
        k_core_hash<F><<<(count + 63) / 64, 64, 0, st>>>(msgs, off, len, count, out);
    }

    static FamilyOps table(const char* name, unsigned func)
    {
        FamilyOps o{};
        s_func = func;
        o.name = name;
        o.func = func;
        o.n = (unsigned)F::N;
        o.len = (unsigned)F::LEN;
        o.ctx_bytes = sizeof(Ctx);
        o.make_ctx = make_ctx;
        o.keygen_chains = keygen_chains;
        o.ltree_level = ltree_level;
        o.tree_level = tree_level;
        o.keygen_subtree = keygen_subtree;
        o.hpre_bytes = sizeof(typename F::HPre);
        o.verify_partition = verify_partition;
        o.verify_prep = verify_prep;
        o.verify_prep_part = verify_prep_part;
        o.verify_scatter = verify_scatter;
        o.verify_chains = verify_chains;
        o.verify_ltree = verify_ltree;
        o.verify_root = verify_root;
        o.verify_ltree_warp = verify_ltree_warp;
        o.verify_persist = verify_persist;
        o.verify_persist_multi = verify_persist_multi;
        o.sign_prep = sign_prep;
        o.sign_hmsg = sign_hmsg;
        o.sign_prep_rest = sign_prep_rest;
        o.sign_chains = sign_chains;
        o.core_hash = core_hash;
        return o;
    }
};

}  // namespace xb
