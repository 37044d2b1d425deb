// Host-side launch table of one hash family.  Each fam_*.cu translation
// unit instantiates the kernels of xmss_kernels.cuh for its family and
// fills one FamilyOps; the engine picks the table by (func, n).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace xb {

struct LeafRef;
struct TreeJob;
struct VerifyArgs;
struct SignArgs;
struct PersistArgs;
struct PersistJobs;

// Kinds of the batches of a persistent multi-batch launch.
enum : uint32_t { kJobVerify = 0, kJobKeygen = 1, kJobSign = 2 };

struct FamilyOps {
    const char* name;
    unsigned func, n, len;
    size_t ctx_bytes;  // sizeof(F::Ctx)
    void (*make_ctx)(const uint8_t* pub, uint32_t pub_stride, const uint8_t* sks, uint32_t sks_stride,
                     const uint8_t* skp, uint32_t skp_stride, uint32_t nkeys, void* ctx, cudaStream_t st);
    void (*keygen_chains)(const TreeJob* jobs, int h, uint64_t slot0, uint64_t nslots, const void* ctx,
                          uint8_t* wpk, LeafRef* refs, cudaStream_t st);
    void (*ltree_level)(const LeafRef* refs, uint32_t nslots, int level, int cnt_in, const uint8_t* src,
                        uint32_t src_stride, uint8_t* dst, uint32_t dst_stride, uint8_t* leaf_out, const void* ctx,
                        const int* status, cudaStream_t st);
    void (*tree_level)(const TreeJob* jobs, uint32_t njobs, int h, int level, uint8_t* nodes, const void* ctx,
                       cudaStream_t st);
    // levels 0..k of every job's tree as in-CTA subtrees of 2^k leaves, one thread per leaf (k = 5, 6, 7; k <= h)
    void (*keygen_subtree)(const TreeJob* jobs, uint32_t njobs, int h, int k, const void* ctx, uint8_t* nodes,
                           cudaStream_t st);
    size_t hpre_bytes;  // sizeof(F::HPre)
    void (*verify_partition)(const VerifyArgs& v, uint32_t blocks_max, uint32_t* sel_short, uint32_t* sel_long,
                             uint32_t* n2, cudaStream_t st);
    void (*verify_prep)(const VerifyArgs& v, const void* ctx, cudaStream_t st);
    // one part of verify_prep: H_msg (part 1) or the h_pre items (part 2)
    void (*verify_prep_part)(const VerifyArgs& v, const void* ctx, cudaStream_t st, int part);
    void (*verify_scatter)(const VerifyArgs& v, uint32_t layer, cudaStream_t st);
    void (*verify_chains)(const VerifyArgs& v, uint32_t layer, const void* ctx, cudaStream_t st);
    void (*verify_ltree)(const VerifyArgs& v, uint32_t layer, int cnt_in, uint32_t node_base, const uint8_t* src,
                         uint32_t src_stride, uint8_t* dst, uint32_t dst_stride, cudaStream_t st);
    void (*verify_root)(const VerifyArgs& v, uint32_t layer, cudaStream_t st);
    void (*verify_ltree_warp)(const VerifyArgs& v, uint32_t layer, cudaStream_t st);  // whole L-tree, warp / sig
    // the whole verify (every layer) as one persistent launch (verify_persist.cuh)
    void (*verify_persist)(const VerifyArgs& v, const PersistArgs& q, cudaStream_t st);
    // several batches of this family's parameter sets as one persistent launch
    void (*verify_persist_multi)(const PersistJobs& jobs, cudaStream_t st);
    void (*sign_prep)(const SignArgs& g, const void* ctx, cudaStream_t st);
    // sign_prep's two parts: R, H_msg, layer 0's chain lengths (no subtree
    // needed); the other layers' chain lengths and the authentication paths
    void (*sign_hmsg)(const SignArgs& g, const void* ctx, cudaStream_t st);
    void (*sign_prep_rest)(const SignArgs& g, const void* ctx, cudaStream_t st);
    void (*sign_chains)(const SignArgs& g, const void* ctx, cudaStream_t st);
    void (*core_hash)(const uint8_t* msgs, const uint64_t* off, const uint64_t* len, uint32_t count, uint8_t* out,
                      cudaStream_t st);
};

// nullptr when (func, n) has no instantiation.
const FamilyOps* family_ops(unsigned func, unsigned n);

// Launch shapes of one hash family (set by the autotuner, tune.cu).  CTA
// sizes are 32, 64 or 128 threads.
struct Tuning {
    uint32_t verify_chain_block = 128;  // k_verify_chains
    uint32_t keygen_chain_block = 128;  // k_keygen_chains, k_sign_chains
    uint32_t level_block = 128;         // L-tree and Merkle-level kernels
    uint32_t split_min = 1024;          // verify batches this large run as two groups ...
    uint32_t short_hmsg_blocks = 16;    // ... split at this many H_msg blocks
    uint32_t prep_split = 1;            // split batches: h_pre in its own launch (1) or in each group's prep (0)
};
Tuning& tuning_for(unsigned func, unsigned n);

// How subtrees of one parameter set are built (set by the autotuner, tune.cu;
// keyed by the parameter set, i.e. its OID).
struct TreeShape {
    uint32_t subtree_height = 0;  // 0: one thread per WOTS chain, a launch per L-tree / Merkle level;
                                  // 5, 6, 7: in-CTA subtrees of 2^k leaves, one thread per leaf
    uint64_t min_leaves = 0;      // builds of fewer leaves use the one-thread-per-chain form
};
TreeShape& tree_shape_for(unsigned func, unsigned n, unsigned full_height, unsigned d);

// The in-CTA subtree height to build `leaves` leaves of subtrees of height
// h with (0: the one-thread-per-chain form).
int subtree_height_for(const TreeShape& s, int h, uint64_t leaves);

extern const FamilyOps kOpsSha256N32;
extern const FamilyOps kOpsSha256N24;
extern const FamilyOps kOpsSha512N64;
extern const FamilyOps kOpsShake128N32;
extern const FamilyOps kOpsShake256N24;
extern const FamilyOps kOpsShake256N32;
extern const FamilyOps kOpsShake256N64;

}  // namespace xb
