/*
 * Batch and device-resident extensions of libxmss_b200.so.
 *
 * These entry points have no single counterpart in the reference's CPU API
 * (cuxmss/xmss.h); each one batches many calls of a reference function and
 * says which.  Their batch shapes follow the reference's GPU host API
 * (cuxmss/gpu/gpu_verify.h, gpu_sign_origin.h, gpu_keypair_origin.h: arrays
 * of signed messages / keys processed in one call), with per-item offsets so
 * messages may have different lengths.
 *
 * Return codes: 0 ok, -1 unknown / mixed OID or bad argument, -3 GPU
 * failure (text in xmss_b200_last_error()).  Per-item results go to the
 * `status` / `ret` arrays with the reference's codes (0, -1, -2).
 *
 * Host-buffer calls are synchronous.  Device-pointer calls (suffix _device)
 * are asynchronous on the given CUDA stream (cudaStream_t passed as void*;
 * NULL = legacy default stream); they share the library's scratch memory, so
 * a call waits for the previous call's work before reusing it.
 */
#ifndef XMSS_B200_H
#define XMSS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Binds the library to a CUDA device (default: the current device at first
 * use).  0 ok, -3 no usable GPU. */
int xmss_b200_init(int device);

/* Text of the last failure on this thread ("" if none). */
const char *xmss_b200_last_error(void);

/* Replaces the randomness source used by xmss_keypair / xmssmt_keypair
 * (default: /dev/urandom as cuxmss/randombytes.c:10-39).  NULL restores it. */
void xmss_b200_set_randombytes(void (*fn)(unsigned char *x, unsigned long long xlen));

/* 1 when (func, n) has a GPU implementation (all seven families of
 * cuxmss/hash.c:29-65 do). */
int xmss_b200_supported(unsigned int func, unsigned int n);

/* Batched xmssmt_core_seed_keypair (xmss_core.c:134-161) for `count` keys of
 * one OID.  seeds: count x 3n bytes (SK_SEED || SK_PRF || PUB_SEED).
 * pk: count x (4 + 2n) and sk: count x (4 + sk_bytes), OID-prefixed as
 * xmss_keypair writes them (xmss.c:10-26). */
int xmss_b200_keypair_batch(uint32_t oid, int mt, uint32_t count, const uint8_t *seeds,
                            uint8_t *pk, uint8_t *sk);

/* Device form of xmss_b200_keypair_batch without OID prefixes:
 * d_pk count x 2n, d_sk count x sk_bytes. */
int xmss_b200_keypair_device(uint32_t oid, int mt, uint32_t count, const uint8_t *d_seeds,
                             uint8_t *d_pk, uint8_t *d_sk, void *stream);

/* Batched xmss[mt]_sign_open (xmss.c:45-60, 95-109).  Signed message i is
 * sm[sm_off[i] .. sm_off[i] + smlen[i]); it is checked against
 * pk[pk_index[i]] (pk_index NULL: pk[i]), pk holding npk OID-prefixed keys
 * (4 + 2n bytes each) of one OID.  status[i] = 0 valid, -1 invalid. */
int xmss_b200_sign_open_batch(int mt, uint32_t count, const uint8_t *sm, const uint64_t *sm_off,
                              const uint64_t *smlen, const uint8_t *pk, uint32_t npk,
                              const uint32_t *pk_index, int *status);

/* Device form of xmss_b200_sign_open_batch: all pointers on the device,
 * d_pk = npk x 2n bytes (root || PUB_SEED, no OID), d_pk_index required. */
int xmss_b200_sign_open_device(uint32_t oid, int mt, uint32_t count, const uint8_t *d_sm,
                               const uint64_t *d_sm_off, const uint64_t *d_smlen,
                               const uint8_t *d_pk, uint32_t npk, const uint32_t *d_pk_index,
                               int *d_status, void *stream);

/* Persistent form of xmss_b200_sign_open_device (same arguments, same
 * statuses): the whole batch, every XMSS^MT layer included, runs as ONE
 * kernel launch whose warps take tasks from a device work queue (a ticket
 * counter over key contexts, H_msg, L-tree precomputation, WOTS chains
 * bucketed longest first, L-tree levels and compute_root, in dependency
 * order).  Every dependency wait inside the launch is bounded; if one runs
 * out (a single H_msg taking seconds, i.e. a message of hundreds of MB)
 * every status of the batch is -3.  Replaces, like xmss_b200_sign_open_device,
 * a loop of xmss[mt]_sign_open calls (xmss.c:45-60, 95-109). */
int xmss_b200_sign_open_device_persistent(uint32_t oid, int mt, uint32_t count, const uint8_t *d_sm,
                                          const uint64_t *d_sm_off, const uint64_t *d_smlen,
                                          const uint8_t *d_pk, uint32_t npk, const uint32_t *d_pk_index,
                                          int *d_status, void *stream);

/* Persistent form over several batches of ANY parameter sets (XMSS and
 * XMSS^MT, every family): the batches of one hash family run as ONE
 * persistent launch (up to 8 batches per launch; each batch's tickets
 * follow the previous batch's in one shared ticket sequence, so the next
 * batch's work fills the SMs during one batch's serial tail), and the
 * families' launches run concurrently on streams forked from `stream` and
 * joined back into it (capturable in a CUDA graph).  Each batch gets the
 * statuses of xmss_b200_sign_open_device; a batch whose dependency wait runs
 * out gets -3 in every status, the others finish.  Asynchronous on stream;
 * 0 ok, -1 bad job (unknown OID, missing pointer), -3 GPU failure. */
typedef struct {
    uint32_t oid;
    int mt;
    uint32_t count;
    const uint8_t *d_sm;
    const uint64_t *d_sm_off;
    const uint64_t *d_smlen;
    const uint8_t *d_pk;         /* npk x 2n (root || PUB_SEED) */
    uint32_t npk;
    const uint32_t *d_pk_index;
    int *d_status;
} xmss_b200_verify_job;

int xmss_b200_sign_open_device_persistent_multi(const xmss_b200_verify_job *jobs, uint32_t njobs, void *stream);

/* Bound of one dependency wait inside a persistent launch, in ns of the
 * GPU's global timer;
 * 0 restores the default of 8 s.  A wait that runs out ends the launch with
 * -3 in every status instead of waiting on; the bound is passed to each
 * launch as an argument, so it applies to launches made after the call.
 * No reference counterpart (the reference has no persistent launch). */
int xmss_b200_set_wait_bound(unsigned long long ns);

/* Pipelined form of xmss_b200_sign_open_batch: enqueues the copy of the
 * signed messages from the caller's memory, the verify, and the copy of the
 * statuses into `status` on `stream` (cudaStream_t as void*) and returns.
 * sm and status should be pinned host memory (pageable memory makes the
 * copies synchronous); they must stay untouched until the stream has
 * passed this call (cudaStreamSynchronize or an event).  sm_off, smlen, pk
 * and pk_index are read before the call returns.  Each stream has its own
 * device buffers, so calls on two or more streams overlap one batch's
 * copies with another's kernels.  A call waits (on the host) only until the
 * previous call on the same stream has copied its inputs to the device;
 * calls on one stream then run one after another on the GPU, so a caller can
 * queue several batches ahead.  No reference counterpart beyond the
 * xmss[mt]_sign_open calls it batches (xmss.c:45-60, 95-109). */
int xmss_b200_sign_open_batch_async(int mt, uint32_t count, const uint8_t *sm, const uint64_t *sm_off,
                                    const uint64_t *smlen, const uint8_t *pk, uint32_t npk,
                                    const uint32_t *pk_index, int *status, void *stream);

/* CUDA-graph form of xmss_b200_sign_open_device for batches of a fixed
 * shape at fixed device addresses (a verifier that refills the same
 * buffers): create runs the verify once (sizing the graph's own scratch)
 * and captures its whole launch sequence; launch replays it with one call,
 * reading whatever the buffers hold then.  Launches of one graph must not
 * overlap each other; destroy waits for the device. */
typedef struct xmss_b200_verify_graph xmss_b200_verify_graph;

int xmss_b200_verify_graph_create(uint32_t oid, int mt, uint32_t count, const uint8_t *d_sm,
                                  const uint64_t *d_sm_off, const uint64_t *d_smlen, const uint8_t *d_pk,
                                  uint32_t npk, const uint32_t *d_pk_index, int *d_status,
                                  xmss_b200_verify_graph **out);
int xmss_b200_verify_graph_launch(xmss_b200_verify_graph *g, void *stream);
void xmss_b200_verify_graph_destroy(xmss_b200_verify_graph *g);

/* Mixed batches: keygen, sign and verify groups of any parameter sets (OIDs,
 * XMSS and XMSS^MT, every hash family) in ONE CUDA graph.  Each group is
 * `count` items of one kind and one parameter set; its launch sequence (the
 * one of xmss_b200_keypair_device / xmss_b200_sign_batch /
 * xmss_b200_sign_open_device) is captured on a stream of its own, forked
 * from and joined back into the launch stream, so the groups run
 * concurrently and the whole batch is a single cudaGraphLaunch.  Every
 * result is byte-identical to the per-kind calls (and to the reference's
 * xmssmt_core_seed_keypair / xmss[mt]_sign / xmss[mt]_sign_open per item).
 *
 * Fields per kind (all d_ pointers on the device, read or written at each
 * launch; host pointers only at create):
 *   XMSS_B200_KEYGEN  d_seeds (count x 3n) -> d_pk (count x 2n, root ||
 *                     PUB_SEED) and d_sk (count x sk_bytes), no OID prefix.
 *   XMSS_B200_SIGN    sk: HOST, count x (4 + sk_bytes), OID-prefixed keys as
 *                     xmss[mt]_keypair writes them (rows may repeat a key:
 *                     its requests take consecutive indices); create does
 *                     the reference's index bookkeeping (xmss_core.c:
 *                     209-239) on them, so on return they are the keys to
 *                     persist, and sets ret[i] (HOST) to 0 or -2 (exhausted:
 *                     that item is not signed).  d_sm + d_sm_off[i] holds
 *                     message i at offset sig_bytes (d_len[i] bytes); launch
 *                     writes the signature before it.
 *   XMSS_B200_VERIFY  d_sm / d_sm_off / d_len (signed-message lengths) /
 *                     d_pk (npk x 2n) / npk / d_pk_index -> d_status, as in
 *                     xmss_b200_sign_open_device.
 * Each signing index is used once: a batch holding sign groups launches at
 * most once (a second launch returns -2 and runs nothing); create signs
 * nothing that leaves the library (its sizing run writes into scratch).
 * Batches of keygen and verify groups may be relaunched after refilling
 * their buffers; launches of one batch must not overlap.  create: 0 ok, -1
 * bad group, -3 GPU failure; destroy waits for the device. */
enum { XMSS_B200_KEYGEN = 1, XMSS_B200_SIGN = 2, XMSS_B200_VERIFY = 3 };

typedef struct {
    int kind;                    /* XMSS_B200_KEYGEN / _SIGN / _VERIFY */
    uint32_t oid;                /* parameter set */
    int mt;                      /* 1: XMSS^MT OID */
    uint32_t count;              /* items */
    const uint8_t *d_seeds;      /* keygen */
    uint8_t *d_pk;               /* keygen: out; verify: in */
    uint8_t *d_sk;               /* keygen */
    uint8_t *sk;                 /* sign: host keys, advanced by create */
    int *ret;                    /* sign: host per-item codes, set by create */
    uint8_t *d_sm;               /* sign: out; verify: in */
    const uint64_t *d_sm_off;    /* sign, verify */
    const uint64_t *d_len;       /* sign: message lengths; verify: signed-message lengths */
    uint32_t npk;                /* verify */
    const uint32_t *d_pk_index;  /* verify */
    int *d_status;               /* verify */
} xmss_b200_batch_group;

typedef struct xmss_b200_batch xmss_b200_batch;

int xmss_b200_batch_create(const xmss_b200_batch_group *groups, uint32_t ngroups, xmss_b200_batch **out);
/* The same batch as persistent launches fed by a device work queue: the
 * groups of one hash family (keygen, sign and verify alike, any parameter
 * sets, up to 8 per launch) run as ONE persistent kernel launch whose warps
 * take the tasks of all of them from one ticket sequence (subtree chains,
 * L-tree levels and Merkle levels, key output, signature preparation and
 * chains, and the verify tasks of xmss_b200_sign_open_device_persistent),
 * the families' launches concurrent on forked streams, all captured in one
 * CUDA graph.  Same results, rules and return codes as
 * xmss_b200_batch_create. */
int xmss_b200_batch_create_persistent(const xmss_b200_batch_group *groups, uint32_t ngroups,
                                      xmss_b200_batch **out);
int xmss_b200_batch_launch(xmss_b200_batch *b, void *stream);
void xmss_b200_batch_destroy(xmss_b200_batch *b);

/* Launch shapes of one hash family (func, n): CTA sizes (32, 64 or 128
 * threads) of the verify chain kernel, of the keygen / sign chain kernels
 * and of the L-tree / Merkle-level kernels, and the split of large verify
 * batches into a short- and a long-H_msg group on two streams (from
 * split_min signatures on, at short_hmsg_blocks hash blocks).  In a split
 * batch, prep_split = 1 runs the L-tree precomputation (h_pre) of both
 * groups as a launch of its own on a third stream, so that each group's
 * chains wait only for its H_msg; 0 runs it inside each group's prep
 * launch.  Results do not depend on any of them.  Defaults: 128, 128,
 * 128, 1024, 16, 1.  Set them while no call of that family runs (they are
 * read at each launch). */
typedef struct {
    uint32_t verify_chain_block;
    uint32_t keygen_chain_block;
    uint32_t level_block;
    uint32_t split_min;
    uint32_t short_hmsg_blocks;
    uint32_t prep_split;
} xmss_b200_tuning;

int xmss_b200_tuning_get(unsigned int func, unsigned int n, xmss_b200_tuning *out);
int xmss_b200_tuning_set(unsigned int func, unsigned int n, const xmss_b200_tuning *t);

/* How the subtrees of one parameter set (OID) are built, for keygen, sign
 * and the server's subtree cache (treehash, xmss_core.c:19-86):
 *   subtree_height 0    one thread per WOTS chain (chains_per_warp 32),
 *                       then one launch per L-tree level and per Merkle
 *                       level;
 *   subtree_height 5-7  in-CTA subtrees: one thread per leaf
 *                       (chains_per_warp 32 x len), whose chains are
 *                       reduced into the L-tree as they finish, a CTA of
 *                       2^k threads reducing its 2^k leaves to one node in
 *                       shared memory; the levels above run across CTAs;
 *   min_leaves          builds with fewer leaves in one call use the first
 *                       form (the in-CTA form runs a leaf's chains one
 *                       after the other, so small builds lack parallelism).
 * chains_per_warp is reported by _get and ignored by _set.  Results do not
 * depend on the shape.  Default: 0 (set by the autotuner or
 * xmss_b200/tuning.json).  0 ok, -1 unknown OID or height out of range. */
typedef struct {
    uint32_t subtree_height;
    uint32_t chains_per_warp;
    uint64_t min_leaves;
} xmss_b200_tree_tuning;

int xmss_b200_tree_tuning_get(uint32_t oid, int mt, xmss_b200_tree_tuning *out);
int xmss_b200_tree_tuning_set(uint32_t oid, int mt, const xmss_b200_tree_tuning *t);

/* Tree autotuner for one parameter set: times keygen slices of 2^12, 2^15
 * and 2^18 leaves (subtrees of the set's height, seeded keys) in the
 * one-thread-per-chain form and as in-CTA subtrees of height 5, 6 and 7,
 * checks that every form gives the same node arrays, and sets the set's
 * shape: the in-CTA height that is fastest at 2^18 leaves if it beats the
 * other form by 2 %, and min_leaves = the smallest slice at which it still
 * does.  best gets the shape; report (if not NULL) a JSON text of every
 * trial.  No reference counterpart (a launch-shape choice).  0 ok, -1
 * unknown OID, -3 failure. */
int xmss_b200_autotune_tree(uint32_t oid, int mt, xmss_b200_tree_tuning *best, char *report, size_t report_cap);

/* Autotuner: times candidate shapes on a synthetic batch of this parameter
 * set (16 seeded keys, `count` signatures of messages log-uniform in
 * 32 B..4 KB, made by this library, and a 4,096-leaf keygen slice), one knob
 * at a time, checks that every candidate accepts every signature, and
 * leaves the fastest shape set for the family.  best gets it; report (if
 * not NULL) a JSON text of every trial.  0 ok, -1 bad argument, -3 failure. */
int xmss_b200_autotune(uint32_t oid, int mt, uint32_t count, xmss_b200_tuning *best, char *report,
                       size_t report_cap);

/* Batched xmss[mt]_sign (xmss.c:28-43, 78-93).  Request i signs
 * msgs[m_off[i] .. + mlen[i]) with sk i (sk: count x (4 + sk_bytes),
 * OID-prefixed, one OID), advancing that sk in place exactly as
 * xmssmt_core_sign does (xmss_core.c:209-239, exhaustion included), and
 * writes sig || message to sm + sm_off[i] (capacity sig_bytes + mlen[i]),
 * its length to smlen[i] and its return code (0, -2) to ret[i].  Requests
 * may carry copies of one key at different indices; each subtree they share
 * is built once. */
int xmss_b200_sign_batch(int mt, uint32_t count, uint8_t *sk, const uint8_t *msgs,
                         const uint64_t *m_off, const uint64_t *mlen, uint8_t *sm,
                         const uint64_t *sm_off, uint64_t *smlen, int *ret);

/* Batched core_hash (hash.c:29-65) of hash family (func, n): out[i] (n
 * bytes) = core_hash(in[off[i] .. off[i] + len[i])).  Exposes the SHA-256,
 * SHA-512 and Keccak cores for testing. */
int xmss_b200_core_hash_batch(unsigned int func, unsigned int n, uint32_t count,
                              const uint8_t *in, const uint64_t *off, const uint64_t *len,
                              uint8_t *out);

/* Work counters of the most recent verify call (host or device form),
 * counted on the GPU: hash blocks absorbed by H_msg, F calls of the WOTS
 * chains and H calls of L-trees and authentication paths.  Waits for that
 * call to finish.  Multiplying by the family's cost per call (SHA-2 with
 * per-key midstates: F = 4, H = 6 compressions) gives the compressions the
 * reference algorithm performs. */
typedef struct {
    unsigned long long hmsg_blocks;
    unsigned long long f_calls;
    unsigned long long h_calls;
} xmss_b200_work;

int xmss_b200_last_verify_work(xmss_b200_work *out);

/* Kernel timing for benchmarks: while enabled, every pipeline records CUDA
 * events around its launches.  xmss_b200_phase_ms waits for the last call and
 * returns its summed kernel time per phase in ms: [0] H_msg / preparation,
 * [1] WOTS chains, [2] L-tree levels, [3] compute_root / auth paths,
 * [4] Merkle tree levels (keygen, sign).  Off by default. */
int xmss_b200_profile(int enable);
int xmss_b200_phase_ms(double ms[5]);

/* Same as xmss_b200_sign_open_device, but allocates nothing: no
 * reference counterpart; it exists for callers that cannot allocate device
 * memory when they verify (a request path that cannot absorb cudaMalloc's
 * device synchronisation and latency, or a process held to a fixed device
 * memory budget).  Its intermediate buffers live in one fixed 8 MiB array in
 * device memory that every GPU using the library holds until exit; a batch
 * that does not fit returns -1 (XMSS-SHA2_10_256 fits up to about 760
 * signatures per call).
 * All calls share that array: calls whose GPU work overlaps race, so callers
 * serialise them.  The first call on each device looks the array up with
 * that device current and should come before any stream capture. */
int xmss_b200_sign_open_device_noalloc(uint32_t oid, int mt, uint32_t count, const uint8_t *d_sm,
                                       const uint64_t *d_sm_off, const uint64_t *d_smlen,
                                       const uint8_t *d_pk, uint32_t npk, const uint32_t *d_pk_index,
                                       int *d_status, void *stream);

/* ---------------------------------------------------------------------------
 * Serving: a request loop over device-resident keys.  No reference
 * counterpart as a whole; each request does what one xmss[mt]_sign
 * (xmss.c:28-43, 78-93) or xmss[mt]_sign_open (xmss.c:45-60, 95-109) call
 * does, with byte-identical results.
 *
 * Requests are submitted from any thread and complete asynchronously.  A
 * dispatcher thread batches whatever is queued whenever one of `slots` batch
 * slots is free (continuous batching: batches admitted while others run
 * overlap on the device), groups each batch by operation and parameter set,
 * and admits it only while free device memory stays above
 * mem_reserve_bytes, shrinking the batch when it does not fit (free memory
 * is read by a monitor thread every 20 ms, and asked again by the
 * dispatcher only when that reading says a batch does not fit).
 *
 * Keys are resident on the device: seeds, PRF key, root, PUB_SEED, a u64
 * one-time index counter advanced with atomicAdd (reservations run in
 * submission order, so request i of a key gets the i-th index), and a cache
 * of the subtrees signing needs (each built once, then authentication paths
 * are copied out of it instead of recomputed as xmss_core.c:253-270 does).
 * Indices run from the sk's index to 2^h - 2; the request that would take
 * 2^h - 1 (signed with a wiped key by the reference, xmss_core.c:212-231)
 * and all after it complete with -2.
 *
 * Completion codes: 0 ok (sign) / valid (verify); -1 invalid signature or
 * bad request; -2 key exhausted; -3 resource or GPU failure.
 * --------------------------------------------------------------------------- */
typedef struct xmss_b200_server xmss_b200_server;

typedef struct {
    uint32_t max_batch;          /* requests per batch (default 4096) */
    uint32_t slots;              /* batches in flight (default 8) */
    uint32_t window_us;          /* a free slot waits up to this long for a batch to fill (default 0) */
    uint32_t reserved0;
    uint64_t tree_pool_bytes;    /* device memory of the subtree cache (default 1 GiB) */
    uint64_t mem_reserve_bytes;  /* device memory admission leaves free (default 1 GiB) */
} xmss_b200_server_config;

typedef struct {
    uint64_t tag;       /* as submitted */
    int32_t ret;        /* completion code */
    uint32_t kind;      /* 0 sign, 1 verify, 2 warm */
    uint64_t index;     /* sign: the one-time index used */
    double latency_us;  /* submission to completion */
} xmss_b200_completion;

typedef struct {
    uint64_t submitted, completed;
    uint64_t batches;          /* slot launches */
    uint64_t sign_groups;      /* per-parameter-set sign launches */
    uint64_t verify_groups;    /* per-parameter-set verify launches */
    uint64_t largest_batch;
    uint64_t deferred_for_memory;
    uint64_t trees_built, tree_hits, trees_evicted;
    double launch_us;  /* dispatcher time planning, staging and launching */
    double finish_us;  /* dispatcher time copying results out */
    double batch_us;   /* summed launch-to-completion time of the batches */
} xmss_b200_server_stats;

/* cfg NULL or zero fields: defaults.  0 ok, -3 failure. */
int xmss_b200_server_create(const xmss_b200_server_config *cfg, xmss_b200_server **out);

/* Completes every submitted request (results are written to the callers'
 * buffers, completions not yet polled are dropped), then frees the server. */
void xmss_b200_server_destroy(xmss_b200_server *srv);

/* Makes a secret key resident: sk is OID-prefixed as xmss[mt]_keypair writes
 * it (xmss.c:18-25).  The server owns the key's state from here on; read it
 * back with xmss_b200_server_export_sk.  0 ok, -1 unknown OID, -3 failure. */
int xmss_b200_server_add_key(xmss_b200_server *srv, int mt, const uint8_t *sk, uint32_t *key_id);

/* Writes the key's current sk (OID-prefixed, index = the next index the
 * server would issue) to sk (4 + sk_bytes bytes).  Indices of requests still
 * queued are not counted: export after they complete. */
int xmss_b200_server_export_sk(xmss_b200_server *srv, uint32_t key_id, uint8_t *sk);

/* Signs m (mlen bytes) with resident key key_id: writes sig || m to sm
 * (capacity sig_bytes + mlen) and its length to *smlen.  m, sm and smlen
 * must stay valid until the request completes. */
int xmss_b200_server_submit_sign(xmss_b200_server *srv, uint32_t key_id, const uint8_t *m, uint64_t mlen,
                                 uint8_t *sm, uint64_t *smlen, uint64_t tag);

/* Verifies sm (smlen bytes) under pk (OID-prefixed, copied at submission);
 * sm must stay valid until the request completes. */
int xmss_b200_server_submit_verify(xmss_b200_server *srv, int mt, const uint8_t *sm, uint64_t smlen,
                                   const uint8_t *pk, uint64_t tag);

/* Builds (or keeps) the subtrees key_id's next signature needs, without
 * taking an index: the cache rebuild after a key is added or restored.
 * Completes as kind 2. */
int xmss_b200_server_submit_warm(xmss_b200_server *srv, uint32_t key_id, uint64_t tag);

/* Takes up to max completions, waiting up to wait_us for the first.
 * Returns how many were written. */
int xmss_b200_server_poll(xmss_b200_server *srv, xmss_b200_completion *out, uint32_t max, uint32_t wait_us);

/* 0 ok, -3 when the dispatcher has failed (text in xmss_b200_last_error()). */
int xmss_b200_server_stats_get(xmss_b200_server *srv, xmss_b200_server_stats *out);

/* Per-batch trace: the server keeps the last 4096 batches.  Times in us;
 * gpu_us spans the batch's first device operation to its last (CUDA events),
 * lane_us is the slowest plan, identified by its operation (0 sign, 1 verify)
 * and OID. */
typedef struct {
    uint64_t seq;
    uint32_t requests, plans;
    uint32_t slow_kind, slow_oid;
    double queue_us;   /* oldest request: submission to launch */
    double launch_us;  /* host planning, staging and launching */
    double gpu_us;
    double lane_us;
    double done_us;    /* launch to completion seen by the dispatcher */
    uint64_t h2d_bytes, d2h_bytes;
    double start_skew_us;  /* latest lane start after the inputs landed */
    double join_us;        /* batch end after the last lane ended */
} xmss_b200_batch_trace;

/* Copies up to max of the most recent batch records, oldest first; returns
 * how many. */
int xmss_b200_server_trace(xmss_b200_server *srv, xmss_b200_batch_trace *out, uint32_t max);

/* Load generator: submits items (sorted by t_us) at their times from a
 * submitting thread while this thread polls, until all complete.  Latency is
 * measured from each item's scheduled time, so a submitter that falls behind
 * shows in the numbers.  ret[i], latency_us[i] and index[i] (sign: the index
 * used) get item i's result; *elapsed_s the time from start to the last
 * completion.  0 ok, -1 bad argument. */
typedef struct {
    double t_us;            /* scheduled submission time, from the start */
    uint32_t kind;          /* 0 sign, 1 verify */
    uint32_t key_id;        /* sign: resident key */
    int32_t mt;             /* verify: 1 for XMSS^MT */
    uint32_t reserved0;
    const uint8_t *in;      /* sign: message; verify: signed message */
    uint64_t inlen;
    uint8_t *sm;            /* sign: output, capacity sig_bytes + inlen */
    uint64_t *smlen;        /* sign: output length */
    const uint8_t *pk;      /* verify: OID-prefixed public key */
} xmss_b200_trace_item;

int xmss_b200_server_replay(xmss_b200_server *srv, const xmss_b200_trace_item *items, uint32_t count, int *ret,
                            double *latency_us, uint64_t *index, double *elapsed_s);

/* ---------------------------------------------------------------------------
 * BDS ("fast") secret keys, as the reference's xmss_core_fast.c builds keep
 * them (xmss_core_fast.c:14-148, 635-653): the plain sk followed by the
 * authentication-path traversal state of 2d - 1 trees and, for XMSS^MT, the
 * WOTS signatures of the lower roots.  Keys are OID-prefixed here.
 * --------------------------------------------------------------------------- */

/* Size of a BDS sk of this parameter set without the OID (0: unknown). */
unsigned long long xmss_b200_bds_sk_bytes(uint32_t oid, int mt);

/* The plain sk (what xmss[mt]_keypair writes) inside a BDS sk: its index,
 * seeds, root and PUB_SEED.  0 ok, -1 unknown OID. */
int xmss_b200_sk_from_bds(int mt, const uint8_t *bds_sk, uint8_t *sk);

/* The BDS sk the reference's fast build holds at this plain sk's index:
 * the traversal of keygen and of every signature below the index is
 * replayed on the host (its hashes looked up in subtrees built on the GPU),
 * so the time grows with the index; indices above 2^24 return -1.  Fields
 * the reference never writes (it leaves the caller's buffer in them) are
 * zero; a wiped key stays wiped.  At the last index (2^h - 1) the cached
 * WOTS signatures are those of this library's sign at that index, which the
 * reference never reads (it wipes the key before signing). */
int xmss_b200_sk_to_bds(int mt, const uint8_t *sk, uint8_t *bds_sk);

/* Compression-rate probe (the roofline denominator): `blocks` x 128 threads
 * each run `iters` dependent SHA-256 compressions (kind 0), Keccak-f[1600]
 * permutations (kind 1) or SHA-512 compressions (kind 2) in registers, on
 * `stream`; kinds 10 + m (m = 0..9) run SHA-256 in pipe mix m, and 20, 21
 * and 23 mixes 0, 1 and 3 with one warp per block (latency of a lone warp).
 * d_sink: blocks x 128
 * u32 of device memory (written almost never). */
int xmss_b200_rate_probe(int kind, uint32_t blocks, uint32_t iters, uint32_t *d_sink, void *stream);

#ifdef __cplusplus
}
#endif

#endif
