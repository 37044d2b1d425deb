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

/* Compression-rate probe (the roofline denominator): `blocks` x 128 threads
 * each run `iters` dependent SHA-256 compressions (kind 0) or Keccak-f[1600]
 * permutations (kind 1) in registers, on `stream`.  d_sink: blocks x 128
 * u32 of device memory (written almost never). */
int xmss_b200_rate_probe(int kind, uint32_t blocks, uint32_t iters, uint32_t *d_sink, void *stream);

#ifdef __cplusplus
}
#endif

#endif
