/*
 * CPU oracle for the XMSS / XMSS^MT hot path (TEST INFRASTRUCTURE ONLY).
 *
 * This is a plain-C restatement of the reference C path of CU-XMSS
 * (cuxmss/xmss_core.c, xmss_commons.c, wots.c, hash.c, hash_address.c,
 * params.c, utils.c) together with SHA-256 / SHA-512 (FIPS 180-4) and
 * Keccak-f[1600] / SHAKE (FIPS 202) written from the standards.
 *
 * It exists to check the CUDA library: only the test suite, the smoke check
 * and the CPU-baseline leg of the benchmark load it.  The product library
 * never links or calls it.
 *
 * Every exported function names the reference function it restates.
 */
#ifndef XMSS_ORACLE_H
#define XMSS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define XO_SHA2 0
#define XO_SHAKE128 1
#define XO_SHAKE256 2

/* Same fields, same order as xmss_params (cuxmss/params.h:15-33). */
typedef struct {
    unsigned int func;
    unsigned int n;
    unsigned int padding_len;
    unsigned int wots_w;
    unsigned int wots_log_w;
    unsigned int wots_len1;
    unsigned int wots_len2;
    unsigned int wots_len;
    unsigned int wots_sig_bytes;
    unsigned int full_height;
    unsigned int tree_height;
    unsigned int d;
    unsigned int index_bytes;
    unsigned int sig_bytes;
    unsigned int pk_bytes;
    unsigned long long sk_bytes;
    unsigned int bds_k;
} xo_params;

/* Hash primitives (FIPS 180-4, FIPS 202). */
void xo_sha256(uint8_t out[32], const uint8_t *in, size_t inlen);
void xo_sha512(uint8_t out[64], const uint8_t *in, size_t inlen);
void xo_shake128(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen);
void xo_shake256(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen);

/* Parameter tables: params.c:7-76, 78-252, 254-375, 377-698, 710-753. */
int xo_str_to_oid(uint32_t *oid, const char *s, int mt);
int xo_parse_oid(xo_params *p, uint32_t oid, int mt);
int xo_initialize_params(xo_params *p);

/* Tweakable hashes: hash.c:70-183. addr is 8 x u32. */
int xo_prf(const xo_params *p, uint8_t *out, const uint8_t in[32], const uint8_t *key);
int xo_prf_keygen(const xo_params *p, uint8_t *out, const uint8_t *in, const uint8_t *key);
int xo_hash_message(const xo_params *p, uint8_t *out, const uint8_t *R,
                    const uint8_t *root, unsigned long long idx,
                    const uint8_t *m, unsigned long long mlen);
int xo_thash_f(const xo_params *p, uint8_t *out, const uint8_t *in,
               const uint8_t *pub_seed, uint32_t addr[8]);
int xo_thash_h(const xo_params *p, uint8_t *out, const uint8_t *in,
               const uint8_t *pub_seed, uint32_t addr[8]);

/* WOTS+: wots.c:117-175. */
void xo_wots_pkgen(const xo_params *p, uint8_t *pk, const uint8_t *seed,
                   const uint8_t *pub_seed, uint32_t addr[8]);
void xo_wots_sign(const xo_params *p, uint8_t *sig, const uint8_t *msg,
                  const uint8_t *seed, const uint8_t *pub_seed, uint32_t addr[8]);
void xo_wots_pk_from_sig(const xo_params *p, uint8_t *pk, const uint8_t *sig,
                         const uint8_t *msg, const uint8_t *pub_seed,
                         uint32_t addr[8]);
void xo_chain_lengths(const xo_params *p, int *lengths, const uint8_t *msg);

/* Trees: xmss_commons.c:16-113, xmss_core.c:19-86. */
void xo_gen_leaf_wots(const xo_params *p, uint8_t *leaf, const uint8_t *sk_seed,
                      const uint8_t *pub_seed, uint32_t ltree_addr[8],
                      uint32_t ots_addr[8]);
void xo_treehash(const xo_params *p, uint8_t *root, uint8_t *auth_path,
                 const uint8_t *sk_seed, const uint8_t *pub_seed,
                 uint32_t leaf_idx, const uint32_t subtree_addr[8]);

/* Full node array of one subtree, computed on `nthreads` host threads.
 * nodes is laid out level by level: level 0 (2^h leaves), level 1, ...,
 * level h (the root); (2^(h+1) - 1) * n bytes in total.  Test helper. */
int xo_tree_nodes(const xo_params *p, uint8_t *nodes, const uint8_t *sk_seed,
                  const uint8_t *pub_seed, uint32_t layer, uint64_t tree,
                  int nthreads);
/* Leaves [first, first+count) of one subtree on nthreads host threads. */
int xo_leaves(const xo_params *p, uint8_t *leaves, const uint8_t *sk_seed,
              const uint8_t *pub_seed, uint32_t layer, uint64_t tree,
              uint32_t first, uint32_t count, int nthreads);

/* Key generation / sign / verify without OID prefix:
 * xmss_core.c:134-161, 183-273; xmss_commons.c:136-215. */
int xo_seed_keypair(const xo_params *p, uint8_t *pk, uint8_t *sk, const uint8_t *seed);
int xo_sign(const xo_params *p, uint8_t *sk, uint8_t *sm, unsigned long long *smlen,
            const uint8_t *m, unsigned long long mlen);
int xo_sign_open(const xo_params *p, uint8_t *m, unsigned long long *mlen,
                 const uint8_t *sm, unsigned long long smlen, const uint8_t *pk);

/* Sign at the sk's current index using precomputed node arrays of every
 * layer's subtree (as written by xo_tree_nodes, one array per layer, passed
 * as a packed buffer ordered layer 0 .. d-1).  Same bytes as xo_sign, used
 * to make large signature fixtures quickly.  Returns as xo_sign. */
int xo_sign_with_trees(const xo_params *p, uint8_t *sk, uint8_t *sm,
                       unsigned long long *smlen, const uint8_t *m,
                       unsigned long long mlen, const uint8_t *layer_nodes);

/* OID-prefixed wrappers: xmss.c:10-109 (keypair takes an explicit seed). */
int xo_api_seed_keypair(uint8_t *pk, uint8_t *sk, uint32_t oid, int mt, const uint8_t *seed);
int xo_api_sign(uint8_t *sk, uint8_t *sm, unsigned long long *smlen,
                const uint8_t *m, unsigned long long mlen, int mt);
int xo_api_sign_open(uint8_t *m, unsigned long long *mlen, const uint8_t *sm,
                     unsigned long long smlen, const uint8_t *pk, int mt);

/* Compression-count model of a verify (used by the benchmark to count
 * algorithmic work): chain steps of the WOTS part of one layer. */
int xo_verify_chain_steps(const xo_params *p, const uint8_t *msg);

#ifdef __cplusplus
}
#endif

#endif
