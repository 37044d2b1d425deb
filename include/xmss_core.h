/*
 * Core XMSS / XMSS^MT calls without OID prefix, drop-in for the reference's
 * xmss_core.h (cuxmss/xmss_core.h:1-85).  GPU-backed; return codes as in
 * xmss.h (-3 = GPU failure, not in the reference).
 */
#ifndef XMSS_CORE_H
#define XMSS_CORE_H

#include "params.h"

#ifdef __cplusplus
extern "C" {
#endif

/* sk size of the plain (non-BDS) format: index_bytes + 4n (xmss_core.c:93-96). */
unsigned long long xmss_xmssmt_core_sk_bytes(const xmss_params *params);

/* xmss_core.c:103-110 */
int xmss_core_keypair(const xmss_params *params, unsigned char *pk, unsigned char *sk);

/* xmss_core.c:116-126 */
int xmss_core_sign(const xmss_params *params, unsigned char *sk,
                   unsigned char *sm, unsigned long long *smlen,
                   const unsigned char *m, unsigned long long mlen);

/* xmss_commons.c:120-130 */
int xmss_core_sign_open(const xmss_params *params,
                        unsigned char *m, unsigned long long *mlen,
                        const unsigned char *sm, unsigned long long smlen,
                        const unsigned char *pk);

/* xmss_core.c:168-177; seed from randombytes(). */
int xmssmt_core_keypair(const xmss_params *params, unsigned char *pk, unsigned char *sk);

/* xmss_core.c:134-161; seed = SK_SEED || SK_PRF || PUB_SEED (3n bytes). */
int xmssmt_core_seed_keypair(const xmss_params *params, unsigned char *pk,
                             unsigned char *sk, unsigned char *seed);

/* xmss_core.c:183-273 */
int xmssmt_core_sign(const xmss_params *params, unsigned char *sk,
                     unsigned char *sm, unsigned long long *smlen,
                     const unsigned char *m, unsigned long long mlen);

/* xmss_commons.c:136-215 */
int xmssmt_core_sign_open(const xmss_params *params,
                          unsigned char *m, unsigned long long *mlen,
                          const unsigned char *sm, unsigned long long smlen,
                          const unsigned char *pk);

#ifdef __cplusplus
}
#endif

#endif
