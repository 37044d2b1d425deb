/*
 * XMSS / XMSS^MT public API, drop-in for the reference's xmss.h
 * (cuxmss/xmss.h:15-64): same six functions, same buffer formats, same
 * return codes.  Every call computes on the GPU (sm_100a) through
 * libxmss_b200.so; there is no CPU fallback.
 *
 * pk = OID (4 bytes, big-endian) || root || PUB_SEED
 * sk = OID || idx (index_bytes, big-endian) || SK_SEED || SK_PRF || root || PUB_SEED
 * sm = idx || R || d x (WOTS signature || auth path) || message
 *
 * Returns 0 on success, -1 for an unknown OID or a failed verification (m
 * zeroed, *mlen = 0), -2 when the key is exhausted, and -3 when the GPU
 * could not run the call (no device, CUDA error); the reference has no -3.
 */
#ifndef XMSS_H
#define XMSS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Replaces xmss_keypair (xmss.c:10-26); seed from randombytes(). */
int xmss_keypair(unsigned char *pk, unsigned char *sk, const uint32_t oid);

/* Replaces xmss_sign (xmss.c:28-43); sk is updated in place. */
int xmss_sign(unsigned char *sk,
              unsigned char *sm, unsigned long long *smlen,
              const unsigned char *m, unsigned long long mlen);

/* Replaces xmss_sign_open (xmss.c:45-60); m needs room for smlen bytes. */
int xmss_sign_open(unsigned char *m, unsigned long long *mlen,
                   const unsigned char *sm, unsigned long long smlen,
                   const unsigned char *pk);

/* Replaces xmssmt_keypair (xmss.c:62-76). */
int xmssmt_keypair(unsigned char *pk, unsigned char *sk, const uint32_t oid);

/* Replaces xmssmt_sign (xmss.c:78-93). */
int xmssmt_sign(unsigned char *sk,
                unsigned char *sm, unsigned long long *smlen,
                const unsigned char *m, unsigned long long mlen);

/* Replaces xmssmt_sign_open (xmss.c:95-109). */
int xmssmt_sign_open(unsigned char *m, unsigned long long *mlen,
                     const unsigned char *sm, unsigned long long smlen,
                     const unsigned char *pk);

#ifdef __cplusplus
}
#endif

#endif
