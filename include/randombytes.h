/*
 * Randomness source of xmss_keypair / xmssmt_keypair, drop-in for the
 * reference's randombytes.h (cuxmss/randombytes.h:1-17).  The library's
 * default reads /dev/urandom like cuxmss/randombytes.c:10-39;
 * xmss_b200_set_randombytes (xmss_b200.h) installs another source.
 */
#ifndef XMSS_RANDOMBYTES_H
#define XMSS_RANDOMBYTES_H

#ifdef __cplusplus
extern "C" {
#endif

void randombytes(unsigned char *x, unsigned long long xlen);

#ifdef __cplusplus
}
#endif

#endif
