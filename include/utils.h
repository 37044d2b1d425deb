/*
 * Big-endian integer <-> byte helpers, drop-in for the reference's utils.h
 * (cuxmss/utils.h:1-25, cuxmss/utils.c:6-30).  Exported by libxmss_b200.so
 * because the reference's own programs call them on sk bytes (for example
 * cuxmss/test/xmss_max_signatures.c reads the index with bytes_to_ull).
 */
#ifndef XMSS_UTILS_H
#define XMSS_UTILS_H

#ifdef __cplusplus
extern "C" {
#endif

/* out[0 .. outlen) = in, most significant byte first (utils.c:6-16). */
void ull_to_bytes(unsigned char *out, unsigned int outlen, unsigned long long in);

/* The integer whose big-endian bytes are in[0 .. inlen) (utils.c:21-30). */
unsigned long long bytes_to_ull(const unsigned char *in, unsigned int inlen);

#ifdef __cplusplus
}
#endif

#endif
