/*
 * Parameter sets of XMSS / XMSS^MT, selected at run time by OID.
 *
 * Drop-in for the reference's params.h (cuxmss/params.h:1-80): same struct
 * layout, same function names, argument meaning and return codes.  The
 * tables cover all 21 XMSS and 56 XMSS^MT OIDs of params.c:7-252.
 */
#ifndef XMSS_PARAMS_H
#define XMSS_PARAMS_H

#include <stdint.h>

/* Internal identifiers of the hash functions (params.h:6-9). */
#define XMSS_SHA2 0
#define XMSS_SHAKE128 1
#define XMSS_SHAKE256 2

/* OID prefix length of pk/sk buffers (params.h:11-12). */
#define XMSS_OID_LEN 4

/* Populated by xmss[mt]_parse_oid (params.h:15-33). */
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
} xmss_params;

#ifdef __cplusplus
extern "C" {
#endif

/* "XMSS-SHA2_10_256" -> 0x00000001; -1 when unknown (params.c:7-76). */
int xmss_str_to_oid(uint32_t *oid, const char *s);

/* "XMSSMT-SHA2_20/2_256" -> 0x00000001; -1 when unknown (params.c:78-252). */
int xmssmt_str_to_oid(uint32_t *oid, const char *s);

/* Fills params for an XMSS OID; -1 when unknown (params.c:254-375). */
int xmss_parse_oid(xmss_params *params, const uint32_t oid);

/* Fills params for an XMSS^MT OID; -1 when unknown (params.c:377-698). */
int xmssmt_parse_oid(xmss_params *params, const uint32_t oid);

/* Derives the remaining fields from full_height, n, d, func, wots_w
 * (params.c:710-753); -1 for an unsupported wots_w. */
int xmss_xmssmt_initialize_params(xmss_params *params);

#ifdef __cplusplus
}
#endif

#endif
