/*
 * Command-line tools over libxmss_b200, drop-in for the reference's ui/
 * programs (cuxmss/ui/keypair.c, sign.c, open.c; built there as
 * ui/xmss[mt]_keypair, _sign, _open).  One source, six binaries: the
 * Makefile compiles it with CLI_KEYPAIR / CLI_SIGN / CLI_OPEN and, for the
 * XMSS^MT tools, XMSSMT.
 *
 * File formats (those of the reference tools):
 *   keypair file  OID || pk  followed by  OID || sk   (pk_bytes, sk_bytes of
 *                 the OID's parameter set; xmss.c:18-25)
 *   signature     sm = sig || m as xmss[mt]_sign writes it
 *
 *   xmss_keypair <params>          writes a new keypair file to stdout
 *   xmss_sign <keypair> <message>  writes sm to stdout and the advanced sk
 *                                  back into the keypair file
 *   xmss_open <keypair> <sm>       "Verification succeeded." (exit 0) or
 *                                  "Verification failed!" (non-zero)
 *
 * Messages, exit codes and file updates follow the reference tools; the one
 * difference is that a sign that fails (exhausted key: -2) reports it and
 * writes no signature, where the reference writes an unset buffer (the
 * wiped key is stored by both).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include "../../include/params.h"
#include "../../include/xmss.h"

#ifdef XMSSMT
#define TOOL_STR_TO_OID xmssmt_str_to_oid
#define TOOL_PARSE_OID xmssmt_parse_oid
#define TOOL_KEYPAIR xmssmt_keypair
#define TOOL_SIGN xmssmt_sign
#define TOOL_OPEN xmssmt_sign_open
#else
#define TOOL_STR_TO_OID xmss_str_to_oid
#define TOOL_PARSE_OID xmss_parse_oid
#define TOOL_KEYPAIR xmss_keypair
#define TOOL_SIGN xmss_sign
#define TOOL_OPEN xmss_sign_open
#endif

static inline uint32_t read_oid(const unsigned char *b)
{
    return ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
}

/* Whole file into a malloc'd buffer; NULL on failure. */
static inline unsigned char *slurp(FILE *f, unsigned long long *len)
{
    if (fseek(f, 0, SEEK_END) != 0) return NULL;
    long n = ftell(f);
    if (n < 0 || fseek(f, 0, SEEK_SET) != 0) return NULL;
    unsigned char *b = malloc(n ? (size_t)n : 1);
    if (!b) return NULL;
    if (n && fread(b, 1, (size_t)n, f) != (size_t)n) {
        free(b);
        return NULL;
    }
    *len = (unsigned long long)n;
    return b;
}

#if defined(CLI_KEYPAIR)
int main(int argc, char **argv)
{
    if (argc != 2) {
        fprintf(stderr, "Expected parameter string (e.g. 'XMSS-SHA2_10_256') as only parameter.\n"
                        "The keypair is written to stdout.\n");
        return -1;
    }
    uint32_t oid = 0;
    xmss_params p;
    TOOL_STR_TO_OID(&oid, argv[1]);
    int r = TOOL_PARSE_OID(&p, oid);
    if (r != 0) {
        fprintf(stderr, "Error parsing oid.\n");
        return r;
    }
    unsigned char *pk = malloc(XMSS_OID_LEN + p.pk_bytes), *sk = malloc(XMSS_OID_LEN + p.sk_bytes);
    if (!pk || !sk) return -1;
    r = TOOL_KEYPAIR(pk, sk, oid);
    if (r != 0) {
        fprintf(stderr, "Key generation failed (%d).\n", r);
        return r;
    }
    fwrite(pk, 1, XMSS_OID_LEN + p.pk_bytes, stdout);
    fwrite(sk, 1, XMSS_OID_LEN + p.sk_bytes, stdout);
    fclose(stdout);
    free(pk);
    free(sk);
    return 0;
}

#elif defined(CLI_SIGN)
int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "Expected keypair and message filenames as two parameters.\n"
                        "The keypair is updated with the changed state, "
                        "and the message + signature is output via stdout.\n");
        return -1;
    }
    FILE *kf = fopen(argv[1], "r+b");
    if (!kf) {
        fprintf(stderr, "Could not open keypair file.\n");
        return -1;
    }
    FILE *mf = fopen(argv[2], "rb");
    if (!mf) {
        fprintf(stderr, "Could not open message file.\n");
        fclose(kf);
        return -1;
    }
    unsigned char oidb[XMSS_OID_LEN];
    xmss_params p;
    int r = -1;
    /* the public key's OID gives the offset of the secret key */
    if (fread(oidb, 1, XMSS_OID_LEN, kf) != XMSS_OID_LEN || (r = TOOL_PARSE_OID(&p, read_oid(oidb))) != 0) {
        fprintf(stderr, "Error parsing public key oid.\n");
        fclose(kf);
        fclose(mf);
        return r ? r : -1;
    }
    const long sk_at = XMSS_OID_LEN + (long)p.pk_bytes;
    if (fseek(kf, sk_at, SEEK_SET) != 0 || fread(oidb, 1, XMSS_OID_LEN, kf) != XMSS_OID_LEN ||
        (r = TOOL_PARSE_OID(&p, read_oid(oidb))) != 0) {
        fprintf(stderr, "Error parsing secret key oid.\n");
        fclose(kf);
        fclose(mf);
        return r ? r : -1;
    }
    unsigned long long mlen = 0, smlen = 0;
    unsigned char *m = slurp(mf, &mlen);
    unsigned char *sk = malloc(XMSS_OID_LEN + p.sk_bytes);
    unsigned char *sm = m ? malloc(p.sig_bytes + mlen) : NULL;
    if (!m || !sk || !sm || fseek(kf, sk_at, SEEK_SET) != 0 ||
        fread(sk, 1, XMSS_OID_LEN + p.sk_bytes, kf) != XMSS_OID_LEN + p.sk_bytes) {
        fprintf(stderr, "Could not read the keypair or message file.\n");
        fclose(kf);
        fclose(mf);
        return -1;
    }
    r = TOOL_SIGN(sk, sm, &smlen, m, mlen);
    /* the key goes back first, also when signing failed (an exhausted key
       comes back wiped, as the reference stores it): a signature never
       leaves before the state that forbids reusing its index is stored */
    if (fseek(kf, sk_at + XMSS_OID_LEN, SEEK_SET) != 0 ||
        fwrite(sk + XMSS_OID_LEN, 1, p.sk_bytes, kf) != p.sk_bytes || fflush(kf) != 0) {
        fprintf(stderr, "Could not update the keypair file.\n");
        r = -1;
    } else if (r == 0) {
        fwrite(sm, 1, smlen, stdout);
    } else {
        fprintf(stderr, "Signing failed (%d).\n", r);
    }
    fclose(kf);
    fclose(mf);
    free(m);
    free(sk);
    free(sm);
    return r;
}

#elif defined(CLI_OPEN)
int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "Expected keypair and signature + message filenames as two parameters.\n"
                        "Keypair file needs only to contain the public key.\n"
                        "The return code 0 indicates verification success.\n");
        return -1;
    }
    FILE *kf = fopen(argv[1], "rb");
    if (!kf) {
        fprintf(stderr, "Could not open keypair file.\n");
        return -1;
    }
    FILE *sf = fopen(argv[2], "rb");
    if (!sf) {
        fprintf(stderr, "Could not open signature + message file.\n");
        fclose(kf);
        return -1;
    }
    unsigned char oidb[XMSS_OID_LEN];
    xmss_params p;
    int r = -1;
    if (fread(oidb, 1, XMSS_OID_LEN, kf) != XMSS_OID_LEN || (r = TOOL_PARSE_OID(&p, read_oid(oidb))) != 0) {
        fprintf(stderr, "Error parsing oid.\n");
        fclose(kf);
        fclose(sf);
        return r ? r : -1;
    }
    unsigned long long smlen = 0, mlen = 0;
    unsigned char *sm = slurp(sf, &smlen);
    unsigned char *pk = malloc(XMSS_OID_LEN + p.pk_bytes);
    unsigned char *m = sm ? malloc(smlen ? smlen : 1) : NULL;
    if (!sm || !pk || !m || fseek(kf, 0, SEEK_SET) != 0 ||
        fread(pk, 1, XMSS_OID_LEN + p.pk_bytes, kf) != XMSS_OID_LEN + p.pk_bytes) {
        fprintf(stderr, "Could not read the keypair or signature file.\n");
        fclose(kf);
        fclose(sf);
        return -1;
    }
    r = TOOL_OPEN(m, &mlen, sm, smlen, pk);
    printf(r ? "Verification failed!\n" : "Verification succeeded.\n");
    fclose(kf);
    fclose(sf);
    free(sm);
    free(pk);
    free(m);
    return r;
}

#else
#error "compile with CLI_KEYPAIR, CLI_SIGN or CLI_OPEN"
#endif
