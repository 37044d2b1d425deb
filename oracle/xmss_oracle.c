/*
 * CPU oracle for the XMSS / XMSS^MT hot path (TEST INFRASTRUCTURE ONLY).
 *
 * A plain-C restatement of the reference CU-XMSS CPU path.  Citations are
 * `file:line` inside the reference project's cuxmss/ directory.  Hash
 * primitives are written from FIPS 180-4 (SHA-256, SHA-512) and FIPS 202
 * (Keccak-f[1600], SHAKE128, SHAKE256); the Keccak round constants and
 * rotation offsets are derived at start-up from the FIPS 202 definitions.
 *
 * Only the tests, the smoke check and the benchmark's CPU-baseline leg use
 * this file; the CUDA library neither links nor calls it.
 */
#include "xmss_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Byte helpers: utils.c:6-30                                               */
/* ------------------------------------------------------------------------ */

static void to_bytes(uint8_t *out, unsigned int outlen, unsigned long long in)
{
    /* Big-endian, most significant byte first (utils.c:9-18). */
    for (int i = (int)outlen - 1; i >= 0; i--) {
        out[i] = (uint8_t)(in & 0xff);
        in >>= 8;
    }
}

static unsigned long long from_bytes(const uint8_t *in, unsigned int inlen)
{
    unsigned long long r = 0;
    for (unsigned int i = 0; i < inlen; i++) {
        r |= ((unsigned long long)in[i]) << (8 * (inlen - 1 - i));
    }
    return r;
}

/* ------------------------------------------------------------------------ */
/* SHA-256 (FIPS 180-4 section 6.2)                                         */
/* ------------------------------------------------------------------------ */

static const uint32_t SHA256_K[64] = {
    0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1,
    0x923f82a4, 0xab1c5ed5, 0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3,
    0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174, 0xe49b69c1, 0xefbe4786,
    0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
    0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147,
    0x06ca6351, 0x14292967, 0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13,
    0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85, 0xa2bfe8a1, 0xa81a664b,
    0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
    0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a,
    0x5b9cca4f, 0x682e6ff3, 0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208,
    0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};

static const uint32_t SHA256_IV[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372,
                                      0xa54ff53a, 0x510e527f, 0x9b05688c,
                                      0x1f83d9ab, 0x5be0cd19};

#define ROR32(x, n) (((x) >> (n)) | ((x) << (32 - (n))))

static void sha256_block(uint32_t st[8], const uint8_t *blk)
{
    uint32_t w[64];
    for (int t = 0; t < 16; t++) {
        w[t] = ((uint32_t)blk[4 * t] << 24) | ((uint32_t)blk[4 * t + 1] << 16) |
               ((uint32_t)blk[4 * t + 2] << 8) | (uint32_t)blk[4 * t + 3];
    }
    for (int t = 16; t < 64; t++) {
        uint32_t s0 = ROR32(w[t - 15], 7) ^ ROR32(w[t - 15], 18) ^ (w[t - 15] >> 3);
        uint32_t s1 = ROR32(w[t - 2], 17) ^ ROR32(w[t - 2], 19) ^ (w[t - 2] >> 10);
        w[t] = w[t - 16] + s0 + w[t - 7] + s1;
    }
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
    uint32_t e = st[4], f = st[5], g = st[6], h = st[7];
    for (int t = 0; t < 64; t++) {
        uint32_t S1 = ROR32(e, 6) ^ ROR32(e, 11) ^ ROR32(e, 25);
        uint32_t ch = (e & f) ^ (~e & g);
        uint32_t t1 = h + S1 + ch + SHA256_K[t] + w[t];
        uint32_t S0 = ROR32(a, 2) ^ ROR32(a, 13) ^ ROR32(a, 22);
        uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
        uint32_t t2 = S0 + mj;
        h = g; g = f; f = e; e = d + t1;
        d = c; c = b; b = a; a = t1 + t2;
    }
    st[0] += a; st[1] += b; st[2] += c; st[3] += d;
    st[4] += e; st[5] += f; st[6] += g; st[7] += h;
}

void xo_sha256(uint8_t out[32], const uint8_t *in, size_t inlen)
{
    uint32_t st[8];
    uint8_t tail[128];
    size_t full = inlen / 64, rem = inlen % 64;
    memcpy(st, SHA256_IV, sizeof(st));
    for (size_t i = 0; i < full; i++) sha256_block(st, in + 64 * i);
    memset(tail, 0, sizeof(tail));
    memcpy(tail, in + 64 * full, rem);
    tail[rem] = 0x80;
    size_t tl = (rem + 9 <= 64) ? 64 : 128;
    to_bytes(tail + tl - 8, 8, (unsigned long long)inlen * 8);
    sha256_block(st, tail);
    if (tl == 128) sha256_block(st, tail + 64);
    for (int i = 0; i < 8; i++) to_bytes(out + 4 * i, 4, st[i]);
}

/* ------------------------------------------------------------------------ */
/* SHA-512 (FIPS 180-4 section 6.4)                                         */
/* ------------------------------------------------------------------------ */

static const uint64_t SHA512_K[80] = {
    0x428a2f98d728ae22ULL, 0x7137449123ef65cdULL, 0xb5c0fbcfec4d3b2fULL,
    0xe9b5dba58189dbbcULL, 0x3956c25bf348b538ULL, 0x59f111f1b605d019ULL,
    0x923f82a4af194f9bULL, 0xab1c5ed5da6d8118ULL, 0xd807aa98a3030242ULL,
    0x12835b0145706fbeULL, 0x243185be4ee4b28cULL, 0x550c7dc3d5ffb4e2ULL,
    0x72be5d74f27b896fULL, 0x80deb1fe3b1696b1ULL, 0x9bdc06a725c71235ULL,
    0xc19bf174cf692694ULL, 0xe49b69c19ef14ad2ULL, 0xefbe4786384f25e3ULL,
    0x0fc19dc68b8cd5b5ULL, 0x240ca1cc77ac9c65ULL, 0x2de92c6f592b0275ULL,
    0x4a7484aa6ea6e483ULL, 0x5cb0a9dcbd41fbd4ULL, 0x76f988da831153b5ULL,
    0x983e5152ee66dfabULL, 0xa831c66d2db43210ULL, 0xb00327c898fb213fULL,
    0xbf597fc7beef0ee4ULL, 0xc6e00bf33da88fc2ULL, 0xd5a79147930aa725ULL,
    0x06ca6351e003826fULL, 0x142929670a0e6e70ULL, 0x27b70a8546d22ffcULL,
    0x2e1b21385c26c926ULL, 0x4d2c6dfc5ac42aedULL, 0x53380d139d95b3dfULL,
    0x650a73548baf63deULL, 0x766a0abb3c77b2a8ULL, 0x81c2c92e47edaee6ULL,
    0x92722c851482353bULL, 0xa2bfe8a14cf10364ULL, 0xa81a664bbc423001ULL,
    0xc24b8b70d0f89791ULL, 0xc76c51a30654be30ULL, 0xd192e819d6ef5218ULL,
    0xd69906245565a910ULL, 0xf40e35855771202aULL, 0x106aa07032bbd1b8ULL,
    0x19a4c116b8d2d0c8ULL, 0x1e376c085141ab53ULL, 0x2748774cdf8eeb99ULL,
    0x34b0bcb5e19b48a8ULL, 0x391c0cb3c5c95a63ULL, 0x4ed8aa4ae3418acbULL,
    0x5b9cca4f7763e373ULL, 0x682e6ff3d6b2b8a3ULL, 0x748f82ee5defb2fcULL,
    0x78a5636f43172f60ULL, 0x84c87814a1f0ab72ULL, 0x8cc702081a6439ecULL,
    0x90befffa23631e28ULL, 0xa4506cebde82bde9ULL, 0xbef9a3f7b2c67915ULL,
    0xc67178f2e372532bULL, 0xca273eceea26619cULL, 0xd186b8c721c0c207ULL,
    0xeada7dd6cde0eb1eULL, 0xf57d4f7fee6ed178ULL, 0x06f067aa72176fbaULL,
    0x0a637dc5a2c898a6ULL, 0x113f9804bef90daeULL, 0x1b710b35131c471bULL,
    0x28db77f523047d84ULL, 0x32caab7b40c72493ULL, 0x3c9ebe0a15c9bebcULL,
    0x431d67c49c100d4cULL, 0x4cc5d4becb3e42b6ULL, 0x597f299cfc657e2aULL,
    0x5fcb6fab3ad6faecULL, 0x6c44198c4a475817ULL};

static const uint64_t SHA512_IV[8] = {
    0x6a09e667f3bcc908ULL, 0xbb67ae8584caa73bULL, 0x3c6ef372fe94f82bULL,
    0xa54ff53a5f1d36f1ULL, 0x510e527fade682d1ULL, 0x9b05688c2b3e6c1fULL,
    0x1f83d9abfb41bd6bULL, 0x5be0cd19137e2179ULL};

#define ROR64(x, n) (((x) >> (n)) | ((x) << (64 - (n))))

static void sha512_block(uint64_t st[8], const uint8_t *blk)
{
    uint64_t w[80];
    for (int t = 0; t < 16; t++) w[t] = from_bytes(blk + 8 * t, 8);
    for (int t = 16; t < 80; t++) {
        uint64_t s0 = ROR64(w[t - 15], 1) ^ ROR64(w[t - 15], 8) ^ (w[t - 15] >> 7);
        uint64_t s1 = ROR64(w[t - 2], 19) ^ ROR64(w[t - 2], 61) ^ (w[t - 2] >> 6);
        w[t] = w[t - 16] + s0 + w[t - 7] + s1;
    }
    uint64_t a = st[0], b = st[1], c = st[2], d = st[3];
    uint64_t e = st[4], f = st[5], g = st[6], h = st[7];
    for (int t = 0; t < 80; t++) {
        uint64_t S1 = ROR64(e, 14) ^ ROR64(e, 18) ^ ROR64(e, 41);
        uint64_t ch = (e & f) ^ (~e & g);
        uint64_t t1 = h + S1 + ch + SHA512_K[t] + w[t];
        uint64_t S0 = ROR64(a, 28) ^ ROR64(a, 34) ^ ROR64(a, 39);
        uint64_t mj = (a & b) ^ (a & c) ^ (b & c);
        uint64_t t2 = S0 + mj;
        h = g; g = f; f = e; e = d + t1;
        d = c; c = b; b = a; a = t1 + t2;
    }
    st[0] += a; st[1] += b; st[2] += c; st[3] += d;
    st[4] += e; st[5] += f; st[6] += g; st[7] += h;
}

void xo_sha512(uint8_t out[64], const uint8_t *in, size_t inlen)
{
    uint64_t st[8];
    uint8_t tail[256];
    size_t full = inlen / 128, rem = inlen % 128;
    memcpy(st, SHA512_IV, sizeof(st));
    for (size_t i = 0; i < full; i++) sha512_block(st, in + 128 * i);
    memset(tail, 0, sizeof(tail));
    memcpy(tail, in + 128 * full, rem);
    tail[rem] = 0x80;
    size_t tl = (rem + 17 <= 128) ? 128 : 256;
    /* 128-bit length; the high 64 bits are zero for any message here. */
    to_bytes(tail + tl - 8, 8, (unsigned long long)inlen * 8);
    sha512_block(st, tail);
    if (tl == 256) sha512_block(st, tail + 128);
    for (int i = 0; i < 8; i++) to_bytes(out + 8 * i, 8, st[i]);
}

/* ------------------------------------------------------------------------ */
/* Keccak-f[1600] and SHAKE (FIPS 202)                                      */
/* ------------------------------------------------------------------------ */

static uint64_t KECCAK_RC[24];
static unsigned KECCAK_RHO[25];
static pthread_once_t keccak_once = PTHREAD_ONCE_INIT;

/* rc(t) from FIPS 202 Algorithm 5 (LFSR x^8 + x^6 + x^5 + x^4 + 1). */
static int keccak_rc_bit(int t)
{
    if (t % 255 == 0) return 1;
    /* R = 10000000 as a bit array, r[0] leftmost; r[8] receives the bit
     * shifted out by "R = 0 || R". */
    int r[9] = {1, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i = 1; i <= t % 255; i++) {
        for (int j = 8; j >= 1; j--) r[j] = r[j - 1];
        r[0] = 0;
        r[0] ^= r[8];
        r[4] ^= r[8];
        r[5] ^= r[8];
        r[6] ^= r[8];
    }
    return r[0];
}

static void keccak_init_tables(void)
{
    for (int ir = 0; ir < 24; ir++) {
        uint64_t rc = 0;
        for (int j = 0; j <= 6; j++) {
            if (keccak_rc_bit(j + 7 * ir)) rc |= 1ULL << ((1 << j) - 1);
        }
        KECCAK_RC[ir] = rc;
    }
    /* rho offsets: FIPS 202 Algorithm 2. */
    KECCAK_RHO[0] = 0;
    int x = 1, y = 0;
    for (int t = 0; t < 24; t++) {
        KECCAK_RHO[x + 5 * y] = (unsigned)(((t + 1) * (t + 2) / 2) % 64);
        int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
}

static uint64_t rol64(uint64_t v, unsigned n)
{
    return n ? ((v << n) | (v >> (64 - n))) : v;
}

static void keccak_f1600(uint64_t A[25])
{
    pthread_once(&keccak_once, keccak_init_tables);
    for (int ir = 0; ir < 24; ir++) {
        uint64_t C[5], D[5], B[25];
        for (int x = 0; x < 5; x++)
            C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
        for (int x = 0; x < 5; x++)
            D[x] = C[(x + 4) % 5] ^ rol64(C[(x + 1) % 5], 1);
        for (int i = 0; i < 25; i++) A[i] ^= D[i % 5];
        /* rho and pi: B[y, 2x+3y] = rot(A[x, y], r[x, y]) */
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++)
                B[y + 5 * ((2 * x + 3 * y) % 5)] = rol64(A[x + 5 * y], KECCAK_RHO[x + 5 * y]);
        /* chi */
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++)
                A[x + 5 * y] = B[x + 5 * y] ^ (~B[(x + 1) % 5 + 5 * y] & B[(x + 2) % 5 + 5 * y]);
        /* iota */
        A[0] ^= KECCAK_RC[ir];
    }
}

static void shake(unsigned rate, uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen)
{
    uint64_t A[25];
    uint8_t blk[200];
    memset(A, 0, sizeof(A));
    while (inlen >= rate) {
        for (unsigned i = 0; i < rate / 8; i++) {
            uint64_t v = 0;
            for (int b = 0; b < 8; b++) v |= (uint64_t)in[8 * i + b] << (8 * b);
            A[i] ^= v;
        }
        keccak_f1600(A);
        in += rate;
        inlen -= rate;
    }
    memset(blk, 0, sizeof(blk));
    memcpy(blk, in, inlen);
    blk[inlen] ^= 0x1F;        /* SHAKE domain bits + first pad bit */
    blk[rate - 1] ^= 0x80;     /* last pad bit */
    for (unsigned i = 0; i < rate / 8; i++) {
        uint64_t v = 0;
        for (int b = 0; b < 8; b++) v |= (uint64_t)blk[8 * i + b] << (8 * b);
        A[i] ^= v;
    }
    keccak_f1600(A);
    for (;;) {
        size_t take = outlen < rate ? outlen : rate;
        for (size_t i = 0; i < take; i++) out[i] = (uint8_t)(A[i / 8] >> (8 * (i % 8)));
        out += take;
        outlen -= take;
        if (!outlen) break;
        keccak_f1600(A);
    }
}

void xo_shake128(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen)
{
    shake(168, out, outlen, in, inlen);
}

void xo_shake256(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen)
{
    shake(136, out, outlen, in, inlen);
}

/* ------------------------------------------------------------------------ */
/* Parameter sets: params.c                                                 */
/* ------------------------------------------------------------------------ */

typedef struct {
    const char *name;
    uint32_t oid;
    unsigned func, n, h, d;
} xo_set;

/* XMSS names and OIDs, params.c:7-76 / 254-375. */
static const xo_set XMSS_SETS[] = {
    {"XMSS-SHA2_10_256", 0x01, XO_SHA2, 32, 10, 1},
    {"XMSS-SHA2_16_256", 0x02, XO_SHA2, 32, 16, 1},
    {"XMSS-SHA2_20_256", 0x03, XO_SHA2, 32, 20, 1},
    {"XMSS-SHA2_10_512", 0x04, XO_SHA2, 64, 10, 1},
    {"XMSS-SHA2_16_512", 0x05, XO_SHA2, 64, 16, 1},
    {"XMSS-SHA2_20_512", 0x06, XO_SHA2, 64, 20, 1},
    {"XMSS-SHAKE_10_256", 0x07, XO_SHAKE128, 32, 10, 1},
    {"XMSS-SHAKE_16_256", 0x08, XO_SHAKE128, 32, 16, 1},
    {"XMSS-SHAKE_20_256", 0x09, XO_SHAKE128, 32, 20, 1},
    {"XMSS-SHAKE_10_512", 0x0a, XO_SHAKE256, 64, 10, 1},
    {"XMSS-SHAKE_16_512", 0x0b, XO_SHAKE256, 64, 16, 1},
    {"XMSS-SHAKE_20_512", 0x0c, XO_SHAKE256, 64, 20, 1},
    {"XMSS-SHA2_10_192", 0x0d, XO_SHA2, 24, 10, 1},
    {"XMSS-SHA2_16_192", 0x0e, XO_SHA2, 24, 16, 1},
    {"XMSS-SHA2_20_192", 0x0f, XO_SHA2, 24, 20, 1},
    {"XMSS-SHAKE256_10_256", 0x10, XO_SHAKE256, 32, 10, 1},
    {"XMSS-SHAKE256_16_256", 0x11, XO_SHAKE256, 32, 16, 1},
    {"XMSS-SHAKE256_20_256", 0x12, XO_SHAKE256, 32, 20, 1},
    {"XMSS-SHAKE256_10_192", 0x13, XO_SHAKE256, 24, 10, 1},
    {"XMSS-SHAKE256_16_192", 0x14, XO_SHAKE256, 24, 16, 1},
    {"XMSS-SHAKE256_20_192", 0x15, XO_SHAKE256, 24, 20, 1},
};

/* XMSS^MT: params.c:78-252 / 377-698.  Eight (h, d) shapes per family, in
 * OID order 20/2, 20/4, 40/2, 40/4, 40/8, 60/3, 60/6, 60/12; the families
 * come in OID blocks of 8: SHA2-256, SHA2-512, SHAKE-256, SHAKE-512,
 * SHA2-192, SHAKE256-256, SHAKE256-192. */
static const unsigned MT_H[8] = {20, 20, 40, 40, 40, 60, 60, 60};
static const unsigned MT_D[8] = {2, 4, 2, 4, 8, 3, 6, 12};
static const struct {
    const char *prefix;
    const char *suffix;
    unsigned func, n;
} MT_FAMILIES[7] = {
    {"XMSSMT-SHA2_", "_256", XO_SHA2, 32},
    {"XMSSMT-SHA2_", "_512", XO_SHA2, 64},
    {"XMSSMT-SHAKE_", "_256", XO_SHAKE128, 32},
    {"XMSSMT-SHAKE_", "_512", XO_SHAKE256, 64},
    {"XMSSMT-SHA2_", "_192", XO_SHA2, 24},
    {"XMSSMT-SHAKE256_", "_256", XO_SHAKE256, 32},
    {"XMSSMT-SHAKE256_", "_192", XO_SHAKE256, 24},
};

#include <stdio.h>

int xo_str_to_oid(uint32_t *oid, const char *s, int mt)
{
    if (!mt) {
        for (size_t i = 0; i < sizeof(XMSS_SETS) / sizeof(XMSS_SETS[0]); i++) {
            if (!strcmp(s, XMSS_SETS[i].name)) {
                *oid = XMSS_SETS[i].oid;
                return 0;
            }
        }
        return -1;
    }
    char buf[64];
    for (unsigned f = 0; f < 7; f++) {
        for (unsigned k = 0; k < 8; k++) {
            snprintf(buf, sizeof(buf), "%s%u/%u%s", MT_FAMILIES[f].prefix, MT_H[k],
                     MT_D[k], MT_FAMILIES[f].suffix);
            if (!strcmp(s, buf)) {
                *oid = 8 * f + k + 1;
                return 0;
            }
        }
    }
    return -1;
}

int xo_initialize_params(xo_params *p)
{
    /* params.c:710-753 */
    p->tree_height = p->full_height / p->d;
    if (p->wots_w == 4) {
        p->wots_log_w = 2;
        p->wots_len2 = 5;
    } else if (p->wots_w == 16) {
        p->wots_log_w = 4;
        p->wots_len2 = 3;
    } else if (p->wots_w == 256) {
        p->wots_log_w = 8;
        p->wots_len2 = 2;
    } else {
        return -1;
    }
    p->wots_len1 = 8 * p->n / p->wots_log_w;
    p->wots_len = p->wots_len1 + p->wots_len2;
    p->wots_sig_bytes = p->wots_len * p->n;
    p->index_bytes = (p->d == 1) ? 4 : (p->full_height + 7) / 8;
    p->sig_bytes = p->index_bytes + p->n + p->d * p->wots_sig_bytes + p->full_height * p->n;
    p->pk_bytes = 2 * p->n;
    p->sk_bytes = p->index_bytes + 4 * p->n; /* xmss_core.c:93-96 */
    return 0;
}

int xo_parse_oid(xo_params *p, uint32_t oid, int mt)
{
    memset(p, 0, sizeof(*p));
    if (!mt) {
        if (oid < 1 || oid > 0x15) return -1;
        const xo_set *s = &XMSS_SETS[oid - 1];
        p->func = s->func;
        p->n = s->n;
        p->full_height = s->h;
        p->d = 1;
    } else {
        if (oid < 1 || oid > 0x38) return -1;
        unsigned f = (oid - 1) / 8, k = (oid - 1) % 8;
        p->func = MT_FAMILIES[f].func;
        p->n = MT_FAMILIES[f].n;
        p->full_height = MT_H[k];
        p->d = MT_D[k];
    }
    p->padding_len = (p->n == 24) ? 4 : p->n; /* params.c:293-328 */
    p->wots_w = 16;
    p->bds_k = 0;
    return xo_initialize_params(p);
}

/* ------------------------------------------------------------------------ */
/* Addresses: hash_address.c:1-65 and hash.c:19-25                          */
/* ------------------------------------------------------------------------ */

enum { ADDR_OTS = 0, ADDR_LTREE = 1, ADDR_HASHTREE = 2 };

static void addr_bytes(uint8_t out[32], const uint32_t a[8])
{
    for (int i = 0; i < 8; i++) to_bytes(out + 4 * i, 4, a[i]);
}

static void set_tree(uint32_t a[8], uint64_t tree)
{
    a[1] = (uint32_t)(tree >> 32);
    a[2] = (uint32_t)tree;
}

/* ------------------------------------------------------------------------ */
/* Tweakable hashes: hash.c:29-183                                          */
/* ------------------------------------------------------------------------ */

static int core_hash(const xo_params *p, uint8_t *out, const uint8_t *in, size_t inlen)
{
    /* hash.c:29-65: dispatch by (n, func). */
    uint8_t buf[64];
    if (p->func == XO_SHA2 && (p->n == 24 || p->n == 32)) {
        xo_sha256(buf, in, inlen);
        memcpy(out, buf, p->n);
    } else if (p->func == XO_SHA2 && p->n == 64) {
        xo_sha512(out, in, inlen);
    } else if (p->func == XO_SHAKE128 && p->n == 32) {
        xo_shake128(out, 32, in, inlen);
    } else if (p->func == XO_SHAKE256 && (p->n == 24 || p->n == 32 || p->n == 64)) {
        xo_shake256(out, p->n, in, inlen);
    } else {
        return -1;
    }
    return 0;
}

int xo_prf(const xo_params *p, uint8_t *out, const uint8_t in[32], const uint8_t *key)
{
    /* hash.c:70-81: toByte(3, padding_len) || key || in */
    uint8_t buf[64 + 64 + 32];
    to_bytes(buf, p->padding_len, 3);
    memcpy(buf + p->padding_len, key, p->n);
    memcpy(buf + p->padding_len + p->n, in, 32);
    return core_hash(p, out, buf, p->padding_len + p->n + 32);
}

int xo_prf_keygen(const xo_params *p, uint8_t *out, const uint8_t *in, const uint8_t *key)
{
    /* hash.c:87-98: toByte(4, padding_len) || key || in (n + 32 bytes) */
    uint8_t buf[64 + 64 + 64 + 32];
    to_bytes(buf, p->padding_len, 4);
    memcpy(buf + p->padding_len, key, p->n);
    memcpy(buf + p->padding_len + p->n, in, p->n + 32);
    return core_hash(p, out, buf, p->padding_len + 2 * p->n + 32);
}

int xo_hash_message(const xo_params *p, uint8_t *out, const uint8_t *R,
                    const uint8_t *root, unsigned long long idx,
                    const uint8_t *m, unsigned long long mlen)
{
    /* hash.c:107-120: toByte(2, pl) || R || root || toByte(idx, n) || M.
     * The reference writes this prefix into caller memory in front of M; the
     * oracle builds the same byte string in a fresh buffer. */
    size_t pre = p->padding_len + 3 * p->n;
    uint8_t *buf = (uint8_t *)malloc(pre + mlen + 1);
    if (!buf) return -1;
    to_bytes(buf, p->padding_len, 2);
    memcpy(buf + p->padding_len, R, p->n);
    memcpy(buf + p->padding_len + p->n, root, p->n);
    to_bytes(buf + p->padding_len + 2 * p->n, p->n, idx);
    if (mlen) memcpy(buf + pre, m, mlen);
    int r = core_hash(p, out, buf, pre + mlen);
    free(buf);
    return r;
}

int xo_thash_h(const xo_params *p, uint8_t *out, const uint8_t *in,
               const uint8_t *pub_seed, uint32_t addr[8])
{
    /* hash.c:125-155 */
    uint8_t buf[64 + 3 * 64], mask[2 * 64], ab[32];
    to_bytes(buf, p->padding_len, 1);
    addr[7] = 0;
    addr_bytes(ab, addr);
    xo_prf(p, buf + p->padding_len, ab, pub_seed);
    addr[7] = 1;
    addr_bytes(ab, addr);
    xo_prf(p, mask, ab, pub_seed);
    addr[7] = 2;
    addr_bytes(ab, addr);
    xo_prf(p, mask + p->n, ab, pub_seed);
    for (unsigned i = 0; i < 2 * p->n; i++) buf[p->padding_len + p->n + i] = in[i] ^ mask[i];
    return core_hash(p, out, buf, p->padding_len + 3 * p->n);
}

int xo_thash_f(const xo_params *p, uint8_t *out, const uint8_t *in,
               const uint8_t *pub_seed, uint32_t addr[8])
{
    /* hash.c:157-183 */
    uint8_t buf[64 + 2 * 64], mask[64], ab[32];
    to_bytes(buf, p->padding_len, 0);
    addr[7] = 0;
    addr_bytes(ab, addr);
    xo_prf(p, buf + p->padding_len, ab, pub_seed);
    addr[7] = 1;
    addr_bytes(ab, addr);
    xo_prf(p, mask, ab, pub_seed);
    for (unsigned i = 0; i < p->n; i++) buf[p->padding_len + p->n + i] = in[i] ^ mask[i];
    return core_hash(p, out, buf, p->padding_len + 2 * p->n);
}

/* ------------------------------------------------------------------------ */
/* WOTS+: wots.c                                                            */
/* ------------------------------------------------------------------------ */

static void expand_seed(const xo_params *p, uint8_t *outseeds, const uint8_t *inseed,
                        const uint8_t *pub_seed, uint32_t addr[8])
{
    /* wots.c:14-29: PRF_keygen(SK_SEED, PUB_SEED || ADRS(chain=i, hash=0, km=0)) */
    uint8_t buf[64 + 32];
    addr[6] = 0;
    addr[7] = 0;
    memcpy(buf, pub_seed, p->n);
    for (unsigned i = 0; i < p->wots_len; i++) {
        addr[5] = i;
        addr_bytes(buf + p->n, addr);
        xo_prf_keygen(p, outseeds + i * p->n, buf, inseed);
    }
}

static void gen_chain(const xo_params *p, uint8_t *out, const uint8_t *in,
                      unsigned start, unsigned steps, const uint8_t *pub_seed,
                      uint32_t addr[8])
{
    /* wots.c:38-53 */
    memmove(out, in, p->n);
    for (unsigned i = start; i < start + steps && i < p->wots_w; i++) {
        addr[6] = i;
        xo_thash_f(p, out, out, pub_seed, addr);
    }
}

static void base_w(const xo_params *p, int *output, int out_len, const uint8_t *input)
{
    /* wots.c:60-79 */
    int in = 0, bits = 0;
    unsigned total = 0;
    for (int o = 0; o < out_len; o++) {
        if (bits == 0) {
            total = input[in++];
            bits = 8;
        }
        bits -= (int)p->wots_log_w;
        output[o] = (int)((total >> bits) & (p->wots_w - 1));
    }
}

void xo_chain_lengths(const xo_params *p, int *lengths, const uint8_t *msg)
{
    /* wots.c:82-107: message digits, then the checksum digits. */
    base_w(p, lengths, (int)p->wots_len1, msg);
    int csum = 0;
    for (unsigned i = 0; i < p->wots_len1; i++) csum += (int)p->wots_w - 1 - lengths[i];
    csum <<= (8 - ((p->wots_len2 * p->wots_log_w) % 8));
    uint8_t cb[8];
    unsigned cbl = (p->wots_len2 * p->wots_log_w + 7) / 8;
    to_bytes(cb, cbl, (unsigned long long)csum);
    base_w(p, lengths + p->wots_len1, (int)p->wots_len2, cb);
}

void xo_wots_pkgen(const xo_params *p, uint8_t *pk, const uint8_t *seed,
                   const uint8_t *pub_seed, uint32_t addr[8])
{
    /* wots.c:117-131 */
    expand_seed(p, pk, seed, pub_seed, addr);
    for (unsigned i = 0; i < p->wots_len; i++) {
        addr[5] = i;
        gen_chain(p, pk + i * p->n, pk + i * p->n, 0, p->wots_w - 1, pub_seed, addr);
    }
}

void xo_wots_sign(const xo_params *p, uint8_t *sig, const uint8_t *msg,
                  const uint8_t *seed, const uint8_t *pub_seed, uint32_t addr[8])
{
    /* wots.c:136-154 */
    int lengths[256];
    xo_chain_lengths(p, lengths, msg);
    expand_seed(p, sig, seed, pub_seed, addr);
    for (unsigned i = 0; i < p->wots_len; i++) {
        addr[5] = i;
        gen_chain(p, sig + i * p->n, sig + i * p->n, 0, (unsigned)lengths[i], pub_seed, addr);
    }
}

void xo_wots_pk_from_sig(const xo_params *p, uint8_t *pk, const uint8_t *sig,
                         const uint8_t *msg, const uint8_t *pub_seed, uint32_t addr[8])
{
    /* wots.c:161-175 */
    int lengths[256];
    xo_chain_lengths(p, lengths, msg);
    for (unsigned i = 0; i < p->wots_len; i++) {
        addr[5] = i;
        gen_chain(p, pk + i * p->n, sig + i * p->n, (unsigned)lengths[i],
                  p->wots_w - 1 - (unsigned)lengths[i], pub_seed, addr);
    }
}

int xo_verify_chain_steps(const xo_params *p, const uint8_t *msg)
{
    int lengths[256], s = 0;
    xo_chain_lengths(p, lengths, msg);
    for (unsigned i = 0; i < p->wots_len; i++) s += (int)p->wots_w - 1 - lengths[i];
    return s;
}

/* ------------------------------------------------------------------------ */
/* L-tree, compute_root, leaves: xmss_commons.c                             */
/* ------------------------------------------------------------------------ */

static void l_tree(const xo_params *p, uint8_t *leaf, uint8_t *wots_pk,
                   const uint8_t *pub_seed, uint32_t addr[8])
{
    /* xmss_commons.c:16-49: pairwise, odd node carried up; in place. */
    unsigned l = p->wots_len;
    uint32_t height = 0;
    addr[5] = height;
    while (l > 1) {
        unsigned parents = l >> 1;
        for (unsigned i = 0; i < parents; i++) {
            addr[6] = i;
            xo_thash_h(p, wots_pk + i * p->n, wots_pk + 2 * i * p->n, pub_seed, addr);
        }
        if (l & 1) {
            memcpy(wots_pk + (l >> 1) * p->n, wots_pk + (l - 1) * p->n, p->n);
            l = (l >> 1) + 1;
        } else {
            l >>= 1;
        }
        height++;
        addr[5] = height;
    }
    memcpy(leaf, wots_pk, p->n);
}

static void compute_root(const xo_params *p, uint8_t *root, const uint8_t *leaf,
                         unsigned long leafidx, const uint8_t *auth,
                         const uint8_t *pub_seed, uint32_t addr[8])
{
    /* xmss_commons.c:54-96 */
    uint8_t buf[2 * 64];
    if (leafidx & 1) {
        memcpy(buf + p->n, leaf, p->n);
        memcpy(buf, auth, p->n);
    } else {
        memcpy(buf, leaf, p->n);
        memcpy(buf + p->n, auth, p->n);
    }
    auth += p->n;
    for (unsigned i = 0; i < p->tree_height - 1; i++) {
        addr[5] = i;
        leafidx >>= 1;
        addr[6] = (uint32_t)leafidx;
        if (leafidx & 1) {
            xo_thash_h(p, buf + p->n, buf, pub_seed, addr);
            memcpy(buf, auth, p->n);
        } else {
            xo_thash_h(p, buf, buf, pub_seed, addr);
            memcpy(buf + p->n, auth, p->n);
        }
        auth += p->n;
    }
    addr[5] = p->tree_height - 1;
    leafidx >>= 1;
    addr[6] = (uint32_t)leafidx;
    xo_thash_h(p, root, buf, pub_seed, addr);
}

void xo_gen_leaf_wots(const xo_params *p, uint8_t *leaf, const uint8_t *sk_seed,
                      const uint8_t *pub_seed, uint32_t ltree_addr[8], uint32_t ots_addr[8])
{
    /* xmss_commons.c:104-113 */
    uint8_t pk[256 * 64];
    xo_wots_pkgen(p, pk, sk_seed, pub_seed, ots_addr);
    l_tree(p, leaf, pk, pub_seed, ltree_addr);
}

/* ------------------------------------------------------------------------ */
/* treehash: xmss_core.c:19-86                                              */
/* ------------------------------------------------------------------------ */

void xo_treehash(const xo_params *p, uint8_t *root, uint8_t *auth_path,
                 const uint8_t *sk_seed, const uint8_t *pub_seed,
                 uint32_t leaf_idx, const uint32_t subtree_addr[8])
{
    uint8_t stack[(20 + 1) * 64];
    unsigned heights[20 + 1];
    unsigned offset = 0;
    uint32_t ots[8] = {0}, lt[8] = {0}, node[8] = {0};
    for (int i = 0; i < 3; i++) ots[i] = lt[i] = node[i] = subtree_addr[i];
    ots[3] = ADDR_OTS;
    lt[3] = ADDR_LTREE;
    node[3] = ADDR_HASHTREE;
    for (uint32_t idx = 0; idx < (1u << p->tree_height); idx++) {
        lt[4] = idx;
        ots[4] = idx;
        xo_gen_leaf_wots(p, stack + offset * p->n, sk_seed, pub_seed, lt, ots);
        offset++;
        heights[offset - 1] = 0;
        if ((leaf_idx ^ 0x1) == idx) memcpy(auth_path, stack + (offset - 1) * p->n, p->n);
        while (offset >= 2 && heights[offset - 1] == heights[offset - 2]) {
            uint32_t tree_idx = idx >> (heights[offset - 1] + 1);
            node[5] = heights[offset - 1];
            node[6] = tree_idx;
            xo_thash_h(p, stack + (offset - 2) * p->n, stack + (offset - 2) * p->n, pub_seed, node);
            offset--;
            heights[offset - 1]++;
            if (((leaf_idx >> heights[offset - 1]) ^ 0x1) == tree_idx)
                memcpy(auth_path + heights[offset - 1] * p->n, stack + (offset - 1) * p->n, p->n);
        }
    }
    memcpy(root, stack, p->n);
}

/* ------------------------------------------------------------------------ */
/* Threaded full-tree helper (test infrastructure)                          */
/* ------------------------------------------------------------------------ */

typedef struct {
    const xo_params *p;
    uint8_t *leaves;
    const uint8_t *sk_seed, *pub_seed;
    uint32_t layer;
    uint64_t tree;
    uint32_t first, count, stride, tid;
} leaf_job;

static void *leaf_worker(void *arg)
{
    leaf_job *j = (leaf_job *)arg;
    uint32_t ots[8] = {0}, lt[8] = {0};
    ots[0] = lt[0] = j->layer;
    set_tree(ots, j->tree);
    set_tree(lt, j->tree);
    ots[3] = ADDR_OTS;
    lt[3] = ADDR_LTREE;
    for (uint32_t i = j->tid; i < j->count; i += j->stride) {
        uint32_t idx = j->first + i;
        lt[4] = idx;
        ots[4] = idx;
        xo_gen_leaf_wots(j->p, j->leaves + (size_t)i * j->p->n, j->sk_seed, j->pub_seed, lt, ots);
    }
    return NULL;
}

int xo_leaves(const xo_params *p, uint8_t *leaves, const uint8_t *sk_seed,
              const uint8_t *pub_seed, uint32_t layer, uint64_t tree,
              uint32_t first, uint32_t count, int nthreads)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    leaf_job jobs[256];
    for (int t = 0; t < nthreads; t++) {
        jobs[t] = (leaf_job){p, leaves, sk_seed, pub_seed, layer, tree, first, count,
                             (uint32_t)nthreads, (uint32_t)t};
        if (pthread_create(&th[t], NULL, leaf_worker, &jobs[t])) return -1;
    }
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
    return 0;
}

int xo_tree_nodes(const xo_params *p, uint8_t *nodes, const uint8_t *sk_seed,
                  const uint8_t *pub_seed, uint32_t layer, uint64_t tree, int nthreads)
{
    uint32_t nleaves = 1u << p->tree_height;
    if (xo_leaves(p, nodes, sk_seed, pub_seed, layer, tree, 0, nleaves, nthreads)) return -1;
    uint32_t node[8] = {0};
    node[0] = layer;
    set_tree(node, tree);
    node[3] = ADDR_HASHTREE;
    uint8_t *lvl = nodes;
    uint32_t cnt = nleaves;
    for (unsigned h = 0; h < p->tree_height; h++) {
        uint8_t *up = lvl + (size_t)cnt * p->n;
        for (uint32_t i = 0; i < cnt / 2; i++) {
            node[5] = h;
            node[6] = i;
            xo_thash_h(p, up + (size_t)i * p->n, lvl + (size_t)2 * i * p->n, pub_seed, node);
        }
        lvl = up;
        cnt /= 2;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Key generation, sign, verify: xmss_core.c / xmss_commons.c               */
/* ------------------------------------------------------------------------ */

int xo_seed_keypair(const xo_params *p, uint8_t *pk, uint8_t *sk, const uint8_t *seed)
{
    /* xmss_core.c:134-161.  sk = idx || SK_SEED || SK_PRF || root || PUB_SEED */
    uint8_t auth[20 * 64];
    uint32_t top[8] = {0};
    top[0] = p->d - 1;
    memset(sk, 0, p->index_bytes);
    sk += p->index_bytes;
    memcpy(sk, seed, 2 * p->n);
    memcpy(sk + 3 * p->n, seed + 2 * p->n, p->n);
    memcpy(pk + p->n, sk + 3 * p->n, p->n);
    xo_treehash(p, pk, auth, sk, pk + p->n, 0, top);
    memcpy(sk + 2 * p->n, pk, p->n);
    return 0;
}

/* Shared tail of xo_sign / xo_sign_with_trees (xmss_core.c:183-273).  When
 * layer_nodes is NULL every layer's subtree is recomputed by treehash; else
 * the root and auth path are read from the precomputed node arrays. */
static int sign_impl(const xo_params *p, uint8_t *sk, uint8_t *sm,
                     unsigned long long *smlen, const uint8_t *m,
                     unsigned long long mlen, const uint8_t *layer_nodes)
{
    const uint8_t *sk_seed = sk + p->index_bytes;
    const uint8_t *sk_prf = sk + p->index_bytes + p->n;
    const uint8_t *pub_root = sk + p->index_bytes + 2 * p->n;
    const uint8_t *pub_seed = sk + p->index_bytes + 3 * p->n;
    uint8_t root[64], idx32[32];
    uint32_t ots[8] = {0};
    ots[3] = ADDR_OTS;

    memmove(sm + p->sig_bytes, m, mlen);
    *smlen = p->sig_bytes + mlen;

    unsigned long long idx = from_bytes(sk, p->index_bytes);
    /* Exhaustion handling, xmss_core.c:212-231: the sk is wiped; the index
     * 2^h - 1 still signs (with the wiped sk), anything above returns -2. */
    if (idx >= ((1ULL << p->full_height) - 1)) {
        memset(sk, 0xFF, p->index_bytes);
        memset(sk + p->index_bytes, 0, (size_t)(p->sk_bytes - p->index_bytes));
        if (idx > ((1ULL << p->full_height) - 1)) return -2;
        if (p->full_height == 64 && idx == ((1ULL << p->full_height) - 1)) return -2;
    }
    memcpy(sm, sk, p->index_bytes);
    to_bytes(sk, p->index_bytes, idx + 1);

    to_bytes(idx32, 32, idx);
    xo_prf(p, sm + p->index_bytes, idx32, sk_prf);
    xo_hash_message(p, root, sm + p->index_bytes, pub_root, idx, sm + p->sig_bytes, mlen);
    sm += p->index_bytes + p->n;

    size_t nodes_per_layer = ((size_t)2 << p->tree_height) - 1;
    for (unsigned i = 0; i < p->d; i++) {
        uint32_t idx_leaf = (uint32_t)(idx & ((1ULL << p->tree_height) - 1));
        idx >>= p->tree_height;
        ots[0] = i;
        set_tree(ots, idx);
        ots[4] = idx_leaf;
        xo_wots_sign(p, sm, root, sk_seed, pub_seed, ots);
        sm += p->wots_sig_bytes;
        if (!layer_nodes) {
            xo_treehash(p, root, sm, sk_seed, pub_seed, idx_leaf, ots);
        } else {
            const uint8_t *lvl = layer_nodes + (size_t)i * nodes_per_layer * p->n;
            uint32_t cnt = 1u << p->tree_height;
            for (unsigned h = 0; h < p->tree_height; h++) {
                memcpy(sm + h * p->n, lvl + (size_t)((idx_leaf >> h) ^ 1) * p->n, p->n);
                lvl += (size_t)cnt * p->n;
                cnt >>= 1;
            }
            memcpy(root, lvl, p->n);
        }
        sm += p->tree_height * p->n;
    }
    return 0;
}

int xo_sign(const xo_params *p, uint8_t *sk, uint8_t *sm, unsigned long long *smlen,
            const uint8_t *m, unsigned long long mlen)
{
    return sign_impl(p, sk, sm, smlen, m, mlen, NULL);
}

int xo_sign_with_trees(const xo_params *p, uint8_t *sk, uint8_t *sm,
                       unsigned long long *smlen, const uint8_t *m,
                       unsigned long long mlen, const uint8_t *layer_nodes)
{
    return sign_impl(p, sk, sm, smlen, m, mlen, layer_nodes);
}

int xo_sign_open(const xo_params *p, uint8_t *m, unsigned long long *mlen,
                 const uint8_t *sm, unsigned long long smlen, const uint8_t *pk)
{
    /* xmss_commons.c:136-215 */
    const uint8_t *pub_root = pk;
    const uint8_t *pub_seed = pk + p->n;
    uint8_t wots_pk[256 * 64], leaf[64], root[64];
    uint32_t ots[8] = {0}, lt[8] = {0}, node[8] = {0};
    ots[3] = ADDR_OTS;
    lt[3] = ADDR_LTREE;
    node[3] = ADDR_HASHTREE;

    *mlen = smlen - p->sig_bytes;
    unsigned long long idx = from_bytes(sm, p->index_bytes);
    /* The reference stages M at m + sig_bytes; the message hash input is the
     * same byte string either way. */
    memmove(m + p->sig_bytes, sm + p->sig_bytes, *mlen);
    xo_hash_message(p, root, sm + p->index_bytes, pk, idx, m + p->sig_bytes, *mlen);
    sm += p->index_bytes + p->n;
    for (unsigned i = 0; i < p->d; i++) {
        uint32_t idx_leaf = (uint32_t)(idx & ((1ULL << p->tree_height) - 1));
        idx >>= p->tree_height;
        ots[0] = lt[0] = node[0] = i;
        set_tree(ots, idx);
        set_tree(lt, idx);
        set_tree(node, idx);
        ots[4] = idx_leaf;
        xo_wots_pk_from_sig(p, wots_pk, sm, root, pub_seed, ots);
        sm += p->wots_sig_bytes;
        lt[4] = idx_leaf;
        l_tree(p, leaf, wots_pk, pub_seed, lt);
        compute_root(p, root, leaf, idx_leaf, sm, pub_seed, node);
        sm += p->tree_height * p->n;
    }
    if (memcmp(root, pub_root, p->n)) {
        memset(m, 0, *mlen);
        *mlen = 0;
        return -1;
    }
    memcpy(m, sm, *mlen);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* OID-prefixed wrappers: xmss.c:10-109                                     */
/* ------------------------------------------------------------------------ */

static uint32_t read_oid(const uint8_t *b)
{
    return (uint32_t)from_bytes(b, 4);
}

int xo_api_seed_keypair(uint8_t *pk, uint8_t *sk, uint32_t oid, int mt, const uint8_t *seed)
{
    xo_params p;
    if (xo_parse_oid(&p, oid, mt)) return -1;
    to_bytes(pk, 4, oid);
    to_bytes(sk, 4, oid);
    return xo_seed_keypair(&p, pk + 4, sk + 4, seed);
}

int xo_api_sign(uint8_t *sk, uint8_t *sm, unsigned long long *smlen,
                const uint8_t *m, unsigned long long mlen, int mt)
{
    xo_params p;
    if (xo_parse_oid(&p, read_oid(sk), mt)) return -1;
    return xo_sign(&p, sk + 4, sm, smlen, m, mlen);
}

int xo_api_sign_open(uint8_t *m, unsigned long long *mlen, const uint8_t *sm,
                     unsigned long long smlen, const uint8_t *pk, int mt)
{
    xo_params p;
    if (xo_parse_oid(&p, read_oid(pk), mt)) return -1;
    return xo_sign_open(&p, m, mlen, sm, smlen, pk + 4);
}
