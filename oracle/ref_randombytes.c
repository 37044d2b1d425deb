/*
 * Deterministic stand-in for the reference's randombytes.c (which reads
 * /dev/urandom, cuxmss/randombytes.c:10-39), linked into the reference build
 * under oracle/_ref only.  The stream is SHAKE-free on purpose: a 64-bit
 * xorshift seeded by ref_randombytes_seed(), so parity runs of the reference
 * are reproducible.  Test infrastructure only.
 */
#include <stdint.h>

static uint64_t state = 0x9E3779B97F4A7C15ULL;

void ref_randombytes_seed(uint64_t seed)
{
    state = seed ? seed : 0x9E3779B97F4A7C15ULL;
}

void randombytes(unsigned char *x, unsigned long long xlen)
{
    while (xlen--) {
        state ^= state << 13;
        state ^= state >> 7;
        state ^= state << 17;
        *x++ = (unsigned char)(state >> 24);
    }
}
