// Hash cores for sm_100a: SHA-256 and SHA-512 compressions (FIPS 180-4) and
// Keccak-f[1600] (FIPS 202), all register resident and fully unrolled so that
// round constants become immediates and rotates become funnel shifts.
//
// Messages are handled as arrays of 32-bit words whose count is a compile-time
// constant; SHA-2 words are big-endian (word i = bytes 4i..4i+3, most
// significant first), Keccak words are little-endian (lane = w[2i] | w[2i+1]<<32).
#pragma once

#include <cstdint>

namespace xb {

__device__ __forceinline__ uint32_t ror32(uint32_t x, int n) { return __funnelshift_r(x, x, n); }
__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

// Pipe balancing.  SHA-256 here is bound by the integer ALU pipe (rotates,
// LOP3 and IADD3 all issue there) while the FMA pipe idles.  An integer
// multiply-add with a multiplier the compiler cannot see (read from constant
// memory, always 1 at run time) executes on the FMA pipe, so additions
// written as a * one + b move off the ALU pipe; right shifts by k likewise
// become mul.hi by 2^(32-k).  Results are bit-identical.
static __constant__ uint32_t xb_pipe_one = 1u;
static __constant__ uint32_t xb_pipe_zero = 0u;

// v | (dep & 0) with a zero the compiler cannot see: makes v depend on dep,
// which keeps two otherwise independent compressions from being interleaved
// (each interleaved compression holds another ~24 registers).
__device__ __forceinline__ uint32_t after(uint32_t v, uint32_t dep)
{
    uint32_t r;
    asm("and.b32 %0, %1, %2;" : "=r"(r) : "r"(dep), "r"(xb_pipe_zero));
    return v | r;
}
static __constant__ uint32_t xb_pipe_pow2[33] = {
    0u,        1u << 1,  1u << 2,  1u << 3,  1u << 4,  1u << 5,  1u << 6,  1u << 7,  1u << 8,
    1u << 9,   1u << 10, 1u << 11, 1u << 12, 1u << 13, 1u << 14, 1u << 15, 1u << 16, 1u << 17,
    1u << 18,  1u << 19, 1u << 20, 1u << 21, 1u << 22, 1u << 23, 1u << 24, 1u << 25, 1u << 26,
    1u << 27,  1u << 28, 1u << 29, 1u << 30, 1u << 31, 0u};

__device__ __forceinline__ uint32_t fma_add(uint32_t a, uint32_t b)
{
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(xb_pipe_one), "r"(b));
    return r;
}

// x >> k for 0 < k < 32 on the FMA pipe
template <int K>
__device__ __forceinline__ uint32_t fma_shr(uint32_t x)
{
    uint32_t r;
    asm("mul.hi.u32 %0, %1, %2;" : "=r"(r) : "r"(x), "r"(xb_pipe_pow2[32 - K]));
    return r;
}

// ---------------------------------------------------------------------------
// SHA-256 compression (FIPS 180-4 6.2.2).  `w` is consumed (message schedule
// is expanded in place in a 16-word window).  MIX selects how the work is
// spread over the ALU and FMA pipes: 0 all on ALU, 1 the additions on FMA,
// 2 additions and the schedule's right shifts on FMA; 3 is the ALU form
// re-associated for latency: e' = (d + h + K + W) + S1 + Ch and
// a' = ((h + K + W) + S0 + Maj) + S1 + Ch, so each round has three dependent
// levels (rotate, xor, add) on both the a and the e path instead of four.
// ---------------------------------------------------------------------------
#ifndef XB_SHA256_MIX
#define XB_SHA256_MIX 0
#endif

template <int MIX>
__device__ __forceinline__ void sha256_compress_t(uint32_t (&st)[8], uint32_t (&w)[16])
{
    const uint32_t K[64] = {
        0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u,
        0x923f82a4u, 0xab1c5ed5u, 0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u,
        0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u, 0xe49b69c1u, 0xefbe4786u,
        0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
        0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u,
        0x06ca6351u, 0x14292967u, 0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u,
        0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u, 0xa2bfe8a1u, 0xa81a664bu,
        0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
        0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au,
        0x5b9cca4fu, 0x682e6ff3u, 0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u,
        0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
    uint32_t e = st[4], f = st[5], g = st[6], h = st[7];
#pragma unroll
    for (int t = 0; t < 64; t++) {
        if (t >= 16) {
            const uint32_t x15 = w[(t - 15) & 15], x2 = w[(t - 2) & 15];
            if constexpr (MIX == 0 || MIX == 3) {
                const uint32_t s0 = ror32(x15, 7) ^ ror32(x15, 18) ^ (x15 >> 3);
                const uint32_t s1 = ror32(x2, 17) ^ ror32(x2, 19) ^ (x2 >> 10);
                w[t & 15] += s0 + w[(t - 7) & 15] + s1;
            } else {
                const uint32_t r0 = (MIX == 2) ? fma_shr<3>(x15) : (x15 >> 3);
                const uint32_t r1 = (MIX == 2) ? fma_shr<10>(x2) : (x2 >> 10);
                const uint32_t s0 = ror32(x15, 7) ^ ror32(x15, 18) ^ r0;
                const uint32_t s1 = ror32(x2, 17) ^ ror32(x2, 19) ^ r1;
                w[t & 15] = fma_add(s1, fma_add(s0, w[t & 15] + w[(t - 7) & 15]));
            }
        }
        const uint32_t S1 = ror32(e, 6) ^ ror32(e, 11) ^ ror32(e, 25);
        const uint32_t ch = g ^ (e & (f ^ g));
        const uint32_t S0 = ror32(a, 2) ^ ror32(a, 13) ^ ror32(a, 22);
        const uint32_t mj = (a & b) | (c & (a | b));
        if constexpr (MIX == 0) {
            const uint32_t t1 = h + S1 + ch + K[t] + w[t & 15];
            h = g; g = f; f = e; e = d + t1;
            d = c; c = b; b = a; a = t1 + S0 + mj;
        } else if constexpr (MIX == 3) {
            const uint32_t hkw = h + K[t] + w[t & 15];
            const uint32_t dhkw = d + hkw;
            const uint32_t s1c = S1 + ch;
            h = g; g = f; f = e; e = dhkw + s1c;
            d = c; c = b; b = a; a = (hkw + S0 + mj) + s1c;
        } else {
            const uint32_t t1 = fma_add(ch, fma_add(S1, h + K[t] + w[t & 15]));
            h = g; g = f; f = e; e = fma_add(d, t1);
            d = c; c = b; b = a; a = fma_add(S0, fma_add(mj, t1));
        }
    }
    st[0] += a; st[1] += b; st[2] += c; st[3] += d;
    st[4] += e; st[5] += f; st[6] += g; st[7] += h;
}

// Rotations on the FMA pipe.  x * 2^(32-k) is a 64-bit product whose high
// word is x >> k and whose low word is x << (32-k); the two have no bit in
// common, so their sum is rotr(x, k).  The power of two comes from constant
// memory, so the multiplies stay multiplies (IMAD) instead of becoming
// shifts (ALU pipe).
template <int K>
__device__ __forceinline__ uint32_t fma_ror(uint32_t x)
{
    uint32_t lo, r;
    asm("mul.lo.u32 %0, %1, %2;" : "=r"(lo) : "r"(x), "r"(xb_pipe_pow2[32 - K]));
    asm("mad.hi.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(x), "r"(xb_pipe_pow2[32 - K]), "r"(lo));
    return r;
}

template <int K>
__device__ __forceinline__ uint32_t fma_ror_wide(uint32_t x)
{
    uint32_t lo, hi;
    asm("{\n\t.reg .u64 t;\n\tmul.wide.u32 t, %2, %3;\n\tmov.b64 {%0, %1}, t;\n\t}"
        : "=r"(lo), "=r"(hi)
        : "r"(x), "r"(xb_pipe_pow2[32 - K]));
    return fma_add(lo, hi);
}

// SHA-256 compression with more of the ALU work moved to the FMA pipe than
// sha256_compress_t<1> (compare with the rate probe; results identical):
//   4  the schedule's w[t-16] + w[t-7] and the final state additions too
//   5  4, and one rotation of each of S0 and S1 as fma_ror
//   6  4, and the same rotations as fma_ror_wide
//   7  5, and h + K[t] + W[t] as two multiply-adds
//   8  5, and the schedule's shifts (fma_shr) and one rotation of each of
//      s0 and s1 as fma_ror
//   9  4, and every rotation of S0 and S1 as fma_ror
template <int MIX>
__device__ __forceinline__ void sha256_compress_x(uint32_t (&st)[8], uint32_t (&w)[16])
{
    const uint32_t K[64] = {
        0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u,
        0x923f82a4u, 0xab1c5ed5u, 0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u,
        0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u, 0xe49b69c1u, 0xefbe4786u,
        0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
        0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u,
        0x06ca6351u, 0x14292967u, 0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u,
        0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u, 0xa2bfe8a1u, 0xa81a664bu,
        0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
        0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au,
        0x5b9cca4fu, 0x682e6ff3u, 0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u,
        0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
    static_assert(MIX >= 4 && MIX <= 9, "pipe mix");
    uint32_t a = st[0], b = st[1], c = st[2], d = st[3];
    uint32_t e = st[4], f = st[5], g = st[6], h = st[7];
#pragma unroll
    for (int t = 0; t < 64; t++) {
        if (t >= 16) {
            const uint32_t x15 = w[(t - 15) & 15], x2 = w[(t - 2) & 15];
            uint32_t s0, s1;
            if constexpr (MIX == 8) {
                s0 = fma_ror<7>(x15) ^ ror32(x15, 18) ^ fma_shr<3>(x15);
                s1 = fma_ror<17>(x2) ^ ror32(x2, 19) ^ fma_shr<10>(x2);
            } else {
                s0 = ror32(x15, 7) ^ ror32(x15, 18) ^ (x15 >> 3);
                s1 = ror32(x2, 17) ^ ror32(x2, 19) ^ (x2 >> 10);
            }
            w[t & 15] = fma_add(s1, fma_add(s0, fma_add(w[t & 15], w[(t - 7) & 15])));
        }
        uint32_t S1, S0;
        if constexpr (MIX == 5 || MIX == 7 || MIX == 8) {
            S1 = fma_ror<6>(e) ^ ror32(e, 11) ^ ror32(e, 25);
            S0 = fma_ror<2>(a) ^ ror32(a, 13) ^ ror32(a, 22);
        } else if constexpr (MIX == 6) {
            S1 = fma_ror_wide<6>(e) ^ ror32(e, 11) ^ ror32(e, 25);
            S0 = fma_ror_wide<2>(a) ^ ror32(a, 13) ^ ror32(a, 22);
        } else if constexpr (MIX == 9) {
            S1 = fma_ror<6>(e) ^ fma_ror<11>(e) ^ fma_ror<25>(e);
            S0 = fma_ror<2>(a) ^ fma_ror<13>(a) ^ fma_ror<22>(a);
        } else {
            S1 = ror32(e, 6) ^ ror32(e, 11) ^ ror32(e, 25);
            S0 = ror32(a, 2) ^ ror32(a, 13) ^ ror32(a, 22);
        }
        const uint32_t ch = g ^ (e & (f ^ g));
        const uint32_t mj = (a & b) | (c & (a | b));
        uint32_t hkw;
        if constexpr (MIX == 7) {
            hkw = fma_add(h, fma_add(w[t & 15], K[t]));
        } else {
            hkw = h + K[t] + w[t & 15];
        }
        const uint32_t t1 = fma_add(ch, fma_add(S1, hkw));
        h = g; g = f; f = e; e = fma_add(d, t1);
        d = c; c = b; b = a; a = fma_add(S0, fma_add(mj, t1));
    }
    st[0] = fma_add(st[0], a); st[1] = fma_add(st[1], b); st[2] = fma_add(st[2], c); st[3] = fma_add(st[3], d);
    st[4] = fma_add(st[4], e); st[5] = fma_add(st[5], f); st[6] = fma_add(st[6], g); st[7] = fma_add(st[7], h);
}

template <int MIX>
__device__ __forceinline__ void sha256_compress_any(uint32_t (&st)[8], uint32_t (&w)[16])
{
    if constexpr (MIX >= 4) {
        sha256_compress_x<MIX>(st, w);
    } else {
        sha256_compress_t<MIX>(st, w);
    }
}

__device__ __forceinline__ void sha256_compress(uint32_t (&st)[8], uint32_t (&w)[16])
{
    sha256_compress_t<XB_SHA256_MIX>(st, w);
}

__device__ __forceinline__ void sha256_iv(uint32_t (&st)[8])
{
    st[0] = 0x6a09e667u; st[1] = 0xbb67ae85u; st[2] = 0x3c6ef372u; st[3] = 0xa54ff53au;
    st[4] = 0x510e527fu; st[5] = 0x9b05688cu; st[6] = 0x1f83d9abu; st[7] = 0x5be0cd19u;
}

// ---------------------------------------------------------------------------
// SHA-256 on state slots, for compressions that resume after a known prefix of
// rounds.  Role r (0 = a, ..., 7 = h) of round t lives in slot (r - t) & 7, so
// a round rewrites two slots and moves nothing, and the slots after any round
// can be stored and resumed from.  Round and schedule arithmetic are those of
// sha256_compress_t<MIX> (MIX 0, 1, 2).
// ---------------------------------------------------------------------------
__host__ __device__ constexpr uint32_t sha256_k(int t)
{
    constexpr uint32_t K[64] = {
        0x428a2f98u, 0x71374491u, 0xb5c0fbcfu, 0xe9b5dba5u, 0x3956c25bu, 0x59f111f1u,
        0x923f82a4u, 0xab1c5ed5u, 0xd807aa98u, 0x12835b01u, 0x243185beu, 0x550c7dc3u,
        0x72be5d74u, 0x80deb1feu, 0x9bdc06a7u, 0xc19bf174u, 0xe49b69c1u, 0xefbe4786u,
        0x0fc19dc6u, 0x240ca1ccu, 0x2de92c6fu, 0x4a7484aau, 0x5cb0a9dcu, 0x76f988dau,
        0x983e5152u, 0xa831c66du, 0xb00327c8u, 0xbf597fc7u, 0xc6e00bf3u, 0xd5a79147u,
        0x06ca6351u, 0x14292967u, 0x27b70a85u, 0x2e1b2138u, 0x4d2c6dfcu, 0x53380d13u,
        0x650a7354u, 0x766a0abbu, 0x81c2c92eu, 0x92722c85u, 0xa2bfe8a1u, 0xa81a664bu,
        0xc24b8b70u, 0xc76c51a3u, 0xd192e819u, 0xd6990624u, 0xf40e3585u, 0x106aa070u,
        0x19a4c116u, 0x1e376c08u, 0x2748774cu, 0x34b0bcb5u, 0x391c0cb3u, 0x4ed8aa4au,
        0x5b9cca4fu, 0x682e6ff3u, 0x748f82eeu, 0x78a5636fu, 0x84c87814u, 0x8cc70208u,
        0x90befffau, 0xa4506cebu, 0xbef9a3f7u, 0xc67178f2u};
    return K[t];
}

// W[t] for t >= 16 into the 16-word window (FIPS 180-4 6.2.2 step 1).
template <int MIX>
__device__ __forceinline__ void sha256_sched(uint32_t (&w)[16], int t)
{
    const uint32_t x15 = w[(t - 15) & 15], x2 = w[(t - 2) & 15];
    if constexpr (MIX == 0) {
        const uint32_t s0 = ror32(x15, 7) ^ ror32(x15, 18) ^ (x15 >> 3);
        const uint32_t s1 = ror32(x2, 17) ^ ror32(x2, 19) ^ (x2 >> 10);
        w[t & 15] += s0 + w[(t - 7) & 15] + s1;
    } else {
        const uint32_t r0 = (MIX == 2) ? fma_shr<3>(x15) : (x15 >> 3);
        const uint32_t r1 = (MIX == 2) ? fma_shr<10>(x2) : (x2 >> 10);
        const uint32_t s0 = ror32(x15, 7) ^ ror32(x15, 18) ^ r0;
        const uint32_t s1 = ror32(x2, 17) ^ ror32(x2, 19) ^ r1;
        w[t & 15] = fma_add(s1, fma_add(s0, w[t & 15] + w[(t - 7) & 15]));
    }
}

// Round t on slots (t must be a constant after unrolling).
template <int MIX>
__device__ __forceinline__ void sha256_round_s(uint32_t (&s)[8], int t, uint32_t wt)
{
    const uint32_t a = s[(0 - t) & 7], b = s[(1 - t) & 7], c = s[(2 - t) & 7];
    const uint32_t e = s[(4 - t) & 7], f = s[(5 - t) & 7], g = s[(6 - t) & 7];
    uint32_t& d = s[(3 - t) & 7];
    uint32_t& h = s[(7 - t) & 7];
    const uint32_t S1 = ror32(e, 6) ^ ror32(e, 11) ^ ror32(e, 25);
    const uint32_t ch = g ^ (e & (f ^ g));
    const uint32_t S0 = ror32(a, 2) ^ ror32(a, 13) ^ ror32(a, 22);
    const uint32_t mj = (a & b) | (c & (a | b));
    if constexpr (MIX == 0) {
        const uint32_t t1 = h + S1 + ch + sha256_k(t) + wt;
        d += t1;
        h = t1 + S0 + mj;
    } else {
        const uint32_t t1 = fma_add(ch, fma_add(S1, h + sha256_k(t) + wt));
        d = fma_add(d, t1);
        h = fma_add(S0, fma_add(mj, t1));
    }
}

// The slots after rounds 0..7 from the IV with W0..W7 = 0: the first block of
// every hash whose input starts with toByte(0, 32) (thash_f's core block).
struct Sha256Slots {
    uint32_t v[8];
};
__host__ __device__ constexpr uint32_t sha256_ror_c(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }
__host__ __device__ constexpr Sha256Slots sha256_zero_prefix8()
{
    Sha256Slots s{{0x6a09e667u, 0xbb67ae85u, 0x3c6ef372u, 0xa54ff53au, 0x510e527fu, 0x9b05688cu, 0x1f83d9abu,
                   0x5be0cd19u}};
    for (int t = 0; t < 8; t++) {
        const uint32_t a = s.v[(0 - t) & 7], b = s.v[(1 - t) & 7], c = s.v[(2 - t) & 7];
        const uint32_t e = s.v[(4 - t) & 7], f = s.v[(5 - t) & 7], g = s.v[(6 - t) & 7];
        const uint32_t S1 = sha256_ror_c(e, 6) ^ sha256_ror_c(e, 11) ^ sha256_ror_c(e, 25);
        const uint32_t S0 = sha256_ror_c(a, 2) ^ sha256_ror_c(a, 13) ^ sha256_ror_c(a, 22);
        const uint32_t t1 = s.v[(7 - t) & 7] + S1 + (g ^ (e & (f ^ g))) + sha256_k(t);
        s.v[(3 - t) & 7] += t1;
        s.v[(7 - t) & 7] = t1 + S0 + ((a & b) | (c & (a | b)));
    }
    return s;
}

// A 32-bit shared-memory load the compiler keeps where it is written (not
// hoisted out of a loop into registers that would stay live across it).
__device__ __forceinline__ uint32_t lds_u32(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"((uint32_t)__cvta_generic_to_shared(p)));
    return v;
}

// The rounds of one compression resumed from slots s; on return s holds the
// final slots and the caller adds its chaining value (the feed-forward):
//   skip 0  s = the chaining value, rounds 0..63;
//   skip 6  s = the slots after rounds 0..5, and the shared-memory words
//           pre[0], pre[stride], ..., pre[4 * stride] = W16..W20 (which read
//           only W0..W5 and W9..W15);
//   skip 8  s = the slots after rounds 0..7 (w[0..7] still hold W0..W7).
// `skip` must be the same for every thread of a warp (a branch, not a select).
template <int MIX>
__device__ __forceinline__ void sha256_rounds_resume(uint32_t (&s)[8], uint32_t (&w)[16], int skip,
                                                     const uint32_t* pre, int stride)
{
    if (skip == 0) {
#pragma unroll
        for (int t = 0; t < 6; t++) sha256_round_s<MIX>(s, t, w[t]);
    }
    if (skip != 8) {
#pragma unroll
        for (int t = 6; t < 8; t++) sha256_round_s<MIX>(s, t, w[t]);
    }
#pragma unroll
    for (int t = 8; t < 16; t++) sha256_round_s<MIX>(s, t, w[t]);
    if (skip == 6) {
#pragma unroll
        for (int t = 16; t < 21; t++) w[t & 15] = lds_u32(pre + (t - 16) * stride);
    } else {
#pragma unroll
        for (int t = 16; t < 21; t++) sha256_sched<MIX>(w, t);
    }
#pragma unroll
    for (int t = 16; t < 21; t++) sha256_round_s<MIX>(s, t, w[t & 15]);
#pragma unroll
    for (int t = 21; t < 64; t++) {
        sha256_sched<MIX>(w, t);
        sha256_round_s<MIX>(s, t, w[t & 15]);
    }
}

// SHA-256 of a message of MW big-endian words (4*MW bytes), from the IV.
template <int MW>
__device__ __forceinline__ void sha256_words(uint32_t (&out)[8], const uint32_t (&m)[MW])
{
    constexpr int NB = (MW * 4 + 9 + 63) / 64;
    uint32_t st[8];
    sha256_iv(st);
#pragma unroll
    for (int b = 0; b < NB; b++) {
        uint32_t w[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int k = 16 * b + j;
            w[j] = (k < MW) ? m[k < MW ? k : 0] : (k == MW ? 0x80000000u : 0u);
        }
        if (b == NB - 1) {
            w[14] = 0;
            w[15] = (uint32_t)(MW * 32);
        }
        sha256_compress(st, w);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = st[i];
}

// ---------------------------------------------------------------------------
// SHA-512 compression (FIPS 180-4 6.4.2).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t ror64(uint64_t x, int n) { return (x >> n) | (x << (64 - n)); }

// Round constants in constant memory: the rounds after the first 16 run as
// a loop over 16-round blocks (see sha512_compress).
static __constant__ uint64_t kSha512K[80] = {
        0x428a2f98d728ae22ull, 0x7137449123ef65cdull, 0xb5c0fbcfec4d3b2full, 0xe9b5dba58189dbbcull,
        0x3956c25bf348b538ull, 0x59f111f1b605d019ull, 0x923f82a4af194f9bull, 0xab1c5ed5da6d8118ull,
        0xd807aa98a3030242ull, 0x12835b0145706fbeull, 0x243185be4ee4b28cull, 0x550c7dc3d5ffb4e2ull,
        0x72be5d74f27b896full, 0x80deb1fe3b1696b1ull, 0x9bdc06a725c71235ull, 0xc19bf174cf692694ull,
        0xe49b69c19ef14ad2ull, 0xefbe4786384f25e3ull, 0x0fc19dc68b8cd5b5ull, 0x240ca1cc77ac9c65ull,
        0x2de92c6f592b0275ull, 0x4a7484aa6ea6e483ull, 0x5cb0a9dcbd41fbd4ull, 0x76f988da831153b5ull,
        0x983e5152ee66dfabull, 0xa831c66d2db43210ull, 0xb00327c898fb213full, 0xbf597fc7beef0ee4ull,
        0xc6e00bf33da88fc2ull, 0xd5a79147930aa725ull, 0x06ca6351e003826full, 0x142929670a0e6e70ull,
        0x27b70a8546d22ffcull, 0x2e1b21385c26c926ull, 0x4d2c6dfc5ac42aedull, 0x53380d139d95b3dfull,
        0x650a73548baf63deull, 0x766a0abb3c77b2a8ull, 0x81c2c92e47edaee6ull, 0x92722c851482353bull,
        0xa2bfe8a14cf10364ull, 0xa81a664bbc423001ull, 0xc24b8b70d0f89791ull, 0xc76c51a30654be30ull,
        0xd192e819d6ef5218ull, 0xd69906245565a910ull, 0xf40e35855771202aull, 0x106aa07032bbd1b8ull,
        0x19a4c116b8d2d0c8ull, 0x1e376c085141ab53ull, 0x2748774cdf8eeb99ull, 0x34b0bcb5e19b48a8ull,
        0x391c0cb3c5c95a63ull, 0x4ed8aa4ae3418acbull, 0x5b9cca4f7763e373ull, 0x682e6ff3d6b2b8a3ull,
        0x748f82ee5defb2fcull, 0x78a5636f43172f60ull, 0x84c87814a1f0ab72ull, 0x8cc702081a6439ecull,
        0x90befffa23631e28ull, 0xa4506cebde82bde9ull, 0xbef9a3f7b2c67915ull, 0xc67178f2e372532bull,
        0xca273eceea26619cull, 0xd186b8c721c0c207ull, 0xeada7dd6cde0eb1eull, 0xf57d4f7fee6ed178ull,
        0x06f067aa72176fbaull, 0x0a637dc5a2c898a6ull, 0x113f9804bef90daeull, 0x1b710b35131c471bull,
        0x28db77f523047d84ull, 0x32caab7b40c72493ull, 0x3c9ebe0a15c9bebcull, 0x431d67c49c100d4cull,
        0x4cc5d4becb3e42b6ull, 0x597f299cfc657e2aull, 0x5fcb6fab3ad6faecull, 0x6c44198c4a475817ull};

// One round on the state v[8] whose roles rotate: at round j, a is
// v[(8 - j) & 7] ... h is v[(15 - j) & 7]; j is a compile-time constant once
// the caller's loop is unrolled, so v stays in registers.
__device__ __forceinline__ void sha512_round(uint64_t (&v)[8], int j, uint64_t k, uint64_t wj)
{
    const uint64_t a = v[(8 - j) & 7], b = v[(9 - j) & 7], c = v[(10 - j) & 7];
    const uint64_t e = v[(12 - j) & 7], f = v[(13 - j) & 7], g = v[(14 - j) & 7];
    const uint64_t S1 = ror64(e, 14) ^ ror64(e, 18) ^ ror64(e, 41);
    const uint64_t ch = g ^ (e & (f ^ g));
    const uint64_t t1 = v[(15 - j) & 7] + S1 + ch + k + wj;
    const uint64_t S0 = ror64(a, 28) ^ ror64(a, 34) ^ ror64(a, 39);
    const uint64_t mj = (a & b) | (c & (a | b));
    v[(11 - j) & 7] += t1;           // d + t1 is the next round's e
    v[(15 - j) & 7] = t1 + S0 + mj;  // the slot of h holds the next round's a
}

// FIPS 180-4 6.4.2.  The first 16 rounds take the message words as they
// are; rounds 16..79 run as four passes of one unrolled 16-round block that
// extends the schedule in place (16 is a multiple of 8, so the state roles
// line up from pass to pass).  The rolled form keeps a kernel's SHA-512 code
// small: fully unrolled, the four compressions of an F call did not stay in
// the instruction cache (instruction fetch was the top stall).
__device__ __forceinline__ void sha512_compress(uint64_t (&st)[8], uint64_t (&w)[16])
{
    uint64_t v[8];
#pragma unroll
    for (int i = 0; i < 8; i++) v[i] = st[i];
#pragma unroll
    for (int j = 0; j < 16; j++) sha512_round(v, j, kSha512K[j], w[j]);
#pragma unroll 1
    for (int r = 16; r < 80; r += 16) {
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const uint64_t x15 = w[(j + 1) & 15], x2 = w[(j + 14) & 15];
            const uint64_t s0 = ror64(x15, 1) ^ ror64(x15, 8) ^ (x15 >> 7);
            const uint64_t s1 = ror64(x2, 19) ^ ror64(x2, 61) ^ (x2 >> 6);
            w[j] += s0 + w[(j + 9) & 15] + s1;
            sha512_round(v, j, kSha512K[r + j], w[j]);
        }
    }
#pragma unroll
    for (int i = 0; i < 8; i++) st[i] += v[i];
}

__device__ __forceinline__ void sha512_iv(uint64_t (&st)[8])
{
    st[0] = 0x6a09e667f3bcc908ull; st[1] = 0xbb67ae8584caa73bull;
    st[2] = 0x3c6ef372fe94f82bull; st[3] = 0xa54ff53a5f1d36f1ull;
    st[4] = 0x510e527fade682d1ull; st[5] = 0x9b05688c2b3e6c1full;
    st[6] = 0x1f83d9abfb41bd6bull; st[7] = 0x5be0cd19137e2179ull;
}

__device__ __forceinline__ uint64_t join64(uint32_t hi, uint32_t lo)
{
    return ((uint64_t)hi << 32) | lo;
}

// SHA-512 of a message of MW big-endian 32-bit words (MW even), from the IV;
// out holds 16 big-endian 32-bit words.
template <int MW>
__device__ __forceinline__ void sha512_words(uint32_t (&out)[16], const uint32_t (&m)[MW])
{
    static_assert(MW % 2 == 0, "SHA-512 messages here are whole 64-bit words");
    constexpr int MQ = MW / 2;
    constexpr int NB = (MW * 4 + 17 + 127) / 128;
    uint64_t st[8];
    sha512_iv(st);
#pragma unroll
    for (int b = 0; b < NB; b++) {
        uint64_t w[16];
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int k = 16 * b + j;
            w[j] = (k < MQ) ? join64(m[2 * (k < MQ ? k : 0)], m[2 * (k < MQ ? k : 0) + 1])
                            : (k == MQ ? 0x8000000000000000ull : 0ull);
        }
        if (b == NB - 1) {
            w[14] = 0;
            w[15] = (uint64_t)MW * 32;
        }
        sha512_compress(st, w);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
        out[2 * i] = (uint32_t)(st[i] >> 32);
        out[2 * i + 1] = (uint32_t)st[i];
    }
}

// ---------------------------------------------------------------------------
// Keccak-f[1600] (FIPS 202 3.2-3.3).  Lane A[x + 5y].
// ---------------------------------------------------------------------------
template <int N>
__device__ __forceinline__ uint64_t rol64c(uint64_t x)
{
    if constexpr (N == 0) {
        return x;
    } else {
        return (x << N) | (x >> (64 - N));
    }
}

// rho offsets r[x + 5y] (FIPS 202 Algorithm 2)
template <int I>
struct KeccakRho {
    static constexpr int tbl[25] = {0,  1,  62, 28, 27, 36, 44, 6,  55, 20, 3,  10, 43,
                                    25, 39, 41, 45, 15, 21, 8,  18, 2,  61, 56, 14};
    static constexpr int value = tbl[I];
};

template <int I>
__device__ __forceinline__ void keccak_rho_pi(uint64_t (&B)[25], const uint64_t (&A)[25],
                                              const uint64_t (&D)[5])
{
    constexpr int x = I % 5, y = I / 5;
    constexpr int dst = y + 5 * ((2 * x + 3 * y) % 5);
    B[dst] = rol64c<KeccakRho<I>::value>(A[I] ^ D[x]);
    if constexpr (I + 1 < 25) keccak_rho_pi<I + 1>(B, A, D);
}

__device__ __forceinline__ void keccak_f1600(uint64_t (&A)[25])
{
    const uint64_t RC[24] = {
        0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808aull, 0x8000000080008000ull,
        0x000000000000808bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
        0x000000000000008aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000aull,
        0x000000008000808bull, 0x800000000000008bull, 0x8000000000008089ull, 0x8000000000008003ull,
        0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800aull, 0x800000008000000aull,
        0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};
#pragma unroll
    for (int r = 0; r < 24; r++) {
        uint64_t C[5], D[5], B[25];
#pragma unroll
        for (int x = 0; x < 5; x++) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
#pragma unroll
        for (int x = 0; x < 5; x++) D[x] = C[(x + 4) % 5] ^ rol64c<1>(C[(x + 1) % 5]);
        keccak_rho_pi<0>(B, A, D);
#pragma unroll
        for (int y = 0; y < 5; y++) {
#pragma unroll
            for (int x = 0; x < 5; x++) {
                A[x + 5 * y] = B[x + 5 * y] ^ (~B[(x + 1) % 5 + 5 * y] & B[(x + 2) % 5 + 5 * y]);
            }
        }
        A[0] ^= RC[r];
    }
}

// Round constants for the partly rolled permutation below.
static __constant__ uint64_t kKeccakRC[24] = {
    0x0000000000000001ull, 0x0000000000008082ull, 0x800000000000808aull, 0x8000000080008000ull,
    0x000000000000808bull, 0x0000000080000001ull, 0x8000000080008081ull, 0x8000000000008009ull,
    0x000000000000008aull, 0x0000000000000088ull, 0x0000000080008009ull, 0x000000008000000aull,
    0x000000008000808bull, 0x800000000000008bull, 0x8000000000008089ull, 0x8000000000008003ull,
    0x8000000000008002ull, 0x8000000000000080ull, 0x000000000000800aull, 0x800000008000000aull,
    0x8000000080008081ull, 0x8000000000008080ull, 0x0000000080000001ull, 0x8000000080008008ull};

// Keccak-f[1600] with U rounds per loop pass (U divides 24): the form for
// the throughput-bound chain kernels, whose fully unrolled F call (three
// permutations) does not stay in the instruction cache.  The serial H_msg
// keeps keccak_f1600: rolling measured 1.5x its latency.
template <int U>
__device__ __forceinline__ void keccak_f1600_u(uint64_t (&A)[25])
{
    static_assert(24 % U == 0, "U must divide 24");
#pragma unroll 1
    for (int r = 0; r < 24; r += U) {
#pragma unroll
        for (int q = 0; q < U; q++) {
            uint64_t C[5], D[5], B[25];
#pragma unroll
            for (int x = 0; x < 5; x++) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
#pragma unroll
            for (int x = 0; x < 5; x++) D[x] = C[(x + 4) % 5] ^ rol64c<1>(C[(x + 1) % 5]);
            keccak_rho_pi<0>(B, A, D);
#pragma unroll
            for (int y = 0; y < 5; y++) {
#pragma unroll
                for (int x = 0; x < 5; x++) {
                    A[x + 5 * y] = B[x + 5 * y] ^ (~B[(x + 1) % 5 + 5 * y] & B[(x + 2) % 5 + 5 * y]);
                }
            }
            A[0] ^= kKeccakRC[r + q];
        }
    }
}

// Keccak-f[1600] spread over a warp: lane t < 25 holds state lane
// A[t] = A[x + 5y] (x = t % 5, y = t / 5) as two 32-bit halves; lanes 25-31
// carry zeros and take part in the shuffles.  One round is the FIPS 202
// step mappings with the state exchanged by shuffles:
//   theta  every lane gathers its column (4 shuffles), then the parities of
//          columns x - 1 and x + 1 of its own row (2 shuffles);
//   rho    a rotation by the lane's own offset;
//   pi     a gather: lane (X, Y) takes lane (x, X) with 2x + 3X = Y (mod 5);
//   chi    the lanes x + 1 and x + 2 of the row (2 shuffles);
//   iota   lane 0.
// A serial chain of permutations (H_msg of a long message) runs ~4x faster
// this way than in one thread, whose fully unrolled permutation does not fit
// the instruction cache; the thread form stays the throughput form.
struct KeccakWarpLane {
    uint32_t col[4];    // lanes of the own column, other rows
    uint32_t xm, xp;    // lanes x - 1 and x + 1 of the own row
    uint32_t pi_src;    // source lane of the pi gather
    uint32_t c1, c2;    // lanes x + 1 and x + 2 of the own row (chi)
    uint32_t rot;       // rho offset mod 32
    bool swap;          // rho offset >= 32
    __device__ __forceinline__ KeccakWarpLane()
    {
        constexpr uint8_t kRho[25] = {0,  1,  62, 28, 27, 36, 44, 6,  55, 20, 3,  10, 43,
                                      25, 39, 41, 45, 15, 21, 8,  18, 2,  61, 56, 14};
        const uint32_t t = threadIdx.x & 31, tt = t < 25 ? t : 0;
        const uint32_t x = tt % 5, y = tt / 5;
#pragma unroll
        for (int k = 1; k <= 4; k++) col[k - 1] = x + 5 * ((y + k) % 5);
        xm = (x + 4) % 5 + 5 * y;
        xp = (x + 1) % 5 + 5 * y;
        // pi: the lane at (X, Y) = (x, y) here receives lane (x', X) with
        // 2x' + 3X = Y (mod 5), i.e. x' = 3 (Y - 3X) mod 5
        const uint32_t xs = (3 * ((y + 5 * 3 - 3 * x) % 5)) % 5;
        pi_src = xs + 5 * x;
        c1 = (x + 1) % 5 + 5 * y;
        c2 = (x + 2) % 5 + 5 * y;
        uint32_t r = 0;
#pragma unroll
        for (int i = 0; i < 25; i++)
            if ((uint32_t)i == tt) r = kRho[i];
        swap = r >= 32;
        rot = r & 31;
    }
};

__device__ __forceinline__ void rotl64_pair(uint32_t& lo, uint32_t& hi, uint32_t n)
{
    const uint32_t l = __funnelshift_l(hi, lo, n), h = __funnelshift_l(lo, hi, n);
    lo = l;
    hi = h;
}

__device__ __forceinline__ void keccak_f1600_warp(uint32_t& lo, uint32_t& hi, const KeccakWarpLane& k)
{
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll 1
    for (int r = 0; r < 24; r++) {
        // theta
        uint32_t cl = lo, ch = hi;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            cl ^= __shfl_sync(0xffffffffu, lo, k.col[i]);
            ch ^= __shfl_sync(0xffffffffu, hi, k.col[i]);
        }
        const uint32_t ml = __shfl_sync(0xffffffffu, cl, k.xm), mh = __shfl_sync(0xffffffffu, ch, k.xm);
        uint32_t pl = __shfl_sync(0xffffffffu, cl, k.xp), ph = __shfl_sync(0xffffffffu, ch, k.xp);
        rotl64_pair(pl, ph, 1);
        lo ^= ml ^ pl;
        hi ^= mh ^ ph;
        // rho (own offset), then pi (gather)
        if (k.swap) {
            const uint32_t t = lo;
            lo = hi;
            hi = t;
        }
        rotl64_pair(lo, hi, k.rot);
        const uint32_t bl = __shfl_sync(0xffffffffu, lo, k.pi_src), bh = __shfl_sync(0xffffffffu, hi, k.pi_src);
        // chi
        const uint32_t b1l = __shfl_sync(0xffffffffu, bl, k.c1), b1h = __shfl_sync(0xffffffffu, bh, k.c1);
        const uint32_t b2l = __shfl_sync(0xffffffffu, bl, k.c2), b2h = __shfl_sync(0xffffffffu, bh, k.c2);
        lo = bl ^ (~b1l & b2l);
        hi = bh ^ (~b1h & b2h);
        // iota
        if (lane == 0) {
            const uint64_t rc = kKeccakRC[r];
            lo ^= (uint32_t)rc;
            hi ^= (uint32_t)(rc >> 32);
        }
        if (lane >= 25) lo = hi = 0;
    }
}

// SHAKE with rate RATEW 32-bit words (42 = SHAKE128, 34 = SHAKE256) over a
// message of MW little-endian words; writes the first OUTW output words.
// U < 24: the permutation runs U rounds per loop pass (keccak_f1600_u).
template <int RATEW, int MW, int OUTW, int U = 24>
__device__ __forceinline__ void shake_words(uint32_t (&out)[OUTW], const uint32_t (&m)[MW])
{
    static_assert(OUTW <= RATEW, "output fits in one squeeze block");
    constexpr int NB = (MW * 4) / (RATEW * 4) + 1;  // absorbed blocks incl. padding
    uint64_t A[25];
#pragma unroll
    for (int i = 0; i < 25; i++) A[i] = 0;
#pragma unroll
    for (int b = 0; b < NB; b++) {
#pragma unroll
        for (int i = 0; i < RATEW / 2; i++) {
            uint32_t lo = 0, hi = 0;
            const int k0 = b * RATEW + 2 * i, k1 = k0 + 1;
            if (k0 < MW) lo = m[k0 < MW ? k0 : 0];
            else if (k0 == MW) lo = 0x1Fu;
            if (k1 < MW) hi = m[k1 < MW ? k1 : 0];
            else if (k1 == MW) hi = 0x1Fu;
            if (b == NB - 1 && 2 * i + 1 == RATEW - 1) hi ^= 0x80000000u;
            A[i] ^= ((uint64_t)hi << 32) | lo;
        }
        if constexpr (U < 24) {
            keccak_f1600_u<U>(A);
        } else {
            keccak_f1600(A);
        }
    }
#pragma unroll
    for (int i = 0; i < OUTW; i++) out[i] = (i & 1) ? (uint32_t)(A[i / 2] >> 32) : (uint32_t)A[i / 2];
}

}  // namespace xb
