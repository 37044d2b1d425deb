// Tweakable hash families of XMSS (the reference's hash.c), one struct per
// (hash function, n) pair that the parameter tables can select
// (cuxmss/hash.c:29-65 core_hash dispatch):
//
//   Sha256N32   SHA-256,        n = 32, padding_len = 32   (midstate form)
//   Sha512N64   SHA-512,        n = 64, padding_len = 64   (midstate form)
//   Sha256N24   SHA-256 / 24 B, n = 24, padding_len = 4
//   Shake128N32 SHAKE128,       n = 32, padding_len = 32
//   Shake256N24 / N32 / N64     SHAKE256, padding_len = 4 / 32 / 64
//
// Every family exposes the same interface over n-byte values held as NW
// 32-bit words in the family's message-word order (big-endian words for
// SHA-2, little-endian words for Keccak):
//   Ctx                 per-key precomputation (seeds, midstates)
//   make_ctx            builds it from PUB_SEED, SK_SEED, SK_PRF
//   load / store        bytes <-> words
//   thash_f, thash_h    hash.c:157-183, 125-155 (ADRS word 7 is overwritten)
//   prf_keygen          hash.c:87-98 with in = PUB_SEED || ADRS
//   prf_r               hash.c:70-81 with key = SK_PRF, in = toByte(idx, 32)
//   hmsg                hash.c:107-120 over a message in global memory
//   byte_at             byte k of an n-byte value (for base_w)
//   HPre, h_pre, h_fin  thash_h split in two: h_pre is the part that depends
//                       only on the address (the three PRFs, and for the
//                       midstate forms the first core block toByte(1)||key);
//                       h_fin finishes the hash from (l, r).  Verify computes
//                       every h_pre of a signature in parallel up front, so
//                       the serial L-tree / authentication-path steps cost
//                       h_fin only (2 compressions instead of 6 for SHA-2).
//
// For the SHA-2 sets with padding_len = n the first block of PRF, PRF_keygen
// and the R-PRF is toByte(X, n) || key and is constant per key, so its
// compression is done once per key ("midstate"); F then costs 4 and H 6
// compressions instead of 6 and 9.
#pragma once

#include <cstdint>
#include <type_traits>

#include "hashcore.cuh"

namespace xb {

// ---------------------------------------------------------------------------
// Byte access helpers.
// ---------------------------------------------------------------------------

// Four message bytes starting at offset o (zero past mlen), packed
// little-endian (byte o in bits 0..7).  Uses two aligned word loads when the
// whole aligned pair lies inside [m, m + mlen); callers guarantee that the
// 3 bytes before m are readable (m is 4-byte aligned, or preceded by the
// signature in an sm buffer).
__device__ __forceinline__ uint32_t fetch4_le(const uint8_t* m, uint64_t mlen, uint64_t o)
{
    if (o + 8 <= mlen) {
        const uintptr_t addr = (uintptr_t)(m + o);
        const uint32_t* a = (const uint32_t*)(addr & ~(uintptr_t)3);
        const int sh = (int)(addr & 3) * 8;
        const uint32_t lo = __ldg(a);
        if (!sh) return lo;
        return __funnelshift_r(lo, __ldg(a + 1), sh);
    }
    uint32_t v = 0;
#pragma unroll
    for (int i = 0; i < 4; i++)
        if (o + i < mlen) v |= (uint32_t)__ldg(m + o + i) << (8 * i);
    return v;
}

// NW little-endian words from bytes at p (any alignment; 16-byte vector
// loads where p is 16-byte aligned, as n-byte nodes of the node arrays are).
template <int NW>
__device__ __forceinline__ void load_le(uint32_t (&v)[NW], const uint8_t* p)
{
    if constexpr (NW % 4 == 0) {
        if (((uintptr_t)p & 15) == 0) {
#pragma unroll
            for (int i = 0; i < NW; i += 4) {
                const uint4 q = *(const uint4*)(p + 4 * i);
                v[i] = q.x;
                v[i + 1] = q.y;
                v[i + 2] = q.z;
                v[i + 3] = q.w;
            }
            return;
        }
    }
    if (((uintptr_t)p & 3) == 0) {
#pragma unroll
        for (int i = 0; i < NW; i++) v[i] = ((const uint32_t*)p)[i];
    } else {
#pragma unroll
        for (int i = 0; i < NW; i++)
            v[i] = (uint32_t)p[4 * i] | ((uint32_t)p[4 * i + 1] << 8) |
                   ((uint32_t)p[4 * i + 2] << 16) | ((uint32_t)p[4 * i + 3] << 24);
    }
}

template <int NW>
__device__ __forceinline__ void store_le(uint8_t* p, const uint32_t (&v)[NW])
{
    if (((uintptr_t)p & 15) == 0 && NW % 4 == 0) {
#pragma unroll
        for (int i = 0; i < NW; i += 4)
            *(uint4*)(p + 4 * i) = make_uint4(v[i], v[i + 1], v[i + 2], v[i + 3]);
    } else if (((uintptr_t)p & 3) == 0) {
#pragma unroll
        for (int i = 0; i < NW; i++) ((uint32_t*)p)[i] = v[i];
    } else {
#pragma unroll
        for (int i = 0; i < NW; i++) {
            p[4 * i] = (uint8_t)v[i];
            p[4 * i + 1] = (uint8_t)(v[i] >> 8);
            p[4 * i + 2] = (uint8_t)(v[i] >> 16);
            p[4 * i + 3] = (uint8_t)(v[i] >> 24);
        }
    }
}

// ---------------------------------------------------------------------------
// Shared pieces of every family.
// ---------------------------------------------------------------------------
template <int N_, int PL_, bool BE_>
struct FamBase {
    static constexpr int N = N_;
    static constexpr int NW = N_ / 4;
    static constexpr int PL = PL_;   // padding_len
    static constexpr int PW = PL_ / 4;
    static constexpr int LEN1 = 2 * N_;  // w = 16
    static constexpr int LEN2 = 3;
    static constexpr int LEN = LEN1 + LEN2;
    static constexpr bool BE = BE_;

    // Message word for a big-endian u32 value (ADRS words, toByte fields).
    __device__ __forceinline__ static uint32_t mw(uint32_t x) { return BE ? x : bswap32(x); }

    __device__ __forceinline__ static void load(uint32_t (&v)[NW], const uint8_t* p)
    {
        load_le<NW>(v, p);
        if (BE) {
#pragma unroll
            for (int i = 0; i < NW; i++) v[i] = bswap32(v[i]);
        }
    }
    __device__ __forceinline__ static void store(uint8_t* p, const uint32_t (&v)[NW])
    {
        if (BE) {
            uint32_t t[NW];
#pragma unroll
            for (int i = 0; i < NW; i++) t[i] = bswap32(v[i]);
            store_le<NW>(p, t);
        } else {
            store_le<NW>(p, v);
        }
    }
    __device__ __forceinline__ static uint32_t byte_at(const uint32_t (&v)[NW], int k)
    {
        const uint32_t w = v[k >> 2];
        return BE ? (w >> (24 - 8 * (k & 3))) & 0xFF : (w >> (8 * (k & 3))) & 0xFF;
    }
};

// ---------------------------------------------------------------------------
// Generic family: every call hashes an explicit word message with core().
// ---------------------------------------------------------------------------
template <class Core, int N_, int PL_>
struct GenericFam : FamBase<N_, PL_, Core::BE> {
    using B = FamBase<N_, PL_, Core::BE>;
    using B::mw;
    static constexpr int NW = B::NW, PW = B::PW;

    struct Ctx {
        uint32_t pub[NW];
        uint32_t sks[NW];
        uint32_t skp[NW];
    };

    __device__ static void make_ctx(Ctx& c, const uint8_t* pub, const uint8_t* sks, const uint8_t* skp)
    {
        B::load(c.pub, pub);
#pragma unroll
        for (int i = 0; i < NW; i++) c.sks[i] = c.skp[i] = 0;
        if (sks) B::load(c.sks, sks);
        if (skp) B::load(c.skp, skp);
    }

    template <int MW>
    __device__ __forceinline__ static void set_pad(uint32_t (&m)[MW], uint32_t x)
    {
#pragma unroll
        for (int i = 0; i < PW - 1; i++) m[i] = 0;
        m[PW - 1] = mw(x);
    }

    // PRF(PUB_SEED, ADRS), hash.c:70-81
    __device__ __forceinline__ static void prf_adrs(uint32_t (&out)[NW], const Ctx& c, const uint32_t (&a)[8])
    {
        uint32_t m[PW + NW + 8];
        set_pad(m, 3);
#pragma unroll
        for (int i = 0; i < NW; i++) m[PW + i] = c.pub[i];
#pragma unroll
        for (int i = 0; i < 8; i++) m[PW + NW + i] = mw(a[i]);
        Core::template digest<PW + NW + 8, NW>(out, m);
    }

    __device__ static void thash_f(uint32_t (&x)[NW], const Ctx& c, uint32_t (&a)[8])
    {
        uint32_t m[PW + 2 * NW], mask[NW], key[NW];
        a[7] = 0;
        prf_adrs(key, c, a);
        a[7] = 1;
        prf_adrs(mask, c, a);
        set_pad(m, 0);
#pragma unroll
        for (int i = 0; i < NW; i++) {
            m[PW + i] = key[i];
            m[PW + NW + i] = x[i] ^ mask[i];
        }
        Core::template digest<PW + 2 * NW, NW>(x, m);
    }

    __device__ static void thash_h(uint32_t (&o)[NW], const uint32_t (&l)[NW], const uint32_t (&r)[NW],
                                   const Ctx& c, uint32_t (&a)[8])
    {
        uint32_t m[PW + 3 * NW], t[NW];
        set_pad(m, 1);
        a[7] = 0;
        prf_adrs(t, c, a);
#pragma unroll
        for (int i = 0; i < NW; i++) m[PW + i] = t[i];
        a[7] = 1;
        prf_adrs(t, c, a);
#pragma unroll
        for (int i = 0; i < NW; i++) m[PW + NW + i] = l[i] ^ t[i];
        a[7] = 2;
        prf_adrs(t, c, a);
#pragma unroll
        for (int i = 0; i < NW; i++) m[PW + 2 * NW + i] = r[i] ^ t[i];
        Core::template digest<PW + 3 * NW, NW>(o, m);
    }

    struct HPre {
        uint32_t key[NW];
        uint32_t m1[NW];
        uint32_t m2[NW];
    };

    __device__ static void h_pre(HPre& o, const Ctx& c, uint32_t (&a)[8])
    {
        a[7] = 0;
        prf_adrs(o.key, c, a);
        a[7] = 1;
        prf_adrs(o.m1, c, a);
        a[7] = 2;
        prf_adrs(o.m2, c, a);
    }

    __device__ static void h_fin(uint32_t (&o)[NW], const HPre& p, const uint32_t (&l)[NW], const uint32_t (&r)[NW])
    {
        uint32_t m[PW + 3 * NW];
        set_pad(m, 1);
#pragma unroll
        for (int i = 0; i < NW; i++) {
            m[PW + i] = p.key[i];
            m[PW + NW + i] = l[i] ^ p.m1[i];
            m[PW + 2 * NW + i] = r[i] ^ p.m2[i];
        }
        Core::template digest<PW + 3 * NW, NW>(o, m);
    }

    __device__ static void prf_keygen(uint32_t (&o)[NW], const Ctx& c, const uint32_t (&a)[8])
    {
        uint32_t m[PW + 2 * NW + 8];
        set_pad(m, 4);
#pragma unroll
        for (int i = 0; i < NW; i++) {
            m[PW + i] = c.sks[i];
            m[PW + NW + i] = c.pub[i];
        }
#pragma unroll
        for (int i = 0; i < 8; i++) m[PW + 2 * NW + i] = mw(a[i]);
        Core::template digest<PW + 2 * NW + 8, NW>(o, m);
    }

    __device__ static void prf_r(uint32_t (&o)[NW], const Ctx& c, uint64_t idx)
    {
        uint32_t m[PW + NW + 8];
        set_pad(m, 3);
#pragma unroll
        for (int i = 0; i < NW; i++) m[PW + i] = c.skp[i];
#pragma unroll
        for (int i = 0; i < 6; i++) m[PW + NW + i] = 0;
        m[PW + NW + 6] = mw((uint32_t)(idx >> 32));
        m[PW + NW + 7] = mw((uint32_t)idx);
        Core::template digest<PW + NW + 8, NW>(o, m);
    }
};

// ---------------------------------------------------------------------------
// Core hash adaptors for GenericFam.
// ---------------------------------------------------------------------------
struct CoreSha256 {
    static constexpr bool BE = true;
    template <int MW, int OW>
    __device__ __forceinline__ static void digest(uint32_t (&out)[OW], const uint32_t (&m)[MW])
    {
        uint32_t full[8];
        sha256_words<MW>(full, m);
#pragma unroll
        for (int i = 0; i < OW; i++) out[i] = full[i];  // n = 24 truncates (hash.c:35-38)
    }
};

// ROLL < 24: the permutation runs ROLL rounds per loop pass (chain kernels).
template <int RATEW, int ROLL = 24>
struct CoreShake {
    static constexpr bool BE = false;
    template <int MW, int OW>
    __device__ __forceinline__ static void digest(uint32_t (&out)[OW], const uint32_t (&m)[MW])
    {
        shake_words<RATEW, MW, OW, ROLL>(out, m);
    }
};

using Sha256N24 = GenericFam<CoreSha256, 24, 4>;
using Shake128N32 = GenericFam<CoreShake<42>, 32, 32>;
using Shake256N24 = GenericFam<CoreShake<34>, 24, 4>;
using Shake256N32 = GenericFam<CoreShake<34>, 32, 32>;
using Shake256N64 = GenericFam<CoreShake<34>, 64, 64>;

// The chain kernels' form of the SHAKE families (same key context): the
// permutation partly rolled, so that their F calls fit the instruction cache.
#ifndef XB_KECCAK_CHAIN_ROLL
#define XB_KECCAK_CHAIN_ROLL 4
#endif
using Shake128N32Chain = GenericFam<CoreShake<42, XB_KECCAK_CHAIN_ROLL>, 32, 32>;
using Shake256N24Chain = GenericFam<CoreShake<34, XB_KECCAK_CHAIN_ROLL>, 24, 4>;
using Shake256N32Chain = GenericFam<CoreShake<34, XB_KECCAK_CHAIN_ROLL>, 32, 32>;
using Shake256N64Chain = GenericFam<CoreShake<34, XB_KECCAK_CHAIN_ROLL>, 64, 64>;

// ---------------------------------------------------------------------------
// SHA-256, n = 32, padding_len = 32: midstate form.
// ---------------------------------------------------------------------------
struct Sha256N32Ctx {
    uint32_t pub[8];
    uint32_t sks[8];
    uint32_t prf_mid[8];  // compress(IV, toByte(3,32) || PUB_SEED)
    uint32_t kg_mid[8];   // compress(IV, toByte(4,32) || SK_SEED)
    uint32_t r_mid[8];    // compress(IV, toByte(3,32) || SK_PRF)
};

struct Sha256N32HPre {
    uint32_t c[8];   // state after the first core block toByte(1,32) || key
    uint32_t m1[8];
    uint32_t m2[8];
};

// MIX is the SHA-256 pipe mix (hashcore.cuh): kernels that keep many warps
// busy use the FMA-pipe form, serial / latency-bound ones the plain form.
template <int MIX>
struct Sha256N32T : FamBase<32, 32, true> {
    using Ctx = Sha256N32Ctx;
    using HPre = Sha256N32HPre;
    __device__ __forceinline__ static void compress(uint32_t (&st)[8], uint32_t (&w)[16])
    {
        sha256_compress_t<MIX>(st, w);
    }

    __device__ __forceinline__ static void mid(uint32_t (&st)[8], uint32_t x, const uint32_t (&k)[8])
    {
        uint32_t w[16];
#pragma unroll
        for (int i = 0; i < 7; i++) w[i] = 0;
        w[7] = x;
#pragma unroll
        for (int i = 0; i < 8; i++) w[8 + i] = k[i];
        sha256_iv(st);
        compress(st, w);
    }

    __device__ static void make_ctx(Ctx& c, const uint8_t* pub, const uint8_t* sks, const uint8_t* skp)
    {
        uint32_t t[8];
        load(c.pub, pub);
        mid(c.prf_mid, 3, c.pub);
#pragma unroll
        for (int i = 0; i < 8; i++) c.sks[i] = 0;
        if (sks) load(c.sks, sks);
        mid(c.kg_mid, 4, c.sks);
#pragma unroll
        for (int i = 0; i < 8; i++) t[i] = 0;
        if (skp) load(t, skp);
        mid(c.r_mid, 3, t);
    }

    // PRF(PUB_SEED, ADRS): one compression from the PRF midstate.
    __device__ __forceinline__ static void prf_adrs(uint32_t (&out)[8], const Ctx& c, const uint32_t (&a)[8])
    {
        uint32_t w[16];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            w[i] = a[i];
            out[i] = c.prf_mid[i];
        }
        w[8] = 0x80000000u;
#pragma unroll
        for (int i = 9; i < 15; i++) w[i] = 0;
        w[15] = 768;
        compress(out, w);
    }

    __device__ static void thash_f(uint32_t (&x)[8], const Ctx& c, uint32_t (&a)[8])
    {
        uint32_t key[8], t[8], w[16];
        a[7] = 1;
        prf_adrs(t, c, a);  // mask
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] ^= t[i];
        a[7] = after(0, t[7]);  // key PRF strictly after the mask PRF
        prf_adrs(key, c, a);
#pragma unroll
        for (int i = 0; i < 8; i++) {
            w[i] = 0;
            w[8 + i] = key[i];
        }
        sha256_iv(t);
        compress(t, w);
#pragma unroll
        for (int i = 0; i < 8; i++) w[i] = x[i];
        w[8] = 0x80000000u;
#pragma unroll
        for (int i = 9; i < 15; i++) w[i] = 0;
        w[15] = 768;
        compress(t, w);
#pragma unroll
        for (int i = 0; i < 8; i++) x[i] = t[i];
    }

    // thash_h runs as one loop over its six compressions around a single
    // compression body: the tree kernels that call it are throughput bound,
    // and separately inlined bodies overflow the instruction cache.
    // thash_h in one loop with the masks folded into the inputs as soon as
    // they exist: 0 mask PRF (km 1) -> l ^= m1, 1 mask PRF (km 2) -> r ^= m2,
    // 2 key PRF (km 0), 3 toByte(1,32) || key, 4 l || r, 5 padding.
    // o may alias l or r.
    __device__ static void thash_h(uint32_t (&o)[8], const uint32_t (&l)[8], const uint32_t (&r)[8],
                                   const Ctx& c, uint32_t (&a)[8])
    {
        uint32_t lc[8], rc[8], t[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            lc[i] = l[i];
            rc[i] = r[i];
        }
#pragma unroll 1
        for (uint32_t k = 0; k < 6; k++) {
            uint32_t st[8], w[16];
            if (k <= 2) {
#pragma unroll
                for (int i = 0; i < 7; i++) w[i] = a[i];
                w[7] = (k == 2) ? 0u : k + 1;
                w[8] = 0x80000000u;
#pragma unroll
                for (int i = 9; i < 15; i++) w[i] = 0;
                w[15] = 768;
#pragma unroll
                for (int i = 0; i < 8; i++) st[i] = c.prf_mid[i];
            } else if (k == 3) {
#pragma unroll
                for (int i = 0; i < 7; i++) w[i] = 0;
                w[7] = 1;
#pragma unroll
                for (int i = 0; i < 8; i++) w[8 + i] = t[i];
                sha256_iv(st);
            } else if (k == 4) {
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = lc[i];
                    w[8 + i] = rc[i];
                    st[i] = t[i];
                }
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) st[i] = t[i];
                w[0] = 0x80000000u;
#pragma unroll
                for (int i = 1; i < 15; i++) w[i] = 0;
                w[15] = 1024;
            }
            compress(st, w);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                if (k == 0) lc[i] ^= st[i];
                else if (k == 1) rc[i] ^= st[i];
                else t[i] = st[i];
            }
        }
#pragma unroll
        for (int i = 0; i < 8; i++) o[i] = t[i];
        a[7] = 2;  // as set_key_and_mask leaves it (hash.c:146-147)
    }

    __device__ static void h_pre(HPre& o, const Ctx& c, uint32_t (&a)[8])
    {
        uint32_t t[8], w[16];
        a[7] = 0;
        prf_adrs(t, c, a);
#pragma unroll
        for (int i = 0; i < 7; i++) w[i] = 0;
        w[7] = 1;
#pragma unroll
        for (int i = 0; i < 8; i++) w[8 + i] = t[i];
        sha256_iv(o.c);
        compress(o.c, w);
        a[7] = 1;
        prf_adrs(o.m1, c, a);
        a[7] = 2;
        prf_adrs(o.m2, c, a);
    }

    // o may alias l or r.
    __device__ static void h_fin(uint32_t (&o)[8], const HPre& p, const uint32_t (&l)[8], const uint32_t (&r)[8])
    {
        uint32_t w[16], st[8];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            w[i] = l[i] ^ p.m1[i];
            w[8 + i] = r[i] ^ p.m2[i];
            st[i] = p.c[i];
        }
        compress(st, w);
        w[0] = 0x80000000u;
#pragma unroll
        for (int i = 1; i < 15; i++) w[i] = 0;
        w[15] = 1024;
        compress(st, w);
#pragma unroll
        for (int i = 0; i < 8; i++) o[i] = st[i];
    }

    __device__ static void prf_keygen(uint32_t (&o)[8], const Ctx& c, const uint32_t (&a)[8])
    {
        uint32_t w[16];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            w[i] = c.pub[i];
            w[8 + i] = a[i];
            o[i] = c.kg_mid[i];
        }
        compress(o, w);
        w[0] = 0x80000000u;
#pragma unroll
        for (int i = 1; i < 15; i++) w[i] = 0;
        w[15] = 1024;
        compress(o, w);
    }

    // A whole WOTS chain in one loop over compression sub-steps, so the kernel
    // holds a single copy of the (fully unrolled, ~1,400-instruction)
    // compression: with the four compressions of F inlined separately the
    // chain loop no longer fits the instruction cache.  With keygen, the chain
    // starts with PRF_keygen (2 sub-steps, hash.c:87-98) from the address in
    // `a` (hash = key_and_mask = 0); then `steps` F calls at hash addresses
    // start .. start + steps - 1, 4 sub-steps each: mask PRF, key PRF,
    // toByte(0) || key, (x ^ mask) || padding (hash.c:157-183).
    //
    // chain_skip: the same chain with the work it repeats done once.  Rounds 0..5 of both PRF blocks read
    // only ADRS words 0..5 (layer, tree, type, OTS address, chain index), which
    // no step of a chain changes, and so do schedule words W16..W20 (with the
    // padding words W9..W15): they are computed once per chain into shared
    // memory, and each PRF compression resumes at round 6.  The core block
    // toByte(0, 32) || key has W0..W7 = 0, so its rounds 0..7 from the IV are a
    // constant and it resumes at round 8.  Per F call that is 20 of 256 rounds
    // and 10 of 192 schedule words fewer.  Only the 8-word value that must
    // outlive a compression (`carry`: the chain value, or the state after
    // toByte(0) || key for the last block) is held in registers across it; the
    // PRF feed-forward (the PUB_SEED midstate) is read from shared memory
    // after the rounds.  Callers launch at most 128 threads per CTA (the
    // shared array has one column per thread).
    static constexpr bool kHasChain = true;

    __device__ static void chain_skip(uint32_t (&x)[8], const Ctx& c, const uint32_t (&a)[8], uint32_t start,
                                      uint32_t steps, bool keygen)
    {
        // per thread, word i at pre[128 * i]: slots after round 5 (0..7),
        // W16..W20 (8..12), the PRF midstate (13..20)
        __shared__ uint32_t chain_pre[21 * 128];
        uint32_t* pre = chain_pre + threadIdx.x;
        {
            uint32_t p[8], w[16];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                p[i] = c.prf_mid[i];
                pre[128 * (13 + i)] = p[i];
            }
#pragma unroll
            for (int t = 0; t < 6; t++) {
                w[t] = a[t];
                sha256_round_s<MIX>(p, t, a[t]);
            }
            w[9] = w[10] = w[11] = w[12] = w[13] = w[14] = 0;
            w[15] = 768;
#pragma unroll
            for (int t = 16; t < 21; t++) sha256_sched<MIX>(w, t);
#pragma unroll
            for (int i = 0; i < 8; i++) pre[128 * i] = p[i];
#pragma unroll
            for (int i = 0; i < 5; i++) pre[128 * (8 + i)] = w[i];
        }
        constexpr Sha256Slots z8 = sha256_zero_prefix8();
        uint32_t tmp[8];  // key, then the state after toByte(0) || key
        const uint32_t pre_n = keygen ? 2 : 0;
        const uint32_t total = pre_n + 4 * steps;
#pragma unroll 1
        for (uint32_t j = 0; j < total; j++) {
            uint32_t s[8], w[16], carry[8];
            int skip = 0;
            const uint32_t jj = j - pre_n;
            const uint32_t phase = (j < pre_n) ? 4 + j : (jj & 3);
            const uint32_t hash = start + (jj >> 2);
            if (phase <= 1) {  // PRF(PUB_SEED, ADRS) with key_and_mask 1 (mask), then 0 (key)
#pragma unroll
                for (int i = 0; i < 6; i++) w[i] = a[i];
                w[6] = hash;
                w[7] = 1 - phase;
                w[8] = 0x80000000u;
#pragma unroll
                for (int i = 9; i < 15; i++) w[i] = 0;
                w[15] = 768;
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    s[i] = lds_u32(pre + 128 * i);
                    carry[i] = x[i];
                }
                skip = 6;
            } else if (phase == 2) {  // toByte(0, 32) || key from the IV
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = 0;
                    w[8 + i] = tmp[i];
                    s[i] = z8.v[i];
                    carry[i] = x[i];
                }
                skip = 8;
            } else if (phase == 3) {  // (x ^ mask) || padding of 96 bytes
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = x[i];
                    s[i] = tmp[i];
                    carry[i] = tmp[i];
                }
                w[8] = 0x80000000u;
#pragma unroll
                for (int i = 9; i < 15; i++) w[i] = 0;
                w[15] = 768;
            } else if (phase == 4) {  // PRF_keygen: PUB_SEED || ADRS from the SK_SEED midstate
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = c.pub[i];
                    s[i] = c.kg_mid[i];
                    carry[i] = s[i];
                }
#pragma unroll
                for (int i = 0; i < 6; i++) w[8 + i] = a[i];
                w[14] = 0;
                w[15] = 0;
            } else {  // PRF_keygen padding block (128 bytes)
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    s[i] = x[i];
                    carry[i] = x[i];
                }
                w[0] = 0x80000000u;
#pragma unroll
                for (int i = 1; i < 15; i++) w[i] = 0;
                w[15] = 1024;
            }
            sha256_rounds_resume<MIX>(s, w, skip, pre + 128 * 8, 128);
            if (phase == 0) {  // x ^= mask
#pragma unroll
                for (int i = 0; i < 8; i++) x[i] = carry[i] ^ (lds_u32(pre + 128 * (13 + i)) + s[i]);
            } else if (phase == 1) {  // key
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    x[i] = carry[i];
                    tmp[i] = lds_u32(pre + 128 * (13 + i)) + s[i];
                }
            } else if (phase == 2) {
                uint32_t iv[8];
                sha256_iv(iv);
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    x[i] = carry[i];
                    tmp[i] = iv[i] + s[i];
                }
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) x[i] = carry[i] + s[i];
            }
        }
    }

    // chain_plain: one compression body from the chaining value each time.
    __device__ static void chain_plain(uint32_t (&x)[8], const Ctx& c, const uint32_t (&a)[8], uint32_t start,
                                       uint32_t steps, bool keygen)
    {
        uint32_t tmp[8];  // key, then the state after toByte(0) || key
        const uint32_t pre = keygen ? 2 : 0;
        const uint32_t total = pre + 4 * steps;
#pragma unroll 1
        for (uint32_t j = 0; j < total; j++) {
            uint32_t st[8], w[16];
            const uint32_t jj = j - pre;
            const uint32_t phase = (j < pre) ? 4 + j : (jj & 3);
            const uint32_t hash = start + (jj >> 2);
            if (phase <= 1) {  // PRF(PUB_SEED, ADRS) with key_and_mask 1 (mask), then 0 (key)
#pragma unroll
                for (int i = 0; i < 6; i++) w[i] = a[i];
                w[6] = hash;
                w[7] = 1 - phase;
                w[8] = 0x80000000u;
#pragma unroll
                for (int i = 9; i < 15; i++) w[i] = 0;
                w[15] = 768;
#pragma unroll
                for (int i = 0; i < 8; i++) st[i] = c.prf_mid[i];
            } else if (phase == 2) {  // toByte(0, 32) || key from the IV
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = 0;
                    w[8 + i] = tmp[i];
                }
                sha256_iv(st);
            } else if (phase == 3) {  // (x ^ mask) || padding of 96 bytes
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = x[i];
                    st[i] = tmp[i];
                }
                w[8] = 0x80000000u;
#pragma unroll
                for (int i = 9; i < 15; i++) w[i] = 0;
                w[15] = 768;
            } else if (phase == 4) {  // PRF_keygen: PUB_SEED || ADRS from the SK_SEED midstate
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = c.pub[i];
                    st[i] = c.kg_mid[i];
                }
#pragma unroll
                for (int i = 0; i < 6; i++) w[8 + i] = a[i];
                w[14] = 0;
                w[15] = 0;
            } else {  // PRF_keygen padding block (128 bytes)
#pragma unroll
                for (int i = 0; i < 8; i++) st[i] = x[i];
                w[0] = 0x80000000u;
#pragma unroll
                for (int i = 1; i < 15; i++) w[i] = 0;
                w[15] = 1024;
            }
            compress(st, w);
            if (phase == 0) {
#pragma unroll
                for (int i = 0; i < 8; i++) x[i] ^= st[i];
            } else if (phase <= 2) {
#pragma unroll
                for (int i = 0; i < 8; i++) tmp[i] = st[i];
            } else {
#pragma unroll
                for (int i = 0; i < 8; i++) x[i] = st[i];
            }
        }
    }

    // Chains that start with PRF_keygen (keygen, sign: every chain 15 steps
    // or the signature's lengths, all from the secret seed) take the form
    // that skips the repeated prefix rounds (keygen 6.8% faster on B200);
    // verify chains keep the plain loop, where the same form measured no
    // faster per chain and 2.5% slower per split verify batch.  `keygen` is a
    // literal at every call site, so each kernel holds one of the two loops.
    __device__ __forceinline__ static void chain(uint32_t (&x)[8], const Ctx& c, const uint32_t (&a)[8],
                                                 uint32_t start, uint32_t steps, bool keygen)
    {
        if (keygen) chain_skip(x, c, a, start, steps, true);
        else chain_plain(x, c, a, start, steps, false);
    }

    __device__ static void prf_r(uint32_t (&o)[8], const Ctx& c, uint64_t idx)
    {
        uint32_t w[16];
#pragma unroll
        for (int i = 0; i < 6; i++) w[i] = 0;
        w[6] = (uint32_t)(idx >> 32);
        w[7] = (uint32_t)idx;
        w[8] = 0x80000000u;
#pragma unroll
        for (int i = 9; i < 15; i++) w[i] = 0;
        w[15] = 768;
#pragma unroll
        for (int i = 0; i < 8; i++) o[i] = c.r_mid[i];
        compress(o, w);
    }
};

using Sha256N32 = Sha256N32T<0>;
using Sha256N32Fma = Sha256N32T<1>;

// ---------------------------------------------------------------------------
// SHA-512, n = 64, padding_len = 64: midstate form over 64-bit words.
// ---------------------------------------------------------------------------
struct Sha512N64 : FamBase<64, 64, true> {
    struct Ctx {
        uint32_t pub[16];
        uint32_t sks[16];
        uint64_t prf_mid[8];
        uint64_t kg_mid[8];
        uint64_t r_mid[8];
    };

    __device__ __forceinline__ static void mid(uint64_t (&st)[8], uint64_t x, const uint32_t (&k)[16])
    {
        uint64_t w[16];
#pragma unroll
        for (int i = 0; i < 7; i++) w[i] = 0;
        w[7] = x;
#pragma unroll
        for (int i = 0; i < 8; i++) w[8 + i] = join64(k[2 * i], k[2 * i + 1]);
        sha512_iv(st);
        sha512_compress(st, w);
    }

    __device__ __forceinline__ static void out16(uint32_t (&o)[16], const uint64_t (&st)[8])
    {
#pragma unroll
        for (int i = 0; i < 8; i++) {
            o[2 * i] = (uint32_t)(st[i] >> 32);
            o[2 * i + 1] = (uint32_t)st[i];
        }
    }

    __device__ static void make_ctx(Ctx& c, const uint8_t* pub, const uint8_t* sks, const uint8_t* skp)
    {
        uint32_t t[16];
        load(c.pub, pub);
        mid(c.prf_mid, 3, c.pub);
#pragma unroll
        for (int i = 0; i < 16; i++) c.sks[i] = 0;
        if (sks) load(c.sks, sks);
        mid(c.kg_mid, 4, c.sks);
#pragma unroll
        for (int i = 0; i < 16; i++) t[i] = 0;
        if (skp) load(t, skp);
        mid(c.r_mid, 3, t);
    }

    __device__ __forceinline__ static void prf_adrs(uint64_t (&st)[8], const Ctx& c, const uint32_t (&a)[8])
    {
        uint64_t w[16];
#pragma unroll
        for (int i = 0; i < 4; i++) w[i] = join64(a[2 * i], a[2 * i + 1]);
        w[4] = 0x8000000000000000ull;
#pragma unroll
        for (int i = 5; i < 15; i++) w[i] = 0;
        w[15] = 1280;  // (64 + 64 + 32) * 8
#pragma unroll
        for (int i = 0; i < 8; i++) st[i] = c.prf_mid[i];
        sha512_compress(st, w);
    }

    // The WOTS chain (wots.c:38-53) as one loop over compression sub-steps -
    // PRF key, toByte(0, 64) || key, PRF mask, (x ^ mask) || padding per F
    // call, PRF_keygen first for keygen - so a chain kernel holds a single
    // SHA-512 compression body.
    static constexpr bool kHasChain = true;

    __device__ static void chain(uint32_t (&x)[16], const Ctx& c, const uint32_t (&a)[8], uint32_t start,
                                 uint32_t steps, bool keygen)
    {
        uint64_t tmp[8], mask[8];  // key, then the state after toByte(0) || key; the mask
        const uint32_t pre = keygen ? 1 : 0;
        const uint32_t total = pre + 4 * steps;
#pragma unroll 1
        for (uint32_t j = 0; j < total; j++) {
            uint64_t st[8], w[16];
            const uint32_t jj = j - pre;
            const uint32_t phase = (j < pre) ? 4 : (jj & 3);
            const uint32_t hash = start + (jj >> 2);
            if (phase == 0 || phase == 2) {  // PRF(PUB_SEED, ADRS), key_and_mask 0 (key) or 1 (mask)
#pragma unroll
                for (int i = 0; i < 3; i++) w[i] = join64(a[2 * i], a[2 * i + 1]);
                w[3] = join64(hash, phase >> 1);
                w[4] = 0x8000000000000000ull;
#pragma unroll
                for (int i = 5; i < 15; i++) w[i] = 0;
                w[15] = 1280;  // (64 + 64 + 32) * 8
#pragma unroll
                for (int i = 0; i < 8; i++) st[i] = c.prf_mid[i];
            } else if (phase == 1) {  // toByte(0, 64) || key from the IV
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = 0;
                    w[8 + i] = tmp[i];
                }
                sha512_iv(st);
            } else if (phase == 3) {  // (x ^ mask) || padding of 192 bytes
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = join64(x[2 * i], x[2 * i + 1]) ^ mask[i];
                    st[i] = tmp[i];
                }
                w[8] = 0x8000000000000000ull;
#pragma unroll
                for (int i = 9; i < 15; i++) w[i] = 0;
                w[15] = 1536;  // 192 * 8
            } else {  // PRF_keygen: PUB_SEED || ADRS from the SK_SEED midstate
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    w[i] = join64(c.pub[2 * i], c.pub[2 * i + 1]);
                    st[i] = c.kg_mid[i];
                }
#pragma unroll
                for (int i = 0; i < 4; i++) w[8 + i] = join64(a[2 * i], a[2 * i + 1]);
                w[12] = 0x8000000000000000ull;
                w[13] = 0;
                w[14] = 0;
                w[15] = 1792;  // (64 + 64 + 64 + 32) * 8
            }
            sha512_compress(st, w);
            if (phase <= 1) {
#pragma unroll
                for (int i = 0; i < 8; i++) tmp[i] = st[i];
            } else if (phase == 2) {
#pragma unroll
                for (int i = 0; i < 8; i++) mask[i] = st[i];
            } else {
                out16(x, st);
            }
        }
    }

    __device__ static void thash_f(uint32_t (&x)[16], const Ctx& c, uint32_t (&a)[8])
    {
        uint64_t t[8], st[8], w[16];
        a[7] = 0;
        prf_adrs(t, c, a);  // key
#pragma unroll
        for (int i = 0; i < 8; i++) {
            w[i] = 0;
            w[8 + i] = t[i];
        }
        sha512_iv(st);
        sha512_compress(st, w);
        a[7] = 1;
        prf_adrs(t, c, a);  // mask
#pragma unroll
        for (int i = 0; i < 8; i++) w[i] = join64(x[2 * i], x[2 * i + 1]) ^ t[i];
        w[8] = 0x8000000000000000ull;
#pragma unroll
        for (int i = 9; i < 15; i++) w[i] = 0;
        w[15] = 1536;  // 192 * 8
        sha512_compress(st, w);
        out16(x, st);
    }

    __device__ static void thash_h(uint32_t (&o)[16], const uint32_t (&l)[16], const uint32_t (&r)[16],
                                   const Ctx& c, uint32_t (&a)[8])
    {
        uint64_t t[8], st[8], w[16];
        a[7] = 0;
        prf_adrs(t, c, a);
#pragma unroll
        for (int i = 0; i < 7; i++) w[i] = 0;
        w[7] = 1;
#pragma unroll
        for (int i = 0; i < 8; i++) w[8 + i] = t[i];
        sha512_iv(st);
        sha512_compress(st, w);
        a[7] = 1;
        prf_adrs(t, c, a);
#pragma unroll
        for (int i = 0; i < 8; i++) w[i] = join64(l[2 * i], l[2 * i + 1]) ^ t[i];
        a[7] = 2;
        prf_adrs(t, c, a);
#pragma unroll
        for (int i = 0; i < 8; i++) w[8 + i] = join64(r[2 * i], r[2 * i + 1]) ^ t[i];
        sha512_compress(st, w);
        w[0] = 0x8000000000000000ull;
#pragma unroll
        for (int i = 1; i < 15; i++) w[i] = 0;
        w[15] = 2048;  // 256 * 8
        sha512_compress(st, w);
        out16(o, st);
    }

    struct HPre {
        uint64_t c[8];  // state after toByte(1,64) || key
        uint64_t m1[8];
        uint64_t m2[8];
    };

    __device__ static void h_pre(HPre& o, const Ctx& c, uint32_t (&a)[8])
    {
        uint64_t t[8], w[16];
        a[7] = 0;
        prf_adrs(t, c, a);
#pragma unroll
        for (int i = 0; i < 7; i++) w[i] = 0;
        w[7] = 1;
#pragma unroll
        for (int i = 0; i < 8; i++) w[8 + i] = t[i];
        sha512_iv(o.c);
        sha512_compress(o.c, w);
        a[7] = 1;
        prf_adrs(o.m1, c, a);
        a[7] = 2;
        prf_adrs(o.m2, c, a);
    }

    __device__ static void h_fin(uint32_t (&o)[16], const HPre& p, const uint32_t (&l)[16], const uint32_t (&r)[16])
    {
        uint64_t st[8], w[16];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            st[i] = p.c[i];
            w[i] = join64(l[2 * i], l[2 * i + 1]) ^ p.m1[i];
            w[8 + i] = join64(r[2 * i], r[2 * i + 1]) ^ p.m2[i];
        }
        sha512_compress(st, w);
        w[0] = 0x8000000000000000ull;
#pragma unroll
        for (int i = 1; i < 15; i++) w[i] = 0;
        w[15] = 2048;
        sha512_compress(st, w);
        out16(o, st);
    }

    __device__ static void prf_keygen(uint32_t (&o)[16], const Ctx& c, const uint32_t (&a)[8])
    {
        uint64_t st[8], w[16];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            w[i] = join64(c.pub[2 * i], c.pub[2 * i + 1]);
            st[i] = c.kg_mid[i];
        }
#pragma unroll
        for (int i = 0; i < 4; i++) w[8 + i] = join64(a[2 * i], a[2 * i + 1]);
        w[12] = 0x8000000000000000ull;
        w[13] = 0;
        w[14] = 0;
        w[15] = 1792;  // (64 + 64 + 64 + 32) * 8
        sha512_compress(st, w);
        out16(o, st);
    }

    __device__ static void prf_r(uint32_t (&o)[16], const Ctx& c, uint64_t idx)
    {
        uint64_t st[8], w[16];
        w[0] = 0;
        w[1] = 0;
        w[2] = 0;
        w[3] = idx;
        w[4] = 0x8000000000000000ull;
#pragma unroll
        for (int i = 5; i < 15; i++) w[i] = 0;
        w[15] = 1280;
#pragma unroll
        for (int i = 0; i < 8; i++) st[i] = c.r_mid[i];
        sha512_compress(st, w);
        out16(o, st);
    }
};

// ---------------------------------------------------------------------------
// H_msg (hash.c:107-120): toByte(2, pl) || R || root || toByte(idx, n) || M,
// streamed block by block from global memory.  One thread per message.
// ---------------------------------------------------------------------------
template <class F>
struct HMsgPrefix {
    static constexpr int W = F::PW + 3 * F::NW;  // prefix words
    uint32_t w[W];
    __device__ __forceinline__ void build(const uint32_t (&R)[F::NW], const uint32_t (&root)[F::NW], uint64_t idx)
    {
#pragma unroll
        for (int i = 0; i < F::PW - 1; i++) w[i] = 0;
        w[F::PW - 1] = F::mw(2);
#pragma unroll
        for (int i = 0; i < F::NW; i++) {
            w[F::PW + i] = R[i];
            w[F::PW + F::NW + i] = root[i];
            w[F::PW + 2 * F::NW + i] = 0;
        }
        w[W - 1] = F::mw((uint32_t)idx);
        w[W - 2] = F::mw((uint32_t)(idx >> 32));
    }
};

// Stream word k (4 bytes at offset 4k) of prefix || M as a little-endian
// packed value.
template <class F>
__device__ __forceinline__ uint32_t stream_le(const HMsgPrefix<F>& pre, const uint8_t* m, uint64_t mlen, uint64_t k)
{
    if (k < (uint64_t)HMsgPrefix<F>::W) {
        const uint32_t v = pre.w[k];
        return F::BE ? bswap32(v) : v;
    }
    return fetch4_le(m, mlen, 4 * (k - HMsgPrefix<F>::W));
}

// SHA-256 / SHA-512 / SHAKE streaming over the padded stream prefix || M,
// cut into blocks of BW 32-bit words (16 for SHA-256, 32 for SHA-512, the
// rate for SHAKE).  H_msg is a serial chain of compressions per thread, so
// its latency is the cost of one block times the blocks:
//   * head blocks (those holding prefix words) are unrolled, so the prefix
//     stays in registers;
//   * body blocks lie inside M with a word to spare: BW + 1 aligned words
//     are loaded one block ahead of the compression that consumes them and
//     funnel-shifted into place (M need not be 4-byte aligned);
//   * the tail blocks (end of M, padding, length) use bounded loads.
// absorb(w, last) consumes one block of little-endian packed words (bytes
// in stream order); pad(o, L) gives the padding bits of the word at stream
// byte o of a stream of L bytes.
template <int BW>
__device__ __forceinline__ void body_load(uint32_t (&a)[BW + 1], const uint32_t* q, uint64_t j0)
{
#pragma unroll
    for (int i = 0; i <= BW; i++) a[i] = __ldg(q + j0 + i);
}

template <class F, int BW, class Absorb, class Pad>
__device__ __forceinline__ void hmsg_stream(const HMsgPrefix<F>& pre, const uint8_t* m, uint64_t mlen, uint64_t nb,
                                            Absorb&& absorb, Pad&& pad)
{
    constexpr int W = HMsgPrefix<F>::W;
    constexpr int PB = (W + BW - 1) / BW;  // blocks holding prefix words
    const uint64_t L = 4ull * W + mlen;
    // bounded word s of the padded stream (little-endian packed)
    auto bounded = [&](uint64_t s) -> uint32_t {
        const uint64_t o = 4 * s;
        uint32_t le = (o < L) ? fetch4_le(m, mlen, o - 4ull * W) : 0;
        return le | pad(o, L);
    };
#pragma unroll
    for (int b = 0; b < PB; b++) {
        if ((uint64_t)b < nb) {
            uint32_t w[BW];
#pragma unroll
            for (int i = 0; i < BW; i++) {
                const int s = b * BW + i;
                if (s < W) {
                    const uint32_t v = pre.w[s < W ? s : 0];
                    w[i] = F::BE ? bswap32(v) : v;
                } else {
                    w[i] = bounded((uint64_t)s);
                }
            }
            absorb(w, (uint64_t)b + 1 == nb);
        }
    }
    // body: blocks b >= PB whose message words j0 .. j0 + BW (one spare)
    // lie inside M, j0 = BW * b - W
    const int64_t words = (int64_t)(mlen / 4);
    const int64_t lim = words + W - BW - 1;
    uint64_t bE = lim >= 0 ? (uint64_t)(lim / BW) + 1 : 0;
    if (bE < (uint64_t)PB) bE = PB;
    if (bE > nb) bE = nb;
    const uintptr_t addr = (uintptr_t)m;
    const uint32_t* q = (const uint32_t*)(addr & ~(uintptr_t)3);
    const int sh = (int)(addr & 3) * 8;
    uint32_t nxt[BW + 1];
    if (bE > (uint64_t)PB) body_load<BW>(nxt, q, (uint64_t)BW * PB - W);
    for (uint64_t b = PB; b < bE; b++) {
        uint32_t w[BW];
#pragma unroll
        for (int i = 0; i < BW; i++) w[i] = __funnelshift_r(nxt[i], nxt[i + 1], sh);
        if (b + 1 < bE) body_load<BW>(nxt, q, (uint64_t)BW * (b + 1) - W);
        absorb(w, false);
    }
    for (uint64_t b = bE; b < nb; b++) {
        uint32_t w[BW];
#pragma unroll
        for (int i = 0; i < BW; i++) w[i] = bounded((uint64_t)BW * b + i);
        absorb(w, b + 1 == nb);
    }
}

template <class F, int KIND>  // KIND 0 = SHA-256, 1 = SHA-512
struct HMsgImpl;

template <class F>
struct HMsgImpl<F, 0> {
    __device__ static void run(uint32_t (&out)[F::NW], const HMsgPrefix<F>& pre, const uint8_t* m, uint64_t mlen)
    {
        const uint64_t L = 4ull * HMsgPrefix<F>::W + mlen;
        const uint64_t nb = (L + 9 + 63) / 64;
        uint32_t st[8];
        sha256_iv(st);
        hmsg_stream<F, 16>(
            pre, m, mlen, nb,
            [&](uint32_t (&w)[16], bool last) {
#pragma unroll
                for (int j = 0; j < 16; j++) w[j] = bswap32(w[j]);
                if (last) {
                    w[14] = (uint32_t)((L * 8) >> 32);
                    w[15] = (uint32_t)(L * 8);
                }
                sha256_compress(st, w);
            },
            [](uint64_t o, uint64_t L_) -> uint32_t { return (o <= L_ && L_ < o + 4) ? 0x80u << (8 * (L_ - o)) : 0u; });
#pragma unroll
        for (int i = 0; i < F::NW; i++) out[i] = st[i];
    }
};

template <class F>
struct HMsgImpl<F, 1> {
    __device__ static void run(uint32_t (&out)[F::NW], const HMsgPrefix<F>& pre, const uint8_t* m, uint64_t mlen)
    {
        const uint64_t L = 4ull * HMsgPrefix<F>::W + mlen;
        const uint64_t nb = (L + 17 + 127) / 128;
        uint64_t st[8];
        sha512_iv(st);
        hmsg_stream<F, 32>(
            pre, m, mlen, nb,
            [&](uint32_t (&w)[32], bool last) {
                uint64_t w64[16];
#pragma unroll
                for (int j = 0; j < 16; j++) w64[j] = join64(bswap32(w[2 * j]), bswap32(w[2 * j + 1]));
                if (last) {
                    w64[14] = 0;
                    w64[15] = L * 8;
                }
                sha512_compress(st, w64);
            },
            [](uint64_t o, uint64_t L_) -> uint32_t { return (o <= L_ && L_ < o + 4) ? 0x80u << (8 * (L_ - o)) : 0u; });
        uint32_t o16[16];
#pragma unroll
        for (int i = 0; i < 8; i++) {
            o16[2 * i] = (uint32_t)(st[i] >> 32);
            o16[2 * i + 1] = (uint32_t)st[i];
        }
#pragma unroll
        for (int i = 0; i < F::NW; i++) out[i] = o16[i];
    }
};

template <class F, int RATEW>
__device__ void hmsg_shake(uint32_t (&out)[F::NW], const HMsgPrefix<F>& pre, const uint8_t* m, uint64_t mlen)
{
    const uint64_t L = 4ull * HMsgPrefix<F>::W + mlen;
    const uint64_t nb = L / (4 * RATEW) + 1;
    uint64_t A[25];
#pragma unroll
    for (int i = 0; i < 25; i++) A[i] = 0;
    hmsg_stream<F, RATEW>(
        pre, m, mlen, nb,
        [&](uint32_t (&w)[RATEW], bool last) {
            if (last) w[RATEW - 1] ^= 0x80000000u;
#pragma unroll
            for (int i = 0; i < RATEW / 2; i++) A[i] ^= join64(w[2 * i + 1], w[2 * i]);
            keccak_f1600(A);
        },
        [](uint64_t o, uint64_t L_) -> uint32_t { return (o <= L_ && L_ < o + 4) ? 0x1Fu << (8 * (L_ - o)) : 0u; });
#pragma unroll
    for (int i = 0; i < F::NW; i++) out[i] = (i & 1) ? (uint32_t)(A[i / 2] >> 32) : (uint32_t)A[i / 2];
}

// H_msg of ONE message by a whole warp (SHAKE families), every lane taking
// part: lane t < RATEW / 2 absorbs the 64-bit word t of each rate block (its
// loads of the next block are issued before the current permutation), and
// keccak_f1600_warp runs the permutation across the lanes.  Same bytes as
// hmsg_shake (prefix || M, pad 0x1F ... 0x80); every lane gets the digest.
template <class F, int RATEW>
__device__ void hmsg_shake_warp(uint32_t (&out)[F::NW], const HMsgPrefix<F>& pre, const uint8_t* m, uint64_t mlen)
{
    constexpr int W = HMsgPrefix<F>::W;
    const uint64_t L = 4ull * W + mlen;
    const uint64_t nb = L / (4 * RATEW) + 1;
    const uint32_t lane = threadIdx.x & 31;
    const KeccakWarpLane kl;
    // word s (4 bytes at offset 4s) of the padded stream, little-endian
    auto word = [&](uint64_t s) -> uint32_t {
        const uint64_t o = 4 * s;
        uint32_t v = 0;
        if (s < (uint64_t)W) {
#pragma unroll
            for (int i = 0; i < W; i++)
                if ((uint64_t)i == s) v = pre.w[i];
        } else if (o < L) {
            v = fetch4_le(m, mlen, o - 4ull * W);
        }
        if (o <= L && L < o + 4) v |= 0x1Fu << (8 * (L - o));
        return v;
    };
    uint32_t lo = 0, hi = 0, nl = 0, nh = 0;
    if (lane < RATEW / 2) {
        nl = word(2 * lane);
        nh = word(2 * lane + 1);
    }
    for (uint64_t b = 0; b < nb; b++) {
        if (lane < RATEW / 2) {
            lo ^= nl;
            hi ^= nh;
            if (b + 1 == nb && lane == RATEW / 2 - 1) hi ^= 0x80000000u;
            if (b + 1 < nb) {
                const uint64_t s = (b + 1) * RATEW + 2 * lane;
                nl = word(s);
                nh = word(s + 1);
            }
        }
        keccak_f1600_warp(lo, hi, kl);
    }
#pragma unroll
    for (int i = 0; i < F::NW; i++) out[i] = __shfl_sync(0xffffffffu, (i & 1) ? hi : lo, i / 2);
}

template <class F> struct HMsgKind;
template <int M> struct HMsgKind<Sha256N32T<M>> { static constexpr int v = 0; };
template <> struct HMsgKind<Sha256N24> { static constexpr int v = 0; };
template <> struct HMsgKind<Sha512N64> { static constexpr int v = 1; };
template <> struct HMsgKind<Shake128N32> { static constexpr int v = 42; };
template <> struct HMsgKind<Shake256N24> { static constexpr int v = 34; };
template <> struct HMsgKind<Shake256N32> { static constexpr int v = 34; };
template <> struct HMsgKind<Shake256N64> { static constexpr int v = 34; };

// 16 big-endian words of the 64-byte block at m + o, which lies entirely in
// [m, m + mlen).  Reads never go past m + mlen; like fetch4_le they may read
// up to 3 bytes before m + o when it is not 4-byte aligned.
__device__ __forceinline__ void load_block64_be(uint32_t (&w)[16], const uint8_t* m, uint64_t mlen, uint64_t o)
{
    const uint8_t* p = m + o;
    const uintptr_t a = (uintptr_t)p;
    if ((a & 15) == 0) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint4 v = __ldg((const uint4*)p + i);
            w[4 * i] = bswap32(v.x);
            w[4 * i + 1] = bswap32(v.y);
            w[4 * i + 2] = bswap32(v.z);
            w[4 * i + 3] = bswap32(v.w);
        }
    } else if ((a & 3) == 0) {
#pragma unroll
        for (int i = 0; i < 16; i++) w[i] = bswap32(__ldg((const uint32_t*)p + i));
    } else if (o + 68 <= mlen) {
        // 17 aligned words cover the block; the last one ends before m + mlen
        const uint32_t* q = (const uint32_t*)(a & ~(uintptr_t)3);
        const int sh = (int)(a & 3) * 8;
        uint32_t lo = __ldg(q);
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const uint32_t hi = __ldg(q + i + 1);
            w[i] = bswap32(__funnelshift_r(lo, hi, sh));
            lo = hi;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 16; i++) w[i] = bswap32(fetch4_le(m, mlen, o + 4 * i));
    }
}

// H_msg for SHA-256 with n = 32: the 128-byte prefix is exactly two blocks,
// so M starts block aligned; full message blocks are loaded one block ahead
// of the compression that consumes them.  H_msg is a serial chain, so the
// prefix, body and tail compressions are written out (a single-body loop
// measured slower here: its per-block setup lengthens the chain).
__device__ __forceinline__ void hmsg_sha256_n32(uint32_t (&out)[8], const uint32_t (&R)[8],
                                                       const uint32_t (&root)[8], uint64_t idx, const uint8_t* m,
                                                       uint64_t mlen)
{
    uint32_t st[8], w[16];
    sha256_iv(st);
#pragma unroll
    for (int i = 0; i < 7; i++) w[i] = 0;
    w[7] = 2;
#pragma unroll
    for (int i = 0; i < 8; i++) w[8 + i] = R[i];
    sha256_compress(st, w);
#pragma unroll
    for (int i = 0; i < 8; i++) w[i] = root[i];
#pragma unroll
    for (int i = 8; i < 14; i++) w[i] = 0;
    w[14] = (uint32_t)(idx >> 32);
    w[15] = (uint32_t)idx;
    sha256_compress(st, w);
    const uint64_t nfull = mlen / 64;
    uint32_t nxt[16];
    if (nfull) load_block64_be(nxt, m, mlen, 0);
    for (uint64_t b = 0; b < nfull; b++) {
#pragma unroll
        for (int i = 0; i < 16; i++) w[i] = nxt[i];
        if (b + 1 < nfull) load_block64_be(nxt, m, mlen, 64 * (b + 1));
        sha256_compress(st, w);
    }
    const uint64_t L = 128 + mlen;
    const uint64_t o0 = 64 * nfull;
    const int tail_blocks = ((mlen - o0) + 9 > 64) ? 2 : 1;
    for (int b = 0; b < tail_blocks; b++) {
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const uint64_t o = o0 + 64 * b + 4 * j;
            uint32_t le = (o < mlen) ? fetch4_le(m, mlen, o) : 0;
            if (o <= mlen && mlen < o + 4) le |= 0x80u << (8 * (mlen - o));
            w[j] = bswap32(le);
        }
        if (b == tail_blocks - 1) {
            w[14] = (uint32_t)((L * 8) >> 32);
            w[15] = (uint32_t)(L * 8);
        }
        sha256_compress(st, w);
    }
#pragma unroll
    for (int i = 0; i < 8; i++) out[i] = st[i];
}

template <class F>
__device__ void hmsg(uint32_t (&out)[F::NW], const uint32_t (&R)[F::NW], const uint32_t (&root)[F::NW],
                     uint64_t idx, const uint8_t* m, uint64_t mlen)
{
    if constexpr (std::is_same<typename F::Ctx, Sha256N32Ctx>::value) {
        hmsg_sha256_n32(out, R, root, idx, m, mlen);
    } else {
        HMsgPrefix<F> pre;
        pre.build(R, root, idx);
        constexpr int K = HMsgKind<F>::v;
        if constexpr (K == 0 || K == 1) {
            HMsgImpl<F, K>::run(out, pre, m, mlen);
        } else {
            hmsg_shake<F, K>(out, pre, m, mlen);
        }
    }
}

// H_msg by a whole warp (one message per warp) for the families whose
// permutation has a warp form (SHAKE); kWarpHmsg<F> says which.
template <class F>
constexpr bool kWarpHmsg = HMsgKind<F>::v >= 34;

template <class F>
__device__ void hmsg_warp(uint32_t (&out)[F::NW], const uint32_t (&R)[F::NW], const uint32_t (&root)[F::NW],
                          uint64_t idx, const uint8_t* m, uint64_t mlen)
{
    static_assert(kWarpHmsg<F>, "warp H_msg is the SHAKE form");
    HMsgPrefix<F> pre;
    pre.build(R, root, idx);
    hmsg_shake_warp<F, HMsgKind<F>::v>(out, pre, m, mlen);
}

}  // namespace xb
