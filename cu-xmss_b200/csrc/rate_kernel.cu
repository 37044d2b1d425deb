// Compression-rate probe: every thread runs `iters` dependent SHA-256
// compressions (or Keccak-f[1600] permutations) entirely in registers.  It
// measures the chip's sustained rate for the same compression code the XMSS
// kernels use and is the denominator of their roofline fraction.
#include <cstdint>

#include "engine.h"
#include "hashcore.cuh"

namespace xb {

template <int MIX>
__global__ void __launch_bounds__(128) k_sha256_rate(uint32_t iters, uint32_t seed, uint32_t* __restrict__ sink)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t st[8];
    sha256_iv(st);
    st[0] ^= t;
    st[1] ^= seed;
#pragma unroll 1
    for (uint32_t i = 0; i < iters; i++) {
        uint32_t w[16];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            w[j] = st[j];
            w[8 + j] = st[j] ^ i;
        }
        sha256_compress_any<MIX>(st, w);
    }
    uint32_t x = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) x ^= st[j];
    if (x == 0x9E3779B9u) sink[t] = x;  // practically never; keeps the work live
}

__global__ void __launch_bounds__(128) k_keccak_rate(uint32_t iters, uint32_t seed, uint32_t* __restrict__ sink)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t A[25];
#pragma unroll
    for (int j = 0; j < 25; j++) A[j] = ((uint64_t)t << 32) ^ seed ^ j;
#pragma unroll 1
    for (uint32_t i = 0; i < iters; i++) {
        A[0] ^= i;
        keccak_f1600_u<4>(A);  // the form the chain kernels run (4 rounds per loop pass)
    }
    uint64_t x = 0;
#pragma unroll
    for (int j = 0; j < 25; j++) x ^= A[j];
    if ((uint32_t)x == 0x9E3779B9u) sink[t] = (uint32_t)x;
}

__global__ void __launch_bounds__(128) k_sha512_rate(uint32_t iters, uint32_t seed, uint32_t* __restrict__ sink)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t st[8];
    sha512_iv(st);
    st[0] ^= t;
    st[1] ^= seed;
#pragma unroll 1
    for (uint32_t i = 0; i < iters; i++) {
        uint64_t w[16];
#pragma unroll
        for (int j = 0; j < 8; j++) {
            w[j] = st[j];
            w[8 + j] = st[j] ^ i;
        }
        sha512_compress(st, w);
    }
    uint64_t x = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) x ^= st[j];
    if ((uint32_t)x == 0x9E3779B9u) sink[t] = (uint32_t)x;
}

// kind 0: SHA-256 as the XMSS kernels compile it; 1: Keccak-f[1600];
// 2: SHA-512 compressions;
// 10 + m: SHA-256 with pipe mix m, 0..9 (for comparing the variants);
// 20 + m: the same with one warp per block (latency of a lone thread).
void launch_rate(int kind, uint32_t blocks, uint32_t iters, uint32_t* sink, cudaStream_t st)
{
    switch (kind) {
        case 13: k_sha256_rate<3><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 20: k_sha256_rate<0><<<blocks, 32, 0, st>>>(iters, 0x1234567u, sink); break;
        case 21: k_sha256_rate<1><<<blocks, 32, 0, st>>>(iters, 0x1234567u, sink); break;
        case 23: k_sha256_rate<3><<<blocks, 32, 0, st>>>(iters, 0x1234567u, sink); break;
        case 0: k_sha256_rate<XB_SHA256_MIX><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 1: k_keccak_rate<<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 2: k_sha512_rate<<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 10: k_sha256_rate<0><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 11: k_sha256_rate<1><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 12: k_sha256_rate<2><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 14: k_sha256_rate<4><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 15: k_sha256_rate<5><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 16: k_sha256_rate<6><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 17: k_sha256_rate<7><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 18: k_sha256_rate<8><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        case 19: k_sha256_rate<9><<<blocks, 128, 0, st>>>(iters, 0x1234567u, sink); break;
        default: break;
    }
}

}  // namespace xb
