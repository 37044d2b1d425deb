// C-ABI of libxmss_b200: the reference's xmss.h / xmss_core.h calls and the
// batch extensions of xmss_b200.h, all computed on the GPU.
//
// Host code here only parses OIDs, moves bytes and keeps the secret-key index
// bookkeeping of the reference (xmss_core.c:209-239); every hash runs in the
// kernels of xmss_kernels.cuh.
#include <fcntl.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/params.h"
#include "../../include/randombytes.h"
#include "../../include/utils.h"
#include "../../include/xmss.h"
#include "../../include/xmss_b200.h"
#include "../../include/xmss_core.h"
#include "engine.h"
#include "xmss_kernels.cuh"

using xb::Engine;

namespace {

thread_local std::string g_err;
void (*g_rng)(unsigned char*, unsigned long long) = nullptr;

constexpr int kOk = 0, kBad = -1, kExhausted = -2, kGpu = -3;

uint64_t be_read(const uint8_t* p, unsigned len)
{
    uint64_t r = 0;
    for (unsigned i = 0; i < len; i++) r = (r << 8) | p[i];
    return r;
}

void be_write(uint8_t* p, unsigned len, uint64_t v)
{
    for (int i = (int)len - 1; i >= 0; i--) {
        p[i] = (uint8_t)(v & 0xff);
        v >>= 8;
    }
}

int parse(xmss_params* p, uint32_t oid, int mt)
{
    return mt ? xmssmt_parse_oid(p, oid) : xmss_parse_oid(p, oid);
}

// Runs f under the engine lock, turning failures into return codes.
template <class Fn>
int guarded(Fn&& f)
{
    try {
        Engine& e = Engine::get();
        std::lock_guard<std::mutex> g(e.mu);
        g_err.clear();
        return f(e);
    } catch (const std::invalid_argument& ex) {
        g_err = ex.what();
        return kBad;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return kGpu;
    }
}

// -- keygen -----------------------------------------------------------------

int keypair_host(const xmss_params& p, uint32_t count, const uint8_t* seeds, uint8_t* pk, uint8_t* sk,
                 size_t pk_stride, size_t sk_stride)
{
    return guarded([&](Engine& e) {
        const xb::FamilyOps* ops = xb::ops_for(p);
        cudaStream_t st = e.stream();
        e.begin(st);
        const size_t n = p.n, seed_b = (size_t)count * 3 * n, pk_b = (size_t)count * 2 * n,
                     sk_b = (size_t)count * p.sk_bytes;
        uint8_t* h = e.h_stage.as<uint8_t>(seed_b + pk_b + sk_b);
        memcpy(h, seeds, seed_b);
        uint8_t* d = e.d_in.as<uint8_t>(seed_b + pk_b + sk_b);
        XB_CUDA(cudaMemcpyAsync(d, h, seed_b, cudaMemcpyHostToDevice, st));
        e.keypair(ops, p, count, d, d + seed_b, d + seed_b + pk_b, st);
        XB_CUDA(cudaMemcpyAsync(h + seed_b, d + seed_b, pk_b + sk_b, cudaMemcpyDeviceToHost, st));
        e.end(st);
        XB_CUDA(cudaStreamSynchronize(st));
        for (uint32_t k = 0; k < count; k++) {
            memcpy(pk + k * pk_stride, h + seed_b + k * 2 * n, 2 * n);
            memcpy(sk + k * sk_stride, h + seed_b + pk_b + k * p.sk_bytes, p.sk_bytes);
        }
        return kOk;
    });
}

// -- sign -------------------------------------------------------------------

// Index bookkeeping of xmssmt_core_sign (xmss_core.c:209-239) on one sk (no
// OID).  Returns kExhausted or kOk; on kOk *idx is the index to sign with and
// idx_bytes the bytes that go into the signature.
int sk_advance(const xmss_params& p, uint8_t* sk, uint64_t* idx, uint8_t* idx_bytes)
{
    const uint64_t i = be_read(sk, p.index_bytes);
    const uint64_t last = (p.full_height >= 64) ? ~0ull : ((1ull << p.full_height) - 1);
    if (i >= last) {
        memset(sk, 0xFF, p.index_bytes);
        memset(sk + p.index_bytes, 0, (size_t)(p.sk_bytes - p.index_bytes));
        if (i > last) return kExhausted;
        if (p.full_height == 64 && i == last) return kExhausted;
    }
    memcpy(idx_bytes, sk, p.index_bytes);
    be_write(sk, p.index_bytes, i + 1);
    *idx = i;
    return kOk;
}

// Signs `count` requests.  sk rows (no OID) at sk + r * sk_stride; messages
// m[r] of mlen[r] bytes; output sm[r] (sig || message).
int sign_host(const xmss_params& p, uint32_t count, uint8_t* sk, size_t sk_stride, const uint8_t* const* m,
              const uint64_t* mlen, uint8_t* const* sm, uint64_t* smlen, int* ret)
{
    // Bookkeeping first, exactly as the reference orders it: the message is
    // placed and *smlen set even when the key turns out to be exhausted.
    std::vector<uint32_t> live;
    std::vector<uint64_t> idx;
    std::vector<uint8_t> ibytes((size_t)count * 8);
    for (uint32_t r = 0; r < count; r++) {
        memmove(sm[r] + p.sig_bytes, m[r], mlen[r]);
        smlen[r] = p.sig_bytes + mlen[r];
        uint64_t i = 0;
        ret[r] = sk_advance(p, sk + r * sk_stride, &i, &ibytes[(size_t)r * 8]);
        if (ret[r] == kOk) {
            live.push_back(r);
            idx.push_back(i);
        }
    }
    if (live.empty()) return kOk;
    return guarded([&](Engine& e) {
        const xb::FamilyOps* ops = xb::ops_for(p);
        cudaStream_t st = e.stream();
        e.begin(st);
        const uint32_t L = (uint32_t)live.size();
        std::vector<uint8_t> keys((size_t)L * p.sk_bytes);
        std::vector<uint64_t> off(L), ml(L);
        uint64_t total = 0;
        for (uint32_t k = 0; k < L; k++) {
            const uint32_t r = live[k];
            memcpy(&keys[(size_t)k * p.sk_bytes], sk + r * sk_stride, p.sk_bytes);
            off[k] = total;
            ml[k] = mlen[r];
            total += (p.sig_bytes + mlen[r] + 15) & ~15ull;
        }
        const size_t meta = 2 * L * sizeof(uint64_t);
        uint8_t* h = e.h_stage.as<uint8_t>(total + meta);
        for (uint32_t k = 0; k < L; k++) memcpy(h + off[k] + p.sig_bytes, sm[live[k]] + p.sig_bytes, ml[k]);
        memcpy(h + total, off.data(), L * sizeof(uint64_t));
        memcpy(h + total + L * sizeof(uint64_t), ml.data(), L * sizeof(uint64_t));
        uint8_t* d = e.d_in.as<uint8_t>(total + meta);
        XB_CUDA(cudaMemcpyAsync(d, h, total + meta, cudaMemcpyHostToDevice, st));
        e.sign(ops, p, L, keys.data(), idx.data(), d, (const uint64_t*)(d + total),
               (const uint64_t*)(d + total + L * sizeof(uint64_t)), st);
        XB_CUDA(cudaMemcpyAsync(h, d, total, cudaMemcpyDeviceToHost, st));
        e.end(st);
        XB_CUDA(cudaStreamSynchronize(st));
        for (uint32_t k = 0; k < L; k++) {
            const uint32_t r = live[k];
            memcpy(sm[r], h + off[k], p.sig_bytes);
            memcpy(sm[r], &ibytes[(size_t)r * 8], p.index_bytes);  // memcpy(sm, sk, ib)
        }
        return kOk;
    });
}

// -- verify -----------------------------------------------------------------

int verify_host(const xmss_params& p, uint32_t count, const uint8_t* sm, const uint64_t* sm_off,
                const uint64_t* smlen, const uint8_t* pk_noid, size_t pk_stride, uint32_t npk,
                const uint32_t* pk_index, int* status)
{
    return guarded([&](Engine& e) {
        const xb::FamilyOps* ops = xb::ops_for(p);
        if (!count) return kOk;
        cudaStream_t st = e.stream();
        e.begin(st);
        uint64_t raw = 0;
        for (uint32_t i = 0; i < count; i++) raw = std::max(raw, sm_off[i] + smlen[i]);
        const uint64_t span = (raw + 15) & ~15ull;
        const size_t n2 = 2 * (size_t)p.n;
        const size_t o_off = span, o_len = o_off + count * 8, o_pk = o_len + count * 8,
                     o_idx = o_pk + ((npk * n2 + 15) & ~(size_t)15), o_st = o_idx + ((count * 4 + 15) & ~(size_t)15),
                     total = o_st + count * 4;
        uint8_t* d = e.d_in.as<uint8_t>(total);
        // The signed messages go straight from the caller's memory (a direct
        // DMA when it is pinned); the small arrays are staged.
        if (raw) XB_CUDA(cudaMemcpyAsync(d, sm, raw, cudaMemcpyHostToDevice, st));
        uint8_t* h = e.h_stage.as<uint8_t>(total - o_off);
        memcpy(h, sm_off, count * 8);
        memcpy(h + (o_len - o_off), smlen, count * 8);
        for (uint32_t k = 0; k < npk; k++) memcpy(h + (o_pk - o_off) + k * n2, pk_noid + k * pk_stride, n2);
        uint32_t* hi = (uint32_t*)(h + (o_idx - o_off));
        for (uint32_t i = 0; i < count; i++) {
            hi[i] = pk_index ? pk_index[i] : i;
            if (hi[i] >= npk) throw std::invalid_argument("pk_index out of range");
        }
        XB_CUDA(cudaMemcpyAsync(d + o_off, h, o_st - o_off, cudaMemcpyHostToDevice, st));
        e.verify(ops, p, count, d, (const uint64_t*)(d + o_off), (const uint64_t*)(d + o_len), d + o_pk, npk,
                 (const uint32_t*)(d + o_idx), (int*)(d + o_st), st);
        XB_CUDA(cudaMemcpyAsync(status, d + o_st, count * 4, cudaMemcpyDeviceToHost, st));
        e.end(st);
        XB_CUDA(cudaStreamSynchronize(st));
        return kOk;
    });
}

// Single sign_open with the reference's treatment of m (xmss_commons.c:
// 150-209): the message is staged at m + sig_bytes behind the H_msg prefix,
// then copied to m on success or m[0..mlen) zeroed on failure.
int sign_open_one(const xmss_params& p, uint8_t* m, unsigned long long* mlen, const uint8_t* sm,
                  unsigned long long smlen, const uint8_t* pk)
{
    if (smlen < p.sig_bytes) {  // the reference underflows here
        *mlen = 0;
        return kBad;
    }
    const unsigned long long ml = smlen - p.sig_bytes;
    *mlen = ml;
    const uint64_t idx = be_read(sm, p.index_bytes);
    memmove(m + p.sig_bytes, sm + p.sig_bytes, ml);
    uint8_t* pre = m + p.sig_bytes - p.padding_len - 3 * p.n;
    be_write(pre, p.padding_len, 2);
    memcpy(pre + p.padding_len, sm + p.index_bytes, p.n);
    memcpy(pre + p.padding_len + p.n, pk, p.n);
    be_write(pre + p.padding_len + 2 * p.n, p.n, idx);
    const uint64_t off = 0, len = smlen;
    int status = -1;
    int r = verify_host(p, 1, sm, &off, &len, pk, 2 * p.n, 1, nullptr, &status);
    if (r != kOk) {
        *mlen = 0;
        return r;
    }
    if (status != 0) {
        memset(m, 0, ml);
        *mlen = 0;
        return kBad;
    }
    memmove(m, sm + p.sig_bytes, ml);
    return kOk;
}

int keypair_api(uint8_t* pk, uint8_t* sk, uint32_t oid, int mt)
{
    xmss_params p;
    if (parse(&p, oid, mt)) return kBad;
    be_write(pk, XMSS_OID_LEN, oid);
    be_write(sk, XMSS_OID_LEN, oid);
    return xmssmt_core_keypair(&p, pk + XMSS_OID_LEN, sk + XMSS_OID_LEN);
}

int sign_api(uint8_t* sk, uint8_t* sm, unsigned long long* smlen, const uint8_t* m, unsigned long long mlen, int mt)
{
    xmss_params p;
    if (parse(&p, (uint32_t)be_read(sk, XMSS_OID_LEN), mt)) return kBad;
    return xmssmt_core_sign(&p, sk + XMSS_OID_LEN, sm, smlen, m, mlen);
}

int sign_open_api(uint8_t* m, unsigned long long* mlen, const uint8_t* sm, unsigned long long smlen,
                  const uint8_t* pk, int mt)
{
    xmss_params p;
    if (parse(&p, (uint32_t)be_read(pk, XMSS_OID_LEN), mt)) return kBad;
    return sign_open_one(p, m, mlen, sm, smlen, pk + XMSS_OID_LEN);
}

}  // namespace

namespace xb {
// Lets other translation units of the library report through
// xmss_b200_last_error.
void set_last_error(const std::string& msg) { g_err = msg; }
// The reference's index bookkeeping of one sign (sk without OID): 0 or -2.
int sign_advance(const xmss_params& p, uint8_t* sk, uint64_t* idx, uint8_t* idx_bytes)
{
    return sk_advance(p, sk, idx, idx_bytes);
}
}  // namespace xb

// ===========================================================================
// randombytes.h
// ===========================================================================

extern "C" __attribute__((weak)) void randombytes(unsigned char* x, unsigned long long xlen)
{
    if (g_rng) {
        g_rng(x, xlen);
        return;
    }
    // Same source as cuxmss/randombytes.c:10-39.
    static int fd = -1;
    while (fd == -1) {
        fd = open("/dev/urandom", O_RDONLY);
        if (fd == -1) sleep(1);
    }
    while (xlen > 0) {
        const ssize_t r = read(fd, x, xlen < 1048576 ? (size_t)xlen : 1048576);
        if (r < 1) {
            sleep(1);
            continue;
        }
        x += r;
        xlen -= (unsigned long long)r;
    }
}

// ===========================================================================
// utils.h
// ===========================================================================

extern "C" void ull_to_bytes(unsigned char* out, unsigned int outlen, unsigned long long in)
{
    be_write(out, outlen, in);
}

extern "C" unsigned long long bytes_to_ull(const unsigned char* in, unsigned int inlen)
{
    return be_read(in, inlen);
}

// ===========================================================================
// xmss_core.h
// ===========================================================================

extern "C" unsigned long long xmss_xmssmt_core_sk_bytes(const xmss_params* params)
{
    return params->index_bytes + 4ull * params->n;
}

extern "C" int xmssmt_core_seed_keypair(const xmss_params* params, unsigned char* pk, unsigned char* sk,
                                        unsigned char* seed)
{
    return keypair_host(*params, 1, seed, pk, sk, 2 * params->n, params->sk_bytes);
}

extern "C" int xmssmt_core_keypair(const xmss_params* params, unsigned char* pk, unsigned char* sk)
{
    std::vector<unsigned char> seed(3 * params->n);
    randombytes(seed.data(), seed.size());
    return xmssmt_core_seed_keypair(params, pk, sk, seed.data());
}

extern "C" int xmss_core_keypair(const xmss_params* params, unsigned char* pk, unsigned char* sk)
{
    return xmssmt_core_keypair(params, pk, sk);
}

extern "C" int xmssmt_core_sign(const xmss_params* params, unsigned char* sk, unsigned char* sm,
                                unsigned long long* smlen, const unsigned char* m, unsigned long long mlen)
{
    const uint8_t* mp = m;
    uint8_t* smp = sm;
    uint64_t ml = mlen, sl = 0;
    int ret = 0;
    int r = sign_host(*params, 1, sk, params->sk_bytes, &mp, &ml, &smp, &sl, &ret);
    *smlen = sl;
    return r != kOk ? r : ret;
}

extern "C" int xmss_core_sign(const xmss_params* params, unsigned char* sk, unsigned char* sm,
                              unsigned long long* smlen, const unsigned char* m, unsigned long long mlen)
{
    return xmssmt_core_sign(params, sk, sm, smlen, m, mlen);
}

extern "C" int xmssmt_core_sign_open(const xmss_params* params, unsigned char* m, unsigned long long* mlen,
                                     const unsigned char* sm, unsigned long long smlen, const unsigned char* pk)
{
    return sign_open_one(*params, m, mlen, sm, smlen, pk);
}

extern "C" int xmss_core_sign_open(const xmss_params* params, unsigned char* m, unsigned long long* mlen,
                                   const unsigned char* sm, unsigned long long smlen, const unsigned char* pk)
{
    return xmssmt_core_sign_open(params, m, mlen, sm, smlen, pk);
}

// ===========================================================================
// xmss.h
// ===========================================================================

extern "C" int xmss_keypair(unsigned char* pk, unsigned char* sk, const uint32_t oid)
{
    return keypair_api(pk, sk, oid, 0);
}

extern "C" int xmss_sign(unsigned char* sk, unsigned char* sm, unsigned long long* smlen, const unsigned char* m,
                         unsigned long long mlen)
{
    return sign_api(sk, sm, smlen, m, mlen, 0);
}

extern "C" int xmss_sign_open(unsigned char* m, unsigned long long* mlen, const unsigned char* sm,
                              unsigned long long smlen, const unsigned char* pk)
{
    return sign_open_api(m, mlen, sm, smlen, pk, 0);
}

extern "C" int xmssmt_keypair(unsigned char* pk, unsigned char* sk, const uint32_t oid)
{
    return keypair_api(pk, sk, oid, 1);
}

extern "C" int xmssmt_sign(unsigned char* sk, unsigned char* sm, unsigned long long* smlen, const unsigned char* m,
                           unsigned long long mlen)
{
    return sign_api(sk, sm, smlen, m, mlen, 1);
}

extern "C" int xmssmt_sign_open(unsigned char* m, unsigned long long* mlen, const unsigned char* sm,
                                unsigned long long smlen, const unsigned char* pk)
{
    return sign_open_api(m, mlen, sm, smlen, pk, 1);
}

// ===========================================================================
// xmss_b200.h
// ===========================================================================

extern "C" int xmss_b200_init(int device)
{
    try {
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
            g_err = "no usable CUDA device";
            return kGpu;
        }
        XB_CUDA(cudaSetDevice(device));
        Engine& e = Engine::get();
        if (e.device() != device) {
            g_err = "library already bound to device " + std::to_string(e.device());
            return kBad;
        }
        return kOk;
    } catch (const std::exception& ex) {
        g_err = ex.what();
        return kGpu;
    }
}

extern "C" const char* xmss_b200_last_error(void) { return g_err.c_str(); }

extern "C" void xmss_b200_set_randombytes(void (*fn)(unsigned char*, unsigned long long)) { g_rng = fn; }

extern "C" int xmss_b200_supported(unsigned int func, unsigned int n) { return xb::family_ops(func, n) != nullptr; }

extern "C" int xmss_b200_keypair_batch(uint32_t oid, int mt, uint32_t count, const uint8_t* seeds, uint8_t* pk,
                                       uint8_t* sk)
{
    xmss_params p;
    if (parse(&p, oid, mt)) return kBad;
    const size_t pks = XMSS_OID_LEN + 2 * p.n, sks = XMSS_OID_LEN + p.sk_bytes;
    for (uint32_t k = 0; k < count; k++) {
        be_write(pk + k * pks, XMSS_OID_LEN, oid);
        be_write(sk + k * sks, XMSS_OID_LEN, oid);
    }
    return keypair_host(p, count, seeds, pk + XMSS_OID_LEN, sk + XMSS_OID_LEN, pks, sks);
}

extern "C" int xmss_b200_keypair_device(uint32_t oid, int mt, uint32_t count, const uint8_t* d_seeds, uint8_t* d_pk,
                                        uint8_t* d_sk, void* stream)
{
    xmss_params p;
    if (parse(&p, oid, mt)) return kBad;
    return guarded([&](Engine& e) {
        const xb::FamilyOps* ops = xb::ops_for(p);
        cudaStream_t st = (cudaStream_t)stream;
        e.begin(st);
        e.keypair(ops, p, count, d_seeds, d_pk, d_sk, st);
        e.end(st);
        return kOk;
    });
}

extern "C" int xmss_b200_sign_open_batch(int mt, uint32_t count, const uint8_t* sm, const uint64_t* sm_off,
                                         const uint64_t* smlen, const uint8_t* pk, uint32_t npk,
                                         const uint32_t* pk_index, int* status)
{
    if (!npk) return count ? kBad : kOk;
    const uint32_t oid = (uint32_t)be_read(pk, XMSS_OID_LEN);
    xmss_params p;
    if (parse(&p, oid, mt)) return kBad;
    const size_t pks = XMSS_OID_LEN + 2 * p.n;
    for (uint32_t k = 1; k < npk; k++)
        if ((uint32_t)be_read(pk + k * pks, XMSS_OID_LEN) != oid) {
            g_err = "xmss_b200_sign_open_batch: public keys of different OIDs";
            return kBad;
        }
    return verify_host(p, count, sm, sm_off, smlen, pk + XMSS_OID_LEN, pks, npk, pk_index, status);
}

namespace {

// Buffers of one caller stream for xmss_b200_sign_open_batch_async: scratch
// and staging that grow stream-ordered on that stream, a second stream for
// the split of large batches, and the point where the stream's last call
// has copied its pinned staging to the device.
struct StreamCtx {
    xb::SplitStreams split;
    xb::Workspace w;
    xb::DevBuf d;
    xb::PinnedBuf h;
    cudaEvent_t staged = nullptr;
    bool pending = false;
};

std::map<cudaStream_t, std::unique_ptr<StreamCtx>> g_stream_ctx;  // guarded by Engine::mu

StreamCtx& stream_ctx(cudaStream_t st)
{
    auto& c = g_stream_ctx[st];
    if (!c) {
        auto n = std::make_unique<StreamCtx>();
        n->w.order_on(st);
        n->d.order_on(st);
        n->h.keep_old_blocks();
        n->split.create();
        n->w.split = &n->split;
        XB_CUDA(cudaEventCreateWithFlags(&n->staged, cudaEventDisableTiming));
        c = std::move(n);
    }
    return *c;
}

}  // namespace

extern "C" int xmss_b200_sign_open_batch_async(int mt, uint32_t count, const uint8_t* sm, const uint64_t* sm_off,
                                               const uint64_t* smlen, const uint8_t* pk, uint32_t npk,
                                               const uint32_t* pk_index, int* status, void* stream)
{
    if (!npk) return count ? kBad : kOk;
    const uint32_t oid = (uint32_t)be_read(pk, XMSS_OID_LEN);
    xmss_params p;
    if (parse(&p, oid, mt)) return kBad;
    const size_t pks = XMSS_OID_LEN + 2 * p.n;
    for (uint32_t k = 1; k < npk; k++)
        if ((uint32_t)be_read(pk + k * pks, XMSS_OID_LEN) != oid) {
            g_err = "xmss_b200_sign_open_batch_async: public keys of different OIDs";
            return kBad;
        }
    if (!count) return kOk;
    return guarded([&](Engine& e) {
        const xb::FamilyOps* ops = xb::ops_for(p);
        cudaStream_t st = (cudaStream_t)stream;
        XB_CUDA(cudaSetDevice(e.device()));
        StreamCtx& c = stream_ctx(st);
        // The staging block is rewritten below, so the stream's previous call
        // must have copied it to the device; its kernels and its status copy
        // may still be queued (the device buffers are reused in stream order).
        if (c.pending) XB_CUDA(cudaEventSynchronize(c.staged));
        uint64_t raw = 0;
        for (uint32_t i = 0; i < count; i++) raw = std::max(raw, sm_off[i] + smlen[i]);
        const uint64_t span = (raw + 15) & ~15ull;
        const size_t n2 = 2 * (size_t)p.n;
        const size_t o_off = span, o_len = o_off + count * 8, o_pk = o_len + count * 8,
                     o_idx = o_pk + ((npk * n2 + 15) & ~(size_t)15), o_st = o_idx + ((count * 4 + 15) & ~(size_t)15),
                     total = o_st + count * 4;
        uint8_t* h = c.h.as<uint8_t>(total - o_off);
        memcpy(h, sm_off, count * 8);
        memcpy(h + (o_len - o_off), smlen, count * 8);
        for (uint32_t k = 0; k < npk; k++) memcpy(h + (o_pk - o_off) + k * n2, pk + XMSS_OID_LEN + k * pks, n2);
        uint32_t* hi = (uint32_t*)(h + (o_idx - o_off));
        for (uint32_t i = 0; i < count; i++) {
            hi[i] = pk_index ? pk_index[i] : i;
            if (hi[i] >= npk) throw std::invalid_argument("pk_index out of range");
        }
        uint8_t* d = c.d.as<uint8_t>(total);
        if (raw) XB_CUDA(cudaMemcpyAsync(d, sm, raw, cudaMemcpyHostToDevice, st));
        XB_CUDA(cudaMemcpyAsync(d + o_off, h, o_st - o_off, cudaMemcpyHostToDevice, st));
        XB_CUDA(cudaEventRecord(c.staged, st));
        c.pending = true;
        e.verify(ops, p, count, d, (const uint64_t*)(d + o_off), (const uint64_t*)(d + o_len), d + o_pk, npk,
                 (const uint32_t*)(d + o_idx), (int*)(d + o_st), st, c.w, true);
        XB_CUDA(cudaMemcpyAsync(status, d + o_st, count * 4, cudaMemcpyDeviceToHost, st));
        XB_CUDA(cudaGetLastError());
        return kOk;
    });
}

extern "C" int xmss_b200_sign_open_device(uint32_t oid, int mt, uint32_t count, const uint8_t* d_sm,
                                          const uint64_t* d_sm_off, const uint64_t* d_smlen, const uint8_t* d_pk,
                                          uint32_t npk, const uint32_t* d_pk_index, int* d_status, void* stream)
{
    xmss_params p;
    if (parse(&p, oid, mt)) return kBad;
    if (count && (!d_pk_index || !npk)) return kBad;
    return guarded([&](Engine& e) {
        const xb::FamilyOps* ops = xb::ops_for(p);
        cudaStream_t st = (cudaStream_t)stream;
        e.begin(st);
        e.verify(ops, p, count, d_sm, d_sm_off, d_smlen, d_pk, npk, d_pk_index, d_status, st);
        e.end(st);
        return kOk;
    });
}

extern "C" int xmss_b200_sign_open_device_persistent(uint32_t oid, int mt, uint32_t count, const uint8_t* d_sm,
                                                     const uint64_t* d_sm_off, const uint64_t* d_smlen,
                                                     const uint8_t* d_pk, uint32_t npk, const uint32_t* d_pk_index,
                                                     int* d_status, void* stream)
{
    xmss_params p;
    if (parse(&p, oid, mt)) return kBad;
    if (count && (!d_pk_index || !npk)) return kBad;
    return guarded([&](Engine& e) {
        const xb::FamilyOps* ops = xb::ops_for(p);
        cudaStream_t st = (cudaStream_t)stream;
        e.begin(st);
        e.verify_persistent(ops, p, count, d_sm, d_sm_off, d_smlen, d_pk, npk, d_pk_index, d_status, st);
        e.end(st);
        return kOk;
    });
}

extern "C" int xmss_b200_sign_open_device_persistent_multi(const xmss_b200_verify_job* jobs, uint32_t njobs,
                                                           void* stream)
{
    if (njobs && !jobs) return kBad;
    std::vector<Engine::PersistJob> js(njobs);
    for (uint32_t i = 0; i < njobs; i++) {
        const xmss_b200_verify_job& j = jobs[i];
        if (parse(&js[i].p, j.oid, j.mt)) return kBad;
        if (j.count && (!j.d_pk_index || !j.npk || !j.d_sm || !j.d_sm_off || !j.d_smlen || !j.d_pk || !j.d_status))
            return kBad;
        js[i].count = j.count;
        js[i].d_sm = j.d_sm;
        js[i].d_sm_off = j.d_sm_off;
        js[i].d_smlen = j.d_smlen;
        js[i].d_pk = j.d_pk;
        js[i].npk = j.npk;
        js[i].d_pk_index = j.d_pk_index;
        js[i].d_status = j.d_status;
    }
    return guarded([&](Engine& e) {
        for (auto& j : js) j.ops = xb::ops_for(j.p);
        cudaStream_t st = (cudaStream_t)stream;
        e.begin(st);
        e.verify_persistent_multi(js, st);
        e.end(st);
        return kOk;
    });
}

extern "C" int xmss_b200_set_wait_bound(unsigned long long ns)
{
    return guarded([&](Engine& e) {
        e.persist_wait_ns = ns ? ns : Engine::kDefaultWaitNs;
        return kOk;
    });
}

extern "C" int xmss_b200_sign_batch(int mt, uint32_t count, uint8_t* sk, const uint8_t* msgs,
                                    const uint64_t* m_off, const uint64_t* mlen, uint8_t* sm,
                                    const uint64_t* sm_off, uint64_t* smlen, int* ret)
{
    if (!count) return kOk;
    const uint32_t oid = (uint32_t)be_read(sk, XMSS_OID_LEN);
    xmss_params p;
    if (parse(&p, oid, mt)) return kBad;
    const size_t sks = XMSS_OID_LEN + p.sk_bytes;
    std::vector<const uint8_t*> mp(count);
    std::vector<uint8_t*> sp(count);
    for (uint32_t r = 0; r < count; r++) {
        if ((uint32_t)be_read(sk + r * sks, XMSS_OID_LEN) != oid) {
            g_err = "xmss_b200_sign_batch: secret keys of different OIDs";
            return kBad;
        }
        mp[r] = msgs + m_off[r];
        sp[r] = sm + sm_off[r];
    }
    return sign_host(p, count, sk + XMSS_OID_LEN, sks, mp.data(), mlen, sp.data(), smlen, ret);
}

extern "C" int xmss_b200_core_hash_batch(unsigned int func, unsigned int n, uint32_t count, const uint8_t* in,
                                         const uint64_t* off, const uint64_t* len, uint8_t* out)
{
    const xb::FamilyOps* ops = xb::family_ops(func, n);
    if (!ops) return kBad;
    if (!count) return kOk;
    return guarded([&](Engine& e) {
        cudaStream_t st = e.stream();
        e.begin(st);
        uint64_t raw = 0;
        for (uint32_t i = 0; i < count; i++) raw = std::max(raw, off[i] + len[i]);
        const uint64_t span = (raw + 15) & ~15ull;
        const size_t o_off = span, o_len = o_off + count * 8, o_out = o_len + count * 8, total = o_out + count * n;
        uint8_t* d = e.d_in.as<uint8_t>(total);
        uint8_t* h = e.h_stage.as<uint8_t>(total);
        memcpy(h, in, raw);
        memcpy(h + o_off, off, count * 8);
        memcpy(h + o_len, len, count * 8);
        XB_CUDA(cudaMemcpyAsync(d, h, o_out, cudaMemcpyHostToDevice, st));
        e.core_hash(ops, count, d, (const uint64_t*)(d + o_off), (const uint64_t*)(d + o_len), d + o_out, st);
        XB_CUDA(cudaMemcpyAsync(out, d + o_out, (size_t)count * n, cudaMemcpyDeviceToHost, st));
        e.end(st);
        XB_CUDA(cudaStreamSynchronize(st));
        return kOk;
    });
}

extern "C" int xmss_b200_profile(int enable)
{
    return guarded([&](Engine& e) {
        e.profiling = enable != 0;
        return kOk;
    });
}

extern "C" int xmss_b200_phase_ms(double ms[5])
{
    return guarded([&](Engine& e) {
        e.phase_ms(ms);
        return kOk;
    });
}

extern "C" int xmss_b200_rate_probe(int kind, uint32_t blocks, uint32_t iters, uint32_t* d_sink, void* stream)
{
    if ((kind != 0 && kind != 1 && kind != 2 && (kind < 10 || kind > 19) && kind != 20 && kind != 21 && kind != 23) || !blocks ||
        !d_sink)
        return kBad;
    return guarded([&](Engine& e) {
        cudaStream_t st = (cudaStream_t)stream;
        e.begin(st);
        xb::launch_rate(kind, blocks, iters, d_sink, st);
        e.end(st);
        return kOk;
    });
}

extern "C" int xmss_b200_last_verify_work(xmss_b200_work* out)
{
    return guarded([&](Engine& e) {
        unsigned long long w[3];
        e.last_verify_work(w);
        out->hmsg_blocks = w[0];
        out->f_calls = w[1];
        out->h_calls = w[2];
        return kOk;
    });
}
