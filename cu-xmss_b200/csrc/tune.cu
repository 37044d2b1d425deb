// Launch-shape table per hash family and the autotuner that fills it
// (xmss_b200_tuning_get / _set, xmss_b200_autotune).
//
// The knobs are the CTA sizes of the chain kernels (verify; keygen and
// sign), of the L-tree / Merkle-level kernels, and the split of large verify
// batches into a short- and a long-H_msg group (the batch size from which
// it applies, the H_msg length that separates the groups, whether the
// L-tree precomputation runs as a launch of its own).  The tuner builds
// its own synthetic batch of the parameter set (seeded keys and signatures
// of messages log-uniform in 32 B..4 KB, made by this library), times each
// candidate with CUDA events (median of seven after a warm-up run, L2
// flushed before each), checks that every candidate accepts every
// signature, searches one knob at a time and moves a knob only for a
// candidate at least 2 % faster than its current value.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <random>
#include <tuple>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/params.h"
#include "../../include/xmss_b200.h"
#include "engine.h"
#include "xmss_kernels.cuh"

namespace xb {
void set_last_error(const std::string& msg);  // api.cu

Tuning& tuning_for(unsigned func, unsigned n)
{
    static Tuning table[3][3];  // func x (n = 24, 32, 64)
    const unsigned f = func < 3 ? func : 0;
    const unsigned i = n == 24 ? 0 : (n == 64 ? 2 : 1);
    return table[f][i];
}

TreeShape& tree_shape_for(unsigned func, unsigned n, unsigned full_height, unsigned d)
{
    // (func, n, full height, layers) names one parameter set of params.c
    static std::mutex mu;
    static std::map<std::tuple<unsigned, unsigned, unsigned, unsigned>, TreeShape> table;
    std::lock_guard<std::mutex> g(mu);
    return table[std::make_tuple(func, n, full_height, d)];
}

int subtree_height_for(const TreeShape& s, int h, uint64_t leaves)
{
    const int k = (int)s.subtree_height;
    if (k < 5 || k > 7 || leaves < s.min_leaves) return 0;
    return h >= k ? k : (h >= 5 ? h : 0);
}
}  // namespace xb

namespace {

// The kernels are compiled for at most 128 threads per CTA (a higher bound
// costs the 168-register families an SM-resident CTA).
bool block_ok(uint32_t b) { return b == 32 || b == 64 || b == 128; }

void to_c(const xb::Tuning& t, xmss_b200_tuning* o)
{
    o->verify_chain_block = t.verify_chain_block;
    o->keygen_chain_block = t.keygen_chain_block;
    o->level_block = t.level_block;
    o->split_min = t.split_min;
    o->short_hmsg_blocks = t.short_hmsg_blocks;
    o->prep_split = t.prep_split;
}

}  // namespace

extern "C" int xmss_b200_tuning_get(unsigned func, unsigned n, xmss_b200_tuning* out)
{
    if (!xb::family_ops(func, n) || !out) return -1;
    to_c(xb::tuning_for(func, n), out);
    return 0;
}

extern "C" int xmss_b200_tuning_set(unsigned func, unsigned n, const xmss_b200_tuning* t)
{
    if (!xb::family_ops(func, n) || !t || !block_ok(t->verify_chain_block) || !block_ok(t->keygen_chain_block) ||
        !block_ok(t->level_block) || !t->split_min || !t->short_hmsg_blocks || t->prep_split > 1) {
        xb::set_last_error("xmss_b200_tuning_set: unknown family or shape out of range");
        return -1;
    }
    // plain stores: set shapes while no call of this family is launching
    xb::Tuning& d = xb::tuning_for(func, n);
    d.verify_chain_block = t->verify_chain_block;
    d.keygen_chain_block = t->keygen_chain_block;
    d.level_block = t->level_block;
    d.split_min = t->split_min;
    d.short_hmsg_blocks = t->short_hmsg_blocks;
    d.prep_split = t->prep_split;
    return 0;
}

namespace {

xb::TreeShape* shape_of(uint32_t oid, int mt, xmss_params* p)
{
    if ((mt ? xmssmt_parse_oid(p, oid) : xmss_parse_oid(p, oid)) != 0 || !xb::family_ops(p->func, p->n)) return nullptr;
    return &xb::tree_shape_for(p->func, p->n, p->full_height, p->d);
}

}  // namespace

extern "C" int xmss_b200_tree_tuning_get(uint32_t oid, int mt, xmss_b200_tree_tuning* out)
{
    xmss_params p;
    const xb::TreeShape* s = shape_of(oid, mt, &p);
    if (!s || !out) return -1;
    out->subtree_height = s->subtree_height;
    out->chains_per_warp = s->subtree_height ? 32 * p.wots_len : 32;
    out->min_leaves = s->min_leaves;
    return 0;
}

extern "C" int xmss_b200_tree_tuning_set(uint32_t oid, int mt, const xmss_b200_tree_tuning* t)
{
    xmss_params p;
    xb::TreeShape* s = shape_of(oid, mt, &p);
    if (!s || !t || (t->subtree_height != 0 && (t->subtree_height < 5 || t->subtree_height > 7))) {
        xb::set_last_error("xmss_b200_tree_tuning_set: unknown OID or subtree height other than 0, 5, 6, 7");
        return -1;
    }
    s->subtree_height = t->subtree_height;
    s->min_leaves = t->min_leaves;
    return 0;
}

extern "C" int xmss_b200_autotune(uint32_t oid, int mt, uint32_t count, xmss_b200_tuning* best, char* report,
                                  size_t report_cap)
{
    xmss_params p;
    if ((mt ? xmssmt_parse_oid(&p, oid) : xmss_parse_oid(&p, oid)) != 0 || count < 64 || count > (1u << 20)) {
        xb::set_last_error("xmss_b200_autotune: unknown OID or count outside 64..2^20");
        return -1;
    }
    std::string rep;
    try {
        xb::Engine& e = xb::Engine::get();
        std::lock_guard<std::mutex> lk(e.mu);
        XB_CUDA(cudaSetDevice(e.device()));
        const xb::FamilyOps* ops = xb::ops_for(p);
        xb::Tuning& tn = xb::tuning_for(p.func, p.n);
        cudaStream_t st = e.stream();
        xb::Workspace w;
        xb::SplitStreams ss;
        ss.create();
        w.split = &ss;
        const size_t n = p.n;

        // ---- synthetic batch: keys, then signatures at indices of each
        // key's first subtrees (so that signing builds few of them) ----
        std::mt19937_64 rng(0x5EEDull ^ oid ^ ((uint64_t)mt << 32));
        const uint32_t nk = p.tree_height >= 16 ? 2 : 16;  // keygen of big subtrees takes seconds
        std::vector<uint8_t> seeds((size_t)nk * 3 * n);
        for (auto& b : seeds) b = (uint8_t)rng();
        xb::DevBuf d_seeds, d_pk, d_sk, d_sm, d_off, d_len, d_kix, d_st, d_tree_jobs, d_tree_nodes;
        XB_CUDA(cudaMemcpy(d_seeds.get(seeds.size()), seeds.data(), seeds.size(), cudaMemcpyHostToDevice));
        e.keypair(ops, p, nk, d_seeds.as<uint8_t>(0), d_pk.as<uint8_t>((size_t)nk * 2 * n),
                  d_sk.as<uint8_t>((size_t)nk * p.sk_bytes), st, w);
        std::vector<uint8_t> sk((size_t)nk * p.sk_bytes);
        XB_CUDA(cudaMemcpyAsync(sk.data(), d_sk.get(1), sk.size(), cudaMemcpyDeviceToHost, st));
        XB_CUDA(cudaStreamSynchronize(st));
        const uint64_t idx_span = std::min<uint64_t>(1ull << std::min(p.tree_height, 20u),
                                                     (1ull << std::min(p.full_height, 62u)) - 1);
        std::vector<uint8_t> rows((size_t)count * p.sk_bytes);
        std::vector<uint64_t> idx(count), off(count), mlen(count), smlen(count);
        std::vector<uint32_t> kix(count);
        uint64_t total = 0;
        for (uint32_t r = 0; r < count; r++) {
            kix[r] = r % nk;
            idx[r] = rng() % idx_span;
            memcpy(&rows[(size_t)r * p.sk_bytes], &sk[(size_t)kix[r] * p.sk_bytes], p.sk_bytes);
            for (unsigned b = 0; b < p.index_bytes; b++)
                rows[(size_t)r * p.sk_bytes + b] = (uint8_t)(idx[r] >> (8 * (p.index_bytes - 1 - b)));
            mlen[r] = (uint64_t)std::exp(std::log(32.0) + (std::log(4096.0) - std::log(32.0)) *
                                                              ((double)(rng() >> 11) / (double)(1ull << 53)));
            off[r] = total;
            smlen[r] = p.sig_bytes + mlen[r];
            total += (smlen[r] + 15) & ~15ull;
        }
        std::vector<uint8_t> sm(total);
        for (uint32_t r = 0; r < count; r++) {
            // the signing kernels write everything after the index bytes
            for (unsigned b = 0; b < p.index_bytes; b++)
                sm[off[r] + b] = (uint8_t)(idx[r] >> (8 * (p.index_bytes - 1 - b)));
            for (uint64_t i = 0; i < mlen[r]; i++) sm[off[r] + p.sig_bytes + i] = (uint8_t)rng();
        }
        XB_CUDA(cudaMemcpy(d_sm.get(total), sm.data(), total, cudaMemcpyHostToDevice));
        XB_CUDA(cudaMemcpy(d_off.get(count * 8), off.data(), count * 8, cudaMemcpyHostToDevice));
        XB_CUDA(cudaMemcpy(d_len.get(count * 8), mlen.data(), count * 8, cudaMemcpyHostToDevice));
        e.sign(ops, p, count, rows.data(), idx.data(), d_sm.as<uint8_t>(0), d_off.as<uint64_t>(0),
               d_len.as<uint64_t>(0), st, w);
        XB_CUDA(cudaMemcpy(d_len.get(count * 8), smlen.data(), count * 8, cudaMemcpyHostToDevice));
        XB_CUDA(cudaMemcpy(d_kix.get(count * 4), kix.data(), count * 4, cudaMemcpyHostToDevice));
        int* status = d_st.as<int>(count);

        // keygen slice: 2^12 leaves in subtrees of height min(h, 12)
        const int kh = (int)std::min(p.tree_height, 12u);
        const uint32_t kjobs = 1u << (12 - kh);
        const uint64_t tree_bytes = ((2ull << kh) - 1) * n;
        std::vector<xb::TreeJob> jobs(kjobs);
        for (uint32_t j = 0; j < kjobs; j++) jobs[j] = xb::TreeJob{j % nk, 0, j / nk, j * tree_bytes};
        XB_CUDA(cudaMemcpy(d_tree_jobs.get(kjobs * sizeof(xb::TreeJob)), jobs.data(), kjobs * sizeof(xb::TreeJob),
                           cudaMemcpyHostToDevice));
        xb::DevBuf kctx_buf;
        void* gctx = kctx_buf.get((size_t)nk * ops->ctx_bytes);
        {
            // the keygen slice needs the secret seeds: contexts from the key rows
            std::vector<uint8_t> mat((size_t)nk * 4 * n);
            for (uint32_t k = 0; k < nk; k++)
                memcpy(&mat[(size_t)k * 4 * n], &sk[(size_t)k * p.sk_bytes + p.index_bytes], 4 * n);
            xb::DevBuf d_mat;
            XB_CUDA(cudaMemcpy(d_mat.get(mat.size()), mat.data(), mat.size(), cudaMemcpyHostToDevice));
            uint8_t* dm = d_mat.as<uint8_t>(0);
            ops->make_ctx(dm + 3 * n, 4 * n, dm, 4 * n, dm + n, 4 * n, nk, gctx, st);
            XB_CUDA(cudaStreamSynchronize(st));
        }

        cudaEvent_t a, b;
        XB_CUDA(cudaEventCreate(&a));
        XB_CUDA(cudaEventCreate(&b));
        // L2 (126 MB) is flushed before every timed run, as production calls
        // find it: inputs and scratch arrive from HBM
        xb::DevBuf flush;
        void* fl = flush.get(256ull << 20);
        auto timed = [&](auto&& run) {
            run();
            std::vector<float> t;
            for (int i = 0; i < 7; i++) {
                XB_CUDA(cudaMemsetAsync(fl, i, 256ull << 20, st));
                XB_CUDA(cudaEventRecord(a, st));
                run();
                XB_CUDA(cudaEventRecord(b, st));
                XB_CUDA(cudaEventSynchronize(b));
                float ms = 0;
                XB_CUDA(cudaEventElapsedTime(&ms, a, b));
                t.push_back(ms);
            }
            std::sort(t.begin(), t.end());
            return (double)t[3];
        };
        std::vector<int> h_status(count);
        auto verify_ms = [&]() {
            const double ms = timed([&] {
                e.verify(ops, p, count, d_sm.as<uint8_t>(0), d_off.as<uint64_t>(0), d_len.as<uint64_t>(0),
                         d_pk.as<uint8_t>(0), nk, d_kix.as<uint32_t>(0), status, st, w, true);
            });
            XB_CUDA(cudaMemcpy(h_status.data(), status, count * 4, cudaMemcpyDeviceToHost));
            for (int s : h_status)
                if (s != 0) throw std::runtime_error("a candidate shape rejected a valid signature");
            return ms;
        };
        auto keygen_ms = [&]() {
            return timed([&] {
                e.build_trees(ops, d_tree_jobs.as<xb::TreeJob>(0), kjobs, kh,
                              d_tree_nodes.as<uint8_t>(kjobs * tree_bytes), gctx, st, w);
            });
        };

        char line[256];
        rep = "{\"oid\": " + std::to_string(oid) + ", \"mt\": " + std::to_string(mt) + ", \"func\": " +
              std::to_string(p.func) + ", \"n\": " + std::to_string(p.n) + ", \"count\": " + std::to_string(count) +
              ", \"trials\": [";
        bool first = true;
        auto note = [&](const char* knob, uint32_t v, double vms, double kms) {
            snprintf(line, sizeof line, "%s{\"knob\": \"%s\", \"value\": %u, \"verify_ms\": %.4f, \"keygen_ms\": %.4f}",
                     first ? "" : ", ", knob, v, vms, kms);
            rep += line;
            first = false;
        };
        // A knob leaves its current value only for a candidate at least 2 %
        // faster: smaller differences are within run-to-run noise.
        constexpr double kGain = 0.98;
        const uint32_t blocks[3] = {32, 64, 128};
        auto pick = [&](uint32_t& knob, const char* name, auto&& cost) {
            const uint32_t cur = knob;
            double cur_t = 0, bt = 1e30;
            uint32_t bestv = cur;
            for (uint32_t v : blocks) {
                knob = v;
                const double t = cost(name, v);
                if (v == cur) cur_t = t;
                if (t < bt) bt = t, bestv = v;
            }
            knob = bt < kGain * cur_t ? bestv : cur;
        };
        // 1. verify chains; 2. level kernels (both pipelines use them);
        // 3. keygen / sign chains
        pick(tn.verify_chain_block, "verify_chain_block", [&](const char* k, uint32_t v) {
            const double ms = verify_ms();
            note(k, v, ms, -1);
            return ms;
        });
        pick(tn.level_block, "level_block", [&](const char* k, uint32_t v) {
            const double vm = verify_ms(), km = keygen_ms();
            note(k, v, vm, km);
            return vm + km;
        });
        pick(tn.keygen_chain_block, "keygen_chain_block", [&](const char* k, uint32_t v) {
            const double km = keygen_ms();
            note(k, v, -1, km);
            return km;
        });
        // 4. split of this batch size: as it is, off, or on at each H_msg boundary
        {
            const uint32_t keep_min = tn.split_min, keep_short = tn.short_hmsg_blocks;
            const double cur_t = verify_ms();
            note("split_current", count >= keep_min ? keep_short : 0, cur_t, -1);
            double bt = 1e30;
            uint32_t best_min = keep_min, best_short = keep_short;
            tn.split_min = count + 1;
            const double off_t = verify_ms();
            note("split_off", 0, off_t, -1);
            if (off_t < bt) bt = off_t, best_min = count + 1;
            for (uint32_t sb : {8u, 16u, 32u}) {
                tn.split_min = count;
                tn.short_hmsg_blocks = sb;
                const double ms = verify_ms();
                note("short_hmsg_blocks", sb, ms, -1);
                if (ms < bt) bt = ms, best_min = count, best_short = sb;
            }
            if (bt < kGain * cur_t) {
                // batches from this size on follow the choice; smaller ones
                // keep the previous threshold when it was lower
                tn.split_min = best_min == count ? std::min(keep_min, count) : std::max(keep_min, count + 1);
                tn.short_hmsg_blocks = best_short;
            } else {
                tn.split_min = keep_min;
                tn.short_hmsg_blocks = keep_short;
            }
        }
        // 5. where this batch splits: h_pre in its own launch or in each group's prep
        if (count >= tn.split_min) {
            const uint32_t keep = tn.prep_split;
            const double cur_t = verify_ms();
            note("prep_split", keep, cur_t, -1);
            tn.prep_split = 1 - keep;
            const double alt_t = verify_ms();
            note("prep_split", tn.prep_split, alt_t, -1);
            if (!(alt_t < kGain * cur_t)) tn.prep_split = keep;
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        XB_CUDA(cudaStreamSynchronize(st));
        ss.destroy();
        xmss_b200_tuning bt;
        to_c(tn, &bt);
        if (best) *best = bt;
        snprintf(line, sizeof line,
                 "], \"best\": {\"verify_chain_block\": %u, \"keygen_chain_block\": %u, \"level_block\": %u, "
                 "\"split_min\": %u, \"short_hmsg_blocks\": %u, \"prep_split\": %u}}",
                 bt.verify_chain_block, bt.keygen_chain_block, bt.level_block, bt.split_min, bt.short_hmsg_blocks,
                 bt.prep_split);
        rep += line;
    } catch (const std::exception& ex) {
        xb::set_last_error(std::string("xmss_b200_autotune: ") + ex.what());
        return -3;
    }
    if (report && report_cap) {
        const size_t k = std::min(report_cap - 1, rep.size());
        memcpy(report, rep.data(), k);
        report[k] = 0;
    }
    return 0;
}

// Tree-building shape of one parameter set: keygen of slices of 2^12, 2^15
// and 2^18 leaves (subtrees of the set's height, seeded keys, L2 flushed
// before each timed run, median of five), one thread per chain against
// in-CTA subtrees of height 5, 6 and 7; every candidate's node arrays must
// equal those of the one-thread-per-chain form.  The best in-CTA height at
// the largest slice is kept if it is at least 2 % faster there, with
// min_leaves = the smallest slice at which it still is.
extern "C" int xmss_b200_autotune_tree(uint32_t oid, int mt, xmss_b200_tree_tuning* best, char* report,
                                       size_t report_cap)
{
    xmss_params p;
    xb::TreeShape* shape = shape_of(oid, mt, &p);
    if (!shape) {
        xb::set_last_error("xmss_b200_autotune_tree: unknown OID");
        return -1;
    }
    std::string rep;
    try {
        xb::Engine& e = xb::Engine::get();
        std::lock_guard<std::mutex> lk(e.mu);
        XB_CUDA(cudaSetDevice(e.device()));
        const xb::FamilyOps* ops = xb::ops_for(p);
        cudaStream_t st = e.stream();
        xb::Workspace w;
        const size_t n = p.n;
        const int h = (int)p.tree_height;
        constexpr uint32_t nk = 4;
        std::mt19937_64 rng(0x7EE5ull ^ oid ^ ((uint64_t)mt << 32));
        std::vector<uint8_t> mat((size_t)nk * 4 * n);
        for (auto& b : mat) b = (uint8_t)rng();
        xb::DevBuf d_mat, d_ctx, d_jobs, d_nodes, d_ref, flush;
        XB_CUDA(cudaMemcpy(d_mat.get(mat.size()), mat.data(), mat.size(), cudaMemcpyHostToDevice));
        uint8_t* dm = d_mat.as<uint8_t>(0);
        void* ctx = d_ctx.get((size_t)nk * ops->ctx_bytes);
        ops->make_ctx(dm + 3 * n, 4 * n, dm, 4 * n, dm + n, 4 * n, nk, ctx, st);
        void* fl = flush.get(256ull << 20);
        cudaEvent_t a, b;
        XB_CUDA(cudaEventCreate(&a));
        XB_CUDA(cudaEventCreate(&b));
        char line[256];
        rep = "{\"oid\": " + std::to_string(oid) + ", \"mt\": " + std::to_string(mt) + ", \"trials\": [";
        bool first = true;
        const int sizes[3] = {12, 15, 18};
        double t_at[3][8] = {};
        for (int si = 0; si < 3; si++) {
            const int lg = std::max(sizes[si], h);  // at least one subtree
            const uint32_t njobs = 1u << (lg - h);
            const uint64_t tree_bytes = ((2ull << h) - 1) * n;
            std::vector<xb::TreeJob> jobs(njobs);
            for (uint32_t j = 0; j < njobs; j++) jobs[j] = xb::TreeJob{j % nk, 0, j / nk, j * tree_bytes};
            XB_CUDA(cudaMemcpy(d_jobs.get(njobs * sizeof(xb::TreeJob)), jobs.data(), njobs * sizeof(xb::TreeJob),
                               cudaMemcpyHostToDevice));
            const size_t bytes = (size_t)njobs * tree_bytes;
            uint8_t* nodes = d_nodes.as<uint8_t>(bytes);
            uint8_t* ref = d_ref.as<uint8_t>(bytes);
            std::vector<uint8_t> h_ref(bytes), h_got(bytes);
            for (int k : {0, 5, 6, 7}) {
                if (k > h) continue;
                auto run = [&] {
                    e.build_trees(ops, d_jobs.as<xb::TreeJob>(0), njobs, h, nodes, ctx, st, w, k);
                };
                run();
                std::vector<float> t;
                for (int i = 0; i < 5; i++) {
                    XB_CUDA(cudaMemsetAsync(fl, i, 256ull << 20, st));
                    XB_CUDA(cudaEventRecord(a, st));
                    run();
                    XB_CUDA(cudaEventRecord(b, st));
                    XB_CUDA(cudaEventSynchronize(b));
                    float ms = 0;
                    XB_CUDA(cudaEventElapsedTime(&ms, a, b));
                    t.push_back(ms);
                }
                std::sort(t.begin(), t.end());
                t_at[si][k] = t[2];
                if (k == 0) {
                    XB_CUDA(cudaMemcpy(h_ref.data(), nodes, bytes, cudaMemcpyDeviceToHost));
                } else {
                    XB_CUDA(cudaMemcpy(h_got.data(), nodes, bytes, cudaMemcpyDeviceToHost));
                    if (h_got != h_ref) throw std::runtime_error("in-CTA subtrees differ from the per-chain form");
                }
                snprintf(line, sizeof line, "%s{\"leaves_log2\": %d, \"subtree_height\": %d, \"ms\": %.4f}",
                         first ? "" : ", ", lg, k, (double)t[2]);
                rep += line;
                first = false;
            }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        constexpr double kGain = 0.98;
        int kb = 0;
        for (int k : {5, 6, 7})
            if (k <= h && t_at[2][k] > 0 && t_at[2][k] < kGain * t_at[2][0] &&
                (kb == 0 || t_at[2][k] < t_at[2][kb]))
                kb = k;
        uint64_t min_leaves = 0;
        if (kb) {
            min_leaves = 1ull << std::max(sizes[2], h);
            for (int si = 1; si >= 0; si--) {
                if (t_at[si][kb] > 0 && t_at[si][kb] < kGain * t_at[si][0])
                    min_leaves = 1ull << std::max(sizes[si], h);
                else
                    break;
            }
        }
        shape->subtree_height = (uint32_t)kb;
        shape->min_leaves = min_leaves;
        xmss_b200_tree_tuning out;
        xmss_b200_tree_tuning_get(oid, mt, &out);
        if (best) *best = out;
        snprintf(line, sizeof line, "], \"best\": {\"subtree_height\": %u, \"chains_per_warp\": %u, \"min_leaves\": %llu}}",
                 out.subtree_height, out.chains_per_warp, (unsigned long long)out.min_leaves);
        rep += line;
    } catch (const std::exception& ex) {
        xb::set_last_error(std::string("xmss_b200_autotune_tree: ") + ex.what());
        return -3;
    }
    if (report && report_cap) {
        const size_t k = std::min(report_cap - 1, rep.size());
        memcpy(report, rep.data(), k);
        report[k] = 0;
    }
    return 0;
}
