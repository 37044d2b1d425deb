// BDS ("fast") secret keys of the reference's xmss_core_fast.c builds.
//
// Such a key is the plain sk (index, SK_SEED, SK_PRF, root, PUB_SEED)
// followed by the traversal state of 2d - 1 trees (Buchmann-Dahmen-Szydlo
// authentication-path traversal: stack, authentication path, keep nodes,
// treehash instances, retained nodes) and, for XMSS^MT, the cached WOTS
// signatures of the lower roots (xmss_core_fast.c:14-148, 635-653).  The
// signatures are the same as the plain algorithm's; only the sk differs.
//
// Import keeps the plain fields.  Export rebuilds the state the reference
// holds after signing every index below the key's: it replays the
// reference's traversal (keygen, then each signature's state update) on the
// host, and every hash the traversal would compute - a leaf, or the parent
// of two nodes - is looked up in subtree node arrays built by this
// library's keygen kernels.  Replay time grows with the index.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/params.h"
#include "../../include/xmss_b200.h"
#include "../../include/xmss_core.h"
#include "engine.h"
#include "xmss_kernels.cuh"

namespace xb {
void set_last_error(const std::string& msg);  // api.cu
}

namespace {

constexpr uint64_t kMaxReplay = 1ull << 24;  // signatures an export may replay

uint64_t be_get(const uint8_t* p, unsigned len)
{
    uint64_t r = 0;
    for (unsigned i = 0; i < len; i++) r = (r << 8) | p[i];
    return r;
}

void be_put(uint8_t* p, unsigned len, uint64_t v)
{
    for (int i = (int)len - 1; i >= 0; i--, v >>= 8) p[i] = (uint8_t)v;
}

bool parse(int mt, uint32_t oid, xmss_params* p)
{
    return (mt ? xmssmt_parse_oid(p, oid) : xmss_parse_oid(p, oid)) == 0;
}

// Bytes of one tree's serialized state (xmss_core_fast.c:38-78, 635-653).
uint64_t state_bytes(const xmss_params& p)
{
    const uint64_t h = p.tree_height, n = p.n, k = p.bds_k;
    return (h + 1) * n + 4 + (h + 1) + h * n + (h >> 1) * n + (h - k) * (7 + n) + ((1ull << k) - k - 1) * n + 4;
}

uint64_t bds_sk_bytes(const xmss_params& p)
{
    return p.index_bytes + 4ull * p.n + (2ull * p.d - 1) * state_bytes(p) + (p.d - 1ull) * p.wots_sig_bytes;
}

// Node arrays of one key's subtrees, built on the GPU in batches and kept on
// the host while the replay moves forward through the trees of each layer.
class Subtrees {
   public:
    Subtrees(xb::Engine& e, const xmss_params& p, const uint8_t* keymat) : e_(e), p_(p)
    {
        ops_ = xb::ops_for(p);
        const size_t n = p.n;
        XB_CUDA(cudaSetDevice(e.device()));
        uint8_t* dk = dkey_.as<uint8_t>(4 * n);
        XB_CUDA(cudaMemcpy(dk, keymat, 4 * n, cudaMemcpyHostToDevice));
        // key row: SK_SEED | SK_PRF | root | PUB_SEED
        ops_->make_ctx(dk + 3 * n, 4 * n, dk, 4 * n, dk + n, 4 * n, 1, ctx_.get(ops_->ctx_bytes), e.stream());
        XB_CUDA(cudaStreamSynchronize(e.stream()));
        tree_bytes_ = ((2ull << p.tree_height) - 1) * n;
    }

    // n bytes of node (height, index) of subtree (layer, tree).
    const uint8_t* node(uint32_t layer, uint64_t tree, uint32_t height, uint64_t index)
    {
        auto it = cache_.find({layer, tree});
        if (it == cache_.end()) {
            build(layer, tree);
            it = cache_.find({layer, tree});
        }
        const int h = (int)p_.tree_height;
        return it->second.data() + (xb::level_offset(h, (int)height) + index) * p_.n;
    }

   private:
    void build(uint32_t layer, uint64_t first)
    {
        // drop trees of this layer the replay has left behind
        for (auto it = cache_.begin(); it != cache_.end();)
            it = (it->first.first == layer && it->first.second + 1 < first) ? cache_.erase(it) : std::next(it);
        const uint32_t shift = p_.tree_height * (layer + 1);
        const uint64_t ntrees = shift >= p_.full_height ? 1 : 1ull << (p_.full_height - shift);
        const uint64_t batch =
            std::min<uint64_t>(ntrees - first, std::max<uint64_t>(1, (64ull << 20) / tree_bytes_));
        std::vector<xb::TreeJob> jobs(batch);
        for (uint64_t t = 0; t < batch; t++) jobs[t] = xb::TreeJob{0, layer, first + t, t * tree_bytes_};
        cudaStream_t st = e_.stream();
        xb::TreeJob* dj = djobs_.as<xb::TreeJob>(batch);
        XB_CUDA(cudaMemcpyAsync(dj, jobs.data(), batch * sizeof(xb::TreeJob), cudaMemcpyHostToDevice, st));
        uint8_t* dn = dnodes_.as<uint8_t>(batch * tree_bytes_);
        e_.build_trees(ops_, dj, (uint32_t)batch, (int)p_.tree_height, dn, ctx_.get(1), st, w_,
                       xb::Engine::subtree_k(p_, (uint32_t)batch));
        std::vector<uint8_t> all(batch * tree_bytes_);
        XB_CUDA(cudaMemcpyAsync(all.data(), dn, all.size(), cudaMemcpyDeviceToHost, st));
        XB_CUDA(cudaStreamSynchronize(st));
        for (uint64_t t = 0; t < batch; t++)
            cache_[{layer, first + t}].assign(all.begin() + t * tree_bytes_, all.begin() + (t + 1) * tree_bytes_);
    }

    xb::Engine& e_;
    xmss_params p_;
    const xb::FamilyOps* ops_ = nullptr;
    uint64_t tree_bytes_ = 0;
    xb::DevBuf dkey_, ctx_, djobs_, dnodes_;
    xb::Workspace w_;
    std::map<std::pair<uint32_t, uint64_t>, std::vector<uint8_t>> cache_;
};

// Traversal state of one tree, field for field as serialized.
struct Treehash {
    uint8_t h = 0;
    uint32_t next_idx = 0;
    uint8_t stackusage = 0, completed = 0;
    std::vector<uint8_t> node;
};

struct State {
    std::vector<uint8_t> stack;  // (h + 1) nodes, stale slots included
    uint32_t stackoffset = 0;
    std::vector<uint8_t> stacklevels;
    std::vector<uint8_t> auth, keep, retain;
    std::vector<Treehash> th;
    uint32_t next_leaf = 0;
};

// The reference's traversal over one key, hashes replaced by node lookups.
class Replay {
   public:
    Replay(const xmss_params& p, Subtrees& nodes) : p_(p), nodes_(nodes), n_(p.n), h_(p.tree_height), k_(p.bds_k)
    {
        states_.resize(2 * p.d - 1);
        for (State& s : states_) {
            s.stack.assign((h_ + 1) * n_, 0);
            s.stacklevels.assign(h_ + 1, 0);
            s.auth.assign(h_ * n_, 0);
            s.keep.assign((h_ >> 1) * n_, 0);
            s.retain.assign(((1u << k_) - k_ - 1) * n_, 0);
            s.th.resize(h_ - k_);
            for (Treehash& t : s.th) t.node.assign(n_, 0);
        }
    }

    // Key generation: every layer's first tree (xmss_core_fast.c:656-709, 858-916).
    void keygen()
    {
        for (uint32_t i = 0; i < p_.d; i++) init_tree(states_[i], i, 0);
    }

    // The state update of the signature at index idx (xmss_core_fast.c:
    // 710-856 for XMSS, 917-1121 for XMSS^MT).
    void sign_update(uint64_t idx)
    {
        if (p_.d == 1) {
            if (idx < (1ull << h_) - 1) {
                round(states_[0], (uint32_t)idx, 0, 0);
                treehash_updates(states_[0], (h_ - k_) >> 1, 0, 0);
            }
            return;
        }
        const uint32_t d = p_.d, H = p_.full_height;
        const uint64_t lim = H >= 64 ? ~0ull : (1ull << H);
        int swapped_upto = -1;
        uint32_t updates = (h_ - k_) >> 1;
        uint64_t tree = idx >> h_;
        uint64_t leaf = idx & ((1ull << h_) - 1);
        if ((1 + tree) * (1ull << h_) + leaf < lim) next_leaf_update(states_[d], 0, tree + 1);
        for (uint32_t i = 0; i < d; i++) {
            const uint32_t sh = h_ * (i + 1);
            const uint64_t mask = sh >= 64 ? ~0ull : (1ull << sh) - 1;
            if (((idx + 1) & mask) != 0) {
                leaf = (idx >> (h_ * i)) & ((1ull << h_) - 1);
                tree = sh >= 64 ? 0 : idx >> sh;
                if ((int)i == swapped_upto + 1) round(states_[i], (uint32_t)leaf, i, tree);
                updates = treehash_updates(states_[i], updates, i, tree);
                const uint32_t rem = H - h_ * i;
                const uint64_t lim_i = rem >= 64 ? ~0ull : (1ull << rem);
                if ((1 + tree) * (1ull << h_) + leaf < lim_i && i > 0 && updates > 0 &&
                    states_[d + i].next_leaf < lim) {
                    next_leaf_update(states_[d + i], i, tree + 1);
                    updates--;
                }
            } else if (idx < lim - 1) {
                std::swap(states_[d + i], states_[i]);
                states_[d + i].stackoffset = 0;
                states_[d + i].next_leaf = 0;
                updates--;  // the WOTS signature of the new root counts as one update
                swapped_upto = (int)i;
                for (Treehash& t : states_[i].th) t.completed = 1;
            }
        }
    }

    // Serialized states in the key's byte order (xmss_core_fast.c:38-78).
    void serialize(uint8_t* out) const
    {
        for (const State& s : states_) {
            memcpy(out, s.stack.data(), s.stack.size());
            out += s.stack.size();
            be_put(out, 4, s.stackoffset);
            out += 4;
            memcpy(out, s.stacklevels.data(), s.stacklevels.size());
            out += s.stacklevels.size();
            memcpy(out, s.auth.data(), s.auth.size());
            out += s.auth.size();
            memcpy(out, s.keep.data(), s.keep.size());
            out += s.keep.size();
            for (const Treehash& t : s.th) {
                *out++ = t.h;
                be_put(out, 4, t.next_idx);
                out += 4;
                *out++ = t.stackusage;
                *out++ = t.completed;
                memcpy(out, t.node.data(), n_);
                out += n_;
            }
            memcpy(out, s.retain.data(), s.retain.size());
            out += s.retain.size();
            be_put(out, 4, s.next_leaf);
            out += 4;
        }
    }

   private:
    uint8_t* slot(std::vector<uint8_t>& v, size_t i) { return v.data() + i * n_; }
    void put(uint8_t* dst, const uint8_t* src) { memcpy(dst, src, n_); }
    const uint8_t* leaf(uint32_t layer, uint64_t tree, uint64_t i) { return nodes_.node(layer, tree, 0, i); }
    const uint8_t* parent(uint32_t layer, uint64_t tree, uint32_t child_height, uint64_t parent_index)
    {
        return nodes_.node(layer, tree, child_height + 1, parent_index);
    }
    size_t retain_slot(uint32_t nodeh, uint64_t i) const
    {
        return (1u << (h_ - 1 - nodeh)) + nodeh - h_ + (((i >> nodeh) - 3) >> 1);
    }

    // Node completed at height nodeh while leaf i was added: the nodes the
    // traversal keeps (authentication path of leaf 0, the next treehash
    // results, retained nodes).
    void keep_completed(State& s, uint32_t nodeh, uint64_t i, const uint8_t* v)
    {
        if ((i >> nodeh) == 1) {
            put(slot(s.auth, nodeh), v);
        } else if (nodeh < h_ - k_ && (i >> nodeh) == 3) {
            put(s.th[nodeh].node.data(), v);
        } else if (nodeh >= h_ - k_) {
            put(slot(s.retain, retain_slot(nodeh, i)), v);
        }
    }

    // treehash_init (xmss_core_fast.c:216-284): the whole tree through a
    // local stack; the state's own stack is untouched.
    void init_tree(State& s, uint32_t layer, uint64_t tree)
    {
        for (uint32_t i = 0; i < h_ - k_; i++) {
            s.th[i].h = (uint8_t)i;
            s.th[i].completed = 1;
            s.th[i].stackusage = 0;
        }
        std::vector<uint8_t> stack((h_ + 1) * n_, 0);
        std::vector<uint32_t> levels(h_ + 1, 0);
        uint32_t so = 0;
        for (uint64_t i = 0; i < (1ull << h_); i++) {
            put(slot(stack, so), leaf(layer, tree, i));
            levels[so] = 0;
            so++;
            if (h_ - k_ > 0 && i == 3) put(s.th[0].node.data(), slot(stack, so));
            while (so > 1 && levels[so - 1] == levels[so - 2]) {
                const uint32_t nodeh = levels[so - 1];
                keep_completed(s, nodeh, i, slot(stack, so - 1));
                put(slot(stack, so - 2), parent(layer, tree, nodeh, i >> (nodeh + 1)));
                levels[so - 2]++;
                so--;
            }
        }
    }

    // treehash_update (xmss_core_fast.c:406-450)
    void treehash_update(State& s, Treehash& t, uint32_t layer, uint64_t tree)
    {
        const uint8_t* v = leaf(layer, tree, t.next_idx);
        uint32_t height = 0;
        while (t.stackusage > 0 && s.stacklevels[s.stackoffset - 1] == height) {
            v = parent(layer, tree, height, t.next_idx >> (height + 1));
            height++;
            t.stackusage--;
            s.stackoffset--;
        }
        if (height == t.h) {
            put(t.node.data(), v);
            t.completed = 1;
        } else {
            put(slot(s.stack, s.stackoffset), v);
            t.stackusage++;
            s.stacklevels[s.stackoffset] = (uint8_t)height;
            s.stackoffset++;
            t.next_idx++;
        }
    }

    uint32_t min_height_on_stack(const State& s, const Treehash& t) const
    {
        uint32_t r = h_;
        for (uint32_t i = 0; i < t.stackusage; i++) r = std::min<uint32_t>(r, s.stacklevels[s.stackoffset - i - 1]);
        return r;
    }

    // bds_treehash_update (xmss_core_fast.c:458-494): spend up to `updates`
    // leaf computations on the instance with the lowest pending node.  The
    // reference returns the remainder as a (signed) char into an unsigned
    // int, which matters once a swap has taken the budget below zero.
    uint32_t treehash_updates(State& s, uint32_t updates, uint32_t layer, uint64_t tree)
    {
        uint32_t used = 0;
        for (uint32_t j = 0; j < updates; j++) {
            uint32_t l_min = h_, level = h_ - k_;
            for (uint32_t i = 0; i < h_ - k_; i++) {
                const Treehash& t = s.th[i];
                const uint32_t low = t.completed ? h_ : (t.stackusage == 0 ? i : min_height_on_stack(s, t));
                if (low < l_min) {
                    level = i;
                    l_min = low;
                }
            }
            if (level == h_ - k_) break;
            treehash_update(s, s.th[level], layer, tree);
            used++;
        }
        return (uint32_t)(int32_t)(int8_t)(uint8_t)(updates - used);
    }

    // bds_state_update (xmss_core_fast.c:500-553): one more leaf of the next
    // tree onto its stack.
    void next_leaf_update(State& s, uint32_t layer, uint64_t tree)
    {
        const uint64_t i = s.next_leaf;
        if (i == (1ull << h_)) return;
        put(slot(s.stack, s.stackoffset), leaf(layer, tree, i));
        s.stacklevels[s.stackoffset] = 0;
        s.stackoffset++;
        if (h_ - k_ > 0 && i == 3) put(s.th[0].node.data(), slot(s.stack, s.stackoffset));
        while (s.stackoffset > 1 && s.stacklevels[s.stackoffset - 1] == s.stacklevels[s.stackoffset - 2]) {
            const uint32_t nodeh = s.stacklevels[s.stackoffset - 1];
            keep_completed(s, nodeh, i, slot(s.stack, s.stackoffset - 1));
            put(slot(s.stack, s.stackoffset - 2), parent(layer, tree, nodeh, i >> (nodeh + 1)));
            s.stacklevels[s.stackoffset - 2]++;
            s.stackoffset--;
        }
        s.next_leaf++;
    }

    // bds_round (xmss_core_fast.c:559-633): the authentication path of leaf
    // leaf_idx + 1 from that of leaf_idx.
    void round(State& s, uint32_t leaf_idx, uint32_t layer, uint64_t tree)
    {
        uint32_t tau = h_;
        for (uint32_t i = 0; i < h_; i++)
            if (!((leaf_idx >> i) & 1)) {
                tau = i;
                break;
            }
        if (!((leaf_idx >> (tau + 1)) & 1) && tau < h_ - 1) put(slot(s.keep, tau >> 1), slot(s.auth, tau));
        if (tau == 0) {
            put(slot(s.auth, 0), leaf(layer, tree, leaf_idx));
            return;
        }
        put(slot(s.auth, tau), parent(layer, tree, tau - 1, leaf_idx >> tau));
        for (uint32_t i = 0; i < tau; i++) {
            if (i < h_ - k_) {
                put(slot(s.auth, i), s.th[i].node.data());
            } else {
                const size_t off = (1u << (h_ - 1 - i)) + i - h_, row = ((leaf_idx >> i) - 1) >> 1;
                put(slot(s.auth, i), slot(s.retain, off + row));
            }
        }
        for (uint32_t i = 0; i < std::min(tau, h_ - k_); i++) {
            const uint64_t start = (uint64_t)leaf_idx + 1 + 3ull * (1ull << i);
            if (start < (1ull << h_)) {
                s.th[i].h = (uint8_t)i;
                s.th[i].next_idx = (uint32_t)start;
                s.th[i].completed = 0;
                s.th[i].stackusage = 0;
            }
        }
    }

    xmss_params p_;
    Subtrees& nodes_;
    const uint32_t n_, h_, k_;
    std::vector<State> states_;
};

}  // namespace

extern "C" unsigned long long xmss_b200_bds_sk_bytes(uint32_t oid, int mt)
{
    xmss_params p;
    if (!parse(mt, oid, &p)) return 0;
    return bds_sk_bytes(p);
}

extern "C" int xmss_b200_sk_from_bds(int mt, const uint8_t* bds_sk, uint8_t* sk)
{
    xmss_params p;
    const uint32_t oid = (uint32_t)be_get(bds_sk, XMSS_OID_LEN);
    if (!parse(mt, oid, &p)) return -1;
    memcpy(sk, bds_sk, XMSS_OID_LEN + p.index_bytes + 4 * p.n);  // OID, index, SK_SEED, SK_PRF, root, PUB_SEED
    return 0;
}

extern "C" int xmss_b200_sk_to_bds(int mt, const uint8_t* sk, uint8_t* bds_sk)
{
    xmss_params p;
    const uint32_t oid = (uint32_t)be_get(sk, XMSS_OID_LEN);
    if (!parse(mt, oid, &p)) return -1;
    const uint64_t idx = be_get(sk + XMSS_OID_LEN, p.index_bytes);
    const uint64_t last = p.full_height >= 64 ? ~0ull : (1ull << p.full_height) - 1;
    const size_t plain = p.index_bytes + 4ull * p.n;
    uint8_t* out = bds_sk + XMSS_OID_LEN;
    memcpy(bds_sk, sk, XMSS_OID_LEN + plain);
    memset(out + plain, 0, bds_sk_bytes(p) - plain);
    if (idx > last) return 0;  // a wiped key: index all ones, everything else zero (as the reference leaves it)
    if (idx > kMaxReplay) {
        xb::set_last_error("xmss_b200_sk_to_bds: index above 2^24, too many signatures to replay");
        return -1;
    }
    try {
        xb::Engine& e = xb::Engine::get();
        std::lock_guard<std::mutex> g(e.mu);
        Subtrees nodes(e, p, sk + XMSS_OID_LEN + p.index_bytes);
        Replay r(p, nodes);
        r.keygen();
        for (uint64_t i = 0; i < idx; i++) r.sign_update(i);
        r.serialize(out + plain);
    } catch (const std::exception& ex) {
        xb::set_last_error(std::string("xmss_b200_sk_to_bds: ") + ex.what());
        return -3;
    }
    if (p.d > 1) {
        // cached WOTS signatures of the lower roots: those the signature at
        // idx carries for layers 1 .. d-1
        std::vector<uint8_t> skc(sk + XMSS_OID_LEN, sk + XMSS_OID_LEN + p.sk_bytes), sm(p.sig_bytes);
        unsigned long long smlen = 0;
        const int rc = xmssmt_core_sign(&p, skc.data(), sm.data(), &smlen, sm.data(), 0);
        if (rc != 0) return rc;
        const size_t layer_bytes = p.wots_sig_bytes + (size_t)p.tree_height * p.n;
        uint8_t* wots = out + plain + (2ull * p.d - 1) * state_bytes(p);
        for (uint32_t i = 1; i < p.d; i++)
            memcpy(wots + (i - 1) * p.wots_sig_bytes, sm.data() + p.index_bytes + p.n + i * layer_bytes,
                   p.wots_sig_bytes);
    }
    return 0;
}
