// Run-time parameter tables (the reference's params.c API, cuxmss/params.c).
//
// The 21 XMSS sets are listed by name; the 56 XMSS^MT sets are generated
// from their structure: OIDs come in blocks of eight (h, d) shapes per hash
// family (params.c:78-252 names, params.c:377-698 values).
#include <cstdio>
#include <cstring>

#include "../../include/params.h"

namespace {

struct XmssSet {
    const char* name;
    unsigned func, n, h;
};

// OID = index + 1 (params.c:7-76, 254-375)
const XmssSet kXmss[21] = {
    {"XMSS-SHA2_10_256", XMSS_SHA2, 32, 10},     {"XMSS-SHA2_16_256", XMSS_SHA2, 32, 16},
    {"XMSS-SHA2_20_256", XMSS_SHA2, 32, 20},     {"XMSS-SHA2_10_512", XMSS_SHA2, 64, 10},
    {"XMSS-SHA2_16_512", XMSS_SHA2, 64, 16},     {"XMSS-SHA2_20_512", XMSS_SHA2, 64, 20},
    {"XMSS-SHAKE_10_256", XMSS_SHAKE128, 32, 10}, {"XMSS-SHAKE_16_256", XMSS_SHAKE128, 32, 16},
    {"XMSS-SHAKE_20_256", XMSS_SHAKE128, 32, 20}, {"XMSS-SHAKE_10_512", XMSS_SHAKE256, 64, 10},
    {"XMSS-SHAKE_16_512", XMSS_SHAKE256, 64, 16}, {"XMSS-SHAKE_20_512", XMSS_SHAKE256, 64, 20},
    {"XMSS-SHA2_10_192", XMSS_SHA2, 24, 10},     {"XMSS-SHA2_16_192", XMSS_SHA2, 24, 16},
    {"XMSS-SHA2_20_192", XMSS_SHA2, 24, 20},     {"XMSS-SHAKE256_10_256", XMSS_SHAKE256, 32, 10},
    {"XMSS-SHAKE256_16_256", XMSS_SHAKE256, 32, 16}, {"XMSS-SHAKE256_20_256", XMSS_SHAKE256, 32, 20},
    {"XMSS-SHAKE256_10_192", XMSS_SHAKE256, 24, 10}, {"XMSS-SHAKE256_16_192", XMSS_SHAKE256, 24, 16},
    {"XMSS-SHAKE256_20_192", XMSS_SHAKE256, 24, 20},
};

// XMSS^MT shapes inside each block of eight OIDs.
const unsigned kMtH[8] = {20, 20, 40, 40, 40, 60, 60, 60};
const unsigned kMtD[8] = {2, 4, 2, 4, 8, 3, 6, 12};

struct MtFamily {
    const char* prefix;
    const char* suffix;
    unsigned func, n;
};
const MtFamily kMtFam[7] = {
    {"XMSSMT-SHA2_", "_256", XMSS_SHA2, 32},      {"XMSSMT-SHA2_", "_512", XMSS_SHA2, 64},
    {"XMSSMT-SHAKE_", "_256", XMSS_SHAKE128, 32}, {"XMSSMT-SHAKE_", "_512", XMSS_SHAKE256, 64},
    {"XMSSMT-SHA2_", "_192", XMSS_SHA2, 24},      {"XMSSMT-SHAKE256_", "_256", XMSS_SHAKE256, 32},
    {"XMSSMT-SHAKE256_", "_192", XMSS_SHAKE256, 24},
};

int finish(xmss_params* p, unsigned func, unsigned n, unsigned h, unsigned d)
{
    p->func = func;
    p->n = n;
    p->padding_len = (n == 24) ? 4 : n;
    p->full_height = h;
    p->d = d;
    p->wots_w = 16;
    p->bds_k = 0;
    return xmss_xmssmt_initialize_params(p);
}

}  // namespace

extern "C" int xmss_str_to_oid(uint32_t* oid, const char* s)
{
    for (unsigned i = 0; i < 21; i++) {
        if (!strcmp(s, kXmss[i].name)) {
            *oid = i + 1;
            return 0;
        }
    }
    return -1;
}

extern "C" int xmssmt_str_to_oid(uint32_t* oid, const char* s)
{
    char buf[64];
    for (unsigned f = 0; f < 7; f++) {
        for (unsigned k = 0; k < 8; k++) {
            snprintf(buf, sizeof(buf), "%s%u/%u%s", kMtFam[f].prefix, kMtH[k], kMtD[k], kMtFam[f].suffix);
            if (!strcmp(s, buf)) {
                *oid = 8 * f + k + 1;
                return 0;
            }
        }
    }
    return -1;
}

extern "C" int xmss_parse_oid(xmss_params* p, const uint32_t oid)
{
    if (oid < 1 || oid > 21) return -1;
    const XmssSet& s = kXmss[oid - 1];
    return finish(p, s.func, s.n, s.h, 1);
}

extern "C" int xmssmt_parse_oid(xmss_params* p, const uint32_t oid)
{
    if (oid < 1 || oid > 56) return -1;
    const unsigned f = (oid - 1) / 8, k = (oid - 1) % 8;
    return finish(p, kMtFam[f].func, kMtFam[f].n, kMtH[k], kMtD[k]);
}

extern "C" int xmss_xmssmt_initialize_params(xmss_params* p)
{
    // params.c:710-753
    p->tree_height = p->full_height / p->d;
    switch (p->wots_w) {
        case 4: p->wots_log_w = 2; p->wots_len2 = 5; break;
        case 16: p->wots_log_w = 4; p->wots_len2 = 3; break;
        case 256: p->wots_log_w = 8; p->wots_len2 = 2; break;
        default: return -1;
    }
    p->wots_len1 = 8 * p->n / p->wots_log_w;
    p->wots_len = p->wots_len1 + p->wots_len2;
    p->wots_sig_bytes = p->wots_len * p->n;
    p->index_bytes = (p->d == 1) ? 4 : (p->full_height + 7) / 8;
    p->sig_bytes = p->index_bytes + p->n + p->d * p->wots_sig_bytes + p->full_height * p->n;
    p->pk_bytes = 2 * p->n;
    p->sk_bytes = p->index_bytes + 4ull * p->n;  // xmss_core.c:93-96
    return 0;
}
