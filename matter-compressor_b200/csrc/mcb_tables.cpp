// mcb_tables.cpp -- host-side tables (see mcb_tables.h). Compiled without
// floating-point contraction so every f32 expression rounds like the
// reference's strict build.
#include "mcb_tables.h"

#include <math.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>

namespace mcb {

namespace {

// Trained p0 endpoint tables at q=1 (lo) and q=12 (hi), class order SIG, MAG,
// EOB, MASK, MASKU, MASKA, FLAG, DC (src/mc_codec.c:108,121-140). Slots not
// listed are the untrained 2048.
struct ClassRow { const uint16_t *v; int n; };
const uint16_t kLoSig[] = {115, 110, 112, 144, 3866, 3522, 3330, 948, 3939, 3723, 3483, 2383,
                           4007, 3795, 3575, 3130, 4042, 3912, 3805, 3686, 4064, 4064, 4028, 4064};
const uint16_t kHiSig[] = {456, 335, 535, 1133, 3950, 3755, 3590, 2892, 4064, 4051, 3990, 3686};
const uint16_t kLoMag[] = {1996, 1234, 948, 743, 595, 539, 441, 421, 333, 358, 297, 305};
const uint16_t kHiMag[] = {2121, 1410, 1081, 863, 746, 631, 569, 508, 465, 431, 399, 370};
const uint16_t kLoEob[] = {32, 32, 32, 32, 32, 32, 32, 32, 32, 92, 285, 2295, 4064};
const uint16_t kHiEob[] = {59, 32, 32, 32, 32, 63, 92, 315, 2273, 4064, 4064};
const uint16_t kMask[] = {4025, 3064, 2995, 827, 2107, 473, 576, 50};
const uint16_t kMaskU[] = {250, 1713, 2961, 2991};
const uint16_t kMaskA[] = {3936, 32};
const uint16_t kFlag[] = {1023, 4064, 4064, 4064};
const uint16_t kDc[] = {3873, 366, 1820, 2056, 2040, 2055, 2041, 2045};

template <int N>
ClassRow row(const uint16_t (&a)[N]) { return {a, N}; }

void baked(uint16_t lo[8][32], uint16_t hi[8][32]) {
    const ClassRow los[8] = {row(kLoSig), row(kLoMag), row(kLoEob), row(kMask),
                             row(kMaskU), row(kMaskA), row(kFlag), row(kDc)};
    const ClassRow his[8] = {row(kHiSig), row(kHiMag), row(kHiEob), row(kMask),
                             row(kMaskU), row(kMaskA), row(kFlag), row(kDc)};
    for (int c = 0; c < 8; ++c) {
        for (int s = 0; s < 32; ++s) {
            lo[c][s] = s < los[c].n ? los[c].v[s] : 2048;
            hi[c][s] = s < his[c].n ? his[c].v[s] : 2048;
        }
    }
}

std::mutex g_pri_mu;
bool g_pri_override = false;
uint16_t g_pri_lo[8][32], g_pri_hi[8][32];
std::atomic<uint32_t> g_pri_gen{1};

int l1(int idx) { return (idx >> 8) + ((idx >> 4) & 15) + (idx & 15); }

}  // namespace

void table_cos(float cmf[16][16]) {
    for (int k = 0; k < 16; ++k) {
        double ck = (k == 0) ? sqrt(1.0 / 16) : sqrt(2.0 / 16);
        for (int n = 0; n < 16; ++n) {
            double arg = 3.14159265358979323846 * (2.0 * n + 1.0) * k / (2.0 * 16);
            cmf[k][n] = (float)(ck * cos(arg));
        }
    }
}

void table_scan(uint16_t scan[kN3]) {
    int order[kN3];
    for (int i = 0; i < kN3; ++i) order[i] = i;
    std::sort(order, order + kN3, [](int a, int b) {
        int fa = l1(a), fb = l1(b);
        return fa != fb ? fa < fb : a < b;
    });
    for (int p = 0; p < kN3; ++p) {
        int band = std::min(l1(order[p]) * 8 / 48, 7);
        scan[p] = (uint16_t)(order[p] | (band << 12));
    }
}

uint32_t priors_set(const uint16_t *plo, const uint16_t *phi) {
    std::lock_guard<std::mutex> g(g_pri_mu);
    if (plo && phi) {
        memcpy(g_pri_lo, plo, sizeof g_pri_lo);
        memcpy(g_pri_hi, phi, sizeof g_pri_hi);
        g_pri_override = true;
    } else {
        g_pri_override = false;
    }
    return ++g_pri_gen;
}

uint32_t priors_generation() { return g_pri_gen.load(); }

void priors_active(uint16_t lo[8][32], uint16_t hi[8][32]) {
    std::lock_guard<std::mutex> g(g_pri_mu);
    if (g_pri_override) {
        memcpy(lo, g_pri_lo, sizeof g_pri_lo);
        memcpy(hi, g_pri_hi, sizeof g_pri_hi);
    } else {
        baked(lo, hi);
    }
}

void table_qtab(float q, QTab *t) {
    memset(t, 0, sizeof *t);
    t->q = q;
    for (int f = 0; f < 48; ++f) {
        float w = powf(1.0f + (float)f, 0.65f);
        float st = q * w;
        t->step[f] = st;
        t->dz8[f] = 0.80f * st;
        t->dz4[f] = 0.40f * st;
        t->rstep[f] = 1.0f / st;
    }
    uint16_t lo[8][32], hi[8][32], pri[8][32];
    priors_active(lo, hi);
    // w = log2(q)/3.585 clamped to [0,1], interpolated in single precision
    float w = 0.0f;
    if (q > 1.0f) w = ((float)(log((double)q) / log(2.0)) - 0.0f) / (3.585f - 0.0f);
    if (w < 0) w = 0;
    if (w > 1) w = 1;
    for (int c = 0; c < 8; ++c)
        for (int s = 0; s < 32; ++s) {
            float v = (float)lo[c][s] + (float)((int)hi[c][s] - (int)lo[c][s]) * w;
            v = v + 0.5f;
            pri[c][s] = (uint16_t)v;
        }
    enum { SIG = 0, MAG = 1, EOB = 2, FLAG = 6, DC = 7 };
    for (int i = 0; i < 2; ++i) t->ctx[kCtxFlag + i] = pri[FLAG][i];
    for (int i = 0; i < 8; ++i) t->ctx[kCtxDc + i] = pri[DC][i];
    for (int i = 0; i < 14; ++i) t->ctx[kCtxEob + i] = pri[EOB][i];
    for (int i = 0; i < 32; ++i) t->ctx[kCtxSig + i] = pri[SIG][i];
    for (int i = 0; i < 12; ++i) t->ctx[kCtxMag + i] = pri[MAG][i];
}

}  // namespace mcb
