/*
 * mc_oracle.c -- CPU restatement of matter-compressor's 16^3 block codec.
 *
 * TEST INFRASTRUCTURE ONLY (see mc_oracle.h). Written as a plain, readable
 * restatement of the reference's algorithm: one function per reference
 * routine, each citing the file:line it follows. Build with strict IEEE
 * single precision (no FMA contraction, no fast-math): oracle/Makefile.
 *
 * Corrupt-stream policy (shared with the CUDA decoder): the reference's
 * unbounded Exp-Golomb prefix loop (src/mc_codec.c:235,272) is capped at
 * OR_EG_CAP one-bits; hitting the cap ends the block's entropy decode (the
 * coefficients and corrections decoded so far stand). Shifts by >= 32 follow
 * x86 semantics (count taken mod 32), and integer wrap-around follows the
 * two's-complement behaviour the reference's gcc build exhibits.
 */
#include "mc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define OR_N3      4096
#define OR_EG_CAP  64

/* ------------------------------------------------------------------ priors */
/* Trained p0 tables (P(bit==0) in 1/4096), src/mc_codec.c:121-140. Each class
 * lists its trained slots; every slot not listed is the untrained 2048. The
 * class order is SIG, MAG, EOB, MASK, MASKU, MASKA, FLAG, DC
 * (src/mc_codec.c:108). */
static const uint16_t PLO_SIG[] = {115,110,112,144,3866,3522,3330,948,3939,3723,3483,2383,
                                   4007,3795,3575,3130,4042,3912,3805,3686,4064,4064,4028,4064};
static const uint16_t PHI_SIG[] = {456,335,535,1133,3950,3755,3590,2892,4064,4051,3990,3686};
static const uint16_t PLO_MAG[] = {1996,1234,948,743,595,539,441,421,333,358,297,305};
static const uint16_t PHI_MAG[] = {2121,1410,1081,863,746,631,569,508,465,431,399,370};
static const uint16_t PLO_EOB[] = {32,32,32,32,32,32,32,32,32,92,285,2295,4064};
static const uint16_t PHI_EOB[] = {59,32,32,32,32,63,92,315,2273,4064,4064};
static const uint16_t P_MASK[]  = {4025,3064,2995,827,2107,473,576,50};
static const uint16_t P_MASKU[] = {250,1713,2961,2991};
static const uint16_t P_MASKA[] = {3936,32};
static const uint16_t P_FLAG[]  = {1023,4064,4064,4064};
static const uint16_t P_DC[]    = {3873,366,1820,2056,2040,2055,2041,2045};

#define NSLOT 32
enum { C_SIG = 0, C_MAG, C_EOB, C_MASK, C_MASKU, C_MASKA, C_FLAG, C_DC };

static void fill_class(uint16_t row[NSLOT], const uint16_t *v, size_t n) {
    for (int s = 0; s < NSLOT; ++s) row[s] = 2048;
    for (size_t s = 0; s < n; ++s) row[s] = v[s];
}
#define FILL(row, arr) fill_class(row, arr, sizeof(arr) / sizeof(arr[0]))

static void baked_tables(uint16_t lo[8][NSLOT], uint16_t hi[8][NSLOT]) {
    FILL(lo[C_SIG], PLO_SIG);   FILL(hi[C_SIG], PHI_SIG);
    FILL(lo[C_MAG], PLO_MAG);   FILL(hi[C_MAG], PHI_MAG);
    FILL(lo[C_EOB], PLO_EOB);   FILL(hi[C_EOB], PHI_EOB);
    FILL(lo[C_MASK], P_MASK);   FILL(hi[C_MASK], P_MASK);
    FILL(lo[C_MASKU], P_MASKU); FILL(hi[C_MASKU], P_MASKU);
    FILL(lo[C_MASKA], P_MASKA); FILL(hi[C_MASKA], P_MASKA);
    FILL(lo[C_FLAG], P_FLAG);   FILL(hi[C_FLAG], P_FLAG);
    FILL(lo[C_DC], P_DC);       FILL(hi[C_DC], P_DC);
}

static int      g_override = 0;
static uint16_t g_ovr_lo[8][NSLOT], g_ovr_hi[8][NSLOT];

void or_set_priors(const uint16_t *plo, const uint16_t *phi) {
    if (plo && phi) {
        memcpy(g_ovr_lo, plo, sizeof g_ovr_lo);
        memcpy(g_ovr_hi, phi, sizeof g_ovr_hi);
        g_override = 1;
    } else {
        g_override = 0;
    }
}

/* src/mc_codec.c:156-167: weight w = log2(q)/3.585 clamped to [0,1] (q<=1 -> 0),
 * p = (u16)(lo + (hi-lo)*w + 0.5f) evaluated in single precision. */
void or_priors_for_q(float q, uint16_t out[256]) {
    uint16_t lo[8][NSLOT], hi[8][NSLOT];
    if (g_override) {
        memcpy(lo, g_ovr_lo, sizeof lo);
        memcpy(hi, g_ovr_hi, sizeof hi);
    } else {
        baked_tables(lo, hi);
    }
    const float span = 3.585f - 0.0f;
    float w;
    if (q <= 1.0f) w = 0.0f;
    else w = ((float)(log((double)q) / log(2.0)) - 0.0f) / span;
    if (w < 0) w = 0;
    if (w > 1) w = 1;
    for (int c = 0; c < 8; ++c)
        for (int s = 0; s < NSLOT; ++s) {
            int d = (int)hi[c][s] - (int)lo[c][s];
            float v = (float)lo[c][s] + (float)d * w;
            v = v + 0.5f;
            out[c * NSLOT + s] = (uint16_t)v;
        }
}

float or_sanitize_q(float q) {
    if (!(q > 0.0f) || q > 1024.0f) return 8.0f;   /* src/mc_codec.c:496 */
    return q;
}

/* ------------------------------------------------------------ fixed tables */
static float    g_cos[16][16];     /* cmf[k][n], src/mc_codec_float.h:70-78 */
static uint16_t g_scan[OR_N3];     /* scan position -> raster index        */
static int      g_ready = 0;

static int l1_of(int idx) { return (idx >> 8) + ((idx >> 4) & 15) + (idx & 15); }

static int scan_less(const void *a, const void *b) {
    int ia = *(const uint16_t *)a, ib = *(const uint16_t *)b;
    int fa = l1_of(ia), fb = l1_of(ib);
    if (fa != fb) return fa - fb;
    return ia - ib;
}

static void tables_init(void) {
    if (g_ready) return;
    for (int k = 0; k < 16; ++k) {
        double ck = (k == 0) ? sqrt(1.0 / 16) : sqrt(2.0 / 16);
        for (int n = 0; n < 16; ++n) {
            /* same double expression order as src/mc_codec_float.h:75 */
            double arg = 3.14159265358979323846 * (2.0 * n + 1.0) * k / (2.0 * 16);
            g_cos[k][n] = (float)(ck * cos(arg));
        }
    }
    for (int i = 0; i < OR_N3; ++i) g_scan[i] = (uint16_t)i;
    qsort(g_scan, OR_N3, sizeof g_scan[0], scan_less);   /* total order: unique result */
    g_ready = 1;
}

void or_scan_table(uint16_t scan[4096]) {
    tables_init();
    memcpy(scan, g_scan, sizeof g_scan);
}

/* band of a raster index: floor(L1*8/48) capped at 7 (src/mc_codec.c:305-308). */
static int band_of(int idx) {
    int b = l1_of(idx) * 8 / 48;
    return b > 7 ? 7 : b;
}

/* step = q * (1+L1)^0.65, rstep = 1/step (src/mc_codec.c:542-552). */
void or_step_table(float q, float step[4096], float rstep[4096]) {
    for (int i = 0; i < OR_N3; ++i) {
        float w = powf(1.0f + (float)l1_of(i), 0.65f);
        step[i] = q * w;
        rstep[i] = 1.0f / step[i];
    }
}

/* -------------------------------------------------------- range encoder */
/* LZMA-style carry-propagating encoder, src/mc_codec.c:95,178-195,209-215. */
typedef struct {
    uint8_t *buf; size_t cap, len;
    uint64_t low; uint32_t range;
    uint8_t cache; uint64_t pending;    /* pending = the reference's cache_size */
} renc;

static void re_init(renc *e, uint8_t *buf, size_t cap) {
    e->buf = buf; e->cap = cap; e->len = 0;
    e->low = 0; e->range = 0xFFFFFFFFu; e->cache = 0; e->pending = 1;
}
static void re_emit(renc *e, uint8_t b) {
    if (e->len < e->cap) e->buf[e->len] = b;
    e->len++;
}
static void re_shift(renc *e) {
    uint32_t top = (uint32_t)(e->low >> 32);
    if (top != 0 || e->low < 0xFF000000ull) {
        uint8_t carry = (uint8_t)top;
        uint8_t first = (uint8_t)(e->cache + carry);
        re_emit(e, first);
        for (uint64_t i = 1; i < e->pending; ++i) re_emit(e, (uint8_t)(0xFF + carry));
        e->pending = 0;
        e->cache = (uint8_t)(e->low >> 24);
    }
    e->pending++;
    e->low = (e->low << 8) & 0xFFFFFFFFull;
}
static void re_norm(renc *e) {
    while (e->range < (1u << 24)) { re_shift(e); e->range <<= 8; }
}
static void re_bit(renc *e, uint16_t *p0, int bit) {
    uint32_t r0 = (e->range >> 12) * (uint32_t)*p0;
    if (!bit) { e->range = r0; *p0 = (uint16_t)(*p0 + ((4096 - *p0) >> 4)); }
    else { e->low += r0; e->range -= r0; *p0 = (uint16_t)(*p0 - (*p0 >> 4)); }
    re_norm(e);
}
static void re_bypass(renc *e, int bit) {
    e->range >>= 1;
    if (bit) e->low += e->range;
    re_norm(e);
}
static void re_bypass_bits(renc *e, uint32_t v, int k) {
    /* more than 16 bits go out as 16-bit pieces, most significant first */
    while (k > 16) { re_bypass_bits(e, (v >> (k - 16)) & 0xFFFFu, 16); k -= 16; }
    if (k == 0) return;
    e->range >>= k;
    e->low += (uint64_t)(v & ((1u << k) - 1)) * e->range;
    re_norm(e);
}
static void re_finish(renc *e) { for (int i = 0; i < 5; ++i) re_shift(e); }

static int bitlen(uint32_t v) { int n = 0; while (v) { v >>= 1; ++n; } return n; }

/* order-0 Exp-Golomb in bypass bits (src/mc_codec.c:229-233). */
static void re_expgolomb(renc *e, uint32_t v) {
    uint32_t t = v + 1;
    int nb = t ? bitlen(t) - 1 : 0;
    for (int i = 0; i < nb; ++i) re_bypass(e, 1);
    re_bypass(e, 0);
    if (nb) re_bypass_bits(e, (v + 1) & ((1u << nb) - 1), nb);
}

/* -------------------------------------------------------- range decoder */
/* src/mc_codec.c:96,197-226: bytes past the payload read as zero. */
typedef struct {
    const uint8_t *buf; size_t len, pos;
    uint32_t code, range;
    int bad;          /* set once an Exp-Golomb prefix reaches OR_EG_CAP */
} rdec;

static uint8_t rd_byte(rdec *d) { return d->pos < d->len ? d->buf[d->pos++] : 0; }
static void rd_init(rdec *d, const uint8_t *buf, size_t len) {
    d->buf = buf; d->len = len; d->pos = 0; d->code = 0; d->range = 0xFFFFFFFFu; d->bad = 0;
    for (int i = 0; i < 5; ++i) d->code = (d->code << 8) | rd_byte(d);
}
static void rd_norm(rdec *d) {
    while (d->range < (1u << 24)) { d->code = (d->code << 8) | rd_byte(d); d->range <<= 8; }
}
static int rd_bit(rdec *d, uint16_t *p0) {
    uint32_t r0 = (d->range >> 12) * (uint32_t)*p0;
    int bit;
    if (d->code < r0) { d->range = r0; bit = 0; *p0 = (uint16_t)(*p0 + ((4096 - *p0) >> 4)); }
    else { d->code -= r0; d->range -= r0; bit = 1; *p0 = (uint16_t)(*p0 - (*p0 >> 4)); }
    rd_norm(d);
    return bit;
}
static int rd_bypass(rdec *d) {
    d->range >>= 1;
    int bit = d->code >= d->range;
    if (bit) d->code -= d->range;
    rd_norm(d);
    return bit;
}
static uint32_t rd_bypass_bits(rdec *d, int k) {
    uint32_t v = 0;
    while (k > 16) { v = (v << 16) | rd_bypass_bits(d, 16); k -= 16; }
    if (k == 0) return v;
    d->range >>= k;
    uint32_t q = d->code / d->range;
    uint32_t m = (1u << k) - 1;
    if (q > m) q = m;
    d->code -= q * d->range;
    rd_norm(d);
    return (v << k) | q;
}
/* src/mc_codec.c:234-238, with the prefix capped (see file header). */
static uint32_t rd_expgolomb(rdec *d) {
    int nb = 0;
    while (rd_bypass(d)) {
        if (++nb >= OR_EG_CAP) { d->bad = 1; return 0; }
    }
    if (!nb) return 0;
    return ((1u << (nb & 31)) | rd_bypass_bits(d, nb)) - 1;
}

/* ------------------------------------------------------ context sets */
typedef struct {
    uint16_t sig[32];   /* band*4 + density  (src/mc_codec.c:249-259) */
    uint16_t mag[12];   /* unary magnitude ladder                      */
    uint16_t eob[14];   /* EOB bit-length prefix (src/mc_codec.c:311-313) */
    uint16_t flag[2];   /* header bins (src/mc_codec.c:714,747)          */
    uint16_t dc[8];
} ctxset;

static void ctx_load(ctxset *c, const uint16_t pri[256]) {
    for (int i = 0; i < 32; ++i) c->sig[i] = pri[C_SIG * NSLOT + i];
    for (int i = 0; i < 12; ++i) c->mag[i] = pri[C_MAG * NSLOT + i];
    for (int i = 0; i < 14; ++i) c->eob[i] = pri[C_EOB * NSLOT + i];
    for (int i = 0; i < 2; ++i)  c->flag[i] = pri[C_FLAG * NSLOT + i];
    for (int i = 0; i < 8; ++i)  c->dc[i] = pri[C_DC * NSLOT + i];
}

static int density(uint32_t hist) {
    int n = __builtin_popcount(hist & 0xFFFFu);
    return n < 3 ? n : 3;
}

/* ------------------------------------------------------------ transform */
/* DCT-III of one line, even/odd halves with sequential single-precision
 * accumulation in ascending k, zero coefficients skipped
 * (src/mc_codec_float.h:98-105). */
static void idct_line(const float *in, int si, float *out, int so) {
    int any = 0;
    for (int i = 0; i < 16; ++i) if (in[i * si] != 0.0f) { any = 1; break; }
    if (!any) { for (int i = 0; i < 16; ++i) out[i * so] = 0.0f; return; }
    float ev[8], od[8];
    for (int n = 0; n < 8; ++n) { ev[n] = 0.0f; od[n] = 0.0f; }
    for (int k = 0; k < 16; k += 2) {
        float v = in[k * si];
        if (v != 0.0f) for (int n = 0; n < 8; ++n) ev[n] += g_cos[k][n] * v;
    }
    for (int k = 1; k < 16; k += 2) {
        float v = in[k * si];
        if (v != 0.0f) for (int n = 0; n < 8; ++n) od[n] += g_cos[k][n] * v;
    }
    for (int n = 0; n < 8; ++n) {
        out[n * so] = ev[n] + od[n];
        out[(15 - n) * so] = ev[n] - od[n];
    }
}
/* DCT-II of one line (src/mc_codec_float.h:83-95). */
static void fdct_line(const float *in, int si, float *out, int so) {
    int any = 0;
    for (int i = 0; i < 16; ++i) if (in[i * si] != 0.0f) { any = 1; break; }
    if (!any) { for (int i = 0; i < 16; ++i) out[i * so] = 0.0f; return; }
    float s[8], d[8];
    for (int n = 0; n < 8; ++n) {
        s[n] = in[n * si] + in[(15 - n) * si];
        d[n] = in[n * si] - in[(15 - n) * si];
    }
    for (int k = 0; k < 16; k += 2) {
        float a = 0.0f;
        for (int n = 0; n < 8; ++n) a += g_cos[k][n] * s[n];
        out[k * so] = a;
    }
    for (int k = 1; k < 16; k += 2) {
        float a = 0.0f;
        for (int n = 0; n < 8; ++n) a += g_cos[k][n] * d[n];
        out[k * so] = a;
    }
}
/* Separable 3D transform, passes along x, then y, then z. The reference
 * transforms contiguous lines and rotates the cube between passes
 * (src/mc_codec_float.h:128-158); indexing the axes directly is the same
 * arithmetic on the same values. Layout is [z][y][x]. */
typedef void (*line_fn)(const float *, int, float *, int);
static void transform3(line_fn f, const float *src, float *dst) {
    float a[OR_N3], b[OR_N3];
    for (int z = 0; z < 16; ++z) for (int y = 0; y < 16; ++y)
        f(src + z * 256 + y * 16, 1, a + z * 256 + y * 16, 1);
    for (int z = 0; z < 16; ++z) for (int x = 0; x < 16; ++x)
        f(a + z * 256 + x, 16, b + z * 256 + x, 16);
    for (int y = 0; y < 16; ++y) for (int x = 0; x < 16; ++x)
        f(b + y * 16 + x, 256, dst + y * 16 + x, 256);
}

/* dead-zone reconstruction (src/mc_codec_float.h:185-190). */
static float dequant(int32_t lv, float step) {
    if (!lv) return 0.0f;
    float a = (float)(lv < 0 ? -lv : lv);
    float r = (a - 1.0f) * step;
    r = r + 0.80f * step;
    r = r + 0.40f * step;
    return lv < 0 ? -r : r;
}

static uint8_t clamp_u8(int v) { return (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v); }

/* ---------------------------------------------------------- block encode */
/* src/mc_codec.c:629-736. */
uint32_t or_enc_block(const uint8_t vox[4096], float q_in, int tau, uint8_t *out, uint32_t cap) {
    tables_init();
    float q = or_sanitize_q(q_in);
    if (tau < 0) tau = 0;
    long sum = 0, cnt = 0;
    for (int i = 0; i < OR_N3; ++i) { sum += vox[i]; cnt += vox[i] != 0; }
    if (!cnt) return 0;
    int dc = (int)((sum + OR_N3 / 2) / OR_N3);

    float blk[OR_N3], coef[OR_N3], step[OR_N3], rstep[OR_N3];
    or_step_table(q, step, rstep);
    for (int i = 0; i < OR_N3; ++i) blk[i] = (float)((int)vox[i] - dc);
    transform3(fdct_line, blk, coef);

    /* fused quantiser: t = |c|*rstep + (1-0.8), clamp [0,32767], truncate
     * (src/mc_codec.c:686-692) */
    static const float bias = 1.0f - 0.80f;
    int16_t lv[OR_N3];
    for (int i = 0; i < OR_N3; ++i) {
        float c = coef[i];
        float t = fabsf(c) * rstep[i];
        t = t + bias;
        if (!(t > 0.0f)) t = 0.0f;
        if (!(t < 32767.0f)) t = 32767.0f;
        int v = (int)t;
        lv[i] = (int16_t)(c < 0.0f ? -v : v);
    }

    /* max-error corrections against the local reconstruction (:697-708) */
    uint16_t cpos[OR_N3];
    int32_t  cdel[OR_N3];
    int ncorr = 0;
    if (tau > 0) {
        float rc[OR_N3], rb[OR_N3];
        for (int i = 0; i < OR_N3; ++i) rc[i] = dequant(lv[i], step[i]);
        transform3(idct_line, rc, rb);
        for (int i = 0; i < OR_N3; ++i) {
            int v = clamp_u8((int)lrintf(rb[i]) + dc);
            int err = (int)vox[i] - v;
            int ae = err < 0 ? -err : err;
            if (ae > tau) { cpos[ncorr] = (uint16_t)i; cdel[ncorr] = err < 0 ? -(ae - tau) : (ae - tau); ncorr++; }
        }
    }

    uint16_t pri[256];
    or_priors_for_q(q, pri);
    ctxset cx;
    ctx_load(&cx, pri);
    renc e;
    re_init(&e, out, cap);
    re_bit(&e, &cx.flag[0], 0);              /* reserved bit (was "mixed") */
    re_bit(&e, &cx.flag[1], ncorr > 0);
    for (int b = 0; b < 8; ++b) re_bit(&e, &cx.dc[b], (dc >> (7 - b)) & 1);

    /* coefficients: EOB, then significance/magnitude/sign (src/mc_codec.c:330-350) */
    int eob = 0;
    for (int p = OR_N3 - 1; p >= 0; --p) if (lv[g_scan[p]]) { eob = p + 1; break; }
    {   /* EOB prefix + suffix (src/mc_codec.c:314-320); 13 prefix bins for n=4096 */
        int k = bitlen((uint32_t)eob);
        for (int i = 0; i < k; ++i) re_bit(&e, &cx.eob[i], 1);
        if (k < 13) re_bit(&e, &cx.eob[k], 0);
        if (k > 1) re_bypass_bits(&e, (uint32_t)eob & ((1u << (k - 1)) - 1), k - 1);
    }
    uint32_t hist = 0;
    for (int p = 0; p < eob; ++p) {
        int idx = g_scan[p];
        int v = lv[idx];
        if (p != eob - 1) re_bit(&e, &cx.sig[band_of(idx) * 4 + density(hist)], v != 0);
        hist = (hist << 1) | (v != 0);
        if (!v) continue;
        /* magnitude: unary over 12 adaptive rungs, then Exp-Golomb (:260-267) */
        uint32_t m = (uint32_t)(v < 0 ? -v : v), rest = m - 1;
        int k = 0;
        while (rest > 0 && k < 11) { re_bit(&e, &cx.mag[k], 1); rest--; k++; }
        if (rest == 0) re_bit(&e, &cx.mag[k], 0);
        else { re_bit(&e, &cx.mag[11], 1); re_expgolomb(&e, rest); }
        re_bypass(&e, v < 0);
    }
    if (ncorr > 0) {   /* [eg count-1][eg gap, sign, eg |d|-1]* (:721-729) */
        re_expgolomb(&e, (uint32_t)(ncorr - 1));
        uint32_t prev = 0;
        for (int c = 0; c < ncorr; ++c) {
            re_expgolomb(&e, (uint32_t)cpos[c] - prev);
            prev = cpos[c];
            int32_t D = cdel[c];
            re_bypass(&e, D < 0);
            re_expgolomb(&e, (uint32_t)(D < 0 ? -D : D) - 1);
        }
    }
    re_finish(&e);
    return (uint32_t)e.len;
}

/* ---------------------------------------------------------- block decode */
/* Entropy stage of src/mc_codec.c:739-757 and :353-375. info[]: 0 dc, 1 flags,
 * 2..4 extents z,y,x (-1 none), 5 eob, 6 nonzeros, 7 bad-stream flag. The
 * decoder state is returned for the correction stage. */
static void entropy_decode(rdec *d, ctxset *cx, int16_t lv[4096], int info[8]) {
    int flags = 0, dc = 0;
    flags |= rd_bit(d, &cx->flag[0]) ? 1 : 0;
    flags |= rd_bit(d, &cx->flag[1]) ? 2 : 0;
    for (int b = 0; b < 8; ++b) dc = (dc << 1) | rd_bit(d, &cx->dc[b]);
    memset(lv, 0, OR_N3 * sizeof lv[0]);

    uint32_t eob;
    {   /* src/mc_codec.c:321-327 */
        int k = 0;
        while (k < 13 && rd_bit(d, &cx->eob[k])) k++;
        if (k == 0) eob = 0;
        else if (k == 1) eob = 1;
        else eob = (1u << (k - 1)) | rd_bypass_bits(d, k - 1);
        if (eob > OR_N3) eob = OR_N3;
    }
    int ez = -1, ey = -1, ex = -1, nnz = 0;
    uint32_t hist = 0;
    for (uint32_t p = 0; p < eob && !d->bad; ++p) {
        int idx = g_scan[p];
        int sig = (p == eob - 1) ? 1 : rd_bit(d, &cx->sig[band_of(idx) * 4 + density(hist)]);
        hist = (hist << 1) | (uint32_t)sig;
        if (!sig) continue;
        /* src/mc_codec.c:268-275 */
        uint32_t v = 0, m;
        int k = 0;
        while (k < 11 && rd_bit(d, &cx->mag[k])) { v++; k++; }
        if (k < 11) m = v + 1;
        else if (!rd_bit(d, &cx->mag[11])) m = v + 1;
        else m = v + rd_expgolomb(d) + 1;
        if (d->bad) break;
        int neg = rd_bypass(d);
        lv[idx] = (int16_t)(neg ? -(int32_t)m : (int32_t)m);
        nnz++;
        int cz = idx >> 8, cy = (idx >> 4) & 15, cxx = idx & 15;
        if (cz > ez) ez = cz;
        if (cy > ey) ey = cy;
        if (cxx > ex) ex = cxx;
    }
    info[0] = dc; info[1] = flags; info[2] = ez; info[3] = ey; info[4] = ex;
    info[5] = (int)eob; info[6] = nnz; info[7] = d->bad;
}

static void block_ctx(float q, ctxset *cx) {
    uint16_t pri[256];
    or_priors_for_q(q, pri);
    ctx_load(cx, pri);
}

void or_dec_block_levels(const uint8_t *p, uint32_t plen, float q_in, int16_t levels[4096], int info[8]) {
    tables_init();
    float q = or_sanitize_q(q_in);
    ctxset cx;
    block_ctx(q, &cx);
    rdec d;
    rd_init(&d, p, plen);
    entropy_decode(&d, &cx, levels, info);
}

void or_dec_block(const uint8_t *p, uint32_t plen, float q_in, uint8_t dst[4096]) {
    tables_init();
    float q = or_sanitize_q(q_in);
    ctxset cx;
    block_ctx(q, &cx);
    rdec d;
    rd_init(&d, p, plen);
    int16_t lv[OR_N3];
    int info[8];
    entropy_decode(&d, &cx, lv, info);
    int dc = info[0], flags = info[1];
    if (info[2] < 0) {
        memset(dst, dc, OR_N3);   /* constant block (src/mc_codec.c:757-759) */
        if (!(flags & 2)) return;
    } else {
        float step[OR_N3], rstep[OR_N3], coef[OR_N3], blk[OR_N3];
        or_step_table(q, step, rstep);
        for (int i = 0; i < OR_N3; ++i) coef[i] = dequant(lv[i], step[i]);
        transform3(idct_line, coef, blk);
        for (int i = 0; i < OR_N3; ++i) dst[i] = clamp_u8((int)lrintf(blk[i]) + dc);
    }
    if ((flags & 2) && !d.bad) {   /* sparse corrections (src/mc_codec.c:770-782) */
        uint32_t ncorr = rd_expgolomb(&d) + 1, pos = 0;
        if (ncorr > OR_N3) ncorr = OR_N3;
        for (uint32_t c = 0; c < ncorr && !d.bad; ++c) {
            pos += rd_expgolomb(&d);
            if (d.bad) break;
            int neg = rd_bypass(&d);
            uint32_t m = rd_expgolomb(&d) + 1;
            if (d.bad) break;
            if (pos >= OR_N3) break;
            uint32_t delta = neg ? 0u - m : m;            /* wrapping int add */
            dst[pos] = clamp_u8((int)((uint32_t)dst[pos] + delta));
        }
    }
}

/* ------------------------------------------------------------ fraction map */
/* 4096 nibbles, 4 adaptive bins each, context = bucket of the previous nibble
 * (0 / 1..14 / 15), MSB first (src/mc_codec.c:600-621). Contexts start at 2048. */
static int nib_bucket(int prev) { return prev == 0 ? 0 : prev == 15 ? 2 : 1; }

uint32_t or_enc_fracmap(const uint8_t frac[4096], uint8_t *out, uint32_t cap) {
    uint16_t c[3][4];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 4; ++j) c[i][j] = 2048;
    renc e;
    re_init(&e, out, cap);
    int prev = 0;
    for (int i = 0; i < OR_N3; ++i) {
        int v = frac[i] & 15, b = nib_bucket(prev);
        for (int bit = 3; bit >= 0; --bit) re_bit(&e, &c[b][bit], (v >> bit) & 1);
        prev = v;
    }
    re_finish(&e);
    return (uint32_t)e.len;
}

void or_dec_fracmap(const uint8_t *in, uint32_t len, uint8_t frac[4096]) {
    uint16_t c[3][4];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 4; ++j) c[i][j] = 2048;
    rdec d;
    rd_init(&d, in, len);
    int prev = 0;
    for (int i = 0; i < OR_N3; ++i) {
        int v = 0, b = nib_bucket(prev);
        for (int bit = 3; bit >= 0; --bit) v |= rd_bit(&d, &c[b][bit]) << bit;
        frac[i] = (uint8_t)v;
        prev = v;
    }
}

/* round(15 * count/4096), at least 1 when any voxel is set (src/mc_codec.c:820-822) */
uint8_t or_frac_nibble(const uint8_t vox[4096]) {
    int cnt = 0;
    for (int i = 0; i < OR_N3; ++i) cnt += vox[i] != 0;
    int f = (cnt * 15 + 2048) / 4096;
    if (cnt && !f) f = 1;
    return (uint8_t)f;
}

/* ------------------------------------------------------------------ XXH64 */
/* The published XXH64 algorithm (as used at src/mc_codec.c:393-414). */
static const uint64_t XP1 = 0x9E3779B185EBCA87ull, XP2 = 0xC2B2AE3D27D4EB4Full,
                      XP3 = 0x165667B19E3779F9ull, XP4 = 0x85EBCA77C2B2AE63ull,
                      XP5 = 0x27D4EB2F165667C5ull;
static uint64_t rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
static uint64_t xround(uint64_t acc, uint64_t in) { return rotl64(acc + in * XP2, 31) * XP1; }
static uint64_t ld64(const uint8_t *p) { uint64_t v; memcpy(&v, p, 8); return v; }
static uint32_t ld32(const uint8_t *p) { uint32_t v; memcpy(&v, p, 4); return v; }

uint64_t or_xxh64(const void *data, size_t len, uint64_t seed) {
    const uint8_t *p = (const uint8_t *)data, *end = p + len;
    uint64_t h;
    if (len >= 32) {
        uint64_t acc[4] = {seed + XP1 + XP2, seed + XP2, seed, seed - XP1};
        while (end - p >= 32) {
            for (int i = 0; i < 4; ++i) acc[i] = xround(acc[i], ld64(p + 8 * i));
            p += 32;
        }
        h = rotl64(acc[0], 1) + rotl64(acc[1], 7) + rotl64(acc[2], 12) + rotl64(acc[3], 18);
        for (int i = 0; i < 4; ++i) h = (h ^ xround(0, acc[i])) * XP1 + XP4;
    } else {
        h = seed + XP5;
    }
    h += (uint64_t)len;
    for (; end - p >= 8; p += 8) h = rotl64(h ^ xround(0, ld64(p)), 27) * XP1 + XP4;
    if (end - p >= 4) { h = rotl64(h ^ ((uint64_t)ld32(p) * XP1), 23) * XP2 + XP3; p += 4; }
    for (; p < end; ++p) h = rotl64(h ^ ((uint64_t)*p * XP5), 11) * XP1;
    h ^= h >> 33; h *= XP2; h ^= h >> 29; h *= XP3; h ^= h >> 32;
    return h;
}

/* --------------------------------------------------------------- chunk blob */
/* blob = [f32 q][u64 hash][u16 fmaplen][fmap][512 B bitmap][u16 len per present
 * block][payloads in block order] (src/mc_archive.h:147-151). */
#define BLOB_HDR 14
#define SEED_CHAIN 0x6D636368756E6Bull

static unsigned popcount_bytes(const uint8_t *p, size_t n) {
    unsigned c = 0;
    for (size_t i = 0; i < n; ++i) c += (unsigned)__builtin_popcount(p[i]);
    return c;
}

/* src/mc_archive.c:76-88: the chain seeds each segment's hash with the
 * running value and XORs the result in. */
uint64_t or_blob_hash(const uint8_t *blob, uint64_t blob_len) {
    uint16_t fml;
    memcpy(&fml, blob + 12, 2);
    const uint8_t *fmap = blob + BLOB_HDR, *bm = fmap + fml, *lens = bm + 512;
    unsigned np = popcount_bytes(bm, 512);
    uint64_t pay = (uint64_t)BLOB_HDR + fml + 512 + 2ull * np;
    uint64_t h = or_xxh64(fmap, fml, SEED_CHAIN);
    h ^= or_xxh64(bm, 512, h);
    h ^= or_xxh64(lens, 2ull * np, h);
    h ^= or_xxh64(blob + pay, blob_len - pay, h);
    return h;
}

static void gather_block(const uint8_t *vox256, int bi, uint8_t blk[4096]) {
    int bz = bi >> 8, by = (bi >> 4) & 15, bx = bi & 15;
    for (int z = 0; z < 16; ++z) for (int y = 0; y < 16; ++y)
        memcpy(blk + z * 256 + y * 16,
               vox256 + ((size_t)(bz * 16 + z) * 256 + (by * 16 + y)) * 256 + bx * 16, 16);
}

size_t or_encode_chunk(const uint8_t *vox256, float header_q, float q_in, int tau, uint8_t *out, size_t cap) {
    float q = or_sanitize_q(q_in);
    uint8_t *frac = calloc(OR_N3, 1);
    uint16_t *len = calloc(OR_N3, 2);
    uint8_t bm[512] = {0};
    size_t pay_cap = (size_t)OR_N3 * 17408;
    uint8_t *pay = malloc(pay_cap);
    size_t pay_len = 0;
    unsigned np = 0;
    uint8_t blk[OR_N3];
    for (int bi = 0; bi < OR_N3; ++bi) {
        gather_block(vox256, bi, blk);
        frac[bi] = or_frac_nibble(blk);
        uint32_t l = or_enc_block(blk, q, tau, pay + pay_len, 17408);
        if (l) { bm[bi >> 3] |= (uint8_t)(1u << (bi & 7)); len[np++] = (uint16_t)l; pay_len += l; }
    }
    size_t total = 0;
    if (np) {
        uint8_t fmap[2112];
        uint32_t fml = or_enc_fracmap(frac, fmap, sizeof fmap);
        if (fml > sizeof fmap) fml = sizeof fmap;
        total = BLOB_HDR + fml + 512 + 2ull * np + pay_len;
        if (total <= cap) {
            uint8_t *w = out;
            uint16_t f16 = (uint16_t)fml;
            uint64_t h = 0;
            memcpy(w, &header_q, 4); memcpy(w + 12, &f16, 2);
            memcpy(w + BLOB_HDR, fmap, fml);
            memcpy(w + BLOB_HDR + fml, bm, 512);
            memcpy(w + BLOB_HDR + fml + 512, len, 2ull * np);
            memcpy(w + BLOB_HDR + fml + 512 + 2ull * np, pay, pay_len);
            h = or_blob_hash(w, total);
            memcpy(w + 4, &h, 8);
        }
    }
    free(frac); free(len); free(pay);
    return total;
}

/* locate block bi's payload in a blob: offsets are the running sum of the
 * present blocks' lengths in block order (src/mc_archive.h:175-206). */
static int blob_block(const uint8_t *blob, uint64_t blob_len, int bi, uint64_t *off, uint32_t *plen) {
    uint16_t fml;
    memcpy(&fml, blob + 12, 2);
    const uint8_t *bm = blob + BLOB_HDR + fml;
    if (!((bm[bi >> 3] >> (bi & 7)) & 1)) return 0;
    unsigned np = popcount_bytes(bm, 512);
    const uint8_t *lens = bm + 512;
    uint64_t pos = (uint64_t)BLOB_HDR + fml + 512 + 2ull * np;
    unsigned slot = 0;
    for (int b = 0; b < bi; ++b)
        if ((bm[b >> 3] >> (b & 7)) & 1) { uint16_t l; memcpy(&l, lens + 2 * slot, 2); pos += l; slot++; }
    uint16_t l;
    memcpy(&l, lens + 2 * slot, 2);
    if (pos + l > blob_len) return 0;
    *off = pos; *plen = l;
    return 1;
}

void or_decode_chunk_block(const uint8_t *blob, uint64_t blob_len, int bz, int by, int bx, uint8_t dst[4096]) {
    float q;
    memcpy(&q, blob, 4);
    uint64_t off; uint32_t l;
    if (!blob_block(blob, blob_len, (bz * 16 + by) * 16 + bx, &off, &l)) { memset(dst, 0, OR_N3); return; }
    or_dec_block(blob + off, l, q, dst);
}

void or_decode_chunk(const uint8_t *blob, uint64_t blob_len, uint8_t *out256) {
    float q;
    memcpy(&q, blob, 4);
    uint16_t fml;
    memcpy(&fml, blob + 12, 2);
    const uint8_t *bm = blob + BLOB_HDR + fml;
    unsigned np = popcount_bytes(bm, 512);
    const uint8_t *lens = bm + 512;
    uint64_t pos = (uint64_t)BLOB_HDR + fml + 512 + 2ull * np;
    unsigned slot = 0;
    uint8_t blk[OR_N3];
    for (int bi = 0; bi < OR_N3; ++bi) {
        int present = (bm[bi >> 3] >> (bi & 7)) & 1;
        if (present) {
            uint16_t l;
            memcpy(&l, lens + 2 * slot, 2);
            slot++;
            if (pos + l <= blob_len) or_dec_block(blob + pos, l, q, blk);
            else memset(blk, 0, OR_N3);
            pos += l;
        } else {
            memset(blk, 0, OR_N3);
        }
        int bz = bi >> 8, by = (bi >> 4) & 15, bx = bi & 15;
        for (int z = 0; z < 16; ++z) for (int y = 0; y < 16; ++y)
            memcpy(out256 + ((size_t)(bz * 16 + z) * 256 + (by * 16 + y)) * 256 + bx * 16,
                   blk + z * 256 + y * 16, 16);
    }
}

/* ---- decode-side deblocking (src/mc_codec.c:561-595) ----
 * One face: p1 p0 | q0 q1 along the axis, q0 at index i, the others `step`
 * apart (src/mc_codec.c:563-574). Air voxels (0) are never touched; a step
 * across the face as large as beta is a real edge and is kept; otherwise p0
 * and q0 move towards each other by a clamped 4:1 difference, air neighbours
 * standing in as their face voxel, and stay inside [1, 255]. */
static void db_face(uint8_t *v, size_t total, size_t i, size_t step, int beta, int tc) {
    const int p0 = v[i - step], q0 = v[i];
    if (p0 == 0 || q0 == 0) return;
    const int d = q0 - p0;
    if ((d < 0 ? -d : d) >= beta) return;
    const int p1 = v[i - 2 * step];
    const int q1 = i + step < total ? v[i + step] : 0;
    const int pn = p1 ? p1 : p0, qn = q1 ? q1 : q0;
    int delta = (4 * d + (pn - qn) + 4) >> 3;   /* arithmetic shift: floor */
    if (delta > tc) delta = tc;
    if (delta < -tc) delta = -tc;
    int a = p0 + delta, b = q0 - delta;
    a = a < 1 ? 1 : (a > 255 ? 255 : a);
    b = b < 1 ? 1 : (b > 255 ? 255 : b);
    v[i - step] = (uint8_t)a;
    v[i] = (uint8_t)b;
}

/* Gate and clamp from the quality (src/mc_codec.c:577-578), then the x, y and
 * z faces in that order (:580-594). */
void or_deblock(uint8_t *vol, int nz, int ny, int nx, float quality) {
    const int beta = (int)(3.0f * quality + 6.0f);
    const int tc = (int)(0.5f * quality + 1.0f);
    const size_t sy = (size_t)nx, sz = (size_t)ny * (size_t)nx, total = sz * (size_t)nz;
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 16; x < nx; x += 16) db_face(vol, total, z * sz + y * sy + x, 1, beta, tc);
    for (int z = 0; z < nz; ++z)
        for (int y = 16; y < ny; y += 16)
            for (int x = 0; x < nx; ++x) db_face(vol, total, z * sz + y * sy + x, sy, beta, tc);
    for (int z = 16; z < nz; z += 16)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) db_face(vol, total, z * sz + y * sy + x, sz, beta, tc);
}

/* ---- LOD decimation (src/mc_archive.c:63-72) ---- */
void or_decimate(const uint8_t *src, int DZ, int DY, int DX, uint8_t *dst) {
    const int hz = (DZ + 1) / 2, hy = (DY + 1) / 2, hx = (DX + 1) / 2;
    for (int z = 0; z < hz; ++z)
        for (int y = 0; y < hy; ++y)
            for (int x = 0; x < hx; ++x) {
                int sum = 0, n = 0;
                for (int c = 0; c < 8; ++c) {
                    const int sz = 2 * z + (c >> 2), sy = 2 * y + ((c >> 1) & 1), sx = 2 * x + (c & 1);
                    if (sz >= DZ || sy >= DY || sx >= DX) continue;
                    const int v = src[((size_t)sz * DY + sy) * DX + sx];
                    if (v) { sum += v; n++; }
                }
                dst[((size_t)z * hy + y) * hx + x] = n ? (uint8_t)((sum + n / 2) / n) : 0;
            }
}

uint8_t or_voxel_source(void *ud, int x, int y, int z) {
    const or_volume_src *s = (const or_volume_src *)ud;
    if ((unsigned)z >= (unsigned)s->nz || (unsigned)y >= (unsigned)s->ny || (unsigned)x >= (unsigned)s->nx) return 0;
    return s->v[((size_t)z * s->ny + y) * s->nx + x];
}
