/*
 * qt_oracle.c — TEST INFRASTRUCTURE ONLY (the oracle; never linked into the product).
 *
 * A plain-C, scalar restatement of the reference S3TC codec path of
 * drewcassidy/quicktex (v0.3.1). Every function cites the reference
 * file:line it follows (paths relative to the reference project root).
 * It is pinned two ways by the CPU tests: against the golden vectors of the
 * reference's own tests (tests/golden), and against the unmodified reference
 * compiled from its sources (oracle/_ref/libqtref.so) on seeded inputs.
 *
 * Floating point: x86-64 GCC -O2 with -ffp-contract=off, i.e. IEEE binary32
 * with every operation rounded, in the reference's operation order — the
 * same arithmetic the reference's shipped build performs.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* enums (reference values: BC1Encoder.h:57-100, Interpolator.h:30)          */
/* ------------------------------------------------------------------------- */
enum { CM_INCOMPLETE = 0x00, CM_THREE = 0x03, CM_FOUR = 0x04, CM_THREE_BLACK = 0x13 };
enum { EM_NONE = 0, EM_FASTER = 1, EM_CHECK2 = 2, EM_FULL = 3 };
enum { EP_LS = 0, EP_BB = 1, EP_BBINT = 2, EP_PCA = 3 };
enum { IT_IDEAL = 0, IT_ROUND = 1, IT_NVIDIA = 2, IT_AMD = 3 };

static __thread char g_err[256];

/* Candidate-evaluation (CE) counter: one CE = the SSD of one texel against
 * one palette colour plus its compare/select. Counted per FindSelectors call
 * without the reference's early exits (a full call always costs its texels x
 * candidates): Full 4-colour 64, Full 3-colour 48, Check2 32 + 16
 * projections = 48, Faster/None 16 projections = 16, and the single-colour
 * trial 16. Data-dependent stops (cluster fit at zero error, LS convergence,
 * the endpoint search stop rule) are honoured because they stop the calls. */
static __thread unsigned long long t_ce;
static unsigned long long g_ce;
/* The part of t_ce spent in second four-colour cluster-fit passes that repeat the first
 * pass's trials: the pass's input gives the same start hash and texel order as the first
 * pass's input (or its error is already 0), so it cannot change the result. An encoder may
 * skip them with identical output; counted so that executed work can be told apart from
 * the reference's. */
static __thread unsigned long long t_ce_rep;
static unsigned long long g_ce_rep;
/* the start hash and texel order of the last refine_block_cf's input */
static __thread int t_cf_start;
static __thread uint32_t t_cf_order[16];
static int fail(const char *m) { snprintf(g_err, sizeof g_err, "%s", m); return 1; }
const char *qo_last_error(void) { return g_err; }

/* ------------------------------------------------------------------------- */
/* tables                                                                    */
/* ------------------------------------------------------------------------- */
static uint8_t orders4[969][4], orders3[153][3];
static uint16_t best4[969][128], best3[153][32];
static uint16_t hash4[4096], hash3[256];
static float factors4[969][4], factors3[153][4];
/* OrderTable.cpp:43-44 — kept literally: the 3-colour list is NOT in bin order
 * (bin 1 -> ordering 15, bin 2 -> ordering 89), and GetHash indexes it by bin. */
static const uint16_t single_hash4[4] = {15, 700, 753, 515};
static const uint16_t single_hash3[3] = {12, 15, 89};
/* OrderTable.cpp:40-41: least-squares normal-equation weights
 * {s^2, s(n-s), s(n-s), (n-s)^2} for selector s of an n+1 colour palette. */
static const float weights4[4][4] = {{0, 0, 0, 9}, {1, 2, 2, 4}, {4, 2, 2, 1}, {9, 0, 0, 0}};
static const float weights3[3][4] = {{0, 0, 0, 4}, {1, 1, 1, 1}, {4, 0, 0, 0}};

typedef struct { uint8_t high, low, error; } match_t;
static match_t match5[4][256], match6[4][256]; /* per interpolator type */

/* ------------------------------------------------------------------------- */
/* util.h:110-126, 145-154                                                   */
/* ------------------------------------------------------------------------- */
static int s8to5(int v) { int v2 = v * 31 + 128; return (v2 + (v2 >> 8)) >> 8; }
static int s8to6(int v) { int v2 = v * 63 + 128; return (v2 + (v2 >> 8)) >> 8; }
static int s5to8(int v) { return (v << 3) | (v >> 2); }
static int s6to8(int v) { return (v << 2) | (v >> 4); }
static uint8_t clamp255(int32_t i) { return (uint8_t)(((uint32_t)i & 0xFFFFFF00u) ? (~(i >> 31)) : i); }
static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

typedef struct { uint8_t r, g, b, a; } color_t;
static color_t mkcolor(int r, int g, int b) { color_t c = {(uint8_t)r, (uint8_t)g, (uint8_t)b, 255}; return c; }
static int ch(color_t c, int i) { return i == 0 ? c.r : i == 1 ? c.g : i == 2 ? c.b : c.a; }
static void setch(color_t *c, int i, int v) {
    if (i == 0) c->r = (uint8_t)v; else if (i == 1) c->g = (uint8_t)v; else if (i == 2) c->b = (uint8_t)v; else c->a = (uint8_t)v;
}
static int is_black(color_t c) { return (c.r | c.g | c.b) < 4; } /* Color.h:82 */
static int same_color(color_t a, color_t b) { return a.r == b.r && a.g == b.g && a.b == b.b && a.a == b.a; }
static uint16_t pack565(color_t c) { return (uint16_t)(c.b | (c.g << 5) | (c.r << 11)); } /* Color.cpp:41-46 */
static color_t scale_from_565(color_t c) { return mkcolor(s5to8(c.r), s6to8(c.g), s5to8(c.b)); } /* Color.cpp:116 */
static color_t scale_to_565(color_t c) { return mkcolor(s8to5(c.r), s8to6(c.g), s8to5(c.b)); }   /* Color.cpp:115 */

/* Color.h:87-95 */
static const float mid5[32] = {.015686f, .047059f, .078431f, .111765f, .145098f, .176471f, .207843f, .241176f, .274510f, .305882f, .337255f,
                               .370588f, .403922f, .435294f, .466667f, .5f,      .533333f, .564706f, .596078f, .629412f, .662745f, .694118f,
                               .725490f, .758824f, .792157f, .823529f, .854902f, .888235f, .921569f, .952941f, .984314f, 1e+37f};
static const float mid6[64] = {.007843f, .023529f, .039216f, .054902f, .070588f, .086275f, .101961f, .117647f, .133333f, .149020f, .164706f,
                               .180392f, .196078f, .211765f, .227451f, .245098f, .262745f, .278431f, .294118f, .309804f, .325490f, .341176f,
                               .356863f, .372549f, .388235f, .403922f, .419608f, .435294f, .450980f, .466667f, .482353f, .500000f, .517647f,
                               .533333f, .549020f, .564706f, .580392f, .596078f, .611765f, .627451f, .643137f, .658824f, .674510f, .690196f,
                               .705882f, .721569f, .737255f, .754902f, .772549f, .788235f, .803922f, .819608f, .835294f, .850980f, .866667f,
                               .882353f, .898039f, .913725f, .929412f, .945098f, .960784f, .976471f, .992157f, 1e+37f};

/* x86-64 cvttss2si: out-of-range and NaN give INT_MIN. */
static int f2i_trunc(float v) {
    if (!(v > -2147483904.0f && v < 2147483648.0f)) return INT_MIN;
    return (int)v;
}

/* Color::PreciseRound565, Color.cpp:66-86 */
static color_t precise_round565(const float v[4]) {
    int tr = f2i_trunc(v[0] * 31.0f), tg = f2i_trunc(v[1] * 63.0f), tb = f2i_trunc(v[2] * 31.0f);
    int r = clampi(tr, 0, 31), g = clampi(tg, 0, 63), b = clampi(tb, 0, 31);
    r += v[0] > mid5[r];
    g += v[1] > mid6[g];
    b += v[2] > mid5[b];
    return mkcolor(r, g, b);
}

/* ------------------------------------------------------------------------- */
/* interpolators, Interpolator.cpp:47-138                                    */
/* ------------------------------------------------------------------------- */
static int interp8(int t, int v0, int v1) {
    switch (t) {
        case IT_ROUND: return (v0 * 2 + v1 + 1) / 3;           /* :76 */
        case IT_AMD: return (v0 * 43 + v1 * 21 + 32) >> 6;     /* :136 */
        default: return (v0 * 2 + v1) / 3;                     /* :67 (Nvidia inherits) */
    }
}
static int interp_half8(int t, int v0, int v1) {
    return t == IT_AMD ? ((v0 + v1 + 1) >> 1) : ((v0 + v1) / 2); /* :138, :69 */
}
static int nv_interp5(int v0, int v1) { return ((2 * v0 + v1) * 22) / 8; }              /* :81-84 */
static int nv_interp6(int v0, int v1) { int gd = v1 - v0; return (256 * v0 + (gd / 4) + 128 + gd * 80) >> 8; } /* :86-90 */
static int nv_half5(int v0, int v1) { return ((v0 + v1) * 33) / 8; }                    /* :92-95 */
static int nv_half6(int v0, int v1) { int gd = v1 - v0; return (256 * v0 + gd / 4 + 128 + gd * 128) >> 8; }   /* :97-101 */
static int interp5(int t, int v0, int v1) { return t == IT_NVIDIA ? nv_interp5(v0, v1) : interp8(t, s5to8(v0), s5to8(v1)); }
static int interp6(int t, int v0, int v1) { return t == IT_NVIDIA ? nv_interp6(v0, v1) : interp8(t, s6to8(v0), s6to8(v1)); }

/* Interpolator::InterpolateBC1 (:57-73) and InterpolatorNvidia::InterpolateBC1 (:103-120) */
static void interpolate_bc1(int t, color_t low, color_t high, int use_3color, color_t out[4]) {
    out[0] = scale_from_565(low);
    out[1] = scale_from_565(high);
    if (t == IT_NVIDIA) {
        if (!use_3color) {
            out[2] = mkcolor(nv_interp5(low.r, high.r), nv_interp6(low.g, high.g), nv_interp5(low.b, high.b));
            out[3] = mkcolor(nv_interp5(high.r, low.r), nv_interp6(high.g, low.g), nv_interp5(high.b, low.b));
        } else {
            out[2] = mkcolor(nv_half5(low.r, high.r), nv_half6(low.g, high.g), nv_half5(low.b, high.b));
            out[3] = (color_t){0, 0, 0, 0};
        }
        return;
    }
    if (use_3color) {
        out[2] = mkcolor(interp_half8(t, out[0].r, out[1].r), interp_half8(t, out[0].g, out[1].g), interp_half8(t, out[0].b, out[1].b));
        out[3] = (color_t){0, 0, 0, 0};
    } else {
        out[2] = mkcolor(interp8(t, out[0].r, out[1].r), interp8(t, out[0].g, out[1].g), interp8(t, out[0].b, out[1].b));
        out[3] = mkcolor(interp8(t, out[1].r, out[0].r), interp8(t, out[1].g, out[0].g), interp8(t, out[1].b, out[0].b));
    }
}

/* SingleColorTable<B, N>, SingleColorTable.h:46-90 (N does not enter the computation) */
static void build_match_table(int t, int bits, match_t tab[256]) {
    int size = 1 << bits;
    int ideal = (t == IT_IDEAL || t == IT_ROUND);
    int use8 = (t != IT_NVIDIA);
    for (int i = 0; i < 256; i++) {
        unsigned error = 256;
        for (int low = 0; low < size; low++) {
            int low8 = bits == 5 ? s5to8(low) : s6to8(low);
            for (int high = 0; high < size; high++) {
                int high8 = bits == 5 ? s5to8(high) : s6to8(high);
                int value;
                if (use8) value = interp8(t, high8, low8) & 0xFF;
                else value = (bits == 5 ? interp5(t, high, low) : interp6(t, high, low)) & 0xFF;
                unsigned e = (unsigned)abs(value - i);
                if (ideal) e += (unsigned)(abs(high8 - low8) * 3) / 100;
                if (e < error || (e == error && low == high)) {
                    tab[i].low = (uint8_t)low;
                    tab[i].high = (uint8_t)high;
                    tab[i].error = (uint8_t)e;
                    error = e;
                }
            }
        }
    }
}

/* OrderTable<N>::Generate, OrderTable.h:57-89 */
static void gen_factors(int n, int count, const uint8_t *hist, float (*fac)[4], uint16_t *hashes) {
    const float denom = n == 4 ? 3.0f : 2.0f;
    for (int i = 0; i < count; i++) {
        const uint8_t *h = hist + i * n;
        int any16 = 0;
        unsigned packed = 0;
        for (int s = 0; s < n; s++) any16 |= h[s] == 16;
        for (int s = 0; s < n - 1; s++) packed |= (unsigned)h[s] << (4 * s);
        if (!any16) hashes[packed] = (uint16_t)i;
        float m[4] = {0, 0, 0, 0};
        for (int s = 0; s < n; s++) {
            const float *w = n == 4 ? weights4[s] : weights3[s];
            for (int k = 0; k < 4; k++) m[k] = m[k] + w[k] * (float)h[s];
        }
        float det = (m[0] * m[3]) - (m[1] * m[2]);
        if (fabsf(det) < 1e-8f) {
            fac[i][0] = fac[i][1] = fac[i][2] = fac[i][3] = 0.0f;
        } else {
            float t = m[0]; m[0] = m[3]; m[3] = t;
            m[1] = m[1] * -1.0f; m[2] = m[2] * -1.0f;
            float s = (denom / 255.0f) / det;
            for (int k = 0; k < 4; k++) fac[i][k] = m[k] * s;
        }
    }
}

int qo_init(const char *table_path) {
    FILE *f = fopen(table_path, "rb");
    if (!f) return fail("cannot open order tables");
    static uint8_t raw[262208];
    size_t n = fread(raw, 1, sizeof raw, f);
    fclose(f);
    if (n != sizeof raw || memcmp(raw, "QTOT", 4) != 0) return fail("bad order tables file");
    memcpy(orders4, raw + 8, sizeof orders4);
    memcpy(orders3, raw + 8 + sizeof orders4, sizeof orders3);
    for (int i = 0; i < 969 * 128; i++) ((uint16_t *)best4)[i] = (uint16_t)(raw[4352 + 2 * i] | (raw[4352 + 2 * i + 1] << 8));
    for (int i = 0; i < 153 * 32; i++) ((uint16_t *)best3)[i] = (uint16_t)(raw[252416 + 2 * i] | (raw[252416 + 2 * i + 1] << 8));
    memset(hash4, 0, sizeof hash4);
    memset(hash3, 0, sizeof hash3);
    gen_factors(4, 969, &orders4[0][0], factors4, hash4);
    gen_factors(3, 153, &orders3[0][0], factors3, hash3);
    for (int t = 0; t < 4; t++) {
        build_match_table(t, 5, match5[t]);
        build_match_table(t, 6, match6[t]);
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* BC1 encoder                                                               */
/* ------------------------------------------------------------------------- */
typedef struct {
    int color_mode, interp, error_mode, endpoint_mode;
    int two_ls, two_ep, two_cf, exhaustive;
    unsigned search_rounds, orderings4, orderings3, power_iters;
} bc1p_t;

/* BC1Encoder::SetLevel, BC1Encoder.cpp:74-249 */
static int set_level(bc1p_t *p, unsigned level) {
    if (level > 19) return fail("Level out of range, bust be between 0 and 18 inclusive");
    p->two_ls = p->two_ep = p->two_cf = p->exhaustive = 0;
    p->power_iters = 4;
    p->error_mode = EM_CHECK2;
    p->endpoint_mode = EP_PCA;
    p->search_rounds = 0;
    p->orderings3 = p->orderings4 = 0;
    switch (level) {
        case 0: p->endpoint_mode = EP_BBINT; break;
        case 1: p->endpoint_mode = EP_LS; break;
        case 2: break;
        case 3: p->two_ls = 1; break;
        case 4: p->two_ls = 1; p->error_mode = EM_FULL; p->power_iters = 6; break;
        default:
        case 5: p->two_ls = 1; p->error_mode = EM_FASTER; break;
        case 6: p->two_ls = 1; p->orderings4 = 1; p->orderings3 = 1; p->error_mode = EM_FASTER; break;
        case 7: p->two_ls = 1; p->error_mode = EM_FASTER; p->orderings4 = 4; p->orderings3 = 1; break;
        case 8: p->two_ls = 1; p->error_mode = EM_FASTER; p->orderings4 = 8; p->orderings3 = 1; break;
        case 9: p->two_ls = 1; p->error_mode = EM_CHECK2; p->orderings4 = 11; p->orderings3 = 3; break;
        case 10: p->two_ls = 1; p->error_mode = EM_CHECK2; p->orderings4 = 20; p->orderings3 = 8; break;
        case 11: p->two_ls = 1; p->error_mode = EM_CHECK2; p->orderings4 = 28; p->orderings3 = 16; break;
        case 12: p->two_ls = 1; p->error_mode = EM_CHECK2; p->orderings4 = 32; p->orderings3 = 32; break;
        case 13: p->two_ls = p->two_ep = 1; p->error_mode = EM_FULL; p->orderings4 = 32; p->orderings3 = 32; p->search_rounds = 20; p->power_iters = 6; break;
        case 14: p->two_ls = p->two_ep = 1; p->error_mode = EM_FULL; p->orderings4 = 32; p->orderings3 = 32; p->search_rounds = 32; p->power_iters = 6; break;
        case 15: p->two_ls = p->two_ep = 1; p->error_mode = EM_FULL; p->orderings4 = 56; p->orderings3 = 32; p->search_rounds = 32; p->power_iters = 6; break;
        case 16: p->two_ls = p->two_ep = 1; p->error_mode = EM_FULL; p->orderings4 = 80; p->orderings3 = 32; p->search_rounds = 256; p->power_iters = 6; break;
        case 17: p->two_ls = p->two_ep = 1; p->error_mode = EM_FULL; p->orderings4 = 128; p->orderings3 = 32; p->search_rounds = 256; break;
        case 18: p->two_ls = p->two_ep = p->two_cf = 1; p->error_mode = EM_FULL; p->orderings4 = 128; p->orderings3 = 32; p->search_rounds = 256; p->power_iters = 6; break;
        case 19: p->two_ls = p->two_ep = p->two_cf = p->exhaustive = 1; p->error_mode = EM_FULL; p->orderings4 = 128; p->orderings3 = 32; p->search_rounds = 256; p->power_iters = 6; break;
    }
    p->orderings4 = p->orderings4 < 1 ? 1 : (p->orderings4 > 128 ? 128 : p->orderings4); /* :247-248 */
    p->orderings3 = p->orderings3 < 1 ? 1 : (p->orderings3 > 32 ? 32 : p->orderings3);
    return 0;
}

/* BC1Encoder.h:147-153 */
typedef struct {
    color_t low, high;
    uint8_t sel[16];
    int color_mode;
    unsigned error;
} result_t;

static void result_init(result_t *r) {
    memset(r, 0, sizeof *r);
    r->low = r->high = mkcolor(0, 0, 0);
    r->color_mode = CM_INCOMPLETE;
    r->error = UINT_MAX;
}

/* ColorBlock::Metrics, ColorBlock.h:88-117 */
typedef struct {
    color_t min, max, avg;
    int is_greyscale, has_black;
    int sums[3];
} metrics_t;

static metrics_t get_metrics(const color_t px[16], int ignore_black) {
    metrics_t m;
    m.min = mkcolor(255, 255, 255);
    m.max = mkcolor(0, 0, 0);
    m.avg = mkcolor(0, 0, 0); /* default Color() when no texel counts */
    m.has_black = 0;
    m.is_greyscale = 1;
    m.sums[0] = m.sums[1] = m.sums[2] = 0;
    int total = 0;
    for (int i = 0; i < 16; i++) {
        color_t v = px[i];
        int blk = is_black(v);
        m.has_black |= blk;
        if (ignore_black && blk) continue;
        m.is_greyscale &= (v.r == v.g) && (v.r == v.b);
        for (int c = 0; c < 3; c++) {
            int x = ch(v, c);
            if (x < ch(m.min, c)) setch(&m.min, c, x);
            if (x > ch(m.max, c)) setch(&m.max, c, x);
            m.sums[c] += x;
        }
        total++;
    }
    if (total > 0) {
        /* (sums + total/2) / total; the w lane gives alpha (0 + total/2)/total = 0 */
        m.avg = mkcolor((m.sums[0] + total / 2) / total, (m.sums[1] + total / 2) / total, (m.sums[2] + total / 2) / total);
        m.avg.a = (uint8_t)((total / 2) / total);
    }
    return m;
}

typedef struct {
    bc1p_t p;
} enc_t;

/* FindEndpointsSingleColor(result, color, is_3color), BC1Encoder.cpp:443-456 */
static void find_endpoints_single_color(const bc1p_t *p, result_t *r, color_t c, int is3) {
    /* the 3-colour tables equal the 4-colour ones (SingleColorTable.h: N is unused) */
    match_t mr = match5[p->interp][c.r], mg = match6[p->interp][c.g], mb = match5[p->interp][c.b];
    r->color_mode = is3 ? CM_THREE : CM_FOUR;
    r->error = (unsigned)mr.error + mg.error + mb.error;
    r->low = mkcolor(mr.low, mg.low, mb.low);
    r->high = mkcolor(mr.high, mg.high, mb.high);
}

/* FindEndpointsSingleColor(result, pixels, color, is_3color), BC1Encoder.cpp:458-471:
 * the error is measured against colors[2] of the endpoints held BEFORE the
 * lookup, over all four channels (alpha included, palette alpha = 255). */
static void find_endpoints_single_color_px(const bc1p_t *p, result_t *r, const color_t px[16], color_t c, int is3) {
    color_t cols[4];
    interpolate_bc1(p->interp, r->low, r->high, is3, cols);
    color_t rv = cols[2];
    t_ce += 16;
    find_endpoints_single_color(p, r, c, is3);
    r->error = 0;
    for (int i = 0; i < 16; i++) {
        int dr = px[i].r - rv.r, dg = px[i].g - rv.g, db = px[i].b - rv.b, da = px[i].a - rv.a;
        r->error += (unsigned)(dr * dr + dg * dg + db * db + da * da);
        r->sel[i] = 1;
    }
}

/* FindEndpoints, BC1Encoder.cpp:473-677 */
static void find_endpoints(const bc1p_t *p, result_t *r, const color_t px[16], const metrics_t *m, int mode, int ignore_black) {
    if (m->is_greyscale) { /* :474-494 */
        int fr = px[0].r;
        if (m->max.r - m->min.r < 2) {
            r->low = mkcolor(s8to5(fr), s8to6(fr), s8to5(fr));
            r->high = r->low;
        } else {
            r->low = mkcolor(s8to5(m->min.r), s8to6(m->min.r), s8to5(m->min.r));
            r->high = mkcolor(s8to5(m->max.r), s8to6(m->max.r), s8to5(m->max.r));
        }
    } else if (mode == EP_LS) { /* :495-552 */
        int d[3] = {m->max.r - m->min.r, m->max.g - m->min.g, m->max.b - m->min.b};
        float l[4] = {0, 0, 0, 0}, h[4] = {0, 0, 0, 0};
        int c0 = (d[0] >= d[1] && d[0] >= d[2]) ? 0 : ((d[1] >= d[2] && d[1] >= d[0]) ? 1 : 2); /* Color.cpp:95-99 */
        l[c0] = (float)ch(m->min, c0);
        h[c0] = (float)ch(m->min, c0);
        unsigned sxy[3] = {0, 0, 0}; /* uninitialised in the reference (:510); zero here */
        for (int i = 0; i < 16; i++)
            for (int c = 0; c < 3; c++) sxy[c] += (unsigned)(ch(px[i], c0) * ch(px[i], c));
        const unsigned sum_x = (unsigned)m->sums[c0];
        const unsigned sum_xx = sxy[c0];
        float den = (float)(16u * sum_xx) - (float)(sum_x * sum_x);
        if (fabsf(den) > 1e-8f) {
            for (int i = 1; i < 3; i++) {
                int c = (c0 + i) % 3;
                unsigned sum_y = (unsigned)m->sums[c], sum_xy = sxy[c];
                float a = (float)((16u * sum_xy) - (sum_x * sum_y)) / den;
                float b = (float)((sum_xx * sum_y) - (sum_xy * sum_x)) / den;
                l[c] = b + (a * l[c0]);
                h[c] = b + (a * h[c0]);
            }
        }
        for (int c = 0; c < 3; c++) {
            float inset = (h[c] - l[c]) / 16.0f;
            l[c] = ((l[c] + inset) / 255.0f);
            h[c] = ((h[c] - inset) / 255.0f);
        }
        r->low = precise_round565(l);
        r->high = precise_round565(h);
    } else if (mode == EP_BB) { /* :553-580 */
        float l[4] = {0, 0, 0, 0}, h[4] = {0, 0, 0, 0};
        const float bias = 8.0f / 255.0f;
        for (int c = 0; c < 3; c++) {
            l[c] = (float)ch(m->min, c) / 255.0f;
            h[c] = (float)ch(m->max, c) / 255.0f;
            float inset = (h[c] - l[c] - bias) / 16.0f;
            l[c] += inset;
            h[c] -= inset;
        }
        int cxz = 0, cyz = 0;
        for (int i = 0; i < 16; i++) { /* note the precedence: b*r - avg.r (:572-573) */
            int b = (int)px[i].b - m->avg.b;
            cxz += b * (int)px[i].r - m->avg.r;
            cyz += b * (int)px[i].g - m->avg.g;
        }
        if (cxz < 0) { float t = l[0]; l[0] = h[0]; h[0] = t; }
        if (cyz < 0) { float t = l[1]; l[1] = h[1]; h[1] = t; }
        r->low = precise_round565(l);
        r->high = precise_round565(h);
    } else if (mode == EP_BBINT) { /* :581-605 */
        color_t mn = mkcolor(0, 0, 0), mx = mkcolor(0, 0, 0);
        for (int c = 0; c < 3; c++) {
            int inset = ((int)(ch(m->max, c) - ch(m->min, c)) - 8) >> 4;
            setch(&mn, c, clamp255(ch(m->min, c) + inset));
            setch(&mx, c, clamp255(ch(m->max, c) - inset));
        }
        int cxz = 0, cyz = 0;
        for (int i = 0; i < 16; i++) {
            int b = (int)px[i].b - m->avg.b;
            cxz += b * (int)px[i].r - m->avg.r;
            cyz += b * (int)px[i].g - m->avg.g;
        }
        if (cxz < 0) { uint8_t t = mn.r; mn.r = mx.r; mx.r = t; }
        if (cyz < 0) { uint8_t t = mn.g; mn.g = mx.g; mx.g = t; }
        r->low = scale_to_565(mn);
        r->high = scale_to_565(mx);
    } else if (mode == EP_PCA) { /* :606-674 */
        float mn[4] = {(float)m->min.r, (float)m->min.g, (float)m->min.b, 0};
        float mx[4] = {(float)m->max.r, (float)m->max.g, (float)m->max.b, 0};
        float av[4] = {(float)m->avg.r, (float)m->avg.g, (float)m->avg.b, 0};
        float axis[4] = {306, 601, 117, 0};
        float cov[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
        for (int i = 0; i < 16; i++) {
            if (ignore_black && is_black(px[i])) continue;
            float v[4] = {(float)px[i].r, (float)px[i].g, (float)px[i].b, 0};
            float d[4];
            for (int k = 0; k < 4; k++) d[k] = v[k] - av[k];
            for (int c1 = 0; c1 < 3; c1++)
                for (int c2 = c1; c2 < 3; c2++) cov[c1][c2] += (d[c1] * d[c2]);
        }
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) cov[a][b] = cov[a][b] / 255.0f;
        for (int a = 0; a < 3; a++) /* Matrix4x4::Mirror, Matrix4x4.cpp:41-47 */
            for (int b = a + 1; b < 4; b++) cov[b][a] = cov[a][b];
        float delta[4];
        for (int k = 0; k < 4; k++) delta[k] = mx[k] - mn[k];
        if (cov[0][2] < 0) delta[0] = -delta[0];
        if (cov[1][2] < 0) delta[1] = -delta[1];
        for (unsigned it = 0; it < p->power_iters; it++) { /* Matrix4x4.cpp:33-39, Vector4.h:53-57 */
            float nd[4];
            for (int rr = 0; rr < 4; rr++) {
                float s = 0;
                for (int k = 0; k < 4; k++) s += delta[k] * cov[rr][k];
                nd[rr] = s;
            }
            memcpy(delta, nd, sizeof nd);
        }
        float k = 0; /* Vector4::MaxAbs(3) */
        for (int c = 0; c < 3; c++) { float a = fabsf(delta[c]); if (a > k) k = a; }
        if (k >= 2) {
            float s = 2048.0f / k;
            for (int c = 0; c < 4; c++) axis[c] = delta[c] * s;
        }
        for (int c = 0; c < 4; c++) axis[c] = axis[c] * 16.0f;
        float min_dot = INFINITY, max_dot = -INFINITY;
        int min_i = 0, max_i = 0;
        for (int i = 0; i < 16; i++) {
            if (ignore_black && is_black(px[i])) continue;
            float v[4] = {(float)px[i].r, (float)px[i].g, (float)px[i].b, 0};
            float dot = 0;
            for (int c = 0; c < 4; c++) dot += v[c] * axis[c];
            if (dot > max_dot) { max_dot = dot; max_i = i; }
            if (dot < min_dot) { min_dot = dot; min_i = i; }
        }
        r->low = scale_to_565(px[min_i]);
        r->high = scale_to_565(px[max_i]);
    }
    r->color_mode = CM_INCOMPLETE;
}

static unsigned sqr3(int a, int b, int c) { return (unsigned)(a * a + b * b + c * c); }

/* FindSelectors<M>, BC1Encoder.cpp:679-779 */
static void find_selectors(const bc1p_t *p, int M, result_t *r, const color_t px[16], int em) {
    int cc = M & 0x0F;
    color_t cols[4];
    interpolate_bc1(p->interp, r->low, r->high, cc == 3, cols);
    int cv[4][3];
    int order[4];
    if (cc == 4) { order[0] = 0; order[1] = 2; order[2] = 3; order[3] = 1; }
    else { order[0] = 0; order[1] = 2; order[2] = 1; order[3] = 3; }
    for (int j = 0; j < 4; j++) { cv[j][0] = cols[order[j]].r; cv[j][1] = cols[order[j]].g; cv[j][2] = cols[order[j]].b; }
    unsigned total = 0;
    t_ce += (em == EM_FULL) ? (M == CM_THREE ? 48u : 64u) : (em == EM_CHECK2 ? 48u : 16u);
    if (em == EM_NONE || em == EM_FASTER) {
        int ax[3] = {cv[3][0] - cv[0][0], cv[3][1] - cv[0][1], cv[3][2] - cv[0][2]};
        int dots[4];
        for (int j = 0; j < 4; j++) dots[j] = ax[0] * cv[j][0] + ax[1] * cv[j][1] + ax[2] * cv[j][2];
        int t0 = dots[0] + dots[1], t1 = dots[1] + dots[2], t2 = dots[2] + dots[3];
        for (int c = 0; c < 3; c++) ax[c] *= 2;
        for (int i = 0; i < 16; i++) {
            int pv[3] = {px[i].r, px[i].g, px[i].b};
            int dot = ax[0] * pv[0] + ax[1] * pv[1] + ax[2] * pv[2];
            int level = (dot <= t0) + (dot < t1) + (dot < t2);
            int s = 3 - level;
            if (em == EM_FASTER) {
                total += sqr3(pv[0] - cv[s][0], pv[1] - cv[s][1], pv[2] - cv[s][2]);
                if (i % 4 != 0 && total >= r->error) break;
            }
            r->sel[i] = (uint8_t)s;
        }
    } else if (em == EM_CHECK2) {
        int ax[3] = {cv[3][0] - cv[0][0], cv[3][1] - cv[0][1], cv[3][2] - cv[0][2]};
        const float f = 4.0f / ((float)sqr3(ax[0], ax[1], ax[2]) + .00000125f);
        for (int i = 0; i < 16; i++) {
            int pv[3] = {px[i].r, px[i].g, px[i].b};
            int dd = (pv[0] - cv[0][0]) * ax[0] + (pv[1] - cv[0][1]) * ax[1] + (pv[2] - cv[0][2]) * ax[2];
            float sel_f = (float)dd * f + 0.5f;
            int s = clampi(f2i_trunc(sel_f), 1, 3);
            unsigned e0 = sqr3(cv[s - 1][0] - pv[0], cv[s - 1][1] - pv[1], cv[s - 1][2] - pv[2]);
            unsigned e1 = sqr3(cv[s][0] - pv[0], cv[s][1] - pv[1], cv[s][2] - pv[2]);
            int bs = s;
            unsigned be = e1;
            if (e0 == e1) {
                if (bs == 1) bs = 0;
            } else if (e0 < be) {
                bs = s - 1;
                be = e0;
            }
            total += be;
            if (total >= r->error) break;
            r->sel[i] = (uint8_t)bs;
        }
    } else { /* EM_FULL */
        int max_sel = (M == CM_THREE) ? 3 : 4;
        for (int i = 0; i < 16; i++) {
            unsigned be = UINT_MAX;
            int bs = 0;
            int pv[3] = {px[i].r, px[i].g, px[i].b};
            for (int j = 0; j < max_sel; j++) {
                unsigned e = sqr3(cv[j][0] - pv[0], cv[j][1] - pv[1], cv[j][2] - pv[2]);
                if (e < be || (e == be && j == 3)) { be = e; bs = j; }
            }
            total += be;
            if (total >= r->error) break;
            r->sel[i] = (uint8_t)bs;
        }
    }
    r->error = total;
    r->color_mode = M;
}

/* RefineEndpointsLS<FourColor>(result, pixels, metrics), BC1Encoder.cpp:781-825.
 * Only ever instantiated for FourColor, so no texel is skipped and the
 * 4-colour weights apply whatever the block's colour mode. */
static int refine_endpoints_ls_px(result_t *r, const color_t px[16], const metrics_t *m) {
    float q00[4] = {0, 0, 0, 0};
    float mat[4] = {0, 0, 0, 0};
    for (int i = 0; i < 16; i++) {
        int s = r->sel[i];
        q00[0] += (float)(px[i].r * s);
        q00[1] += (float)(px[i].g * s);
        q00[2] += (float)(px[i].b * s);
        for (int k = 0; k < 4; k++) mat[k] += weights4[s][k];
    }
    float det = (mat[0] * mat[3]) - (mat[1] * mat[2]);
    if (fabsf(det) < 1e-8f) {
        r->color_mode = CM_INCOMPLETE;
        return 0;
    }
    float t = mat[0]; mat[0] = mat[3]; mat[3] = t;
    mat[1] = mat[1] * -1.0f;
    mat[2] = mat[2] * -1.0f;
    float sc = (3.0f / 255.0f) / det;
    for (int k = 0; k < 4; k++) mat[k] = mat[k] * sc;
    float q10[4], lo[4], hi[4];
    for (int c = 0; c < 3; c++) q10[c] = (float)(m->sums[c] * 3) - q00[c];
    q10[3] = 0.0f - q00[3];
    for (int c = 0; c < 4; c++) {
        lo[c] = (mat[0] * q00[c]) + (mat[1] * q10[c]);
        hi[c] = (mat[2] * q00[c]) + (mat[3] * q10[c]);
    }
    r->color_mode = CM_FOUR;
    r->low = precise_round565(lo);
    r->high = precise_round565(hi);
    return 1;
}

/* RefineEndpointsLS<M>(result, sums, matrix, hash), BC1Encoder.cpp:827-850 */
static void refine_endpoints_ls_sums(int M, result_t *r, float sums[17][4], const float mat[4], int hash) {
    int n = M & 0x0F;
    float denom = (float)(n - 1);
    float q10[4] = {0, 0, 0, 0}, q00[4], lo[4], hi[4];
    int level = 0;
    for (int i = 0; i < n - 1; i++) {
        level += n == 4 ? orders4[hash][i] : orders3[hash][i];
        for (int c = 0; c < 4; c++) q10[c] += sums[level][c];
    }
    for (int c = 0; c < 4; c++) q00[c] = (sums[16][c] * denom) - q10[c];
    for (int c = 0; c < 4; c++) {
        lo[c] = (mat[0] * q00[c]) + (mat[1] * q10[c]);
        hi[c] = (mat[2] * q00[c]) + (mat[3] * q10[c]);
    }
    r->color_mode = M;
    r->low = precise_round565(lo);
    r->high = precise_round565(hi);
}

/* RefineBlockLS<M>, BC1Encoder.cpp:852-875 */
static void refine_block_ls(const bc1p_t *p, int M, result_t *r, const color_t px[16], const metrics_t *m, int em, unsigned passes) {
    for (unsigned pass = 0; pass < passes; pass++) {
        result_t t = *r;
        if (!refine_endpoints_ls_px(&t, px, m)) find_endpoints_single_color_px(p, &t, px, m->avg, M != CM_FOUR);
        else find_selectors(p, M, &t, px, em);
        if (same_color(t.low, r->low) && same_color(t.high, r->high)) break;
        if (em == EM_NONE || t.error < r->error) *r = t;
        else return;
    }
}

static int is_single_color_hash(int n, int hash) {
    if (n == 4) return hash == single_hash4[0] || hash == single_hash4[1] || hash == single_hash4[2] || hash == single_hash4[3];
    return hash == single_hash3[0] || hash == single_hash3[1] || hash == single_hash3[2];
}

static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}

/* RefineBlockCF<M>, BC1Encoder.cpp:877-928 */
static void refine_block_cf(const bc1p_t *p, int M, result_t *r, const color_t px[16], const metrics_t *m, int em, unsigned orderings) {
    int n = M & 0x0F;
    result_t orig = *r;
    int hist[4] = {0, 0, 0, 0};
    for (int i = 0; i < 16; i++) hist[orig.sel[i]]++; /* Histogram.h:39-45 */
    int start = -1; /* OrderTable::GetHash, OrderTable.h:91-104 */
    for (int i = 0; i < n; i++)
        if (hist[i] == 16) { start = n == 4 ? single_hash4[i] : single_hash3[i]; break; }
    if (start < 0) {
        unsigned packed = 0;
        for (int i = 0; i < n - 1; i++) packed |= (unsigned)hist[i] << (4 * i);
        start = n == 4 ? hash4[packed] : hash3[packed];
    }
    color_t hi8 = scale_from_565(orig.high), lo8 = scale_from_565(orig.low);
    float axis[4] = {(float)(hi8.r - lo8.r), (float)(hi8.g - lo8.g), (float)(hi8.b - lo8.b), (float)(hi8.a - lo8.a)};
    float cvec[16][4];
    uint32_t dots[16];
    for (int i = 0; i < 16; i++) {
        cvec[i][0] = (float)px[i].r; cvec[i][1] = (float)px[i].g; cvec[i][2] = (float)px[i].b; cvec[i][3] = 0;
        float d = 0;
        for (int c = 0; c < 4; c++) d += cvec[i][c] * axis[c];
        int dot = 0x1000000 + f2i_trunc(d);
        dots[i] = ((uint32_t)dot << 4) | (uint32_t)i;
    }
    qsort(dots, 16, sizeof dots[0], cmp_u32);
    t_cf_start = start;
    for (int i = 0; i < 16; i++) t_cf_order[i] = dots[i] & 0xF;
    float sums[17][4];
    memset(sums, 0, sizeof sums);
    for (int i = 0; i < 16; i++) {
        int q = dots[i] & 0xF;
        for (int c = 0; c < 4; c++) sums[i + 1][c] = sums[i][c] + cvec[q][c];
    }
    unsigned total = p->exhaustive ? (n == 4 ? 969u : 153u) : orderings;
    for (unsigned q = 0; q < total; q++) {
        int th = p->exhaustive ? (int)q : (n == 4 ? best4[start][q] : best3[start][q]);
        const float *mat = n == 4 ? factors4[th] : factors3[th];
        result_t t = orig;
        if (is_single_color_hash(n, th)) {
            find_endpoints_single_color_px(p, &t, px, m->avg, n == 3);
        } else {
            refine_endpoints_ls_sums(M, &t, sums, mat, th);
            find_selectors(p, M, &t, px, em);
        }
        if (t.error < r->error) *r = t;
        if (t.error == 0) break;
    }
}

/* EndpointSearch, BC1Encoder.cpp:930-996 */
static void endpoint_search(const bc1p_t *p, result_t *r, const color_t px[16]) {
    static const int vox[16][4] = {{1, 0, 0, 3},  {0, 1, 0, 4},   {0, 0, 1, 5},   {-1, 0, 0, 0}, {0, -1, 0, 1}, {0, 0, -1, 2},
                                   {1, 1, 0, 9},  {1, 0, 1, 10},  {0, 1, 1, 11},  {-1, -1, 0, 6}, {-1, 0, -1, 7}, {0, -1, -1, 8},
                                   {-1, 1, 0, 13}, {1, -1, 0, 12}, {0, -1, 1, 15}, {0, 1, -1, 14}};
    unsigned prev = 0;
    int forbidden = -1;
    for (unsigned i = 0; i < p->search_rounds; i++) {
        unsigned vi = i & 15;
        if ((int)(i & 31) == forbidden) continue;
        const int *d = vox[vi];
        result_t t = *r;
        color_t *e = (i & 16) ? &t.low : &t.high;
        e->r = (uint8_t)clampi(e->r + d[0], 0, 31);
        e->g = (uint8_t)clampi(e->g + d[1], 0, 63);
        e->b = (uint8_t)clampi(e->b + d[2], 0, 31);
        switch (r->color_mode) {
            default:
            case CM_FOUR: find_selectors(p, CM_FOUR, &t, px, p->error_mode); break;
            case CM_THREE: find_selectors(p, CM_THREE, &t, px, EM_FULL); break;
            case CM_THREE_BLACK: find_selectors(p, CM_THREE_BLACK, &t, px, EM_FULL); break;
        }
        if (t.error < r->error) {
            *r = t;
            forbidden = d[3] | (int)(i & 16);
            prev = i;
        }
        if (i - prev > 32) break;
    }
}

static void put_u16(uint8_t *o, uint16_t v) { o[0] = (uint8_t)(v & 0xFF); o[1] = (uint8_t)(v >> 8); }

/* WriteBlockSolid, BC1Encoder.cpp:345-393 */
static void write_block_solid(const bc1p_t *p, color_t c, uint8_t out[8]) {
    uint8_t mask = 0xAA;
    uint16_t mn, mx;
    if ((c.r | c.g | c.b) == 0) {
        mn = 0; mx = 1; mask = 0x55;
    } else {
        result_t r, r3;
        result_init(&r);
        find_endpoints_single_color(p, &r, c, 0);
        if (p->color_mode & CM_THREE) {
            result_init(&r3);
            find_endpoints_single_color(p, &r3, c, 1);
            if (r3.error < r.error) r = r3;
        }
        mn = pack565(r.low);
        mx = pack565(r.high);
        if (r.color_mode == CM_FOUR) {
            if (mn == mx) {
                if (mn > 0) { mn--; mask = 0; }
                else { mx = 1; mn = 0; mask = 0x55; }
            } else if (mx < mn) {
                uint16_t t = mn; mn = mx; mx = t;
                mask = 0xFF;
            }
        } else if (mx > mn) {
            uint16_t t = mn; mn = mx; mx = t;
        }
    }
    put_u16(out, mx);
    put_u16(out + 2, mn);
    out[4] = out[5] = out[6] = out[7] = mask;
}

/* WriteBlock, BC1Encoder.cpp:395-441 */
static void write_block(const result_t *r, uint8_t out[8]) {
    uint16_t ep1 = pack565(r->low), ep0 = pack565(r->high);
    uint8_t lut[4];
    if (r->color_mode & CM_FOUR) {
        lut[0] = 1; lut[1] = 3; lut[2] = 2; lut[3] = 0;
        if (ep1 > ep0) {
            uint16_t t = ep1; ep1 = ep0; ep0 = t;
            lut[0] = 0; lut[1] = 2; lut[2] = 3; lut[3] = 1;
        } else if (ep1 == ep0) {
            if (ep1 > 0) { ep1--; memset(lut, 0, 4); }
            else { ep0 = 1; ep1 = 0; memset(lut, 1, 4); }
        }
    } else {
        lut[0] = 1; lut[1] = 2; lut[2] = 0; lut[3] = 3;
        if (ep1 < ep0) {
            uint16_t t = ep1; ep1 = ep0; ep0 = t;
            lut[0] = 0; lut[1] = 2; lut[2] = 1; lut[3] = 3;
        }
    }
    put_u16(out, ep0);
    put_u16(out + 2, ep1);
    for (int y = 0; y < 4; y++) { /* BC1Block.cpp:37-43: row y = byte y, texel x at bits 2x */
        uint8_t b = 0;
        for (int x = 0; x < 4; x++) b |= (uint8_t)(lut[r->sel[y * 4 + x]] << (2 * x));
        out[4 + y] = b;
    }
}

/* BC1Encoder::EncodeBlock, BC1Encoder.cpp:261-342 */
static void encode_bc1_block(const bc1p_t *p, const color_t px[16], uint8_t out[8]) {
    int solid = 1;
    for (int i = 1; i < 16; i++) solid &= same_color(px[i], px[0]);
    if (solid) { write_block_solid(p, px[0], out); return; }

    metrics_t m = get_metrics(px, 0);
    const int use_likely = p->exhaustive || p->orderings3 > 0 || p->orderings4 > 0;
    int needs_err = use_likely;
    needs_err |= p->color_mode == CM_THREE;
    needs_err |= (p->color_mode == CM_THREE_BLACK) && m.has_black;
    needs_err |= p->error_mode != EM_NONE;
    needs_err |= p->search_rounds > 0;
    int em = needs_err ? p->error_mode : EM_NONE;
    unsigned ls_passes = p->two_ls ? 2 : 1, cf_passes = p->two_cf ? 2 : 1;
    unsigned ep_passes = (needs_err && p->two_ep) ? 2 : 1;

    result_t orig, res;
    result_init(&orig);
    result_init(&res);
    for (unsigned round = 0; round < ep_passes; round++) {
        int mode = round == 1 ? EP_BB : p->endpoint_mode;
        result_t to, tr;
        result_init(&to);
        find_endpoints(p, &to, px, &m, mode, 0);
        tr = to;
        find_selectors(p, CM_FOUR, &tr, px, em);
        refine_block_ls(p, CM_FOUR, &tr, px, &m, em, ls_passes);
        if (!needs_err || tr.error < res.error) { res = tr; orig = to; }
    }
    if (res.error > 0 && use_likely) {
        int start1 = 0;
        uint32_t order1[16];
        for (unsigned it = 0; it < cf_passes; it++) {
            const unsigned long long ce0 = t_ce;
            const unsigned err0 = res.error;
            refine_block_cf(p, CM_FOUR, &res, px, &m, p->error_mode, p->orderings4);
            if (it == 0) {
                start1 = t_cf_start;
                memcpy(order1, t_cf_order, sizeof order1);
            } else if (err0 == 0 || (t_cf_start == start1 && !memcmp(t_cf_order, order1, sizeof order1))) {
                t_ce_rep += t_ce - ce0;
            }
        }
    }

    if (res.error > 0 && (p->color_mode & CM_THREE)) {
        result_t t = orig;
        find_selectors(p, CM_THREE, &t, px, EM_FULL);
        refine_block_ls(p, CM_THREE, &t, px, &m, EM_FULL, ls_passes);
        if (t.error > 0 && use_likely)
            for (unsigned it = 0; it < cf_passes; it++) refine_block_cf(p, CM_THREE, &t, px, &m, EM_FULL, p->orderings3);
        if (t.error < res.error) res = t;
    }

    if (res.error > 0 && p->color_mode == CM_THREE_BLACK && m.has_black && !is_black(m.max)) {
        result_t t;
        result_init(&t);
        metrics_t mnb = get_metrics(px, 1);
        find_endpoints(p, &t, px, &mnb, EP_PCA, 1);
        find_selectors(p, CM_THREE_BLACK, &t, px, EM_FULL);
        refine_block_ls(p, CM_THREE_BLACK, &t, px, &mnb, EM_FULL, ls_passes);
        if (t.error < res.error) res = t;
    }

    if (res.error > 0 && p->search_rounds > 0) endpoint_search(p, &res, px);
    write_block(&res, out);
}

/* ------------------------------------------------------------------------- */
/* BC4, BC4Encoder.cpp:30-71, BC4Block.cpp                                  */
/* ------------------------------------------------------------------------- */
static void encode_bc4_block(const color_t px[16], int channel, uint8_t out[8]) {
    int mn = 255, mx = 0;
    for (int i = 0; i < 16; i++) { int v = ch(px[i], channel); if (v < mn) mn = v; if (v > mx) mx = v; }
    if (mx == mn) { /* BC4Block(min): solid */
        out[0] = out[1] = (uint8_t)mn;
        memset(out + 2, 0, 6);
        return;
    }
    static const uint8_t levels[8] = {1, 7, 6, 5, 4, 3, 2, 0};
    const int bias = 4 - mn * 14, delta = mx - mn;
    int th[7];
    for (int i = 0; i < 7; i++) th[i] = delta * (1 + 2 * i) - bias;
    uint64_t bits = 0;
    for (int i = 0; i < 16; i++) {
        int v = ch(px[i], channel) * 14;
        int lvl = 0;
        for (int c = 0; c < 7; c++) lvl += v >= th[c];
        bits |= (uint64_t)levels[lvl] << (3 * i); /* row-major, 3 bits each (BC4Block.cpp:36-42) */
    }
    out[0] = (uint8_t)mx;
    out[1] = (uint8_t)mn;
    for (int k = 0; k < 6; k++) out[2 + k] = (uint8_t)(bits >> (8 * k));
}

/* BC4Block::GetValues6/8, BC4Block.cpp:44-64 */
static void bc4_values(const uint8_t blk[8], int v[8]) {
    int a0 = blk[0], a1 = blk[1];
    v[0] = a0; v[1] = a1;
    if (a0 <= a1) {
        v[2] = (a0 * 4 + a1) / 5; v[3] = (a0 * 3 + a1 * 2) / 5; v[4] = (a0 * 2 + a1 * 3) / 5; v[5] = (a0 + a1 * 4) / 5;
        v[6] = 0; v[7] = 255;
    } else {
        v[2] = (a0 * 6 + a1) / 7; v[3] = (a0 * 5 + a1 * 2) / 7; v[4] = (a0 * 4 + a1 * 3) / 7;
        v[5] = (a0 * 3 + a1 * 4) / 7; v[6] = (a0 * 2 + a1 * 5) / 7; v[7] = (a0 + a1 * 6) / 7;
    }
}

/* ------------------------------------------------------------------------- */
/* texture loops: RawTexture::GetBlock (Texture.h:89-112, wrap at edges),   */
/* BlockEncoder::Encode (Encoder.h:36-56), BlockDecoder::Decode             */
/* (Decoder.h:36-54) with RawTexture::SetBlock (Texture.h:114-134)          */
/* ------------------------------------------------------------------------- */
static void get_block(const uint8_t *rgba, int w, int h, int bx, int by, color_t px[16]) {
    for (int y = 0; y < 4; y++)
        for (int x = 0; x < 4; x++) {
            int sx = (bx * 4 + x) % w, sy = (by * 4 + y) % h;
            const uint8_t *s = rgba + 4 * ((size_t)sy * w + sx);
            px[y * 4 + x] = (color_t){s[0], s[1], s[2], s[3]};
        }
}

/* decode writes in the reference's order (by, bx, x, y); later writes win */
static void set_block(uint8_t *rgba, int w, int h, int bx, int by, const color_t px[16]) {
    for (int x = 0; x < 4; x++)
        for (int y = 0; y < 4; y++) {
            int tx = (bx * 4 + x) % w, ty = (by * 4 + y) % h;
            uint8_t *d = rgba + 4 * ((size_t)ty * w + tx);
            color_t c = px[y * 4 + x];
            d[0] = c.r; d[1] = c.g; d[2] = c.b; d[3] = c.a;
        }
}

typedef void (*block_fn)(const void *ctx, const color_t px[16], uint8_t *out);

static int encode_texture(const uint8_t *rgba, int w, int h, const void *ctx, block_fn fn, int bsize, uint8_t *out, int mode) {
    if (w <= 0 || h <= 0) return fail("Texture width must be greater than 0");
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    long n = (long)bw * bh;
    if (mode == 1) {
#pragma omp parallel for schedule(dynamic, 64)
        for (long i = 0; i < n; i++) {
            color_t px[16];
            get_block(rgba, w, h, (int)(i % bw), (int)(i / bw), px);
            t_ce = t_ce_rep = 0;
            fn(ctx, px, out + i * bsize);
#pragma omp atomic
            g_ce += t_ce;
#pragma omp atomic
            g_ce_rep += t_ce_rep;
        }
    } else {
        for (long i = 0; i < n; i++) {
            color_t px[16];
            get_block(rgba, w, h, (int)(i % bw), (int)(i / bw), px);
            t_ce = t_ce_rep = 0;
            fn(ctx, px, out + i * bsize);
            g_ce += t_ce;
            g_ce_rep += t_ce_rep;
        }
    }
    return 0;
}

static void fn_bc1(const void *ctx, const color_t px[16], uint8_t *out) { encode_bc1_block((const bc1p_t *)ctx, px, out); }
static void fn_bc3(const void *ctx, const color_t px[16], uint8_t *out) {
    encode_bc4_block(px, 3, out);                  /* BC3Block: alpha BC4 first (BC3Block.h:38-39) */
    encode_bc1_block((const bc1p_t *)ctx, px, out + 8);
}
typedef struct { int c0, c1; } chan_t;
static void fn_bc4(const void *ctx, const color_t px[16], uint8_t *out) { encode_bc4_block(px, ((const chan_t *)ctx)->c0, out); }
static void fn_bc5(const void *ctx, const color_t px[16], uint8_t *out) {
    encode_bc4_block(px, ((const chan_t *)ctx)->c0, out);
    encode_bc4_block(px, ((const chan_t *)ctx)->c1, out + 8);
}

static int make_params(bc1p_t *p, int level, int color_mode, int interp, const int *ov) {
    if (color_mode != CM_FOUR && color_mode != CM_THREE && color_mode != CM_THREE_BLACK)
        return fail("Encoder color mode must be FourColor, ThreeColor, or ThreeColorBlack");
    if (interp < 0 || interp > 3) return fail("Invalid interpolator type");
    if (set_level(p, (unsigned)level)) return 1;
    p->color_mode = color_mode;
    p->interp = interp;
    if (ov) {
        if (ov[0] >= 0) p->error_mode = ov[0];
        if (ov[1] >= 0) p->endpoint_mode = ov[1];
        if (ov[2] >= 0) p->two_ls = ov[2] != 0;
        if (ov[3] >= 0) p->two_ep = ov[3] != 0;
        if (ov[4] >= 0) p->two_cf = ov[4] != 0;
        if (ov[5] >= 0) p->exhaustive = ov[5] != 0;
        if (ov[6] >= 0) p->search_rounds = (unsigned)ov[6];
        if (ov[7] >= 0) p->orderings4 = ov[7] < 1 ? 1 : (ov[7] > 128 ? 128 : (unsigned)ov[7]);
        if (ov[8] >= 0) p->orderings3 = ov[8] < 1 ? 1 : (ov[8] > 32 ? 32 : (unsigned)ov[8]);
        if (ov[9] >= 0) p->power_iters = ov[9] < 4 ? 4 : (ov[9] > 10 ? 10 : (unsigned)ov[9]);
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* exported C-ABI (mirrors oracle/ref_harness.cpp)                           */
/* ------------------------------------------------------------------------- */
/* total candidate evaluations of the encodes since the last reset */
unsigned long long qo_ce_count(void) { return g_ce; }
/* of those, the evaluations in repeated second cluster-fit passes */
unsigned long long qo_ce_repeated_count(void) { return g_ce_rep; }
void qo_ce_reset(void) { g_ce = g_ce_rep = 0; }

int qo_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void qo_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int qo_bc1_level_params(int level, int color_mode, int *out) {
    bc1p_t p;
    if (make_params(&p, level, color_mode, 0, NULL)) return 1;
    out[0] = p.error_mode; out[1] = p.endpoint_mode; out[2] = p.two_ls; out[3] = p.two_ep; out[4] = p.two_cf;
    out[5] = p.exhaustive; out[6] = (int)p.search_rounds; out[7] = (int)p.orderings4; out[8] = (int)p.orderings3;
    out[9] = (int)p.power_iters;
    return 0;
}

int qo_bc1_encode(const uint8_t *rgba, int w, int h, int level, int color_mode, int interp, const int *ov, uint8_t *out, int mode) {
    bc1p_t p;
    if (make_params(&p, level, color_mode, interp, ov)) return 1;
    return encode_texture(rgba, w, h, &p, fn_bc1, 8, out, mode);
}

int qo_bc3_encode(const uint8_t *rgba, int w, int h, int level, int interp, uint8_t *out, int mode) {
    bc1p_t p; /* BC3Encoder.h:39-42: BC1 in FourColor + BC4 on channel 3 */
    if (make_params(&p, level, CM_FOUR, interp, NULL)) return 1;
    return encode_texture(rgba, w, h, &p, fn_bc3, 16, out, mode);
}

int qo_bc4_encode(const uint8_t *rgba, int w, int h, int channel, uint8_t *out, int mode) {
    if (channel < 0 || channel > 3) return fail("Channel out of range");
    chan_t c = {channel, channel};
    return encode_texture(rgba, w, h, &c, fn_bc4, 8, out, mode);
}

int qo_bc5_encode(const uint8_t *rgba, int w, int h, int c0, int c1, uint8_t *out, int mode) {
    if (c0 < 0 || c0 > 3 || c1 < 0 || c1 > 3) return fail("Channel out of range");
    chan_t c = {c0, c1};
    return encode_texture(rgba, w, h, &c, fn_bc5, 16, out, mode);
}

/* BC1Decoder::DecodeBlock, BC1Decoder.cpp:33-52 */
static void decode_bc1_block(const uint8_t blk[8], int interp, int write_alpha, int allow_3color, color_t px[16]) {
    uint16_t c0 = (uint16_t)(blk[0] | (blk[1] << 8)), c1 = (uint16_t)(blk[2] | (blk[3] << 8));
    color_t lo = {(uint8_t)((c0 >> 11) & 0x1F), (uint8_t)((c0 >> 5) & 0x3F), (uint8_t)(c0 & 0x1F), 255};
    color_t hi = {(uint8_t)((c1 >> 11) & 0x1F), (uint8_t)((c1 >> 5) & 0x3F), (uint8_t)(c1 & 0x1F), 255};
    color_t cols[4];
    interpolate_bc1(interp, lo, hi, allow_3color && (c1 >= c0), cols); /* Interpolator.cpp:52-55 */
    for (int i = 0; i < 16; i++) {
        int s = (blk[4 + i / 4] >> (2 * (i % 4))) & 3;
        px[i] = cols[s];
        if (!write_alpha) px[i].a = 255;
    }
}

static void bc4_decode_into(const uint8_t blk[8], int channel, color_t px[16]) { /* BC4Decoder.cpp:29-43 */
    int v[8];
    bc4_values(blk, v);
    uint64_t bits = 0;
    for (int k = 0; k < 6; k++) bits |= (uint64_t)blk[2 + k] << (8 * k);
    for (int i = 0; i < 16; i++) setch(&px[i], channel, v[(bits >> (3 * i)) & 7]);
}

static void clear_block(color_t px[16]) {
    for (int i = 0; i < 16; i++) px[i] = (color_t){0, 0, 0, 255};
}

int qo_bc1_decode(const uint8_t *blocks, int w, int h, int interp, int write_alpha, uint8_t *out) {
    if (w <= 0 || h <= 0) return fail("Texture width must be greater than 0");
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            color_t px[16];
            decode_bc1_block(blocks + 8 * ((size_t)by * bw + bx), interp, write_alpha, 1, px);
            set_block(out, w, h, bx, by, px);
        }
    return 0;
}

int qo_bc3_decode(const uint8_t *blocks, int w, int h, int interp, uint8_t *out) {
    if (w <= 0 || h <= 0) return fail("Texture width must be greater than 0");
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            const uint8_t *b = blocks + 16 * ((size_t)by * bw + bx);
            color_t px[16];
            decode_bc1_block(b + 8, interp, 0, 0, px); /* BC3Decoder.cpp:27: 4-colour only */
            bc4_decode_into(b, 3, px);
            set_block(out, w, h, bx, by, px);
        }
    return 0;
}

int qo_bc4_decode(const uint8_t *blocks, int w, int h, int channel, uint8_t *out) {
    if (w <= 0 || h <= 0) return fail("Texture width must be greater than 0");
    if (channel < 0 || channel > 3) return fail("Channel out of range");
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            color_t px[16];
            clear_block(px);
            bc4_decode_into(blocks + 8 * ((size_t)by * bw + bx), channel, px);
            set_block(out, w, h, bx, by, px);
        }
    return 0;
}

int qo_bc5_decode(const uint8_t *blocks, int w, int h, int c0, int c1, uint8_t *out) {
    if (w <= 0 || h <= 0) return fail("Texture width must be greater than 0");
    if (c0 < 0 || c0 > 3 || c1 < 0 || c1 > 3) return fail("Channel out of range");
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            const uint8_t *b = blocks + 16 * ((size_t)by * bw + bx);
            color_t px[16];
            clear_block(px);
            bc4_decode_into(b, c0, px);
            bc4_decode_into(b + 8, c1, px);
            set_block(out, w, h, bx, by, px);
        }
    return 0;
}
