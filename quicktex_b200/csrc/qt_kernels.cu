// qt_kernels.cu — sm_100a kernels of the S3TC encode/decode path.
//
// Mapping. BC1 (and the colour half of BC3) runs one 4x4 block per group of
// 16 lanes (two blocks per warp). Each phase of the reference encoder
// (BC1Encoder::EncodeBlock, BC1Encoder.cpp:261-342) picks its own lane
// mapping:
//   * texel-parallel  (lane = texel): metrics, FindEndpoints, FindSelectors,
//     RefineEndpointsLS(pixels). Every sum the reference accumulates over texels
//     is integer-valued (in int or in float below 2^24), so warp reductions
//     (redux.sync) give the reference's exact values in any order.
//   * ordering-parallel (lane = cluster-fit ordering): RefineBlockCF. All
//     orderings start from the same `orig` result, so the reference's
//     sequential "keep if strictly better, stop at zero error" loop equals an
//     argmin over (error, ordering index).
//   * round-parallel (lane = search round): EndpointSearch. Rounds between two
//     improvements all start from the same result, so 16 consecutive rounds are
//     evaluated speculatively and the first improving one (or the stop rule)
//     decides, exactly as the sequential loop would.
// The reference's FindSelectors early exits never change an accepted result
// (every exit bound is >= the later acceptance bound), so full errors are
// computed instead.
//
// Floating point. Every operation whose rounding matters is written with an
// explicit round-to-nearest intrinsic (__fadd_rn, __fmul_rn, __fdiv_rn), in
// the reference's operation order; the compiler never contracts these into
// FMAs. Plain float arithmetic (and fmaf) is used only where every operand and
// result is an integer below 2^24, i.e. exact.
//
// BC4/BC5 encode and all decoders are HBM-bound: one thread per block,
// 16-byte row loads/stores where the texture is 4-aligned.

#include <cuda_runtime.h>

#include <cfloat>
#include <climits>
#include <cstdint>
#include <cstdlib>

#include "qt_internal.h"

namespace qtk {

// ---------------------------------------------------------------------------
// constant tables
// ---------------------------------------------------------------------------
struct DevTables {
    uint16_t best4[969 * 128];
    uint16_t best3[153 * 32];
    uint16_t hash4[4096];
    uint16_t hash3[256];
    float4 factors4[969];
    float4 factors3[153];
    uint32_t orders4[969];
    uint32_t orders3[153];
    uint32_t match5[4][256];
    uint32_t match6[4][256];
};
static_assert(sizeof(DevTables) == sizeof(HostTables), "device and host table images must match");

__device__ DevTables g_tab;

// Color::PreciseRound565 rounding points (Color.h:87-95); the values must be
// these exact floats for the rounding to match.
__constant__ float c_mid5[32] = {.015686f, .047059f, .078431f, .111765f, .145098f, .176471f, .207843f, .241176f,
                                 .274510f, .305882f, .337255f, .370588f, .403922f, .435294f, .466667f, .5f,
                                 .533333f, .564706f, .596078f, .629412f, .662745f, .694118f, .725490f, .758824f,
                                 .792157f, .823529f, .854902f, .888235f, .921569f, .952941f, .984314f, 1e+37f};
__constant__ float c_mid6[64] = {
    .007843f, .023529f, .039216f, .054902f, .070588f, .086275f, .101961f, .117647f, .133333f, .149020f, .164706f,
    .180392f, .196078f, .211765f, .227451f, .245098f, .262745f, .278431f, .294118f, .309804f, .325490f, .341176f,
    .356863f, .372549f, .388235f, .403922f, .419608f, .435294f, .450980f, .466667f, .482353f, .500000f, .517647f,
    .533333f, .549020f, .564706f, .580392f, .596078f, .611765f, .627451f, .643137f, .658824f, .674510f, .690196f,
    .705882f, .721569f, .737255f, .754902f, .772549f, .788235f, .803922f, .819608f, .835294f, .850980f, .866667f,
    .882353f, .898039f, .913725f, .929412f, .945098f, .960784f, .976471f, .992157f, 1e+37f};

// EndpointSearch voxel steps (BC1Encoder.cpp:933-950): dr, dg, db in 2-bit
// two's complement fields (bits 0-1, 2-3, 4-5) and the opposite step's index
// in bits 8-11.
__constant__ uint16_t c_voxels[16] = {
    0x301, 0x404, 0x510, 0x003, 0x10C, 0x230, 0x905, 0xA11, 0xB14, 0x60F, 0x733, 0x83C, 0xD07, 0xC0D, 0xF1C, 0xE34};

constexpr int CM_INCOMPLETE = 0x00, CM_THREE = 0x03, CM_FOUR = 0x04, CM_TB = 0x13;
constexpr int EM_NONE = 0, EM_FASTER = 1, EM_CHECK2 = 2, EM_FULL = 3;
constexpr int EP_LS = 0, EP_BB = 1, EP_BBINT = 2, EP_PCA = 3;
constexpr int IT_IDEAL = 0, IT_ROUND = 1, IT_NVIDIA = 2, IT_AMD = 3;

constexpr int kGroupsPerCta = 8;  // 16-lane groups per 128-thread CTA

// BC4 selector for each threshold count (BC4Encoder.cpp:46 Levels {1,7,6,5,4,3,2,0}), 3 bits each
constexpr uint32_t kBC4Levels = 1u | (7u << 3) | (6u << 6) | (5u << 9) | (4u << 12) | (3u << 15) | (2u << 18) | (0u << 21);

// ---------------------------------------------------------------------------
// scalar helpers (util.h:110-154, Color.cpp)
// ---------------------------------------------------------------------------
__device__ __forceinline__ int s8to5(int v) { int v2 = v * 31 + 128; return (v2 + (v2 >> 8)) >> 8; }
__device__ __forceinline__ int s8to6(int v) { int v2 = v * 63 + 128; return (v2 + (v2 >> 8)) >> 8; }
__device__ __forceinline__ int s5to8(int v) { return (v << 3) | (v >> 2); }
__device__ __forceinline__ int s6to8(int v) { return (v << 2) | (v >> 4); }
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
__device__ __forceinline__ int clamp255(int i) { return ((unsigned)i & 0xFFFFFF00u) ? ((~(i >> 31)) & 0xFF) : i; }
// float -> int with x86 cvttss2si semantics (INT_MIN when out of range or NaN)
__device__ __forceinline__ int f2i_x86(float v) {
    return (v > -2147483904.0f && v < 2147483648.0f) ? __float2int_rz(v) : INT_MIN;
}
// 5:6:5 endpoint packed as Pack565Unscaled (Color.cpp:41-46)
__device__ __forceinline__ int epr(int e) { return e >> 11; }
__device__ __forceinline__ int epg(int e) { return (e >> 5) & 63; }
__device__ __forceinline__ int epb(int e) { return e & 31; }
__device__ __forceinline__ int eppack(int r, int g, int b) { return (r << 11) | (g << 5) | b; }
__device__ __forceinline__ int sel4(int a0, int a1, int a2, int a3, int s) {
    return s == 0 ? a0 : (s == 1 ? a1 : (s == 2 ? a2 : a3));
}
__device__ __forceinline__ float sel4f(float a0, float a1, float a2, float a3, int s) {
    return s == 0 ? a0 : (s == 1 ? a1 : (s == 2 ? a2 : a3));
}
__device__ __forceinline__ unsigned sq3(int a, int b, int c) { return (unsigned)(a * a + b * b + c * c); }

// Color::PreciseRound565 (Color.cpp:66-86)
__device__ __forceinline__ int precise_round565(float v0, float v1, float v2, const float *mid5, const float *mid6) {
    int r = clampi(f2i_x86(__fmul_rn(v0, 31.0f)), 0, 31);
    int g = clampi(f2i_x86(__fmul_rn(v1, 63.0f)), 0, 63);
    int b = clampi(f2i_x86(__fmul_rn(v2, 31.0f)), 0, 31);
    r += v0 > mid5[r];
    g += v1 > mid6[g];
    b += v2 > mid5[b];
    return eppack(r, g, b);
}

// PreciseRound565 of a cluster-fit trial's endpoint. The trial endpoints are table factors
// times sums of at most 3 * 16 * 255: over the factor tables |v| * 63 < 9500, finite and far
// inside int range, so truncation needs no x86 out-of-range case; the unsigned conversion
// saturates negatives to 0, which is the lower clamp.
__device__ __forceinline__ int precise_round565_cf(float v0, float v1, float v2, const float *mid5, const float *mid6) {
    int r = (int)min(__float2uint_rz(__fmul_rn(v0, 31.0f)), 31u);
    int g = (int)min(__float2uint_rz(__fmul_rn(v1, 63.0f)), 63u);
    int b = (int)min(__float2uint_rz(__fmul_rn(v2, 31.0f)), 31u);
    r += v0 > mid5[r];
    g += v1 > mid6[g];
    b += v2 > mid5[b];
    return eppack(r, g, b);
}

// ---------------------------------------------------------------------------
// interpolators (Interpolator.cpp:47-138)
// ---------------------------------------------------------------------------
// a, b are channel values (non-negative), so unsigned division gives the same quotients
template <int IT> __device__ __forceinline__ int i8(int a, int b) {
    const unsigned ua = (unsigned)a, ub = (unsigned)b;
    if (IT == IT_ROUND) return (int)((ua * 2 + ub + 1) / 3);
    if (IT == IT_AMD) return (int)((ua * 43 + ub * 21 + 32) >> 6);
    return (int)((ua * 2 + ub) / 3);
}
template <int IT> __device__ __forceinline__ int h8(int a, int b) {
    return (int)(IT == IT_AMD ? (((unsigned)a + (unsigned)b + 1) >> 1) : (((unsigned)a + (unsigned)b) / 2));
}
__device__ __forceinline__ int nv5(int a, int b) { return (int)((((unsigned)a * 2 + (unsigned)b) * 22) / 8); }
__device__ __forceinline__ int nv6(int a, int b) { int gd = b - a; return (256 * a + (gd / 4) + 128 + gd * 80) >> 8; }
__device__ __forceinline__ int nvh5(int a, int b) { return (int)((((unsigned)a + (unsigned)b) * 33) / 8); }
__device__ __forceinline__ int nvh6(int a, int b) { int gd = b - a; return (256 * a + gd / 4 + 128 + gd * 128) >> 8; }

// Palette in FindSelectors' internal selector order (BC1Encoder.cpp:684-693):
// four colours {c0, c2, c3, c1}, three colours {c0, c2, c1, c3=black}.
struct Pal {
    int r0, g0, b0, r1, g1, b1, r2, g2, b2, r3, g3, b3;
};

template <int IT> __device__ __forceinline__ Pal make_pal(int lo, int hi, bool three) {
    const int lr = epr(lo), lg = epg(lo), lb = epb(lo), hr = epr(hi), hg = epg(hi), hb = epb(hi);
    const int ar = s5to8(lr), ag = s6to8(lg), ab = s5to8(lb);  // colors[0]
    const int br = s5to8(hr), bg = s6to8(hg), bb = s5to8(hb);  // colors[1]
    int cr, cg, cb, dr, dg, db;                                // colors[2], colors[3]
    if (IT == IT_NVIDIA) {
        if (!three) {
            cr = nv5(lr, hr); cg = nv6(lg, hg); cb = nv5(lb, hb);
            dr = nv5(hr, lr); dg = nv6(hg, lg); db = nv5(hb, lb);
        } else {
            cr = nvh5(lr, hr); cg = nvh6(lg, hg); cb = nvh5(lb, hb);
            dr = dg = db = 0;
        }
    } else if (three) {
        cr = h8<IT>(ar, br); cg = h8<IT>(ag, bg); cb = h8<IT>(ab, bb);
        dr = dg = db = 0;
    } else {
        cr = i8<IT>(ar, br); cg = i8<IT>(ag, bg); cb = i8<IT>(ab, bb);
        dr = i8<IT>(br, ar); dg = i8<IT>(bg, ag); db = i8<IT>(bb, ab);
    }
    Pal p;
    p.r0 = ar; p.g0 = ag; p.b0 = ab;
    p.r1 = cr; p.g1 = cg; p.b1 = cb;
    if (!three) {
        p.r2 = dr; p.g2 = dg; p.b2 = db;
        p.r3 = br; p.g3 = bg; p.b3 = bb;
    } else {
        p.r2 = br; p.g2 = bg; p.b2 = bb;
        p.r3 = dr; p.g3 = dg; p.b3 = db;
    }
    return p;
}

// ---------------------------------------------------------------------------
// per-CTA shared state of the BC1 kernel. File scope, so that the phase
// functions below (kept __noinline__: one copy each, a small instruction
// working set per launch) reach the block being encoded without passing it.
// ---------------------------------------------------------------------------
__shared__ float s_mid5[32], s_mid6[64];
__shared__ uint16_t s_vox[16];
__shared__ uint32_t s_px[kGroupsPerCta][16];      // the block's texels, RGBA8
__shared__ float4 s_pf[kGroupsPerCta][16];        // (r, g, b, r^2+g^2+b^2) as exact floats
__shared__ int s_sum[kGroupsPerCta][17 * 3];       // cluster-fit prefix sums
__shared__ uint16_t s_row[kGroupsPerCta][128];     // BestOrders row of the current cluster fit
__shared__ int s_met[kGroupsPerCta][2][16];        // metrics: [0] all texels, [1] ignoring black
__shared__ int s_pp[kGroupsPerCta];                // sum over the block of r^2 + g^2 + b^2

// metric slots
constexpr int MT_MN = 0, MT_MX = 3, MT_AV = 6, MT_SUM = 9, MT_GREY = 12, MT_BLACK = 13;

struct Grp {
    unsigned gm;  // the group's 16 lanes within the warp
    int lane;     // texel index in phases that map lanes to texels
    int g;        // group index within the CTA
};
__device__ __forceinline__ Grp grp() {
    Grp G;
    G.lane = threadIdx.x & 15;
    G.g = threadIdx.x >> 4;
    G.gm = 0xFFFFu << (threadIdx.x & 16);
    return G;
}

struct Res {  // EncodeResults (BC1Encoder.h:147-153); endpoints packed 5:6:5
    int lo, hi;
    uint32_t sel;  // 16 x 2-bit internal selectors, texel i at bits 2i
    int mode;
    uint32_t err;
};

__device__ __forceinline__ Res res_init() {
    Res r;
    r.lo = r.hi = 0;
    r.sel = 0;
    r.mode = CM_INCOMPLETE;
    r.err = UINT_MAX;
    return r;
}

struct SelErr {
    uint32_t sel, err;
};

__device__ __forceinline__ unsigned gsum(unsigned m, unsigned v) { return __reduce_add_sync(m, v); }
__device__ __forceinline__ unsigned gmin(unsigned m, unsigned v) { return __reduce_min_sync(m, v); }
__device__ __forceinline__ unsigned gmax(unsigned m, unsigned v) { return __reduce_max_sync(m, v); }
__device__ __forceinline__ unsigned gor(unsigned m, unsigned v) { return __reduce_or_sync(m, v); }

// Selector-search kinds: the (colour mode, error mode) pairs FindSelectors is
// ever called with. Three-colour searches are always ErrorMode::Full
// (BC1Encoder.cpp:313-333, 978-984).
constexpr int K_F4_NONE = 0, K_F4_FASTER = 1, K_F4_CHECK2 = 2, K_F4_FULL = 3, K_T3 = 4, K_TB = 5;
__host__ __device__ constexpr bool kind_three(int k) { return k >= K_T3; }
__host__ __device__ constexpr int kind_mode(int k) { return k == K_T3 ? CM_THREE : (k == K_TB ? CM_TB : CM_FOUR); }
__device__ __forceinline__ int kind_for(int M, int em) { return M == CM_THREE ? K_T3 : (M == CM_TB ? K_TB : em); }

// ColorBlock::GetMetrics (ColorBlock.h:88-117), into s_met[g][which]
__device__ __noinline__ void get_metrics(int which, bool ignore_black) {
    const Grp G = grp();
    const uint32_t v = s_px[G.g][G.lane];
    const int p[3] = {(int)(v & 0xFF), (int)((v >> 8) & 0xFF), (int)((v >> 16) & 0xFF)};
    const bool blk = (p[0] | p[1] | p[2]) < 4;
    const bool has_black = __any_sync(G.gm, blk);
    const bool inc = !(ignore_black && blk);
    const bool grey = __all_sync(G.gm, !inc || (p[0] == p[1] && p[0] == p[2]));
    const int total = __popc(__ballot_sync(G.gm, inc) & G.gm);
    int *M = s_met[G.g][which];
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const int mn = (int)gmin(G.gm, inc ? p[c] : 255), mx = (int)gmax(G.gm, inc ? p[c] : 0);
        const int sm = (int)gsum(G.gm, inc ? p[c] : 0);
        if (G.lane == 0) {
            M[MT_MN + c] = mn;
            M[MT_MX + c] = mx;
            M[MT_SUM + c] = sm;
            M[MT_AV + c] = total > 0 ? (sm + total / 2) / total : 0;
        }
    }
    if (G.lane == 0) {
        M[MT_GREY] = grey;
        M[MT_BLACK] = has_black;
    }
    __syncwarp(G.gm);
}

// ---------------------------------------------------------------------------
// FindSelectors<M>(error_mode), texel-parallel (BC1Encoder.cpp:679-779)
// ---------------------------------------------------------------------------
template <int IT, int K> __device__ __noinline__ SelErr fs_tp(int lo, int hi) {
    const Grp G = grp();
    const uint32_t v = s_px[G.g][G.lane];
    const int pr = v & 0xFF, pg = (v >> 8) & 0xFF, pb = (v >> 16) & 0xFF;
    const Pal P = make_pal<IT>(lo, hi, kind_three(K));
    int s;
    unsigned e;
    if (K == K_F4_NONE || K == K_F4_FASTER) {
        const int ar = P.r3 - P.r0, ag = P.g3 - P.g0, ab = P.b3 - P.b0;
        const int d0 = ar * P.r0 + ag * P.g0 + ab * P.b0, d1 = ar * P.r1 + ag * P.g1 + ab * P.b1;
        const int d2 = ar * P.r2 + ag * P.g2 + ab * P.b2, d3 = ar * P.r3 + ag * P.g3 + ab * P.b3;
        const int t0 = d0 + d1, t1 = d1 + d2, t2 = d2 + d3;
        const int dot = 2 * ar * pr + 2 * ag * pg + 2 * ab * pb;
        s = 3 - ((dot <= t0) + (dot < t1) + (dot < t2));
        e = K == K_F4_FASTER ? sq3(pr - sel4(P.r0, P.r1, P.r2, P.r3, s), pg - sel4(P.g0, P.g1, P.g2, P.g3, s),
                                   pb - sel4(P.b0, P.b1, P.b2, P.b3, s))
                             : 0u;
    } else if (K == K_F4_CHECK2) {
        const int ar = P.r3 - P.r0, ag = P.g3 - P.g0, ab = P.b3 - P.b0;
        const float f = __fdiv_rn(4.0f, __fadd_rn(__uint2float_rn(sq3(ar, ag, ab)), .00000125f));
        const int dd = (pr - P.r0) * ar + (pg - P.g0) * ag + (pb - P.b0) * ab;
        const float sf = __fadd_rn(__fmul_rn(__int2float_rn(dd), f), 0.5f);
        const int sl = clampi(f2i_x86(sf), 1, 3);
        const unsigned e0 = sq3(sel4(P.r0, P.r1, P.r2, P.r3, sl - 1) - pr, sel4(P.g0, P.g1, P.g2, P.g3, sl - 1) - pg,
                                sel4(P.b0, P.b1, P.b2, P.b3, sl - 1) - pb);
        const unsigned e1 = sq3(sel4(P.r0, P.r1, P.r2, P.r3, sl) - pr, sel4(P.g0, P.g1, P.g2, P.g3, sl) - pg,
                                sel4(P.b0, P.b1, P.b2, P.b3, sl) - pb);
        s = sl;
        e = e1;
        if (e0 == e1) {
            if (s == 1) s = 0;  // prefer the endpoint (:736-738)
        } else if (e0 < e) {
            s = sl - 1;
            e = e0;
        }
    } else {
        const unsigned e0 = sq3(P.r0 - pr, P.g0 - pg, P.b0 - pb), e1 = sq3(P.r1 - pr, P.g1 - pg, P.b1 - pb);
        const unsigned e2 = sq3(P.r2 - pr, P.g2 - pg, P.b2 - pb);
        s = 0;
        e = e0;
        if (e1 < e) { e = e1; s = 1; }
        if (e2 < e) { e = e2; s = 2; }
        if (K != K_T3) {
            const unsigned e3 = sq3(P.r3 - pr, P.g3 - pg, P.b3 - pb);
            if (e3 <= e) { e = e3; s = 3; }  // ties prefer selector 3 (:762)
        }
    }
    SelErr o;
    o.err = gsum(G.gm, e);
    o.sel = gor(G.gm, (unsigned)s << (2 * G.lane));
    return o;
}

template <int IT> __device__ __forceinline__ SelErr fs_any(int K, int lo, int hi) {
    switch (K) {
        case K_F4_NONE: return fs_tp<IT, K_F4_NONE>(lo, hi);
        case K_F4_FASTER: return fs_tp<IT, K_F4_FASTER>(lo, hi);
        case K_F4_CHECK2: return fs_tp<IT, K_F4_CHECK2>(lo, hi);
        case K_F4_FULL: return fs_tp<IT, K_F4_FULL>(lo, hi);
        case K_T3: return fs_tp<IT, K_T3>(lo, hi);
        default: return fs_tp<IT, K_TB>(lo, hi);
    }
}

// ---------------------------------------------------------------------------
// lane-serial block error: one lane evaluates all 16 texels for its own
// endpoints (error only; the winner's selectors come from fs_tp)
// ---------------------------------------------------------------------------
template <int IT, int K> __device__ __forceinline__ float block_err(const float4 *pf, int lo, int hi) {
    const Pal P = make_pal<IT>(lo, hi, kind_three(K));
    float tot = 0.0f;
    if (K == K_F4_FULL || K == K_T3 || K == K_TB) {
        // sum_t min_j |p_t - c_j|^2 = sum_t |p_t|^2 + sum_t min_j (|c_j|^2 - 2 p_t.c_j), in exact integers:
        // p.c by one dp4a on the packed texel (the colour's alpha byte is 0), the first sum is per block
        const uint32_t *px = s_px[grp().g];
        const uint32_t c0 = P.r0 | (P.g0 << 8) | (P.b0 << 16), c1 = P.r1 | (P.g1 << 8) | (P.b1 << 16);
        const uint32_t c2 = P.r2 | (P.g2 << 8) | (P.b2 << 16), c3 = P.r3 | (P.g3 << 8) | (P.b3 << 16);
        const int v0 = (int)sq3(P.r0, P.g0, P.b0), v1 = (int)sq3(P.r1, P.g1, P.b1);
        const int v2 = (int)sq3(P.r2, P.g2, P.b2), v3 = (int)sq3(P.r3, P.g3, P.b3);
        int t0 = 0, t1 = 0;
#pragma unroll 2
        for (int i = 0; i < 16; i += 2) {
            const uint32_t u = px[i], q = px[i + 1];
            int m = v0 - 2 * (int)__dp4a(u, c0, 0u), n = v0 - 2 * (int)__dp4a(q, c0, 0u);
            m = min(m, v1 - 2 * (int)__dp4a(u, c1, 0u));
            n = min(n, v1 - 2 * (int)__dp4a(q, c1, 0u));
            m = min(m, v2 - 2 * (int)__dp4a(u, c2, 0u));
            n = min(n, v2 - 2 * (int)__dp4a(q, c2, 0u));
            if (K != K_T3) {
                m = min(m, v3 - 2 * (int)__dp4a(u, c3, 0u));
                n = min(n, v3 - 2 * (int)__dp4a(q, c3, 0u));
            }
            t0 += m;
            t1 += n;
        }
        tot = (float)(s_pp[grp().g] + t0 + t1);
    } else if (K == K_F4_FASTER) {
        const int ar = P.r3 - P.r0, ag = P.g3 - P.g0, ab = P.b3 - P.b0;
        const int d0 = ar * P.r0 + ag * P.g0 + ab * P.b0, d1 = ar * P.r1 + ag * P.g1 + ab * P.b1;
        const int d2 = ar * P.r2 + ag * P.g2 + ab * P.b2, d3 = ar * P.r3 + ag * P.g3 + ab * P.b3;
        const float t0 = (float)(d0 + d1), t1 = (float)(d1 + d2), t2 = (float)(d2 + d3);
        const float a2r = 2.0f * ar, a2g = 2.0f * ag, a2b = 2.0f * ab;
#pragma unroll 4
        for (int i = 0; i < 16; i++) {
            const float4 p = pf[i];
            const float dot = fmaf(p.z, a2b, fmaf(p.y, a2g, p.x * a2r));
            const int s = 3 - ((int)(dot <= t0) + (int)(dot < t1) + (int)(dot < t2));  // selector = 3 - level
            const float dr = p.x - (float)sel4(P.r0, P.r1, P.r2, P.r3, s);
            const float dg = p.y - (float)sel4(P.g0, P.g1, P.g2, P.g3, s);
            const float db = p.z - (float)sel4(P.b0, P.b1, P.b2, P.b3, s);
            tot += fmaf(db, db, fmaf(dg, dg, dr * dr));
        }
    } else if (K == K_F4_CHECK2) {
        const int ar = P.r3 - P.r0, ag = P.g3 - P.g0, ab = P.b3 - P.b0;
        const float f = __fdiv_rn(4.0f, __fadd_rn(__uint2float_rn(sq3(ar, ag, ab)), .00000125f));
        const float far_ = (float)ar, fag = (float)ag, fab = (float)ab;
        const float c0r = (float)P.r0, c0g = (float)P.g0, c0b = (float)P.b0;
#pragma unroll 4
        for (int i = 0; i < 16; i++) {
            const float4 p = pf[i];
            const float dd = fmaf(p.z - c0b, fab, fmaf(p.y - c0g, fag, (p.x - c0r) * far_));
            const float sf = __fadd_rn(__fmul_rn(dd, f), 0.5f);
            const int sl = clampi(f2i_x86(sf), 1, 3);
            const float ar0 = (float)sel4(P.r0, P.r1, P.r2, P.r3, sl - 1) - p.x;
            const float ag0 = (float)sel4(P.g0, P.g1, P.g2, P.g3, sl - 1) - p.y;
            const float ab0 = (float)sel4(P.b0, P.b1, P.b2, P.b3, sl - 1) - p.z;
            const float ar1 = (float)sel4(P.r0, P.r1, P.r2, P.r3, sl) - p.x;
            const float ag1 = (float)sel4(P.g0, P.g1, P.g2, P.g3, sl) - p.y;
            const float ab1 = (float)sel4(P.b0, P.b1, P.b2, P.b3, sl) - p.z;
            tot += fminf(fmaf(ab0, ab0, fmaf(ag0, ag0, ar0 * ar0)), fmaf(ab1, ab1, fmaf(ag1, ag1, ar1 * ar1)));
        }
    }
    return tot;
}

// ---------------------------------------------------------------------------
// FindEndpointsSingleColor(result, pixels, color, is_3color), texel-parallel
// (BC1Encoder.cpp:443-471): the error is taken against colors[2] of the
// endpoints held BEFORE the table lookup, over RGBA (palette alpha 255).
// ---------------------------------------------------------------------------
struct SC {
    int lo, hi;
    uint32_t err;
};

template <int IT> __device__ __noinline__ SC single_color_px(int stale_lo, int stale_hi, bool is3, int which) {
    const Grp G = grp();
    const uint32_t v = s_px[G.g][G.lane];
    const Pal P = make_pal<IT>(stale_lo, stale_hi, is3);  // colors[2] is internal index 1 in both orders
    const int dr = (int)(v & 0xFF) - P.r1, dg = (int)((v >> 8) & 0xFF) - P.g1, db = (int)((v >> 16) & 0xFF) - P.b1;
    const int da = (int)(v >> 24) - 255;
    SC o;
    o.err = gsum(G.gm, (unsigned)(dr * dr + dg * dg + db * db + da * da));
    const int *M = s_met[G.g][which];
    const uint32_t mr = g_tab.match5[IT][M[MT_AV]], mg = g_tab.match6[IT][M[MT_AV + 1]], mb = g_tab.match5[IT][M[MT_AV + 2]];
    o.lo = eppack((mr >> 8) & 0xFF, (mg >> 8) & 0xFF, (mb >> 8) & 0xFF);
    o.hi = eppack(mr & 0xFF, mg & 0xFF, mb & 0xFF);
    return o;
}

// ---------------------------------------------------------------------------
// FindEndpoints (BC1Encoder.cpp:473-677), texel-parallel
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fdot4_rn(float a0, float a1, float a2, float a3, float b0, float b1, float b2, float b3) {
    // Vector4::Dot (Vector4.h:53-57): sum from 0, left to right
    float s = __fadd_rn(0.0f, __fmul_rn(a0, b0));
    s = __fadd_rn(s, __fmul_rn(a1, b1));
    s = __fadd_rn(s, __fmul_rn(a2, b2));
    return __fadd_rn(s, __fmul_rn(a3, b3));
}

__device__ __noinline__ int2 find_endpoints(int mode, bool ignore_black, int power_iters, int which) {
    const Grp G = grp();
    const uint32_t v = s_px[G.g][G.lane];
    const int pr = v & 0xFF, pg = (v >> 8) & 0xFF, pb = (v >> 16) & 0xFF;
    const int *M = s_met[G.g][which];
    const int mn[3] = {M[MT_MN], M[MT_MN + 1], M[MT_MN + 2]}, mx[3] = {M[MT_MX], M[MT_MX + 1], M[MT_MX + 2]};
    const int av[3] = {M[MT_AV], M[MT_AV + 1], M[MT_AV + 2]};
    int lo, hi;
    if (M[MT_GREY]) {  // :474-494
        const int fr = (int)(s_px[G.g][0] & 0xFF);
        if (mx[0] - mn[0] < 2) {
            lo = hi = eppack(s8to5(fr), s8to6(fr), s8to5(fr));
        } else {
            lo = eppack(s8to5(mn[0]), s8to6(mn[0]), s8to5(mn[0]));
            hi = eppack(s8to5(mx[0]), s8to6(mx[0]), s8to5(mx[0]));
        }
    } else if (mode == EP_LS) {  // :495-552
        const int d0 = mx[0] - mn[0], d1 = mx[1] - mn[1], d2 = mx[2] - mn[2];
        const int c0 = (d0 >= d1 && d0 >= d2) ? 0 : ((d1 >= d2 && d1 >= d0) ? 1 : 2);  // Color::MaxChannelRGB
        const int p[3] = {pr, pg, pb};
        const int px0 = c0 == 0 ? pr : (c0 == 1 ? pg : pb);
        unsigned sxy[3];
#pragma unroll
        for (int c = 0; c < 3; c++) sxy[c] = gsum(G.gm, (unsigned)(px0 * p[c]));  // zero-initialised (:510 is not)
        float l[3] = {0.f, 0.f, 0.f}, h[3] = {0.f, 0.f, 0.f};
        const float mn0 = (float)(c0 == 0 ? mn[0] : (c0 == 1 ? mn[1] : mn[2]));
        const unsigned sum_x = (unsigned)M[MT_SUM + c0], sum_xx = c0 == 0 ? sxy[0] : (c0 == 1 ? sxy[1] : sxy[2]);
#pragma unroll
        for (int c = 0; c < 3; c++)
            if (c == c0) l[c] = h[c] = mn0;
        const float den = __fsub_rn(__uint2float_rn(16u * sum_xx), __uint2float_rn(sum_x * sum_x));
        if (fabsf(den) > 1e-8f) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
                if (c == c0) continue;
                const unsigned sum_y = (unsigned)M[MT_SUM + c], sum_xy = sxy[c];
                const float a = __fdiv_rn(__uint2float_rn((16u * sum_xy) - (sum_x * sum_y)), den);
                const float b = __fdiv_rn(__uint2float_rn((sum_xx * sum_y) - (sum_xy * sum_x)), den);
                l[c] = __fadd_rn(b, __fmul_rn(a, mn0));
                h[c] = __fadd_rn(b, __fmul_rn(a, mn0));
            }
        }
#pragma unroll
        for (int c = 0; c < 3; c++) {
            const float inset = __fdiv_rn(__fsub_rn(h[c], l[c]), 16.0f);
            l[c] = __fdiv_rn(__fadd_rn(l[c], inset), 255.0f);
            h[c] = __fdiv_rn(__fsub_rn(h[c], inset), 255.0f);
        }
        lo = precise_round565(l[0], l[1], l[2], s_mid5, s_mid6);
        hi = precise_round565(h[0], h[1], h[2], s_mid5, s_mid6);
    } else if (mode == EP_BB || mode == EP_BBINT) {  // :553-605
        const int b = pb - av[2];
        const int cxz = (int)gsum(G.gm, (unsigned)(b * pr - av[0]));  // b * r - avg.r, as written (:572)
        const int cyz = (int)gsum(G.gm, (unsigned)(b * pg - av[1]));
        if (mode == EP_BB) {
            const float bias = __fdiv_rn(8.0f, 255.0f);
            float l[3], h[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                l[c] = __fdiv_rn((float)mn[c], 255.0f);
                h[c] = __fdiv_rn((float)mx[c], 255.0f);
                const float inset = __fdiv_rn(__fsub_rn(__fsub_rn(h[c], l[c]), bias), 16.0f);
                l[c] = __fadd_rn(l[c], inset);
                h[c] = __fsub_rn(h[c], inset);
            }
            if (cxz < 0) { const float t = l[0]; l[0] = h[0]; h[0] = t; }
            if (cyz < 0) { const float t = l[1]; l[1] = h[1]; h[1] = t; }
            lo = precise_round565(l[0], l[1], l[2], s_mid5, s_mid6);
            hi = precise_round565(h[0], h[1], h[2], s_mid5, s_mid6);
        } else {
            int a[3], z[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const int inset = ((mx[c] - mn[c]) - 8) >> 4;
                a[c] = clamp255(mn[c] + inset);
                z[c] = clamp255(mx[c] - inset);
            }
            if (cxz < 0) { const int t = a[0]; a[0] = z[0]; z[0] = t; }
            if (cyz < 0) { const int t = a[1]; a[1] = z[1]; z[1] = t; }
            lo = eppack(s8to5(a[0]), s8to6(a[1]), s8to5(a[2]));
            hi = eppack(s8to5(z[0]), s8to6(z[1]), s8to5(z[2]));
        }
    } else {  // PCA, :606-674
        const bool blk = (pr | pg | pb) < 4;
        const bool inc = !(ignore_black && blk);
        const int dr = pr - av[0], dg = pg - av[1], db = pb - av[2];
        // covariance from identity, accumulated over included texels: exact integers
        const int s00 = (int)gsum(G.gm, inc ? (unsigned)(dr * dr) : 0u);
        const int s01 = (int)gsum(G.gm, inc ? (unsigned)(dr * dg) : 0u);
        const int s02 = (int)gsum(G.gm, inc ? (unsigned)(dr * db) : 0u);
        const int s11 = (int)gsum(G.gm, inc ? (unsigned)(dg * dg) : 0u);
        const int s12 = (int)gsum(G.gm, inc ? (unsigned)(dg * db) : 0u);
        const int s22 = (int)gsum(G.gm, inc ? (unsigned)(db * db) : 0u);
        const float k255 = 255.0f;
        const float c00 = __fdiv_rn((float)(1 + s00), k255), c01 = __fdiv_rn((float)s01, k255);
        const float c02 = __fdiv_rn((float)s02, k255), c11 = __fdiv_rn((float)(1 + s11), k255);
        const float c12 = __fdiv_rn((float)s12, k255), c22 = __fdiv_rn((float)(1 + s22), k255);
        const float c33 = __fdiv_rn(1.0f, k255), z = __fdiv_rn(0.0f, k255);
        float d0 = __fsub_rn((float)mx[0], (float)mn[0]);
        float d1 = __fsub_rn((float)mx[1], (float)mn[1]);
        float d2 = __fsub_rn((float)mx[2], (float)mn[2]);
        float d3 = __fsub_rn(0.0f, 0.0f);
        if (c02 < 0) d0 = -d0;
        if (c12 < 0) d1 = -d1;
        for (int it = 0; it < power_iters; it++) {  // Matrix4x4 * Vector4 (Matrix4x4.cpp:33-39), mirrored rows
            const float n0 = fdot4_rn(d0, d1, d2, d3, c00, c01, c02, z);
            const float n1 = fdot4_rn(d0, d1, d2, d3, c01, c11, c12, z);
            const float n2 = fdot4_rn(d0, d1, d2, d3, c02, c12, c22, z);
            const float n3 = fdot4_rn(d0, d1, d2, d3, z, z, z, c33);
            d0 = n0; d1 = n1; d2 = n2; d3 = n3;
        }
        float k = 0.0f;  // Vector4::MaxAbs(3)
        if (fabsf(d0) > k) k = fabsf(d0);
        if (fabsf(d1) > k) k = fabsf(d1);
        if (fabsf(d2) > k) k = fabsf(d2);
        float a0 = 306.0f, a1 = 601.0f, a2 = 117.0f, a3 = 0.0f;
        if (k >= 2) {
            const float s = __fdiv_rn(2048.0f, k);
            a0 = __fmul_rn(d0, s); a1 = __fmul_rn(d1, s); a2 = __fmul_rn(d2, s); a3 = __fmul_rn(d3, s);
        }
        a0 = __fmul_rn(a0, 16.0f); a1 = __fmul_rn(a1, 16.0f); a2 = __fmul_rn(a2, 16.0f); a3 = __fmul_rn(a3, 16.0f);
        const float dot = fdot4_rn((float)pr, (float)pg, (float)pb, 0.0f, a0, a1, a2, a3);
        // first index of the maximum / minimum (strict > / < scan, :654-670)
        float vmax = inc ? dot : -INFINITY, vmin = inc ? dot : INFINITY;
        int imax = G.lane, imin = G.lane;
#pragma unroll
        for (int off = 8; off >= 1; off >>= 1) {
            const float ov = __shfl_xor_sync(G.gm, vmax, off, 16);
            const int oi = __shfl_xor_sync(G.gm, imax, off, 16);
            if (ov > vmax || (ov == vmax && oi < imax)) { vmax = ov; imax = oi; }
            const float ow = __shfl_xor_sync(G.gm, vmin, off, 16);
            const int oj = __shfl_xor_sync(G.gm, imin, off, 16);
            if (ow < vmin || (ow == vmin && oj < imin)) { vmin = ow; imin = oj; }
        }
        const uint32_t pmin = s_px[G.g][imin], pmax = s_px[G.g][imax];
        lo = eppack(s8to5(pmin & 0xFF), s8to6((pmin >> 8) & 0xFF), s8to5((pmin >> 16) & 0xFF));
        hi = eppack(s8to5(pmax & 0xFF), s8to6((pmax >> 8) & 0xFF), s8to5((pmax >> 16) & 0xFF));
    }
    return make_int2(lo, hi);
}

// ---------------------------------------------------------------------------
// RefineBlockLS<M> (BC1Encoder.cpp:852-875) with
// RefineEndpointsLS<FourColor>(result, pixels, metrics) (:781-825). Only the
// FourColor instantiation of the latter is ever called (:860): no texel is
// skipped and the 4-colour weights apply to every colour mode.
// ---------------------------------------------------------------------------
template <int IT, int K> __device__ __noinline__ Res refine_ls(Res r, int passes, int which) {
    const Grp G = grp();
    const uint32_t v = s_px[G.g][G.lane];
    const int pr = v & 0xFF, pg = (v >> 8) & 0xFF, pb = (v >> 16) & 0xFF;
    const int *M = s_met[G.g][which];
    for (int pass = 0; pass < passes; pass++) {
        Res t = r;
        const int s = (t.sel >> (2 * G.lane)) & 3;
        const int n1 = __popc(__ballot_sync(G.gm, s == 1) & G.gm), n2 = __popc(__ballot_sync(G.gm, s == 2) & G.gm);
        const int n3 = __popc(__ballot_sync(G.gm, s == 3) & G.gm), n0 = 16 - n1 - n2 - n3;
        // sum of OrderTable<4>::Weights[sel] = {s^2, s(3-s), s(3-s), (3-s)^2}: exact small integers
        float m0 = (float)(n1 + 4 * n2 + 9 * n3), m1 = (float)(2 * n1 + 2 * n2), m2 = m1, m3 = (float)(9 * n0 + 4 * n1 + n2);
        const float q00r = (float)(int)gsum(G.gm, (unsigned)(pr * s));
        const float q00g = (float)(int)gsum(G.gm, (unsigned)(pg * s));
        const float q00b = (float)(int)gsum(G.gm, (unsigned)(pb * s));
        const float det = __fsub_rn(__fmul_rn(m0, m3), __fmul_rn(m1, m2));
        if (fabsf(det) < 1e-8f) {  // not multicolour: FindEndpointsSingleColor on the average
            const SC sc = single_color_px<IT>(t.lo, t.hi, K != K_F4_NONE && kind_three(K), which);
            t.lo = sc.lo;
            t.hi = sc.hi;
            t.err = sc.err;
            t.sel = 0x55555555u;
            t.mode = kind_three(K) ? CM_THREE : CM_FOUR;
        } else {
            const float tt = m0; m0 = m3; m3 = tt;
            m1 = -m1;
            m2 = -m2;
            const float sc = __fdiv_rn(__fdiv_rn(3.0f, 255.0f), det);
            m0 = __fmul_rn(m0, sc); m1 = __fmul_rn(m1, sc); m2 = __fmul_rn(m2, sc); m3 = __fmul_rn(m3, sc);
            const float q10r = (float)(M[MT_SUM] * 3) - q00r, q10g = (float)(M[MT_SUM + 1] * 3) - q00g;
            const float q10b = (float)(M[MT_SUM + 2] * 3) - q00b;
            t.lo = precise_round565(__fadd_rn(__fmul_rn(m0, q00r), __fmul_rn(m1, q10r)),
                                    __fadd_rn(__fmul_rn(m0, q00g), __fmul_rn(m1, q10g)),
                                    __fadd_rn(__fmul_rn(m0, q00b), __fmul_rn(m1, q10b)), s_mid5, s_mid6);
            t.hi = precise_round565(__fadd_rn(__fmul_rn(m2, q00r), __fmul_rn(m3, q10r)),
                                    __fadd_rn(__fmul_rn(m2, q00g), __fmul_rn(m3, q10g)),
                                    __fadd_rn(__fmul_rn(m2, q00b), __fmul_rn(m3, q10b)), s_mid5, s_mid6);
            const SelErr se = fs_tp<IT, K>(t.lo, t.hi);
            t.sel = se.sel;
            t.err = se.err;
            t.mode = kind_mode(K);
        }
        if (t.lo == r.lo && t.hi == r.hi) break;
        if (K == K_F4_NONE || t.err < r.err) r = t;
        else break;
    }
    return r;
}

template <int IT> __device__ __forceinline__ Res refine_ls_any(int K, Res r, int passes, int which) {
    switch (K) {
        case K_F4_NONE: return refine_ls<IT, K_F4_NONE>(r, passes, which);
        case K_F4_FASTER: return refine_ls<IT, K_F4_FASTER>(r, passes, which);
        case K_F4_CHECK2: return refine_ls<IT, K_F4_CHECK2>(r, passes, which);
        case K_F4_FULL: return refine_ls<IT, K_F4_FULL>(r, passes, which);
        case K_T3: return refine_ls<IT, K_T3>(r, passes, which);
        default: return refine_ls<IT, K_TB>(r, passes, which);
    }
}

__device__ __forceinline__ bool is_single_hash(bool four, int h) {
    return four ? (h == 15 || h == 700 || h == 753 || h == 515) : (h == 12 || h == 15 || h == 89);
}

// RefineEndpointsLS<M>(result, sums, matrix, hash) (BC1Encoder.cpp:827-850):
// q10 = sums at the ordering's cumulative selector counts (exact integers)
__device__ __forceinline__ int2 ls_from_sums(const int *S, float4 f, uint32_t o, bool four) {
    const int l1 = o & 0xFF, l2 = l1 + ((o >> 8) & 0xFF), l3 = l2 + ((o >> 16) & 0xFF);
    int qr = S[3 * l1] + S[3 * l2], qg = S[3 * l1 + 1] + S[3 * l2 + 1], qb = S[3 * l1 + 2] + S[3 * l2 + 2];
    if (four) {
        qr += S[3 * l3];
        qg += S[3 * l3 + 1];
        qb += S[3 * l3 + 2];
    }
    const float denom = four ? 3.0f : 2.0f;
    const float fr = (float)qr, fg = (float)qg, fb = (float)qb;
    const float q0r = (float)S[48] * denom - fr, q0g = (float)S[49] * denom - fg, q0b = (float)S[50] * denom - fb;
    const int lo = precise_round565(__fadd_rn(__fmul_rn(f.x, q0r), __fmul_rn(f.y, fr)),
                                    __fadd_rn(__fmul_rn(f.x, q0g), __fmul_rn(f.y, fg)),
                                    __fadd_rn(__fmul_rn(f.x, q0b), __fmul_rn(f.y, fb)), s_mid5, s_mid6);
    const int hi = precise_round565(__fadd_rn(__fmul_rn(f.z, q0r), __fmul_rn(f.w, fr)),
                                    __fadd_rn(__fmul_rn(f.z, q0g), __fmul_rn(f.w, fg)),
                                    __fadd_rn(__fmul_rn(f.z, q0b), __fmul_rn(f.w, fb)), s_mid5, s_mid6);
    return make_int2(lo, hi);
}

// ---------------------------------------------------------------------------
// RefineBlockCF<M> (BC1Encoder.cpp:877-928)
// ---------------------------------------------------------------------------
template <int IT, int K> __device__ __noinline__ Res refine_cf(Res r, unsigned orderings, bool exhaustive, int which) {
    constexpr bool four = !kind_three(K);
    constexpr int M = kind_mode(K);
    const Grp G = grp();
    const Res orig = r;
    // Histogram of the selectors -> start ordering (OrderTable::GetHash, OrderTable.h:91-104)
    const uint32_t w = orig.sel;
    const int n1 = __popc(w & ~(w >> 1) & 0x55555555u), n2 = __popc(~w & (w >> 1) & 0x55555555u);
    const int n3 = __popc(w & (w >> 1) & 0x55555555u), n0 = 16 - n1 - n2 - n3;
    int start;
    if (four) {  // SingleColorHashes (OrderTable.cpp:43-44), looked up by bin
        start = n0 == 16 ? 15 : n1 == 16 ? 700 : n2 == 16 ? 753 : n3 == 16 ? 515 : (int)g_tab.hash4[n0 | (n1 << 4) | (n2 << 8)];
    } else {
        start = n0 == 16 ? 12 : n1 == 16 ? 15 : n2 == 16 ? 89 : (int)g_tab.hash3[n0 | (n1 << 4)];
    }
    const unsigned total = exhaustive ? (four ? 969u : 153u) : orderings;
    uint16_t *row = s_row[G.g];
    if (!exhaustive) {  // stage the BestOrders row (8 or 2 entries per lane)
        const uint16_t *src = four ? g_tab.best4 + start * 128 : g_tab.best3 + start * 32;
        for (unsigned q = G.lane; q < total; q += 16) row[q] = src[q] & 0x7FFF;  // without the single-colour flag
    }
    // projection onto high - low, sort, prefix sums (:891-909); all values exact integers
    const uint32_t v = s_px[G.g][G.lane];
    const int pr = v & 0xFF, pg = (v >> 8) & 0xFF, pb = (v >> 16) & 0xFF;
    const int axr = s5to8(epr(orig.hi)) - s5to8(epr(orig.lo));
    const int axg = s6to8(epg(orig.hi)) - s6to8(epg(orig.lo));
    const int axb = s5to8(epb(orig.hi)) - s5to8(epb(orig.lo));
    const uint32_t key = ((uint32_t)(0x1000000 + pr * axr + pg * axg + pb * axb) << 4) | (uint32_t)G.lane;
    int rank = 0;  // keys are distinct (the texel index is in the low bits)
#pragma unroll
    for (int i = 0; i < 16; i++) rank += __shfl_sync(G.gm, key, i, 16) < key;
    int sr = 0, sg = 0, sb = 0;  // sum of the texels ranked at or below this lane's position
#pragma unroll 4
    for (int j = 0; j < 16; j++) {
        if (__shfl_sync(G.gm, rank, j, 16) <= G.lane) {
            const uint32_t u = s_px[G.g][j];
            sr += u & 0xFF;
            sg += (u >> 8) & 0xFF;
            sb += (u >> 16) & 0xFF;
        }
    }
    int *S = s_sum[G.g];
    S[3 * (G.lane + 1) + 0] = sr;
    S[3 * (G.lane + 1) + 1] = sg;
    S[3 * (G.lane + 1) + 2] = sb;
    if (G.lane == 0) S[0] = S[1] = S[2] = 0;
    __syncwarp(G.gm);

    // the single-colour trial is the same for every single-colour ordering of this call
    const SC sc = single_color_px<IT>(orig.lo, orig.hi, !four, which);

    if (total <= 4) {
        // few orderings: evaluate them in sequence, texel-parallel (the reference's loop as written)
        for (unsigned q = 0; q < total; q++) {
            const int th = exhaustive ? (int)q : (int)row[q];
            Res t;
            if (is_single_hash(four, th)) {
                t.lo = sc.lo;
                t.hi = sc.hi;
                t.err = sc.err;
                t.sel = 0x55555555u;
            } else {
                const int2 e = ls_from_sums(S, four ? g_tab.factors4[th] : g_tab.factors3[th],
                                            four ? g_tab.orders4[th] : g_tab.orders3[th], four);
                t.lo = e.x;
                t.hi = e.y;
                const SelErr se = fs_tp<IT, K>(t.lo, t.hi);
                t.sel = se.sel;
                t.err = se.err;
            }
            t.mode = M;
            if (t.err < r.err) r = t;
            if (t.err == 0) break;
        }
    } else {
        // ordering-parallel: lane l evaluates orderings l, l+16, ...; argmin over (error, index)
        const float4 *pf = s_pf[G.g];
        float best = INFINITY;
        int bq = 0x7FFF, blo = 0, bhi = 0;
        unsigned q = G.lane;
        int th = 0;
        float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
        uint32_t o = 0;
        if (q < total) {
            th = exhaustive ? (int)q : (int)row[q];
            f = four ? g_tab.factors4[th] : g_tab.factors3[th];
            o = four ? g_tab.orders4[th] : g_tab.orders3[th];
        }
        for (; q < total; q += 16) {
            // prefetch the next ordering's table entries while this one is evaluated
            const unsigned qn = q + 16;
            int thn = 0;
            float4 fn = f;
            uint32_t on = o;
            if (qn < total) {
                thn = exhaustive ? (int)qn : (int)row[qn];
                fn = four ? g_tab.factors4[thn] : g_tab.factors3[thn];
                on = four ? g_tab.orders4[thn] : g_tab.orders3[thn];
            }
            int lo, hi;
            float e;
            if (is_single_hash(four, th)) {
                lo = sc.lo;
                hi = sc.hi;
                e = (float)sc.err;
            } else {
                const int2 ep = ls_from_sums(S, f, o, four);
                lo = ep.x;
                hi = ep.y;
                e = block_err<IT, K>(pf, lo, hi);
            }
            if (e < best) {
                best = e;
                bq = (int)q;
                blo = lo;
                bhi = hi;
            }
            th = thn;
            f = fn;
            o = on;
        }
        const uint32_t be = best == INFINITY ? UINT_MAX : (uint32_t)best;
        const uint32_t min_e = gmin(G.gm, be);
        const uint32_t min_q = gmin(G.gm, be == min_e ? (uint32_t)bq : 0xFFFFu);
        if (min_e < orig.err) {
            const int wl = (int)(min_q & 15);
            r.lo = __shfl_sync(G.gm, blo, wl, 16);
            r.hi = __shfl_sync(G.gm, bhi, wl, 16);
            r.err = min_e;
            r.mode = M;
            const int wth = exhaustive ? (int)min_q : (int)row[min_q];
            r.sel = is_single_hash(four, wth) ? 0x55555555u : fs_tp<IT, K>(r.lo, r.hi).sel;
        }
    }
    __syncwarp(G.gm);  // s_sum and s_row are rewritten by the next call
    return r;
}

template <int IT> __device__ __forceinline__ Res refine_cf_any(int K, Res r, unsigned orderings, bool exhaustive, int which) {
    switch (K) {
        case K_F4_NONE: return refine_cf<IT, K_F4_NONE>(r, orderings, exhaustive, which);
        case K_F4_FASTER: return refine_cf<IT, K_F4_FASTER>(r, orderings, exhaustive, which);
        case K_F4_CHECK2: return refine_cf<IT, K_F4_CHECK2>(r, orderings, exhaustive, which);
        case K_F4_FULL: return refine_cf<IT, K_F4_FULL>(r, orderings, exhaustive, which);
        default: return refine_cf<IT, K_T3>(r, orderings, exhaustive, which);
    }
}

// ---------------------------------------------------------------------------
// EndpointSearch (BC1Encoder.cpp:930-996), round-parallel speculation
// ---------------------------------------------------------------------------
template <int IT, int K> __device__ __noinline__ Res endpoint_search(Res r, unsigned rounds) {
    const Grp G = grp();
    const float4 *pf = s_pf[G.g];
    const unsigned sh = (G.gm & 0xFFFFu) ? 0 : 16;
    unsigned prev = 0, i0 = 0;
    int forbidden = -1;
    bool moved = false;
    while (i0 < rounds) {
        const unsigned i = i0 + (unsigned)G.lane;
        const bool active = i < rounds && (int)(i & 31) != forbidden;
        const uint16_t vx = s_vox[i & 15];
        const int ddr = ((int)((unsigned)vx << 30)) >> 30, ddg = ((int)((unsigned)vx << 28)) >> 30;
        const int ddb = ((int)((unsigned)vx << 26)) >> 30;
        int lo = r.lo, hi = r.hi;
        if (i & 16) lo = eppack(clampi(epr(lo) + ddr, 0, 31), clampi(epg(lo) + ddg, 0, 63), clampi(epb(lo) + ddb, 0, 31));
        else hi = eppack(clampi(epr(hi) + ddr, 0, 31), clampi(epg(hi) + ddg, 0, 63), clampi(epb(hi) + ddb, 0, 31));
        float e = INFINITY;
        if (active) e = block_err<IT, K>(pf, lo, hi);
        const bool improve = active && e < (float)r.err;
        const bool stop = active && (i - prev > 32);
        const unsigned bi = (__ballot_sync(G.gm, improve) >> sh) & 0xFFFFu;
        const unsigned bs = (__ballot_sync(G.gm, stop) >> sh) & 0xFFFFu;
        const int fi = bi ? __ffs(bi) - 1 : 16, fs = bs ? __ffs(bs) - 1 : 16;
        if (bi && fi <= fs) {  // the first improving round is accepted
            const unsigned j = i0 + (unsigned)fi;
            r.lo = __shfl_sync(G.gm, lo, fi, 16);
            r.hi = __shfl_sync(G.gm, hi, fi, 16);
            r.err = (uint32_t)__shfl_sync(G.gm, e, fi, 16);
            forbidden = (int)((s_vox[j & 15] >> 8) & 15) | (int)(j & 16);
            prev = j;
            i0 = j + 1;
            moved = true;
        } else if (bs) {  // that round did not improve and i - prev > 32: stop
            break;
        } else {
            i0 += 16;
        }
    }
    if (moved) r.sel = fs_tp<IT, K>(r.lo, r.hi).sel;  // selectors of the accepted endpoints
    return r;
}

template <int IT> __device__ __forceinline__ Res endpoint_search_any(int K, Res r, unsigned rounds) {
    switch (K) {
        case K_F4_NONE: return endpoint_search<IT, K_F4_NONE>(r, rounds);
        case K_F4_FASTER: return endpoint_search<IT, K_F4_FASTER>(r, rounds);
        case K_F4_CHECK2: return endpoint_search<IT, K_F4_CHECK2>(r, rounds);
        case K_F4_FULL: return endpoint_search<IT, K_F4_FULL>(r, rounds);
        case K_T3: return endpoint_search<IT, K_T3>(r, rounds);
        default: return endpoint_search<IT, K_TB>(r, rounds);
    }
}

// ---------------------------------------------------------------------------
// block writers (BC1Encoder.cpp:345-441, BC1Block.h:66-80)
// ---------------------------------------------------------------------------
template <int IT> __device__ __forceinline__ uint2 write_block_solid(uint32_t c) {
    const int cr = c & 0xFF, cg = (c >> 8) & 0xFF, cb = (c >> 16) & 0xFF;
    uint32_t mask = 0xAA;
    int mn, mx;
    if ((cr | cg | cb) == 0) {
        mn = 0; mx = 1; mask = 0x55;
    } else {
        // FindEndpointsSingleColor(color); the 3-colour tables equal the 4-colour
        // ones (SingleColorTable.h: N unused), so the 3-colour trial never wins.
        const uint32_t mr = g_tab.match5[IT][cr], mg = g_tab.match6[IT][cg], mb = g_tab.match5[IT][cb];
        mn = eppack((mr >> 8) & 0xFF, (mg >> 8) & 0xFF, (mb >> 8) & 0xFF);
        mx = eppack(mr & 0xFF, mg & 0xFF, mb & 0xFF);
        if (mn == mx) {
            if (mn > 0) { mn--; mask = 0; }
            else { mx = 1; mn = 0; mask = 0x55; }
        } else if (mx < mn) {
            const int t = mn; mn = mx; mx = t;
            mask = 0xFF;
        }
    }
    return make_uint2((uint32_t)mx | ((uint32_t)mn << 16), mask * 0x01010101u);
}

__device__ __forceinline__ uint2 write_block(const Res &r) {
    int ep1 = r.lo, ep0 = r.hi;
    uint32_t lut;  // 4 x 2-bit entries
    if (r.mode & CM_FOUR) {
        lut = 1 | (3 << 2) | (2 << 4) | (0 << 6);
        if (ep1 > ep0) {
            const int t = ep1; ep1 = ep0; ep0 = t;
            lut = 0 | (2 << 2) | (3 << 4) | (1 << 6);
        } else if (ep1 == ep0) {
            if (ep1 > 0) { ep1--; lut = 0; }
            else { ep0 = 1; ep1 = 0; lut = 0x55; }
        }
    } else {
        lut = 1 | (2 << 2) | (0 << 4) | (3 << 6);
        if (ep1 < ep0) {
            const int t = ep1; ep1 = ep0; ep0 = t;
            lut = 0 | (2 << 2) | (1 << 4) | (3 << 6);
        }
    }
    uint32_t sel = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) sel |= ((lut >> (2 * ((r.sel >> (2 * i)) & 3))) & 3) << (2 * i);
    return make_uint2((uint32_t)ep0 | ((uint32_t)ep1 << 16), sel);
}

// ---------------------------------------------------------------------------
// BC1Encoder::EncodeBlock (BC1Encoder.cpp:261-342) for the group's block
// ---------------------------------------------------------------------------
template <int IT> __device__ __forceinline__ uint2 encode_bc1_group(const Grp &G, const qt_bc1_params &p, int color_mode) {
    if (__all_sync(G.gm, s_px[G.g][G.lane] == s_px[G.g][0])) return write_block_solid<IT>(s_px[G.g][0]);

    get_metrics(0, false);
    const bool has_black = s_met[G.g][0][MT_BLACK] != 0;
    const bool use_likely = p.exhaustive || p.orderings3 > 0 || p.orderings4 > 0;
    bool needs_err = use_likely;
    needs_err |= color_mode == CM_THREE;
    needs_err |= (color_mode == CM_TB) && has_black;
    needs_err |= p.error_mode != EM_NONE;
    needs_err |= p.search_rounds > 0;
    const int em = needs_err ? p.error_mode : EM_NONE;
    const int ls_passes = p.two_ls_passes ? 2 : 1, cf_passes = p.two_cf_passes ? 2 : 1;
    const int ep_passes = (needs_err && p.two_ep_passes) ? 2 : 1;
    const int k4 = kind_for(CM_FOUR, em);

    Res orig = res_init(), res = res_init();
    for (int round = 0; round < ep_passes; round++) {
        const int2 ep = find_endpoints(round == 1 ? EP_BB : p.endpoint_mode, false, (int)p.power_iterations, 0);
        Res to = res_init();
        to.lo = ep.x;
        to.hi = ep.y;
        Res tr = to;
        const SelErr se = fs_any<IT>(k4, tr.lo, tr.hi);
        tr.sel = se.sel;
        tr.err = se.err;
        tr.mode = CM_FOUR;
        tr = refine_ls_any<IT>(k4, tr, ls_passes, 0);
        if (!needs_err || tr.err < res.err) {
            res = tr;
            orig = to;
        }
    }
    if (res.err > 0 && use_likely)
        for (int it = 0; it < cf_passes; it++) res = refine_cf_any<IT>(kind_for(CM_FOUR, p.error_mode), res, p.orderings4, p.exhaustive, 0);

    if (res.err > 0 && (color_mode & CM_THREE)) {
        Res t = orig;
        const SelErr se = fs_tp<IT, K_T3>(t.lo, t.hi);
        t.sel = se.sel;
        t.err = se.err;
        t.mode = CM_THREE;
        t = refine_ls<IT, K_T3>(t, ls_passes, 0);
        if (t.err > 0 && use_likely)
            for (int it = 0; it < cf_passes; it++) t = refine_cf<IT, K_T3>(t, p.orderings3, p.exhaustive, 0);
        if (t.err < res.err) res = t;
    }

    if (res.err > 0 && color_mode == CM_TB && has_black) {
        const int *M0 = s_met[G.g][0];
        if (!((M0[MT_MX] | M0[MT_MX + 1] | M0[MT_MX + 2]) < 4)) {
            get_metrics(1, true);
            const int2 ep = find_endpoints(EP_PCA, true, (int)p.power_iterations, 1);
            Res t = res_init();
            t.lo = ep.x;
            t.hi = ep.y;
            const SelErr se = fs_tp<IT, K_TB>(t.lo, t.hi);
            t.sel = se.sel;
            t.err = se.err;
            t.mode = CM_TB;
            t = refine_ls<IT, K_TB>(t, ls_passes, 1);
            if (t.err < res.err) res = t;
        }
    }

    if (res.err > 0 && p.search_rounds > 0) {
        const int M = res.mode == CM_THREE ? CM_THREE : (res.mode == CM_TB ? CM_TB : CM_FOUR);
        res = endpoint_search_any<IT>(kind_for(M, M == CM_FOUR ? p.error_mode : EM_FULL), res, p.search_rounds);
    }
    return write_block(res);
}

// BC4Encoder::EncodeBlock (BC4Encoder.cpp:30-71) for the group's block; returns the 8 bytes
__device__ __forceinline__ uint2 encode_bc4_group(const Grp &G, int ch) {
    const int v = (int)((s_px[G.g][G.lane] >> (8 * ch)) & 0xFF);
    const int mn = (int)gmin(G.gm, (unsigned)v), mx = (int)gmax(G.gm, (unsigned)v);
    if (mn == mx) return make_uint2((uint32_t)mn | ((uint32_t)mn << 8), 0u);
    const int bias = 4 - mn * 14, delta = mx - mn, x = v * 14;
    int lvl = 0;
#pragma unroll
    for (int c = 0; c < 7; c++) lvl += x >= delta * (1 + 2 * c) - bias;
    const uint32_t s = (kBC4Levels >> (3 * lvl)) & 7u;
    const int bit = 3 * G.lane;
    const uint32_t lo = gor(G.gm, bit < 32 ? s << bit : 0u);
    const uint32_t hi = gor(G.gm, bit >= 32 ? s << (bit - 32) : (bit + 3 > 32 ? s >> (32 - bit) : 0u));
    // bytes: a0=max, a1=min, then 48 selector bits little endian
    return make_uint2((uint32_t)mx | ((uint32_t)mn << 8) | (lo << 16), (lo >> 16) | (hi << 16));
}

// ---------------------------------------------------------------------------
// BC1 / BC3 encode kernel: one block per 16-lane group, grid-stride
// ---------------------------------------------------------------------------
template <int IT>
__global__ void __launch_bounds__(128, 6) k_bc1_encode(const uint8_t *__restrict__ rgba, int w, int h, int bw, long b_begin,
                                                       long nblocks, qt_bc1_params p, uint8_t *__restrict__ out, int bc3) {
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
        if (i < 32) s_mid5[i] = c_mid5[i];
        s_mid6[i] = c_mid6[i];
        if (i < 16) s_vox[i] = c_voxels[i];
    }
    __syncthreads();
    const Grp G = grp();
    const int color_mode = bc3 ? CM_FOUR : p.color_mode;  // BC3Encoder.h:39-40

    for (long b = b_begin + (long)blockIdx.x * kGroupsPerCta + G.g; b < nblocks; b += (long)gridDim.x * kGroupsPerCta) {
        const int by = (int)(b / bw), bx = (int)(b - (long)by * bw);
        int sx = bx * 4 + (G.lane & 3), sy = by * 4 + (G.lane >> 2);
        if (sx >= w) sx %= w;  // RawTexture::GetBlock wraps at the edges (Texture.h:105-108)
        if (sy >= h) sy %= h;
        const uint32_t v = *reinterpret_cast<const uint32_t *>(rgba + ((size_t)sy * w + sx) * 4);
        const float fr = (float)(v & 0xFF), fg = (float)((v >> 8) & 0xFF), fb = (float)((v >> 16) & 0xFF);
        s_px[G.g][G.lane] = v;
        s_pf[G.g][G.lane] = make_float4(fr, fg, fb, fr * fr + fg * fg + fb * fb);
        const unsigned pp = gsum(G.gm, sq3((int)(v & 0xFF), (int)((v >> 8) & 0xFF), (int)((v >> 16) & 0xFF)));
        if (G.lane == 0) s_pp[G.g] = (int)pp;
        __syncwarp(G.gm);
        const uint2 blk = encode_bc1_group<IT>(G, p, color_mode);
        if (bc3) {
            const uint2 a = encode_bc4_group(G, 3);
            if (G.lane == 0) reinterpret_cast<uint4 *>(out)[b] = make_uint4(a.x, a.y, blk.x, blk.y);
        } else if (G.lane == 0) {
            reinterpret_cast<uint2 *>(out)[b] = blk;
        }
        __syncwarp(G.gm);
    }
}

// ---------------------------------------------------------------------------
// thread-per-block kernels: BC4/BC5 encode, all decoders
//
// These move 72-80 bytes of HBM traffic per block, so at full bandwidth an SM
// has ~400 thread-instructions per block to spend. The per-block work is kept
// well under that: byte selection with PRMT (__byte_perm), one multiply-high
// per texel for the BC4 level, 32-bit block indices where they fit, and one
// kernel instantiation per format so nothing branches on it per block.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_block_thread(const uint8_t *__restrict__ rgba, int w, int h, int bx, int by,
                                                  bool fast, uint32_t px[16]) {
    if (fast) {
#pragma unroll
        for (int y = 0; y < 4; y++) {
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(rgba + ((size_t)(by * 4 + y) * w + bx * 4) * 4));
            px[4 * y] = q.x; px[4 * y + 1] = q.y; px[4 * y + 2] = q.z; px[4 * y + 3] = q.w;
        }
    } else {
#pragma unroll
        for (int y = 0; y < 4; y++)
#pragma unroll
            for (int x = 0; x < 4; x++) {
                const int sx = (bx * 4 + x) % w, sy = (by * 4 + y) % h;
                px[4 * y + x] = __ldg(reinterpret_cast<const uint32_t *>(rgba + ((size_t)sy * w + sx) * 4));
            }
    }
}

// The Levels table of BC4Encoder.cpp:45 ({1,7,6,5,4,3,2,0}: threshold count -> selector) as bytes for PRMT.
constexpr uint32_t kBC4MapLo = 1u | (7u << 8) | (6u << 16) | (5u << 24);
constexpr uint32_t kBC4MapHi = 4u | (3u << 8) | (2u << 16) | (0u << 24);

// Exact division of n < 4096 by d = 2*delta (delta 1..255) as __umulhi(n, M[delta]):
// M = (floor(2^(12+l) / d) + 1) << (20 - l), l = ceil(log2 d) (Granlund & Montgomery,
// "Division by invariant integers using multiplication", 1994, Thm 4.2, N = 12 bits).
struct BC4Magic {
    uint32_t m[256];
};
constexpr BC4Magic make_bc4_magic() {
    BC4Magic t{};
    for (int delta = 1; delta < 256; delta++) {
        const uint32_t d = 2u * (uint32_t)delta;
        int l = 0;
        while ((1u << l) < d) l++;
        const uint64_t m = (1ull << (12 + l)) / d + 1;
        t.m[delta] = (uint32_t)(m << (20 - l));
    }
    return t;
}
__device__ const BC4Magic g_bc4_magic = make_bc4_magic();

// BC4Encoder::EncodeBlock (BC4Encoder.cpp:30-71) on channel ch. The reference
// counts the thresholds delta*(1+2c) - bias (c = 0..6) that 14*value reaches;
// for min <= value <= max that count is exactly
// min(7, floor((14*(value - min) + 4 + delta) / (2*delta))), taken here with one
// multiply-high per texel (equal for every (min, max, value), checked exhaustively).
__device__ __forceinline__ uint2 bc4_block_thread(const uint32_t px[16], int ch) {
    const uint32_t sel = 0x4440u | (uint32_t)ch;  // byte ch of the texel, zeros above
    uint32_t v[16];
    uint32_t mn = 255u, mx = 0u;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        v[i] = __byte_perm(px[i], 0u, sel);
        mn = min(mn, v[i]);
        mx = max(mx, v[i]);
    }
    if (mn == mx) return make_uint2(mn | (mn << 8), 0u);  // BC4Block(min): solid
    const uint32_t delta = mx - mn;
    const uint32_t M = __ldg(&g_bc4_magic.m[delta]);
    const uint32_t K = 4u + delta - 14u * mn;  // 14*value + K == 14*(value - min) + 4 + delta (mod 2^32)
    uint32_t lo = 0u, hi = 0u;                 // selector bits 0..31 and 32..47
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t lvl = min(__umulhi(14u * v[i] + K, M), 7u);
        const uint32_t s = __byte_perm(kBC4MapLo, kBC4MapHi, lvl) & 7u;
        if (i < 10) {
            lo |= s << (3 * i);
        } else if (i == 10) {
            lo |= s << 30;
            hi |= s >> 2;
        } else {
            hi |= s << (3 * i - 32);
        }
    }
    return make_uint2(mx | (mn << 8) | (lo << 16), (lo >> 16) | (hi << 16));
}

__device__ __forceinline__ uint32_t min_u16x2(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("min.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
__device__ __forceinline__ uint32_t max_u16x2(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("max.u16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

// BC5Encoder::EncodeBlock (BC5Encoder.cpp:25-30): BC4 of channel c0, then of c1,
// with the two channels carried side by side in 16-bit halves. One packed
// min/max per texel covers both channels, and one IMAD forms both numerators
// 14*value + K: a negative low-half K borrows one from the high half, which its
// high constant pre-compensates, so each half holds its channel's exact value.
// Per channel the rest is bc4_block_thread's arithmetic.
__device__ __forceinline__ uint4 bc5_block_thread(const uint32_t px[16], int c0, int c1) {
    const uint32_t sel = 0x4040u | (uint32_t)c0 | ((uint32_t)c1 << 8);  // byte c0 -> bits 0..7, byte c1 -> bits 16..23
    uint32_t v[16];
    uint32_t mn = 0x00FF00FFu, mx = 0u;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        v[i] = __byte_perm(px[i], 0u, sel);
        mn = min_u16x2(mn, v[i]);
        mx = max_u16x2(mx, v[i]);
    }
    const uint32_t mn0 = mn & 0xFFFFu, mn1 = mn >> 16, d0 = (mx & 0xFFFFu) - mn0, d1 = (mx >> 16) - mn1;
    const uint32_t M0 = __ldg(&g_bc4_magic.m[d0]), M1 = __ldg(&g_bc4_magic.m[d1]);  // m[0] = 0: solid, fixed below
    const int K0 = 4 + (int)d0 - 14 * (int)mn0, K1 = 4 + (int)d1 - 14 * (int)mn1;
    const uint32_t Kp = ((uint32_t)K0 & 0xFFFFu) + ((uint32_t)(K1 - (K0 < 0 ? 1 : 0)) << 16);
    uint32_t lo0 = 0u, hi0 = 0u, lo1 = 0u, hi1 = 0u;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t num = 14u * v[i] + Kp;
        const uint32_t l0 = min(__umulhi(num & 0xFFFFu, M0), 7u), l1 = min(__umulhi(num >> 16, M1), 7u);
        const uint32_t s0 = __byte_perm(kBC4MapLo, kBC4MapHi, l0) & 7u, s1 = __byte_perm(kBC4MapLo, kBC4MapHi, l1) & 7u;
        if (i < 10) {
            lo0 |= s0 << (3 * i);
            lo1 |= s1 << (3 * i);
        } else if (i == 10) {
            lo0 |= s0 << 30;
            hi0 |= s0 >> 2;
            lo1 |= s1 << 30;
            hi1 |= s1 >> 2;
        } else {
            hi0 |= s0 << (3 * i - 32);
            hi1 |= s1 << (3 * i - 32);
        }
    }
    const uint32_t mx0 = mn0 + d0, mx1 = mn1 + d1;
    uint4 r;
    r.x = d0 ? (mx0 | (mn0 << 8) | (lo0 << 16)) : (mn0 | (mn0 << 8));  // BC4Block(min) when solid
    r.y = d0 ? ((lo0 >> 16) | (hi0 << 16)) : 0u;
    r.z = d1 ? (mx1 | (mn1 << 8) | (lo1 << 16)) : (mn1 | (mn1 << 8));
    r.w = d1 ? ((lo1 >> 16) | (hi1 << 16)) : 0u;
    return r;
}

// One thread per block. Idx is uint32_t whenever the block count and the grid fit
// 31 bits (the common case: no 64-bit division per block), else uint64_t.
template <bool BC5, typename Idx>
__global__ void __launch_bounds__(256) k_bc4_encode(const uint8_t *__restrict__ rgba, int w, int h, Idx bw, Idx b_begin,
                                                    Idx nblocks, int c0, int c1, int aligned, uint8_t *__restrict__ out) {
    for (Idx b = b_begin + (Idx)blockIdx.x * blockDim.x + threadIdx.x; b < nblocks; b += (Idx)gridDim.x * blockDim.x) {
        const int by = (int)(b / bw), bx = (int)(b - (Idx)by * bw);
        const bool fast = aligned && (bx * 4 + 4 <= w) && (by * 4 + 4 <= h);
        uint32_t px[16];
        load_block_thread(rgba, w, h, bx, by, fast, px);
        if (BC5) reinterpret_cast<uint4 *>(out)[b] = bc5_block_thread(px, c0, c1);
        else reinterpret_cast<uint2 *>(out)[b] = bc4_block_thread(px, c0);
    }
}

// BC1 palette for decoding: Interpolator::Interpolate565BC1 (Interpolator.cpp:52-55)
template <int IT>
__device__ __forceinline__ void bc1_palette(uint32_t c0, uint32_t c1, bool allow3, bool write_alpha, uint32_t col[4]) {
    const int lo = (int)c0, hi = (int)c1;  // packed 5:6:5 == eppack layout
    const bool three = allow3 && (c1 >= c0);
    const Pal P = make_pal<IT>(lo, hi, three);
    // back to BC1 index order: colors[0]=c0, [1]=c1, [2], [3]
    uint32_t a3 = three ? 0u : 255u;
    if (!write_alpha) a3 = 255u;
    col[0] = (uint32_t)P.r0 | ((uint32_t)P.g0 << 8) | ((uint32_t)P.b0 << 16) | 0xFF000000u;
    col[2] = (uint32_t)P.r1 | ((uint32_t)P.g1 << 8) | ((uint32_t)P.b1 << 16) | 0xFF000000u;
    if (!three) {
        col[3] = (uint32_t)P.r2 | ((uint32_t)P.g2 << 8) | ((uint32_t)P.b2 << 16) | 0xFF000000u;
        col[1] = (uint32_t)P.r3 | ((uint32_t)P.g3 << 8) | ((uint32_t)P.b3 << 16) | 0xFF000000u;
    } else {
        col[1] = (uint32_t)P.r2 | ((uint32_t)P.g2 << 8) | ((uint32_t)P.b2 << 16) | 0xFF000000u;
        col[3] = (uint32_t)P.r3 | ((uint32_t)P.g3 << 8) | ((uint32_t)P.b3 << 16) | (a3 << 24);
    }
}

// BC4Block::GetValues (BC4Block.cpp:44-64), the 8 values as bytes: lo = values 0..3, hi = 4..7
__device__ __forceinline__ uint2 bc4_value_bytes(uint32_t a0, uint32_t a1) {
    uint32_t v2, v3, v4, v5, v6, v7;
    if (a0 <= a1) {  // GetValues6 (BC4Block.cpp:44-53)
        v2 = (a0 * 4 + a1) / 5; v3 = (a0 * 3 + a1 * 2) / 5; v4 = (a0 * 2 + a1 * 3) / 5; v5 = (a0 + a1 * 4) / 5;
        v6 = 0; v7 = 255;
    } else {  // GetValues8 (:55-64)
        v2 = (a0 * 6 + a1) / 7; v3 = (a0 * 5 + a1 * 2) / 7; v4 = (a0 * 4 + a1 * 3) / 7;
        v5 = (a0 * 3 + a1 * 4) / 7; v6 = (a0 * 2 + a1 * 5) / 7; v7 = (a0 + a1 * 6) / 7;
    }
    return make_uint2(a0 | (a1 << 8) | (v2 << 16) | (v3 << 24), v4 | (v5 << 8) | (v6 << 16) | (v7 << 24));
}

// Four 2-bit (BC1) or 3-bit (BC4) indices of one texel row, one per nibble: a PRMT selector.
__device__ __forceinline__ uint32_t nibbles2(uint32_t x) {
    x = (x & 0x0Fu) | ((x & 0xF0u) << 4);
    return (x & 0x0303u) | ((x & 0x0C0Cu) << 2);
}
__device__ __forceinline__ uint32_t nibbles3(uint32_t x) {
    return (x & 0x7u) | ((x & 0x38u) << 1) | ((x & 0x1C0u) << 2) | ((x & 0xE00u) << 3);
}

// The BC4 values of texel row y (4 texels), one byte each, from the 48 selector bits
__device__ __forceinline__ uint32_t bc4_row(uint2 vals, uint32_t sel_lo, uint32_t sel_hi, int y) {
    const uint32_t x = y == 0 ? sel_lo : y == 1 ? (sel_lo >> 12) : y == 2 ? __funnelshift_r(sel_lo, sel_hi, 24) : (sel_hi >> 4);
    return __byte_perm(vals.x, vals.y, nibbles3(x & 0xFFFu));
}

// Decode of one block into px[16] (RGBA8 words), for FMT 1 (BC1Decoder.cpp:33-55),
// 3 (BC3Decoder.cpp:26-31: BC1 colours without 3-colour mode, then BC4 into alpha),
// 4 (BC4Decoder.cpp:29-43 into channel c0 of (0,0,0,255)) and
// 5 (BC5Decoder.cpp:25-30: c0, then c1).
template <int FMT, int IT>
__device__ __forceinline__ void decode_texels(const uint8_t *__restrict__ blocks, size_t b, int write_alpha, int c0,
                                              int c1, uint32_t px[16]) {
    if (FMT == 1 || FMT == 3) {
        uint2 cb, ab = make_uint2(0u, 0u);
        if (FMT == 1) {
            cb = __ldg(reinterpret_cast<const uint2 *>(blocks) + b);
        } else {
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(blocks) + b);
            ab = make_uint2(q.x, q.y);
            cb = make_uint2(q.z, q.w);
        }
        uint32_t col[4];
        bc1_palette<IT>(cb.x & 0xFFFF, cb.x >> 16, FMT == 1, FMT == 1 && write_alpha, col);
        // channel planes: byte k of each = that channel of col[k]
        const uint32_t A = __byte_perm(col[0], col[1], 0x5140), B = __byte_perm(col[2], col[3], 0x5140);
        const uint32_t C = __byte_perm(col[0], col[1], 0x7362), D = __byte_perm(col[2], col[3], 0x7362);
        const uint32_t Rp = __byte_perm(A, B, 0x5410), Gp = __byte_perm(A, B, 0x7632);
        const uint32_t Bp = __byte_perm(C, D, 0x5410), Ap = __byte_perm(C, D, 0x7632);
        uint2 av = make_uint2(0u, 0u);
        uint32_t slo = 0u, shi = 0u;
        if (FMT == 3) {
            av = bc4_value_bytes(ab.x & 0xFF, (ab.x >> 8) & 0xFF);
            slo = (ab.x >> 16) | (ab.y << 16);
            shi = ab.y >> 16;
        }
#pragma unroll
        for (int y = 0; y < 4; y++) {
            const uint32_t S = nibbles2((cb.y >> (8 * y)) & 0xFFu);
            const uint32_t Rr = __byte_perm(Rp, 0u, S), Gr = __byte_perm(Gp, 0u, S), Br = __byte_perm(Bp, 0u, S);
            const uint32_t Ar = FMT == 3 ? bc4_row(av, slo, shi, y) : __byte_perm(Ap, 0u, S);
            const uint32_t X = __byte_perm(Rr, Gr, 0x5140), Y = __byte_perm(Br, Ar, 0x5140);
            const uint32_t X2 = __byte_perm(Rr, Gr, 0x7362), Y2 = __byte_perm(Br, Ar, 0x7362);
            px[4 * y + 0] = __byte_perm(X, Y, 0x5410);
            px[4 * y + 1] = __byte_perm(X, Y, 0x7632);
            px[4 * y + 2] = __byte_perm(X2, Y2, 0x5410);
            px[4 * y + 3] = __byte_perm(X2, Y2, 0x7632);
        }
    } else {
        uint2 q0, q1 = make_uint2(0u, 0u);
        if (FMT == 4) {
            q0 = __ldg(reinterpret_cast<const uint2 *>(blocks) + b);
        } else {
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(blocks) + b);
            q0 = make_uint2(q.x, q.y);
            q1 = make_uint2(q.z, q.w);
        }
        // texel k of a row: byte c0 <- value k, other bytes of (0,0,0,255); BC5 then byte c1 <- value k
        const uint32_t base0 = 0x7444u & ~(0xFu << (4 * c0));
        const uint32_t base1 = 0x3210u & ~(0xFu << (4 * c1));
        const uint2 v0 = bc4_value_bytes(q0.x & 0xFF, (q0.x >> 8) & 0xFF);
        const uint32_t lo0 = (q0.x >> 16) | (q0.y << 16), hi0 = q0.y >> 16;
        uint2 v1 = make_uint2(0u, 0u);
        uint32_t lo1 = 0u, hi1 = 0u;
        if (FMT == 5) {
            v1 = bc4_value_bytes(q1.x & 0xFF, (q1.x >> 8) & 0xFF);
            lo1 = (q1.x >> 16) | (q1.y << 16);
            hi1 = q1.y >> 16;
        }
#pragma unroll
        for (int y = 0; y < 4; y++) {
            const uint32_t W0 = bc4_row(v0, lo0, hi0, y);
            const uint32_t W1 = FMT == 5 ? bc4_row(v1, lo1, hi1, y) : 0u;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                uint32_t t = __byte_perm(W0, 0xFF000000u, base0 | ((uint32_t)k << (4 * c0)));
                if (FMT == 5) t = __byte_perm(t, W1, base1 | ((uint32_t)(4 + k) << (4 * c1)));
                px[4 * y + k] = t;
            }
        }
    }
}

// Store of a decoded block. Every texel of every block is decoded, and a texel
// is stored only if no later block (in the reference's by, bx, x, y write
// order) writes the same wrapped position: source (px, py) is final iff
// px + w >= 4*bw and py + h >= 4*bh (RawTexture::SetBlock, Texture.h:114-134).
__device__ __forceinline__ void store_block(const uint32_t px[16], int w, int h, int bw, int bh, int bx, int by,
                                            bool aligned, uint8_t *__restrict__ rgba) {
    const bool interior = aligned && bx > 0 && by > 0 && bx * 4 + 4 <= w && by * 4 + 4 <= h;
    if (interior) {
#pragma unroll
        for (int y = 0; y < 4; y++)
            *reinterpret_cast<uint4 *>(rgba + ((size_t)(by * 4 + y) * w + bx * 4) * 4) =
                make_uint4(px[4 * y], px[4 * y + 1], px[4 * y + 2], px[4 * y + 3]);
    } else {
#pragma unroll
        for (int y = 0; y < 4; y++)
#pragma unroll
            for (int x = 0; x < 4; x++) {
                const int sx = bx * 4 + x, sy = by * 4 + y;
                if (sx + w >= 4 * bw && sy + h >= 4 * bh)
                    *reinterpret_cast<uint32_t *>(rgba + ((size_t)(sy % h) * w + (sx % w)) * 4) = px[4 * y + x];
            }
    }
}

template <int FMT, int IT>
__device__ __forceinline__ void decode_block_fmt(const uint8_t *__restrict__ blocks, int w, int h, int bw, int bh,
                                                 size_t b, int bx, int by, int write_alpha, int c0, int c1,
                                                 bool aligned, uint8_t *__restrict__ rgba) {
    uint32_t px[16];
    decode_texels<FMT, IT>(blocks, b, write_alpha, c0, c1, px);
    store_block(px, w, h, bw, bh, bx, by, aligned, rgba);
}

// Runtime-format decode of block b (the batch kernel's entry).
template <int IT>
__device__ __forceinline__ void decode_block(const uint8_t *__restrict__ blocks, int w, int h, int bw, int bh, long b,
                                             int fmt, int write_alpha, int c0, int c1, int aligned,
                                             uint8_t *__restrict__ rgba) {
    const int by = (int)(b / bw), bx = (int)(b - (long)by * bw);
    switch (fmt) {
        case 1: decode_block_fmt<1, IT>(blocks, w, h, bw, bh, (size_t)b, bx, by, write_alpha, c0, c1, aligned, rgba); break;
        case 3: decode_block_fmt<3, IT>(blocks, w, h, bw, bh, (size_t)b, bx, by, write_alpha, c0, c1, aligned, rgba); break;
        case 4: decode_block_fmt<4, IT>(blocks, w, h, bw, bh, (size_t)b, bx, by, write_alpha, c0, c1, aligned, rgba); break;
        default: decode_block_fmt<5, IT>(blocks, w, h, bw, bh, (size_t)b, bx, by, write_alpha, c0, c1, aligned, rgba); break;
    }
}

// One thread per block; Idx as in k_bc4_encode.
template <int FMT, int IT, typename Idx>
__global__ void __launch_bounds__(256) k_decode(const uint8_t *__restrict__ blocks, int w, int h, Idx bw, int bh,
                                                Idx b_begin, Idx nblocks, int write_alpha, int c0, int c1, int aligned,
                                                uint8_t *__restrict__ rgba) {
    for (Idx b = b_begin + (Idx)blockIdx.x * blockDim.x + threadIdx.x; b < nblocks; b += (Idx)gridDim.x * blockDim.x) {
        const int by = (int)(b / bw), bx = (int)(b - (Idx)by * bw);
        decode_block_fmt<FMT, IT>(blocks, w, h, (int)bw, bh, (size_t)b, bx, by, write_alpha, c0, c1, aligned != 0, rgba);
    }
}

#include "qt_bc1_thread.cuh"

// ---------------------------------------------------------------------------
// persistent batch kernel: many textures, any format / op / level, one launch.
// A warp claims one tile (consecutive blocks of one texture) at a time; its
// lanes take the tile's blocks, one block per thread.
// ---------------------------------------------------------------------------
template <int IT> __device__ __noinline__ uint2 encode_bc1_batch(const qt_bc1_params *p, int color_mode, int pp) {
    return tpb::encode_block<IT>(*p, color_mode, pp);
}

__device__ __forceinline__ void batch_block(const BatchItemDev &__restrict__ I, long b) {
    const bool aligned = ((I.w & 3) == 0) && ((reinterpret_cast<uintptr_t>(I.op == QT_OP_ENCODE ? I.src : I.dst) & 15) == 0);
    if (I.op == QT_OP_DECODE) {
        switch (I.interp) {
            case IT_IDEAL: decode_block<IT_IDEAL>(I.src, I.w, I.h, I.bw, I.bh, b, I.fmt, I.write_alpha, I.c0, I.c1, aligned, I.dst); break;
            case IT_ROUND: decode_block<IT_ROUND>(I.src, I.w, I.h, I.bw, I.bh, b, I.fmt, I.write_alpha, I.c0, I.c1, aligned, I.dst); break;
            case IT_NVIDIA: decode_block<IT_NVIDIA>(I.src, I.w, I.h, I.bw, I.bh, b, I.fmt, I.write_alpha, I.c0, I.c1, aligned, I.dst); break;
            default: decode_block<IT_AMD>(I.src, I.w, I.h, I.bw, I.bh, b, I.fmt, I.write_alpha, I.c0, I.c1, aligned, I.dst); break;
        }
        return;
    }
    const int by = (int)(b / I.bw), bx = (int)(b - (long)by * I.bw);
    uint32_t v[16];
    load_block_thread(I.src, I.w, I.h, bx, by, aligned && (bx * 4 + 4 <= I.w) && (by * 4 + 4 <= I.h), v);
    if (I.fmt == 4 || I.fmt == 5) {
        if (I.fmt == 5) reinterpret_cast<uint4 *>(I.dst)[b] = bc5_block_thread(v, I.c0, I.c1);
        else reinterpret_cast<uint2 *>(I.dst)[b] = bc4_block_thread(v, I.c0);
        return;
    }
    int pp = 0;
#pragma unroll
    for (int i = 0; i < 16; i++) {
        tpb::t_px[i][threadIdx.x] = v[i];
        const uint32_t u = v[i] & 0x00FFFFFFu;
        pp += (int)__dp4a(u, u, 0u);
    }
    const int cm = I.fmt == 3 ? CM_FOUR : I.p.color_mode;  // BC3Encoder.h:39-40
    uint2 blk;
    switch (I.p.interpolator) {
        case IT_IDEAL: blk = encode_bc1_batch<IT_IDEAL>(&I.p, cm, pp); break;
        case IT_ROUND: blk = encode_bc1_batch<IT_ROUND>(&I.p, cm, pp); break;
        case IT_NVIDIA: blk = encode_bc1_batch<IT_NVIDIA>(&I.p, cm, pp); break;
        default: blk = encode_bc1_batch<IT_AMD>(&I.p, cm, pp); break;
    }
    if (I.fmt == 3) {
#pragma unroll
        for (int i = 0; i < 16; i++) v[i] = tpb::t_px[i][threadIdx.x];
        const uint2 a = bc4_block_thread(v, 3);
        reinterpret_cast<uint4 *>(I.dst)[b] = make_uint4(a.x, a.y, blk.x, blk.y);
    } else {
        reinterpret_cast<uint2 *>(I.dst)[b] = blk;
    }
}

// ctl[0] is the queue head (atomically advanced by each warp), ctl[1] the number of tiles.
__global__ void __launch_bounds__(tpb::kThreads, 4) k_batch(const BatchItemDev *__restrict__ items,
                                                            const TileDev *__restrict__ tiles, uint32_t *__restrict__ ctl) {
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
        if (i < 32) s_mid5[i] = c_mid5[i];
        s_mid6[i] = c_mid6[i];
        if (i < 16) s_vox[i] = c_voxels[i];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint32_t ntiles = ctl[1];
    while (true) {
        uint32_t t = 0;
        if (lane == 0) t = atomicAdd(&ctl[0], 1u);
        t = __shfl_sync(0xFFFFFFFFu, t, 0);
        if (t >= ntiles) break;
        const TileDev T = tiles[t];
        // the descriptor stays in (L1-cached) global memory: copying it to registers spills
        const BatchItemDev &I = items[T.item];
        for (uint32_t k = lane; k < T.count; k += 32) batch_block(I, (long)T.start + k);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// host-side launchers
// ---------------------------------------------------------------------------
static int num_sms() {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    return sms;
}

static int grid_for(long work, int per_cta) {
    const long need = (work + per_cta - 1) / per_cta;
    const long cap = (long)num_sms() * 64;
    return (int)(need < cap ? (need > 0 ? need : 1) : cap);
}

int upload_tables(int device) {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_tab, &host_tables(), sizeof(DevTables));
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaSetDevice(prev);
    return (int)e;
}

// BC1 mapping: 0 = one block per thread, 1 = one block per 16-lane group.
// QT_BC1_MAPPING=thread|group overrides the default for comparison runs.
static int bc1_mapping() {
    static int m = -1;
    if (m < 0) {
        const char *e = getenv("QT_BC1_MAPPING");
        m = (e && e[0] == 'g') ? 1 : 0;
    }
    return m;
}

// below this many blocks the split pass costs more than idle solid lanes do
constexpr long kSplitMinBlocks = 16384;

long defer_min_blocks() { return 2L * num_sms() * 4 * tpb::kThreads; }

// the four-colour cluster fit runs twice (EncodeBlock, BC1Encoder.cpp:299-302); exactly then
// encode_block, given a Deferred, stops blocks before the second pass
static bool cf2_pass(const qt_bc1_params &p) {
    return p.two_cf_passes && (p.exhaustive || p.orderings3 > 0 || p.orderings4 > 0);
}

int launch_bc1_encode_range(const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3,
                            long b_begin, long b_end, void *stream) {
    const int bw = (w + 3) / 4;
    const long n = b_end - b_begin;
    if (n <= 0) return 0;
    cudaStream_t s = (cudaStream_t)stream;
    if (bc1_mapping() == 0) {
        const int aligned = ((w & 3) == 0) && ((reinterpret_cast<uintptr_t>(rgba) & 15) == 0);
        const int g = grid_for(n, tpb::kThreads);
        if (n < kSplitMinBlocks || n > 0xFFFFFFFFL) {
            switch (p.interpolator) {
                case IT_IDEAL: k_bc1_thread<IT_IDEAL, false><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, b_begin, b_end, p, out, bc3, aligned, nullptr, nullptr); break;
                case IT_ROUND: k_bc1_thread<IT_ROUND, false><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, b_begin, b_end, p, out, bc3, aligned, nullptr, nullptr); break;
                case IT_NVIDIA: k_bc1_thread<IT_NVIDIA, false><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, b_begin, b_end, p, out, bc3, aligned, nullptr, nullptr); break;
                default: k_bc1_thread<IT_AMD, false><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, b_begin, b_end, p, out, bc3, aligned, nullptr, nullptr); break;
            }
            return (int)cudaGetLastError();
        }
        // solid blocks first, then the encoder over the rest (list + count, stream-ordered scratch);
        // with EndpointSearch, the encoder queues the searches and k_bc1_search runs them
        // deferred only when the queue holds at least two searches per resident lane of the
        // search kernel: below that no lane gets a second entry to refill from, and the extra
        // pass costs more than it saves (measured at L18: -5% at 1024^2, +10% at 2048^2)
        const bool defer = p.search_rounds > 0 && n >= defer_min_blocks();
        // and the second four-colour cluster-fit pass, when there is one, runs in its own pass
        // for the blocks where it can change the result
        const bool cf2 = defer && cf2_pass(p);
        const size_t words = 64 + (size_t)n + (defer ? 18 * (size_t)n : 0) + (cf2 ? 6 * (size_t)n : 0);
        uint32_t *scratch = nullptr;
        cudaError_t e = scratch_alloc((void **)&scratch, words * sizeof(uint32_t), s);
        if (e != cudaSuccess) return (int)e;
        uint32_t *count = scratch, *list = scratch + 64;
        e = cudaMemsetAsync(scratch, 0, 64 * sizeof(uint32_t), s);  // list count, queue counts and heads
        if (e == cudaSuccess && defer) {
            SearchQueues q;
            q.count = scratch + 1;
            q.head = scratch + 4;
            q.cap = n;
            uint32_t *qb = list + n;
            q.b = qb;
            q.lohi = qb + 3 * (size_t)n;
            q.err = qb + 6 * (size_t)n;
            q.sel = qb + 9 * (size_t)n;
            q.mode = qb + 12 * (size_t)n;
            FinishQueue fq;  // searches that moved the endpoints
            fq.count = scratch + 16;
            fq.b = qb + 15 * (size_t)n;
            fq.lohi = fq.b + (size_t)n;
            fq.mode = fq.b + 2 * (size_t)n;
            Cf2Queue c{};
            if (cf2) {
                uint32_t *cb = qb + 18 * (size_t)n;
                c.count = scratch + 8;
                c.b = cb;
                c.lohi = cb + (size_t)n;
                c.err = cb + 2 * (size_t)n;
                c.sel = cb + 3 * (size_t)n;
                c.mode = cb + 4 * (size_t)n;
                c.orig = cb + 5 * (size_t)n;
                c.cap = n;
            }
            const int gs = grid_for(n, 256);
            const int gsearch = num_sms() * 4;
            switch (p.interpolator) {
#define QT_DEFER(I)                                                                                                        \
    k_bc1_split<I><<<gs, 256, 0, s>>>(rgba, w, h, bw, b_begin, b_end, out, bc3, aligned, list, count);                      \
    k_bc1_defer<I><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, p, out, bc3, aligned, list, count, q, c);                    \
    if (cf2) k_bc1_cf2<I><<<gsearch, tpb::kThreads, 0, s>>>(rgba, w, h, bw, p, out, bc3, aligned, c, q);                    \
    k_bc1_search<I><<<gsearch, tpb::kThreads, 0, s>>>(rgba, w, h, bw, p, out, bc3, aligned, q, fq);                       \
    k_bc1_finish<I><<<gsearch, tpb::kThreads, 0, s>>>(rgba, w, h, bw, p, out, bc3, aligned, fq);
                case IT_IDEAL: QT_DEFER(IT_IDEAL) break;
                case IT_ROUND: QT_DEFER(IT_ROUND) break;
                case IT_NVIDIA: QT_DEFER(IT_NVIDIA) break;
                default: QT_DEFER(IT_AMD) break;
#undef QT_DEFER
            }
            e = cudaGetLastError();
        } else if (e == cudaSuccess) {
            const int gs = grid_for(n, 256);
            switch (p.interpolator) {
                case IT_IDEAL:
                    k_bc1_split<IT_IDEAL><<<gs, 256, 0, s>>>(rgba, w, h, bw, b_begin, b_end, out, bc3, aligned, list, count);
                    k_bc1_thread<IT_IDEAL, true><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, 0, 0, p, out, bc3, aligned, list, count);
                    break;
                case IT_ROUND:
                    k_bc1_split<IT_ROUND><<<gs, 256, 0, s>>>(rgba, w, h, bw, b_begin, b_end, out, bc3, aligned, list, count);
                    k_bc1_thread<IT_ROUND, true><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, 0, 0, p, out, bc3, aligned, list, count);
                    break;
                case IT_NVIDIA:
                    k_bc1_split<IT_NVIDIA><<<gs, 256, 0, s>>>(rgba, w, h, bw, b_begin, b_end, out, bc3, aligned, list, count);
                    k_bc1_thread<IT_NVIDIA, true><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, 0, 0, p, out, bc3, aligned, list, count);
                    break;
                default:
                    k_bc1_split<IT_AMD><<<gs, 256, 0, s>>>(rgba, w, h, bw, b_begin, b_end, out, bc3, aligned, list, count);
                    k_bc1_thread<IT_AMD, true><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, 0, 0, p, out, bc3, aligned, list, count);
                    break;
            }
            e = cudaGetLastError();
        }
        scratch_free(scratch, s);
        return (int)e;
    }
    const int grid = grid_for(n, kGroupsPerCta);
    switch (p.interpolator) {
        case IT_IDEAL: k_bc1_encode<IT_IDEAL><<<grid, 128, 0, s>>>(rgba, w, h, bw, b_begin, b_end, p, out, bc3); break;
        case IT_ROUND: k_bc1_encode<IT_ROUND><<<grid, 128, 0, s>>>(rgba, w, h, bw, b_begin, b_end, p, out, bc3); break;
        case IT_NVIDIA: k_bc1_encode<IT_NVIDIA><<<grid, 128, 0, s>>>(rgba, w, h, bw, b_begin, b_end, p, out, bc3); break;
        default: k_bc1_encode<IT_AMD><<<grid, 128, 0, s>>>(rgba, w, h, bw, b_begin, b_end, p, out, bc3); break;
    }
    return (int)cudaGetLastError();
}

int bc1_encode_kernels(long n, const qt_bc1_params &p) {
    if (n <= 0) return 0;
    if (bc1_mapping() != 0 || n < kSplitMinBlocks || n > 0xFFFFFFFFL) return 1;
    if (p.search_rounds == 0 || n < defer_min_blocks()) return 2;
    return cf2_pass(p) ? 5 : 4;  // split, encoder, (second cluster-fit pass,) search, finish
}

int launch_bc1_encode(const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3, void *stream) {
    return launch_bc1_encode_range(rgba, w, h, p, out, bc3, 0, (long)((w + 3) / 4) * ((h + 3) / 4), stream);
}

int batch_sms() { return num_sms(); }

int batch_ctas_per_sm() {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch, tpb::kThreads, 0) != cudaSuccess || n <= 0) n = 1;
    return n;
}

int launch_batch(const BatchItemDev *items, const TileDev *tiles, uint32_t *ctl, int grid, void *stream) {
    if (grid <= 0) grid = num_sms() * batch_ctas_per_sm();
    k_batch<<<grid, tpb::kThreads, 0, (cudaStream_t)stream>>>(items, tiles, ctl);
    return (int)cudaGetLastError();
}

// Grid of one thread per block when it fits (uint32_t indices), else a
// grid-stride loop over 64-bit indices.
static bool small_index(long n, int *grid) {
    const long ctas = (n + 255) / 256;
    if (n <= 0x7FFFFFFFL && ctas <= 0x7FFFFFFFL / 256) {
        *grid = (int)(ctas > 0 ? ctas : 1);
        return true;
    }
    *grid = num_sms() * 64;
    return false;
}

int launch_bc4_encode_range(const uint8_t *rgba, int w, int h, int c0, int c1, bool bc5, uint8_t *out, long b_begin,
                            long b_end, void *stream) {
    const int bw = (w + 3) / 4;
    if (b_end <= b_begin) return 0;
    const int aligned = ((w & 3) == 0) && ((reinterpret_cast<uintptr_t>(rgba) & 15) == 0);
    cudaStream_t s = (cudaStream_t)stream;
    int grid = 0;
    if (small_index(b_end, &grid)) {
        grid = (int)((b_end - b_begin + 255) / 256);
        const uint32_t ubw = (uint32_t)bw, u0 = (uint32_t)b_begin, un = (uint32_t)b_end;
        if (bc5) k_bc4_encode<true, uint32_t><<<grid, 256, 0, s>>>(rgba, w, h, ubw, u0, un, c0, c1, aligned, out);
        else k_bc4_encode<false, uint32_t><<<grid, 256, 0, s>>>(rgba, w, h, ubw, u0, un, c0, c1, aligned, out);
    } else {
        const uint64_t ubw = (uint64_t)bw, u0 = (uint64_t)b_begin, un = (uint64_t)b_end;
        if (bc5) k_bc4_encode<true, uint64_t><<<grid, 256, 0, s>>>(rgba, w, h, ubw, u0, un, c0, c1, aligned, out);
        else k_bc4_encode<false, uint64_t><<<grid, 256, 0, s>>>(rgba, w, h, ubw, u0, un, c0, c1, aligned, out);
    }
    return (int)cudaGetLastError();
}

int launch_bc4_encode(const uint8_t *rgba, int w, int h, int c0, int c1, bool bc5, uint8_t *out, void *stream) {
    return launch_bc4_encode_range(rgba, w, h, c0, c1, bc5, out, 0, (long)((w + 3) / 4) * ((h + 3) / 4), stream);
}

template <int FMT, int IT, typename Idx>
static void launch_decode_t(int grid, cudaStream_t s, const uint8_t *blocks, int w, int h, int bw, int bh, long b0,
                            long n, int write_alpha, int c0, int c1, int aligned, uint8_t *rgba) {
    k_decode<FMT, IT, Idx><<<grid, 256, 0, s>>>(blocks, w, h, (Idx)bw, bh, (Idx)b0, (Idx)n, write_alpha, c0, c1, aligned, rgba);
}

template <typename Idx>
static void launch_decode_idx(int fmt, int interp, int grid, cudaStream_t s, const uint8_t *blocks, int w, int h,
                              int bw, int bh, long b0, long n, int write_alpha, int c0, int c1, int aligned, uint8_t *rgba) {
#define QT_DEC(F, I) launch_decode_t<F, I, Idx>(grid, s, blocks, w, h, bw, bh, b0, n, write_alpha, c0, c1, aligned, rgba)
    if (fmt == 4) { QT_DEC(4, IT_IDEAL); return; }
    if (fmt == 5) { QT_DEC(5, IT_IDEAL); return; }
    if (fmt == 1) {
        switch (interp) {
            case IT_IDEAL: QT_DEC(1, IT_IDEAL); break;
            case IT_ROUND: QT_DEC(1, IT_ROUND); break;
            case IT_NVIDIA: QT_DEC(1, IT_NVIDIA); break;
            default: QT_DEC(1, IT_AMD); break;
        }
        return;
    }
    switch (interp) {
        case IT_IDEAL: QT_DEC(3, IT_IDEAL); break;
        case IT_ROUND: QT_DEC(3, IT_ROUND); break;
        case IT_NVIDIA: QT_DEC(3, IT_NVIDIA); break;
        default: QT_DEC(3, IT_AMD); break;
    }
#undef QT_DEC
}

int launch_decode_range(int fmt, const uint8_t *blocks, int w, int h, int interp, int write_alpha, int c0, int c1,
                        uint8_t *rgba, long b_begin, long b_end, void *stream) {
    const int bw = (w + 3) / 4, bh = (h + 3) / 4;
    if (b_end <= b_begin) return 0;
    const int aligned = ((w & 3) == 0) && ((reinterpret_cast<uintptr_t>(rgba) & 15) == 0);
    int grid = 0;
    if (small_index(b_end, &grid)) {
        grid = (int)((b_end - b_begin + 255) / 256);
        launch_decode_idx<uint32_t>(fmt, interp, grid, (cudaStream_t)stream, blocks, w, h, bw, bh, b_begin, b_end, write_alpha, c0, c1, aligned, rgba);
    } else {
        launch_decode_idx<uint64_t>(fmt, interp, grid, (cudaStream_t)stream, blocks, w, h, bw, bh, b_begin, b_end, write_alpha, c0, c1, aligned, rgba);
    }
    return (int)cudaGetLastError();
}

int launch_decode(int fmt, const uint8_t *blocks, int w, int h, int interp, int write_alpha, int c0, int c1,
                  uint8_t *rgba, void *stream) {
    return launch_decode_range(fmt, blocks, w, h, interp, write_alpha, c0, c1, rgba, 0,
                               (long)((w + 3) / 4) * ((h + 3) / 4), stream);
}

}  // namespace qtk
