// qt_kernels.cu — sm_100a kernels of the S3TC encode/decode path and their
// launchers.
//
// Mapping. Every kernel runs one 4x4 block per thread. BC1 (and the colour
// half of BC3) runs the reference encoder (BC1Encoder::EncodeBlock,
// BC1Encoder.cpp:261-342) sequentially per thread, in its order; those
// kernels are in qt_bc1_thread.cuh, included below. The reference's
// FindSelectors early exits never change an accepted result (every exit bound
// is >= the later acceptance bound), so full errors are computed instead.
//
// Floating point. Every operation whose rounding matters is written with an
// explicit round-to-nearest intrinsic (__fadd_rn, __fmul_rn, __fdiv_rn), in
// the reference's operation order; the compiler never contracts these into
// FMAs. Plain float arithmetic (and fmaf) is used only where every operand and
// result is an integer below 2^24, i.e. exact.
//
// BC4/BC5 encode and all decoders are HBM-bound: one thread per block,
// 16-byte row loads/stores where the texture is 4-aligned. The persistent
// batch kernel (k_batch) runs any mix of them from a device work queue.

#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cstdint>
#include <cstdlib>
#include <type_traits>

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
// per-CTA shared copies of small constant tables (read by every BC1 kernel)
// ---------------------------------------------------------------------------
__shared__ float s_mid5[32], s_mid6[64];
__shared__ uint16_t s_vox[16];

// Selector-search kinds: the (colour mode, error mode) pairs FindSelectors is
// ever called with. Three-colour searches are always ErrorMode::Full
// (BC1Encoder.cpp:313-333, 978-984).
constexpr int K_F4_NONE = 0, K_F4_FASTER = 1, K_F4_CHECK2 = 2, K_F4_FULL = 3, K_T3 = 4, K_TB = 5;
__host__ __device__ constexpr bool kind_three(int k) { return k >= K_T3; }
__host__ __device__ constexpr int kind_mode(int k) { return k == K_T3 ? CM_THREE : (k == K_TB ? CM_TB : CM_FOUR); }
__device__ __forceinline__ int kind_for(int M, int em) { return M == CM_THREE ? K_T3 : (M == CM_TB ? K_TB : em); }

// Vector4::Dot (Vector4.h:53-57) in the reference's rounding: sum from 0, left to right
__device__ __forceinline__ float fdot4_rn(float a0, float a1, float a2, float a3, float b0, float b1, float b2, float b3) {
    float s = __fadd_rn(0.0f, __fmul_rn(a0, b0));
    s = __fadd_rn(s, __fmul_rn(a1, b1));
    s = __fadd_rn(s, __fmul_rn(a2, b2));
    return __fadd_rn(s, __fmul_rn(a3, b3));
}

__device__ __forceinline__ bool is_single_hash(bool four, int h) {
    return four ? (h == 15 || h == 700 || h == 753 || h == 515) : (h == 12 || h == 15 || h == 89);
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

// WriteBlock of an EncodeResults (BC1Encoder.h:147-153): endpoints packed 5:6:5, sel the 16
// 2-bit internal selectors (texel i at bits 2i), mode its colour mode
__device__ __forceinline__ uint2 write_block(int lo, int hi, uint32_t sel_in, int mode) {
    int ep1 = lo, ep0 = hi;
    uint32_t lut;  // 4 x 2-bit entries
    if (mode & CM_FOUR) {
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
    for (int i = 0; i < 16; i++) sel |= ((lut >> (2 * ((sel_in >> (2 * i)) & 3))) & 3) << (2 * i);
    return make_uint2((uint32_t)ep0 | ((uint32_t)ep1 << 16), sel);
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

// Selector packing shared by the BC4 and BC5 encoders. A level q (0..9, see below) indexes
// the Levels table with one PTX prmt.b32: a selector nibble 0..7 copies byte q of
// {kBC4MapHi:kBC4MapLo}, and 8 or 9 copies the sign of byte 0 or 1 (map 1 and 7: sign 0), i.e. 0,
// which is map[7], the selector of every level >= 7. So no clamp and no mask are needed: the
// other result bytes hold map[0] = 1 (selector nibble 0), a known constant. Selector words are then
// accumulated with IMAD, acc += word << 3j, and that constant's contribution is subtracted once at
// the end (the arithmetic is exact modulo 2^32 and the 3-bit fields never overlap).
// (CUDA's __byte_perm takes only the low 3 bits of each nibble, so it would map 8 and 9 to
// map[0] and map[1]; the lookup needs the PTX instruction's sign-replicate mode.)
__device__ __forceinline__ uint32_t prmt_levels(uint32_t selector) {
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(kBC4MapLo), "r"(kBC4MapHi), "r"(selector));
    return d;
}
constexpr uint32_t kPermOnes = 0x01010100u;  // prmt result bytes 1..3 for a selector < 16
template <int N>
__host__ __device__ constexpr uint32_t perm_garbage(uint32_t word) {  // sum of word << 3j, j < N
    uint32_t c = 0;
    for (int j = 0; j < N; j++) c += word << (3 * j);
    return c;
}

// BC4Encoder::EncodeBlock (BC4Encoder.cpp:30-71) on channel ch. The reference
// counts the thresholds delta*(1+2c) - bias (c = 0..6) that 14*value reaches;
// for min <= value <= max that count is exactly
// min(7, floor((14*(value - min) + 4 + delta) / (2*delta))), and the division is
// a multiply-high by g_bc4_magic (exact for numerators below 4096; both facts
// checked for every (min, max, value)). The level itself, floor(...), is at most 9
// (delta >= 1), so the prmt table lookup above takes it unclamped.
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
    uint32_t a0 = 0u, a1 = 0u;                 // texels 0..9 (30 bits), 10..15 (18 bits)
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t q = __umulhi(14u * v[i] + K, M);
        const uint32_t word = prmt_levels(q);  // selector in byte 0
        if (i < 10) a0 += word << (3 * i);
        else a1 += word << (3 * (i - 10));
    }
    a0 -= perm_garbage<10>(kPermOnes);
    a1 -= perm_garbage<6>(kPermOnes);
    const uint32_t lo = a0 | (a1 << 30), hi = a1 >> 2;  // selector bits 0..31 and 32..47
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
// Both levels then index the Levels table in one prmt (selector nibbles 0 and 2),
// which puts channel c0's selector in byte 0 and c1's in byte 2 of one word; five
// texels' words accumulate into one register (two 15-bit fields, 3 bits per
// texel), as in bc4_block_thread.
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
    uint32_t g[4] = {0u, 0u, 0u, 0u};  // texels 0-4, 5-9, 10-14, 15: c0 fields in bits 0..14, c1 in 16..30
#pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t num = 14u * v[i] + Kp;
        const uint32_t q0 = __umulhi(num & 0xFFFFu, M0), q1 = __umulhi(num >> 16, M1);  // levels 0..9
        const uint32_t word = prmt_levels(q0 + (q1 << 8));  // selectors in bytes 0, 2
        g[i / 5] += word << (3 * (i % 5));
    }
    constexpr uint32_t kOnes2 = 0x01000100u;  // prmt result bytes 1 and 3 (selector nibbles 1, 3 = 0)
    g[0] -= perm_garbage<5>(kOnes2);
    g[1] -= perm_garbage<5>(kOnes2);
    g[2] -= perm_garbage<5>(kOnes2);
    g[3] -= perm_garbage<1>(kOnes2);
    // channel fields: 15 + 15 + 15 + 3 bits -> selector bits 0..31 (lo) and 32..47 (hi)
    const uint32_t f00 = g[0] & 0xFFFFu, f01 = g[1] & 0xFFFFu, f02 = g[2] & 0xFFFFu, f03 = g[3] & 0xFFFFu;
    const uint32_t f10 = g[0] >> 16, f11 = g[1] >> 16, f12 = g[2] >> 16, f13 = g[3] >> 16;
    const uint32_t lo0 = f00 | (f01 << 15) | (f02 << 30), hi0 = (f02 >> 2) | (f03 << 13);
    const uint32_t lo1 = f10 | (f11 << 15) | (f12 << 30), hi1 = (f12 >> 2) | (f13 << 13);
    const uint32_t mx0 = mn0 + d0, mx1 = mn1 + d1;
    uint4 r;
    r.x = d0 ? (mx0 | (mn0 << 8) | (lo0 << 16)) : (mn0 | (mn0 << 8));  // BC4Block(min) when solid
    r.y = d0 ? ((lo0 >> 16) | (hi0 << 16)) : 0u;
    r.z = d1 ? (mx1 | (mn1 << 8) | (lo1 << 16)) : (mn1 | (mn1 << 8));
    r.w = d1 ? ((lo1 >> 16) | (hi1 << 16)) : 0u;
    return r;
}

// One thread per block. Idx is uint32_t whenever the block count and the grid fit
// 31 bits (the common case: no 64-bit division per block), else uint64_t. BC5 is held to
// 40 registers (6 CTAs of 256 threads per SM instead of 5 at its natural 44): its loads
// need the extra warps in flight (measured 0.83 -> 0.88 of HBM at 16384^2, bit-identical).
// BC4 gives no minimum (0), where the compiler also settles at 40 registers; an explicit
// minimum of 1 to 4 CTAs lets it take 52-56 and costs BC4 a tenth of its bandwidth.
//
// BC4: one block per thread. BC5 (two channels' arithmetic per texel) was latency-bound, so its
// grid is persistent (the SMs filled at the kernel's occupancy) and each thread's next block
// arrives by cp.async into shared memory while it encodes the current one: the rows are
// transposed there ([buffer][texel row][thread], 16 bytes each), so a warp's copies and reads
// are conflict-free, and the block in flight holds no registers (0.88 -> 0.905 of HBM; the same
// for BC4 measured 0.97 -> 0.91, so BC4 keeps the plain loop). Edge blocks of a texture whose
// width is not a multiple of 4 (or an unaligned base) are loaded directly, with the wrap rule.
template <bool BC5, typename Idx>
__global__ void __launch_bounds__(256, BC5 ? 6 : 0) k_bc4_encode(const uint8_t *__restrict__ rgba, int w, int h, Idx bw, Idx b_begin,
                                                    Idx nblocks, int c0, int c1, int aligned, uint8_t *__restrict__ out) {
    if constexpr (!BC5) {
        for (Idx b = b_begin + (Idx)blockIdx.x * blockDim.x + threadIdx.x; b < nblocks; b += (Idx)gridDim.x * blockDim.x) {
            const int by = (int)(b / bw), bx = (int)(b - (Idx)by * bw);
            uint32_t px[16];
            load_block_thread(rgba, w, h, bx, by, aligned && (bx * 4 + 4 <= w) && (by * 4 + 4 <= h), px);
            reinterpret_cast<uint2 *>(out)[b] = bc4_block_thread(px, c0);
        }
        return;
    }
    __shared__ uint4 stage[2][4][256];
    const Idx stride = (Idx)gridDim.x * blockDim.x;
    // the row copies of block bb into buffer buf, when it is an aligned interior block
    auto prefetch = [&](Idx bb, int buf) -> bool {
        if (bb >= nblocks) return false;
        const int by = (int)(bb / bw), bx = (int)(bb - (Idx)by * bw);
        if (!(aligned && (bx * 4 + 4 <= w) && (by * 4 + 4 <= h))) return false;
#pragma unroll
        for (int y = 0; y < 4; y++)
            __pipeline_memcpy_async(&stage[buf][y][threadIdx.x], rgba + ((size_t)(by * 4 + y) * w + bx * 4) * 4, 16);
        return true;
    };
    Idx b = b_begin + (Idx)blockIdx.x * blockDim.x + threadIdx.x;
    bool staged = prefetch(b, 0);
    __pipeline_commit();
    for (int buf = 0; b < nblocks; b += stride, buf ^= 1) {
        const bool next = prefetch(b + stride, buf ^ 1);
        __pipeline_commit();
        __pipeline_wait_prior(1);  // this block's copies (the group before the newest) have landed
        uint32_t px[16];
        if (staged) {
#pragma unroll
            for (int y = 0; y < 4; y++) {
                const uint4 q = stage[buf][y][threadIdx.x];
                px[4 * y] = q.x; px[4 * y + 1] = q.y; px[4 * y + 2] = q.z; px[4 * y + 3] = q.w;
            }
        } else {
            const int by = (int)(b / bw), bx = (int)(b - (Idx)by * bw);
            load_block_thread(rgba, w, h, bx, by, false, px);
        }
        reinterpret_cast<uint4 *>(out)[b] = bc5_block_thread(px, c0, c1);
        staged = next;
    }
    __pipeline_wait_prior(0);
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

// below this many blocks the split pass costs more than idle solid lanes do
constexpr long kSplitMinBlocks = 16384;

long defer_min_blocks() { return 2L * num_sms() * 4 * tpb::kThreads; }

// the four-colour cluster fit runs twice (EncodeBlock, BC1Encoder.cpp:299-302); exactly then
// encode_block, given a Deferred, stops blocks before the second pass
static bool cf2_pass(const qt_bc1_params &p) {
    return p.two_cf_passes && (p.exhaustive || p.orderings3 > 0 || p.orderings4 > 0);
}

// The specialised encoder (k_bc1_fast) for a setting without EndpointSearch: its four-colour
// selector kind is the error mode (every setting has cluster-fit orderings, so it needs block
// errors: BC1Encoder.cpp:267-276); its colour mode is the setting's, four-colour for BC3. With
// list/count the blocks are the listed ones.
template <int IT, int K4>
static void launch_fast_k(int g, cudaStream_t s, const uint8_t *rgba, int w, int h, int bw, long b0, long b1,
                          const qt_bc1_params &p, uint8_t *out, bool bc3, int aligned, const uint32_t *list,
                          const uint32_t *count) {
    const int cm = bc3 ? CM_FOUR : p.color_mode;  // BC3Encoder.h:39-40
    if (cm == CM_FOUR)
        k_bc1_fast<IT, K4, CM_FOUR><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count);
    else if (cm == CM_THREE)
        k_bc1_fast<IT, K4, CM_THREE><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count);
    else
        k_bc1_fast<IT, K4, CM_TB><<<g, tpb::kThreads, 0, s>>>(rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count);
}

template <int IT>
static void launch_fast_it(int g, cudaStream_t s, const uint8_t *rgba, int w, int h, int bw, long b0, long b1,
                           const qt_bc1_params &p, uint8_t *out, bool bc3, int aligned, const uint32_t *list,
                           const uint32_t *count) {
    switch (p.error_mode) {
        case EM_NONE: launch_fast_k<IT, K_F4_NONE>(g, s, rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count); break;
        case EM_FASTER: launch_fast_k<IT, K_F4_FASTER>(g, s, rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count); break;
        case EM_CHECK2: launch_fast_k<IT, K_F4_CHECK2>(g, s, rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count); break;
        default: launch_fast_k<IT, K_F4_FULL>(g, s, rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count); break;
    }
}

static void launch_fast(int g, cudaStream_t s, const uint8_t *rgba, int w, int h, int bw, long b0, long b1,
                        const qt_bc1_params &p, uint8_t *out, bool bc3, int aligned, const uint32_t *list,
                        const uint32_t *count) {
    switch (p.interpolator) {
        case IT_IDEAL: launch_fast_it<IT_IDEAL>(g, s, rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count); break;
        case IT_ROUND: launch_fast_it<IT_ROUND>(g, s, rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count); break;
        case IT_NVIDIA: launch_fast_it<IT_NVIDIA>(g, s, rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count); break;
        default: launch_fast_it<IT_AMD>(g, s, rgba, w, h, bw, b0, b1, p, out, bc3, aligned, list, count); break;
    }
}

template <typename F>
static void by_interp(int interpolator, F &&f) {
    switch (interpolator) {
        case IT_IDEAL: f(std::integral_constant<int, IT_IDEAL>()); break;
        case IT_ROUND: f(std::integral_constant<int, IT_ROUND>()); break;
        case IT_NVIDIA: f(std::integral_constant<int, IT_NVIDIA>()); break;
        default: f(std::integral_constant<int, IT_AMD>()); break;
    }
}

// Scratch of the deferred path over n blocks, in 32-bit words: a 64-word header (word 0 the
// list count, 1-3 the search queues' counts, 4-6 their heads, 8-9 the second-pass queue's
// counts, 16 the finish queue's count, 32-63 the list counts of a texture encoded in parts),
// the list of non-solid blocks, the three search queues (5 arrays each), the finish queue (3
// arrays) and, with the second cluster-fit pass, its queue (6 arrays).
constexpr int kPartCount0 = 32, kMaxParts = 32;
static size_t defer_words(long n, bool cf2) { return 64 + 19 * (size_t)n + (cf2 ? 6 * (size_t)n : 0); }

struct DeferQueues {
    SearchQueues q;
    FinishQueue fq;
    Cf2Queue c;
};

static DeferQueues defer_layout(uint32_t *scratch, long n, bool cf2) {
    DeferQueues d{};
    uint32_t *qb = scratch + 64 + n;
    d.q.count = scratch + 1;
    d.q.head = scratch + 4;
    d.q.cap = n;
    d.q.b = qb;
    d.q.lohi = qb + 3 * (size_t)n;
    d.q.err = qb + 6 * (size_t)n;
    d.q.sel = qb + 9 * (size_t)n;
    d.q.mode = qb + 12 * (size_t)n;
    d.fq.count = scratch + 16;  // searches that moved the endpoints
    d.fq.b = qb + 15 * (size_t)n;
    d.fq.lohi = d.fq.b + (size_t)n;
    d.fq.mode = d.fq.b + 2 * (size_t)n;
    if (cf2) {
        uint32_t *cb = qb + 18 * (size_t)n;
        d.c.count = scratch + 8;
        d.c.b = cb;
        d.c.lohi = cb + (size_t)n;
        d.c.err = cb + 2 * (size_t)n;
        d.c.sel = cb + 3 * (size_t)n;
        d.c.mode = cb + 4 * (size_t)n;
        d.c.orig = cb + 5 * (size_t)n;
        d.c.cap = n;
    }
    return d;
}

// The deferred path's first passes over the blocks [b0, b1): the split pass lists the
// non-solid blocks in list/count, the encoder runs each to its first cluster-fit pass and
// queues what remains (second pass, 3-colour trials, EndpointSearch) in d.
template <int I>
static void defer_front(const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3, int aligned,
                        const DeferQueues &d, uint32_t *list, uint32_t *count, long b0, long b1, cudaStream_t s) {
    const int bw = (w + 3) / 4;
    const long n = b1 - b0;
    k_bc1_split<I><<<grid_for(n, 256), 256, 0, s>>>(rgba, w, h, bw, b0, b1, out, bc3, aligned, list, count);
    k_bc1_defer<I><<<grid_for(n, tpb::kThreads), tpb::kThreads, 0, s>>>(rgba, w, h, bw, p, out, bc3, aligned, list,
                                                                          count, d.q, d.c);
}

// ... and its passes over the queues: second cluster-fit pass and 3-colour trials (cf2),
// EndpointSearch with lane refill, and the selectors of the searches that moved.
template <int I>
static void defer_back(const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3, int aligned,
                       const DeferQueues &d, bool cf2, cudaStream_t s) {
    const int bw = (w + 3) / 4;
    const int gsearch = num_sms() * 4;
    if (cf2) k_bc1_cf2<I><<<gsearch, tpb::kThreads, 0, s>>>(rgba, w, h, bw, p, out, bc3, aligned, d.c, d.q);
    k_bc1_search<I><<<gsearch, tpb::kThreads, 0, s>>>(rgba, w, h, bw, p, out, bc3, aligned, d.q, d.fq);
    k_bc1_finish<I><<<gsearch, tpb::kThreads, 0, s>>>(rgba, w, h, bw, p, out, bc3, aligned, d.fq);
}

static int texel_aligned(const uint8_t *rgba, int w) {
    return ((w & 3) == 0) && ((reinterpret_cast<uintptr_t>(rgba) & 15) == 0);
}

bool bc1_parts_eligible(long nblocks, const qt_bc1_params &p) {
    return p.search_rounds > 0 && nblocks >= defer_min_blocks() && nblocks <= 0xFFFFFFFFL;
}

int bc1_parts_begin(Bc1Parts &ps, long nblocks, const qt_bc1_params &p, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    ps = Bc1Parts{};
    if (!bc1_parts_eligible(nblocks, p)) return (int)cudaErrorInvalidValue;
    ps.n = nblocks;
    ps.cf2 = cf2_pass(p);
    cudaError_t e = scratch_alloc((void **)&ps.scratch, defer_words(nblocks, ps.cf2) * sizeof(uint32_t), s);
    if (e != cudaSuccess) {
        ps.scratch = nullptr;
        return (int)e;
    }
    e = cudaMemsetAsync(ps.scratch, 0, 64 * sizeof(uint32_t), s);
    return (int)e;
}

int bc1_parts_add(Bc1Parts &ps, const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3,
                  long b_begin, long b_end, void *stream) {
    if (!ps.scratch || ps.parts >= kMaxParts || b_begin < 0 || b_end > ps.n || b_end <= b_begin)
        return (int)cudaErrorInvalidValue;
    // part k lists its non-solid blocks in its own slice of the list (at most b_end - b_begin
    // of them) and counts them in header word 32 + k; the queues are shared
    uint32_t *list = ps.scratch + 64 + b_begin, *count = ps.scratch + kPartCount0 + ps.parts++;
    const DeferQueues d = defer_layout(ps.scratch, ps.n, ps.cf2);
    cudaStream_t s = (cudaStream_t)stream;
    by_interp(p.interpolator, [&](auto I) {
        defer_front<decltype(I)::value>(rgba, w, h, p, out, bc3, texel_aligned(rgba, w), d, list, count, b_begin, b_end, s);
    });
    return (int)cudaGetLastError();
}

int bc1_parts_end(Bc1Parts &ps, const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3,
                  void *stream) {
    if (!ps.scratch) return (int)cudaErrorInvalidValue;
    const DeferQueues d = defer_layout(ps.scratch, ps.n, ps.cf2);
    cudaStream_t s = (cudaStream_t)stream;
    by_interp(p.interpolator, [&](auto I) {
        defer_back<decltype(I)::value>(rgba, w, h, p, out, bc3, texel_aligned(rgba, w), d, ps.cf2, s);
    });
    const cudaError_t e = cudaGetLastError();
    bc1_parts_free(ps, stream);
    return (int)e;
}

void bc1_parts_free(Bc1Parts &ps, void *stream) {
    if (ps.scratch) scratch_free(ps.scratch, (cudaStream_t)stream);
    ps.scratch = nullptr;
}

int launch_bc1_encode_range(const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3,
                            long b_begin, long b_end, void *stream) {
    const int bw = (w + 3) / 4;
    const long n = b_end - b_begin;
    if (n <= 0) return 0;
    cudaStream_t s = (cudaStream_t)stream;
    {
        const int aligned = texel_aligned(rgba, w);
        const int g = grid_for(n, tpb::kThreads);
        if ((n < kSplitMinBlocks || n > 0xFFFFFFFFL) && p.search_rounds == 0) {
            launch_fast(g, s, rgba, w, h, bw, b_begin, b_end, p, out, bc3, aligned, nullptr, nullptr);
            return (int)cudaGetLastError();
        }
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
        const size_t words = defer ? defer_words(n, cf2) : 64 + (size_t)n;
        uint32_t *scratch = nullptr;
        cudaError_t e = scratch_alloc((void **)&scratch, words * sizeof(uint32_t), s);
        if (e != cudaSuccess) return (int)e;
        uint32_t *count = scratch, *list = scratch + 64;
        e = cudaMemsetAsync(scratch, 0, 64 * sizeof(uint32_t), s);  // list count, queue counts and heads
        if (e == cudaSuccess && defer) {
            const DeferQueues d = defer_layout(scratch, n, cf2);
            by_interp(p.interpolator, [&](auto I) {
                defer_front<decltype(I)::value>(rgba, w, h, p, out, bc3, aligned, d, list, count, b_begin, b_end, s);
                defer_back<decltype(I)::value>(rgba, w, h, p, out, bc3, aligned, d, cf2, s);
            });
            e = cudaGetLastError();
        } else if (e == cudaSuccess && p.search_rounds == 0) {
            const int gs = grid_for(n, 256);
            switch (p.interpolator) {
                case IT_IDEAL: k_bc1_split<IT_IDEAL><<<gs, 256, 0, s>>>(rgba, w, h, bw, b_begin, b_end, out, bc3, aligned, list, count); break;
                case IT_ROUND: k_bc1_split<IT_ROUND><<<gs, 256, 0, s>>>(rgba, w, h, bw, b_begin, b_end, out, bc3, aligned, list, count); break;
                case IT_NVIDIA: k_bc1_split<IT_NVIDIA><<<gs, 256, 0, s>>>(rgba, w, h, bw, b_begin, b_end, out, bc3, aligned, list, count); break;
                default: k_bc1_split<IT_AMD><<<gs, 256, 0, s>>>(rgba, w, h, bw, b_begin, b_end, out, bc3, aligned, list, count); break;
            }
            launch_fast(g, s, rgba, w, h, bw, 0, 0, p, out, bc3, aligned, list, count);
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
}

int bc1_encode_kernels(long n, const qt_bc1_params &p) {
    if (n <= 0) return 0;
    if (n < kSplitMinBlocks || n > 0xFFFFFFFFL) return 1;
    if (p.search_rounds == 0 || n < defer_min_blocks()) return 2;
    return cf2_pass(p) ? 5 : 4;  // split, encoder, (second cluster-fit pass,) search, finish
}

int launch_bc1_encode(const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3, void *stream) {
    return launch_bc1_encode_range(rgba, w, h, p, out, bc3, 0, (long)((w + 3) / 4) * ((h + 3) / 4), stream);
}

int batch_sms() { return num_sms(); }

static int batch_ctas_per_sm_at(int threads) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch, threads, 0) != cudaSuccess || n <= 0) n = 1;
    return n;
}

int batch_ctas_per_sm() { return batch_ctas_per_sm_at(tpb::kThreads); }

int launch_batch(const BatchItemDev *items, const TileDev *tiles, uint32_t *ctl, int grid, int threads, void *stream) {
    // the kernel's shared-memory columns hold tpb::kThreads threads; smaller CTAs use a prefix
    if (threads != 32 && threads != 64 && threads != tpb::kThreads) return (int)cudaErrorInvalidValue;
    if (grid <= 0) grid = num_sms() * batch_ctas_per_sm_at(threads);
    k_batch<<<grid, threads, 0, (cudaStream_t)stream>>>(items, tiles, ctl);
    return (int)cudaGetLastError();
}

int launch_batch(const BatchItemDev *items, const TileDev *tiles, uint32_t *ctl, int grid, void *stream) {
    return launch_batch(items, tiles, ctl, grid, tpb::kThreads, stream);
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
        if (bc5) {  // persistent: at most the CTAs the SMs hold at once (each thread then loops,
                    // its next block's copies in flight while it encodes)
            static int resident = 0;
            if (resident <= 0) {  // 32 KB of staging per CTA: the shared-memory carveout that fits 6
                int per_sm = 0;
                const void *k = (const void *)k_bc4_encode<true, uint32_t>;
                cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
                const cudaError_t oe = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, 256, 0);
                cudaGetLastError();
                resident = num_sms() * (oe == cudaSuccess && per_sm > 0 ? per_sm : 1);
            }
            grid = std::min(grid, resident);
        }
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
