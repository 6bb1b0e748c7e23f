// qt_bc1_thread.cuh — thread-per-block BC1/BC3 encoder (included by qt_kernels.cu).
//
// One thread encodes one 4x4 block, following BC1Encoder::EncodeBlock
// (BC1Encoder.cpp:261-342) step by step, with no cross-lane work: no
// replicated scalar code, no reductions, 32 blocks in flight per warp. The
// block's texels and cluster-fit prefix sums live in shared memory in a
// transposed layout ([item][thread]), so every per-texel access of a warp is
// one conflict-free shared load and the loops stay rolled (a small instruction
// footprint); the sort keys live in registers. Float arithmetic uses explicit
// round-to-nearest intrinsics in the reference's operation order; every texel
// sum is an exact integer.

namespace tpb {

constexpr int kThreads = 128;

// -2 and -1 that the compiler cannot fold: d * kNeg2 + v stays one IMAD on the FMA pipe. The
// Full trial-error loops use it for half of their |c|^2 - 2 p.c terms, so that the integer ALU
// pipe (min, add) and the FMA pipe (dp4a, IMAD) share the work; the loops whose comparisons and
// selects already fill the ALU pipe (Check2 and Faster, and FindSelectors in Full mode) for every
// term and for p.axis. Measured over the plain expressions, which compile to ALU instructions:
// Check2 L0 +2.5-4%, L10 +2-4.5%; Faster (which also selects among four errors instead of
// among palette words) L5 +4.5-7%, L7 +12%, BC3 L5 +8%; FindSelectors' Full loop +1-2% at the
// three-colour settings.
__constant__ int kNeg2 = -2;
__constant__ int kNeg1 = -1;

__shared__ uint32_t t_px[16][kThreads];     // texel i of the thread's block
__shared__ uint32_t t_srg[17][kThreads];    // cluster-fit prefix sums: r | g << 16
__shared__ uint16_t t_sb[17][kThreads];     //                          b

struct R {  // EncodeResults (BC1Encoder.h:147-153); endpoints packed 5:6:5
    int lo, hi;
    uint32_t sel;
    int mode;
    uint32_t err;
};

__device__ __forceinline__ R rinit() {
    R r;
    r.lo = r.hi = 0;
    r.sel = 0;
    r.mode = CM_INCOMPLETE;
    r.err = UINT_MAX;
    return r;
}

struct M {  // ColorBlock::Metrics (ColorBlock.h:88-117)
    int mn[3], mx[3], av[3], sum[3];
    bool grey, has_black;
};

__device__ __forceinline__ uint32_t px(int i) { return t_px[i][threadIdx.x]; }
__device__ __forceinline__ int cr(uint32_t v) { return v & 0xFF; }
__device__ __forceinline__ int cg(uint32_t v) { return (v >> 8) & 0xFF; }
__device__ __forceinline__ int cb(uint32_t v) { return (v >> 16) & 0xFF; }
__device__ __forceinline__ bool black(uint32_t v) { return (cr(v) | cg(v) | cb(v)) < 4; }

// Texels i..i+3 as one word per channel (byte k = texel i + k), for dp4a over four texels
__device__ __forceinline__ void channel_words(int i, uint32_t &R, uint32_t &G, uint32_t &B) {
    const uint32_t v0 = px(i), v1 = px(i + 1), v2 = px(i + 2), v3 = px(i + 3);
    const uint32_t t01 = __byte_perm(v0, v1, 0x5140), t23 = __byte_perm(v2, v3, 0x5140);  // r r g g
    const uint32_t u01 = __byte_perm(v0, v1, 0x7362), u23 = __byte_perm(v2, v3, 0x7362);  // b b a a
    R = __byte_perm(t01, t23, 0x5410);
    G = __byte_perm(t01, t23, 0x7632);
    B = __byte_perm(u01, u23, 0x5410);
}

__device__ __forceinline__ M metrics_body(bool ignore_black) {
    M m;
    int total = 0;
    // two channels per word (r | b << 16, g | a << 16): packed 16-bit min, max and sums (at most
    // 16 x 255 per half); the alpha half is carried along and dropped
    uint32_t mn_rb = 0x00FF00FFu, mn_ga = 0x00FF00FFu, mx_rb = 0u, mx_ga = 0u, s_rb = 0u, s_ga = 0u;
    bool grey = true, has_black = false;
#pragma unroll 4
    for (int i = 0; i < 16; i++) {
        const uint32_t v = px(i);
        const bool b = (v & 0x00FCFCFCu) == 0u;  // (r | g | b) < 4
        has_black |= b;
        if (ignore_black && b) continue;
        const uint32_t rb = v & 0x00FF00FFu, ga = (v >> 8) & 0x00FF00FFu;
        grey &= (v & 0x00FFFFFFu) == (v & 0xFFu) * 0x010101u;
        asm("min.u16x2 %0, %0, %1;" : "+r"(mn_rb) : "r"(rb));
        asm("min.u16x2 %0, %0, %1;" : "+r"(mn_ga) : "r"(ga));
        asm("max.u16x2 %0, %0, %1;" : "+r"(mx_rb) : "r"(rb));
        asm("max.u16x2 %0, %0, %1;" : "+r"(mx_ga) : "r"(ga));
        s_rb += rb;
        s_ga += ga;
        total++;
    }
    m.has_black = has_black;
    m.grey = grey;
    m.mn[0] = (int)(mn_rb & 0xFFFFu); m.mn[1] = (int)(mn_ga & 0xFFFFu); m.mn[2] = (int)(mn_rb >> 16);
    m.mx[0] = (int)(mx_rb & 0xFFFFu); m.mx[1] = (int)(mx_ga & 0xFFFFu); m.mx[2] = (int)(mx_rb >> 16);
    m.sum[0] = (int)(s_rb & 0xFFFFu); m.sum[1] = (int)(s_ga & 0xFFFFu); m.sum[2] = (int)(s_rb >> 16);
#pragma unroll
    for (int c = 0; c < 3; c++) m.av[c] = total > 0 ? (m.sum[c] + total / 2) / total : 0;
    return m;
}

// Each phase exists twice: its body (__forceinline__, *_body) and a __noinline__ copy under the
// plain name, one per template instance. The generic kernels call the copies, which keeps
// their instruction working set small when one kernel serves every setting; the specialised
// kernels (k_bc1_fast: one selector kind, no EndpointSearch) inline the bodies, which saves
// the call overhead where the per-block work is small. INL picks one at compile time.
__device__ __noinline__ M metrics(bool ignore_black) { return metrics_body(ignore_black); }
template <bool INL> __device__ __forceinline__ M metrics_(bool ignore_black) {
    if constexpr (INL) return metrics_body(ignore_black);
    else return metrics(ignore_black);
}

// Check2's projected selector (BC1Encoder.cpp:723-729) is trunc(fl(fl(dd * f) + 0.5)) clamped to
// [1, 3], dd = (p - c0).axis an exact integer, f = fl(4 / den). Rounding is monotone, so the selector
// is >= s exactly when dd reaches the smallest integer with fl(fl(dd * f) + 0.5) >= s. Over every
// |axis|^2 in [0, 3 * 255^2] that integer is ceil(fl(fl(s - 0.5) * fl(den / 4))) or one more
// (checked exhaustively), so one evaluation of the rounded expression finds it.
__device__ __forceinline__ int check2_threshold(float f, float quarter_den, float s) {
    const int est = __float2int_ru(__fmul_rn(__fadd_rn(s, -0.5f), quarter_den));
    return est + (int)!(__fadd_rn(__fmul_rn(__int2float_rn(est), f), 0.5f) >= s);
}

// FindSelectors<M>(error_mode), BC1Encoder.cpp:679-779; K is one of the selector kinds (K_*)
template <int IT, int K> __device__ __forceinline__ uint2 find_selectors_body(int lo, int hi) {
    const Pal P = make_pal<IT>(lo, hi, kind_three(K));
    // palette colours (internal order) as packed RGB words and their |c|^2: the error of texel p
    // against colour k is |p|^2 + v_k - 2 p.c_k, exact in integers (dp4a)
    const uint32_t c0 = P.r0 | (P.g0 << 8) | (P.b0 << 16), c1 = P.r1 | (P.g1 << 8) | (P.b1 << 16);
    const uint32_t c2 = P.r2 | (P.g2 << 8) | (P.b2 << 16), c3 = P.r3 | (P.g3 << 8) | (P.b3 << 16);
    const int v0 = (int)__dp4a(c0, c0, 0u), v1 = (int)__dp4a(c1, c1, 0u);
    const int v2 = (int)__dp4a(c2, c2, 0u), v3 = (int)__dp4a(c3, c3, 0u);
    uint32_t sel = 0, tot = 0;
    if (K == K_F4_NONE || K == K_F4_FASTER) {
        const int ar = P.r3 - P.r0, ag = P.g3 - P.g0, ab = P.b3 - P.b0;
        const int d0 = ar * P.r0 + ag * P.g0 + ab * P.b0, d1 = ar * P.r1 + ag * P.g1 + ab * P.b1;
        const int d2 = ar * P.r2 + ag * P.g2 + ab * P.b2, d3 = ar * P.r3 + ag * P.g3 + ab * P.b3;
        const int t0 = d0 + d1, t1 = d1 + d2, t2 = d2 + d3;
        const int h0 = t0 >> 1, h1 = (t1 - 1) >> 1, h2 = (t2 - 1) >> 1;  // floor division
#pragma unroll 4
        for (int i = 0; i < 16; i++) {
            const uint32_t v = px(i);
            // 2 p.axis, with axis = palette entry 3 - entry 0 (the palette words' byte 3 is 0)
            const int p0 = (int)__dp4a(v, c0, 0u), p3 = (int)__dp4a(v, c3, 0u);
            const int pd = p0 * kNeg1 + p3;  // p.axis; 2 p.axis <= t0 exactly when p.axis <= h0 ...
            const int s = 3 - ((pd <= h0) + (pd <= h1) + (pd <= h2));
            if (K == K_F4_FASTER) {
                const uint32_t u = v & 0x00FFFFFFu;
                const int p1 = (int)__dp4a(v, c1, 0u), p2 = (int)__dp4a(v, c2, 0u);
                const int q0 = p0 * kNeg2 + v0, q1 = p1 * kNeg2 + v1, q2 = p2 * kNeg2 + v2, q3 = p3 * kNeg2 + v3;
                const int e = s == 0 ? q0 : s == 1 ? q1 : s == 2 ? q2 : q3;
                tot += (uint32_t)((int)__dp4a(u, u, 0u) + e);
            }
            sel |= (uint32_t)s << (2 * i);
        }
    } else if (K == K_F4_CHECK2) {
        const int ar = P.r3 - P.r0, ag = P.g3 - P.g0, ab = P.b3 - P.b0;
        const float den = __fadd_rn(__uint2float_rn(sq3(ar, ag, ab)), .00000125f);
        const float f = __fdiv_rn(4.0f, den), quarter = __fmul_rn(den, 0.25f);
        const int dbase = P.r0 * ar + P.g0 * ag + P.b0 * ab;
        // the projected selector is >= 2 (>= 3) exactly when p.axis - c0.axis reaches the threshold
        const int u2 = check2_threshold(f, quarter, 2.0f) + dbase, u3 = check2_threshold(f, quarter, 3.0f) + dbase;
#pragma unroll 4
        for (int i = 0; i < 16; i++) {
            const uint32_t v = px(i), u = v & 0x00FFFFFFu;
            const int p0 = (int)__dp4a(v, c0, 0u), p1 = (int)__dp4a(v, c1, 0u);
            const int p2 = (int)__dp4a(v, c2, 0u), p3 = (int)__dp4a(v, c3, 0u);
            const int pd = p0 * kNeg1 + p3;  // p.axis
            const bool two = pd >= u2, three = pd >= u3;
            const int sl = three ? 3 : two ? 2 : 1;
            // the two candidates sl-1 and sl
            const int q0 = p0 * kNeg2 + v0, q1 = p1 * kNeg2 + v1, q2 = p2 * kNeg2 + v2, q3 = p3 * kNeg2 + v3;
            const int e0 = three ? q2 : two ? q1 : q0;
            const int e1 = three ? q3 : two ? q2 : q1;
            int s = sl, e = e1;
            if (e0 == e1) {
                if (s == 1) s = 0;
            } else if (e0 < e) {
                s = sl - 1;
                e = e0;
            }
            tot += (uint32_t)(e + (int)__dp4a(u, u, 0u));
            sel |= (uint32_t)s << (2 * i);
        }
    } else {
#pragma unroll 4
        for (int i = 0; i < 16; i++) {
            const uint32_t u = px(i) & 0x00FFFFFFu;
            const int pp = (int)__dp4a(u, u, 0u);
            // ties keep the lower index except selector 3 (:762)
            int e = (int)__dp4a(u, c0, 0u) * kNeg2 + v0, s = 0;
            const int e1 = (int)__dp4a(u, c1, 0u) * kNeg2 + v1;
            if (e1 < e) { e = e1; s = 1; }
            const int e2 = (int)__dp4a(u, c2, 0u) * kNeg2 + v2;
            if (e2 < e) { e = e2; s = 2; }
            if (K != K_T3) {
                const int e3 = (int)__dp4a(u, c3, 0u) * kNeg2 + v3;
                if (e3 <= e) { e = e3; s = 3; }
            }
            tot += (uint32_t)(e + pp);
            sel |= (uint32_t)s << (2 * i);
        }
    }
    return make_uint2(sel, tot);
}

template <int IT, int K> __device__ __noinline__ uint2 find_selectors(int lo, int hi) {
    return find_selectors_body<IT, K>(lo, hi);
}
template <int IT, int K, bool INL> __device__ __forceinline__ uint2 find_selectors_(int lo, int hi) {
    if constexpr (INL) return find_selectors_body<IT, K>(lo, hi);
    else return find_selectors<IT, K>(lo, hi);
}

template <int IT> __device__ __forceinline__ uint2 fs_any(int K, int lo, int hi) {
    switch (K) {
        case K_F4_NONE: return find_selectors<IT, K_F4_NONE>(lo, hi);
        case K_F4_FASTER: return find_selectors<IT, K_F4_FASTER>(lo, hi);
        case K_F4_CHECK2: return find_selectors<IT, K_F4_CHECK2>(lo, hi);
        case K_F4_FULL: return find_selectors<IT, K_F4_FULL>(lo, hi);
        case K_T3: return find_selectors<IT, K_T3>(lo, hi);
        default: return find_selectors<IT, K_TB>(lo, hi);
    }
}

// error of the endpoints only (the cluster-fit and search trials); same as find_selectors' total
template <int IT, int K> __device__ __forceinline__ uint32_t block_error(int lo, int hi, int pp_sum) {
    const Pal P = make_pal<IT>(lo, hi, kind_three(K));
    if (K == K_F4_FULL || K == K_T3 || K == K_TB) {
        const uint32_t c0 = P.r0 | (P.g0 << 8) | (P.b0 << 16), c1 = P.r1 | (P.g1 << 8) | (P.b1 << 16);
        const uint32_t c2 = P.r2 | (P.g2 << 8) | (P.b2 << 16), c3 = P.r3 | (P.g3 << 8) | (P.b3 << 16);
        const int v0 = (int)__dp4a(c0, c0, 0u), v1 = (int)__dp4a(c1, c1, 0u);
        const int v2 = (int)__dp4a(c2, c2, 0u), v3 = (int)__dp4a(c3, c3, 0u);
        int t0 = 0, t1 = 0;
#pragma unroll 4
        for (int i = 0; i < 16; i += 2) {
            const uint32_t u = px(i), q = px(i + 1);
            int m = v0 - 2 * (int)__dp4a(u, c0, 0u), n = v0 - 2 * (int)__dp4a(q, c0, 0u);
            m = min(m, (int)__dp4a(u, c1, 0u) * kNeg2 + v1);
            n = min(n, (int)__dp4a(q, c1, 0u) * kNeg2 + v1);
            m = min(m, v2 - 2 * (int)__dp4a(u, c2, 0u));
            n = min(n, v2 - 2 * (int)__dp4a(q, c2, 0u));
            if (K != K_T3) {
                m = min(m, (int)__dp4a(u, c3, 0u) * kNeg2 + v3);
                n = min(n, (int)__dp4a(q, c3, 0u) * kNeg2 + v3);
            }
            t0 += m;
            t1 += n;
        }
        return (uint32_t)(pp_sum + t0 + t1);
    }
    if (K == K_F4_CHECK2 || K == K_F4_FASTER) {
        // The total of FindSelectors' Check2 / Faster modes (BC1Encoder.cpp:697-749) without the
        // selectors: ties choose between selectors of equal error, so they do not change it. The
        // axis is palette entry 3 - entry 0, so p.axis = p.c3 - p.c0 from the same dp4a products.
        const uint32_t c0 = P.r0 | (P.g0 << 8) | (P.b0 << 16), c1 = P.r1 | (P.g1 << 8) | (P.b1 << 16);
        const uint32_t c2 = P.r2 | (P.g2 << 8) | (P.b2 << 16), c3 = P.r3 | (P.g3 << 8) | (P.b3 << 16);
        const int v0 = (int)__dp4a(c0, c0, 0u), v1 = (int)__dp4a(c1, c1, 0u);
        const int v2 = (int)__dp4a(c2, c2, 0u), v3 = (int)__dp4a(c3, c3, 0u);
        const int ar = P.r3 - P.r0, ag = P.g3 - P.g0, ab = P.b3 - P.b0;
        int t = 0;
        if (K == K_F4_CHECK2) {
            const float den = __fadd_rn(__uint2float_rn(sq3(ar, ag, ab)), .00000125f);
            const float f = __fdiv_rn(4.0f, den), quarter = __fmul_rn(den, 0.25f);
            const int dbase = P.r0 * ar + P.g0 * ag + P.b0 * ab;
            // selector >= 2 (>= 3) exactly when p.axis - c0.axis reaches the threshold
            const int u2 = check2_threshold(f, quarter, 2.0f) + dbase, u3 = check2_threshold(f, quarter, 3.0f) + dbase;
#pragma unroll 4
            for (int i = 0; i < 16; i++) {
                const uint32_t u = px(i);  // the palette words' byte 3 is 0: alpha drops out of dp4a
                const int d0 = (int)__dp4a(u, c0, 0u), d1 = (int)__dp4a(u, c1, 0u);
                const int d2 = (int)__dp4a(u, c2, 0u), d3 = (int)__dp4a(u, c3, 0u);
                const int pd = d0 * kNeg1 + d3;
                const bool two = pd >= u2, three = pd >= u3;
                const int e0 = d0 * kNeg2 + v0, e1 = d1 * kNeg2 + v1, e2 = d2 * kNeg2 + v2, e3 = d3 * kNeg2 + v3;
                const int ea = three ? e2 : two ? e1 : e0;
                const int eb = three ? e3 : two ? e2 : e1;
                t += min(ea, eb);
            }
        } else {
            const int d0 = ar * P.r0 + ag * P.g0 + ab * P.b0, d1 = ar * P.r1 + ag * P.g1 + ab * P.b1;
            const int d2 = ar * P.r2 + ag * P.g2 + ab * P.b2, d3 = ar * P.r3 + ag * P.g3 + ab * P.b3;
            const int t0 = d0 + d1, t1 = d1 + d2, t2 = d2 + d3;
            const int h0 = t0 >> 1, h1 = (t1 - 1) >> 1, h2 = (t2 - 1) >> 1;  // floor division
#pragma unroll 4
            for (int i = 0; i < 16; i++) {
                const uint32_t u = px(i);
                const int p0 = (int)__dp4a(u, c0, 0u), p1 = (int)__dp4a(u, c1, 0u);
                const int p2 = (int)__dp4a(u, c2, 0u), p3 = (int)__dp4a(u, c3, 0u);
                const int pd = p0 * kNeg1 + p3;
                const int s = 3 - ((pd <= h0) + (pd <= h1) + (pd <= h2));
                const int q0 = p0 * kNeg2 + v0, q1 = p1 * kNeg2 + v1, q2 = p2 * kNeg2 + v2, q3 = p3 * kNeg2 + v3;
                t += s == 0 ? q0 : s == 1 ? q1 : s == 2 ? q2 : q3;
            }
        }
        return (uint32_t)(pp_sum + t);
    }
    return find_selectors<IT, K>(lo, hi).y;
}

// FindEndpointsSingleColor(result, pixels, color, is_3color) (BC1Encoder.cpp:458-471)
template <int IT> __device__ __forceinline__ R single_color_body(int stale_lo, int stale_hi, int ar, int ag, int ab, bool is3) {
    const Pal P = make_pal<IT>(stale_lo, stale_hi, is3);  // colors[2] is internal index 1
    // sum over texels of |p - c|^2 in RGBA with c = (colors[2], 255), as
    // sum |p|^2 - 2 sum p.c + 16 |c|^2 (exact in integers): two dp4a per texel
    const uint32_t c = (uint32_t)P.r1 | ((uint32_t)P.g1 << 8) | ((uint32_t)P.b1 << 16) | 0xFF000000u;
    uint32_t pp = 0, pc = 0;
#pragma unroll 4
    for (int i = 0; i < 16; i++) {
        const uint32_t v = px(i);
        pp = __dp4a(v, v, pp);
        pc = __dp4a(v, c, pc);
    }
    const uint32_t e = pp - 2u * pc + 16u * __dp4a(c, c, 0u);
    const uint32_t mr = g_tab.match5[IT][ar], mg = g_tab.match6[IT][ag], mb = g_tab.match5[IT][ab];
    R r;
    r.lo = eppack((mr >> 8) & 0xFF, (mg >> 8) & 0xFF, (mb >> 8) & 0xFF);
    r.hi = eppack(mr & 0xFF, mg & 0xFF, mb & 0xFF);
    r.err = e;
    r.sel = 0x55555555u;
    r.mode = is3 ? CM_THREE : CM_FOUR;
    return r;
}

template <int IT> __device__ __noinline__ R single_color(int stale_lo, int stale_hi, int ar, int ag, int ab, bool is3) {
    return single_color_body<IT>(stale_lo, stale_hi, ar, ag, ab, is3);
}
template <int IT, bool INL>
__device__ __forceinline__ R single_color_(int stale_lo, int stale_hi, int ar, int ag, int ab, bool is3) {
    if constexpr (INL) return single_color_body<IT>(stale_lo, stale_hi, ar, ag, ab, is3);
    else return single_color<IT>(stale_lo, stale_hi, ar, ag, ab, is3);
}

// FindEndpoints (BC1Encoder.cpp:473-677)
__device__ __forceinline__ int2 find_endpoints_body(const M &m, int mode, bool ignore_black, int power_iters) {
    int lo, hi;
    if (m.grey) {
        const int fr = cr(px(0));
        if (m.mx[0] - m.mn[0] < 2) {
            lo = hi = eppack(s8to5(fr), s8to6(fr), s8to5(fr));
        } else {
            lo = eppack(s8to5(m.mn[0]), s8to6(m.mn[0]), s8to5(m.mn[0]));
            hi = eppack(s8to5(m.mx[0]), s8to6(m.mx[0]), s8to5(m.mx[0]));
        }
    } else if (mode == EP_LS) {
        const int d0 = m.mx[0] - m.mn[0], d1 = m.mx[1] - m.mn[1], d2 = m.mx[2] - m.mn[2];
        const int c0 = (d0 >= d1 && d0 >= d2) ? 0 : ((d1 >= d2 && d1 >= d0) ? 1 : 2);
        unsigned sxy0 = 0, sxy1 = 0, sxy2 = 0;  // zero-initialised (:510 is not)
        for (int i = 0; i < 16; i++) {
            const uint32_t v = px(i);
            const int p0 = c0 == 0 ? cr(v) : (c0 == 1 ? cg(v) : cb(v));
            sxy0 += (unsigned)(p0 * cr(v));
            sxy1 += (unsigned)(p0 * cg(v));
            sxy2 += (unsigned)(p0 * cb(v));
        }
        const unsigned sxy[3] = {sxy0, sxy1, sxy2};
        float l[3] = {0.f, 0.f, 0.f}, h[3] = {0.f, 0.f, 0.f};
        const float mn0 = (float)m.mn[c0];
        l[c0] = h[c0] = mn0;
        const unsigned sum_x = (unsigned)m.sum[c0], sum_xx = sxy[c0];
        const float den = __fsub_rn(__uint2float_rn(16u * sum_xx), __uint2float_rn(sum_x * sum_x));
        if (fabsf(den) > 1e-8f) {
            for (int i = 1; i < 3; i++) {
                const int c = (c0 + i) % 3;
                const unsigned sum_y = (unsigned)m.sum[c], sum_xy = sxy[c];
                const float a = __fdiv_rn(__uint2float_rn((16u * sum_xy) - (sum_x * sum_y)), den);
                const float b = __fdiv_rn(__uint2float_rn((sum_xx * sum_y) - (sum_xy * sum_x)), den);
                l[c] = __fadd_rn(b, __fmul_rn(a, l[c0]));
                h[c] = __fadd_rn(b, __fmul_rn(a, h[c0]));
            }
        }
        for (int c = 0; c < 3; c++) {
            const float inset = __fdiv_rn(__fsub_rn(h[c], l[c]), 16.0f);
            l[c] = __fdiv_rn(__fadd_rn(l[c], inset), 255.0f);
            h[c] = __fdiv_rn(__fsub_rn(h[c], inset), 255.0f);
        }
        lo = precise_round565(l[0], l[1], l[2], s_mid5, s_mid6);
        hi = precise_round565(h[0], h[1], h[2], s_mid5, s_mid6);
    } else if (mode == EP_BB || mode == EP_BBINT) {
        // sum over the 16 texels of (b - avg.b) * r - avg.r and (b - avg.b) * g - avg.g, as written
        // (:572-573), from raw moments: sum br - avg.b sum r - 16 avg.r (exact in integers)
        uint32_t rb = 0, gb = 0;
#pragma unroll
        for (int i = 0; i < 16; i += 4) {
            uint32_t R, G, B;
            channel_words(i, R, G, B);
            rb = __dp4a(R, B, rb);
            gb = __dp4a(G, B, gb);
        }
        const int cxz = (int)rb - m.av[2] * m.sum[0] - 16 * m.av[0];
        const int cyz = (int)gb - m.av[2] * m.sum[1] - 16 * m.av[1];
        if (mode == EP_BB) {
            const float bias = __fdiv_rn(8.0f, 255.0f);
            float l[3], h[3];
            for (int c = 0; c < 3; c++) {
                l[c] = __fdiv_rn((float)m.mn[c], 255.0f);
                h[c] = __fdiv_rn((float)m.mx[c], 255.0f);
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
            for (int c = 0; c < 3; c++) {
                const int inset = ((m.mx[c] - m.mn[c]) - 8) >> 4;
                a[c] = clamp255(m.mn[c] + inset);
                z[c] = clamp255(m.mx[c] - inset);
            }
            if (cxz < 0) { const int t = a[0]; a[0] = z[0]; z[0] = t; }
            if (cyz < 0) { const int t = a[1]; a[1] = z[1]; z[1] = t; }
            lo = eppack(s8to5(a[0]), s8to6(a[1]), s8to5(a[2]));
            hi = eppack(s8to5(z[0]), s8to6(z[1]), s8to5(z[2]));
        }
    } else {  // PCA
        int s00 = 0, s01 = 0, s02 = 0, s11 = 0, s12 = 0, s22 = 0;
        if (ignore_black) {
            for (int i = 0; i < 16; i++) {
                const uint32_t v = px(i);
                if (black(v)) continue;
                const int dr = cr(v) - m.av[0], dg = cg(v) - m.av[1], db = cb(v) - m.av[2];
                s00 += dr * dr; s01 += dr * dg; s02 += dr * db; s11 += dg * dg; s12 += dg * db; s22 += db * db;
            }
        } else {
            // the same sums over all 16 texels from raw moments, exactly in integers:
            // sum (x - a)(y - b) = sum xy - b sum x - a sum y + 16 a b. The raw moments come four
            // texels at a time: one word per channel of four texels' bytes, one dp4a per product.
            uint32_t rr = 0, rg = 0, rb = 0, gg = 0, gb = 0, bb = 0;
#pragma unroll
            for (int i = 0; i < 16; i += 4) {
                uint32_t R, G, B;
                channel_words(i, R, G, B);
                rr = __dp4a(R, R, rr); rg = __dp4a(R, G, rg); rb = __dp4a(R, B, rb);
                gg = __dp4a(G, G, gg); gb = __dp4a(G, B, gb); bb = __dp4a(B, B, bb);
            }
            const int a0 = m.av[0], a1 = m.av[1], a2 = m.av[2], S0 = m.sum[0], S1 = m.sum[1], S2 = m.sum[2];
            s00 = (int)rr - 2 * a0 * S0 + 16 * a0 * a0;
            s01 = (int)rg - a1 * S0 - a0 * S1 + 16 * a0 * a1;
            s02 = (int)rb - a2 * S0 - a0 * S2 + 16 * a0 * a2;
            s11 = (int)gg - 2 * a1 * S1 + 16 * a1 * a1;
            s12 = (int)gb - a2 * S1 - a1 * S2 + 16 * a1 * a2;
            s22 = (int)bb - 2 * a2 * S2 + 16 * a2 * a2;
        }
        const float k255 = 255.0f;
        const float c00 = __fdiv_rn((float)(1 + s00), k255), c01 = __fdiv_rn((float)s01, k255);
        const float c02 = __fdiv_rn((float)s02, k255), c11 = __fdiv_rn((float)(1 + s11), k255);
        const float c12 = __fdiv_rn((float)s12, k255), c22 = __fdiv_rn((float)(1 + s22), k255);
        const float c33 = __fdiv_rn(1.0f, k255), z = __fdiv_rn(0.0f, k255);
        float d0 = __fsub_rn((float)m.mx[0], (float)m.mn[0]);
        float d1 = __fsub_rn((float)m.mx[1], (float)m.mn[1]);
        float d2 = __fsub_rn((float)m.mx[2], (float)m.mn[2]);
        float d3 = __fsub_rn(0.0f, 0.0f);
        if (c02 < 0) d0 = -d0;
        if (c12 < 0) d1 = -d1;
        for (int it = 0; it < power_iters; it++) {
            const float n0 = fdot4_rn(d0, d1, d2, d3, c00, c01, c02, z);
            const float n1 = fdot4_rn(d0, d1, d2, d3, c01, c11, c12, z);
            const float n2 = fdot4_rn(d0, d1, d2, d3, c02, c12, c22, z);
            const float n3 = fdot4_rn(d0, d1, d2, d3, z, z, z, c33);
            d0 = n0; d1 = n1; d2 = n2; d3 = n3;
        }
        float k = 0.0f;
        if (fabsf(d0) > k) k = fabsf(d0);
        if (fabsf(d1) > k) k = fabsf(d1);
        if (fabsf(d2) > k) k = fabsf(d2);
        float a0 = 306.0f, a1 = 601.0f, a2 = 117.0f, a3 = 0.0f;
        if (k >= 2) {
            const float s = __fdiv_rn(2048.0f, k);
            a0 = __fmul_rn(d0, s); a1 = __fmul_rn(d1, s); a2 = __fmul_rn(d2, s); a3 = __fmul_rn(d3, s);
        }
        a0 = __fmul_rn(a0, 16.0f); a1 = __fmul_rn(a1, 16.0f); a2 = __fmul_rn(a2, 16.0f); a3 = __fmul_rn(a3, 16.0f);
        float min_dot = INFINITY, max_dot = -INFINITY;
        int min_i = 0, max_i = 0;
        for (int i = 0; i < 16; i++) {
            const uint32_t v = px(i);
            if (ignore_black && black(v)) continue;
            const float dot = fdot4_rn((float)cr(v), (float)cg(v), (float)cb(v), 0.0f, a0, a1, a2, a3);
            if (dot > max_dot) { max_dot = dot; max_i = i; }
            if (dot < min_dot) { min_dot = dot; min_i = i; }
        }
        const uint32_t pmin = px(min_i), pmax = px(max_i);
        lo = eppack(s8to5(cr(pmin)), s8to6(cg(pmin)), s8to5(cb(pmin)));
        hi = eppack(s8to5(cr(pmax)), s8to6(cg(pmax)), s8to5(cb(pmax)));
    }
    return make_int2(lo, hi);
}

__device__ __noinline__ int2 find_endpoints(const M &m, int mode, bool ignore_black, int power_iters) {
    return find_endpoints_body(m, mode, ignore_black, power_iters);
}
template <bool INL> __device__ __forceinline__ int2 find_endpoints_(const M &m, int mode, bool ignore_black, int power_iters) {
    if constexpr (INL) return find_endpoints_body(m, mode, ignore_black, power_iters);
    else return find_endpoints(m, mode, ignore_black, power_iters);
}

// RefineBlockLS<M> with RefineEndpointsLS<FourColor>(pixels) (BC1Encoder.cpp:781-825, 852-875)
template <int IT, int K, bool INL> __device__ __forceinline__ R refine_ls_body(R r, const M &m, int passes) {
    for (int pass = 0; pass < passes; pass++) {
        R t = r;
        // sum of selector x colour per channel, two channels per word (r | b << 16, g | a << 16:
        // at most 16 x 3 x 255 = 12240 per half, no carry), and the selector histogram by popcount
        uint32_t acc_rb = 0, acc_ga = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            const uint32_t v = px(i), s = (t.sel >> (2 * i)) & 3u;
            acc_rb = s * (v & 0x00FF00FFu) + acc_rb;
            acc_ga = s * ((v >> 8) & 0x00FF00FFu) + acc_ga;
        }
        const int q0r = (int)(acc_rb & 0xFFFFu), q0g = (int)(acc_ga & 0xFFFFu), q0b = (int)(acc_rb >> 16);
        const uint32_t w = t.sel;
        const int n1 = __popc(w & ~(w >> 1) & 0x55555555u), n2 = __popc(~w & (w >> 1) & 0x55555555u);
        const int n3 = __popc(w & (w >> 1) & 0x55555555u);
        const int n0 = 16 - n1 - n2 - n3;
        float m0 = (float)(n1 + 4 * n2 + 9 * n3), m1 = (float)(2 * n1 + 2 * n2), m2 = m1, m3 = (float)(9 * n0 + 4 * n1 + n2);
        const float det = __fsub_rn(__fmul_rn(m0, m3), __fmul_rn(m1, m2));
        if (fabsf(det) < 1e-8f) {
            t = single_color_<IT, INL>(t.lo, t.hi, m.av[0], m.av[1], m.av[2], kind_three(K));
        } else {
            const float tt = m0; m0 = m3; m3 = tt;
            m1 = -m1;
            m2 = -m2;
            const float sc = __fdiv_rn(__fdiv_rn(3.0f, 255.0f), det);
            m0 = __fmul_rn(m0, sc); m1 = __fmul_rn(m1, sc); m2 = __fmul_rn(m2, sc); m3 = __fmul_rn(m3, sc);
            const float f0r = (float)q0r, f0g = (float)q0g, f0b = (float)q0b;
            const float q10r = (float)(m.sum[0] * 3) - f0r, q10g = (float)(m.sum[1] * 3) - f0g, q10b = (float)(m.sum[2] * 3) - f0b;
            t.lo = precise_round565(__fadd_rn(__fmul_rn(m0, f0r), __fmul_rn(m1, q10r)),
                                    __fadd_rn(__fmul_rn(m0, f0g), __fmul_rn(m1, q10g)),
                                    __fadd_rn(__fmul_rn(m0, f0b), __fmul_rn(m1, q10b)), s_mid5, s_mid6);
            t.hi = precise_round565(__fadd_rn(__fmul_rn(m2, f0r), __fmul_rn(m3, q10r)),
                                    __fadd_rn(__fmul_rn(m2, f0g), __fmul_rn(m3, q10g)),
                                    __fadd_rn(__fmul_rn(m2, f0b), __fmul_rn(m3, q10b)), s_mid5, s_mid6);
            const uint2 se = find_selectors_<IT, K, INL>(t.lo, t.hi);
            t.sel = se.x;
            t.err = se.y;
            t.mode = kind_mode(K);
        }
        if (t.lo == r.lo && t.hi == r.hi) break;
        if (K == K_F4_NONE || t.err < r.err) r = t;
        else break;
    }
    return r;
}

template <int IT, int K> __device__ __noinline__ R refine_ls(R r, const M &m, int passes) {
    return refine_ls_body<IT, K, false>(r, m, passes);
}
template <int IT, int K, bool INL> __device__ __forceinline__ R refine_ls_(R r, const M &m, int passes) {
    if constexpr (INL) return refine_ls_body<IT, K, true>(r, m, passes);
    else return refine_ls<IT, K>(r, m, passes);
}

template <int IT> __device__ __forceinline__ R refine_ls_any(int K, R r, const M &m, int passes) {
    switch (K) {
        case K_F4_NONE: return refine_ls<IT, K_F4_NONE>(r, m, passes);
        case K_F4_FASTER: return refine_ls<IT, K_F4_FASTER>(r, m, passes);
        case K_F4_CHECK2: return refine_ls<IT, K_F4_CHECK2>(r, m, passes);
        case K_F4_FULL: return refine_ls<IT, K_F4_FULL>(r, m, passes);
        case K_T3: return refine_ls<IT, K_T3>(r, m, passes);
        default: return refine_ls<IT, K_TB>(r, m, passes);
    }
}

// Ascending sort of 16 keys in registers: Batcher's odd-even merge network (63
// compare-exchanges, each an unsigned min and max).
__device__ __forceinline__ void sort16(uint32_t k[16]) {
    constexpr int kNet[63][2] = {{0, 1}, {2, 3}, {0, 2}, {1, 3}, {1, 2}, {4, 5}, {6, 7}, {4, 6}, {5, 7}, {5, 6}, {0, 4}, {2, 6}, {2, 4}, {1, 5}, {3, 7}, {3, 5}, {1, 2}, {3, 4}, {5, 6}, {8, 9}, {10, 11}, {8, 10}, {9, 11}, {9, 10}, {12, 13}, {14, 15}, {12, 14}, {13, 15}, {13, 14}, {8, 12}, {10, 14}, {10, 12}, {9, 13}, {11, 15}, {11, 13}, {9, 10}, {11, 12}, {13, 14}, {0, 8}, {4, 12}, {4, 8}, {2, 10}, {6, 14}, {6, 10}, {2, 4}, {6, 8}, {10, 12}, {1, 9}, {5, 13}, {5, 9}, {3, 11}, {7, 15}, {7, 11}, {3, 5}, {7, 9}, {11, 13}, {1, 2}, {3, 4}, {5, 6}, {7, 8}, {9, 10}, {11, 12}, {13, 14}};
#pragma unroll
    for (int c = 0; c < 63; c++) {
        const uint32_t a = k[kNet[c][0]], b = k[kNet[c][1]];
        k[kNet[c][0]] = min(a, b);
        k[kNet[c][1]] = max(a, b);
    }
}

// OrderTable::GetHash of the selectors' histogram (OrderTable.h:91-104), the first
// ordering of RefineBlockCF (BC1Encoder.cpp:886-889)
__device__ __forceinline__ int cf_start_hash(bool four, uint32_t w) {
    const int n1 = __popc(w & ~(w >> 1) & 0x55555555u), n2 = __popc(~w & (w >> 1) & 0x55555555u);
    const int n3 = __popc(w & (w >> 1) & 0x55555555u), n0 = 16 - n1 - n2 - n3;
    if (four) return n0 == 16 ? 15 : n1 == 16 ? 700 : n2 == 16 ? 753 : n3 == 16 ? 515 : (int)g_tab.hash4[n0 | (n1 << 4) | (n2 << 8)];
    return n0 == 16 ? 12 : n1 == 16 ? 15 : n2 == 16 ? 89 : (int)g_tab.hash3[n0 | (n1 << 4)];
}

// RefineBlockCF's sort key of texel i (BC1Encoder.cpp:895-900): its dot with the axis, then i
__device__ __forceinline__ uint32_t cf_key(uint32_t v, int axr, int axg, int axb, int i) {
    return ((uint32_t)(0x1000000 + cr(v) * axr + cg(v) * axg + cb(v) * axb) << 4) | (uint32_t)i;
}

// RefineBlockCF's trials (BC1Encoder.cpp:905-927) depend on its input only through the
// start hash (the histogram of the input selectors) and the texel order along the input's
// axis; its single-colour trial depends on neither. A second pass whose input gives the
// same hash and order as the first pass's input runs the same trials against a best error
// that is already the minimum of them, so it changes nothing. True when r (the first
// pass's result) gives start hash `start` and texel order `order` (rank k -> texel in
// nibble k).
__device__ __forceinline__ bool cf_same_trials(bool four, const R &r, int start, uint64_t order) {
    if (cf_start_hash(four, r.sel) != start) return false;
    const int axr = s5to8(epr(r.hi)) - s5to8(epr(r.lo));
    const int axg = s6to8(epg(r.hi)) - s6to8(epg(r.lo));
    const int axb = s5to8(epb(r.hi)) - s5to8(epb(r.lo));
    // the keys under r's axis, read in the first pass's order, must still increase
    int i = (int)(order & 0xF);
    uint32_t prev = cf_key(px(i), axr, axg, axb, i);
    bool same = true;
#pragma unroll 4
    for (int k = 1; k < 16; k++) {
        i = (int)((order >> (4 * k)) & 0xF);
        const uint32_t key = cf_key(px(i), axr, axg, axb, i);
        same &= prev < key;
        prev = key;
    }
    return same;
}

// RefineBlockCF<M> (BC1Encoder.cpp:877-928): the reference's loop as written. With ORDER,
// *order_out receives the texel order of the input (rank k -> texel in nibble k).
template <int IT, int K, bool ORDER, bool INL>
__device__ __forceinline__ R refine_cf_body(R r, const M &m, unsigned orderings, bool exhaustive, int pp_sum, uint64_t *order_out) {
    constexpr bool four = !kind_three(K);
    const int tid = threadIdx.x;
    const R orig = r;
    const int start = cf_start_hash(four, orig.sel);
    // projection keys, rank by counting (keys are distinct), prefix sums in rank order
    const int axr = s5to8(epr(orig.hi)) - s5to8(epr(orig.lo));
    const int axg = s6to8(epg(orig.hi)) - s6to8(epg(orig.lo));
    const int axb = s5to8(epb(orig.hi)) - s5to8(epb(orig.lo));
    uint32_t key[16];
#pragma unroll
    for (int i = 0; i < 16; i++) key[i] = cf_key(px(i), axr, axg, axb, i);
    sort16(key);  // the keys are distinct, so this is the reference's std::sort order
    uint64_t order = 0;
    uint32_t arg = 0, ab = 0;
    t_srg[0][tid] = 0;
    t_sb[0][tid] = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {  // prefix sums of the colours in rank order
        const int i = (int)(key[k] & 15);
        const uint32_t v = px(i);
        arg += (uint32_t)cr(v) | ((uint32_t)cg(v) << 16);
        ab += (uint32_t)cb(v);
        t_srg[k + 1][tid] = arg;
        t_sb[k + 1][tid] = (uint16_t)ab;
        if (ORDER) order |= (uint64_t)i << (4 * k);
    }
    if (ORDER) *order_out = order;
    const float t16r = (float)(arg & 0xFFFF), t16g = (float)(arg >> 16), t16b = (float)ab;
    const float denom = four ? 3.0f : 2.0f;
    const unsigned total = exhaustive ? (four ? 969u : 153u) : orderings;
    const uint16_t *row = four ? g_tab.best4 + start * 128 : g_tab.best3 + start * 32;
    bool sc_done = false, from_ls = false;
    R sc;
    for (unsigned q = 0; q < total; q++) {
        // BestOrders entries carry bit 15 for the single-colour orderings
        const int raw = exhaustive ? (int)q : (int)row[q], th = raw & 0x7FFF;
        const bool single = exhaustive ? is_single_hash(four, th) : raw >= 0x8000;
        R t;
        if (single) {
            if (!sc_done) {  // the same trial for every single-colour ordering of this call
                sc = single_color_<IT, INL>(orig.lo, orig.hi, m.av[0], m.av[1], m.av[2], !four);
                sc.mode = kind_mode(K);
                sc_done = true;
            }
            t = sc;
        } else {
            const float4 f = four ? g_tab.factors4[th] : g_tab.factors3[th];
            const uint32_t o = four ? g_tab.orders4[th] : g_tab.orders3[th];
            const int l1 = o & 0xFF, l2 = l1 + ((o >> 8) & 0xFF), l3 = l2 + ((o >> 16) & 0xFF);
            uint32_t qrg = t_srg[l1][tid] + t_srg[l2][tid], qb = (uint32_t)t_sb[l1][tid] + t_sb[l2][tid];
            if (four) {
                qrg += t_srg[l3][tid];
                qb += t_sb[l3][tid];
            }
            const float fr = (float)(qrg & 0xFFFF), fg = (float)(qrg >> 16), fb = (float)qb;
            // integers below 2^24 (sums of at most 3 x 16 x 255): exact whether fused or not, so one FMA
            const float q0r = __fmaf_rn(t16r, denom, -fr), q0g = __fmaf_rn(t16g, denom, -fg), q0b = __fmaf_rn(t16b, denom, -fb);
            t.lo = precise_round565_cf(__fadd_rn(__fmul_rn(f.x, q0r), __fmul_rn(f.y, fr)),
                                    __fadd_rn(__fmul_rn(f.x, q0g), __fmul_rn(f.y, fg)),
                                    __fadd_rn(__fmul_rn(f.x, q0b), __fmul_rn(f.y, fb)), s_mid5, s_mid6);
            t.hi = precise_round565_cf(__fadd_rn(__fmul_rn(f.z, q0r), __fmul_rn(f.w, fr)),
                                    __fadd_rn(__fmul_rn(f.z, q0g), __fmul_rn(f.w, fg)),
                                    __fadd_rn(__fmul_rn(f.z, q0b), __fmul_rn(f.w, fb)), s_mid5, s_mid6);
            t.err = block_error<IT, K>(t.lo, t.hi, pp_sum);
            t.sel = 0;  // filled for the winner below
            t.mode = kind_mode(K);
        }
        if (t.err < r.err) {
            r = t;
            from_ls = !single;
        }
        if (t.err == 0) break;
    }
    if (from_ls) r.sel = find_selectors_<IT, K, INL>(r.lo, r.hi).x;  // selectors of the winning LS trial
    return r;
}

template <int IT, int K, bool ORDER = false>
__device__ __noinline__ R refine_cf(R r, const M &m, unsigned orderings, bool exhaustive, int pp_sum, uint64_t *order_out = nullptr) {
    return refine_cf_body<IT, K, ORDER, false>(r, m, orderings, exhaustive, pp_sum, order_out);
}
template <int IT, int K, bool INL>
__device__ __forceinline__ R refine_cf_(R r, const M &m, unsigned orderings, bool exhaustive, int pp_sum) {
    if constexpr (INL) return refine_cf_body<IT, K, false, true>(r, m, orderings, exhaustive, pp_sum, nullptr);
    else return refine_cf<IT, K>(r, m, orderings, exhaustive, pp_sum);
}

// EndpointSearch (BC1Encoder.cpp:930-996): the reference's sequential loop
template <int IT, int K> __device__ __noinline__ R endpoint_search(R r, unsigned rounds, int pp_sum) {
    unsigned prev = 0;
    int forbidden = -1;
    bool moved = false;
    for (unsigned i = 0; i < rounds; i++) {
        if ((int)(i & 31) == forbidden) continue;
        const uint16_t vx = s_vox[i & 15];
        const int ddr = ((int)((unsigned)vx << 30)) >> 30, ddg = ((int)((unsigned)vx << 28)) >> 30;
        const int ddb = ((int)((unsigned)vx << 26)) >> 30;
        int lo = r.lo, hi = r.hi;
        if (i & 16) lo = eppack(clampi(epr(lo) + ddr, 0, 31), clampi(epg(lo) + ddg, 0, 63), clampi(epb(lo) + ddb, 0, 31));
        else hi = eppack(clampi(epr(hi) + ddr, 0, 31), clampi(epg(hi) + ddg, 0, 63), clampi(epb(hi) + ddb, 0, 31));
        const uint32_t e = block_error<IT, K>(lo, hi, pp_sum);
        if (e < r.err) {
            r.lo = lo;
            r.hi = hi;
            r.err = e;
            forbidden = (int)((vx >> 8) & 15) | (int)(i & 16);
            prev = i;
            moved = true;
        }
        if (i - prev > 32) break;
    }
    if (moved) r.sel = find_selectors<IT, K>(r.lo, r.hi).x;
    return r;
}

template <int IT, bool ORDER = false>
__device__ __forceinline__ R refine_cf_any(int K, R r, const M &m, unsigned o, bool ex, int pp, uint64_t *order = nullptr) {
    switch (K) {
        case K_F4_NONE: return refine_cf<IT, K_F4_NONE, ORDER>(r, m, o, ex, pp, order);
        case K_F4_FASTER: return refine_cf<IT, K_F4_FASTER, ORDER>(r, m, o, ex, pp, order);
        case K_F4_CHECK2: return refine_cf<IT, K_F4_CHECK2, ORDER>(r, m, o, ex, pp, order);
        case K_F4_FULL: return refine_cf<IT, K_F4_FULL, ORDER>(r, m, o, ex, pp, order);
        default: return refine_cf<IT, K_T3, ORDER>(r, m, o, ex, pp, order);
    }
}

template <int IT> __device__ __forceinline__ R search_any(int K, R r, unsigned rounds, int pp) {
    switch (K) {
        case K_F4_NONE: return endpoint_search<IT, K_F4_NONE>(r, rounds, pp);
        case K_F4_FASTER: return endpoint_search<IT, K_F4_FASTER>(r, rounds, pp);
        case K_F4_CHECK2: return endpoint_search<IT, K_F4_CHECK2>(r, rounds, pp);
        case K_F4_FULL: return endpoint_search<IT, K_F4_FULL>(r, rounds, pp);
        case K_T3: return endpoint_search<IT, K_T3>(r, rounds, pp);
        default: return endpoint_search<IT, K_TB>(r, rounds, pp);
    }
}

__device__ __forceinline__ uint2 write(const R &r) { return write_block(r.lo, r.hi, r.sel, r.mode); }

// A block whose remaining work runs later in a pass of its own: its result so far.
// need: EndpointSearch, in k_bc1_search; queue is the search queue of its colour mode
// (0 four-colour, 1 three-colour, 2 three-colour + black).
// cf2: the rest of EncodeBlock after the first four-colour cluster-fit pass, in k_bc1_cf2:
// the second pass when pass2, then the 3-colour trials; orig holds the endpoints the
// 3-colour trial starts from.
struct Deferred {
    bool need, cf2, pass2;
    int queue;
    R r, orig;
};

// EncodeBlock from the 3-colour trials on (BC1Encoder.cpp:305-341): res is the
// four-colour result after its cluster-fit passes, orig the endpoints before the
// four-colour refinement. With `d`, a block that needs EndpointSearch stops before it
// and is returned in *d instead. INL inlines the phase bodies; without SEARCH the caller
// guarantees p.search_rounds == 0 and no search code is compiled in.
template <int IT, bool INL = false, bool SEARCH = true>
__device__ __forceinline__ uint2 encode_tail(const qt_bc1_params &p, int color_mode, int pp_sum, const M &m, R res,
                                             const R &orig, Deferred *d) {
    const bool use_likely = p.exhaustive || p.orderings3 > 0 || p.orderings4 > 0;
    const int ls_passes = p.two_ls_passes ? 2 : 1, cf_passes = p.two_cf_passes ? 2 : 1;
    if (res.err > 0 && (color_mode & CM_THREE)) {
        R t = orig;
        const uint2 se = find_selectors_<IT, K_T3, INL>(t.lo, t.hi);
        t.sel = se.x;
        t.err = se.y;
        t.mode = CM_THREE;
        t = refine_ls_<IT, K_T3, INL>(t, m, ls_passes);
        if (t.err > 0 && use_likely)
            for (int it = 0; it < cf_passes; it++) t = refine_cf_<IT, K_T3, INL>(t, m, p.orderings3, p.exhaustive, pp_sum);
        if (t.err < res.err) res = t;
    }

    if (res.err > 0 && color_mode == CM_TB && m.has_black && !((m.mx[0] | m.mx[1] | m.mx[2]) < 4)) {
        const M mnb = metrics_<INL>(true);
        const int2 ep = find_endpoints_<INL>(mnb, EP_PCA, true, (int)p.power_iterations);
        R t = rinit();
        t.lo = ep.x;
        t.hi = ep.y;
        const uint2 se = find_selectors_<IT, K_TB, INL>(t.lo, t.hi);
        t.sel = se.x;
        t.err = se.y;
        t.mode = CM_TB;
        t = refine_ls_<IT, K_TB, INL>(t, mnb, ls_passes);
        if (t.err < res.err) res = t;
    }

    if (SEARCH && res.err > 0 && p.search_rounds > 0) {
        const int Md = res.mode == CM_THREE ? CM_THREE : (res.mode == CM_TB ? CM_TB : CM_FOUR);
        if (d) {
            d->need = true;
            d->queue = Md == CM_FOUR ? 0 : (Md == CM_THREE ? 1 : 2);
            d->r = res;
            return make_uint2(0u, 0u);
        }
        if constexpr (SEARCH)
            res = search_any<IT>(kind_for(Md, Md == CM_FOUR ? p.error_mode : EM_FULL), res, p.search_rounds, pp_sum);
    }
    return write(res);
}

// BC1Encoder::EncodeBlock (BC1Encoder.cpp:261-342), one thread. With `d`, a block that
// needs EndpointSearch stops before it, and at settings with two four-colour cluster-fit
// passes a block stops after the first when the second can change its result or when the
// 3-colour trials follow; either is returned in *d instead.
// Specialised form (k_bc1_fast): K4 >= 0 fixes the four-colour selector kind at compile time
// (the caller guarantees kind_for(CM_FOUR, p.error_mode) == K4 and, without SEARCH,
// p.search_rounds == 0); INL inlines every phase body; `d` must then be null.
template <int IT, int K4 = -1, bool INL = false, bool SEARCH = true>
__device__ __forceinline__ uint2 encode_block(const qt_bc1_params &p, int color_mode, int pp_sum, Deferred *d = nullptr) {
    const uint32_t c0 = px(0);
    bool solid = true;
    for (int i = 1; i < 16; i++) solid &= px(i) == c0;
    if (solid) return write_block_solid<IT>(c0);

    const M m = metrics_<INL>(false);
    const bool use_likely = p.exhaustive || p.orderings3 > 0 || p.orderings4 > 0;
    bool needs_err = use_likely;
    needs_err |= color_mode == CM_THREE;
    needs_err |= (color_mode == CM_TB) && m.has_black;
    needs_err |= p.error_mode != EM_NONE;
    needs_err |= p.search_rounds > 0;
    const int em = needs_err ? p.error_mode : EM_NONE;
    const int ls_passes = p.two_ls_passes ? 2 : 1, cf_passes = p.two_cf_passes ? 2 : 1;
    const int ep_passes = (needs_err && p.two_ep_passes) ? 2 : 1;
    const int k4 = kind_for(CM_FOUR, em);

    R orig = rinit(), res = rinit();
    for (int round = 0; round < ep_passes; round++) {
        const int2 ep = find_endpoints_<INL>(m, round == 1 ? EP_BB : p.endpoint_mode, false, (int)p.power_iterations);
        R to = rinit();
        to.lo = ep.x;
        to.hi = ep.y;
        R tr = to;
        uint2 se;
        if constexpr (K4 >= 0) se = find_selectors_<IT, K4, INL>(tr.lo, tr.hi);
        else se = fs_any<IT>(k4, tr.lo, tr.hi);
        tr.sel = se.x;
        tr.err = se.y;
        tr.mode = CM_FOUR;
        if constexpr (K4 >= 0) tr = refine_ls_<IT, K4, INL>(tr, m, ls_passes);
        else tr = refine_ls_any<IT>(k4, tr, m, ls_passes);
        if (!needs_err || tr.err < res.err) {
            res = tr;
            orig = to;
        }
    }
    if constexpr (K4 >= 0) {
        if (res.err > 0 && use_likely)
            for (int it = 0; it < cf_passes; it++) res = refine_cf_<IT, K4, INL>(res, m, p.orderings4, p.exhaustive, pp_sum);
    } else if (res.err > 0 && use_likely) {
        const int kcf = kind_for(CM_FOUR, p.error_mode);
        if (d && cf_passes == 2) {
            const int start = cf_start_hash(true, res.sel);
            uint64_t order = 0;
            res = refine_cf_any<IT, true>(kcf, res, m, p.orderings4, p.exhaustive, pp_sum, &order);
            // a zero error cannot drop further; the same trials cannot beat their own minimum
            const bool pass2 = res.err > 0 && !cf_same_trials(true, res, start, order);
            if (pass2 || (res.err > 0 && (color_mode & CM_THREE))) {
                d->cf2 = true;
                d->pass2 = pass2;
                d->r = res;
                d->orig = orig;
                return make_uint2(0u, 0u);
            }
        } else {
            for (int it = 0; it < cf_passes; it++)
                res = refine_cf_any<IT>(kcf, res, m, p.orderings4, p.exhaustive, pp_sum);
        }
    }
    return encode_tail<IT, INL, SEARCH>(p, color_mode, pp_sum, m, res, orig, d);
}

}  // namespace tpb

// one block per thread; BC3 adds the BC4 alpha block on channel 3. With LIST the
// thread's blocks are list[i] for i < *count (the non-solid blocks that
// k_bc1_split left), so no lane of a warp idles on a solid block.
template <int IT, bool LIST>
__global__ void __launch_bounds__(tpb::kThreads, 4) k_bc1_thread(const uint8_t *__restrict__ rgba, int w, int h, int bw,
                                                                   long b_begin, long nblocks, qt_bc1_params p,
                                                                   uint8_t *__restrict__ out, int bc3, int aligned,
                                                                   const uint32_t *__restrict__ list,
                                                                   const uint32_t *__restrict__ count) {
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
        if (i < 32) s_mid5[i] = c_mid5[i];
        s_mid6[i] = c_mid6[i];
        if (i < 16) s_vox[i] = c_voxels[i];
    }
    __syncthreads();
    const int color_mode = bc3 ? CM_FOUR : p.color_mode;  // BC3Encoder.h:39-40
    const long end = LIST ? (long)*count : nblocks;
    for (long i = (LIST ? 0 : b_begin) + (long)blockIdx.x * blockDim.x + threadIdx.x; i < end;
         i += (long)gridDim.x * blockDim.x) {
        const long b = LIST ? (long)list[i] : i;
        const int by = (int)(b / bw), bx = (int)(b - (long)by * bw);
        uint32_t v[16];
        load_block_thread(rgba, w, h, bx, by, aligned && (bx * 4 + 4 <= w) && (by * 4 + 4 <= h), v);
        int pp = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            tpb::t_px[i][threadIdx.x] = v[i];
            const uint32_t u = v[i] & 0x00FFFFFFu;
            pp += (int)__dp4a(u, u, 0u);
        }
        const uint2 blk = tpb::encode_block<IT>(p, color_mode, pp);
        if (bc3) {
#pragma unroll
            for (int i = 0; i < 16; i++) v[i] = tpb::t_px[i][threadIdx.x];
            const uint2 a = bc4_block_thread(v, 3);
            reinterpret_cast<uint4 *>(out)[b] = make_uint4(a.x, a.y, blk.x, blk.y);
        } else {
            reinterpret_cast<uint2 *>(out)[b] = blk;
        }
    }
}

// The same for settings without EndpointSearch (levels 0-12), specialised: the four-colour
// selector kind K4 and the colour mode CM (CM_FOUR for BC3) fixed at compile time and every
// phase inlined, so a launch runs one straight-line path with no calls and no code for the
// other colour modes' trials. With `list`, the blocks are list[i] for i < *count; otherwise
// [b_begin, nblocks). The Faster-selector instance (levels 5-8) is held to 80 registers for 6
// CTAs per SM (measured +2-4% at level 5); the others keep 90-96 registers (5 CTAs), which
// level 10's three-colour trials need (-4% at 80).
template <int IT, int K4, int CM>
__global__ void __launch_bounds__(tpb::kThreads, K4 == K_F4_FASTER ? 6 : 4) k_bc1_fast(const uint8_t *__restrict__ rgba, int w, int h, int bw,
                                                                 long b_begin, long nblocks, qt_bc1_params p,
                                                                 uint8_t *__restrict__ out, int bc3, int aligned,
                                                                 const uint32_t *__restrict__ list,
                                                                 const uint32_t *__restrict__ count) {
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
        if (i < 32) s_mid5[i] = c_mid5[i];
        s_mid6[i] = c_mid6[i];
    }
    __syncthreads();
    constexpr int color_mode = CM;
    const bool listed = list != nullptr;
    const long end = listed ? (long)*count : nblocks;
    for (long i = (listed ? 0 : b_begin) + (long)blockIdx.x * blockDim.x + threadIdx.x; i < end;
         i += (long)gridDim.x * blockDim.x) {
        const long b = listed ? (long)list[i] : i;
        const int by = (int)(b / bw), bx = (int)(b - (long)by * bw);
        uint32_t v[16];
        load_block_thread(rgba, w, h, bx, by, aligned && (bx * 4 + 4 <= w) && (by * 4 + 4 <= h), v);
        int pp = 0;
#pragma unroll
        for (int k = 0; k < 16; k++) {
            tpb::t_px[k][threadIdx.x] = v[k];
            const uint32_t u = v[k] & 0x00FFFFFFu;
            pp += (int)__dp4a(u, u, 0u);
        }
        const uint2 blk = tpb::encode_block<IT, K4, true, false>(p, color_mode, pp);
        if (bc3) {
#pragma unroll
            for (int k = 0; k < 16; k++) v[k] = tpb::t_px[k][threadIdx.x];
            const uint2 a = bc4_block_thread(v, 3);
            reinterpret_cast<uint4 *>(out)[b] = make_uint4(a.x, a.y, blk.x, blk.y);
        } else {
            reinterpret_cast<uint2 *>(out)[b] = blk;
        }
    }
}

// Split pass: one thread per block of [b_begin, b_end). A solid block (all 16
// texels equal in RGBA, ColorBlock::IsSingleColor) is written here, as
// EncodeBlock's first step does (BC1Encoder.cpp:264-266, WriteBlockSolid, plus
// BC3's alpha); every other block's index is appended to list (warp-aggregated).
template <int IT>
__global__ void __launch_bounds__(256) k_bc1_split(const uint8_t *__restrict__ rgba, int w, int h, int bw, long b_begin,
                                                   long b_end, uint8_t *__restrict__ out, int bc3, int aligned,
                                                   uint32_t *__restrict__ list, uint32_t *__restrict__ count) {
    const int lane = threadIdx.x & 31;
    // every lane of a warp runs the same number of iterations, so the ballot sees whole warps
    const long stride = (long)gridDim.x * blockDim.x;
    const long first = b_begin + (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long base_warp = first - lane;
    for (long wb = base_warp; wb < b_end; wb += stride) {
        const long b = wb + lane;
        bool keep = false;
        if (b < b_end) {
            const int by = (int)(b / bw), bx = (int)(b - (long)by * bw);
            uint32_t v[16];
            load_block_thread(rgba, w, h, bx, by, aligned && (bx * 4 + 4 <= w) && (by * 4 + 4 <= h), v);
            bool solid = true;
#pragma unroll
            for (int i = 1; i < 16; i++) solid &= v[i] == v[0];
            if (solid) {
                const uint2 blk = write_block_solid<IT>(v[0]);
                if (bc3) {
                    const uint2 a = bc4_block_thread(v, 3);
                    reinterpret_cast<uint4 *>(out)[b] = make_uint4(a.x, a.y, blk.x, blk.y);
                } else {
                    reinterpret_cast<uint2 *>(out)[b] = blk;
                }
            }
            keep = !solid;
        }
        const uint32_t m = __ballot_sync(0xffffffffu, keep);
        uint32_t pos = 0;
        if (lane == 0 && m) pos = atomicAdd(count, (uint32_t)__popc(m));
        pos = __shfl_sync(0xffffffffu, pos, 0);
        if (keep) list[pos + __popc(m & ((1u << lane) - 1))] = (uint32_t)b;
    }
}

// ---------------------------------------------------------------------------
// EndpointSearch as a separate pass with lane refill. In the single-pass
// kernel a warp runs until the longest of its 32 searches stops (most stop
// after 33 rounds, a few run to 256), so most lanes idle through the search.
// Here the encoder (k_bc1_defer) queues the blocks that need the search, one
// queue per colour mode so that a warp runs one selector kind, and
// k_bc1_search runs one search round per step in every lane: a lane whose
// search has stopped writes its block and takes the next queued one.
// ---------------------------------------------------------------------------
// idle lanes a search warp gathers before it refills them (measured: 4 → +3.1%, 8-16 → +3.5%,
// 24 → +2.5% at level 18 over refilling every lane as soon as it is idle)
constexpr int kRefillBatch = 8;

struct SearchQueues {
    uint32_t *count;  // [3] entries per queue
    uint32_t *head;   // [3] next entry to take
    uint32_t *b, *lohi, *err, *sel, *mode;  // [3][cap] each
    long cap;
};

// Searches that moved the endpoints, finished by k_bc1_finish: the block, its final endpoints
// and colour mode. The reference keeps the selectors of the last accepted trial, which
// FindSelectors computed from those endpoints (BC1Encoder.cpp:974-990); the search rounds here
// compute errors only, so the selectors are computed once at the end. Done inside the refill loop,
// that would run with one lane of the warp active.
struct FinishQueue {
    uint32_t *count;
    uint32_t *b, *lohi, *mode;  // [cap] each
};

// Blocks whose EncodeBlock continues in k_bc1_cf2 after the first four-colour cluster-fit
// pass (one entry per block: its index, the result after the first pass, the endpoints
// before refinement). Entries that run the second pass fill the arrays from the front,
// entries that only run the 3-colour trials from the back, so warps of k_bc1_cf2 see one
// kind.
struct Cf2Queue {
    uint32_t *count;  // [2]: second-pass entries, 3-colour-only entries
    uint32_t *b, *lohi, *err, *sel, *mode, *orig;  // [cap] each
    long cap;
};

__device__ __forceinline__ uint32_t pack_lohi(const tpb::R &r) { return (uint32_t)r.lo | ((uint32_t)r.hi << 16); }

// Appends the lanes' deferred searches to their queues (warp-aggregated). Every lane of
// the warp calls it.
__device__ __forceinline__ void push_searches(const SearchQueues &q, const tpb::Deferred &d, long b, int lane) {
#pragma unroll
    for (int qq = 0; qq < 3; qq++) {
        const bool mine = d.need && d.queue == qq;
        const uint32_t m = __ballot_sync(0xffffffffu, mine);
        if (!m) continue;
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(q.count + qq, (uint32_t)__popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (mine) {
            const long slot = (long)qq * q.cap + base + __popc(m & ((1u << lane) - 1));
            q.b[slot] = (uint32_t)b;
            q.lohi[slot] = pack_lohi(d.r);
            q.err[slot] = d.r.err;
            q.sel[slot] = d.r.sel;
            q.mode[slot] = (uint32_t)d.r.mode;
        }
    }
}

__device__ __forceinline__ void load_tables_smem() {
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
        if (i < 32) s_mid5[i] = c_mid5[i];
        s_mid6[i] = c_mid6[i];
        if (i < 16) s_vox[i] = c_voxels[i];
    }
    __syncthreads();
}

// the block's texels into the thread's shared-memory column; returns sum |p|^2
__device__ __forceinline__ int stage_block(const uint8_t *__restrict__ rgba, int w, int h, int bw, long b, int aligned,
                                           uint32_t v[16]) {
    const int by = (int)(b / bw), bx = (int)(b - (long)by * bw);
    load_block_thread(rgba, w, h, bx, by, aligned && (bx * 4 + 4 <= w) && (by * 4 + 4 <= h), v);
    int pp = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        tpb::t_px[k][threadIdx.x] = v[k];
        const uint32_t u = v[k] & 0x00FFFFFFu;
        pp += (int)__dp4a(u, u, 0u);
    }
    return pp;
}

template <int IT>
__global__ void __launch_bounds__(tpb::kThreads, 4) k_bc1_defer(const uint8_t *__restrict__ rgba, int w, int h, int bw,
                                                                  qt_bc1_params p, uint8_t *__restrict__ out, int bc3,
                                                                  int aligned, const uint32_t *__restrict__ list,
                                                                  const uint32_t *__restrict__ count, SearchQueues q,
                                                                  Cf2Queue c) {
    load_tables_smem();
    const int color_mode = bc3 ? CM_FOUR : p.color_mode;  // BC3Encoder.h:39-40
    const int lane = threadIdx.x & 31;
    const long end = (long)*count, stride = (long)gridDim.x * blockDim.x;
    // warp-uniform iterations, so the ballots below see whole warps
    for (long wb = (long)blockIdx.x * blockDim.x + threadIdx.x - lane; wb < end; wb += stride) {
        const long i = wb + lane;
        tpb::Deferred d;
        d.need = d.cf2 = d.pass2 = false;
        d.queue = 0;
        long b = 0;
        if (i < end) {
            b = (long)list[i];
            uint32_t v[16];
            const int pp = stage_block(rgba, w, h, bw, b, aligned, v);
            const uint2 blk = tpb::encode_block<IT>(p, color_mode, pp, &d);
            if (bc3) {  // the alpha half now; a queued block's colour half is written by a later pass
#pragma unroll
                for (int k = 0; k < 16; k++) v[k] = tpb::t_px[k][threadIdx.x];
                const uint2 a = bc4_block_thread(v, 3);
                reinterpret_cast<uint4 *>(out)[b] = make_uint4(a.x, a.y, blk.x, blk.y);
            } else if (!d.need && !d.cf2) {
                reinterpret_cast<uint2 *>(out)[b] = blk;
            }
        }
        push_searches(q, d, b, lane);
#pragma unroll
        for (int kind = 0; kind < 2; kind++) {
            const bool mine = d.cf2 && d.pass2 == (kind == 0);
            const uint32_t m = __ballot_sync(0xffffffffu, mine);
            if (!m) continue;
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(c.count + kind, (uint32_t)__popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (mine) {
                const long idx = (long)base + __popc(m & ((1u << lane) - 1));
                const long slot = kind == 0 ? idx : c.cap - 1 - idx;
                c.b[slot] = (uint32_t)b;
                c.lohi[slot] = pack_lohi(d.r);
                c.err[slot] = d.r.err;
                c.sel[slot] = d.r.sel;
                c.mode[slot] = (uint32_t)d.r.mode;
                c.orig[slot] = pack_lohi(d.orig);
            }
        }
    }
}

// The queued blocks' second four-colour cluster-fit pass (BC1Encoder.cpp:300-302), for the
// entries that need it, and the rest of EncodeBlock after it; their searches go to the
// search queues. Entries of one kind are uniform work, so a plain grid-stride loop over the
// second-pass entries, then the others, keeps warps full.
template <int IT>
__global__ void __launch_bounds__(tpb::kThreads, 4) k_bc1_cf2(const uint8_t *__restrict__ rgba, int w, int h, int bw,
                                                                qt_bc1_params p, uint8_t *__restrict__ out, int bc3,
                                                                int aligned, Cf2Queue c, SearchQueues q) {
    load_tables_smem();
    const int color_mode = bc3 ? CM_FOUR : p.color_mode;
    const int lane = threadIdx.x & 31;
    const long n2 = (long)c.count[0], end = n2 + (long)c.count[1], stride = (long)gridDim.x * blockDim.x;
    for (long wb = (long)blockIdx.x * blockDim.x + threadIdx.x - lane; wb < end; wb += stride) {
        const long idx = wb + lane;
        tpb::Deferred d;
        d.need = d.cf2 = d.pass2 = false;
        d.queue = 0;
        long b = 0;
        if (idx < end) {
            const bool pass2 = idx < n2;
            const long i = pass2 ? idx : c.cap - 1 - (idx - n2);
            b = (long)c.b[i];
            uint32_t v[16];
            const int pp = stage_block(rgba, w, h, bw, b, aligned, v);
            const tpb::M m = tpb::metrics(false);
            tpb::R res, orig = tpb::rinit();
            const uint32_t lh = c.lohi[i], ol = c.orig[i];
            res.lo = (int)(lh & 0xFFFF);
            res.hi = (int)(lh >> 16);
            res.err = c.err[i];
            res.sel = c.sel[i];
            res.mode = (int)c.mode[i];
            orig.lo = (int)(ol & 0xFFFF);
            orig.hi = (int)(ol >> 16);
            if (pass2) res = tpb::refine_cf_any<IT>(kind_for(CM_FOUR, p.error_mode), res, m, p.orderings4, p.exhaustive, pp);
            const uint2 blk = tpb::encode_tail<IT>(p, color_mode, pp, m, res, orig, &d);
            if (!d.need) {
                if (bc3) reinterpret_cast<uint2 *>(out)[2 * b + 1] = blk;  // the colour half of the 16-byte block
                else reinterpret_cast<uint2 *>(out)[b] = blk;
            }
        }
        push_searches(q, d, b, lane);
    }
}

// One queue of searches (the reference's loop, BC1Encoder.cpp:930-996, one round per step).
template <int IT, int K>
__device__ __forceinline__ void search_queue(int qq, const uint8_t *__restrict__ rgba, int w, int h, int bw,
                                             unsigned rounds, uint8_t *__restrict__ out, int bc3, int aligned,
                                             const SearchQueues &q, const FinishQueue &f) {
    const int lane = threadIdx.x & 31;
    const uint32_t total = q.count[qq];
    bool active = false, drained = false, moved = false, pending = false, pending_write = false;
    long b = 0;
    tpb::R r = tpb::rinit();
    int forbidden = -1, pp = 0;
    unsigned prev = 0, i = 0;
    for (;;) {
        uint32_t need = __ballot_sync(0xffffffffu, !active && !drained);
        // A refill (queue entry, texels) runs with only the refilled lanes active, so it waits for
        // kRefillBatch idle lanes, unless no lane is searching. The lanes' finished searches are
        // settled in the same batch: those that moved the endpoints go to the finish queue
        // (warp-aggregated), the others are written.
        if (__popc(need) < kRefillBatch && __any_sync(0xffffffffu, active)) need = 0;
        if (need) {
            const uint32_t fin = __ballot_sync(0xffffffffu, pending);
            if (fin) {
                uint32_t fbase = 0;
                if (lane == 0) fbase = atomicAdd(f.count, (uint32_t)__popc(fin));
                fbase = __shfl_sync(0xffffffffu, fbase, 0);
                if (pending) {
                    const uint32_t slot = fbase + __popc(fin & ((1u << lane) - 1));
                    f.b[slot] = (uint32_t)b;
                    f.lohi[slot] = pack_lohi(r);
                    f.mode[slot] = (uint32_t)r.mode;
                    pending = false;
                }
            }
            if (pending_write) {  // the queued selectors belong to these endpoints
                const uint2 blk = tpb::write(r);
                if (bc3) reinterpret_cast<uint2 *>(out)[2 * b + 1] = blk;  // the colour half of the 16-byte block
                else reinterpret_cast<uint2 *>(out)[b] = blk;
                pending_write = false;
            }
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(q.head + qq, (uint32_t)__popc(need));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (!active && !drained) {
                const uint32_t idx = base + __popc(need & ((1u << lane) - 1));
                if (idx < total) {
                    const long slot = (long)qq * q.cap + idx;
                    b = (long)q.b[slot];
                    const uint32_t lh = q.lohi[slot];
                    r.lo = (int)(lh & 0xFFFF);
                    r.hi = (int)(lh >> 16);
                    r.err = q.err[slot];
                    r.sel = q.sel[slot];
                    r.mode = (int)q.mode[slot];
                    uint32_t v[16];
                    pp = stage_block(rgba, w, h, bw, b, aligned, v);
                    forbidden = -1;
                    prev = 0;
                    i = 0;
                    moved = false;
                    active = true;
                } else {
                    drained = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, active)) break;
        if (!active) continue;
        bool done = false;
        if ((int)(i & 31) == forbidden) i++;  // skipped by the reference without a stop test
        if (i < rounds) {
            const uint16_t vx = s_vox[i & 15];
            const int ddr = ((int)((unsigned)vx << 30)) >> 30, ddg = ((int)((unsigned)vx << 28)) >> 30;
            const int ddb = ((int)((unsigned)vx << 26)) >> 30;
            int lo = r.lo, hi = r.hi;
            if (i & 16) lo = eppack(clampi(epr(lo) + ddr, 0, 31), clampi(epg(lo) + ddg, 0, 63), clampi(epb(lo) + ddb, 0, 31));
            else hi = eppack(clampi(epr(hi) + ddr, 0, 31), clampi(epg(hi) + ddg, 0, 63), clampi(epb(hi) + ddb, 0, 31));
            const uint32_t e = tpb::block_error<IT, K>(lo, hi, pp);
            if (e < r.err) {
                r.lo = lo;
                r.hi = hi;
                r.err = e;
                forbidden = (int)((vx >> 8) & 15) | (int)(i & 16);
                prev = i;
                moved = true;
            }
            if (i - prev > 32) done = true;
            i++;
        }
        if (i >= rounds) done = true;
        if (done) {  // settled at the lane's next refill
            if (moved) pending = true;  // selectors and block from k_bc1_finish
            else pending_write = true;
            active = false;
        }
    }
}

template <int IT>
__global__ void __launch_bounds__(tpb::kThreads, 4) k_bc1_search(const uint8_t *__restrict__ rgba, int w, int h, int bw,
                                                                   qt_bc1_params p, uint8_t *__restrict__ out, int bc3,
                                                                   int aligned, SearchQueues q, FinishQueue f) {
    load_tables_smem();
    const unsigned rounds = p.search_rounds;
    switch (p.error_mode) {  // four-colour searches use the encoder's error mode (kind_for)
        case EM_NONE: search_queue<IT, K_F4_NONE>(0, rgba, w, h, bw, rounds, out, bc3, aligned, q, f); break;
        case EM_FASTER: search_queue<IT, K_F4_FASTER>(0, rgba, w, h, bw, rounds, out, bc3, aligned, q, f); break;
        case EM_CHECK2: search_queue<IT, K_F4_CHECK2>(0, rgba, w, h, bw, rounds, out, bc3, aligned, q, f); break;
        default: search_queue<IT, K_F4_FULL>(0, rgba, w, h, bw, rounds, out, bc3, aligned, q, f); break;
    }
    search_queue<IT, K_T3>(1, rgba, w, h, bw, rounds, out, bc3, aligned, q, f);
    search_queue<IT, K_TB>(2, rgba, w, h, bw, rounds, out, bc3, aligned, q, f);
}

// The searches that moved the endpoints: FindSelectors on the final endpoints (the selectors the
// reference kept from the last accepted trial, BC1Encoder.cpp:974-990) and WriteBlock, one entry
// per thread. The search kernel appends its queues in order, so a warp's
// entries share a colour mode except where one mode's entries end.
template <int IT>
__global__ void __launch_bounds__(tpb::kThreads, 4) k_bc1_finish(const uint8_t *__restrict__ rgba, int w, int h, int bw,
                                                                   qt_bc1_params p, uint8_t *__restrict__ out, int bc3,
                                                                   int aligned, FinishQueue f) {
    load_tables_smem();
    const long end = (long)*f.count, stride = (long)gridDim.x * blockDim.x;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < end; i += stride) {
        const long b = (long)f.b[i];
        uint32_t v[16];
        stage_block(rgba, w, h, bw, b, aligned, v);
        tpb::R r = tpb::rinit();
        const uint32_t lh = f.lohi[i];
        r.lo = (int)(lh & 0xFFFF);
        r.hi = (int)(lh >> 16);
        r.mode = (int)f.mode[i];
        const int Md = r.mode == CM_THREE ? CM_THREE : (r.mode == CM_TB ? CM_TB : CM_FOUR);
        r.sel = tpb::fs_any<IT>(kind_for(Md, Md == CM_FOUR ? p.error_mode : EM_FULL), r.lo, r.hi).x;
        const uint2 blk = tpb::write(r);
        if (bc3) reinterpret_cast<uint2 *>(out)[2 * b + 1] = blk;  // the colour half of the 16-byte block
        else reinterpret_cast<uint2 *>(out)[b] = blk;
    }
}
