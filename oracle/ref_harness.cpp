// Test infrastructure only: a C-ABI harness over the UNMODIFIED reference codec
// (drewcassidy/quicktex, quicktex/ sources compiled as-is by oracle/Makefile).
//
// It is the "reference" arm of the parity checks and of the CPU baseline: it
// constructs the reference's own encoder/decoder classes and runs them through
// their public Encode/Decode methods (BlockEncoder::Encode, Encoder.h:36-56;
// BlockDecoder::Decode, Decoder.h:36-54), or, in "omp" mode, through
// EncodeBlock/DecodeBlock under an OpenMP loop over every block.
//
// The reference's pybind11 layer cannot construct interpolators
// (s3tc/interpolator/_bindings.cpp:24-54 define no constructors), so this
// harness is the only way to drive IdealRound/Nvidia/AMD through the reference.
//
// Never linked into, loaded by, or called from the product library.

#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>

#include "Color.h"
#include "ColorBlock.h"
#include "Texture.h"
#include "s3tc/bc1/BC1Decoder.h"
#include "s3tc/bc1/BC1Encoder.h"
#include "s3tc/bc3/BC3Decoder.h"
#include "s3tc/bc3/BC3Encoder.h"
#include "s3tc/bc4/BC4Decoder.h"
#include "s3tc/bc4/BC4Encoder.h"
#include "s3tc/bc5/BC5Decoder.h"
#include "s3tc/bc5/BC5Encoder.h"
#include "s3tc/interpolator/Interpolator.h"

#ifdef _OPENMP
#include <omp.h>
#endif

using namespace quicktex;
using namespace quicktex::s3tc;

namespace {

thread_local std::string g_err;

std::shared_ptr<Interpolator> make_interp(int type) {
    return std::shared_ptr<Interpolator>(Interpolator::MakeInterpolator(static_cast<Interpolator::Type>(type)));
}

RawTexture to_raw(const uint8_t *rgba, int w, int h) {
    RawTexture t(w, h);
    std::memcpy(t.Data(), rgba, t.NBytes());
    return t;
}

template <typename B> BlockTexture<B> to_blocks(const uint8_t *data, int w, int h) {
    BlockTexture<B> t(w, h);
    std::memcpy(t.Data(), data, t.NBytes());
    return t;
}

// overrides: [error_mode, endpoint_mode, two_ls, two_ep, two_cf, exhaustive,
//             search_rounds, orderings4, orderings3, power_iterations]; -1 keeps the level's value.
void apply_overrides(BC1Encoder &e, const int *ov) {
    if (!ov) return;
    if (ov[0] >= 0) e.SetErrorMode(static_cast<BC1Encoder::ErrorMode>(ov[0]));
    if (ov[1] >= 0) e.SetEndpointMode(static_cast<BC1Encoder::EndpointMode>(ov[1]));
    if (ov[2] >= 0) e.two_ls_passes = ov[2] != 0;
    if (ov[3] >= 0) e.two_ep_passes = ov[3] != 0;
    if (ov[4] >= 0) e.two_cf_passes = ov[4] != 0;
    if (ov[5] >= 0) e.exhaustive = ov[5] != 0;
    if (ov[6] >= 0) e.SetSearchRounds(static_cast<unsigned>(ov[6]));
    if (ov[7] >= 0) e.SetOrderings4(static_cast<unsigned>(ov[7]));
    if (ov[8] >= 0) e.SetOrderings3(static_cast<unsigned>(ov[8]));
    if (ov[9] >= 0) e.SetPowerIterations(static_cast<unsigned>(ov[9]));
}

// mode 0: the reference's own Encode (OpenMP only where MTThreshold allows it).
// mode 1: OpenMP over EncodeBlock for every block (the fair parallel CPU figure).
template <typename Enc> void run_encode(const Enc &enc, const RawTexture &raw, uint8_t *out, int mode) {
    using Tex = typename Enc::Texture;
    if (mode == 0) {
        Tex t = enc.Encode(raw);
        std::memcpy(out, t.Data(), t.NBytes());
        return;
    }
    Tex t(raw.Width(), raw.Height());
    const int bx = t.BlocksX(), by = t.BlocksY();
    const long n = (long)bx * by;
#pragma omp parallel for schedule(dynamic, 64)
    for (long i = 0; i < n; i++) {
        int x = (int)(i % bx), y = (int)(i / bx);
        auto px = raw.GetBlock<4, 4>(x, y);
        t.SetBlock(x, y, enc.EncodeBlock(px));
    }
    std::memcpy(out, t.Data(), t.NBytes());
}

// Seconds of the fastest of `reps` runs (after one untimed run) of one encode of `raw`: mode 0
// the reference's own Encode, mode 1 OpenMP over EncodeBlock. Only the encode is timed: the
// encoder, its tables and the input texture exist beforehand (the reference's CPU timing plan).
template <typename Enc> double time_encode(const Enc &enc, const RawTexture &raw, int mode, int reps) {
    using Tex = typename Enc::Texture;
    double best = 1e30;
    for (int r = 0; r <= reps; r++) {
        const auto t0 = std::chrono::steady_clock::now();
        if (mode == 0) {
            Tex t = enc.Encode(raw);
            (void)t;
        } else {
            Tex t(raw.Width(), raw.Height());
            const int bx = t.BlocksX(), by = t.BlocksY();
            const long n = (long)bx * by;
#pragma omp parallel for schedule(dynamic, 64)
            for (long i = 0; i < n; i++) {
                int x = (int)(i % bx), y = (int)(i / bx);
                t.SetBlock(x, y, enc.EncodeBlock(raw.GetBlock<4, 4>(x, y)));
            }
        }
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (r > 0 && dt < best) best = dt;
    }
    return best;
}

// The same for one decode: mode 0 the reference's own (serial) Decode, mode 1 OpenMP over
// DecodeBlock (block-aligned sizes only, so no two blocks write the same texel).
template <typename Dec> double time_decode(const Dec &dec, const typename Dec::Texture &tex, int mode, int reps) {
    double best = 1e30;
    for (int r = 0; r <= reps; r++) {
        const auto t0 = std::chrono::steady_clock::now();
        if (mode == 0) {
            RawTexture out = dec.Decode(tex);
            (void)out;
        } else {
            RawTexture out(tex.Width(), tex.Height());
            const int bx = tex.BlocksX(), by = tex.BlocksY();
            const long n = (long)bx * by;
#pragma omp parallel for schedule(dynamic, 256)
            for (long i = 0; i < n; i++) {
                int x = (int)(i % bx), y = (int)(i / bx);
                out.SetBlock<4, 4>(x, y, dec.DecodeBlock(tex.GetBlock(x, y)));
            }
        }
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (r > 0 && dt < best) best = dt;
    }
    return best;
}

template <typename F> int guarded(F &&f) {
    try {
        f();
        return 0;
    } catch (const std::exception &e) {
        g_err = e.what();
        return 1;
    }
}

}  // namespace

extern "C" {

const char *ref_last_error() { return g_err.c_str(); }

int ref_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void ref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// Resolved BC1 settings for a level (BC1Encoder::SetLevel, BC1Encoder.cpp:74-249):
// out = [error_mode, endpoint_mode, two_ls, two_ep, two_cf, exhaustive, search_rounds,
//        orderings4, orderings3, power_iterations]
int ref_bc1_level_params(int level, int color_mode, int *out) {
    return guarded([&] {
        BC1Encoder e((unsigned)level, static_cast<BC1Encoder::ColorMode>(color_mode));
        out[0] = (int)e.GetErrorMode();
        out[1] = (int)e.GetEndpointMode();
        out[2] = e.two_ls_passes;
        out[3] = e.two_ep_passes;
        out[4] = e.two_cf_passes;
        out[5] = e.exhaustive;
        out[6] = (int)e.GetSearchRounds();
        out[7] = (int)e.GetOrderings4();
        out[8] = (int)e.GetOrderings3();
        out[9] = (int)e.GetPowerIterations();
    });
}

int ref_bc1_encode(const uint8_t *rgba, int w, int h, int level, int color_mode, int interp, const int *overrides, uint8_t *out, int mode) {
    return guarded([&] {
        BC1Encoder e((unsigned)level, static_cast<BC1Encoder::ColorMode>(color_mode), make_interp(interp));
        apply_overrides(e, overrides);
        run_encode(e, to_raw(rgba, w, h), out, mode);
    });
}

int ref_bc3_encode(const uint8_t *rgba, int w, int h, int level, int interp, uint8_t *out, int mode) {
    return guarded([&] {
        BC3Encoder e((unsigned)level, make_interp(interp));
        run_encode(e, to_raw(rgba, w, h), out, mode);
    });
}

int ref_bc4_encode(const uint8_t *rgba, int w, int h, int channel, uint8_t *out, int mode) {
    return guarded([&] {
        BC4Encoder e((uint8_t)channel);
        run_encode(e, to_raw(rgba, w, h), out, mode);
    });
}

int ref_bc5_encode(const uint8_t *rgba, int w, int h, int c0, int c1, uint8_t *out, int mode) {
    return guarded([&] {
        BC5Encoder e((uint8_t)c0, (uint8_t)c1);
        run_encode(e, to_raw(rgba, w, h), out, mode);
    });
}

int ref_bc1_decode(const uint8_t *blocks, int w, int h, int interp, int write_alpha, uint8_t *out) {
    return guarded([&] {
        BC1Decoder d(write_alpha != 0, make_interp(interp));
        RawTexture r = d.Decode(to_blocks<BC1Block>(blocks, w, h));
        std::memcpy(out, r.Data(), r.NBytes());
    });
}

int ref_bc3_decode(const uint8_t *blocks, int w, int h, int interp, uint8_t *out) {
    return guarded([&] {
        BC3Decoder d(make_interp(interp));
        RawTexture r = d.Decode(to_blocks<BC3Block>(blocks, w, h));
        std::memcpy(out, r.Data(), r.NBytes());
    });
}

int ref_bc4_decode(const uint8_t *blocks, int w, int h, int channel, uint8_t *out) {
    return guarded([&] {
        BC4Decoder d((uint8_t)channel);
        RawTexture r = d.Decode(to_blocks<BC4Block>(blocks, w, h));
        std::memcpy(out, r.Data(), r.NBytes());
    });
}

int ref_bc5_decode(const uint8_t *blocks, int w, int h, int c0, int c1, uint8_t *out) {
    return guarded([&] {
        BC5Decoder d((uint8_t)c0, (uint8_t)c1);
        RawTexture r = d.Decode(to_blocks<BC5Block>(blocks, w, h));
        std::memcpy(out, r.Data(), r.NBytes());
    });
}

// Timing (CPU baseline): seconds of the fastest of `reps` encodes of fmt (1, 3, 4, 5) on the
// w x h texture; level/color_mode/interp apply to BC1 and BC3, c0/c1 to BC4 (c0) and BC5.
// Returns a negative value on error (message in ref_last_error).
double ref_time_encode(int fmt, const uint8_t *rgba, int w, int h, int level, int color_mode, int interp, int c0,
                       int c1, int mode, int reps) {
    double t = -1.0;
    if (guarded([&] {
            const RawTexture raw = to_raw(rgba, w, h);
            if (fmt == 1) t = time_encode(BC1Encoder((unsigned)level, static_cast<BC1Encoder::ColorMode>(color_mode), make_interp(interp)), raw, mode, reps);
            else if (fmt == 3) t = time_encode(BC3Encoder((unsigned)level, make_interp(interp)), raw, mode, reps);
            else if (fmt == 4) t = time_encode(BC4Encoder((uint8_t)c0), raw, mode, reps);
            else if (fmt == 5) t = time_encode(BC5Encoder((uint8_t)c0, (uint8_t)c1), raw, mode, reps);
            else throw std::invalid_argument("format must be 1, 3, 4 or 5");
        }))
        return -1.0;
    return t;
}

// The same for decoding `blocks` (BC1 with write_alpha = 0; BC3 with the given interpolator).
double ref_time_decode(int fmt, const uint8_t *blocks, int w, int h, int interp, int c0, int c1, int mode, int reps) {
    double t = -1.0;
    if (guarded([&] {
            if (mode == 1 && ((w & 3) || (h & 3))) throw std::invalid_argument("mode 1 needs block-aligned sizes");
            if (fmt == 1) t = time_decode(BC1Decoder(false, make_interp(interp)), to_blocks<BC1Block>(blocks, w, h), mode, reps);
            else if (fmt == 3) t = time_decode(BC3Decoder(make_interp(interp)), to_blocks<BC3Block>(blocks, w, h), mode, reps);
            else if (fmt == 4) t = time_decode(BC4Decoder((uint8_t)c0), to_blocks<BC4Block>(blocks, w, h), mode, reps);
            else if (fmt == 5) t = time_decode(BC5Decoder((uint8_t)c0, (uint8_t)c1), to_blocks<BC5Block>(blocks, w, h), mode, reps);
            else throw std::invalid_argument("format must be 1, 3, 4 or 5");
        }))
        return -1.0;
    return t;
}

}  // extern "C"
