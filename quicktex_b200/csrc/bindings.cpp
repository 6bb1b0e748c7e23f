// bindings.cpp — the `_quicktex` Python extension of quicktex_b200.
//
// Mirrors the reference module (quicktex/_bindings.cpp:38-71,
// quicktex/_bindings.h:38-234, quicktex/s3tc/*/_bindings.cpp): the same
// classes, methods, properties, defaults and exception types, so that
// `quicktex_b200.s3tc.bc1.BC1Encoder(...).encode(tex)` reads like the
// reference's call. Texture objects own host buffers; every encode/decode is
// one call into libquicktex_cuda.so (include/quicktex_cuda.h) with the GIL
// released. One addition: the interpolator classes have constructors, which
// the reference does not expose (s3tc/interpolator/_bindings.cpp:24-54).

#include <pybind11/operators.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <array>
#include <cstdint>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "quicktex_cuda.h"

namespace py = pybind11;
using namespace pybind11::literals;

namespace qtb {

struct Color {
    uint8_t r = 0, g = 0, b = 0, a = 255;
};

}  // namespace qtb

namespace pybind11::detail {
// Color <-> tuple of 3 or 4 ints in [0, 255] (alpha defaults to 255), as the
// reference's caster does (quicktex/_bindings.h:38-82).
template <> struct type_caster<qtb::Color> {
   public:
    PYBIND11_TYPE_CASTER(qtb::Color, const_name("Color"));

    bool load(handle src, bool) {
        if (!src || !PySequence_Check(src.ptr()) || PyUnicode_Check(src.ptr()) || PyBytes_Check(src.ptr())) return false;
        PyObject *t = PySequence_Tuple(src.ptr());
        if (!t) {
            PyErr_Clear();
            return false;
        }
        const Py_ssize_t n = PyTuple_Size(t);
        bool ok = n >= 3 && n <= 4;
        uint8_t ch[4] = {0, 0, 0, 255};
        for (Py_ssize_t i = 0; ok && i < n; i++) {
            PyObject *num = PyNumber_Long(PyTuple_GetItem(t, i));
            if (!num) {
                PyErr_Clear();
                ok = false;
                break;
            }
            const long v = PyLong_AsLong(num);
            Py_DECREF(num);
            if (v < 0 || v > 255) ok = false;
            else ch[i] = (uint8_t)v;
        }
        Py_DECREF(t);
        if (!ok) return false;
        value.r = ch[0];
        value.g = ch[1];
        value.b = ch[2];
        value.a = ch[3];
        return true;
    }

    static handle cast(const qtb::Color &c, return_value_policy, handle) {
        return py::make_tuple((int)c.r, (int)c.g, (int)c.b, (int)c.a).release();
    }
};
}  // namespace pybind11::detail

namespace qtb {

// ---------------------------------------------------------------------------
// status -> Python exception (the reference's pybind11 translations)
// ---------------------------------------------------------------------------
void check(int rc) {
    if (rc == QT_OK) return;
    const std::string msg = qt_last_error();
    switch (rc) {
        case QT_ERR_ARG: throw std::invalid_argument(msg);
        case QT_ERR_RANGE: throw std::out_of_range(msg);
        case QT_ERR_OOM: throw std::bad_alloc();
        default: throw std::runtime_error(msg);
    }
}

// ---------------------------------------------------------------------------
// textures (quicktex/Texture.h)
// ---------------------------------------------------------------------------
// Texel or block storage in the library's cache of pinned host blocks (qt_host_alloc): the
// host-buffer entry points copy it with the copy engines directly, where the reference's
// pageable std::vector would be staged through a pinned ring first (about as much time again
// as the copy itself on a large texture).
class HostBytes {
   public:
    HostBytes() = default;
    explicit HostBytes(size_t n) : n_(n) {
        void *p = nullptr;
        if (qt_host_alloc(n, &p) != QT_OK) throw std::bad_alloc();
        p_ = static_cast<uint8_t *>(p);
    }
    HostBytes(const HostBytes &o) : HostBytes(o.n_) { std::memcpy(p_, o.p_, n_); }
    HostBytes(HostBytes &&o) noexcept : p_(o.p_), n_(o.n_) {
        o.p_ = nullptr;
        o.n_ = 0;
    }
    HostBytes &operator=(HostBytes o) noexcept {
        std::swap(p_, o.p_);
        std::swap(n_, o.n_);
        return *this;
    }
    ~HostBytes() { qt_host_free(p_); }
    uint8_t *data() { return p_; }
    const uint8_t *data() const { return p_; }
    size_t size() const { return n_; }
    uint8_t &operator[](size_t i) { return p_[i]; }

   private:
    uint8_t *p_ = nullptr;
    size_t n_ = 0;
};

// Construction without the initial fill, for textures whose every byte is written next (an
// encoder's result, a texture made from a bytes-like object).
struct NoFill {};

class Texture {
   public:
    virtual ~Texture() = default;
    int Width() const { return w_; }
    int Height() const { return h_; }
    std::tuple<int, int> Size() const { return {w_, h_}; }
    size_t NBytes() const { return data_.size(); }
    uint8_t *Data() { return data_.data(); }
    const uint8_t *Data() const { return data_.data(); }

   protected:
    Texture(int w, int h, size_t nbytes, NoFill) : w_(w), h_(h) {
        if (w <= 0) throw std::invalid_argument("Texture width must be greater than 0");
        if (h <= 0) throw std::invalid_argument("Texture height must be greater than 0");
        data_ = HostBytes(nbytes);
    }
    Texture(int w, int h, size_t nbytes) : Texture(w, h, nbytes, NoFill{}) { std::memset(data_.data(), 0, nbytes); }
    int w_, h_;
    HostBytes data_;
};

inline size_t checked_area(int w, int h) { return (w > 0 && h > 0) ? (size_t)w * (size_t)h : 0; }

class RawTexture : public Texture {
   public:
    RawTexture(int w, int h) : Texture(w, h, checked_area(w, h) * 4, NoFill{}) {
        // Color() = (0, 0, 0, 255) in every texel, one 32-bit store each (the storage is page-aligned)
        std::fill_n(reinterpret_cast<uint32_t *>(data_.data()), data_.size() / 4, 0xFF000000u);
    }
    RawTexture(int w, int h, NoFill f) : Texture(w, h, checked_area(w, h) * 4, f) {}
    Color GetPixel(int x, int y) const {
        const uint8_t *p = data_.data() + ((size_t)y * w_ + x) * 4;
        return Color{p[0], p[1], p[2], p[3]};
    }
    void SetPixel(int x, int y, Color c) {
        uint8_t *p = data_.data() + ((size_t)y * w_ + x) * 4;
        p[0] = c.r;
        p[1] = c.g;
        p[2] = c.b;
        p[3] = c.a;
    }
};

template <size_t N> struct alignas(8) Block {
    static constexpr int Width = 4, Height = 4;
    std::array<uint8_t, N> bytes{};
    bool operator==(const Block &o) const { return bytes == o.bytes; }
};

using Sel4x4 = std::array<std::array<uint8_t, 4>, 4>;

// BC1Block (s3tc/bc1/BC1Block.h:30-125): color0 LE u16, color1 LE u16, row y = byte 4+y, texel x at bits 2x
struct BC1Block : Block<8> {
    static uint16_t pack565(Color c) {
        auto s5 = [](int v) { int v2 = v * 31 + 128; return (v2 + (v2 >> 8)) >> 8; };
        auto s6 = [](int v) { int v2 = v * 63 + 128; return (v2 + (v2 >> 8)) >> 8; };
        return (uint16_t)(s5(c.b) | (s6(c.g) << 5) | (s5(c.r) << 11));
    }
    static Color unpack565(uint16_t v) {
        const int r = (v >> 11) & 31, g = (v >> 5) & 63, b = v & 31;
        return Color{(uint8_t)((r << 3) | (r >> 2)), (uint8_t)((g << 2) | (g >> 4)), (uint8_t)((b << 3) | (b >> 2)), 255};
    }
    uint16_t c0() const { return (uint16_t)(bytes[0] | (bytes[1] << 8)); }
    uint16_t c1() const { return (uint16_t)(bytes[2] | (bytes[3] << 8)); }
    void set_c0(uint16_t v) { bytes[0] = v & 0xFF; bytes[1] = v >> 8; }
    void set_c1(uint16_t v) { bytes[2] = v & 0xFF; bytes[3] = v >> 8; }
    std::tuple<Color, Color> GetColors() const { return {unpack565(c0()), unpack565(c1())}; }
    void SetColors(std::tuple<Color, Color> cs) {
        set_c0(pack565(std::get<0>(cs)));
        set_c1(pack565(std::get<1>(cs)));
    }
    Sel4x4 GetSelectors() const {
        Sel4x4 s{};
        for (int y = 0; y < 4; y++)
            for (int x = 0; x < 4; x++) s[y][x] = (bytes[4 + y] >> (2 * x)) & 3;
        return s;
    }
    void SetSelectors(const Sel4x4 &s) {
        for (auto &row : s)
            for (auto v : row)
                if (v > 3) throw std::invalid_argument("Selector value out of bounds.");
        for (int y = 0; y < 4; y++) {
            uint8_t b = 0;
            for (int x = 0; x < 4; x++) b |= (uint8_t)(s[y][x] << (2 * x));
            bytes[4 + y] = b;
        }
    }
    bool Is3Color() const { return c0() <= c1(); }
};

// BC4Block (s3tc/bc4/BC4Block.h:28-105): a0, a1, 48 selector bits LE, 3 bits per texel, row-major
struct BC4Block : Block<8> {
    uint64_t sel_bits() const {
        uint64_t b = 0;
        for (int k = 0; k < 6; k++) b |= (uint64_t)bytes[2 + k] << (8 * k);
        return b;
    }
    std::tuple<uint8_t, uint8_t> GetAlphas() const { return {bytes[0], bytes[1]}; }
    void SetAlphas(std::tuple<uint8_t, uint8_t> a) {
        bytes[0] = std::get<0>(a);
        bytes[1] = std::get<1>(a);
    }
    Sel4x4 GetSelectors() const {
        const uint64_t b = sel_bits();
        Sel4x4 s{};
        for (int i = 0; i < 16; i++) s[i / 4][i % 4] = (b >> (3 * i)) & 7;
        return s;
    }
    void SetSelectors(const Sel4x4 &s) {
        for (auto &row : s)
            for (auto v : row)
                if (v > 7) throw std::invalid_argument("Selector value out of bounds.");
        uint64_t b = 0;
        for (int i = 0; i < 16; i++) b |= (uint64_t)s[i / 4][i % 4] << (3 * i);
        for (int k = 0; k < 6; k++) bytes[2 + k] = (uint8_t)(b >> (8 * k));
    }
    bool Is6Value() const { return bytes[0] <= bytes[1]; }
    std::array<uint8_t, 8> GetValues() const {  // BC4Block::GetValues6/8 (BC4Block.cpp:44-64)
        const int a0 = bytes[0], a1 = bytes[1];
        if (a0 <= a1)
            return {(uint8_t)a0, (uint8_t)a1, (uint8_t)((a0 * 4 + a1) / 5), (uint8_t)((a0 * 3 + a1 * 2) / 5),
                    (uint8_t)((a0 * 2 + a1 * 3) / 5), (uint8_t)((a0 + a1 * 4) / 5), 0, 0xFF};
        return {(uint8_t)a0, (uint8_t)a1, (uint8_t)((a0 * 6 + a1) / 7), (uint8_t)((a0 * 5 + a1 * 2) / 7),
                (uint8_t)((a0 * 4 + a1 * 3) / 7), (uint8_t)((a0 * 3 + a1 * 4) / 7), (uint8_t)((a0 * 2 + a1 * 5) / 7),
                (uint8_t)((a0 + a1 * 6) / 7)};
    }
};

// BC3Block = BC4 alpha block then BC1 colour block (BC3Block.h:28-58)
struct BC3Block {
    static constexpr int Width = 4, Height = 4;
    BC4Block alpha_block;
    BC1Block color_block;
    bool operator==(const BC3Block &o) const { return alpha_block == o.alpha_block && color_block == o.color_block; }
    std::tuple<BC4Block, BC1Block> GetBlocks() const { return {alpha_block, color_block}; }
    void SetBlocks(std::tuple<BC4Block, BC1Block> b) {
        alpha_block = std::get<0>(b);
        color_block = std::get<1>(b);
    }
};

// BC5Block = two BC4 blocks (BC5Block.h:27-57)
struct BC5Block {
    static constexpr int Width = 4, Height = 4;
    BC4Block chan0_block;
    BC4Block chan1_block;
    bool operator==(const BC5Block &o) const { return chan0_block == o.chan0_block && chan1_block == o.chan1_block; }
    std::tuple<BC4Block, BC4Block> GetBlocks() const { return {chan0_block, chan1_block}; }
    void SetBlocks(std::tuple<BC4Block, BC4Block> b) {
        chan0_block = std::get<0>(b);
        chan1_block = std::get<1>(b);
    }
};
static_assert(sizeof(BC1Block) == 8 && sizeof(BC4Block) == 8 && sizeof(BC3Block) == 16 && sizeof(BC5Block) == 16);

template <typename B> class BlockTexture : public Texture {
   public:
    BlockTexture(int w, int h) : Texture(w, h, (size_t)((w + 3) / 4) * (size_t)((h + 3) / 4) * sizeof(B)) {
        bw_ = (w + 3) / 4;
        bh_ = (h + 3) / 4;
    }
    BlockTexture(int w, int h, NoFill f) : Texture(w, h, (size_t)((w + 3) / 4) * (size_t)((h + 3) / 4) * sizeof(B), f) {
        bw_ = (w + 3) / 4;
        bh_ = (h + 3) / 4;
    }
    int BlocksX() const { return bw_; }
    int BlocksY() const { return bh_; }
    std::tuple<int, int> BlocksXY() const { return {bw_, bh_}; }
    B GetBlock(int x, int y) const {
        B b;
        std::memcpy(&b, data_.data() + ((size_t)y * bw_ + x) * sizeof(B), sizeof(B));
        return b;
    }
    void SetBlock(int x, int y, const B &b) { std::memcpy(data_.data() + ((size_t)y * bw_ + x) * sizeof(B), &b, sizeof(B)); }

   private:
    int bw_, bh_;
};

using BC1Texture = BlockTexture<BC1Block>;
using BC3Texture = BlockTexture<BC3Block>;
using BC4Texture = BlockTexture<BC4Block>;
using BC5Texture = BlockTexture<BC5Block>;

// ---------------------------------------------------------------------------
// interpolators (s3tc/interpolator/Interpolator.h:28-180): identified by type
// ---------------------------------------------------------------------------
class Interpolator {
   public:
    virtual ~Interpolator() = default;
    virtual int Type() const { return QT_INTERP_IDEAL; }
};
class InterpolatorRound final : public Interpolator {
   public:
    int Type() const override { return QT_INTERP_IDEAL_ROUND; }
};
class InterpolatorNvidia final : public Interpolator {
   public:
    int Type() const override { return QT_INTERP_NVIDIA; }
};
class InterpolatorAMD final : public Interpolator {
   public:
    int Type() const override { return QT_INTERP_AMD; }
};
using InterpolatorPtr = std::shared_ptr<Interpolator>;

// ---------------------------------------------------------------------------
// encoders / decoders
// ---------------------------------------------------------------------------
enum class ColorMode : int { Incomplete = 0x00, ThreeColor = 0x03, FourColor = 0x04, UseBlack = 0x10, ThreeColorBlack = 0x13 };
enum class ErrorMode : int { None = 0, Faster = 1, Check2 = 2, Full = 3 };
enum class EndpointMode : int { LeastSquares = 0, BoundingBox = 1, BoundingBoxInt = 2, PCA = 3 };

class BC1Encoder {
   public:
    static constexpr unsigned min_power_iterations = 4;
    static constexpr unsigned max_power_iterations = 10;

    BC1Encoder(unsigned level, ColorMode mode, InterpolatorPtr interp) : interp_(std::move(interp)), mode_(mode) {
        if (mode != ColorMode::FourColor && mode != ColorMode::ThreeColor && mode != ColorMode::ThreeColorBlack)
            throw std::invalid_argument("Encoder color mode must be FourColor, ThreeColor, or ThreeColorBlack");
        if (!interp_) throw std::invalid_argument("interpolator must not be None");
        SetLevel(level);
    }
    BC1Encoder(unsigned level = 5, ColorMode mode = ColorMode::FourColor)
        : BC1Encoder(level, mode, std::make_shared<Interpolator>()) {}

    void SetLevel(unsigned level) { check(qt_bc1_params_for_level(level, (int)mode_, interp_->Type(), &p_)); }

    qt_bc1_params params() const {
        qt_bc1_params p = p_;
        p.color_mode = (int)mode_;
        p.interpolator = interp_->Type();
        return p;
    }

    BC1Texture Encode(const RawTexture &tex) const {
        BC1Texture out(tex.Width(), tex.Height(), NoFill{});  // every block is written
        const qt_bc1_params p = params();
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = qt_bc1_encode_host(tex.Data(), tex.Width(), tex.Height(), &p, out.Data());
        }
        check(rc);
        return out;
    }

    InterpolatorPtr GetInterpolator() const { return interp_; }
    ColorMode GetColorMode() const { return mode_; }
    ErrorMode GetErrorMode() const { return (ErrorMode)p_.error_mode; }
    void SetErrorMode(ErrorMode m) { p_.error_mode = (int)m; }
    EndpointMode GetEndpointMode() const { return (EndpointMode)p_.endpoint_mode; }
    void SetEndpointMode(EndpointMode m) { p_.endpoint_mode = (int)m; }
    unsigned GetSearchRounds() const { return p_.search_rounds; }
    void SetSearchRounds(unsigned r) { p_.search_rounds = r; }
    std::tuple<unsigned, unsigned> GetOrderings() const { return {p_.orderings4, p_.orderings3}; }
    void SetOrderings(std::tuple<unsigned, unsigned> o) {  // clamped (BC1Encoder.cpp:251-256)
        p_.orderings4 = std::min(std::max(std::get<0>(o), 1u), 128u);
        p_.orderings3 = std::min(std::max(std::get<1>(o), 1u), 32u);
    }
    unsigned GetPowerIterations() const { return p_.power_iterations; }
    void SetPowerIterations(unsigned n) { p_.power_iterations = std::min(std::max(n, min_power_iterations), max_power_iterations); }
    bool GetFlag(int which) const {
        return which == 0 ? p_.two_ls_passes : which == 1 ? p_.two_ep_passes : which == 2 ? p_.two_cf_passes : p_.exhaustive;
    }
    void SetFlag(int which, bool v) {
        (which == 0 ? p_.two_ls_passes : which == 1 ? p_.two_ep_passes : which == 2 ? p_.two_cf_passes : p_.exhaustive) = v;
    }

   private:
    InterpolatorPtr interp_;
    ColorMode mode_;
    qt_bc1_params p_{};
};

class BC1Decoder {
   public:
    BC1Decoder(bool write_alpha, InterpolatorPtr interp) : write_alpha(write_alpha), interp_(std::move(interp)) {
        if (!interp_) throw std::invalid_argument("interpolator must not be None");
    }
    explicit BC1Decoder(bool write_alpha = false) : BC1Decoder(write_alpha, std::make_shared<Interpolator>()) {}
    RawTexture Decode(const BC1Texture &tex) const {
        RawTexture out(tex.Width(), tex.Height(), NoFill{});  // every texel is written, defaults included
        const int it = interp_->Type(), wa = write_alpha;
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = qt_bc1_decode_host(tex.Data(), tex.Width(), tex.Height(), it, wa, out.Data());
        }
        check(rc);
        return out;
    }
    InterpolatorPtr GetInterpolator() const { return interp_; }
    bool write_alpha;

   private:
    InterpolatorPtr interp_;
};

class BC4Encoder {
   public:
    explicit BC4Encoder(uint8_t channel = 3) : channel_(channel) {
        if (channel >= 4) throw std::invalid_argument("Channel out of range");
    }
    BC4Texture Encode(const RawTexture &tex) const {
        BC4Texture out(tex.Width(), tex.Height(), NoFill{});  // every block is written
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = qt_bc4_encode_host(tex.Data(), tex.Width(), tex.Height(), channel_, out.Data());
        }
        check(rc);
        return out;
    }
    uint8_t GetChannel() const { return channel_; }

   private:
    uint8_t channel_;
};

class BC4Decoder {
   public:
    explicit BC4Decoder(uint8_t channel = 3) : channel_(channel) {
        if (channel >= 4) throw std::invalid_argument("Channel out of range");
    }
    RawTexture Decode(const BC4Texture &tex) const {
        RawTexture out(tex.Width(), tex.Height(), NoFill{});  // every texel is written, defaults included
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = qt_bc4_decode_host(tex.Data(), tex.Width(), tex.Height(), channel_, out.Data());
        }
        check(rc);
        return out;
    }
    uint8_t GetChannel() const { return channel_; }

   private:
    uint8_t channel_;
};

class BC3Encoder {
   public:
    BC3Encoder(unsigned level, InterpolatorPtr interp)
        : bc1_(std::make_shared<BC1Encoder>(level, ColorMode::FourColor, std::move(interp))), bc4_(std::make_shared<BC4Encoder>(3)) {}
    explicit BC3Encoder(unsigned level = 5) : BC3Encoder(level, std::make_shared<Interpolator>()) {}
    BC3Texture Encode(const RawTexture &tex) const {
        BC3Texture out(tex.Width(), tex.Height(), NoFill{});  // every block is written
        const qt_bc1_params p = bc1_->params();
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = qt_bc3_encode_host(tex.Data(), tex.Width(), tex.Height(), &p, out.Data());
        }
        check(rc);
        return out;
    }
    std::shared_ptr<BC1Encoder> GetBC1Encoder() const { return bc1_; }
    std::shared_ptr<BC4Encoder> GetBC4Encoder() const { return bc4_; }

   private:
    std::shared_ptr<BC1Encoder> bc1_;
    std::shared_ptr<BC4Encoder> bc4_;
};

class BC3Decoder {
   public:
    explicit BC3Decoder(InterpolatorPtr interp)
        : bc1_(std::make_shared<BC1Decoder>(false, std::move(interp))), bc4_(std::make_shared<BC4Decoder>(3)) {}
    BC3Decoder() : BC3Decoder(std::make_shared<Interpolator>()) {}
    RawTexture Decode(const BC3Texture &tex) const {
        RawTexture out(tex.Width(), tex.Height(), NoFill{});  // every texel is written, defaults included
        const int it = bc1_->GetInterpolator()->Type();
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = qt_bc3_decode_host(tex.Data(), tex.Width(), tex.Height(), it, out.Data());
        }
        check(rc);
        return out;
    }
    std::shared_ptr<BC1Decoder> GetBC1Decoder() const { return bc1_; }
    std::shared_ptr<BC4Decoder> GetBC4Decoder() const { return bc4_; }

   private:
    std::shared_ptr<BC1Decoder> bc1_;
    std::shared_ptr<BC4Decoder> bc4_;
};

class BC5Encoder {
   public:
    BC5Encoder(uint8_t c0 = 0, uint8_t c1 = 1) : e0_(std::make_shared<BC4Encoder>(c0)), e1_(std::make_shared<BC4Encoder>(c1)) {}
    BC5Texture Encode(const RawTexture &tex) const {
        BC5Texture out(tex.Width(), tex.Height(), NoFill{});  // every block is written
        const int c0 = e0_->GetChannel(), c1 = e1_->GetChannel();
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = qt_bc5_encode_host(tex.Data(), tex.Width(), tex.Height(), c0, c1, out.Data());
        }
        check(rc);
        return out;
    }
    std::tuple<uint8_t, uint8_t> GetChannels() const { return {e0_->GetChannel(), e1_->GetChannel()}; }
    std::tuple<std::shared_ptr<BC4Encoder>, std::shared_ptr<BC4Encoder>> GetBC4Encoders() const { return {e0_, e1_}; }

   private:
    std::shared_ptr<BC4Encoder> e0_, e1_;
};

class BC5Decoder {
   public:
    BC5Decoder(uint8_t c0 = 0, uint8_t c1 = 1) : d0_(std::make_shared<BC4Decoder>(c0)), d1_(std::make_shared<BC4Decoder>(c1)) {}
    RawTexture Decode(const BC5Texture &tex) const {
        RawTexture out(tex.Width(), tex.Height(), NoFill{});  // every texel is written, defaults included
        const int c0 = d0_->GetChannel(), c1 = d1_->GetChannel();
        int rc;
        {
            py::gil_scoped_release nogil;
            rc = qt_bc5_decode_host(tex.Data(), tex.Width(), tex.Height(), c0, c1, out.Data());
        }
        check(rc);
        return out;
    }
    std::tuple<uint8_t, uint8_t> GetChannels() const { return {d0_->GetChannel(), d1_->GetChannel()}; }
    std::tuple<std::shared_ptr<BC4Decoder>, std::shared_ptr<BC4Decoder>> GetBC4Decoders() const { return {d0_, d1_}; }

   private:
    std::shared_ptr<BC4Decoder> d0_, d1_;
};

// ---------------------------------------------------------------------------
// binding helpers (quicktex/_bindings.h:87-234)
// ---------------------------------------------------------------------------
py::buffer_info request_bytes(py::buffer buf, size_t need) {
    py::buffer_info info = buf.request(false);
    if (info.format != py::format_descriptor<uint8_t>::format())
        throw std::runtime_error("Incompatible format in python buffer: expected a byte array.");
    if (info.ndim != 1) throw std::runtime_error("Incompatible format in python buffer: Incorrect number of dimensions.");
    if (info.shape[0] < (py::ssize_t)need) throw std::runtime_error("Incompatible format in python buffer: 1-D buffer has incorrect length.");
    if (info.strides[0] != 1) throw std::runtime_error("Incompatible format in python buffer: 1-D buffer is not contiguous.");
    return info;
}

template <typename T> T buffer_to_texture(py::buffer buf, int w, int h) {
    T out(w, h, NoFill{});
    py::buffer_info info = request_bytes(buf, out.NBytes());
    std::memcpy(out.Data(), info.ptr, out.NBytes());
    return out;
}

template <typename T> T buffer_to_pod(py::buffer buf) {
    py::buffer_info info = request_bytes(buf, sizeof(T));
    T out;
    std::memcpy(&out, info.ptr, sizeof(T));
    return out;
}

int py_index(int v, int size, const char *name) {
    if (v < -size || v >= size) throw std::out_of_range(std::string(name) + " value out of range");
    return v < 0 ? size + v : v;
}

template <typename Cls, typename Get, typename Set, typename Ext> void def_subscript_2d(Cls &c, Get get, Set set, Ext ext) {
    using T = typename Cls::type;
    using V = decltype((std::declval<T &>().*get)(0, 0));
    c.def(
        "__getitem__",
        [get, ext](T &self, std::tuple<int, int> k) {
            auto s = (self.*ext)();
            return (self.*get)(py_index(std::get<0>(k), std::get<0>(s), "x"), py_index(std::get<1>(k), std::get<1>(s), "y"));
        },
        "key"_a);
    c.def(
        "__setitem__",
        [set, ext](T &self, std::tuple<int, int> k, const V &v) {
            auto s = (self.*ext)();
            (self.*set)(py_index(std::get<0>(k), std::get<0>(s), "x"), py_index(std::get<1>(k), std::get<1>(s), "y"), v);
        },
        "key"_a, "value"_a);
}

template <typename B> py::class_<B> bind_block(py::module_ &m, const char *name) {
    py::class_<B> c(m, name, py::buffer_protocol());
    c.def_static("frombytes", &buffer_to_pod<B>, "data"_a, "Create a new block by copying a bytes-like object.");
    c.def_property_readonly_static("width", [](py::object) { return B::Width; });
    c.def_property_readonly_static("height", [](py::object) { return B::Height; });
    c.def_property_readonly_static("size", [](py::object) { return std::make_tuple(B::Width, B::Height); });
    c.def_property_readonly_static("nbytes", [](py::object) { return sizeof(B); });
    c.def(py::self == py::self);
    c.def_buffer([](B &b) { return py::buffer_info(reinterpret_cast<uint8_t *>(&b), sizeof(B)); });
    c.def("tobytes", [](const B &b) { return py::bytes(reinterpret_cast<const char *>(&b), sizeof(B)); });
    return c;
}

template <typename B> py::class_<BlockTexture<B>, Texture> bind_block_texture(py::module_ &m, const char *name) {
    using T = BlockTexture<B>;
    py::class_<T, Texture> c(m, name);
    c.def(py::init<int, int>(), "width"_a, "height"_a);
    c.def_static("from_bytes", &buffer_to_texture<T>, "data"_a, "width"_a, "height"_a);
    // no reference counterpart: a texture whose blocks the caller writes next (a device-to-host
    // copy straight into its storage), without the zero fill
    c.def_static("_uninitialized", [](int w, int h) { return T(w, h, NoFill{}); }, "width"_a, "height"_a);
    c.def_property_readonly("width_blocks", &T::BlocksX);
    c.def_property_readonly("height_blocks", &T::BlocksY);
    c.def_property_readonly("size_blocks", &T::BlocksXY);
    def_subscript_2d(c, &T::GetBlock, &T::SetBlock, &T::BlocksXY);
    return c;
}

}  // namespace qtb

using namespace qtb;

PYBIND11_MODULE(_quicktex, m) {
    m.doc() = "B200 (sm_100a) S3TC encode/decode behind the quicktex module interface";
    m.attr("__version__") = qt_version();

    py::class_<Texture> texture(m, "Texture", py::buffer_protocol());
    texture.def_property_readonly("nbytes", &Texture::NBytes);
    texture.def_property_readonly("size", &Texture::Size);
    texture.def_property_readonly("width", &Texture::Width);
    texture.def_property_readonly("height", &Texture::Height);
    texture.def_buffer([](Texture &t) { return py::buffer_info(t.Data(), (py::ssize_t)t.NBytes()); });
    texture.def("tobytes", [](const Texture &t) { return py::bytes(reinterpret_cast<const char *>(t.Data()), t.NBytes()); });

    py::class_<RawTexture, Texture> raw(m, "RawTexture");
    raw.def(py::init<int, int>(), "width"_a, "height"_a);
    raw.def_static("frombytes", &buffer_to_texture<RawTexture>, "data"_a, "width"_a, "height"_a);
    def_subscript_2d(raw, &RawTexture::GetPixel, &RawTexture::SetPixel, &RawTexture::Size);

    py::module_ s3tc = m.def_submodule("_s3tc", "S3TC block compression on B200");

    // interpolators
    py::module_ mi = s3tc.def_submodule("_interpolator", "BC1 interpolation modes");
    py::class_<Interpolator, std::shared_ptr<Interpolator>> ideal(mi, "Interpolator");
    ideal.def(py::init<>());
    py::class_<InterpolatorRound, Interpolator, std::shared_ptr<InterpolatorRound>>(mi, "InterpolatorRound").def(py::init<>());
    py::class_<InterpolatorNvidia, Interpolator, std::shared_ptr<InterpolatorNvidia>>(mi, "InterpolatorNvidia").def(py::init<>());
    py::class_<InterpolatorAMD, Interpolator, std::shared_ptr<InterpolatorAMD>>(mi, "InterpolatorAMD").def(py::init<>());

    // BC1
    py::module_ m1 = s3tc.def_submodule("_bc1", "BC1");
    auto b1 = bind_block<BC1Block>(m1, "BC1Block");
    b1.def(py::init<>());
    b1.def(py::init([](Color c0, Color c1, const Sel4x4 &s) {
               BC1Block b;
               b.SetColors({c0, c1});
               b.SetSelectors(s);
               return b;
           }),
           "color0"_a, "color1"_a, "selectors"_a);
    b1.def_property("endpoints", &BC1Block::GetColors, &BC1Block::SetColors);
    b1.def_property("selectors", &BC1Block::GetSelectors, &BC1Block::SetSelectors);
    b1.def_property_readonly("is_3color", &BC1Block::Is3Color);
    bind_block_texture<BC1Block>(m1, "BC1Texture");

    py::class_<BC1Encoder, std::shared_ptr<BC1Encoder>> e1(m1, "BC1Encoder");
    py::enum_<EndpointMode>(e1, "EndpointMode")
        .value("LeastSquares", EndpointMode::LeastSquares)
        .value("BoundingBox", EndpointMode::BoundingBox)
        .value("BoundingBoxInt", EndpointMode::BoundingBoxInt)
        .value("PCA", EndpointMode::PCA);
    py::enum_<ErrorMode>(e1, "ErrorMode")
        .value("None", ErrorMode::None)
        .value("Faster", ErrorMode::Faster)
        .value("Check2", ErrorMode::Check2)
        .value("Full", ErrorMode::Full);
    py::enum_<ColorMode>(e1, "ColorMode")
        .value("FourColor", ColorMode::FourColor)
        .value("ThreeColor", ColorMode::ThreeColor)
        .value("ThreeColorBlack", ColorMode::ThreeColorBlack);
    e1.def(py::init<unsigned, ColorMode>(), "level"_a = 5, "color_mode"_a = ColorMode::FourColor);
    e1.def(py::init<unsigned, ColorMode, InterpolatorPtr>(), "level"_a, "color_mode"_a, "interpolator"_a);
    e1.def("encode", &BC1Encoder::Encode, "texture"_a);
    e1.def("set_level", &BC1Encoder::SetLevel, "level"_a);
    e1.def_property_readonly("interpolator", &BC1Encoder::GetInterpolator);
    e1.def_property_readonly("color_mode", &BC1Encoder::GetColorMode);
    e1.def_property("error_mode", &BC1Encoder::GetErrorMode, &BC1Encoder::SetErrorMode);
    e1.def_property("endpoint_mode", &BC1Encoder::GetEndpointMode, &BC1Encoder::SetEndpointMode);
    const char *flags[4] = {"two_ls_passes", "two_ep_passes", "two_cf_passes", "exhaustive"};
    for (int i = 0; i < 4; i++)
        e1.def_property(flags[i], [i](const BC1Encoder &e) { return e.GetFlag(i); }, [i](BC1Encoder &e, bool v) { e.SetFlag(i, v); });
    e1.def_property("search_rounds", &BC1Encoder::GetSearchRounds, &BC1Encoder::SetSearchRounds);
    e1.def_property("orderings", &BC1Encoder::GetOrderings, &BC1Encoder::SetOrderings);
    e1.def_property_readonly_static("max_power_iterations", [](py::object) { return BC1Encoder::max_power_iterations; });
    e1.def_property_readonly_static("min_power_iterations", [](py::object) { return BC1Encoder::min_power_iterations; });
    e1.def_property("power_iterations", &BC1Encoder::GetPowerIterations, &BC1Encoder::SetPowerIterations);

    py::class_<BC1Decoder, std::shared_ptr<BC1Decoder>> d1(m1, "BC1Decoder");
    d1.def(py::init<bool>(), "write_alpha"_a = false);
    d1.def(py::init<bool, InterpolatorPtr>(), "write_alpha"_a, "interpolator"_a);
    d1.def("decode", &BC1Decoder::Decode, "texture"_a);
    d1.def_property_readonly("interpolator", &BC1Decoder::GetInterpolator);
    d1.def_readwrite("write_alpha", &BC1Decoder::write_alpha);

    // BC4
    py::module_ m4 = s3tc.def_submodule("_bc4", "BC4");
    auto b4 = bind_block<BC4Block>(m4, "BC4Block");
    b4.def(py::init<>());
    b4.def(py::init([](uint8_t a0, uint8_t a1, const Sel4x4 &s) {
               BC4Block b;
               b.SetAlphas({a0, a1});
               b.SetSelectors(s);
               return b;
           }),
           "endpoint0"_a, "endpoint1"_a, "selectors"_a);
    b4.def_property("endpoints", &BC4Block::GetAlphas, &BC4Block::SetAlphas);
    b4.def_property("selectors", &BC4Block::GetSelectors, &BC4Block::SetSelectors);
    b4.def_property_readonly("values", &BC4Block::GetValues);
    b4.def_property_readonly("is_6value", &BC4Block::Is6Value);
    bind_block_texture<BC4Block>(m4, "BC4Texture");
    py::class_<BC4Encoder, std::shared_ptr<BC4Encoder>> e4(m4, "BC4Encoder");
    e4.def(py::init<uint8_t>(), "channel"_a = 3);
    e4.def("encode", &BC4Encoder::Encode, "texture"_a);
    e4.def_property_readonly("channel", &BC4Encoder::GetChannel);
    py::class_<BC4Decoder, std::shared_ptr<BC4Decoder>> d4(m4, "BC4Decoder");
    d4.def(py::init<uint8_t>(), "channel"_a = 3);
    d4.def("decode", &BC4Decoder::Decode, "texture"_a);
    d4.def_property_readonly("channel", &BC4Decoder::GetChannel);

    // BC3
    py::module_ m3 = s3tc.def_submodule("_bc3", "BC3");
    auto b3 = bind_block<BC3Block>(m3, "BC3Block");
    b3.def(py::init<>());
    b3.def(py::init([](const BC4Block &a, const BC1Block &c) { return BC3Block{a, c}; }), "alpha_block"_a, "color_block"_a);
    b3.def_readwrite("alpha_block", &BC3Block::alpha_block);
    b3.def_readwrite("color_block", &BC3Block::color_block);
    b3.def_property("blocks", &BC3Block::GetBlocks, &BC3Block::SetBlocks);
    bind_block_texture<BC3Block>(m3, "BC3Texture");
    py::class_<BC3Encoder, std::shared_ptr<BC3Encoder>> e3(m3, "BC3Encoder");
    e3.def(py::init<unsigned>(), "level"_a = 5);
    e3.def(py::init<unsigned, InterpolatorPtr>(), "level"_a, "interpolator"_a);
    e3.def("encode", &BC3Encoder::Encode, "texture"_a);
    e3.def_property_readonly("bc1_encoder", &BC3Encoder::GetBC1Encoder);
    e3.def_property_readonly("bc4_encoder", &BC3Encoder::GetBC4Encoder);
    py::class_<BC3Decoder, std::shared_ptr<BC3Decoder>> d3(m3, "BC3Decoder");
    d3.def(py::init<>());
    d3.def(py::init<InterpolatorPtr>(), "interpolator"_a);
    d3.def("decode", &BC3Decoder::Decode, "texture"_a);
    d3.def_property_readonly("bc1_decoder", &BC3Decoder::GetBC1Decoder);
    d3.def_property_readonly("bc4_decoder", &BC3Decoder::GetBC4Decoder);

    // BC5
    py::module_ m5 = s3tc.def_submodule("_bc5", "BC5");
    auto b5 = bind_block<BC5Block>(m5, "BC5Block");
    b5.def(py::init<>());
    b5.def(py::init([](const BC4Block &a, const BC4Block &b) { return BC5Block{a, b}; }), "chan0_block"_a, "chan1_block"_a);
    b5.def_readwrite("chan0_block", &BC5Block::chan0_block);
    b5.def_readwrite("chan1_block", &BC5Block::chan1_block);
    b5.def_property("blocks", &BC5Block::GetBlocks, &BC5Block::SetBlocks);
    bind_block_texture<BC5Block>(m5, "BC5Texture");
    py::class_<BC5Encoder, std::shared_ptr<BC5Encoder>> e5(m5, "BC5Encoder");
    e5.def(py::init<uint8_t, uint8_t>(), "chan0"_a = 0, "chan1"_a = 1);
    e5.def("encode", &BC5Encoder::Encode, "texture"_a);
    e5.def_property_readonly("channels", &BC5Encoder::GetChannels);
    e5.def_property_readonly("bc4_encoders", &BC5Encoder::GetBC4Encoders);
    py::class_<BC5Decoder, std::shared_ptr<BC5Decoder>> d5(m5, "BC5Decoder");
    d5.def(py::init<uint8_t, uint8_t>(), "chan0"_a = 0, "chan1"_a = 1);
    d5.def("decode", &BC5Decoder::Decode, "texture"_a);
    d5.def_property_readonly("channels", &BC5Decoder::GetChannels);
    d5.def_property_readonly("bc4_decoders", &BC5Decoder::GetBC4Decoders);
}
