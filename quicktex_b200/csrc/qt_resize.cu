// qt_resize.cu — BILINEAR downsampling of RGBA8 textures for mip chains
// (qt_resize_bilinear_device in include/quicktex_cuda.h).
//
// quicktex builds each mip level with Pillow: image_utils.resize_no_premultiply
// (quicktex/image_utils.py:40-52) resizes the RGB bands and the alpha band
// separately with Image.resize(size, Image.BILINEAR), and dds.encode
// (quicktex/dds.py:275-280) resizes the ORIGINAL image to every level. Pillow's
// resampler treats each band alike, so the result equals resizing all four
// channels of the RGBA8 texture independently, which is what this file does.
//
// The arithmetic restates Pillow 12.2.0's separable fixed-point resampler
// (src/libImaging/Resample.c: precompute_coeffs, normalize_coeffs_8bpc,
// ImagingResampleHorizontal_8bpc / ImagingResampleVertical_8bpc,
// ImagingResampleInner), a third-party dependency of quicktex:
//   - per output coordinate: scale = in/out, filterscale = max(scale, 1),
//     support = filterscale (the triangle filter's support is 1), centre
//     (x + 0.5)*scale, taps [xmin, xmin + n) with xmin = (int)(centre - support
//     + 0.5) clamped to 0 and end (int)(centre + support + 0.5) clamped to the
//     input size; weight of tap t = tri((t + xmin - centre + 0.5)/filterscale),
//     tri(d) = max(0, 1 - |d|), each divided by their sum (in tap order) when
//     the sum is non-zero, all in double;
//   - weights to fixed point with 22 fraction bits, rounded half away from zero;
//   - each output value = clamp((2^21 + sum(value * weight)) >> 22, 0, 255), 32-bit;
//   - a horizontal pass over the source rows the vertical pass needs, to 8-bit
//     values, then a vertical pass; a pass whose size does not change is skipped.
// The weights are computed here on the host in double (x86-64, no FMA
// contraction), exactly as Pillow does, and the device applies them.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "qt_internal.h"

namespace {

constexpr int kPrecisionBits = 22;  // 32 - 8 - 2

struct Taps {
    int ksize = 0;
    std::vector<int2> bounds;  // per output coordinate: first tap, tap count
    std::vector<int32_t> kk;   // out * ksize fixed-point weights
};

double tri(double x) {
    if (x < 0.0) x = -x;
    return x < 1.0 ? 1.0 - x : 0.0;
}

Taps bilinear_taps(int in_size, int out_size) {
    Taps t;
    const float in0 = 0.0f, in1 = (float)in_size;
    const double scale = (double)(in1 - in0) / out_size;
    const double filterscale = scale < 1.0 ? 1.0 : scale;
    const double support = 1.0 * filterscale;
    t.ksize = (int)std::ceil(support) * 2 + 1;
    t.bounds.resize((size_t)out_size);
    t.kk.assign((size_t)out_size * t.ksize, 0);
    std::vector<double> k((size_t)t.ksize);
    for (int xx = 0; xx < out_size; xx++) {
        const double center = in0 + (xx + 0.5) * scale;
        double ww = 0.0;
        const double ss = 1.0 / filterscale;
        int xmin = (int)(center - support + 0.5);
        if (xmin < 0) xmin = 0;
        int xmax = (int)(center + support + 0.5);
        if (xmax > in_size) xmax = in_size;
        xmax -= xmin;
        for (int x = 0; x < xmax; x++) {
            const double w = tri((x + xmin - center + 0.5) * ss);
            k[(size_t)x] = w;
            ww += w;
        }
        for (int x = 0; x < xmax; x++)
            if (ww != 0.0) k[(size_t)x] /= ww;
        int32_t *row = t.kk.data() + (size_t)xx * t.ksize;
        for (int x = 0; x < xmax; x++) {
            const double v = k[(size_t)x];
            row[x] = v < 0 ? (int32_t)(-0.5 + v * (1 << kPrecisionBits)) : (int32_t)(0.5 + v * (1 << kPrecisionBits));
        }
        t.bounds[(size_t)xx] = make_int2(xmin, xmax);
    }
    return t;
}

__device__ __forceinline__ uint32_t clip8(int v) {
    v >>= kPrecisionBits;
    return (uint32_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
}

__device__ __forceinline__ uint32_t weighted(int s0, int s1, int s2, int s3) {
    return clip8(s0) | (clip8(s1) << 8) | (clip8(s2) << 16) | (clip8(s3) << 24);
}

// rows [y0, y0 + gridDim.y * k) of src (width w) -> dst rows [0, ...) of width dw
__global__ void __launch_bounds__(256) k_resample_h(const uint32_t *__restrict__ src, int w, int y0, int rows,
                                                    uint32_t *__restrict__ dst, int dw, const int2 *__restrict__ bounds,
                                                    const int32_t *__restrict__ kk, int ksize) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= dw) return;
    const int2 b = bounds[x];
    const int32_t *k = kk + (size_t)x * ksize;
    for (int y = blockIdx.y; y < rows; y += gridDim.y) {
        const uint32_t *row = src + (size_t)(y0 + y) * w + b.x;
        int s0 = 1 << (kPrecisionBits - 1), s1 = s0, s2 = s0, s3 = s0;
        for (int t = 0; t < b.y; t++) {
            const uint32_t p = __ldg(row + t);
            const int c = __ldg(k + t);
            s0 += (int)(p & 0xFF) * c;
            s1 += (int)((p >> 8) & 0xFF) * c;
            s2 += (int)((p >> 16) & 0xFF) * c;
            s3 += (int)(p >> 24) * c;
        }
        dst[(size_t)y * dw + x] = weighted(s0, s1, s2, s3);
    }
}

// src (width w, rows indexed by the shifted bounds) -> dst (w x dh)
__global__ void __launch_bounds__(256) k_resample_v(const uint32_t *__restrict__ src, int w, uint32_t *__restrict__ dst,
                                                    int dh, const int2 *__restrict__ bounds,
                                                    const int32_t *__restrict__ kk, int ksize) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= w) return;
    for (int yy = blockIdx.y; yy < dh; yy += gridDim.y) {
        const int2 b = bounds[yy];
        const int32_t *k = kk + (size_t)yy * ksize;
        int s0 = 1 << (kPrecisionBits - 1), s1 = s0, s2 = s0, s3 = s0;
        for (int t = 0; t < b.y; t++) {
            const uint32_t p = __ldg(src + (size_t)(b.x + t) * w + x);
            const int c = __ldg(k + t);
            s0 += (int)(p & 0xFF) * c;
            s1 += (int)((p >> 8) & 0xFF) * c;
            s2 += (int)((p >> 16) & 0xFF) * c;
            s3 += (int)(p >> 24) * c;
        }
        dst[(size_t)yy * w + x] = weighted(s0, s1, s2, s3);
    }
}

// Wide filters (the deep levels of a chain resize the original by up to its full
// size, so one output sums thousands of taps): the taps of one output are split
// over several threads and their partial sums added. The sums are exact 32-bit
// integers, so the order of the additions does not change the result.

// horizontal: one warp per output pixel, lanes stride over the taps (coalesced row reads)
__global__ void __launch_bounds__(256) k_resample_h_wide(const uint32_t *__restrict__ src, int w, int y0, int rows,
                                                         uint32_t *__restrict__ dst, int dw,
                                                         const int2 *__restrict__ bounds,
                                                         const int32_t *__restrict__ kk, int ksize) {
    const int lane = threadIdx.x & 31;
    const long nout = (long)dw * rows;
    for (long o = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; o < nout; o += ((long)gridDim.x * blockDim.x) >> 5) {
        const int y = (int)(o / dw), x = (int)(o - (long)y * dw);
        const int2 b = bounds[x];
        const int32_t *k = kk + (size_t)x * ksize;
        const uint32_t *row = src + (size_t)(y0 + y) * w + b.x;
        int s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int t = lane; t < b.y; t += 32) {
            const uint32_t p = __ldg(row + t);
            const int c = __ldg(k + t);
            s0 += (int)(p & 0xFF) * c;
            s1 += (int)((p >> 8) & 0xFF) * c;
            s2 += (int)((p >> 16) & 0xFF) * c;
            s3 += (int)(p >> 24) * c;
        }
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
            s0 += __shfl_xor_sync(0xffffffffu, s0, d);
            s1 += __shfl_xor_sync(0xffffffffu, s1, d);
            s2 += __shfl_xor_sync(0xffffffffu, s2, d);
            s3 += __shfl_xor_sync(0xffffffffu, s3, d);
        }
        if (lane == 0) {
            const int half = 1 << (kPrecisionBits - 1);
            dst[(size_t)y * dw + x] = weighted(s0 + half, s1 + half, s2 + half, s3 + half);
        }
    }
}

// vertical: a CTA of 32 columns x 8 tap groups; the 8 partial sums of a column meet in shared memory
__global__ void __launch_bounds__(256) k_resample_v_wide(const uint32_t *__restrict__ src, int w,
                                                         uint32_t *__restrict__ dst, int dh,
                                                         const int2 *__restrict__ bounds,
                                                         const int32_t *__restrict__ kk, int ksize) {
    __shared__ int4 part[8][32];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int x = blockIdx.x * 32 + tx;
    for (int yy = blockIdx.y; yy < dh; yy += gridDim.y) {
        const int2 b = bounds[yy];
        const int32_t *k = kk + (size_t)yy * ksize;
        int s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        if (x < w)
            for (int t = ty; t < b.y; t += 8) {
                const uint32_t p = __ldg(src + (size_t)(b.x + t) * w + x);
                const int c = __ldg(k + t);
                s0 += (int)(p & 0xFF) * c;
                s1 += (int)((p >> 8) & 0xFF) * c;
                s2 += (int)((p >> 16) & 0xFF) * c;
                s3 += (int)(p >> 24) * c;
            }
        part[ty][tx] = make_int4(s0, s1, s2, s3);
        __syncthreads();
        if (ty == 0 && x < w) {
            const int half = 1 << (kPrecisionBits - 1);
            int4 a = make_int4(half, half, half, half);
#pragma unroll
            for (int g = 0; g < 8; g++) {
                a.x += part[g][tx].x;
                a.y += part[g][tx].y;
                a.z += part[g][tx].z;
                a.w += part[g][tx].w;
            }
            dst[(size_t)yy * w + x] = weighted(a.x, a.y, a.z, a.w);
        }
        __syncthreads();
    }
}

constexpr int kWideTaps = 16;  // above this many taps per output, the split kernels run

dim3 grid_2d(int x, int y) { return dim3((unsigned)((x + 255) / 256), (unsigned)(y < 65535 ? y : 65535)); }

void resample_h(const uint32_t *in, int w, int y0, int rows, uint32_t *out, int dw, const int2 *b, const int32_t *k,
                int ksize, cudaStream_t s) {
    if (ksize > kWideTaps) {
        const long warps = (long)dw * rows;
        const long ctas = std::min<long>((warps + 7) / 8, 148L * 64);
        k_resample_h_wide<<<(unsigned)ctas, 256, 0, s>>>(in, w, y0, rows, out, dw, b, k, ksize);
    } else {
        k_resample_h<<<grid_2d(dw, rows), 256, 0, s>>>(in, w, y0, rows, out, dw, b, k, ksize);
    }
}

void resample_v(const uint32_t *in, int w, uint32_t *out, int dh, const int2 *b, const int32_t *k, int ksize,
                cudaStream_t s) {
    if (ksize > kWideTaps)
        k_resample_v_wide<<<dim3((unsigned)((w + 31) / 32), (unsigned)(dh < 65535 ? dh : 65535)), 256, 0, s>>>(
            in, w, out, dh, b, k, ksize);
    else
        k_resample_v<<<grid_2d(w, dh), 256, 0, s>>>(in, w, out, dh, b, k, ksize);
}

}  // namespace

extern "C" int qt_resize_bilinear_device(const uint8_t *src, int w, int h, uint8_t *dst, int dw, int dh, void *stream) {
    if (!src || !dst) return qtk::set_error(QT_ERR_ARG, "NULL buffer");
    if (w <= 0 || h <= 0 || dw <= 0 || dh <= 0) return qtk::set_error(QT_ERR_ARG, "Texture sizes must be greater than 0");
    if ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 3)
        return qtk::set_error(QT_ERR_ARG, "resize: buffers must be 4-byte aligned");
    if (int rc = qtk::ensure_current_device(nullptr)) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (dw == w && dh == h) {  // Image.resize to the same size returns a copy
        e = cudaMemcpyAsync(dst, src, (size_t)w * h * 4, cudaMemcpyDeviceToDevice, s);
        return e == cudaSuccess ? QT_OK : qtk::cuda_error((int)e, "resize copy");
    }
    const bool need_h = dw != w, need_v = dh != h;
    const Taps th = bilinear_taps(w, dw);
    Taps tv = bilinear_taps(h, dh);
    const int y_first = tv.bounds[0].x, y_last = tv.bounds[(size_t)dh - 1].x + tv.bounds[(size_t)dh - 1].y;
    if (need_h)
        for (int2 &b : tv.bounds) b.x -= y_first;  // the vertical pass reads the horizontal pass's rows

    // one buffer for both tap tables (stream-ordered, freed after the passes); every table
    // starts on a 16-byte boundary (the bounds are read as 8-byte int2)
    const auto al = [](size_t n) { return (n + 15) / 16 * 16; };
    const size_t bh = th.bounds.size() * sizeof(int2), kh = th.kk.size() * sizeof(int32_t);
    const size_t bv = tv.bounds.size() * sizeof(int2), kv = tv.kk.size() * sizeof(int32_t);
    const size_t o_kh = al(bh), o_bv = al(o_kh + kh), o_kv = al(o_bv + bv);
    std::vector<uint8_t> host(o_kv + kv);
    std::memcpy(host.data(), th.bounds.data(), bh);
    std::memcpy(host.data() + o_kh, th.kk.data(), kh);
    std::memcpy(host.data() + o_bv, tv.bounds.data(), bv);
    std::memcpy(host.data() + o_kv, tv.kk.data(), kv);
    uint8_t *d_taps = nullptr;
    uint32_t *d_tmp = nullptr;
    const int tmp_rows = y_last - y_first;
    if ((e = qtk::scratch_alloc((void **)&d_taps, host.size(), s)) != cudaSuccess) return qtk::cuda_error((int)e, "resize taps");
    // from pageable memory: the call returns once `host` has been staged
    e = cudaMemcpyAsync(d_taps, host.data(), host.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && need_h && need_v) e = qtk::scratch_alloc((void **)&d_tmp, (size_t)dw * tmp_rows * 4, s);
    if (e == cudaSuccess) {
        const int2 *b_h = reinterpret_cast<const int2 *>(d_taps);
        const int32_t *k_h = reinterpret_cast<const int32_t *>(d_taps + o_kh);
        const int2 *b_v = reinterpret_cast<const int2 *>(d_taps + o_bv);
        const int32_t *k_v = reinterpret_cast<const int32_t *>(d_taps + o_kv);
        const uint32_t *in = reinterpret_cast<const uint32_t *>(src);
        uint32_t *out = reinterpret_cast<uint32_t *>(dst);
        if (need_h && need_v) {
            resample_h(in, w, y_first, tmp_rows, d_tmp, dw, b_h, k_h, th.ksize, s);
            resample_v(d_tmp, dw, out, dh, b_v, k_v, tv.ksize, s);
        } else if (need_h) {
            resample_h(in, w, 0, h, out, dw, b_h, k_h, th.ksize, s);
        } else {
            resample_v(in, w, out, dh, b_v, k_v, tv.ksize, s);
        }
        e = cudaGetLastError();
    }
    qtk::scratch_free(d_tmp, s);
    qtk::scratch_free(d_taps, s);
    return e == cudaSuccess ? QT_OK : qtk::cuda_error((int)e, "resize");
}

// ---------------------------------------------------------------------------
// Vertical flip and the BC3nm swizzle of the command-line encoder
// (quicktex/cli/encode.py:52-58: image.transpose(FLIP_TOP_BOTTOM), then
// Image.merge('RGBA', (255, band c1, band c1, band c0))), one texel per thread.
// ---------------------------------------------------------------------------
namespace {

__global__ void __launch_bounds__(256) k_flip_swizzle(const uint32_t *__restrict__ src, int w, int h,
                                                      uint32_t *__restrict__ dst, int flip, int c0, int c1) {
    const long n = (long)w * h;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int y = (int)(i / w), x = (int)(i - (long)y * w);
        uint32_t v = __ldg(src + (size_t)(flip ? h - 1 - y : y) * w + x);
        if (c0 >= 0) {
            const uint32_t a = (v >> (8 * c0)) & 0xFF, g = (v >> (8 * c1)) & 0xFF;
            v = 0xFFu | (g << 8) | (g << 16) | (a << 24);
        }
        dst[i] = v;
    }
}

}  // namespace

extern "C" int qt_flip_swizzle_device(const uint8_t *src, int w, int h, uint8_t *dst, int flip, int c0, int c1,
                                      void *stream) {
    if (!src || !dst) return qtk::set_error(QT_ERR_ARG, "NULL buffer");
    if (w <= 0 || h <= 0) return qtk::set_error(QT_ERR_ARG, "Texture sizes must be greater than 0");
    if ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 3)
        return qtk::set_error(QT_ERR_ARG, "flip/swizzle: buffers must be 4-byte aligned");
    if (c0 >= 0 && (c0 > 3 || c1 < 0 || c1 > 3)) return qtk::set_error(QT_ERR_ARG, "Channel out of range");
    const size_t bytes = (size_t)w * h * 4;
    if (src < dst + bytes && dst < src + bytes) return qtk::set_error(QT_ERR_ARG, "flip/swizzle: buffers overlap");
    if (int rc = qtk::ensure_current_device(nullptr)) return rc;
    const long n = (long)w * h;
    long blocks = (n + 255) / 256;
    if (blocks > 148L * 64) blocks = 148L * 64;
    k_flip_swizzle<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<const uint32_t *>(src), w, h,
                                                                     reinterpret_cast<uint32_t *>(dst), flip != 0,
                                                                     c0 >= 0 ? c0 : -1, c1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? QT_OK : qtk::cuda_error((int)e, "flip/swizzle");
}
