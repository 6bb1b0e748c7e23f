// qt_noalloc.cu — qt_batch_run_noalloc: the batched path without any device
// allocation.
//
// Who needs it: callers that must not allocate GPU memory when they encode —
// an engine or plugin that reserves its whole device budget at start-up and
// forbids allocation afterwards, a latency-critical loop that cannot afford the
// device-wide synchronisation cudaMalloc/cudaFree may imply, or code running
// under a host-side allocator lock. qt_batch_create allocates its queue
// (cudaMalloc, cudaHostAlloc); this entry point instead keeps the queue in a
// fixed array below, part of the library image on every GPU that loads it.
//
// Limits and rules:
//  - at most QT_NOALLOC_MAX_ITEMS textures per call (larger requests fail with
//    QT_ERR_ARG); the tiles are coarsened so that they always fit.
//  - every call reuses the same array and it keeps the last call's contents;
//    the queue head is rewritten to zero on each call. Calls whose GPU work
//    overlaps (e.g. on two streams) race on the array: order them on one
//    stream, or wait for one before issuing the next.
//  - the first call on a device looks up the array's device address (and
//    uploads the codec's constant tables if no other entry point did); make
//    that first call before any stream capture.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "qt_internal.h"

namespace {

constexpr size_t kCtlBytes = 256;
constexpr size_t kItemsBytes = (QT_NOALLOC_MAX_ITEMS * sizeof(qtk::BatchItemDev) + 255) / 256 * 256;
constexpr size_t kTilesBytes = (size_t)QT_NOALLOC_MAX_TILES * sizeof(qtk::TileDev);
static_assert(kCtlBytes + kItemsBytes + kTilesBytes <= QT_NOALLOC_SCRATCH_BYTES, "scratch layout exceeds its size");

// The device work queue of qt_batch_run_noalloc: [control (queue head, tile
// count) | texture descriptors | tiles]. In host code this name is only a
// handle for cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[QT_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch_addr[kMaxDevices];  // device address of g_noalloc_scratch, per device

// host staging: fixed arrays, reused by every call under g_mu (no heap)
qtk::BatchItemDev h_items[QT_NOALLOC_MAX_ITEMS];
qtk::TileDev h_tiles[QT_NOALLOC_MAX_TILES];
uint32_t h_ctl[2];

// tile size and relative per-block cost of an item, from the work its settings imply
void tile_rule(const qt_batch_item &it, uint32_t *tile_blocks, float *cost) {
    if (it.op != QT_OP_ENCODE || it.format == 4 || it.format == 5) {
        *tile_blocks = 2048;
        *cost = it.op == QT_OP_ENCODE ? 0.1f : 0.05f;
        return;
    }
    const qt_bc1_params &p = it.params;
    float c = 1.5f;
    if (p.search_rounds >= 128) c = 25.f;
    else if (p.orderings4 >= 56 || p.search_rounds > 0) c = 15.f;
    else if (p.orderings4 >= 9) c = 4.f;
    else if (p.orderings4 >= 4) c = 2.f;
    *cost = c;
    *tile_blocks = c >= 15.f ? 32u : c >= 2.f ? 64u : 256u;
}

int check_item(const qt_batch_item &it) {
    const int f = it.format;
    if (it.op != QT_OP_ENCODE && it.op != QT_OP_DECODE) return qtk::set_error(QT_ERR_ARG, "batch item: invalid op");
    if (f != 1 && f != 3 && f != 4 && f != 5) return qtk::set_error(QT_ERR_ARG, "batch item: format must be 1, 3, 4 or 5");
    if (it.width <= 0) return qtk::set_error(QT_ERR_ARG, "Texture width must be greater than 0");
    if (it.height <= 0) return qtk::set_error(QT_ERR_ARG, "Texture height must be greater than 0");
    if (!it.src || !it.dst) return qtk::set_error(QT_ERR_ARG, "batch item: NULL buffer");
    const size_t bsz = (f == 3 || f == 5) ? 16 : 8;
    const size_t a_src = it.op == QT_OP_ENCODE ? 4 : bsz, a_dst = it.op == QT_OP_ENCODE ? bsz : 4;
    if (reinterpret_cast<uintptr_t>(it.src) % a_src || reinterpret_cast<uintptr_t>(it.dst) % a_dst)
        return qtk::set_error(QT_ERR_ARG, "batch item: misaligned buffer");
    if (it.chan0 < 0 || it.chan0 > 3 || it.chan1 < 0 || it.chan1 > 3) return qtk::set_error(QT_ERR_ARG, "Channel out of range");
    if (it.op == QT_OP_DECODE && (it.interpolator < 0 || it.interpolator > 3))
        return qtk::set_error(QT_ERR_ARG, "Invalid interpolator type");
    if (it.op == QT_OP_ENCODE && (f == 1 || f == 3)) return qtk::check_bc1_params(&it.params, f == 3);
    return QT_OK;
}

}  // namespace

extern "C" int qt_batch_run_noalloc(const qt_batch_item *items, size_t n, void *stream) {
    if (n && !items) return qtk::set_error(QT_ERR_ARG, "items is NULL");
    if (n > QT_NOALLOC_MAX_ITEMS) {
        char msg[160];
        std::snprintf(msg, sizeof msg, "qt_batch_run_noalloc: %zu textures exceed its fixed limit of %d per call", n,
                      QT_NOALLOC_MAX_ITEMS);
        return qtk::set_error(QT_ERR_ARG, msg);
    }
    std::lock_guard<std::mutex> lk(g_mu);
    int dev = 0;
    if (int rc = qtk::ensure_current_device(&dev)) return rc;
    if (dev >= kMaxDevices) return qtk::set_error(QT_ERR_ARG, "device index out of range");
    if (!g_scratch_addr[dev]) {  // once per device, with that device current
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return qtk::cuda_error((int)e, "cudaGetSymbolAddress");
        g_scratch_addr[dev] = static_cast<unsigned char *>(p);
    }
    if (n == 0) return QT_OK;

    // every item is validated before its sizes are used: widths and heights are positive and
    // each texture's block count fits the 32-bit tile fields (as qt_batch_run requires)
    for (size_t i = 0; i < n; i++) {
        if (int rc = check_item(items[i])) return rc;
        const uint64_t nb = (uint64_t)((items[i].width + 3) / 4) * (uint64_t)((items[i].height + 3) / 4);
        if (nb > 0xFFFFFFFFull) return qtk::set_error(QT_ERR_ARG, "Texture too large");
    }
    // tiles coarsened (x2 at a time) until they fit the fixed queue; every item needs at least
    // one tile and n <= QT_NOALLOC_MAX_ITEMS < QT_NOALLOC_MAX_TILES, so a scale of 2^32 (one tile
    // per item) always fits and the loop ends by then
    uint64_t scale = 1;
    for (int round = 0; round <= 32; round++) {
        uint64_t tiles = 0;
        for (size_t i = 0; i < n; i++) {
            uint32_t tb;
            float c;
            tile_rule(items[i], &tb, &c);
            const uint64_t nb = (uint64_t)((items[i].width + 3) / 4) * (uint64_t)((items[i].height + 3) / 4);
            const uint64_t t = std::max<uint64_t>(1, tb * scale);
            tiles += (nb + t - 1) / t;
        }
        if (tiles <= QT_NOALLOC_MAX_TILES) break;
        scale *= 2;
    }
    uint32_t nt = 0;
    for (size_t i = 0; i < n; i++) {
        const qt_batch_item &it = items[i];
        qtk::BatchItemDev &d = h_items[i];
        d.src = it.src;
        d.dst = it.dst;
        d.w = it.width;
        d.h = it.height;
        d.bw = (it.width + 3) / 4;
        d.bh = (it.height + 3) / 4;
        d.op = it.op;
        d.fmt = it.format;
        d.c0 = (it.format == 4 || it.format == 5) ? it.chan0 : 0;
        d.c1 = it.format == 5 ? it.chan1 : d.c0;
        d.interp = it.interpolator;
        d.write_alpha = it.write_alpha != 0;
        d.p = it.params;
        uint32_t tb;
        float c;
        tile_rule(it, &tb, &c);
        const uint64_t t = std::max<uint64_t>(1, tb * scale);
        const uint64_t nb = (uint64_t)d.bw * d.bh;
        for (uint64_t s0 = 0; s0 < nb; s0 += t) {
            if (nt >= QT_NOALLOC_MAX_TILES) return qtk::set_error(QT_ERR_ARG, "qt_batch_run_noalloc: tile queue full");
            const uint32_t cnt = (uint32_t)std::min<uint64_t>(t, nb - s0);
            // pad carries the tile's cost for the ordering below; the kernel ignores it
            h_tiles[nt++] = {(uint32_t)i, (uint32_t)s0, cnt, (uint32_t)std::min(4.0e9f, c * (float)cnt)};
        }
    }
    std::sort(h_tiles, h_tiles + nt, [](const qtk::TileDev &a, const qtk::TileDev &b) {
        return a.pad != b.pad ? a.pad > b.pad : (a.item != b.item ? a.item < b.item : a.start < b.start);
    });
    h_ctl[0] = 0;  // queue head starts at zero on every call
    h_ctl[1] = nt;

    unsigned char *base = g_scratch_addr[dev];
    uint32_t *d_ctl = reinterpret_cast<uint32_t *>(base);
    qtk::BatchItemDev *d_items = reinterpret_cast<qtk::BatchItemDev *>(base + kCtlBytes);
    qtk::TileDev *d_tiles = reinterpret_cast<qtk::TileDev *>(base + kCtlBytes + kItemsBytes);
    cudaStream_t s = (cudaStream_t)stream;
    // copies from pageable host memory return once the source has been staged, so the fixed
    // host arrays may be refilled by the next call as soon as these return
    cudaError_t e;
    if ((e = cudaMemcpyAsync(d_items, h_items, n * sizeof(qtk::BatchItemDev), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_tiles, h_tiles, nt * sizeof(qtk::TileDev), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_ctl, h_ctl, sizeof h_ctl, cudaMemcpyHostToDevice, s)) != cudaSuccess)
        return qtk::cuda_error((int)e, "qt_batch_run_noalloc upload");
    const int lrc = qtk::launch_batch(d_items, d_tiles, d_ctl, 0, stream);
    return lrc ? qtk::cuda_error(lrc, "qt_batch_run_noalloc launch") : QT_OK;
}
