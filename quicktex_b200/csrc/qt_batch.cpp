// qt_batch.cpp — host side of the batched persistent path (qt_batch_* in
// include/quicktex_cuda.h).
//
// A qt_batch owns, per device: the device work queue (texture descriptors,
// tiles, and a two-word control block: queue head and tile count), pinned
// host staging for it, and a CUDA graph holding the persistent kernel launch.
// Every qt_batch_run cuts the textures into tiles (tile size per format/level
// from the tuning rules), orders the tiles by estimated cost, heaviest first
// (so the long L18 tiles start early and the cheap ones fill the tail),
// uploads the queue, and replays the graph. The graph is re-captured only
// when a queue buffer has to grow.

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "qt_internal.h"

namespace {

constexpr int kLevels = 20;
int fmt_index(int fmt) { return fmt == 1 ? 0 : fmt == 3 ? 1 : fmt == 4 ? 2 : fmt == 5 ? 3 : -1; }
int rule_index(int op, int fmt, int level) {
    const int l = (op == QT_OP_ENCODE && (fmt == 1 || fmt == 3)) ? std::min(std::max(level, 0), kLevels - 1) : 0;
    return (op * 4 + fmt_index(fmt)) * kLevels + l;
}

struct Rule {
    uint32_t tile_blocks;
    float cost;
};

// The preset level whose settings these are (exact match on the fields a
// level sets), else the preset closest in cluster-fit orderings and search
// rounds; used only to pick a tuning rule.
int qtk_level_of(const qt_bc1_params &p) {
    int best = 0;
    long best_d = -1;
    for (int l = 0; l < kLevels; l++) {
        qt_bc1_params q;
        if (qt_bc1_params_for_level((unsigned)l, QT_COLOR_FOUR, 0, &q) != QT_OK) continue;
        if (q.error_mode == p.error_mode && q.endpoint_mode == p.endpoint_mode && q.two_ls_passes == p.two_ls_passes &&
            q.two_ep_passes == p.two_ep_passes && q.two_cf_passes == p.two_cf_passes && q.exhaustive == p.exhaustive &&
            q.search_rounds == p.search_rounds && q.orderings4 == p.orderings4 && q.orderings3 == p.orderings3 &&
            q.power_iterations == p.power_iterations)
            return l;
        const long d = std::labs((long)q.orderings4 * (q.two_cf_passes ? 2 : 1) - (long)p.orderings4 * (p.two_cf_passes ? 2 : 1)) +
                       std::labs((long)q.search_rounds - (long)p.search_rounds) / 4;
        if (best_d < 0 || d < best_d) {
            best_d = d;
            best = l;
        }
    }
    return p.exhaustive ? 19 : best;
}

}  // namespace

struct qt_batch {
    int device = 0;
    std::mutex mu;
    Rule rules[2 * 4 * kLevels];
    int ctas_per_sm = 0;
    int threads = 128;  // per CTA of the persistent kernel
    size_t cap_items = 0, cap_tiles = 0, last_tiles = 0;
    qtk::BatchItemDev *d_items = nullptr, *h_items = nullptr;
    qtk::TileDev *d_tiles = nullptr, *h_tiles = nullptr;
    uint32_t *d_ctl = nullptr, *h_ctl = nullptr;
    cudaEvent_t staged = nullptr;     // the last upload from the pinned staging buffers
    cudaEvent_t done = nullptr;       // the last persistent launch (the queue is in use until then)
    cudaStream_t capture = nullptr;   // private stream the graph is captured on
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;

    qt_batch() {
        for (int op = 0; op < 2; op++)
            for (int f : {1, 3, 4, 5})
                for (int l = 0; l < kLevels; l++) {
                    Rule &r = rules[rule_index(op, f, l)];
                    // a warp takes one tile; tiles are multiples of its 32 lanes
                    if (op == QT_OP_DECODE) {
                        r = {2048, 0.05f};
                    } else if (f == 4 || f == 5) {
                        r = {2048, 0.1f};
                    } else {  // BC1 / BC3 encode: cost grows steeply with the level's cluster fit and search
                        const float c = l >= 17 ? 25.f : l >= 13 ? 15.f : l >= 9 ? 4.f : l >= 7 ? 2.f : l >= 1 ? 1.5f : 1.f;
                        r = {l >= 13 ? 32u : l >= 7 ? 64u : 256u, c + (f == 3 ? 0.1f : 0.f)};
                    }
                }
    }
};

namespace {

void free_buffers(qt_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    cudaFree(b->d_items);
    cudaFree(b->d_tiles);
    cudaFreeHost(b->h_items);
    cudaFreeHost(b->h_tiles);
    b->d_items = b->h_items = nullptr;
    b->d_tiles = b->h_tiles = nullptr;
    b->cap_items = b->cap_tiles = 0;
}

int grow(qt_batch *b, size_t items, size_t tiles) {
    if (items <= b->cap_items && tiles <= b->cap_tiles && b->d_items) return QT_OK;
    if (b->staged) cudaEventSynchronize(b->staged);
    cudaDeviceSynchronize();  // the old queue may still be read by a running launch
    const size_t ni = std::max(items, std::max<size_t>(b->cap_items * 2, 64));
    const size_t nt = std::max(tiles, std::max<size_t>(b->cap_tiles * 2, 1024));
    free_buffers(b);
    cudaError_t e;
    if ((e = cudaMalloc(&b->d_items, ni * sizeof(qtk::BatchItemDev))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_tiles, nt * sizeof(qtk::TileDev))) != cudaSuccess ||
        (e = cudaHostAlloc((void **)&b->h_items, ni * sizeof(qtk::BatchItemDev), cudaHostAllocDefault)) != cudaSuccess ||
        (e = cudaHostAlloc((void **)&b->h_tiles, nt * sizeof(qtk::TileDev), cudaHostAllocDefault)) != cudaSuccess) {
        free_buffers(b);
        cudaGetLastError();
        return qtk::cuda_error((int)e, "allocating the batch queue");
    }
    b->cap_items = ni;
    b->cap_tiles = nt;
    return QT_OK;
}

int check_item(const qt_batch_item &it) {
    if (int rc = qtk::check_item_fields(it)) return rc;
    if (!it.src || !it.dst) return qtk::set_error(QT_ERR_ARG, "batch item: NULL buffer");
    const size_t bsz = (it.format == 3 || it.format == 5) ? 16 : 8;
    const size_t a_src = it.op == QT_OP_ENCODE ? 4 : bsz, a_dst = it.op == QT_OP_ENCODE ? bsz : 4;
    if (reinterpret_cast<uintptr_t>(it.src) % a_src || reinterpret_cast<uintptr_t>(it.dst) % a_dst)
        return qtk::set_error(QT_ERR_ARG, "batch item: misaligned buffer");
    return QT_OK;
}

}  // namespace

int qtk::check_item_fields(const qt_batch_item &it) {
    if (it.op != QT_OP_ENCODE && it.op != QT_OP_DECODE) return qtk::set_error(QT_ERR_ARG, "batch item: invalid op");
    if (fmt_index(it.format) < 0) return qtk::set_error(QT_ERR_ARG, "batch item: format must be 1, 3, 4 or 5");
    if (it.width <= 0) return qtk::set_error(QT_ERR_ARG, "Texture width must be greater than 0");
    if (it.height <= 0) return qtk::set_error(QT_ERR_ARG, "Texture height must be greater than 0");
    if (it.chan0 < 0 || it.chan0 > 3 || it.chan1 < 0 || it.chan1 > 3) return qtk::set_error(QT_ERR_ARG, "Channel out of range");
    if (it.op == QT_OP_DECODE && (it.interpolator < 0 || it.interpolator > 3))
        return qtk::set_error(QT_ERR_ARG, "Invalid interpolator type");
    if (it.op == QT_OP_ENCODE && (it.format == 1 || it.format == 3)) return qtk::check_bc1_params(&it.params, it.format == 3);
    return QT_OK;
}

extern "C" {

int qt_batch_create(int device, qt_batch **out) {
    if (!out) return qtk::set_error(QT_ERR_ARG, "out is NULL");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return qtk::cuda_error((int)e, "cudaSetDevice");
    int rc = qtk::ensure_current_device(nullptr);
    qt_batch *b = nullptr;
    if (rc == QT_OK) {
        b = new qt_batch();
        b->device = device;
        if ((e = cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaMalloc(&b->d_ctl, 2 * sizeof(uint32_t))) != cudaSuccess ||
            (e = cudaHostAlloc((void **)&b->h_ctl, 2 * sizeof(uint32_t), cudaHostAllocDefault)) != cudaSuccess) {
            rc = qtk::cuda_error((int)e, "creating a batch");
            qt_batch_destroy(b);
            b = nullptr;
        }
    }
    cudaSetDevice(prev);
    *out = b;
    return rc;
}

int qt_batch_destroy(qt_batch *b) {
    if (!b) return QT_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    free_buffers(b);
    cudaFree(b->d_ctl);
    cudaFreeHost(b->h_ctl);
    if (b->staged) cudaEventDestroy(b->staged);
    if (b->done) cudaEventDestroy(b->done);
    if (b->capture) cudaStreamDestroy(b->capture);
    cudaSetDevice(prev);
    delete b;
    return QT_OK;
}

int qt_batch_set_rules(qt_batch *b, const qt_tile_rule *rules, size_t n) {
    if (!b || (n && !rules)) return qtk::set_error(QT_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(b->mu);
    for (size_t i = 0; i < n; i++) {
        const qt_tile_rule &r = rules[i];
        if ((r.op != QT_OP_ENCODE && r.op != QT_OP_DECODE) || fmt_index(r.format) < 0 || r.tile_blocks == 0 ||
            !(r.cost_per_block > 0))
            return qtk::set_error(QT_ERR_ARG, "invalid tile rule");
        const bool leveled = r.op == QT_OP_ENCODE && (r.format == 1 || r.format == 3);
        const int l0 = (leveled && r.level >= 0) ? r.level : 0, l1 = (leveled && r.level >= 0) ? r.level : kLevels - 1;
        for (int l = l0; l <= l1; l++) b->rules[rule_index(r.op, r.format, l)] = {r.tile_blocks, r.cost_per_block};
    }
    return QT_OK;
}

int qt_batch_set_grid(qt_batch *b, int ctas_per_sm) {
    if (!b || ctas_per_sm < 0) return qtk::set_error(QT_ERR_ARG, "invalid grid");
    std::lock_guard<std::mutex> lk(b->mu);
    if (ctas_per_sm != b->ctas_per_sm && b->exec) {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
    }
    b->ctas_per_sm = ctas_per_sm;
    return QT_OK;
}

int qt_batch_set_threads(qt_batch *b, int threads_per_cta) {
    if (!b || (threads_per_cta != 32 && threads_per_cta != 64 && threads_per_cta != 128))
        return qtk::set_error(QT_ERR_ARG, "threads per CTA must be 32, 64 or 128");
    std::lock_guard<std::mutex> lk(b->mu);
    if (threads_per_cta != b->threads && b->exec) {
        cudaGraphExecDestroy(b->exec);
        cudaGraphDestroy(b->graph);
        b->exec = nullptr;
        b->graph = nullptr;
    }
    b->threads = threads_per_cta;
    return QT_OK;
}

size_t qt_batch_last_tiles(const qt_batch *b) { return b ? b->last_tiles : 0; }

int qt_copy_async(const qt_copy *copies, size_t n, void *stream) {
    if (n && !copies) return qtk::set_error(QT_ERR_ARG, "copies is NULL");
    for (size_t i = 0; i < n; i++) {
        if (!copies[i].bytes) continue;
        if (!copies[i].dst || !copies[i].src) return qtk::set_error(QT_ERR_ARG, "qt_copy_async: NULL buffer");
        const cudaError_t e = cudaMemcpyAsync(copies[i].dst, copies[i].src, copies[i].bytes, cudaMemcpyDefault,
                                              (cudaStream_t)stream);
        if (e != cudaSuccess) return qtk::cuda_error((int)e, "qt_copy_async");
    }
    return QT_OK;
}

int qt_batch_reserve(qt_batch *b, size_t items, size_t tiles) {
    if (!b) return qtk::set_error(QT_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(b->mu);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b->device) return qtk::set_error(QT_ERR_STATE, "qt_batch_reserve: the batch belongs to another device");
    return grow(b, std::max<size_t>(items, b->cap_items), std::max<size_t>(tiles, b->cap_tiles));
}

int qt_batch_run(qt_batch *b, const qt_batch_item *items, size_t n, void *stream) {
    if (!b || (n && !items)) return qtk::set_error(QT_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(b->mu);
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != b->device) return qtk::set_error(QT_ERR_STATE, "qt_batch_run: the batch belongs to another device");
    if (int rc = qtk::ensure_current_device(nullptr)) return rc;

    // descriptors, and tiles ordered heaviest first
    std::vector<qtk::BatchItemDev> dev(n);
    struct Tile {
        float cost;
        qtk::TileDev t;
    };
    std::vector<Tile> tiles;
    for (size_t i = 0; i < n; i++) {
        const qt_batch_item &it = items[i];
        if (int rc = check_item(it)) return rc;
        qtk::BatchItemDev &d = dev[i];
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
        const uint64_t nb = (uint64_t)d.bw * d.bh;
        if (nb > 0xFFFFFFFFull) return qtk::set_error(QT_ERR_ARG, "Texture too large");
        const bool leveled = it.op == QT_OP_ENCODE && (it.format == 1 || it.format == 3);
        const Rule &r = b->rules[rule_index(it.op, it.format, leveled ? qtk_level_of(it.params) : 0)];
        for (uint64_t s0 = 0; s0 < nb; s0 += r.tile_blocks) {
            const uint32_t cnt = (uint32_t)std::min<uint64_t>(r.tile_blocks, nb - s0);
            tiles.push_back({r.cost * cnt, {(uint32_t)i, (uint32_t)s0, cnt, 0u}});
        }
    }
    std::stable_sort(tiles.begin(), tiles.end(), [](const Tile &a, const Tile &c) { return a.cost > c.cost; });
    b->last_tiles = tiles.size();
    if (tiles.size() > 0xFFFFFFFFull) return qtk::set_error(QT_ERR_ARG, "too many tiles");
    if (tiles.empty()) return QT_OK;

    if (int rc = grow(b, n, tiles.size())) return rc;
    cudaError_t e = cudaEventSynchronize(b->staged);  // the staging buffers are free once the last upload ran
    if (e != cudaSuccess) return qtk::cuda_error((int)e, "batch staging");
    std::memcpy(b->h_items, dev.data(), n * sizeof(qtk::BatchItemDev));
    for (size_t i = 0; i < tiles.size(); i++) b->h_tiles[i] = tiles[i].t;
    b->h_ctl[0] = 0;
    b->h_ctl[1] = (uint32_t)tiles.size();
    cudaStream_t s = (cudaStream_t)stream;
    // runs on other streams: do not overwrite the queue before the previous launch finished reading it
    if ((e = cudaStreamWaitEvent(s, b->done, 0)) != cudaSuccess) return qtk::cuda_error((int)e, "batch ordering");
    if ((e = cudaMemcpyAsync(b->d_items, b->h_items, n * sizeof(qtk::BatchItemDev), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b->d_tiles, b->h_tiles, tiles.size() * sizeof(qtk::TileDev), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b->d_ctl, b->h_ctl, 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaEventRecord(b->staged, s)) != cudaSuccess)
        return qtk::cuda_error((int)e, "batch upload");

    if (!b->exec) {  // capture the persistent launch once; replays read the queue through fixed pointers
        const int grid = b->ctas_per_sm > 0 ? qtk::batch_sms() * b->ctas_per_sm : 0;
        if ((e = cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
            return qtk::cuda_error((int)e, "graph capture");
        const int lrc = qtk::launch_batch(b->d_items, b->d_tiles, b->d_ctl, grid, b->threads, b->capture);
        cudaGraph_t g = nullptr;
        e = cudaStreamEndCapture(b->capture, &g);
        if (lrc != 0) {
            if (g) cudaGraphDestroy(g);
            return qtk::cuda_error(lrc, "batch launch");
        }
        if (e != cudaSuccess) return qtk::cuda_error((int)e, "graph capture");
        if ((e = cudaGraphInstantiate(&b->exec, g, 0)) != cudaSuccess) {
            cudaGraphDestroy(g);
            b->exec = nullptr;
            return qtk::cuda_error((int)e, "graph instantiate");
        }
        b->graph = g;
    }
    if ((e = cudaGraphLaunch(b->exec, s)) != cudaSuccess) return qtk::cuda_error((int)e, "graph launch");
    if ((e = cudaEventRecord(b->done, s)) != cudaSuccess) return qtk::cuda_error((int)e, "graph launch");
    return QT_OK;
}

int qt_batch_run_plain(const qt_batch_item *items, size_t n, void *stream) {
    if (n && !items) return qtk::set_error(QT_ERR_ARG, "items is NULL");
    for (size_t i = 0; i < n; i++) {
        const qt_batch_item &it = items[i];
        if (int rc = check_item(it)) return rc;
        const int w = it.width, h = it.height, f = it.format;
        int rc;
        if (it.op == QT_OP_ENCODE) {
            rc = f == 1   ? qt_bc1_encode_device(it.src, w, h, &it.params, it.dst, stream)
                 : f == 3 ? qt_bc3_encode_device(it.src, w, h, &it.params, it.dst, stream)
                 : f == 4 ? qt_bc4_encode_device(it.src, w, h, it.chan0, it.dst, stream)
                          : qt_bc5_encode_device(it.src, w, h, it.chan0, it.chan1, it.dst, stream);
        } else {
            rc = f == 1   ? qt_bc1_decode_device(it.src, w, h, it.interpolator, it.write_alpha, it.dst, stream)
                 : f == 3 ? qt_bc3_decode_device(it.src, w, h, it.interpolator, it.dst, stream)
                 : f == 4 ? qt_bc4_decode_device(it.src, w, h, it.chan0, it.dst, stream)
                          : qt_bc5_decode_device(it.src, w, h, it.chan0, it.chan1, it.dst, stream);
        }
        if (rc) return rc;
    }
    return QT_OK;
}

}  // extern "C"
