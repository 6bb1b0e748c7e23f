/*
 * quicktex_cuda.h — C-ABI of the B200 (sm_100a) S3TC encode/decode path.
 *
 * This is the drop-in boundary under the `_quicktex` Python module: every
 * entry point replaces one call of the reference codec (drewcassidy/quicktex
 * v0.3.1), cited beside it as `file:line` relative to the reference project
 * root. Plain pointers and sizes only: no C++ or torch types cross it.
 *
 * Conventions
 *  - Return value: QT_OK (0) or a QT_ERR_* status; qt_last_error() gives a
 *    thread-local message for the last failing call on the calling thread.
 *  - Textures are RGBA8, row-major, width*height*4 bytes (RawTexture,
 *    quicktex/Texture.h:64-141). Block textures are row-major arrays of
 *    ceil(w/4)*ceil(h/4) blocks of 8 (BC1, BC4) or 16 (BC3, BC5) bytes
 *    (BlockTexture, quicktex/Texture.h:143-184), in the reference's wire
 *    layout (BC1Block.h:30-125, BC4Block.h:28-105, BC3Block.h:28-58,
 *    BC5Block.h:27-57).
 *  - Encoders read edge blocks with modulo wrap (Texture.h:89-112); decoders
 *    reproduce the reference's wrapped overwrite of edge texels
 *    (Texture.h:114-134 in Decoder.h:45-51 loop order).
 *  - `*_host` calls take HOST buffers and return when the result is in host
 *    memory. `*_device` calls take DEVICE buffers and only enqueue work on
 *    `stream` (a cudaStream_t, NULL = legacy default stream).
 *  - All calls are thread-safe. Each device's constant tables are uploaded
 *    on first use (or by qt_init).
 */
#ifndef QUICKTEX_CUDA_H
#define QUICKTEX_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the pybind layer maps them to the reference's Python exceptions) ---- */
#define QT_OK 0
#define QT_ERR_ARG 1     /* std::invalid_argument -> ValueError (e.g. BC1Encoder.cpp:48-50, 75) */
#define QT_ERR_OOM 2     /* device allocation failed -> MemoryError */
#define QT_ERR_CUDA 3    /* CUDA runtime error -> RuntimeError */
#define QT_ERR_TIMEOUT 4 /* a bounded wait expired -> RuntimeError */
#define QT_ERR_RANGE 5   /* std::out_of_range -> IndexError */
#define QT_ERR_STATE 6   /* object used in the wrong state -> RuntimeError */

/* ---- enum values: identical to the reference's (BC1Encoder.h:57-100, Interpolator.h:30) ---- */
#define QT_COLOR_THREE 0x03
#define QT_COLOR_FOUR 0x04
#define QT_COLOR_THREE_BLACK 0x13
#define QT_ERROR_NONE 0
#define QT_ERROR_FASTER 1
#define QT_ERROR_CHECK2 2
#define QT_ERROR_FULL 3
#define QT_ENDPOINT_LEAST_SQUARES 0
#define QT_ENDPOINT_BOUNDING_BOX 1
#define QT_ENDPOINT_BOUNDING_BOX_INT 2
#define QT_ENDPOINT_PCA 3
#define QT_INTERP_IDEAL 0
#define QT_INTERP_IDEAL_ROUND 1
#define QT_INTERP_NVIDIA 2
#define QT_INTERP_AMD 3

/* Resolved BC1 encoder settings: the state a BC1Encoder holds after its
 * constructor and setters (BC1Encoder.h:102-170). */
typedef struct qt_bc1_params {
    int32_t color_mode;       /* QT_COLOR_* */
    int32_t interpolator;     /* QT_INTERP_* */
    int32_t error_mode;       /* QT_ERROR_* */
    int32_t endpoint_mode;    /* QT_ENDPOINT_* */
    int32_t two_ls_passes;    /* bool */
    int32_t two_ep_passes;    /* bool */
    int32_t two_cf_passes;    /* bool */
    int32_t exhaustive;       /* bool */
    uint32_t search_rounds;   /* any value */
    uint32_t orderings4;      /* clamped to [1, 128] */
    uint32_t orderings3;      /* clamped to [1, 32] */
    uint32_t power_iterations;/* clamped to [4, 10] */
} qt_bc1_params;

/* Fills `out` with the settings of a preset level; replaces the
 * BC1Encoder(level, color_mode, interpolator) constructor and
 * BC1Encoder::SetLevel (BC1Encoder.cpp:47-71, 74-249). level > 19 or an
 * invalid colour mode / interpolator -> QT_ERR_ARG. */
int qt_bc1_params_for_level(unsigned level, int color_mode, int interpolator, qt_bc1_params *out);

/* Clamps and checks a params block the way the reference's setters do
 * (BC1Encoder.cpp:251-258). */
int qt_bc1_params_validate(qt_bc1_params *p);

/* Uploads the constant tables (ordering tables, factor matrices, single-colour
 * match tables: OrderTable.h:57-89, SingleColorTable.h:46-90) to `device`.
 * Optional: every entry point does it on first use of a device. */
int qt_init(int device);

const char *qt_last_error(void);

/* Library version string. */
const char *qt_version(void);

/* ---- encoders: BlockEncoder<T>::Encode (Encoder.h:36-56) ---- */

/* BC1Encoder::Encode -> EncodeBlock (BC1Encoder.cpp:261-342) per block.
 * On textures of 16384 blocks or more the device entry points first write the
 * solid blocks and list the others (stream-ordered scratch of 4 bytes per block
 * from the library's own memory pool, which keeps freed memory cached). */
int qt_bc1_encode_host(const uint8_t *rgba, int width, int height, const qt_bc1_params *params, uint8_t *blocks);
int qt_bc1_encode_device(const uint8_t *rgba, int width, int height, const qt_bc1_params *params, uint8_t *blocks,
                         void *stream);

/* BC3Encoder::Encode -> EncodeBlock (BC3Encoder.cpp:27-32): BC1 in four-colour
 * mode on RGB (params->color_mode is ignored) + BC4 on channel 3. */
int qt_bc3_encode_host(const uint8_t *rgba, int width, int height, const qt_bc1_params *params, uint8_t *blocks);
int qt_bc3_encode_device(const uint8_t *rgba, int width, int height, const qt_bc1_params *params, uint8_t *blocks,
                         void *stream);

/* No reference counterpart: host memory for texture storage from the library's cache of
 * pinned (page-locked) blocks. The *_host entry points copy pinned buffers with the copy
 * engines directly; pageable buffers go through a pinned staging ring first, which costs
 * about as much again on a large texture. A block is page-locked once, when first
 * allocated, and a freed block stays cached for the next allocation of its size class
 * (sizes round up by at most 12.5%; up to 2 GiB stay cached). Blocks under 256 KiB, and
 * all blocks where no pinned memory can be had (no usable GPU, or the system's limit), are
 * ordinary memory, which the entry points stage as usual. Thread-safe. qt_host_free ignores NULL and pointers it did
 * not hand out. The drop-in texture classes keep their texels here. */
int qt_host_alloc(size_t bytes, void **ptr);
void qt_host_free(void *ptr);

/* No reference counterpart: the number of kernels one qt_bc1_encode_device or
 * qt_bc3_encode_device call on a width x height texture launches on the current
 * device with these params (1 = the encoder; 2 = a split pass that writes the solid
 * blocks, then the encoder; 4 = split, encoder, EndpointSearch as its own pass, then a
 * pass that finishes the searches that moved the endpoints; 5 = the same with the
 * second cluster-fit pass of level 18 as its own pass). The host entry points launch
 * this per band. params->color_mode is not checked. */
int qt_bc1_encode_kernels(int width, int height, const qt_bc1_params *params, int *kernels);

/* BC4Encoder(channel)::Encode -> EncodeBlock (BC4Encoder.cpp:30-71). */
int qt_bc4_encode_host(const uint8_t *rgba, int width, int height, int channel, uint8_t *blocks);
int qt_bc4_encode_device(const uint8_t *rgba, int width, int height, int channel, uint8_t *blocks, void *stream);

/* BC5Encoder(chan0, chan1)::Encode -> EncodeBlock (BC5Encoder.cpp:25-30). */
int qt_bc5_encode_host(const uint8_t *rgba, int width, int height, int chan0, int chan1, uint8_t *blocks);
int qt_bc5_encode_device(const uint8_t *rgba, int width, int height, int chan0, int chan1, uint8_t *blocks,
                         void *stream);

/* ---- decoders: BlockDecoder<T>::Decode (Decoder.h:36-54) ---- */

/* BC1Decoder(write_alpha, interpolator)::Decode (BC1Decoder.cpp:31-52). */
int qt_bc1_decode_host(const uint8_t *blocks, int width, int height, int interpolator, int write_alpha, uint8_t *rgba);
int qt_bc1_decode_device(const uint8_t *blocks, int width, int height, int interpolator, int write_alpha,
                         uint8_t *rgba, void *stream);

/* BC3Decoder(interpolator)::Decode (BC3Decoder.cpp:26-32). */
int qt_bc3_decode_host(const uint8_t *blocks, int width, int height, int interpolator, uint8_t *rgba);
int qt_bc3_decode_device(const uint8_t *blocks, int width, int height, int interpolator, uint8_t *rgba, void *stream);

/* BC4Decoder(channel)::Decode (BC4Decoder.cpp:29-50); other channels become (0,0,0,255). */
int qt_bc4_decode_host(const uint8_t *blocks, int width, int height, int channel, uint8_t *rgba);
int qt_bc4_decode_device(const uint8_t *blocks, int width, int height, int channel, uint8_t *rgba, void *stream);

/* BC5Decoder(chan0, chan1)::Decode (BC5Decoder.cpp:25-30). */
int qt_bc5_decode_host(const uint8_t *blocks, int width, int height, int chan0, int chan1, uint8_t *rgba);
int qt_bc5_decode_device(const uint8_t *blocks, int width, int height, int chan0, int chan1, uint8_t *rgba,
                         void *stream);

/* ---- batched persistent path (no reference counterpart: the reference runs one
 * texture per Encode/Decode call, Encoder.h:36-56 / Decoder.h:36-54) ----
 *
 * Many textures of any size, format and level in one launch: every texture is
 * cut into tiles of consecutive blocks (tile size per format/level from a tuning
 * table), the tiles are queued heaviest-first in device memory, and one
 * persistent kernel, replayed from a captured CUDA graph, pulls tiles until the
 * queue is empty. Each texture's output is byte-identical to the single-texture
 * entry points above. */
#define QT_OP_ENCODE 0
#define QT_OP_DECODE 1

typedef struct qt_batch qt_batch;

typedef struct qt_batch_item {
    int32_t op;            /* QT_OP_ENCODE or QT_OP_DECODE */
    int32_t format;        /* 1 = BC1, 3 = BC3, 4 = BC4, 5 = BC5 */
    int32_t width, height; /* texture size in texels */
    const uint8_t *src;    /* device: RGBA8 texels (encode) or blocks (decode) */
    uint8_t *dst;          /* device: blocks (encode) or RGBA8 texels (decode) */
    qt_bc1_params params;  /* BC1/BC3 encode settings */
    int32_t chan0, chan1;  /* BC4 (chan0) / BC5 channels */
    int32_t interpolator;  /* BC1/BC3 decode */
    int32_t write_alpha;   /* BC1 decode */
} qt_batch_item;

/* Tuning rule: tiles of `tile_blocks` blocks and a relative cost per block for
 * (op, format, level); level is ignored for BC4/BC5 and decodes (-1). */
typedef struct qt_tile_rule {
    int32_t op, format, level;
    uint32_t tile_blocks;
    float cost_per_block;
} qt_tile_rule;

int qt_batch_create(int device, qt_batch **out);
int qt_batch_destroy(qt_batch *b);
/* Replace the tuning rules (rules not given keep their defaults). */
int qt_batch_set_rules(qt_batch *b, const qt_tile_rule *rules, size_t n);
/* Persistent grid size in CTAs per SM (0 = the kernel's occupancy limit). */
int qt_batch_set_grid(qt_batch *b, int ctas_per_sm);
/* Threads per CTA of the persistent kernel: 32, 64 or 128 (the default). Work is
 * claimed per warp, so the outputs do not depend on it. */
int qt_batch_set_threads(qt_batch *b, int threads_per_cta);
/* Enqueue one persistent launch over all items on `stream` (device buffers; the
 * call returns once the work is queued). */
int qt_batch_run(qt_batch *b, const qt_batch_item *items, size_t n, void *stream);
/* Number of tiles the last qt_batch_run queued. */
size_t qt_batch_last_tiles(const qt_batch *b);
/* The launch model the batch replaces, for comparison: the same items, one
 * single-texture device entry point call (qt_bc{1,3,4,5}_encode_device /
 * _decode_device) per texture in a native loop, on `stream`. The reference's
 * counterpart is one Encode/Decode call per texture (Encoder.h:36-56,
 * Decoder.h:36-54). Same output bytes as qt_batch_run. */
int qt_batch_run_plain(const qt_batch_item *items, size_t n, void *stream);
/* Size the queue for up to `items` textures and `tiles` tiles now, so that later
 * runs within those limits never reallocate it (a reallocation waits for the
 * device and re-captures the graph). Never shrinks the queue. */
int qt_batch_reserve(qt_batch *b, size_t items, size_t tiles);

/* Many copies in one call (serving front ends staging request payloads): one
 * cudaMemcpyAsync per entry on `stream`, direction taken from the pointers
 * (cudaMemcpyDefault). Host memory should be pinned for the copies to be
 * asynchronous. No counterpart in the reference. */
typedef struct qt_copy {
    void *dst;
    const void *src;
    size_t bytes;
} qt_copy;
int qt_copy_async(const qt_copy *copies, size_t n, void *stream);

/* ---- mip chains ----
 *
 * BILINEAR resize of an RGBA8 texture (w x h -> dw x dh), each channel on its
 * own: the mip-level resize of quicktex's dds.encode / image_utils
 * (quicktex/image_utils.py:40-52 resize_no_premultiply, quicktex/dds.py:275-280),
 * which is Pillow's Image.resize(size, Image.BILINEAR); byte-identical to it.
 * Device buffers, 4-byte aligned; enqueued on `stream` (temporary tap tables
 * and the intermediate rows come from the library's stream-ordered memory pool). */
int qt_resize_bilinear_device(const uint8_t *src, int w, int h, uint8_t *dst, int dw, int dh, void *stream);

/* Vertical flip and/or BC3nm swizzle of an RGBA8 texture, as the command-line
 * encoder prepares images (quicktex/cli/encode.py:52-58): flip != 0 reverses the
 * row order (Image.FLIP_TOP_BOTTOM); c0 >= 0 writes (255, in[c1], in[c1], in[c0])
 * (Image.merge('RGBA', (one, bands[1], bands[1], bands[0])) with the bands at
 * channels c0, c1); c0 < 0 leaves the texels as they are. Device buffers, 4-byte
 * aligned, not overlapping; enqueued on `stream`. */
int qt_flip_swizzle_device(const uint8_t *src, int w, int h, uint8_t *dst, int flip, int c0, int c1, void *stream);

/* ---- serving: continuous batching on one GPU (no counterpart in the reference) ----
 *
 * A qt_server owns a device arena of `memory_budget` bytes, `slots` batch
 * queues with a stream each, and a worker thread. qt_server_submit queues
 * requests and returns at once: each is a qt_batch_item whose src and dst are
 * HOST buffers (the payload and the response buffer; pinned memory makes the
 * copies asynchronous), kept valid by the caller until the request completes.
 * Whenever a slot is free the worker folds the waiting requests, in arrival
 * order, that fit the largest free range of the arena and the batch caps into
 * one persistent launch on that slot's stream: payload uploads, qt_batch_run,
 * response downloads. Batches on different slots overlap on the device.
 * Finished requests are reported by qt_server_poll with their tag, status and
 * completion time. A request needing more than the whole budget completes at
 * once with QT_ERR_RANGE. Response bytes equal those of the single-texture
 * entry points. */
typedef struct qt_server qt_server;
typedef struct qt_server_stats {
    uint64_t batches, requests_done, blocks_done;
    uint32_t max_inflight, pending, inflight, slots;
} qt_server_stats;
int qt_server_create(int device, size_t memory_budget, int slots, size_t max_batch_blocks, size_t max_batch_requests,
                     qt_server **out);
/* Runs every request already submitted to completion, then frees the server. */
int qt_server_destroy(qt_server *s);
/* Tuning rules / grid / CTA size of every slot's queue (as qt_batch_set_rules,
 * qt_batch_set_grid, qt_batch_set_threads). */
int qt_server_set_rules(qt_server *s, const qt_tile_rule *rules, size_t n);
int qt_server_set_grid(qt_server *s, int ctas_per_sm);
int qt_server_set_threads(qt_server *s, int threads_per_cta);
/* Queue n requests; tags[i] is reported with request i's completion. All or
 * nothing: an invalid request -> QT_ERR_ARG and none is queued. */
int qt_server_submit(qt_server *s, const qt_batch_item *items, const uint64_t *tags, size_t n);
/* Up to `cap` completions: tag, status (QT_OK or an error code) and completion
 * time (seconds of qt_server_clock). Waits up to timeout_us (0: no wait) for
 * the first one; *n receives the count. */
int qt_server_poll(qt_server *s, uint64_t *tags, int32_t *status, double *t_done, size_t cap, int64_t timeout_us,
                   size_t *n);
int qt_server_get_stats(qt_server *s, qt_server_stats *out);
/* CLOCK_MONOTONIC in seconds: the clock of the completion times. */
double qt_server_clock(void);

/* ---- the batched path without device allocation (no counterpart in the reference) ----
 *
 * For callers that may not allocate GPU memory when they encode: engines that
 * reserve their whole device budget at start-up, latency-critical loops that
 * cannot take the device-wide synchronisation cudaMalloc/cudaFree may cause,
 * code running under a host allocator lock. Same work and same output bytes as
 * qt_batch_run, but the work queue lives in a fixed array of
 * QT_NOALLOC_SCRATCH_BYTES (384 KiB) inside the library, held on every GPU that
 * loads it until the process exits; the call makes no cudaMalloc/cudaFree and
 * creates no batch object. Inputs and outputs are the caller's device buffers.
 *  - At most QT_NOALLOC_MAX_ITEMS textures per call; more -> QT_ERR_ARG.
 *  - All calls share the one queue, which keeps the last call's contents (its
 *    head is reset on every call): calls whose GPU work overlaps race, so issue
 *    them on one stream or wait for the previous one.
 *  - The first call on a device sets up the queue's device address (and the
 *    constant tables); make it before any stream capture. */
#define QT_NOALLOC_MAX_ITEMS 1024
#define QT_NOALLOC_MAX_TILES 16384
#define QT_NOALLOC_SCRATCH_BYTES (384 * 1024)
int qt_batch_run_noalloc(const qt_batch_item *items, size_t n, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* QUICKTEX_CUDA_H */
