// Internal interface between the host C-ABI (qt_capi.cpp) and the kernels
// translation unit (qt_kernels.cu). Not part of the public boundary.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "quicktex_cuda.h"

namespace qtk {

// Host image of the device-resident constant tables.
struct alignas(16) HostTables {
    uint16_t best4[969 * 128];  // OrderTable<4>::BestOrders (OrderTable4.cpp:996-1965)
    uint16_t best3[153 * 32];   // OrderTable<3>::BestOrders (OrderTable.cpp:165-320)
    uint16_t hash4[4096];       // histogram -> ordering index (OrderTable.h:64)
    uint16_t hash3[256];
    float factors4[969][4];     // 2x2 LS inverse per ordering (OrderTable.h:65-83)
    float factors3[153][4];
    uint32_t orders4[969];      // histogram bytes h0 | h1<<8 | h2<<16 | h3<<24
    uint32_t orders3[153];
    uint32_t match5[4][256];    // single-colour tables per interpolator: high | low<<8 | err<<16
    uint32_t match6[4][256];
};

// Device descriptor of one texture of a batch (built from qt_batch_item).
struct BatchItemDev {
    const uint8_t *src;
    uint8_t *dst;
    int32_t w, h, bw, bh;
    int32_t op;           // QT_OP_ENCODE / QT_OP_DECODE
    int32_t fmt;          // 1, 3, 4, 5
    int32_t c0, c1;       // BC4/BC5 channels
    int32_t interp;       // decode interpolator
    int32_t write_alpha;  // BC1 decode
    qt_bc1_params p;      // BC1/BC3 encode settings
};

// One unit of the device work queue: `count` consecutive blocks of item `item`.
struct TileDev {
    uint32_t item, start, count, pad;
};

// Builds the tables on the host (the factor matrices with the reference's
// float operation order) from the embedded ordering-table blob.
const HostTables &host_tables();

// Shared host helpers (qt_capi.cpp): thread-local error message, status codes,
// per-device table upload on the current device, argument checks.
int set_error(int code, const char *msg);
int cuda_error(int cuda_status, const char *what);
int ensure_current_device(int *dev);
int check_bc1_params(const qt_bc1_params *p, bool bc3);
// Checks of a qt_batch_item other than its buffers: op, format, size, channels,
// interpolator and BC1 settings (qt_batch.cpp).
int check_item_fields(const qt_batch_item &it);
// Stream-ordered scratch from the library's own memory pool on the current
// device (its release threshold is unlimited, so freed memory stays cached
// for the next call instead of going back to the driver at every sync).
cudaError_t scratch_alloc(void **ptr, size_t bytes, cudaStream_t stream);
cudaError_t scratch_free(void *ptr, cudaStream_t stream);

// Kernel-side entry points (qt_kernels.cu). Each returns a cudaError_t value
// cast to int (0 on success). All pointers are device pointers.
int upload_tables(int device);

int launch_bc1_encode(const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3,
                      void *stream);
int launch_bc4_encode(const uint8_t *rgba, int w, int h, int c0, int c1, bool bc5, uint8_t *out, void *stream);
// the same over the blocks [b_begin, b_end) of the texture only (row-major block indices)
int launch_bc1_encode_range(const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3,
                            long b_begin, long b_end, void *stream);
int launch_bc4_encode_range(const uint8_t *rgba, int w, int h, int c0, int c1, bool bc5, uint8_t *out, long b_begin,
                            long b_end, void *stream);
// The fewest blocks for which a BC1/BC3 launch with EndpointSearch runs the search as its own
// refill pass (two searches per resident lane of that pass).
long defer_min_blocks();
// BC1/BC3 encode of one texture whose texels arrive in parts (the row bands of a host upload),
// on the deferred path: bc1_parts_begin allocates and clears the shared scratch on `stream`;
// bc1_parts_add runs the split pass and the encoder over the blocks [b_begin, b_end) on its
// stream once that part's texels are there (the stream ordered after begin's); bc1_parts_end,
// on a stream ordered after every part, runs the second cluster-fit pass, EndpointSearch and the
// finish pass over all parts' queues, then frees the scratch. The result equals one
// launch_bc1_encode over the texture. Only where bc1_parts_eligible holds (settings with
// EndpointSearch, defer_min_blocks() to 2^32 blocks), in at most 32 parts; bc1_parts_free
// releases the scratch after a failure.
struct Bc1Parts {
    uint32_t *scratch = nullptr;
    long n = 0;
    bool cf2 = false;
    int parts = 0;
};
bool bc1_parts_eligible(long nblocks, const qt_bc1_params &p);
int bc1_parts_begin(Bc1Parts &ps, long nblocks, const qt_bc1_params &p, void *stream);
int bc1_parts_add(Bc1Parts &ps, const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3,
                  long b_begin, long b_end, void *stream);
int bc1_parts_end(Bc1Parts &ps, const uint8_t *rgba, int w, int h, const qt_bc1_params &p, uint8_t *out, bool bc3,
                  void *stream);
void bc1_parts_free(Bc1Parts &ps, void *stream);
// kernels one launch_bc1_encode_range over n blocks issues (0 for none): the encoder, plus the
// split pass from kSplitMinBlocks blocks, plus the search pass from defer_min_blocks() blocks
int bc1_encode_kernels(long n, const qt_bc1_params &p);
int launch_decode_range(int fmt, const uint8_t *blocks, int w, int h, int interp, int write_alpha, int c0, int c1,
                        uint8_t *rgba, long b_begin, long b_end, void *stream);
// fmt: 1 = BC1, 3 = BC3, 4 = BC4, 5 = BC5
int launch_decode(int fmt, const uint8_t *blocks, int w, int h, int interp, int write_alpha, int c0, int c1,
                  uint8_t *rgba, void *stream);

// Persistent batch kernel: warps pull tiles from tiles[0 .. ctl[1]) through the
// counter ctl[0] until the queue is empty. grid = CTAs to launch (0 = one wave).
int launch_batch(const BatchItemDev *items, const TileDev *tiles, uint32_t *ctl, int grid, void *stream);
// the same with `threads` per CTA (32, 64 or 128; work is claimed per warp, so any of them
// runs the same tiles); grid <= 0 fills the SMs to the kernel's occupancy at that size
int launch_batch(const BatchItemDev *items, const TileDev *tiles, uint32_t *ctl, int grid, int threads, void *stream);
int batch_ctas_per_sm();
int batch_sms();

}  // namespace qtk
