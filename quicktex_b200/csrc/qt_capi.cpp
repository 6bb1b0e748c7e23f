// qt_capi.cpp — host side of the C-ABI declared in include/quicktex_cuda.h.
//
// Owns the constant tables (built once per process, uploaded once per
// device), a pooled device allocator for the host-buffer entry points, the
// pinned staging of pageable host buffers (a ring per host thread and device,
// a shared pool of copy threads), the cache of pinned host blocks behind
// qt_host_alloc, the thread-local error message, and argument
// checking with the reference's error semantics.
//
// Compiled as plain C++ on x86-64 with -ffp-contract=off: the factor matrices
// of the cluster-fit orderings are computed here with the reference's
// operation order (OrderTable.h:65-83) and must match it bit for bit.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "qt_internal.h"

namespace {
#include "qt_order_blob.inc"  // kOrderBlob[], kOrderBlobSize: quicktex_b200/data/bc1_order_tables.bin
}

namespace {

thread_local std::string g_err;

int set_err(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int cuda_err(cudaError_t e, const char *what) {
    if (e == cudaErrorMemoryAllocation) return set_err(QT_ERR_OOM, "%s: out of device memory", what);
    return set_err(QT_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

// ---------------------------------------------------------------------------
// constant tables
// ---------------------------------------------------------------------------
constexpr size_t kBlobOrders4 = 8, kBlobOrders3 = 8 + 969 * 4, kBlobBest4 = 4352, kBlobBest3 = 4352 + 969 * 128 * 2;

// Interpolators (Interpolator.cpp:47-138)
int interp8(int t, int a, int b) {
    if (t == QT_INTERP_IDEAL_ROUND) return (a * 2 + b + 1) / 3;
    if (t == QT_INTERP_AMD) return (a * 43 + b * 21 + 32) >> 6;
    return (a * 2 + b) / 3;
}
int s5to8(int v) { return (v << 3) | (v >> 2); }
int s6to8(int v) { return (v << 2) | (v >> 4); }
int nv5(int a, int b) { return ((2 * a + b) * 22) / 8; }
int nv6(int a, int b) { int gd = b - a; return (256 * a + (gd / 4) + 128 + gd * 80) >> 8; }

// SingleColorTable<B, N> (SingleColorTable.h:46-90); N does not enter the result.
void build_match(int t, int bits, uint32_t out[256]) {
    const int size = 1 << bits;
    const bool ideal = t == QT_INTERP_IDEAL || t == QT_INTERP_IDEAL_ROUND;
    const bool use8 = t != QT_INTERP_NVIDIA;
    for (int i = 0; i < 256; i++) {
        unsigned error = 256, lo_b = 0, hi_b = 0, err_b = 0;
        for (int lo = 0; lo < size; lo++) {
            const int lo8 = bits == 5 ? s5to8(lo) : s6to8(lo);
            for (int hi = 0; hi < size; hi++) {
                const int hi8 = bits == 5 ? s5to8(hi) : s6to8(hi);
                int value = use8 ? interp8(t, hi8, lo8) : (bits == 5 ? nv5(hi, lo) : nv6(hi, lo));
                value &= 0xFF;
                unsigned e = (unsigned)std::abs(value - i);
                if (ideal) e += (unsigned)(std::abs(hi8 - lo8) * 3) / 100;
                if (e < error || (e == error && lo == hi)) {
                    lo_b = (unsigned)lo;
                    hi_b = (unsigned)hi;
                    err_b = e;
                    error = e;
                }
            }
        }
        out[i] = hi_b | (lo_b << 8) | (err_b << 16);
    }
}

// OrderTable<N>::Generate (OrderTable.h:57-89)
void build_factors(int n, int count, const uint8_t *hist, float (*fac)[4], uint16_t *hashes, uint32_t *orders) {
    // OrderTable<N>::Weights (OrderTable.cpp:40-41): {s^2, s(n-1-s), s(n-1-s), (n-1-s)^2}
    const float w4[4][4] = {{0, 0, 0, 9}, {1, 2, 2, 4}, {4, 2, 2, 1}, {9, 0, 0, 0}};
    const float w3[3][4] = {{0, 0, 0, 4}, {1, 1, 1, 1}, {4, 0, 0, 0}};
    const float denom = n == 4 ? 3.0f : 2.0f;
    for (int i = 0; i < count; i++) {
        const uint8_t *h = hist + (size_t)i * n;
        bool any16 = false;
        unsigned packed = 0;
        uint32_t ord = 0;
        for (int s = 0; s < n; s++) {
            any16 |= h[s] == 16;
            ord |= (uint32_t)h[s] << (8 * s);
        }
        for (int s = 0; s < n - 1; s++) packed |= (unsigned)h[s] << (4 * s);
        if (!any16) hashes[packed] = (uint16_t)i;
        orders[i] = ord;
        float m[4] = {0, 0, 0, 0};
        for (int s = 0; s < n; s++) {
            const float *w = n == 4 ? w4[s] : w3[s];
            for (int k = 0; k < 4; k++) m[k] = m[k] + w[k] * (float)h[s];
        }
        const float det = (m[0] * m[3]) - (m[1] * m[2]);
        if (std::fabs(det) < 1e-8f) {
            fac[i][0] = fac[i][1] = fac[i][2] = fac[i][3] = 0.0f;
        } else {
            const float t = m[0];
            m[0] = m[3];
            m[3] = t;
            m[1] = m[1] * -1.0f;
            m[2] = m[2] * -1.0f;
            const float sc = (denom / 255.0f) / det;
            for (int k = 0; k < 4; k++) fac[i][k] = m[k] * sc;
        }
    }
}

qtk::HostTables *make_tables() {
    auto *t = new qtk::HostTables();
    std::memset(t, 0, sizeof *t);
    if (kOrderBlobSize != 262208 || std::memcmp(kOrderBlob, "QTOT", 4) != 0) {
        std::fprintf(stderr, "quicktex_cuda: embedded ordering tables are corrupt\n");
        std::abort();
    }
    const uint8_t *o4 = kOrderBlob + kBlobOrders4, *o3 = kOrderBlob + kBlobOrders3;
    // bit 15 flags the single-colour orderings (OrderTable<4>::SingleColorHashes {15, 700, 753, 515},
    // OrderTable<3>: {12, 15, 89}), so the encoder tests one bit per trial
    for (int i = 0; i < 969 * 128; i++) {
        const uint16_t h = (uint16_t)(kOrderBlob[kBlobBest4 + 2 * i] | (kOrderBlob[kBlobBest4 + 2 * i + 1] << 8));
        t->best4[i] = (uint16_t)(h | ((h == 15 || h == 700 || h == 753 || h == 515) ? 0x8000 : 0));
    }
    for (int i = 0; i < 153 * 32; i++) {
        const uint16_t h = (uint16_t)(kOrderBlob[kBlobBest3 + 2 * i] | (kOrderBlob[kBlobBest3 + 2 * i + 1] << 8));
        t->best3[i] = (uint16_t)(h | ((h == 12 || h == 15 || h == 89) ? 0x8000 : 0));
    }
    build_factors(4, 969, o4, t->factors4, t->hash4, t->orders4);
    build_factors(3, 153, o3, t->factors3, t->hash3, t->orders3);
    for (int it = 0; it < 4; it++) {
        build_match(it, 5, t->match5[it]);
        build_match(it, 6, t->match6[it]);
    }
    return t;
}

// ---------------------------------------------------------------------------
// per-device state and pooled device buffers
// ---------------------------------------------------------------------------
constexpr int kMaxDevices = 64;
std::mutex g_init_mu;
bool g_inited[kMaxDevices];

int ensure_device(int *dev_out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return set_err(QT_ERR_ARG, "device %d out of range", dev);
    if (dev_out) *dev_out = dev;
    std::lock_guard<std::mutex> lk(g_init_mu);
    if (g_inited[dev]) return QT_OK;
    int rc = qtk::upload_tables(dev);
    if (rc != 0) return cuda_err((cudaError_t)rc, "uploading tables");
    g_inited[dev] = true;
    return QT_OK;
}

// Size-class free lists of device buffers, per device. Buffers are kept for
// reuse (resident across calls) and handed out exclusively.
struct Pool {
    std::mutex mu;
    std::multimap<size_t, void *> free_[kMaxDevices];
};
Pool &pool() {
    static Pool *p = new Pool();
    return *p;
}

size_t size_class(size_t n) {
    size_t c = 4096;
    while (c < n) c <<= 1;
    return c;
}

struct DevBuf {
    void *ptr = nullptr;
    size_t cls = 0;
    int dev = 0;
    ~DevBuf() {
        if (ptr) {
            std::lock_guard<std::mutex> lk(pool().mu);
            pool().free_[dev].emplace(cls, ptr);
        }
    }
};

int acquire(DevBuf &b, int dev, size_t n) {
    b.dev = dev;
    b.cls = size_class(n);
    {
        std::lock_guard<std::mutex> lk(pool().mu);
        auto &fl = pool().free_[dev];
        auto it = fl.find(b.cls);
        if (it != fl.end()) {
            b.ptr = it->second;
            fl.erase(it);
            return QT_OK;
        }
    }
    cudaError_t e = cudaMalloc(&b.ptr, b.cls);
    if (e != cudaSuccess) {
        b.ptr = nullptr;
        cudaGetLastError();
        return cuda_err(e, "cudaMalloc");
    }
    return QT_OK;
}

// the library's stream-ordered scratch pool, one per device, created on first use
std::mutex g_mempool_mu;
cudaMemPool_t g_mempool[kMaxDevices];

// one non-blocking stream per host thread and device for the host-buffer calls
cudaStream_t thread_stream(int dev) {
    thread_local cudaStream_t streams[kMaxDevices] = {};
    if (!streams[dev]) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
    return streams[dev];
}

// ---------------------------------------------------------------------------
// argument checks (reference error texts where it has them)
// ---------------------------------------------------------------------------
int check_dims(int w, int h) {
    if (w <= 0) return set_err(QT_ERR_ARG, "Texture width must be greater than 0");
    if (h <= 0) return set_err(QT_ERR_ARG, "Texture height must be greater than 0");
    if ((long long)w * h > (1LL << 32)) return set_err(QT_ERR_ARG, "Texture too large");
    return QT_OK;
}
int check_channel(int c) {
    return (c < 0 || c > 3) ? set_err(QT_ERR_ARG, "Channel out of range") : QT_OK;
}
int check_interp(int t) {
    return (t < 0 || t > 3) ? set_err(QT_ERR_ARG, "Invalid interpolator type") : QT_OK;
}

int check_ptr(const void *p, size_t align, const char *what) {
    if (!p) return set_err(QT_ERR_ARG, "%s is NULL", what);
    if (reinterpret_cast<uintptr_t>(p) % align) return set_err(QT_ERR_ARG, "%s must be %zu-byte aligned", what, align);
    return QT_OK;
}

int finish_launch(int rc, const char *what) {
    return rc ? cuda_err((cudaError_t)rc, what) : QT_OK;
}

// ---------------------------------------------------------------------------
// Pageable host buffers. A copy from or to pageable memory goes through the CUDA
// driver's own small pinned buffer, filled by one CPU thread, and cudaMemcpyAsync
// returns only when it is done (about a quarter of the pinned-memory rate). The
// drop-in API hands over RawTexture / BlockTexture storage, a pageable std::vector,
// so the host-buffer entry points stage pageable buffers themselves: a ring of
// pinned chunks per host thread and device, filled and drained by a small pool of
// copy threads. The CPU copy of one chunk then overlaps the DMA of the others.
// ---------------------------------------------------------------------------
class CopyPool {
   public:
    static CopyPool &get() {
        static CopyPool *p = new CopyPool();  // never destroyed: its threads live until exit
        return *p;
    }
    // memcpy split over the pool's threads and the caller; returns when all of it is done
    void copy(void *dst, const void *src, size_t n) {
        const size_t kPiece = size_t(512) << 10;  // a band's chunk (~8 MB) still spreads over 12 threads
        const size_t pieces = std::min<size_t>(workers_ + 1, std::max<size_t>(1, n / kPiece));
        if (pieces <= 1) {
            std::memcpy(dst, src, n);
            return;
        }
        const size_t step = ((n + pieces - 1) / pieces + 63) & ~size_t(63);  // pieces * step >= n
        std::atomic<size_t> left(pieces - 1);
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (size_t k = 1; k < pieces; k++) {
                const size_t off = k * step;
                tasks_.push_back({static_cast<uint8_t *>(dst) + off, static_cast<const uint8_t *>(src) + off,
                                  off < n ? std::min(step, n - off) : 0, &left});
            }
            pending_.store(tasks_.size(), std::memory_order_release);
        }
        cv_.notify_all();
        std::memcpy(dst, src, std::min(step, n));
        while (left.load(std::memory_order_acquire) != 0) std::this_thread::yield();
    }

   private:
    struct Task {
        uint8_t *dst;
        const uint8_t *src;
        size_t n;
        std::atomic<size_t> *left;
    };
    // Host memcpy scales to ~12 threads on the 16-core GPU hosts measured (14 GB/s with one,
    // 48 with 8, 60 with 12); the pool takes three quarters of the cores, the caller one more.
    CopyPool() {
        const unsigned hw = std::thread::hardware_concurrency();
        workers_ = std::max(1u, std::min(11u, hw * 3 / 4 > 1 ? hw * 3 / 4 - 1 : 1u));
        for (unsigned i = 0; i < workers_; i++) std::thread([this] { run(); }).detach();
    }
    void run() {
        for (;;) {
            // copies come in bursts (one per staging chunk, a fraction of a millisecond apart):
            // poll a little before sleeping, so the next chunk's pieces start without a wake-up
            for (int spin = 0; spin < 2000 && pending_.load(std::memory_order_acquire) == 0; spin++)
                std::this_thread::yield();
            Task t;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [this] { return !tasks_.empty(); });
                t = tasks_.front();
                tasks_.pop_front();
                pending_.store(tasks_.size(), std::memory_order_release);
            }
            if (t.n) std::memcpy(t.dst, t.src, t.n);
            t.left->fetch_sub(1, std::memory_order_release);
        }
    }
    unsigned workers_ = 1;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Task> tasks_;
    std::atomic<size_t> pending_{0};
};

bool is_pageable(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

// Ring of pinned chunks of one host thread on one device. A chunk is reused only after the
// async copy through it finished (its event); a chunk that received device data is copied to
// its host destination then, or by flush().
struct Stage {
    static constexpr size_t kChunk = size_t(16) << 20;
    static constexpr int kChunks = 4;
    uint8_t *buf = nullptr;
    cudaEvent_t ev[kChunks] = {};
    bool busy[kChunks] = {};
    uint8_t *pend_dst[kChunks] = {};
    size_t pend_len[kChunks] = {};
    int next = 0;

    Stage() = default;
    Stage(const Stage &) = delete;
    Stage &operator=(const Stage &) = delete;
    ~Stage() {  // at thread exit: the ring's pinned memory and events go back (errors ignored:
                // at process exit the runtime may already be gone)
        if (!buf) return;
        flush();
        for (int j = 0; j < kChunks; j++)
            if (ev[j]) cudaEventDestroy(ev[j]);
        cudaFreeHost(buf);
        cudaGetLastError();
    }

    int init() {
        if (buf) return QT_OK;
        cudaError_t e = cudaHostAlloc((void **)&buf, kChunk * kChunks, cudaHostAllocDefault);
        for (int j = 0; j < kChunks && e == cudaSuccess; j++) e = cudaEventCreateWithFlags(&ev[j], cudaEventDisableTiming);
        if (e != cudaSuccess) {
            buf = nullptr;
            return cuda_err(e, "pinned staging buffer");
        }
        return QT_OK;
    }
    uint8_t *chunk(int j) { return buf + (size_t)j * kChunk; }
    int retire(int j) {
        if (!busy[j]) return QT_OK;
        const cudaError_t e = cudaEventSynchronize(ev[j]);
        busy[j] = false;
        if (e != cudaSuccess) return cuda_err(e, "staged copy");
        if (pend_len[j]) CopyPool::get().copy(pend_dst[j], chunk(j), pend_len[j]);
        pend_len[j] = 0;
        return QT_OK;
    }
    int take(int *j) {
        *j = next;
        next = (next + 1) % kChunks;
        return retire(*j);
    }
    int upload(void *dev, const uint8_t *host, size_t n, cudaStream_t s) {
        for (size_t off = 0; off < n; off += kChunk) {
            const size_t len = std::min(kChunk, n - off);
            int j, rc;
            if ((rc = take(&j))) return rc;
            CopyPool::get().copy(chunk(j), host + off, len);
            cudaError_t e = cudaMemcpyAsync(static_cast<uint8_t *>(dev) + off, chunk(j), len, cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaEventRecord(ev[j], s);
            if (e != cudaSuccess) return cuda_err(e, "host-to-device copy");
            busy[j] = true;
        }
        return QT_OK;
    }
    int download(uint8_t *host, const void *dev, size_t n, cudaStream_t s) {
        for (size_t off = 0; off < n; off += kChunk) {
            const size_t len = std::min(kChunk, n - off);
            int j, rc;
            if ((rc = take(&j))) return rc;
            cudaError_t e = cudaMemcpyAsync(chunk(j), static_cast<const uint8_t *>(dev) + off, len, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaEventRecord(ev[j], s);
            if (e != cudaSuccess) return cuda_err(e, "device-to-host copy");
            busy[j] = true;
            pend_dst[j] = host + off;
            pend_len[j] = len;
        }
        return QT_OK;
    }
    int flush() {  // every chunk's copy done and delivered, oldest first
        int rc = QT_OK;
        for (int k = 0; k < kChunks; k++) {
            const int r = retire((next + k) % kChunks);
            if (!rc) rc = r;
        }
        return rc;
    }
};

Stage &thread_stage(int dev) {
    thread_local Stage stages[kMaxDevices];
    return stages[dev];
}

// Cache of pinned host blocks for texture storage (qt_host_alloc). A block is page-locked
// once, when it is first allocated, and kept for reuse when freed: cudaFreeHost synchronises
// the whole device, so it runs only when the cached total passes kMaxCached. Sizes round up
// to an eighth of their power of two (at most 12.5% over). Blocks under 256 KiB, and all blocks
// where no pinned memory can be had (no usable GPU, or the system's limit), come from ordinary
// memory instead; the host-buffer entry points then stage them like any pageable buffer.
class HostCache {
   public:
    static HostCache &get() {
        static HostCache *c = new HostCache();  // never destroyed: blocks may outlive static teardown
        return *c;
    }
    int alloc(size_t n, void **out) {
        if (n > (size_t(1) << 48)) return set_err(QT_ERR_OOM, "host allocation of %zu bytes failed", n);
        const size_t cls = host_class(n);
        {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = free_.find(cls);
            if (it != free_.end()) {
                *out = it->second;
                free_.erase(it);
                cached_ -= cls;
                live_[*out] = {cls, true};
                return QT_OK;
            }
        }
        void *p = nullptr;
        bool pinned = false;
        if (cls >= kMinPinned && !no_pinned_.load(std::memory_order_relaxed)) {
            const cudaError_t e = cudaHostAlloc(&p, cls, cudaHostAllocPortable);
            if (e == cudaSuccess) {
                pinned = true;
            } else {
                cudaGetLastError();
                p = nullptr;
                if (e != cudaErrorMemoryAllocation) no_pinned_.store(true, std::memory_order_relaxed);
            }
        }
        if (!p && posix_memalign(&p, 4096, cls) != 0) return set_err(QT_ERR_OOM, "host allocation of %zu bytes failed", n);
        std::lock_guard<std::mutex> lk(mu_);
        live_[p] = {cls, pinned};
        *out = p;
        return QT_OK;
    }
    void release(void *p) {
        if (!p) return;
        void *drop = nullptr;
        {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = live_.find(p);
            if (it == live_.end()) return;  // not ours
            const Entry e = it->second;
            live_.erase(it);
            if (!e.pinned) {
                std::free(p);
                return;
            }
            if (cached_ + e.cls <= kMaxCached) {
                free_.emplace(e.cls, p);
                cached_ += e.cls;
                return;
            }
            drop = p;
        }
        cudaFreeHost(drop);
        cudaGetLastError();
    }

   private:
    struct Entry {
        size_t cls;
        bool pinned;
    };
    static constexpr size_t kMaxCached = size_t(2) << 30;
    // below this, ordinary memory: staging a small buffer costs less than pinning it
    static constexpr size_t kMinPinned = size_t(256) << 10;
    static size_t host_class(size_t n) {
        if (n == 0) n = 1;
        size_t c = 4096;
        while (c < n) c <<= 1;
        const size_t step = std::max<size_t>(4096, c / 8);
        return (n + step - 1) / step * step;
    }
    std::mutex mu_;
    std::multimap<size_t, void *> free_;
    std::map<void *, Entry> live_;
    size_t cached_ = 0;
    std::atomic<bool> no_pinned_{false};
};

// Host<->device copies of the host-buffer entry points: pinned (or otherwise registered)
// host memory is copied directly, pageable memory through the thread's stage.
struct HostXfer {
    Stage *st = nullptr;  // set when either side is pageable
    bool in_pageable = false, out_pageable = false;
    int begin(int dev, const void *host_in, const void *host_out) {
        in_pageable = is_pageable(host_in);
        out_pageable = is_pageable(host_out);
        if (!in_pageable && !out_pageable) return QT_OK;
        st = &thread_stage(dev);
        return st->init();
    }
    int in(void *dev, const uint8_t *host, size_t n, cudaStream_t s) {
        if (in_pageable) return st->upload(dev, host, n, s);
        const cudaError_t e = cudaMemcpyAsync(dev, host, n, cudaMemcpyHostToDevice, s);
        return e == cudaSuccess ? QT_OK : cuda_err(e, "host-to-device copy");
    }
    int out(uint8_t *host, const void *dev, size_t n, cudaStream_t s) {
        if (out_pageable) return st->download(host, dev, n, s);
        const cudaError_t e = cudaMemcpyAsync(host, dev, n, cudaMemcpyDeviceToHost, s);
        return e == cudaSuccess ? QT_OK : cuda_err(e, "device-to-host copy");
    }
    int finish() { return st ? st->flush() : QT_OK; }
};

// host path: H2D, kernel, D2H on this thread's stream; returns when done
template <typename Launch>
int run_host(const void *src, size_t src_bytes, void *dst, size_t dst_bytes, bool dst_needs_zero, Launch &&launch,
             const char *what) {
    int dev = 0;
    int rc = ensure_device(&dev);
    if (rc) return rc;
    DevBuf din, dout;
    if ((rc = acquire(din, dev, src_bytes)) || (rc = acquire(dout, dev, dst_bytes))) return rc;
    cudaStream_t s = thread_stream(dev);
    HostXfer x;
    if ((rc = x.begin(dev, src, dst))) return rc;
    rc = x.in(din.ptr, static_cast<const uint8_t *>(src), src_bytes, s);
    cudaError_t e = cudaSuccess;
    if (!rc && dst_needs_zero && (e = cudaMemsetAsync(dout.ptr, 0, dst_bytes, s)) != cudaSuccess) rc = cuda_err(e, "memset");
    if (!rc && (rc = launch(din.ptr, dout.ptr, (void *)s))) rc = cuda_err((cudaError_t)rc, what);
    if (!rc) rc = x.out(static_cast<uint8_t *>(dst), dout.ptr, dst_bytes, s);
    const int frc = x.finish();
    e = cudaStreamSynchronize(s);
    if (rc) return rc;
    if (frc) return frc;
    if (e != cudaSuccess) return cuda_err(e, what);
    return QT_OK;
}

// A second stream and an event per host thread and device, for the banded host path.
cudaStream_t thread_stream2(int dev) {
    thread_local cudaStream_t streams[kMaxDevices] = {};
    if (!streams[dev]) cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
    return streams[dev];
}
cudaEvent_t thread_event(int dev, int which = 0) {  // which < 3
    thread_local cudaEvent_t events[kMaxDevices][3] = {};
    if (!events[dev][which]) cudaEventCreateWithFlags(&events[dev][which], cudaEventDisableTiming);
    return events[dev][which];
}

// Host path, pipelined: the texture is cut into bands of block rows (about 4 MB of
// texels in the first, 8 MB in the others). Band k's upload and kernel go on one of two streams, all bands
// first, then the downloads: so uploads, kernels and downloads of different bands
// overlap, and a download into pageable memory (which the runtime completes
// before returning) never holds back a later upload. Encode: a bottom band whose
// last block row wraps (h % 4 != 0) reads texel rows 0-3, so it waits for band 0's
// upload. Decode with h % 4 != 0 writes wrapped texels into the top rows from the
// bottom band, so it is not banded. launch(in, out, b_begin, b_end, stream) runs
// the kernel over the blocks [b_begin, b_end).
template <typename Launch>
int run_host_banded(const uint8_t *src, uint8_t *dst, bool encode, int w, int h, size_t block_bytes, Launch &&launch,
                    const char *what, long min_band_blocks = 0) {
    const int bw = (w + 3) / 4, bh = (h + 3) / 4;
    const size_t texel_row = (size_t)w * 4, block_row = (size_t)bw * block_bytes;
    const size_t texel_bytes = texel_row * (size_t)h, blocks_bytes = block_row * (size_t)bh;
    const size_t per_brow = 4 * texel_row + block_row;
    // ~4 MB of texels in the first band (the kernels start sooner), ~8 MB in the others, and at
    // least min_band_blocks blocks in each: a BC1/BC3 setting with EndpointSearch passes
    // defer_min_blocks(), so a texture too small for the deferred path (run_host_bc1_parts
    // takes the larger ones) is not cut into bands that each pay the search's serial latency.
    // Measured at 4096^2 against 8 MB bands throughout: L0/L10 encode -2.5%, BC4 encode -1.5%,
    // BC1 decode -1% per call; a first band of 1 or 2 MB was no better than 8.
    const size_t min_rows = (size_t)((min_band_blocks + bw - 1) / bw);
    const long rows_cap = (long)std::max<size_t>(std::max<size_t>(1, (size_t(8) << 20) / per_brow), min_rows);
    long rows = (long)std::max<size_t>(std::max<size_t>(1, (size_t(4) << 20) / per_brow), min_rows);
    std::vector<int> cut(1, 0);  // band k covers block rows [cut[k], cut[k + 1])
    for (; cut.back() < bh; rows = std::min(2 * rows, rows_cap))
        cut.push_back((int)std::min<long>(bh, (long)cut.back() + rows));
    const int nbands = (int)cut.size() - 1;
    const bool ragged = (h & 3) != 0;
    const size_t in_bytes = encode ? texel_bytes : blocks_bytes, out_bytes = encode ? blocks_bytes : texel_bytes;
    if (nbands < 2 || (!encode && ragged))
        return run_host(src, in_bytes, dst, out_bytes, false,
                        [&](void *in, void *out, void *st) { return launch(in, out, 0L, (long)bw * bh, st); }, what);
    int dev = 0;
    int rc = ensure_device(&dev);
    if (rc) return rc;
    DevBuf din, dout;
    if ((rc = acquire(din, dev, in_bytes)) || (rc = acquire(dout, dev, out_bytes))) return rc;
    cudaStream_t st[2] = {thread_stream(dev), thread_stream2(dev)};
    cudaEvent_t first_up = thread_event(dev);
    uint8_t *di = static_cast<uint8_t *>(din.ptr), *dout_p = static_cast<uint8_t *>(dout.ptr);
    cudaError_t e = cudaSuccess;
    HostXfer x;
    if ((rc = x.begin(dev, src, dst))) return rc;
    // uploads and kernels
    for (int k = 0; k < nbands && e == cudaSuccess && rc == QT_OK; k++) {
        const int r0 = cut[k], r1 = cut[k + 1];
        cudaStream_t s = st[k & 1];
        size_t off, len;
        if (encode) {
            off = (size_t)(4 * r0) * texel_row;
            len = (size_t)(std::min(h, 4 * r1) - 4 * r0) * texel_row;
        } else {
            off = (size_t)r0 * block_row;
            len = (size_t)(r1 - r0) * block_row;
        }
        rc = x.in(di + off, src + off, len, s);
        if (rc) break;
        if (k == 0) e = cudaEventRecord(first_up, s);
        if (e == cudaSuccess && encode && ragged && k == nbands - 1 && (k & 1)) e = cudaStreamWaitEvent(s, first_up, 0);
        if (e == cudaSuccess) {
            const int lrc = launch(din.ptr, dout.ptr, (long)r0 * bw, (long)r1 * bw, (void *)s);
            if (lrc) rc = cuda_err((cudaError_t)lrc, what);
        }
    }
    // downloads
    for (int k = 0; k < nbands && e == cudaSuccess && rc == QT_OK; k++) {
        const int r0 = cut[k], r1 = cut[k + 1];
        size_t off, len;
        if (encode) {
            off = (size_t)r0 * block_row;
            len = (size_t)(r1 - r0) * block_row;
        } else {
            off = (size_t)(4 * r0) * texel_row;
            len = (size_t)(std::min(h, 4 * r1) - 4 * r0) * texel_row;
        }
        rc = x.out(dst + off, dout_p + off, len, st[k & 1]);
    }
    const int frc = x.finish();
    const cudaError_t e0 = cudaStreamSynchronize(st[0]), e1 = cudaStreamSynchronize(st[1]);
    if (rc) return rc;
    if (frc) return frc;
    if (e != cudaSuccess) return cuda_err(e, what);
    if (e0 != cudaSuccess) return cuda_err(e0, what);
    if (e1 != cudaSuccess) return cuda_err(e1, what);
    return QT_OK;
}

int set_level(qt_bc1_params *p, unsigned level) {
    // BC1Encoder::SetLevel (BC1Encoder.cpp:74-249)
    if (level > 19) return set_err(QT_ERR_ARG, "Level out of range, bust be between 0 and 18 inclusive");
    p->two_ls_passes = p->two_ep_passes = p->two_cf_passes = p->exhaustive = 0;
    p->power_iterations = 4;
    p->error_mode = QT_ERROR_CHECK2;
    p->endpoint_mode = QT_ENDPOINT_PCA;
    p->search_rounds = 0;
    p->orderings3 = p->orderings4 = 0;
    struct Row { int ls, ep, cf, ex, em, epm, o4, o3, sr, pi; };
    // -1 in epm keeps PCA; rows follow the switch in SetLevel
    static const Row rows[20] = {
        {0, 0, 0, 0, QT_ERROR_CHECK2, QT_ENDPOINT_BOUNDING_BOX_INT, 0, 0, 0, 4},  // 0
        {0, 0, 0, 0, QT_ERROR_CHECK2, QT_ENDPOINT_LEAST_SQUARES, 0, 0, 0, 4},     // 1
        {0, 0, 0, 0, QT_ERROR_CHECK2, QT_ENDPOINT_PCA, 0, 0, 0, 4},               // 2
        {1, 0, 0, 0, QT_ERROR_CHECK2, QT_ENDPOINT_PCA, 0, 0, 0, 4},               // 3
        {1, 0, 0, 0, QT_ERROR_FULL, QT_ENDPOINT_PCA, 0, 0, 0, 6},                 // 4
        {1, 0, 0, 0, QT_ERROR_FASTER, QT_ENDPOINT_PCA, 0, 0, 0, 4},               // 5
        {1, 0, 0, 0, QT_ERROR_FASTER, QT_ENDPOINT_PCA, 1, 1, 0, 4},               // 6
        {1, 0, 0, 0, QT_ERROR_FASTER, QT_ENDPOINT_PCA, 4, 1, 0, 4},               // 7
        {1, 0, 0, 0, QT_ERROR_FASTER, QT_ENDPOINT_PCA, 8, 1, 0, 4},               // 8
        {1, 0, 0, 0, QT_ERROR_CHECK2, QT_ENDPOINT_PCA, 11, 3, 0, 4},              // 9
        {1, 0, 0, 0, QT_ERROR_CHECK2, QT_ENDPOINT_PCA, 20, 8, 0, 4},              // 10
        {1, 0, 0, 0, QT_ERROR_CHECK2, QT_ENDPOINT_PCA, 28, 16, 0, 4},             // 11
        {1, 0, 0, 0, QT_ERROR_CHECK2, QT_ENDPOINT_PCA, 32, 32, 0, 4},             // 12
        {1, 1, 0, 0, QT_ERROR_FULL, QT_ENDPOINT_PCA, 32, 32, 20, 6},              // 13
        {1, 1, 0, 0, QT_ERROR_FULL, QT_ENDPOINT_PCA, 32, 32, 32, 6},              // 14
        {1, 1, 0, 0, QT_ERROR_FULL, QT_ENDPOINT_PCA, 56, 32, 32, 6},              // 15
        {1, 1, 0, 0, QT_ERROR_FULL, QT_ENDPOINT_PCA, 80, 32, 256, 6},             // 16
        {1, 1, 0, 0, QT_ERROR_FULL, QT_ENDPOINT_PCA, 128, 32, 256, 4},            // 17
        {1, 1, 1, 0, QT_ERROR_FULL, QT_ENDPOINT_PCA, 128, 32, 256, 6},            // 18
        {1, 1, 1, 1, QT_ERROR_FULL, QT_ENDPOINT_PCA, 128, 32, 256, 6},            // 19
    };
    const Row &r = rows[level];
    p->two_ls_passes = r.ls;
    p->two_ep_passes = r.ep;
    p->two_cf_passes = r.cf;
    p->exhaustive = r.ex;
    p->error_mode = r.em;
    p->endpoint_mode = r.epm;
    p->orderings4 = r.o4 < 1 ? 1u : (unsigned)r.o4;  // clamp to >= 1 (:247-248)
    p->orderings3 = r.o3 < 1 ? 1u : (unsigned)r.o3;
    p->search_rounds = (unsigned)r.sr;
    p->power_iterations = (unsigned)r.pi;
    return QT_OK;
}

int check_params(const qt_bc1_params *p, bool bc3) {
    if (!p) return set_err(QT_ERR_ARG, "params is NULL");
    if (!bc3 && p->color_mode != QT_COLOR_FOUR && p->color_mode != QT_COLOR_THREE && p->color_mode != QT_COLOR_THREE_BLACK)
        return set_err(QT_ERR_ARG, "Encoder color mode must be FourColor, ThreeColor, or ThreeColorBlack");
    if (int rc = check_interp(p->interpolator)) return rc;
    if (p->error_mode < 0 || p->error_mode > 3) return set_err(QT_ERR_ARG, "Invalid error mode");
    if (p->endpoint_mode < 0 || p->endpoint_mode > 3) return set_err(QT_ERR_ARG, "Invalid endpoint mode");
    if (p->orderings4 < 1 || p->orderings4 > 128 || p->orderings3 < 1 || p->orderings3 > 32)
        return set_err(QT_ERR_ARG, "orderings out of range (call qt_bc1_params_validate)");
    if (p->power_iterations < 4 || p->power_iterations > 10)
        return set_err(QT_ERR_ARG, "power_iterations out of range (call qt_bc1_params_validate)");
    return QT_OK;
}

}  // namespace

namespace qtk {
const HostTables &host_tables() {
    static const HostTables *t = make_tables();
    return *t;
}

int set_error(int code, const char *msg) { return set_err(code, "%s", msg); }
int cuda_error(int e, const char *what) { return cuda_err((cudaError_t)e, what); }
int ensure_current_device(int *dev) { return ensure_device(dev); }
int check_bc1_params(const qt_bc1_params *p, bool bc3) { return check_params(p, bc3); }

cudaError_t scratch_alloc(void **ptr, size_t bytes, cudaStream_t stream) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(g_mempool_mu);
        if (!g_mempool[dev]) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            if ((e = cudaMemPoolCreate(&g_mempool[dev], &props)) != cudaSuccess) {
                g_mempool[dev] = nullptr;
                return e;
            }
            uint64_t keep = UINT64_MAX;
            cudaMemPoolSetAttribute(g_mempool[dev], cudaMemPoolAttrReleaseThreshold, &keep);
        }
        pool = g_mempool[dev];
    }
    return cudaMallocFromPoolAsync(ptr, bytes, pool, stream);
}

cudaError_t scratch_free(void *ptr, cudaStream_t stream) { return ptr ? cudaFreeAsync(ptr, stream) : cudaSuccess; }
}  // namespace qtk

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

const char *qt_last_error(void) { return g_err.c_str(); }

const char *qt_version(void) { return "quicktex-b200 0.1.0 (sm_100a)"; }

int qt_bc1_params_for_level(unsigned level, int color_mode, int interpolator, qt_bc1_params *out) {
    if (!out) return set_err(QT_ERR_ARG, "out is NULL");
    if (color_mode != QT_COLOR_FOUR && color_mode != QT_COLOR_THREE && color_mode != QT_COLOR_THREE_BLACK)
        return set_err(QT_ERR_ARG, "Encoder color mode must be FourColor, ThreeColor, or ThreeColorBlack");
    if (int rc = check_interp(interpolator)) return rc;
    qt_bc1_params p;
    if (int rc = set_level(&p, level)) return rc;
    p.color_mode = color_mode;
    p.interpolator = interpolator;
    *out = p;
    return QT_OK;
}

int qt_bc1_params_validate(qt_bc1_params *p) {
    if (!p) return set_err(QT_ERR_ARG, "params is NULL");
    // SetOrderings4/3 and SetPowerIterations clamp (BC1Encoder.cpp:251-258)
    if (p->orderings4 < 1) p->orderings4 = 1;
    if (p->orderings4 > 128) p->orderings4 = 128;
    if (p->orderings3 < 1) p->orderings3 = 1;
    if (p->orderings3 > 32) p->orderings3 = 32;
    if (p->power_iterations < 4) p->power_iterations = 4;
    if (p->power_iterations > 10) p->power_iterations = 10;
    return check_params(p, false);
}

int qt_init(int device) {
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return cuda_err(e, "cudaGetDevice");
    if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_err(e, "cudaSetDevice");
    int rc = ensure_device(nullptr);
    cudaSetDevice(prev);
    return rc;
}

int qt_host_alloc(size_t bytes, void **ptr) {
    if (!ptr) return set_err(QT_ERR_ARG, "ptr is NULL");
    *ptr = nullptr;
    return HostCache::get().alloc(bytes, ptr);
}

void qt_host_free(void *ptr) { HostCache::get().release(ptr); }

// ---- encoders ----
int qt_bc1_encode_device(const uint8_t *rgba, int w, int h, const qt_bc1_params *p, uint8_t *blocks, void *stream) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_params(p, false)) || (rc = check_ptr(rgba, 4, "rgba")) ||
        (rc = check_ptr(blocks, 8, "blocks")) || (rc = ensure_device(nullptr)))
        return rc;
    return finish_launch(qtk::launch_bc1_encode(rgba, w, h, *p, blocks, false, stream), "bc1 encode");
}

int qt_bc3_encode_device(const uint8_t *rgba, int w, int h, const qt_bc1_params *p, uint8_t *blocks, void *stream) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_params(p, true)) || (rc = check_ptr(rgba, 4, "rgba")) ||
        (rc = check_ptr(blocks, 16, "blocks")) || (rc = ensure_device(nullptr)))
        return rc;
    return finish_launch(qtk::launch_bc1_encode(rgba, w, h, *p, blocks, true, stream), "bc3 encode");
}

int qt_bc1_encode_kernels(int w, int h, const qt_bc1_params *p, int *kernels) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_params(p, true)) || (rc = check_ptr(kernels, 4, "kernels")) ||
        (rc = ensure_device(nullptr)))
        return rc;
    *kernels = qtk::bc1_encode_kernels((long)((w + 3) / 4) * ((h + 3) / 4), *p);
    return QT_OK;
}

int qt_bc4_encode_device(const uint8_t *rgba, int w, int h, int channel, uint8_t *blocks, void *stream) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_channel(channel)) || (rc = check_ptr(rgba, 4, "rgba")) ||
        (rc = check_ptr(blocks, 8, "blocks")) || (rc = ensure_device(nullptr)))
        return rc;
    return finish_launch(qtk::launch_bc4_encode(rgba, w, h, channel, channel, false, blocks, stream), "bc4 encode");
}

int qt_bc5_encode_device(const uint8_t *rgba, int w, int h, int c0, int c1, uint8_t *blocks, void *stream) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_channel(c0)) || (rc = check_channel(c1)) ||
        (rc = check_ptr(rgba, 4, "rgba")) || (rc = check_ptr(blocks, 16, "blocks")) || (rc = ensure_device(nullptr)))
        return rc;
    return finish_launch(qtk::launch_bc4_encode(rgba, w, h, c0, c1, true, blocks, stream), "bc5 encode");
}

// Host path of a BC1/BC3 encode on the deferred path (EndpointSearch, defer_min_blocks() or more
// blocks): the texels go up in row bands, ~8 MB first and each band twice the last, on two
// streams in turn; each band's split pass and encoder start when its upload is done and append
// to queues shared by the whole texture; the passes over those queues (second cluster-fit pass,
// search, finish) run once after the last band, and the blocks come back in one download.
// Encoding the bands as independent textures instead would end every band's search pass with
// its own tail of idle lanes. A bottom block row that wraps (h % 4 != 0) reads texel rows 0-3,
// so its band waits for band 0's upload.
int run_host_bc1_parts(const uint8_t *src, uint8_t *dst, int w, int h, size_t block_bytes, const qt_bc1_params &p,
                       bool bc3, const char *what) {
    const int bw = (w + 3) / 4, bh = (h + 3) / 4;
    const size_t texel_row = (size_t)w * 4, block_row = (size_t)bw * block_bytes;
    const size_t in_bytes = texel_row * (size_t)h, out_bytes = block_row * (size_t)bh;
    const int rows_first = (int)std::max<size_t>(1, (size_t(8) << 20) / (4 * texel_row + block_row));
    std::vector<int> cut(1, 0);  // band k covers block rows [cut[k], cut[k + 1])
    for (long rows = rows_first; cut.back() < bh; rows *= 2)
        cut.push_back((int)std::min<long>(bh, (long)cut.back() + rows));
    const int nbands = (int)cut.size() - 1;  // <= 13 for any texture of <= 2^32 texels (bc1_parts_add takes 32)
    int dev = 0;
    int rc = ensure_device(&dev);
    if (rc) return rc;
    DevBuf din, dout;
    if ((rc = acquire(din, dev, in_bytes)) || (rc = acquire(dout, dev, out_bytes))) return rc;
    cudaStream_t st[2] = {thread_stream(dev), thread_stream2(dev)};
    cudaEvent_t ev_first = thread_event(dev, 0), ev_ready = thread_event(dev, 1), ev_join = thread_event(dev, 2);
    uint8_t *di = static_cast<uint8_t *>(din.ptr), *dout_p = static_cast<uint8_t *>(dout.ptr);
    HostXfer x;
    if ((rc = x.begin(dev, src, dst))) return rc;
    qtk::Bc1Parts ps;
    cudaError_t e = cudaSuccess;
    if (const int brc = qtk::bc1_parts_begin(ps, (long)bw * bh, p, st[0])) rc = cuda_err((cudaError_t)brc, what);
    if (!rc && (e = cudaEventRecord(ev_ready, st[0])) == cudaSuccess) e = cudaStreamWaitEvent(st[1], ev_ready, 0);
    for (int k = 0; k < nbands && e == cudaSuccess && rc == QT_OK; k++) {
        const int r0 = cut[k], r1 = cut[k + 1];
        cudaStream_t s = st[k & 1];
        const size_t off = (size_t)(4 * r0) * texel_row, len = (size_t)(std::min(h, 4 * r1) - 4 * r0) * texel_row;
        if ((rc = x.in(di + off, src + off, len, s))) break;
        if (k == 0) e = cudaEventRecord(ev_first, s);
        if (e == cudaSuccess && (h & 3) && k == nbands - 1 && (k & 1)) e = cudaStreamWaitEvent(s, ev_first, 0);
        if (e == cudaSuccess) {
            const int lrc = qtk::bc1_parts_add(ps, di, w, h, p, dout_p, bc3, (long)r0 * bw, (long)r1 * bw, s);
            if (lrc) rc = cuda_err((cudaError_t)lrc, what);
        }
    }
    if (!rc && e == cudaSuccess && (e = cudaEventRecord(ev_join, st[1])) == cudaSuccess)
        e = cudaStreamWaitEvent(st[0], ev_join, 0);
    if (!rc && e == cudaSuccess) {
        const int lrc = qtk::bc1_parts_end(ps, di, w, h, p, dout_p, bc3, st[0]);
        if (lrc) rc = cuda_err((cudaError_t)lrc, what);
    }
    if (!rc && e == cudaSuccess) rc = x.out(dst, dout_p, out_bytes, st[0]);
    const int frc = x.finish();
    const cudaError_t e0 = cudaStreamSynchronize(st[0]), e1 = cudaStreamSynchronize(st[1]);
    qtk::bc1_parts_free(ps, st[0]);  // still held only after a failure
    if (rc) return rc;
    if (frc) return frc;
    if (e != cudaSuccess) return cuda_err(e, what);
    if (e0 != cudaSuccess) return cuda_err(e0, what);
    if (e1 != cudaSuccess) return cuda_err(e1, what);
    return QT_OK;
}

int qt_bc1_encode_host(const uint8_t *rgba, int w, int h, const qt_bc1_params *p, uint8_t *blocks) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_params(p, false)) || (rc = check_ptr(rgba, 1, "rgba")) ||
        (rc = check_ptr(blocks, 1, "blocks")))
        return rc;
    const qt_bc1_params pp = *p;
    if (qtk::bc1_parts_eligible((long)((w + 3) / 4) * ((h + 3) / 4), pp))
        return run_host_bc1_parts(rgba, blocks, w, h, 8, pp, false, "bc1 encode");
    return run_host_banded(rgba, blocks, true, w, h, 8,
                           [&](void *in, void *out, long b0, long b1, void *s) {
                               return qtk::launch_bc1_encode_range((const uint8_t *)in, w, h, pp, (uint8_t *)out, false, b0, b1, s);
                           },
                           "bc1 encode", pp.search_rounds > 0 ? qtk::defer_min_blocks() : 0);
}

int qt_bc3_encode_host(const uint8_t *rgba, int w, int h, const qt_bc1_params *p, uint8_t *blocks) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_params(p, true)) || (rc = check_ptr(rgba, 1, "rgba")) ||
        (rc = check_ptr(blocks, 1, "blocks")))
        return rc;
    const qt_bc1_params pp = *p;
    if (qtk::bc1_parts_eligible((long)((w + 3) / 4) * ((h + 3) / 4), pp))
        return run_host_bc1_parts(rgba, blocks, w, h, 16, pp, true, "bc3 encode");
    return run_host_banded(rgba, blocks, true, w, h, 16,
                           [&](void *in, void *out, long b0, long b1, void *s) {
                               return qtk::launch_bc1_encode_range((const uint8_t *)in, w, h, pp, (uint8_t *)out, true, b0, b1, s);
                           },
                           "bc3 encode", pp.search_rounds > 0 ? qtk::defer_min_blocks() : 0);
}

int qt_bc4_encode_host(const uint8_t *rgba, int w, int h, int channel, uint8_t *blocks) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_channel(channel)) || (rc = check_ptr(rgba, 1, "rgba")) ||
        (rc = check_ptr(blocks, 1, "blocks")))
        return rc;
    return run_host_banded(rgba, blocks, true, w, h, 8,
                           [&](void *in, void *out, long b0, long b1, void *s) {
                               return qtk::launch_bc4_encode_range((const uint8_t *)in, w, h, channel, channel, false, (uint8_t *)out, b0, b1, s);
                           },
                           "bc4 encode");
}

int qt_bc5_encode_host(const uint8_t *rgba, int w, int h, int c0, int c1, uint8_t *blocks) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_channel(c0)) || (rc = check_channel(c1)) ||
        (rc = check_ptr(rgba, 1, "rgba")) || (rc = check_ptr(blocks, 1, "blocks")))
        return rc;
    return run_host_banded(rgba, blocks, true, w, h, 16,
                           [&](void *in, void *out, long b0, long b1, void *s) {
                               return qtk::launch_bc4_encode_range((const uint8_t *)in, w, h, c0, c1, true, (uint8_t *)out, b0, b1, s);
                           },
                           "bc5 encode");
}

// ---- decoders ----
static int decode_device(int fmt, const uint8_t *blocks, int w, int h, int interp, int wa, int c0, int c1, uint8_t *rgba,
                         void *stream) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_interp(interp)) || (rc = check_channel(c0)) || (rc = check_channel(c1)) ||
        (rc = check_ptr(blocks, (fmt == 3 || fmt == 5) ? 16 : 8, "blocks")) || (rc = check_ptr(rgba, 4, "rgba")) ||
        (rc = ensure_device(nullptr)))
        return rc;
    return finish_launch(qtk::launch_decode(fmt, blocks, w, h, interp, wa, c0, c1, rgba, stream), "decode");
}

static int decode_host(int fmt, const uint8_t *blocks, int w, int h, int interp, int wa, int c0, int c1, uint8_t *rgba) {
    int rc;
    if ((rc = check_dims(w, h)) || (rc = check_interp(interp)) || (rc = check_channel(c0)) || (rc = check_channel(c1)) ||
        (rc = check_ptr(blocks, 1, "blocks")) || (rc = check_ptr(rgba, 1, "rgba")))
        return rc;
    const size_t bsize = (fmt == 3 || fmt == 5) ? 16 : 8;
    return run_host_banded(blocks, rgba, false, w, h, bsize,
                           [&](void *in, void *out, long b0, long b1, void *s) {
                               return qtk::launch_decode_range(fmt, (const uint8_t *)in, w, h, interp, wa, c0, c1, (uint8_t *)out, b0, b1, s);
                           },
                           "decode");
}

int qt_bc1_decode_device(const uint8_t *b, int w, int h, int interp, int wa, uint8_t *rgba, void *s) {
    return decode_device(1, b, w, h, interp, wa != 0, 0, 0, rgba, s);
}
int qt_bc3_decode_device(const uint8_t *b, int w, int h, int interp, uint8_t *rgba, void *s) {
    return decode_device(3, b, w, h, interp, 0, 0, 0, rgba, s);
}
int qt_bc4_decode_device(const uint8_t *b, int w, int h, int ch, uint8_t *rgba, void *s) {
    return decode_device(4, b, w, h, 0, 0, ch, ch, rgba, s);
}
int qt_bc5_decode_device(const uint8_t *b, int w, int h, int c0, int c1, uint8_t *rgba, void *s) {
    return decode_device(5, b, w, h, 0, 0, c0, c1, rgba, s);
}
int qt_bc1_decode_host(const uint8_t *b, int w, int h, int interp, int wa, uint8_t *rgba) {
    return decode_host(1, b, w, h, interp, wa != 0, 0, 0, rgba);
}
int qt_bc3_decode_host(const uint8_t *b, int w, int h, int interp, uint8_t *rgba) {
    return decode_host(3, b, w, h, interp, 0, 0, 0, rgba);
}
int qt_bc4_decode_host(const uint8_t *b, int w, int h, int ch, uint8_t *rgba) {
    return decode_host(4, b, w, h, 0, 0, ch, ch, rgba);
}
int qt_bc5_decode_host(const uint8_t *b, int w, int h, int c0, int c1, uint8_t *rgba) {
    return decode_host(5, b, w, h, 0, 0, c0, c1, rgba);
}

}  // extern "C"
