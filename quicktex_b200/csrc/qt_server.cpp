// qt_server.cpp — continuous-batching encode/decode server on one GPU
// (qt_server_* in include/quicktex_cuda.h).
//
// Threads: callers submit (under the server mutex) and poll completions; one
// worker thread owns the device arena, the slots and every CUDA call. The
// worker loop:
//   1. retire finished slots (cudaEventQuery on the slot's last event): mark
//      their requests complete, return their arena range;
//   2. if a slot is free, take waiting requests in arrival order while their
//      bytes fit the largest free range and the batch stays within
//      max_batch_blocks / max_batch_requests, and launch them on that slot:
//      one upload per payload, qt_batch_run (one persistent launch), one
//      download per response, an event;
//   3. with batches in flight and nothing to launch, poll again (yielding);
//      idle, sleep on the submit condition variable.

#include <time.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "qt_internal.h"

namespace {

constexpr size_t kAlign = 256;
size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

double mono_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + (double)ts.tv_nsec * 1e-9;
}

// input / output bytes of a request
size_t block_bytes(int fmt) { return (fmt == 3 || fmt == 5) ? 16 : 8; }
size_t n_blocks(const qt_batch_item &it) { return (size_t)((it.width + 3) / 4) * (size_t)((it.height + 3) / 4); }
size_t in_bytes(const qt_batch_item &it) {
    return it.op == QT_OP_ENCODE ? (size_t)it.width * it.height * 4 : n_blocks(it) * block_bytes(it.format);
}
size_t out_bytes(const qt_batch_item &it) {
    return it.op == QT_OP_ENCODE ? n_blocks(it) * block_bytes(it.format) : (size_t)it.width * it.height * 4;
}

// First-fit free list over [0, size): offset -> length, coalesced on release.
struct Arena {
    size_t size = 0;
    std::map<size_t, size_t> free_;
    void init(size_t n) {
        size = n;
        free_.clear();
        if (n) free_[0] = n;
    }
    size_t largest() const {
        size_t m = 0;
        for (const auto &f : free_) m = std::max(m, f.second);
        return m;
    }
    bool alloc(size_t n, size_t *off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            *off = it->first;
            const size_t rest = it->second - n, o = it->first + n;
            free_.erase(it);
            if (rest) free_[o] = rest;
            return true;
        }
        return false;
    }
    void release(size_t off, size_t n) {
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Req {
    qt_batch_item item;  // src / dst: host buffers
    uint64_t tag;
    size_t in, out;      // aligned device bytes
};

struct Done {
    uint64_t tag;
    int32_t status;
    double t;
};

struct Slot {
    qt_batch *batch = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<Req> reqs;
    size_t off = 0, len = 0;
    bool busy = false;
};

}  // namespace

struct qt_server {
    int device = 0;
    uint8_t *dbase = nullptr;
    Arena arena;
    std::vector<Slot> slots;
    size_t max_blocks = 0, max_reqs = 0;

    std::mutex mu;                      // pending, done, running, stats
    std::condition_variable cv_submit;  // worker waits for work
    std::condition_variable cv_done;    // pollers wait for completions
    std::deque<Req> pending;
    std::deque<Done> done;
    bool running = true;
    qt_server_stats stats{};
    std::thread worker;

    std::vector<qt_batch_item> items;  // worker scratch
};

namespace {

void complete(qt_server *s, Slot &sl, int status) {
    const double t = mono_s();
    uint64_t blocks = 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        for (const Req &r : sl.reqs) {
            s->done.push_back({r.tag, status, t});
            blocks += n_blocks(r.item);
        }
        s->stats.requests_done += sl.reqs.size();
        s->stats.blocks_done += blocks;
    }
    s->cv_done.notify_all();
    s->arena.release(sl.off, sl.len);
    sl.reqs.clear();
    sl.busy = false;
}

void fail_now(qt_server *s, const Req &r, int status) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->done.push_back({r.tag, status, mono_s()});
        s->stats.requests_done++;
    }
    s->cv_done.notify_all();
}

void launch(qt_server *s, Slot &sl) {
    size_t total = 0;
    for (const Req &r : sl.reqs) total += r.in + r.out;
    size_t off = 0;
    if (!s->arena.alloc(total, &off)) {  // cannot happen: admission checked the largest free range
        for (const Req &r : sl.reqs) fail_now(s, r, QT_ERR_STATE);
        sl.reqs.clear();
        return;
    }
    sl.off = off;
    sl.len = total;
    s->items.resize(sl.reqs.size());
    size_t pi = off, po = off;
    for (const Req &r : sl.reqs) po += r.in;
    int rc = QT_OK;
    cudaError_t e = cudaSuccess;
    for (size_t k = 0; k < sl.reqs.size() && e == cudaSuccess; k++) {
        const Req &r = sl.reqs[k];
        qt_batch_item &it = s->items[k];
        it = r.item;
        it.src = s->dbase + pi;
        it.dst = s->dbase + po;
        e = cudaMemcpyAsync(s->dbase + pi, r.item.src, in_bytes(r.item), cudaMemcpyDefault, sl.stream);
        pi += r.in;
        po += r.out;
    }
    if (e != cudaSuccess) rc = qtk::cuda_error((int)e, "server upload");
    if (rc == QT_OK) rc = qt_batch_run(sl.batch, s->items.data(), s->items.size(), sl.stream);
    for (size_t k = 0; k < sl.reqs.size() && rc == QT_OK; k++) {
        const Req &r = sl.reqs[k];
        e = cudaMemcpyAsync(r.item.dst, s->items[k].dst, out_bytes(r.item), cudaMemcpyDefault, sl.stream);
        if (e != cudaSuccess) rc = qtk::cuda_error((int)e, "server download");
    }
    if (rc == QT_OK && (e = cudaEventRecord(sl.done, sl.stream)) != cudaSuccess) rc = qtk::cuda_error((int)e, "server event");
    if (rc != QT_OK) {
        cudaStreamSynchronize(sl.stream);
        complete(s, sl, rc);
        return;
    }
    sl.busy = true;
    std::lock_guard<std::mutex> lk(s->mu);
    s->stats.batches++;
}

void worker_main(qt_server *s) {
    cudaSetDevice(s->device);
    for (;;) {
        uint32_t inflight = 0;
        for (Slot &sl : s->slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.done);
            if (q == cudaSuccess) {
                complete(s, sl, QT_OK);
            } else if (q != cudaErrorNotReady) {
                complete(s, sl, qtk::cuda_error((int)q, "server batch"));
            } else {
                inflight++;
            }
        }
        Slot *free_slot = nullptr;
        for (Slot &sl : s->slots)
            if (!sl.busy) {
                free_slot = &sl;
                break;
            }
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->stats.inflight = inflight;
            s->stats.pending = (uint32_t)std::min<size_t>(s->pending.size(), 0xFFFFFFFFu);
            if (!s->running && s->pending.empty() && inflight == 0) return;
            if (free_slot && !s->pending.empty()) {
                const size_t room = s->arena.largest();
                size_t bytes = 0, blocks = 0;
                while (!s->pending.empty()) {
                    const Req &r = s->pending.front();
                    const size_t need = r.in + r.out, nb = n_blocks(r.item);
                    if (!free_slot->reqs.empty() && (blocks + nb > s->max_blocks || free_slot->reqs.size() >= s->max_reqs))
                        break;
                    if (bytes + need > room) break;
                    free_slot->reqs.push_back(r);
                    s->pending.pop_front();
                    bytes += need;
                    blocks += nb;
                }
                if (!free_slot->reqs.empty()) s->stats.max_inflight = std::max(s->stats.max_inflight, inflight + 1);
            } else if (inflight == 0) {
                s->cv_submit.wait_for(lk, std::chrono::milliseconds(2));
                continue;
            }
        }
        if (free_slot && !free_slot->reqs.empty()) {
            launch(s, *free_slot);
            continue;
        }
        std::this_thread::yield();  // batches in flight, nothing to launch
    }
}

}  // namespace

extern "C" {

double qt_server_clock(void) { return mono_s(); }

int qt_server_create(int device, size_t memory_budget, int slots, size_t max_batch_blocks, size_t max_batch_requests,
                     qt_server **out) {
    if (!out) return qtk::set_error(QT_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (slots < 1 || slots > 64 || memory_budget < kAlign || max_batch_blocks == 0 || max_batch_requests == 0)
        return qtk::set_error(QT_ERR_ARG, "invalid server configuration");
    int prev = 0;
    cudaGetDevice(&prev);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return qtk::cuda_error((int)e, "cudaSetDevice");
    int rc = qtk::ensure_current_device(nullptr);
    qt_server *s = nullptr;
    if (rc == QT_OK) {
        s = new qt_server();
        s->device = device;
        s->max_blocks = max_batch_blocks;
        s->max_reqs = max_batch_requests;
        s->slots.resize((size_t)slots);
        s->stats.slots = (uint32_t)slots;
        memory_budget = memory_budget / kAlign * kAlign;
        if ((e = cudaMalloc(&s->dbase, memory_budget)) != cudaSuccess) rc = qtk::cuda_error((int)e, "allocating the server arena");
        for (Slot &sl : s->slots) {
            if (rc != QT_OK) break;
            if ((rc = qt_batch_create(device, &sl.batch)) != QT_OK) break;
            // sized for the largest batch: no queue reallocation while serving
            if ((rc = qt_batch_reserve(sl.batch, max_batch_requests, max_batch_blocks / 32 + max_batch_requests)) != QT_OK) break;
            if ((e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking)) != cudaSuccess ||
                (e = cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming)) != cudaSuccess)
                rc = qtk::cuda_error((int)e, "creating a server slot");
        }
        if (rc == QT_OK) {
            s->arena.init(memory_budget);
            s->worker = std::thread(worker_main, s);
        } else {
            for (Slot &sl : s->slots) {
                if (sl.batch) qt_batch_destroy(sl.batch);
                if (sl.stream) cudaStreamDestroy(sl.stream);
                if (sl.done) cudaEventDestroy(sl.done);
            }
            cudaFree(s->dbase);
            delete s;
            s = nullptr;
        }
    }
    cudaSetDevice(prev);
    *out = s;
    return rc;
}

int qt_server_destroy(qt_server *s) {
    if (!s) return QT_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->running = false;
    }
    s->cv_submit.notify_all();
    if (s->worker.joinable()) s->worker.join();
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(s->device);
    for (Slot &sl : s->slots) {
        qt_batch_destroy(sl.batch);
        cudaStreamDestroy(sl.stream);
        cudaEventDestroy(sl.done);
    }
    cudaFree(s->dbase);
    cudaSetDevice(prev);
    delete s;
    return QT_OK;
}

int qt_server_set_rules(qt_server *s, const qt_tile_rule *rules, size_t n) {
    if (!s) return qtk::set_error(QT_ERR_ARG, "NULL argument");
    for (Slot &sl : s->slots)
        if (int rc = qt_batch_set_rules(sl.batch, rules, n)) return rc;
    return QT_OK;
}

int qt_server_set_grid(qt_server *s, int ctas_per_sm) {
    if (!s) return qtk::set_error(QT_ERR_ARG, "NULL argument");
    for (Slot &sl : s->slots)
        if (int rc = qt_batch_set_grid(sl.batch, ctas_per_sm)) return rc;
    return QT_OK;
}

int qt_server_set_threads(qt_server *s, int threads_per_cta) {
    if (!s) return qtk::set_error(QT_ERR_ARG, "NULL argument");
    for (Slot &sl : s->slots)
        if (int rc = qt_batch_set_threads(sl.batch, threads_per_cta)) return rc;
    return QT_OK;
}

int qt_server_submit(qt_server *s, const qt_batch_item *items, const uint64_t *tags, size_t n) {
    if (!s || (n && (!items || !tags))) return qtk::set_error(QT_ERR_ARG, "NULL argument");
    for (size_t i = 0; i < n; i++) {
        if (int rc = qtk::check_item_fields(items[i])) return rc;
        if (!items[i].src || !items[i].dst) return qtk::set_error(QT_ERR_ARG, "request: NULL buffer");
    }
    std::vector<Req> oversize;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (!s->running) return qtk::set_error(QT_ERR_STATE, "the server is shutting down");
        for (size_t i = 0; i < n; i++) {
            Req r{items[i], tags[i], align_up(in_bytes(items[i])), align_up(out_bytes(items[i]))};
            if (r.in + r.out > s->arena.size) {
                oversize.push_back(r);
                continue;
            }
            s->pending.push_back(r);
        }
    }
    for (const Req &r : oversize) {
        qtk::set_error(QT_ERR_RANGE, "request exceeds the server's memory budget");
        fail_now(s, r, QT_ERR_RANGE);
    }
    s->cv_submit.notify_one();
    return QT_OK;
}

int qt_server_poll(qt_server *s, uint64_t *tags, int32_t *status, double *t_done, size_t cap, int64_t timeout_us,
                   size_t *n) {
    if (!s || !n || (cap && (!tags || !status || !t_done))) return qtk::set_error(QT_ERR_ARG, "NULL argument");
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->done.empty() && timeout_us > 0)
        s->cv_done.wait_for(lk, std::chrono::microseconds(timeout_us), [s] { return !s->done.empty(); });
    size_t k = 0;
    while (k < cap && !s->done.empty()) {
        const Done &d = s->done.front();
        tags[k] = d.tag;
        status[k] = d.status;
        t_done[k] = d.t;
        s->done.pop_front();
        k++;
    }
    *n = k;
    return QT_OK;
}

int qt_server_get_stats(qt_server *s, qt_server_stats *out) {
    if (!s || !out) return qtk::set_error(QT_ERR_ARG, "NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    return QT_OK;
}

}  // extern "C"
