// Bulk host <-> device transfers through pinned staging slots.
//
// A cudaMemcpy from or to pageable memory runs at the driver's own staging
// rate, a few GB/s, and the bond arrays of a large problem are gigabytes. Here
// up to 16 host threads each own two pinned 4 MB slots: a thread fills one slot
// (converting elements on the way: node ids to device positions, dictionary
// ids, packed flags) while the copy engine moves the other, so a transfer runs
// at the rate of the host threads' memory traffic, up to the PCIe limit, and a
// conversion pass costs no extra sweep over the arrays.
//
// Slots come from a process-wide pool of portable pinned blocks and are reused
// by later transfers (freeing pinned memory is left to process exit). All
// copies go to the caller's stream, so stream-ordered work before and after
// them keeps its order; both functions return once every copy has completed.
#pragma once

#include "bbpd_internal.h"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

namespace bbpd {
namespace staging {

constexpr size_t kSlotBytes = (size_t)4 << 20;
constexpr int kMaxWorkers = 16;
constexpr size_t kDirectBytes = (size_t)2 << 20;   // smaller transfers: one plain copy

struct Pool {
    std::mutex mu;
    std::vector<void *> free;
};

inline Pool &pool()
{
    static Pool *p = new Pool;   // never destroyed: pinned memory outlives static teardown
    return *p;
}

inline void *take_slot()
{
    {
        std::lock_guard<std::mutex> g(pool().mu);
        if (!pool().free.empty()) {
            void *s = pool().free.back();
            pool().free.pop_back();
            return s;
        }
    }
    void *s = nullptr;
    if (cudaHostAlloc(&s, kSlotBytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    return s;
}

inline void give_slot(void *s)
{
    if (!s) return;
    std::lock_guard<std::mutex> g(pool().mu);
    pool().free.push_back(s);
}

inline int workers_for(size_t bytes)
{
    const unsigned hc = std::max(1u, std::thread::hardware_concurrency());
    const size_t per = 2 * kSlotBytes;   // at least two slots' worth per worker
    return (int)std::max<size_t>(1, std::min<size_t>({(size_t)kMaxWorkers, (size_t)hc, bytes / per}));
}

// Worker w of W handles elements [n w / W, n (w + 1) / W) in slot-sized chunks.
template <class Body>
inline int run_workers(int W, Body body)
{
    int dev = 0;
    BBPD_CUDA_TRY(cudaGetDevice(&dev));
    std::vector<cudaError_t> err(W, cudaSuccess);
    std::vector<std::thread> th;
    th.reserve(W);
    for (int w = 0; w < W; w++)
        th.emplace_back([&, w]() {
            cudaError_t e = cudaSetDevice(dev);
            if (e == cudaSuccess) e = body(w);
            err[w] = e;
        });
    for (auto &t : th) t.join();
    for (cudaError_t e : err)
        if (e != cudaSuccess)
            return fail(e == cudaErrorMemoryAllocation ? BBPD_ERR_OOM : BBPD_ERR_CUDA, "staged copy: %s",
                        cudaGetErrorString(e));
    return BBPD_OK;
}

struct Slots {
    void *buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool busy[2] = {false, false};
    cudaError_t open()
    {
        for (int s = 0; s < 2; s++) {
            buf[s] = take_slot();
            if (!buf[s]) return cudaErrorMemoryAllocation;
            cudaError_t e = cudaEventCreateWithFlags(&ev[s], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    // wait for the copies still using the slots, then hand them back
    cudaError_t close()
    {
        cudaError_t r = cudaSuccess;
        for (int s = 0; s < 2; s++) {
            if (busy[s]) {
                cudaError_t e = cudaEventSynchronize(ev[s]);
                if (r == cudaSuccess) r = e;
            }
            if (ev[s]) cudaEventDestroy(ev[s]);
            give_slot(buf[s]);
        }
        return r;
    }
};

// dst[k] = element k for k in [0, n); fill(k0, cnt, out) writes elements
// k0 .. k0 + cnt - 1 to out. Returns after the data is on the device.
template <class T, class Fill>
int upload(T *dst, int64_t n, cudaStream_t st, Fill fill)
{
    if (n <= 0) return BBPD_OK;
    const size_t bytes = sizeof(T) * (size_t)n;
    if (bytes <= kDirectBytes) {
        std::vector<T> h((size_t)n);
        fill(0, n, h.data());
        BBPD_CUDA_TRY(cudaMemcpyAsync(dst, h.data(), bytes, cudaMemcpyHostToDevice, st));
        BBPD_CUDA_TRY(cudaStreamSynchronize(st));
        return BBPD_OK;
    }
    const int W = workers_for(bytes);
    const int64_t chunk = (int64_t)(kSlotBytes / sizeof(T));
    return run_workers(W, [&](int w) -> cudaError_t {
        Slots sl;
        cudaError_t e = sl.open();
        const int64_t lo = n * w / W, hi = n * (w + 1) / W;
        int s = 0;
        for (int64_t k0 = lo; k0 < hi && e == cudaSuccess; k0 += chunk) {
            const int64_t cnt = std::min(chunk, hi - k0);
            if (sl.busy[s]) e = cudaEventSynchronize(sl.ev[s]);
            if (e != cudaSuccess) break;
            fill(k0, cnt, (T *)sl.buf[s]);
            e = cudaMemcpyAsync(dst + k0, sl.buf[s], sizeof(T) * (size_t)cnt, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = cudaEventRecord(sl.ev[s], st);
            sl.busy[s] = e == cudaSuccess;
            s ^= 1;
        }
        cudaError_t c = sl.close();
        return e != cudaSuccess ? e : c;
    });
}

// Plain copy of n elements from host memory.
template <class T>
int upload_copy(T *dst, const T *src, int64_t n, cudaStream_t st)
{
    return upload(dst, n, st, [src](int64_t k0, int64_t cnt, T *out) {
        std::memcpy(out, src + k0, sizeof(T) * (size_t)cnt);
    });
}

// Element k of src for k in [0, n) reaches drain(k0, cnt, in), in chunks,
// after the stream's earlier work. Returns after every chunk is drained.
template <class T, class Drain>
int download(const T *src, int64_t n, cudaStream_t st, Drain drain)
{
    if (n <= 0) return BBPD_OK;
    const size_t bytes = sizeof(T) * (size_t)n;
    if (bytes <= kDirectBytes) {
        std::vector<T> h((size_t)n);
        BBPD_CUDA_TRY(cudaMemcpyAsync(h.data(), src, bytes, cudaMemcpyDeviceToHost, st));
        BBPD_CUDA_TRY(cudaStreamSynchronize(st));
        drain(0, n, h.data());
        return BBPD_OK;
    }
    const int W = workers_for(bytes);
    const int64_t chunk = (int64_t)(kSlotBytes / sizeof(T));
    return run_workers(W, [&](int w) -> cudaError_t {
        Slots sl;
        cudaError_t e = sl.open();
        const int64_t lo = n * w / W, hi = n * (w + 1) / W;
        int s = 0;
        int64_t pk0 = -1, pcnt = 0;   // chunk in flight in the other slot
        for (int64_t k0 = lo; k0 < hi && e == cudaSuccess; k0 += chunk) {
            const int64_t cnt = std::min(chunk, hi - k0);
            e = cudaMemcpyAsync(sl.buf[s], src + k0, sizeof(T) * (size_t)cnt, cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaEventRecord(sl.ev[s], st);
            sl.busy[s] = e == cudaSuccess;
            if (e == cudaSuccess && pk0 >= 0) {
                e = cudaEventSynchronize(sl.ev[s ^ 1]);
                sl.busy[s ^ 1] = false;
                if (e == cudaSuccess) drain(pk0, pcnt, (const T *)sl.buf[s ^ 1]);
            }
            pk0 = k0;
            pcnt = cnt;
            s ^= 1;
        }
        if (e == cudaSuccess && pk0 >= 0) {
            e = cudaEventSynchronize(sl.ev[s ^ 1]);
            sl.busy[s ^ 1] = false;
            if (e == cudaSuccess) drain(pk0, pcnt, (const T *)sl.buf[s ^ 1]);
        }
        cudaError_t c = sl.close();
        return e != cudaSuccess ? e : c;
    });
}

template <class T>
int download_copy(T *dst, const T *src, int64_t n, cudaStream_t st)
{
    return download(src, n, st, [dst](int64_t k0, int64_t cnt, const T *in) {
        std::memcpy(dst + k0, in, sizeof(T) * (size_t)cnt);
    });
}

}  // namespace staging
}  // namespace bbpd
