// es_upload.cu - the pinned staging ring of es_upload.h.
//
// Each chunk of a pageable source is copied into a free ring slot by up to
// kMaxThreads host threads (one memcpy stripe each), then its DMA is enqueued
// and an event recorded; a slot is reused once its event has completed. With
// two slots the host copy of chunk k + 1 overlaps the DMA of chunk k.
#include "es_upload.h"

#include "es_fault.h"

#include <algorithm>
#include <cstring>
#include <thread>

namespace es {

namespace {

constexpr size_t kDirectBelow = size_t(1) << 20;  // smaller copies take the CUDA driver's own staging
constexpr int kMaxThreads = 8;
constexpr size_t kStripeMin = size_t(1) << 20;     // bytes per memcpy thread, at least

int copy_threads()
{
    static const int n = [] {
        const unsigned hw = std::thread::hardware_concurrency();
        return std::max(1, std::min(kMaxThreads, (int)(hw / 2)));
    }();
    return n;
}

// memcpy of n bytes with up to copy_threads() threads, in 64-byte aligned stripes.
void parallel_copy(unsigned char* dst, const unsigned char* src, size_t n)
{
    const int want = (int)std::min<size_t>((size_t)copy_threads(), std::max<size_t>(1, n / kStripeMin));
    if (want <= 1) {
        std::memcpy(dst, src, n);
        return;
    }
    const size_t stripe = ((n + want - 1) / want + 63) & ~size_t(63);
    std::thread workers[kMaxThreads];
    int started = 0;
    for (int t = 1; t < want; t++) {
        const size_t off = (size_t)t * stripe;
        if (off >= n) break;
        const size_t len = std::min(stripe, n - off);
        try {
            workers[t] = std::thread([=] { std::memcpy(dst + off, src + off, len); });
            started = t;
        } catch (...) {  // no thread to be had: this one copies the stripe
            std::memcpy(dst + off, src + off, len);
        }
    }
    std::memcpy(dst, src, std::min(stripe, n));
    for (int t = 1; t <= started; t++)
        if (workers[t].joinable()) workers[t].join();
}

}  // namespace

bool dma_readable(const void* p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();  // an unknown pointer is pageable host memory
        return false;
    }
    return a.type != cudaMemoryTypeUnregistered;
}

cudaError_t Staging::ensure()
{
    if (buf_) return cudaSuccess;
    cudaError_t e = host_malloc(&buf_, kChunk * kSlots);
    for (int k = 0; k < kSlots && e == cudaSuccess; k++) e = cudaEventCreateWithFlags(&done_[k], cudaEventDisableTiming);
    if (e != cudaSuccess) release();
    return e;
}

void Staging::release()
{
    for (int k = 0; k < kSlots; k++) {
        if (done_[k]) {
            if (busy_[k]) cudaEventSynchronize(done_[k]);
            cudaEventDestroy(done_[k]);
        }
        done_[k] = nullptr;
        busy_[k] = false;
    }
    if (buf_) cudaFreeHost(buf_);
    buf_ = nullptr;
}

cudaError_t Staging::h2d(void* dst, const void* src, size_t bytes, cudaStream_t s)
{
    if (bytes == 0) return cudaSuccess;
    if (bytes < kDirectBelow) return copy_async(dst, src, bytes, cudaMemcpyHostToDevice, s);
    if (dma_readable(src)) return copy_async(dst, src, bytes, cudaMemcpyDefault, s);
    cudaError_t e = ensure();
    if (e != cudaSuccess) return e;
    const unsigned char* from = static_cast<const unsigned char*>(src);
    unsigned char* to = static_cast<unsigned char*>(dst);
    int slot = 0;
    for (size_t off = 0; off < bytes; off += kChunk, slot = (slot + 1) % kSlots) {
        const size_t len = std::min(kChunk, bytes - off);
        if (busy_[slot]) {
            if ((e = cudaEventSynchronize(done_[slot])) != cudaSuccess) return e;
            busy_[slot] = false;
        }
        unsigned char* ring = buf_ + (size_t)slot * kChunk;
        parallel_copy(ring, from + off, len);
        if ((e = copy_async(to + off, ring, len, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(done_[slot], s)) != cudaSuccess) {
            cudaStreamSynchronize(s);  // the ring slot is free again only once its DMA is done
            return e;
        }
        busy_[slot] = true;
    }
    return cudaSuccess;
}

}  // namespace es
