// es_upload.h - host-to-device copies of caller arrays held in pageable memory,
// through a pinned staging ring.
//
// A cudaMemcpyAsync from pageable memory is staged by the CUDA driver through its
// own pinned buffers on the calling thread. The grid uploads of the C ABI
// (es_upload_grid, es_batch_add_grid: tens to hundreds of MB per grid) instead
// copy each chunk into a pinned ring slot with several host threads while the
// DMA of the previous chunk runs. A source that is already pinned (or
// registered, managed, device) memory is copied directly, and small copies
// take the CUDA driver's own staging. The reference uploads with clEnqueueWriteBuffer from
// its std::vectors (src/sim/SimulationCL.cpp:121-122).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace es {

class Staging {
public:
    Staging() = default;
    ~Staging() { release(); }
    Staging(const Staging&) = delete;
    Staging& operator=(const Staging&) = delete;

    // Enqueues dst (device) <- src (host, `bytes`) on `s`. When it returns, the
    // source may be reused if it was pageable; a pinned source is read by the
    // DMA until `s` reaches this point. Copies go through es::copy_async, so
    // fault injection counts each chunk as one copy.
    cudaError_t h2d(void* dst, const void* src, size_t bytes, cudaStream_t s);

    // Frees the ring (after its last copies have completed).
    void release();

    static constexpr size_t kChunk = size_t(16) << 20;  // bytes per ring slot
    static constexpr int kSlots = 2;

private:
    cudaError_t ensure();

    unsigned char* buf_ = nullptr;  // pinned, kSlots * kChunk bytes
    cudaEvent_t done_[kSlots] = {};
    bool busy_[kSlots] = {};
};

// True when `p` is host memory the DMA engines can read directly (pinned or
// registered), or managed or device memory.
bool dma_readable(const void* p);

}  // namespace es
