// es_fault.h - host-side fault injection for the error paths of the C ABI.
//
// Every device allocation, host<->device copy and kernel launch of the
// lifetime, integration, batch and grid-build entry points goes through the
// wrappers below. When a plan is armed (es_fault_inject, or ES_FAULT_INJECT in
// the environment), the chosen operation reports a failure:
//   - an allocation fails before it is made (null pointer,
//     cudaErrorMemoryAllocation -> ES_ERR_OOM);
//   - a copy or a launch is issued, its stream is waited on, and only then is
//     the failure reported (-> ES_ERR_LAUNCH). Device and host memory hold
//     what an error-free call would have written and nothing is in flight when
//     the caller's error path runs, so an injected failure exercises the host's
//     error handling and can never turn into a device fault. Under graph
//     capture nothing executes, and the wait is skipped.
// Nothing here touches the GPU beyond the real operation itself.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace es {
namespace fault {

enum Kind : int { kAlloc = 0, kCopy = 1, kLaunch = 2, kKinds = 3 };

// Counts one operation of `kind`; true when the armed plan fails this one.
bool fire(Kind kind);

// The injected error of a copy or a launch that was issued on `s`.
cudaError_t after(Kind kind, cudaStream_t s);

}  // namespace fault

template <class T>
cudaError_t dev_malloc(T** p, size_t bytes)
{
    if (fault::fire(fault::kAlloc)) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(reinterpret_cast<void**>(p), bytes);
}

template <class T>
cudaError_t host_malloc(T** p, size_t bytes)
{
    if (fault::fire(fault::kAlloc)) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMallocHost(reinterpret_cast<void**>(p), bytes);
}

inline cudaError_t copy_async(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s)
{
    const cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, s);
    return e == cudaSuccess ? fault::after(fault::kCopy, s) : e;
}

inline cudaError_t copy_sync(void* dst, const void* src, size_t bytes, cudaMemcpyKind kind)
{
    const cudaError_t e = cudaMemcpy(dst, src, bytes, kind);
    return e == cudaSuccess ? fault::after(fault::kCopy, nullptr) : e;
}

// The status of the kernel launch just made on `s` (cudaGetLastError).
inline cudaError_t launched(cudaStream_t s)
{
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? fault::after(fault::kLaunch, s) : e;
}

}  // namespace es
