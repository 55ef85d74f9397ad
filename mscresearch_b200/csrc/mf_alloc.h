// Device and pinned-host allocation wrapper of the host side.
//
// Every allocation the engine's host code makes goes through these calls.
// They forward to the CUDA runtime and keep a count of live allocations and
// bytes, so tests can check that a failed call leaves nothing behind.  A
// test can also make the k-th next allocation report cudaErrorMemoryAllocation
// without allocating (mf_debug_alloc_fail_after in the C ABI), which drives
// every allocation-failure path of an entry point on the host, with no fault
// on the GPU.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

cudaError_t mf_dmalloc_raw(void **p, size_t bytes);          // cudaMalloc
cudaError_t mf_dfree(void *p);                               // cudaFree
cudaError_t mf_hmalloc_raw(void **p, size_t bytes);          // cudaMallocHost
cudaError_t mf_hostalloc_raw(void **p, size_t bytes, unsigned flags);  // cudaHostAlloc
cudaError_t mf_hfree(void *p);                               // cudaFreeHost
// Stream-ordered device allocation (cudaMallocAsync / cudaFreeAsync): the
// server admits residual slots with it on a side stream while its
// persistent kernel runs.
cudaError_t mf_dmalloc_async_raw(void **p, size_t bytes, cudaStream_t st);
cudaError_t mf_dfree_async(void *p, cudaStream_t st);

template <class T>
inline cudaError_t mf_dmalloc(T **p, size_t bytes) {
    return mf_dmalloc_raw(reinterpret_cast<void **>(p), bytes);
}
template <class T>
inline cudaError_t mf_hmalloc(T **p, size_t bytes) {
    return mf_hmalloc_raw(reinterpret_cast<void **>(p), bytes);
}
template <class T>
inline cudaError_t mf_hostalloc(T **p, size_t bytes, unsigned flags) {
    return mf_hostalloc_raw(reinterpret_cast<void **>(p), bytes, flags);
}

// Device buffers that are freed when the scope ends unless released: an
// allocation sequence that fails half way leaves nothing allocated.
struct DevScope {
    std::vector<void *> p;
    template <class T>
    cudaError_t alloc(T **q, size_t bytes) {
        cudaError_t e = mf_dmalloc(q, bytes);
        if (e == cudaSuccess) p.push_back(*q);
        return e;
    }
    void release() { p.clear(); }
    ~DevScope() {
        for (void *x : p) mf_dfree(x);
    }
};
