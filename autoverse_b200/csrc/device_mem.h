// Device allocations of the engine.  Every cudaMalloc / cudaFree of the
// library goes through dmalloc / dfree, which keep a count of live
// allocations and can be told to fail: after `n` further successful
// allocations the next one returns cudaErrorMemoryAllocation without calling
// the driver.  This is host-side failure injection for the out-of-memory paths
// of the create and reconfigure calls (each must return FLP_ERR_OOM and give
// back everything it allocated); no kernel is involved.
#pragma once

#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

namespace flp {

cudaError_t dmalloc_bytes(void** p, size_t bytes);
void dfree(void* p);

template <class T>
cudaError_t dmalloc(T** p, size_t bytes) {
    return dmalloc_bytes(reinterpret_cast<void**>(p), bytes);
}

// Thrown by the batched, embedded and recorder paths when a device allocation
// fails; their C entry points turn it into FLP_ERR_OOM.
struct DeviceOom : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// cudaErrorMemoryAllocation -> DeviceOom, any other failure -> runtime_error.
inline void throw_cuda(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return;
    const std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (e == cudaErrorMemoryAllocation) throw DeviceOom(m);
    throw std::runtime_error(m);
}

// Temporary device buffers of one scope, freed on every way out of it
// (exceptions included); cudaFree waits for the work that still uses them.
struct DevScratch {
    std::vector<void*> ptrs;
    DevScratch() = default;
    DevScratch(const DevScratch&) = delete;
    DevScratch& operator=(const DevScratch&) = delete;
    ~DevScratch() {
        for (void* p : ptrs) dfree(p);
    }
    template <class T>
    T* add(T* p) {
        ptrs.push_back(p);
        return p;
    }
};

// Waits for `st` on the host, polling, for at most timeout_ms; true when the
// stream finished (its errors are then reported by the caller's next check),
// false when the time ran out with work still pending (nothing is cancelled).
// Any failure reported by the stream query is thrown.
bool wait_stream_for(cudaStream_t st, double timeout_ms);

}  // namespace flp
