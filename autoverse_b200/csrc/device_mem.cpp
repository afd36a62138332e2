// dmalloc / dfree: counted device allocations with host-side failure
// injection (see device_mem.h).
#include "device_mem.h"

#include <atomic>
#include <chrono>
#include <thread>

#include "flowlenia_cuda.h"

namespace flp {

namespace {
std::atomic<long long> g_live{0};
std::atomic<long long> g_fail_after{-1};  // < 0: never fail
}  // namespace

cudaError_t dmalloc_bytes(void** p, size_t bytes) {
    long long n = g_fail_after.load();
    while (n >= 0) {
        if (n == 0) {
            *p = nullptr;
            return cudaErrorMemoryAllocation;
        }
        if (g_fail_after.compare_exchange_weak(n, n - 1)) break;
    }
    const cudaError_t e = cudaMalloc(p, bytes ? bytes : 1);
    if (e == cudaSuccess) g_live.fetch_add(1);
    return e;
}

void dfree(void* p) {
    if (!p) return;
    if (cudaFree(p) == cudaSuccess) g_live.fetch_sub(1);
}

bool wait_stream_for(cudaStream_t st, double timeout_ms) {
    using clock = std::chrono::steady_clock;
    const auto end = clock::now() + std::chrono::duration<double, std::milli>(timeout_ms < 0 ? 0 : timeout_ms);
    for (;;) {
        const cudaError_t e = cudaStreamQuery(st);
        if (e == cudaSuccess) return true;
        if (e != cudaErrorNotReady) throw_cuda(e, "stream query");
        if (clock::now() >= end) return false;
        std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

}  // namespace flp

extern "C" int flp_debug_fail_device_alloc(int64_t after) {
    flp::g_fail_after.store(after < 0 ? -1 : after);
    return FLP_OK;
}

extern "C" int flp_debug_live_device_allocs(int64_t* live) {
    if (!live) return FLP_ERR_INVALID_ARGUMENT;
    *live = flp::g_live.load();
    return FLP_OK;
}
