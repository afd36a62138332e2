// Allocation-free affinity entry point: flp_affinity_noalloc.
//
// Some callers must not allocate device memory: code that enqueues work from
// inside another framework's operator or plugin (an inference-engine plugin's
// enqueue, a compiler runtime's custom call) runs on that framework's stream
// and memory pool, where a cudaMalloc would synchronise the whole device and
// fragment the pool the framework manages.  For them this file runs the
// direct convolution + growth kernel (the same kernel flp_debug_affinity
// launches on the direct path) with its scratch -- the kernel descriptors and
// the wrap-padded stencil taps -- placed in one file-scope device array
// instead of cudaMalloc'd buffers.
//
// The array is NOALLOC_SCRATCH_BYTES (1 MiB) on every device that loads the
// library and lives until the process exits.  It is shared by all calls: each
// call overwrites the descriptors and taps it needs before its kernel runs,
// so nothing stale is read, but calls whose work overlaps on the GPU (two
// streams, or two host threads) race on the array and must be serialised by
// the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "flowlenia_cuda.h"
#include "kernels.h"
#include "schema.h"

namespace flp {

extern thread_local std::string g_last_error;

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(1) << 20;
constexpr int MAX_DEVICES = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[MAX_DEVICES] = {nullptr};

// Device address of the scratch array on the current device.  In host code
// `g_noalloc_scratch` names a host-side shadow, not device memory, so the
// address is looked up once per device with that device current.
int scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        g_last_error = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return FLP_ERR_CUDA;
    }
    if (dev < 0 || dev >= MAX_DEVICES) {
        g_last_error = "device ordinal out of range for the allocation-free path";
        return FLP_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            g_last_error = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
            return FLP_ERR_CUDA;
        }
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return FLP_OK;
}

}  // namespace
}  // namespace flp

using namespace flp;

extern "C" int flp_affinity_noalloc(const char* config_json, const float* d_state, float* d_affinity, void* stream) {
    if (!config_json || !d_state || !d_affinity) {
        g_last_error = "null argument";
        return FLP_ERR_INVALID_ARGUMENT;
    }
    try {
        SimulationConfig c = parse_config(config_json);
        if (c.is_3d()) {
            g_last_error = "flp_affinity_noalloc serves 2D worlds only";
            return FLP_ERR_UNSUPPORTED;
        }
        const int W = c.width, H = c.height, C = c.channels, K = int(c.kernels.size());
        // Descriptors and flipped effective taps, as the engine's direct path
        // builds them (wrap-padded stencil, kernel.rs:98-117).
        std::vector<KDesc> kd(K);
        std::vector<float> taps;
        int rmax = 0;
        for (int k = 0; k < K; ++k) {
            const KernelConfig& kc = c.kernels[k];
            KernelStencil st = build_kernel(kc, c.kernel_radius, 2);
            const int r = st.radius, side = st.size;
            if (r > MAX_DIRECT_RADIUS) {
                g_last_error = "kernel radius " + std::to_string(r) + " exceeds the direct path's maximum of " +
                               std::to_string(MAX_DIRECT_RADIUS);
                return FLP_ERR_INVALID_ARGUMENT;
            }
            rmax = std::max(rmax, r);
            std::vector<float> pad = pad_kernel(st, W, H, 1);
            std::vector<float> eff(size_t(side) * side, 0.f);
            std::vector<char> seen(size_t(W) * H, 0);
            for (int dy = -r; dy <= r; ++dy)
                for (int dx = -r; dx <= r; ++dx) {
                    const int tx = ((dx % W) + W) % W, ty = ((dy % H) + H) % H;
                    const size_t t = size_t(ty) * W + tx;
                    if (seen[t]) continue;
                    seen[t] = 1;
                    eff[size_t(-dy + r) * side + (-dx + r)] = pad[t];
                }
            KDesc d{};
            d.src = kc.source_channel;
            d.tgt = kc.target_channel;
            d.r = r;
            d.tap_off = int(taps.size());
            d.weight = kc.weight;
            d.mu = kc.mu;
            const float sigma_sq_2 = 2.0f * kc.sigma * kc.sigma;
            d.inv2s2 = 1.0f / sigma_sq_2;
            kd[k] = d;
            taps.insert(taps.end(), eff.begin(), eff.end());
        }
        const size_t kd_bytes = ((sizeof(KDesc) * size_t(K) + 255) / 256) * 256;
        const size_t need = kd_bytes + sizeof(float) * taps.size();
        if (need > NOALLOC_SCRATCH_BYTES) {
            g_last_error = "kernel descriptors and taps need " + std::to_string(need) +
                           " bytes; the allocation-free scratch holds " + std::to_string(NOALLOC_SCRATCH_BYTES);
            return FLP_ERR_INVALID_ARGUMENT;
        }
        void* base = nullptr;
        int rc = scratch_address(&base);
        if (rc != FLP_OK) return rc;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        unsigned char* b = static_cast<unsigned char*>(base);
        KDesc* d_kd = reinterpret_cast<KDesc*>(b);
        float* d_taps = reinterpret_cast<float*>(b + kd_bytes);
        cudaError_t e = cudaSuccess;
        if (K) e = cudaMemcpyAsync(d_kd, kd.data(), sizeof(KDesc) * K, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess && !taps.empty())
            e = cudaMemcpyAsync(d_taps, taps.data(), sizeof(float) * taps.size(), cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) {
            g_last_error = std::string("copy into scratch: ") + cudaGetErrorString(e);
            return FLP_ERR_CUDA;
        }
        if (K == 0) {
            e = cudaMemsetAsync(d_affinity, 0, sizeof(float) * size_t(C) * W * H, st);
        } else {
            launch_conv_direct_2d(d_state, d_affinity, d_kd, K, d_taps, W, H, C, rmax, nullptr, st);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) {
            g_last_error = std::string("affinity launch: ") + cudaGetErrorString(e);
            return FLP_ERR_CUDA;
        }
        return FLP_OK;
    } catch (const ConfigError& e) {
        g_last_error = e.what();
        return FLP_ERR_INVALID_CONFIG;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return FLP_ERR_INVALID_ARGUMENT;
    }
}
