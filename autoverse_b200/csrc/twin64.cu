// FP64 twin of the 2D step: the engine's own device functions instantiated in
// double, so that the error of the f32 engine can be stated against an FP64
// build of the same arithmetic.
//
//   * convolution + growth: conv_direct_growth_2d<double> (kernels2d.cu), the
//     engine's direct torus convolution with the growth and the per-target
//     weighted sum in kernel order; taps from build_kernel_t<double> /
//     pad_kernel_t<double> (schema.cpp), the engine's stencil statements;
//   * flow: flow_mix / flow_destination<double> (transport_items.cuh), the
//     per-cell channel sum, Sobel, alpha, flow and destination of every flow
//     kernel, one thread per cell;
//   * reintegration: gather_generic_2d<POW2, double> (transport_items.cuh), the
//     engine's general gather path (bit-equal to its tiled fast paths in f32),
//     one thread per destination, visiting sources in the reference's deposit
//     order.
//
// Parameters are the f32 values the reference uses (config.rs parses f32),
// widened to double, as in the oracle's FP64 twin.  Diagnostic entry point:
// it allocates its own device buffers per call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "flowlenia_cuda.h"
#include "kernels.h"
#include "schema.h"
#include "transport_items.cuh"

namespace flp {

extern thread_local std::string g_last_error;

namespace {

__device__ __forceinline__ size_t at(int x, int y, int W) { return size_t(y) * W + x; }

// Channel sum of A at (x, y), channels added in order (propagator.rs:304-311).
__device__ __forceinline__ double chan_sum64(const double* A, int C, size_t N, size_t i) {
    double a = 0.0;
    for (int c = 0; c < C; ++c) a = rn_add(a, A[size_t(c) * N + i]);
    return a;
}

__global__ void twin_flow_2d(const double* __restrict__ A, const double* __restrict__ U, double* __restrict__ DX,
                             double* __restrict__ DY, int C, int W, int H, FlowParams fp,
                             unsigned long long* dmax_bits) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y;
    if (X >= W || Y >= H) return;
    const size_t N = size_t(W) * H;
    const int xl = wrap_near(X - 1, W), xr = wrap_near(X + 1, W);
    const int yt = wrap_near(Y - 1, H), yb = wrap_near(Y + 1, H);
    const size_t itl = at(xl, yt, W), itc = at(X, yt, W), itr = at(xr, yt, W);
    const size_t iml = at(xl, Y, W), imc = at(X, Y, W), imr = at(xr, Y, W);
    const size_t ibl = at(xl, yb, W), ibc = at(X, yb, W), ibr = at(xr, yb, W);
    const FlowMix<double> f =
        flow_mix(chan_sum64(A, C, N, itl), chan_sum64(A, C, N, itc), chan_sum64(A, C, N, itr),
                 chan_sum64(A, C, N, iml), chan_sum64(A, C, N, imc), chan_sum64(A, C, N, imr),
                 chan_sum64(A, C, N, ibl), chan_sum64(A, C, N, ibc), chan_sum64(A, C, N, ibr), fp);
    double dmax = 0.0;
    for (int c = 0; c < C; ++c) {
        const double* u = U + size_t(c) * N;
        double dx, dy;
        flow_destination(f, u[itl], u[itc], u[itr], u[iml], u[imr], u[ibl], u[ibc], u[ibr], X, Y, fp, dx, dy);
        DX[size_t(c) * N + imc] = dx;
        DY[size_t(c) * N + imc] = dy;
        if (fabs(A[size_t(c) * N + imc]) >= 1e-10f)
            dmax = fmax(dmax, fmax(fabs(dx - double(X)), fabs(dy - double(Y))));
    }
    // non-negative doubles order like their bit patterns; NaN or inf widen the window to the grid
    if (!(dmax <= 1e300)) dmax = 1e300;
    if (dmax > 0.0) atomicMax(dmax_bits, static_cast<unsigned long long>(__double_as_longlong(dmax)));
}

template <bool POW2>
__global__ void twin_gather_2d(const double* __restrict__ DX, const double* __restrict__ DY,
                               const double* __restrict__ A, double* __restrict__ out, int W, int H, int R,
                               FlowParams fp) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y, c = blockIdx.z;
    if (X >= W) return;
    const size_t off = size_t(c) * W * H;
    out[off + at(X, Y, W)] = gather_generic_2d<POW2, double>(DX + off, DY + off, A + off, W, H, X, Y, R, fp);
}

template <class T>
struct DevBuf {
    T* p = nullptr;
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)); }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

}  // namespace
}  // namespace flp

using namespace flp;

extern "C" int flp_twin64_step(const char* config_json, const double* state, double* affinity, double* next) {
    if (!config_json || !state || !next) {
        g_last_error = "null argument";
        return FLP_ERR_INVALID_ARGUMENT;
    }
    try {
        const SimulationConfig c = parse_config(config_json);
        if (c.is_3d()) {
            g_last_error = "flp_twin64_step serves 2D worlds only";
            return FLP_ERR_UNSUPPORTED;
        }
        const int W = c.width, H = c.height, C = c.channels, K = int(c.kernels.size());
        const size_t N = size_t(W) * H;
        // kernel descriptors and flipped effective taps, as the engine's direct
        // path builds them (kernel.rs:98-117), in double
        std::vector<KDesc64> kd(std::max(K, 1));
        std::vector<double> taps;
        int rmax = 0;
        for (int k = 0; k < K; ++k) {
            const KernelConfig& kc = c.kernels[k];
            const KernelStencilT<double> st = build_kernel_t<double>(kc, c.kernel_radius, 2);
            const int r = st.radius, side = st.size;
            rmax = std::max(rmax, r);
            const std::vector<double> pad = pad_kernel_t<double>(st, W, H, 1);
            std::vector<double> eff(size_t(side) * side, 0.0);
            std::vector<char> seen(N, 0);
            for (int dy = -r; dy <= r; ++dy)
                for (int dx = -r; dx <= r; ++dx) {
                    const int tx = ((dx % W) + W) % W, ty = ((dy % H) + H) % H;
                    const size_t t = size_t(ty) * W + tx;
                    if (seen[t]) continue;
                    seen[t] = 1;
                    eff[size_t(-dy + r) * side + (-dx + r)] = pad[t];
                }
            KDesc64 d{};
            d.src = kc.source_channel;
            d.tgt = kc.target_channel;
            d.r = r;
            d.tap_off = int(taps.size());
            d.weight = double(kc.weight);
            d.mu = double(kc.mu);
            const double sigma = double(kc.sigma);
            d.inv2s2 = 1.0 / (2.0 * sigma * sigma);
            kd[k] = d;
            taps.insert(taps.end(), eff.begin(), eff.end());
        }
        const FlowParams fp = flow_params_of(c);
        DevBuf<double> dA, dU, dDX, dDY, dOut, dTaps;
        DevBuf<KDesc64> dKd;
        DevBuf<unsigned long long> dDmax;
        cudaError_t e = cudaSuccess;
        for (auto* b : {&dA, &dU, &dDX, &dDY, &dOut})
            if (e == cudaSuccess) e = b->alloc(size_t(C) * N);
        if (e == cudaSuccess) e = dTaps.alloc(taps.size());
        if (e == cudaSuccess) e = dKd.alloc(kd.size());
        if (e == cudaSuccess) e = dDmax.alloc(1);
        if (e == cudaSuccess) e = cudaMemcpy(dA.p, state, sizeof(double) * C * N, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && !taps.empty())
            e = cudaMemcpy(dTaps.p, taps.data(), sizeof(double) * taps.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dKd.p, kd.data(), sizeof(KDesc64) * kd.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(dDmax.p, 0, sizeof(unsigned long long));
        if (e == cudaSuccess) e = cudaMemset(dU.p, 0, sizeof(double) * C * N);
        if (e != cudaSuccess) {
            g_last_error = std::string("twin set-up: ") + cudaGetErrorString(e);
            return e == cudaErrorMemoryAllocation ? FLP_ERR_OOM : FLP_ERR_CUDA;
        }
        if (K > 0) e = launch_conv_direct_2d_f64(dA.p, dU.p, dKd.p, K, dTaps.p, W, H, C, rmax);
        if (e == cudaSuccess) {
            twin_flow_2d<<<dim3((W + 127) / 128, H), 128>>>(dA.p, dU.p, dDX.p, dDY.p, C, W, H, fp, dDmax.p);
            e = cudaGetLastError();
        }
        unsigned long long bits = 0;
        if (e == cudaSuccess) e = cudaMemcpy(&bits, dDmax.p, sizeof(bits), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            g_last_error = std::string("twin convolution/flow: ") + cudaGetErrorString(e);
            return FLP_ERR_CUDA;
        }
        // Window: every source that can reach a destination, plus one cell; a
        // wider window adds only sources without overlap, which are skipped.
        // Capped like the engine's window (a non-finite displacement reaches
        // every cell); windows wider than the grid take the general path's
        // frame-by-frame visit.
        double dmax = 0.0;
        std::memcpy(&dmax, &bits, sizeof(dmax));
        const double reach = std::ceil(dmax + double(fp.s)) + 1.0;
        const int cap = 2 * std::max(W, H) + 2;
        const int R = reach < double(cap) ? std::max(1, int(reach)) : cap;
        if (fp.area_pow2)
            twin_gather_2d<true><<<dim3((W + 127) / 128, H, C), 128>>>(dDX.p, dDY.p, dA.p, dOut.p, W, H, R, fp);
        else
            twin_gather_2d<false><<<dim3((W + 127) / 128, H, C), 128>>>(dDX.p, dDY.p, dA.p, dOut.p, W, H, R, fp);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(next, dOut.p, sizeof(double) * C * N, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess && affinity)
            e = cudaMemcpy(affinity, dU.p, sizeof(double) * C * N, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) {
            g_last_error = std::string("twin gather: ") + cudaGetErrorString(e);
            return FLP_ERR_CUDA;
        }
        return FLP_OK;
    } catch (const ConfigError& ex) {
        g_last_error = ex.what();
        return FLP_ERR_INVALID_CONFIG;
    } catch (const std::exception& ex) {
        g_last_error = ex.what();
        return FLP_ERR_INVALID_ARGUMENT;
    }
}
