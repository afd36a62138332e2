// 2D step kernels of the Flow Lenia engine (sm_100a):
//   * conv_direct_growth_2d — shared-memory tiled torus convolution with the
//     growth function and the per-target weighted sum fused into its epilogue
//     (src/compute/fft.rs:288-324 + growth.rs:45-59 + propagator.rs:270-279);
//   * transport_2d — one pass that forms the channel sum, both Sobel
//     gradients, alpha, the flow and the reintegrated mass, in gather form
//     (propagator.rs:304-371, gradient.rs:68-108, flow.rs:68-87,
//     reintegration.rs:60-167);
//   * the flow-bound reduction and the FP64 compensated mass reduction.
//
// Arithmetic that the reference performs in f32 is written with explicit
// round-to-nearest intrinsics (__fadd_rn/__fmul_rn/...) so that nvcc cannot
// contract it into FMAs: the per-source destinations, overlap areas and
// deposited masses are then bit-identical to the reference's, and the gather
// visits sources in the reference's scatter order, so the transport stage
// reproduces CpuPropagator bit for bit given the same affinity field.
#include "common.cuh"
#include "kernels.h"
#include "transport_items.cuh"

#include <math.h>

namespace flp {

// ---------------------------------------------------------------------------
// Direct convolution + growth.
// Block 32x8 threads, tile 32x32 outputs (4 per thread, rows ty+8i).
// blockIdx.z selects the target channel; kernels targeting it are applied in
// kernel order and their weighted growth is accumulated in that order.
// ---------------------------------------------------------------------------
constexpr int CD_TW = 32, CD_TH = 32;

// T = float in the engine; the FP64 twin (twin64.cu) instantiates the same
// kernel in double with a descriptor type of double parameters.
__device__ __forceinline__ float r_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double r_fma(double a, double b, double c) { return fma(a, b, c); }

template <class T, class KD>
__global__ void __launch_bounds__(256) conv_direct_growth_2d(const T* __restrict__ A, T* __restrict__ U,
                                                             const KD* __restrict__ kd, int K,
                                                             const T* __restrict__ taps, int W, int H, int rmax,
                                                             int* reset_slot, int nreset) {
    dep_enter();
    extern __shared__ __align__(16) unsigned char conv_sm[];
    T* sm = reinterpret_cast<T*>(conv_sm);
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int tid = ty * 32 + tx;
    const int c = blockIdx.z;
    const int x0 = blockIdx.x * CD_TW, y0 = blockIdx.y * CD_TH;
    const size_t N = size_t(W) * H;
    if (reset_slot && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && tid == 0)
        for (int i = 0; i < nreset; ++i) reset_slot[i] = 0;
    const int Pmax = CD_TW + 2 * rmax;
    T* tile = sm;                                   // (CD_TH + 2r) x (CD_TW + 2r)
    T* tsm = sm + size_t(CD_TH + 2 * rmax) * Pmax;  // taps
    T accu[4] = {T(0), T(0), T(0), T(0)};
    int loaded_src = -1, loaded_r = -1;
    for (int k = 0; k < K; ++k) {
        const KD d = kd[k];
        if (d.tgt != c) continue;
        const int r = d.r, side = 2 * r + 1, P = CD_TW + 2 * r;
        __syncthreads();
        for (int i = tid; i < side * side; i += 256) tsm[i] = taps[d.tap_off + i];
        if (d.src != loaded_src || r != loaded_r) {
            const T* a = A + size_t(d.src) * N;
            const int rows = CD_TH + 2 * r;
            for (int i = tid; i < rows * P; i += 256) {
                int ly = i / P, lx = i - ly * P;
                int gy = wrap_coord(y0 - r + ly, H), gx = wrap_coord(x0 - r + lx, W);
                tile[i] = a[size_t(gy) * W + gx];
            }
            loaded_src = d.src;
            loaded_r = r;
        }
        __syncthreads();
        // Each stencil row is summed on its own (fused multiply-adds), then the
        // row sums are added: two chains of 2r+1 roundings instead of one of
        // (2r+1)^2, which keeps the sum's rounding error near that of an f32 FFT.
        T acc[4] = {T(0), T(0), T(0), T(0)};
        for (int dy = 0; dy < side; ++dy) {
            const T* trow = tsm + dy * side;
            const T* base = tile + (ty + dy) * P + tx;
            T row[4] = {T(0), T(0), T(0), T(0)};
            for (int dx = 0; dx < side; ++dx) {
                const T t = trow[dx];
#pragma unroll
                for (int i = 0; i < 4; ++i) row[i] = r_fma(t, base[(8 * i) * P + dx], row[i]);
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) acc[i] = rn_add(acc[i], row[i]);
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            T diff = rn_sub(acc[i], T(d.mu));
            T e = r_exp(rn_mul(rn_mul(-diff, diff), T(d.inv2s2)));
            T g = rn_sub(rn_mul(T(2), e), T(1));
            accu[i] = rn_add(accu[i], rn_mul(T(d.weight), g));
        }
    }
    T* u = U + size_t(c) * N;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        int y = y0 + ty + 8 * i, x = x0 + tx;
        if (x < W && y < H) u[size_t(y) * W + x] = accu[i];
    }
}

size_t conv_direct_smem_bytes(int rmax) {
    int P = CD_TW + 2 * rmax;
    int side = 2 * rmax + 1;
    return sizeof(float) * (size_t(CD_TH + 2 * rmax) * P + size_t(side) * side);
}

void launch_conv_direct_2d(const float* A, float* U, const KDesc* kd, int K, const float* taps, int W, int H, int C,
                           int rmax, int* reset_slot, cudaStream_t st) {
    dim3 grid((W + CD_TW - 1) / CD_TW, (H + CD_TH - 1) / CD_TH, C);
    size_t smem = conv_direct_smem_bytes(rmax);
    launch_dep(conv_direct_growth_2d<float, KDesc>, grid, dim3(32, 8), smem, st, A, U, kd, K, taps, W, H, rmax,
               reset_slot, 1);
}

// The direct convolution instantiated in double (FP64 twin); its shared
// memory exceeds the default 48 KB above r = 15.
cudaError_t launch_conv_direct_2d_f64(const double* A, double* U, const KDesc64* kd, int K, const double* taps, int W,
                                      int H, int C, int rmax) {
    const int P = CD_TW + 2 * rmax, side = 2 * rmax + 1;
    const size_t smem = sizeof(double) * (size_t(CD_TH + 2 * rmax) * P + size_t(side) * side);
    cudaError_t e = cudaFuncSetAttribute(conv_direct_growth_2d<double, KDesc64>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return e;
    dim3 grid((W + CD_TW - 1) / CD_TW, (H + CD_TH - 1) / CD_TH, C);
    conv_direct_growth_2d<double, KDesc64><<<grid, dim3(32, 8), smem>>>(A, U, kd, K, taps, W, H, rmax, nullptr, 0);
    return cudaGetLastError();
}

size_t flow_smem_bytes(int C) { return flow_smem_bytes_inl(C); }
size_t gather_smem_bytes() { return gather_smem_bytes_inl(1); }

__global__ void __launch_bounds__(256) flow_2d(const float* __restrict__ A, const float* __restrict__ U,
                                               float* __restrict__ DX, float* __restrict__ DY, int C, int W, int H,
                                               FlowParams fp, int* dmax_slot, int* status) {
    dep_enter();
    extern __shared__ __align__(16) float sm[];
    flow_item(sm, A, U, DX, DY, C, W, H, fp, blockIdx.x * FL_W, blockIdx.y * FL_H, dmax_slot, status);
}

// Tile of a gather block: the launch is one wave and a half, and tiles on the
// torus edges (whose threads take the wrap passes) are the slowest, so the
// block index enumerates them first: tiles on an x and a y edge, on an x edge
// only, on a y edge only, then the rest, each category row by row with the
// channels innermost.  ntx x nty tiles per channel, C channels.
__device__ __forceinline__ void gather_tile_of(int b, int ntx, int nty, int C, int& tx, int& ty, int& c) {
    const int ex = min(2, ntx), ix = ntx - ex, ey = min(2, nty), iy = nty - ey;
    const int ncol[4] = {ex, ex, ix, ix}, nrow[4] = {ey, iy, ey, iy};
    int k = 0;
    for (; k < 3; ++k) {
        const int n = ncol[k] * nrow[k] * C;
        if (b < n) break;
        b -= n;
    }
    c = b % C;
    const int t = b / C, col = t % ncol[k], row = t / ncol[k];
    tx = k < 2 ? (col == 0 ? 0 : ntx - 1) : 1 + col;   // edge columns 0 and ntx-1, interior 1..ntx-2
    ty = (k == 0 || k == 2) ? (row == 0 ? 0 : nty - 1) : 1 + row;
}

template <bool POW2, int GBY>
__global__ void __launch_bounds__(256, 3) gather_2d(const float* __restrict__ DX, const float* __restrict__ DY,
                                                    const float* __restrict__ A, float* __restrict__ Anext, int W,
                                                    int H, int C, FlowParams fp, const int* __restrict__ dmax_slot) {
    dep_enter();
    extern __shared__ __align__(16) float sm[];
    int tx, ty, c;
    gather_tile_of(blockIdx.x, (W + GT_W - 1) / GT_W, (H + gt_h(GBY) - 1) / gt_h(GBY), C, tx, ty, c);
    const size_t N = size_t(W) * H;
    gather_item<POW2, GBY>(sm, DX + size_t(c) * N, DY + size_t(c) * N, A + size_t(c) * N, Anext + size_t(c) * N, W,
                           H, fp, *dmax_slot, tx * GT_W, ty * gt_h(GBY));
}

template <int C>
__global__ void __launch_bounds__(256) flow_rows_2d(const float* __restrict__ A, const float* __restrict__ U,
                                                    float* __restrict__ DX, float* __restrict__ DY, int W, int H,
                                                    FlowParams fp, int* dmax_slot, int* status) {
    dep_enter();
    flow_rows_item<C>(A, U, DX, DY, W, H, fp, blockIdx.x * 32, blockIdx.y * FR_H, dmax_slot, status);
}

// One compiled kernel per channel count 1..4 (the register-resident row walk),
// the staged kernel for more channels.
void launch_flow_2d(const float* A, const float* U, float* DX, float* DY, int C, int W, int H,
                    const FlowParams& fp, int* dmax_slot, int* status, cudaStream_t st) {
    if (C >= 1 && C <= 4) {
        const dim3 g((W + 31) / 32, (H + FR_H - 1) / FR_H);
        switch (C) {
            case 1: launch_dep(flow_rows_2d<1>, g, 256, 0, st, A, U, DX, DY, W, H, fp, dmax_slot, status); return;
            case 2: launch_dep(flow_rows_2d<2>, g, 256, 0, st, A, U, DX, DY, W, H, fp, dmax_slot, status); return;
            case 3: launch_dep(flow_rows_2d<3>, g, 256, 0, st, A, U, DX, DY, W, H, fp, dmax_slot, status); return;
            default: launch_dep(flow_rows_2d<4>, g, 256, 0, st, A, U, DX, DY, W, H, fp, dmax_slot, status); return;
        }
    }
    dim3 grid((W + FL_W - 1) / FL_W, (H + FL_H - 1) / FL_H);
    launch_dep(flow_2d, grid, 256, flow_smem_bytes(C), st, A, U, DX, DY, C, W, H, fp, dmax_slot, status);
}

void launch_gather_2d(const float* DX, const float* DY, const float* A, float* Anext, int C, int W, int H,
                      const FlowParams& fp, const int* dmax_slot, int gby, cudaStream_t st) {
    if (gby == 2) {
        const int tiles = ((W + GT_W - 1) / GT_W) * ((H + gt_h(2) - 1) / gt_h(2)) * C;
        const size_t smem = gather_smem_bytes_inl(2);
        if (fp.area_pow2)
            launch_dep(gather_2d<true, 2>, dim3(tiles), 256, smem, st, DX, DY, A, Anext, W, H, C, fp, dmax_slot);
        else
            launch_dep(gather_2d<false, 2>, dim3(tiles), 256, smem, st, DX, DY, A, Anext, W, H, C, fp, dmax_slot);
        return;
    }
    const int tiles = ((W + GT_W - 1) / GT_W) * ((H + gt_h(1) - 1) / gt_h(1)) * C;
    const size_t smem = gather_smem_bytes();
    if (fp.area_pow2)
        launch_dep(gather_2d<true, 1>, dim3(tiles), 256, smem, st, DX, DY, A, Anext, W, H, C, fp, dmax_slot);
    else
        launch_dep(gather_2d<false, 1>, dim3(tiles), 256, smem, st, DX, DY, A, Anext, W, H, C, fp, dmax_slot);
}

void transport_2d_set_attributes() {
    auto set = [](const void* f, size_t bytes) {
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
        cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    };
    set((const void*)flow_2d, flow_smem_bytes(64));
    set((const void*)gather_2d<true, 1>, gather_smem_bytes());
    set((const void*)gather_2d<false, 1>, gather_smem_bytes());
    set((const void*)gather_2d<true, 2>, gather_smem_bytes_inl(2));
    set((const void*)gather_2d<false, 2>, gather_smem_bytes_inl(2));
    cudaFuncSetAttribute(conv_direct_growth_2d<float, KDesc>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         int(conv_direct_smem_bytes(MAX_DIRECT_RADIUS)));
}

__global__ void zero_ints_kernel(int* p, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = 0;
}

void launch_zero_ints(int* p, int n, cudaStream_t st) {
    if (p && n > 0) zero_ints_kernel<<<1, 32, 0, st>>>(p, n);
}

// ---------------------------------------------------------------------------
// FP64 compensated (Neumaier) mass reduction, deterministic two-pass.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void neumaier_add(double& s, double& c, double x) {
    double t = s + x;
    if (fabs(s) >= fabs(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

__device__ __forceinline__ void neumaier_merge(double& s, double& c, double s2, double c2) {
    neumaier_add(s, c, s2);
    c += c2;
}

// Block merge in thread order (deterministic); the result is valid in thread 0.
__device__ void block_neumaier(double& s, double& c) {
    __shared__ double ss[256], cs[256];
    ss[threadIdx.x] = s;
    cs[threadIdx.x] = c;
    __syncthreads();
    if (threadIdx.x < 32) {
        double S = ss[threadIdx.x * 8], Cc = cs[threadIdx.x * 8];
        for (int i = 1; i < 8; ++i) neumaier_merge(S, Cc, ss[threadIdx.x * 8 + i], cs[threadIdx.x * 8 + i]);
        ss[threadIdx.x * 8] = S;
        cs[threadIdx.x * 8] = Cc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double S = ss[0], Cc = cs[0];
        for (int w = 1; w < 32; ++w) neumaier_merge(S, Cc, ss[w * 8], cs[w * 8]);
        s = S;
        c = Cc;
    }
}

__global__ void __launch_bounds__(256) mass_partial(const float* __restrict__ A, size_t n, double2* partial) {
    double s = 0.0, c = 0.0;
    for (size_t i = blockIdx.x * size_t(256) + threadIdx.x; i < n; i += size_t(gridDim.x) * 256)
        neumaier_add(s, c, double(A[i]));
    block_neumaier(s, c);
    if (threadIdx.x == 0) partial[blockIdx.x] = make_double2(s, c);
}

__global__ void __launch_bounds__(256) mass_final(const double2* partial, int np, double* out) {
    double s = 0.0, c = 0.0;
    for (int i = threadIdx.x; i < np; i += 256) neumaier_merge(s, c, partial[i].x, partial[i].y);
    block_neumaier(s, c);
    if (threadIdx.x == 0) out[0] = s + c;
}

void launch_mass_fp64(const float* A, size_t n, double2* partial, int np, double* out, cudaStream_t st) {
    mass_partial<<<np, 256, 0, st>>>(A, n, partial);
    mass_final<<<1, 256, 0, st>>>(partial, np, out);
}

}  // namespace flp
