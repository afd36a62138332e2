// FFT convolution for 3D worlds (replaces CachedConvolver3D,
// src/compute/fft3d.rs:262-452, and growth_accumulate, growth.rs:45-59 /
// propagator3d.rs:147-157).
//
// Spectra are kept x-bin-major, [kx][z][y] (W/2+1 half-spectrum bins), so
// that the x transforms are the 2D row items over the D*H rows of the grid,
// the y transforms are contiguous column items, and the z transforms read NZ
// adjacent y's per z.  A step is five kernels: x R2C, y forward, z forward *
// K^ * z inverse (per kernel), y inverse, x C2R + growth.
#include "common.cuh"
#include "fft_items.cuh"
#include "kernels.h"

namespace flp {

#define FLP_Z_SIZES(X) X(32) X(48) X(64) X(96) X(128) X(192) X(256)

template <int D>
__global__ void __launch_bounds__(256) k_zconv_t(const float2* __restrict__ S, const float2* __restrict__ KH,
                                                 float2* __restrict__ T, const int* __restrict__ slot_of_kernel,
                                                 int Wc, int H, int mode, float scale,
                                                 const float2* __restrict__ twD) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    constexpr int NZ = ZCfg<D>::NZ;
    const int groups = (H + NZ - 1) / NZ;
    const int kx = blockIdx.x / groups, g = blockIdx.x - kx * groups;
    const int k = blockIdx.y;
    const int slot = mode == 0 ? slot_of_kernel[k] : k;
    const int y0 = g * NZ;
    const int ny = min(NZ, H - y0);
    const size_t plane = size_t(D) * H;  // one kx block: [z][y]
    zconv_item<D>(fsm, S + (size_t(slot) * Wc + kx) * plane, mode == 0 ? KH + (size_t(k) * Wc + kx) * plane : nullptr,
                  T + (size_t(k) * Wc + kx) * plane, H, y0, ny, mode, scale, twD);
}

bool fft_z_templated(int D) {
#define X(n) if (D == n) return true;
    FLP_Z_SIZES(X)
#undef X
    return false;
}

void fft3d_set_attributes(size_t max_bytes) {
#define X(n)                                                                                        \
    cudaFuncSetAttribute((const void*)k_zconv_t<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(max_bytes)); \
    cudaFuncSetAttribute((const void*)k_zconv_t<n>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    FLP_Z_SIZES(X)
#undef X
}

void launch_fft_z(const float2* S, const float2* KH, float2* T, const int* slot_of_kernel, int nlines_k, int W, int H,
                  int D, const float2* twD, int mode, float scale, cudaStream_t st) {
    const int Wc = W / 2 + 1;
#define X(n)                                                                                                  \
    if (D == n) {                                                                                             \
        const int groups = (H + ZCfg<n>::NZ - 1) / ZCfg<n>::NZ;                                               \
        launch_dep(k_zconv_t<n>, dim3(Wc * groups, nlines_k), 256, ZCfg<n>::smem, st, S, KH, T, slot_of_kernel, Wc, H, mode, \
                                                                             scale, twD);                     \
        return;                                                                                               \
    }
    FLP_Z_SIZES(X)
#undef X
}

}  // namespace flp
