// Device-side descriptors and helpers shared by the engine's kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace flp {

// Status word bits written by kernels (never trapped; read by the host).
enum : int {
    STATUS_NONFINITE = 1,  // a non-finite total mass reached the flow bound
};

// One convolution kernel (KernelConfig, src/schema/config.rs:54-70) as the
// device needs it.  inv2s2 = 1 / (2*sigma*sigma) evaluated in f32 exactly as
// growth_accumulate does (src/compute/growth.rs:52-53).
struct KDesc {
    int src, tgt;
    int r;        // stencil radius in cells
    int tap_off;  // offset of this kernel's (2r+1)^dims taps in the tap buffer
    float weight, mu, inv2s2;
    float pad;
};

// Flow/reintegration parameters of one world.
struct FlowParams {
    float dt;
    float s;            // distribution_size
    float total_area;   // (2s)*(2s) (or (2s)^3 in 3D), f32 as the reference computes it
    float inv_area;     // exact reciprocal when total_area is a power of two
    float beta_a, nexp;
    float pos_eps;      // absolute margin (cells) for rounding of positions in the gather window
    float inv_beta;     // 1 / beta_a when beta_a is a power of two (exact)
    int beta_pow2;
    int area_pow2;      // 1 when the division by total_area is a multiplication
    int point_mode;     // total_area < 1e-10: nearest-cell deposit
    int wide_square;    // area_pow2 and s >= 0.75: a square is wider than a cell plus any rounding of its ends
};

// Programmatic dependent launch.  The step's kernels are launched with
// programmatic stream serialization (launch_dep below), so a kernel's launch
// is processed while its predecessor in the stream drains; each such kernel
// waits at entry for the predecessor to complete with its writes visible
// (dep_enter) before it touches global memory.  No kernel signals its
// dependents early: the implicit signal at exit was measured faster than
// griddepcontrol.launch_dependents at entry (512x512 step 61.5 vs 65.6 us;
// parameter-embedded 256x256 step 55 vs 90 us), whose waiting blocks hold SM
// resources the running kernel needs.  Launched without the attribute, the
// wait is a no-op.
__device__ __forceinline__ void dep_enter() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Launch with programmatic stream serialization; the kernel must begin with
// dep_enter().  Errors surface through cudaGetLastError like a <<<>>> launch.
template <typename... KArgs, typename... Args>
inline void launch_dep(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args... args) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Float <-> order-preserving int, for atomicMax/atomicMin on floats.
__host__ __device__ inline int float_to_ordered(float f) {
#ifdef __CUDA_ARCH__
    int i = __float_as_int(f);
#else
    int i;
    static_assert(sizeof(float) == sizeof(int), "");
    __builtin_memcpy(&i, &f, 4);
#endif
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__host__ __device__ inline float ordered_to_float(int i) {
    int j = i >= 0 ? i : i ^ 0x7FFFFFFF;
#ifdef __CUDA_ARCH__
    return __int_as_float(j);
#else
    float f;
    __builtin_memcpy(&f, &j, 4);
    return f;
#endif
}

__device__ __forceinline__ int wrap_coord(int c, int size) { return ((c % size) + size) % size; }

// Wrap for coordinates a few sides off the torus: conditional add/subtract
// (no integer division); the loops run at most a handful of times even for
// grids narrower than a tile.
__device__ __forceinline__ int wrap_near(int c, int size) {
    while (c < 0) c += size;
    while (c >= size) c -= size;
    return c;
}

// alpha = clamp((A/beta)^n, 0, 1) with the reference's integer-n fast paths
// (src/compute/flow.rs:14-32).  Division is IEEE (nvcc default prec-div).
__device__ __forceinline__ float flow_alpha(float mass, float beta_a, float n) {
    float ratio = __fdiv_rn(mass, beta_a);
    float p;
    if (n == 1.0f) p = ratio;
    else if (n == 2.0f) p = __fmul_rn(ratio, ratio);
    else if (n == 3.0f) p = __fmul_rn(__fmul_rn(ratio, ratio), ratio);
    else if (n == 4.0f) { float r2 = __fmul_rn(ratio, ratio); p = __fmul_rn(r2, r2); }
    else p = powf(ratio, n);
    if (p < 0.0f) p = 0.0f;
    if (p > 1.0f) p = 1.0f;
    return p;
}

// 2D Sobel, gradient.rs:99-102, evaluated left to right without contraction.
__device__ __forceinline__ void sobel2(float tl, float tc, float tr, float ml, float mr, float bl, float bc, float br,
                                      float& gx, float& gy) {
    float x = __fadd_rn(-tl, tr);
    x = __fsub_rn(x, __fmul_rn(2.0f, ml));
    x = __fadd_rn(x, __fmul_rn(2.0f, mr));
    x = __fsub_rn(x, bl);
    x = __fadd_rn(x, br);
    gx = __fmul_rn(x, 0.125f);
    float y = __fsub_rn(-tl, __fmul_rn(2.0f, tc));
    y = __fsub_rn(y, tr);
    y = __fadd_rn(y, bl);
    y = __fadd_rn(y, __fmul_rn(2.0f, bc));
    y = __fadd_rn(y, br);
    gy = __fmul_rn(y, 0.125f);
}

}  // namespace flp
