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

// The same descriptor with double parameters, for the FP64 twin (twin64.cu).
struct KDesc64 {
    int src, tgt;
    int r;
    int tap_off;
    double weight, mu, inv2s2;
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

// Round-to-nearest arithmetic without contraction, for the f32 engine and for
// the same functions instantiated in double (the FP64 twin, twin64.cu).
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float rn_div(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rn_div(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float r_pow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double r_pow(double a, double b) { return pow(a, b); }
__device__ __forceinline__ float r_exp(float a) { return expf(a); }
__device__ __forceinline__ double r_exp(double a) { return exp(a); }

// alpha = clamp((A/beta)^n, 0, 1) with the reference's integer-n fast paths
// (src/compute/flow.rs:14-32).  Division is IEEE (nvcc default prec-div).
template <class T>
__device__ __forceinline__ T flow_alpha(T mass, T beta_a, T n) {
    T ratio = rn_div(mass, beta_a);
    T p;
    if (n == T(1)) p = ratio;
    else if (n == T(2)) p = rn_mul(ratio, ratio);
    else if (n == T(3)) p = rn_mul(rn_mul(ratio, ratio), ratio);
    else if (n == T(4)) { T r2 = rn_mul(ratio, ratio); p = rn_mul(r2, r2); }
    else p = r_pow(ratio, n);
    if (p < T(0)) p = T(0);
    if (p > T(1)) p = T(1);
    return p;
}

// 2D Sobel, gradient.rs:99-102, evaluated left to right without contraction.
template <class T>
__device__ __forceinline__ void sobel2(T tl, T tc, T tr, T ml, T mr, T bl, T bc, T br, T& gx, T& gy) {
    T x = rn_add(-tl, tr);
    x = rn_sub(x, rn_mul(T(2), ml));
    x = rn_add(x, rn_mul(T(2), mr));
    x = rn_sub(x, bl);
    x = rn_add(x, br);
    gx = rn_mul(x, T(0.125));
    T y = rn_sub(-tl, rn_mul(T(2), tc));
    y = rn_sub(y, tr);
    y = rn_add(y, bl);
    y = rn_add(y, rn_mul(T(2), bc));
    y = rn_add(y, br);
    gy = rn_mul(y, T(0.125));
}

}  // namespace flp
