// Launch interface between the host runtime (engine.cu) and the kernels.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "common.cuh"

namespace flp {

constexpr int MAX_DIRECT_RADIUS = 24;

// Radix plan of one FFT length (radices 4, 2, 3, 5, in that order).
struct FftPlan {
    int L = 1;
    int nst = 0;
    int rad[24] = {0};
};

// Geometry and twiddle tables of one 2D world for the FFT path.
struct FftGeom {
    int NR = 8;  // rows per CTA in the row passes
    int NC = 8;  // columns per CTA in the column pass
    FftPlan pm;  // length W/2
    FftPlan ph;  // length H
    const float2* twM = nullptr;  // exp(-2 pi i t / (W/2)), t < W/2
    const float2* twW = nullptr;  // exp(-2 pi i t / W),     t <= W/2
    const float2* twH = nullptr;  // exp(-2 pi i t / H),     t < H
    const float2* twD = nullptr;  // exp(-2 pi i t / D),     t < D (3D only)
    // Warp-synchronous passes (sizes with a compiled plan): warps per CTA of
    // the row R2C, column and row C2R passes (4 or 8), and whether a column
    // CTA transforms a source once for all the kernels that read it (share)
    // or each kernel's column CTA transforms its own source (more CTAs).
    // Every choice computes the same bits.
    int wpc_r2c = 8, wpc_cols = 8, wpc_c2r = 8;
    int share_cols = 1;
};

bool make_plan(int L, FftPlan& p);

// Flow and reintegration parameters of one world (engine.cu), shared by the
// single-world, batched and differentiable engines.
struct SimulationConfig;
FlowParams flow_params_of(const SimulationConfig& cfg);

}  // namespace flp

struct flp_propagator;

namespace flp {

// What the animation recorder (recorder.cu) reads from a single-world handle:
// the current state buffer (C x D x H x W f32, valid in stream order), the
// handle's stream, the grid and dt.
struct PropView {
    const float* state;
    cudaStream_t stream;
    int width, height, depth, channels;
    float dt;
    int device;
};
PropView prop_view(flp_propagator* h);

// direct convolution + growth
size_t conv_direct_smem_bytes(int rmax);
void launch_conv_direct_2d(const float* A, float* U, const KDesc* kd, int K, const float* taps, int W, int H, int C,
                           int rmax, int* reset_slot, cudaStream_t st);
cudaError_t launch_conv_direct_2d_f64(const double* A, double* U, const KDesc64* kd, int K, const double* taps, int W,
                                      int H, int C, int rmax);

// transport: flow (destinations) then gather
size_t flow_smem_bytes(int C);
size_t gather_smem_bytes();
void transport_2d_set_attributes();
void launch_flow_2d(const float* A, const float* U, float* DX, float* DY, int C, int W, int H,
                    const FlowParams& fp, int* dmax_slot, int* status, cudaStream_t st);
// A: the state the flow pass read (the sources' masses); gby: destination rows
// per thread (1 or 2), both give the same bits.
void launch_gather_2d(const float* DX, const float* DY, const float* A, float* Anext, int C, int W, int H,
                      const FlowParams& fp, const int* dmax_slot, int gby, cudaStream_t st);
void launch_zero_ints(int* p, int n, cudaStream_t st);

// FP64 compensated mass
void launch_mass_fp64(const float* A, size_t n, double2* partial, int np, double* out, cudaStream_t st);

// FFT path
size_t fft_rows_smem(int W, int NR, bool with_u);
size_t fft_cols_smem(int H, int NC);
void fft2d_set_attributes(size_t max_bytes);
// Acopy (optional, widths with a warp-synchronous kernel only): the source
// planes read are also written there, at the same offsets (A may then be
// mapped host memory and Acopy its device copy).
void launch_fft_r2c(const float* A, float2* S, const int* srcs, int nsrc, int W, int H, const FftGeom& g,
                    int* reset_slot, int nreset, cudaStream_t st, float* Acopy = nullptr);
bool fft_rows_copy_width(int W);  // whether launch_fft_r2c takes Acopy for this width
void launch_fft_cols(const float2* S, const float2* KH, float2* T, const int* slot_of_kernel, int K, int W, int H,
                     const FftGeom& g, int mode, float scale, cudaStream_t st);
void launch_fft_r2c_legacy(const float* A, float2* S, const int* srcs, int nsrc, int W, int H, const FftGeom& g,
                           int* reset_slot, int nreset, cudaStream_t st);
void launch_fft_c2r_growth_legacy(const float2* T, float* U, const KDesc* kd, int K, int W, int H, int C,
                                  const FftGeom& g, cudaStream_t st);
void launch_fft_lines(const float2* S, const float2* KH, float2* T, const int* slot_of_kernel, int K, int nlines,
                      int H, const FftGeom& g, int mode, float scale, cudaStream_t st);
void launch_fft_c2r_growth(const float2* T, float* U, const KDesc* kd, int K, int W, int H, int C, const FftGeom& g,
                           cudaStream_t st);
// Column convolution T[k] = IFFT_col(FFT_col(S[slot_of_kernel[k]]) * KH[k])
// for K kernels over nslots source spectra, in `groups` equal groups (worlds
// of a batch: group i holds slots [i*nslots/groups, ...) and kernels
// [i*K/groups, ...)); g.share_cols selects one forward transform per slot.
void launch_fft_cols_conv(const float2* S, const float2* KH, float2* T, const int* slot_of_kernel, int nslots, int K,
                          int groups, int W, int H, const FftGeom& g, cudaStream_t st);
// Inverse row pass without growth: slot j -> plane planes[j] (or j), times
// scale, written or accumulated.  Templated row lengths only.
void launch_fft_c2r_raw(const float2* T, float* out, const int* planes, int nslots, int W, int H, float scale,
                        bool accumulate, const FftGeom& g, cudaStream_t st);

// 3D FFT path: z-axis pass (the x and y passes reuse the 2D row and column passes)
bool fft_row_templated(int M);
bool fft_col_templated(int H);
bool fft_z_templated(int D);
void fft3d_set_attributes(size_t max_bytes);
void launch_fft_z(const float2* S, const float2* KH, float2* T, const int* slot_of_kernel, int nlines_k, int W, int H,
                  int D, const float2* twD, int mode, float scale, cudaStream_t st);

// 3D transport
size_t flow3d_smem_bytes(int C, int nz);
int flow3d_max_channels();
size_t gather3d_smem_bytes();
void transport_3d_set_attributes();
void launch_flow_3d(const float* A, const float* U, float* DX, float* DY, float* DZ, int C, int W, int H,
                    int D, const FlowParams& fp, int* dmax_slot, int* status, cudaStream_t st);
// A: the state the flow pass read (the sources' masses)
void launch_gather_3d(const float* DX, const float* DY, const float* DZ, const float* A, float* Anext, int C, int W,
                      int H, int D, const FlowParams& fp, const int* dmax_slot, cudaStream_t st);

}  // namespace flp
