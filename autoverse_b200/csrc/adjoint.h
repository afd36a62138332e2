// Launch interface of the differentiable step (adjoint.cu, adjoint_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace flp {

constexpr int ADJ_MAX_CHANNELS = 8;  // channels per world in a differentiable batch
constexpr int ADJ_MAX_SRC = 8;       // distinct source channels per world

// One kernel of one world, as the adjoint kernels need it.
struct AdjKern {
    float weight, mu, sigma, inv2s2;
    int src, tgt, slot;  // slot: index of src among the world's distinct sources
    int pad;
};

void launch_flow_worlds(const float* A, const float* U, float* DX, float* DY, int B, int C, int W, int H,
                        const FlowParams* fps, int* dmax, int* status, cudaStream_t st);
// A: the state the flow pass read (the sources' masses)
void launch_gather_worlds(const float* DX, const float* DY, const float* A, float* An, int B, int C, int W, int H,
                          const FlowParams* fps, bool pow2, const int* dmax, cudaStream_t st);
void launch_growth_worlds(const float* conv, float* U, const AdjKern* ak, int B, int K, int C, int N,
                          cudaStream_t st);
void launch_adj_reint(const float* DX, const float* DY, const float* A, const float* G, float* MBAR, float* FXB,
                      float* FYB, int B, int C, int W, int H, const FlowParams* fps, bool pow2, cudaStream_t st);
void launch_adj_flow(const float* A, const float* U, const float* FXB, const float* FYB, float* GUX, float* GUY,
                     float* GSX, float* GSY, float* SBL, double* pgrad, int P, int B, int C, int W, int H,
                     const FlowParams* fps, cudaStream_t st);
void launch_adj_sobel_t(const float* GUX, const float* GUY, const float* GSX, const float* GSY, const float* SBL,
                        const float* MBAR, float* UBAR, float* GOUT, int B, int C, int W, int H, cudaStream_t st);
void launch_adj_growth(const float* conv, const float* UBAR, float* CB, const AdjKern* ak, double* pgrad, int P,
                       int B, int K, int C, int N, cudaStream_t st);
void launch_adj_spectral(const float2* KH, const float2* CBH, const float2* AH, float2* SB, float2* KS,
                         const AdjKern* ak, int B, int K, int nsrc, int nbins, cudaStream_t st);
void adjoint_set_attributes();

}  // namespace flp
