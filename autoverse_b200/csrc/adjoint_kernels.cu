// Kernels of the differentiable step: the forward transport batched over
// worlds of one shape, and the hand-written adjoint of each stage of the
// 2D step (src/compute/propagator.rs:239-420):
//
//   forward                                 adjoint (this file)
//   conv_k = K_k * A_src      (fft.rs)      A_src^ += IFFT(conj(K^) FFT(conv_k^)),
//                                           K_k^ += corr(conv_k^, A_src)   [spectral]
//   U_t = sum w G(conv_k)     (growth.rs)   conv_k^ = U_t^ w G'(conv_k); w^, mu^, sigma^
//   grad S, grad U (Sobel)    (gradient.rs) Sobel transpose
//   alpha = clamp((S/b)^n)    (flow.rs)     alpha^ -> S^, beta^
//   F = (1-a) gU - a gS       (flow.rs)     gU^, gS^, alpha^
//   A' = sum m overlap/(2s)^2 (reintegration.rs) m^ (per source), dest^ from the
//                                           piecewise-linear overlap slopes
//
// Every adjoint kernel is a per-cell gather: no atomics on field values (only
// the per-world parameter sums use FP64 atomics).
#include "adjoint.h"
#include "common.cuh"
#include "kernels.h"
#include "transport_items.cuh"

namespace flp {

// ------------------------------------------------------ forward, batched ----
// Rows per thread of the flow's row walk and destination rows per thread of
// the gather for the differentiable batch (worlds of one shape, whose planes
// together exceed L2): a taller walk reloads fewer halo rows.
#ifndef FLP_ADJ_FR_RPT
#define FLP_ADJ_FR_RPT 8
#endif
#ifndef FLP_ADJ_GBY
#define FLP_ADJ_GBY 2
#endif
constexpr int ADJ_FR_RPT = FLP_ADJ_FR_RPT;
constexpr int ADJ_FR_H = 8 * ADJ_FR_RPT;
constexpr int ADJ_GBY = FLP_ADJ_GBY;

template <int CV>
__global__ void __launch_bounds__(256) k_flow_worlds(const float* __restrict__ A, const float* __restrict__ U,
                                                     float* __restrict__ DX, float* __restrict__ DY, int C, int W,
                                                     int H, const FlowParams* __restrict__ fps, int* dmax,
                                                     int* status) {
    extern __shared__ __align__(16) float sm[];
    const int w = blockIdx.z;
    const size_t off = size_t(w) * C * W * H;
    const FlowParams fp = fps[w];
    if constexpr (CV == 0)
        flow_item(sm, A + off, U + off, DX + off, DY + off, C, W, H, fp, blockIdx.x * FL_W, blockIdx.y * FL_H,
                  dmax + w, status);
    else
        flow_rows_item<CV, ADJ_FR_RPT>(A + off, U + off, DX + off, DY + off, W, H, fp, blockIdx.x * 32,
                                       blockIdx.y * ADJ_FR_H, dmax + w, status);
}

template <bool POW2>
__global__ void __launch_bounds__(256, 3) k_gather_worlds(const float* __restrict__ DX, const float* __restrict__ DY,
                                                          const float* __restrict__ A, float* __restrict__ An, int C,
                                                          int W, int H, const FlowParams* __restrict__ fps,
                                                          const int* __restrict__ dmax) {
    extern __shared__ __align__(16) float sm[];
    const int p = blockIdx.z, w = p / C;
    const size_t off = size_t(p) * W * H;
    const FlowParams fp = fps[w];
    gather_item<POW2, ADJ_GBY>(sm, DX + off, DY + off, A + off, An + off, W, H, fp, dmax[w], blockIdx.x * GT_W,
                               blockIdx.y * gt_h(ADJ_GBY));
}

void launch_flow_worlds(const float* A, const float* U, float* DX, float* DY, int B, int C, int W, int H,
                        const FlowParams* fps, int* dmax, int* status, cudaStream_t st) {
    const int cv = C <= 4 ? C : 0;
    const int th = cv ? ADJ_FR_H : FL_H;
    const dim3 grid((W + FL_W - 1) / FL_W, (H + th - 1) / th, B);
    const size_t smem = cv ? 0 : flow_smem_bytes(C);
    switch (cv) {
        case 1: k_flow_worlds<1><<<grid, 256, smem, st>>>(A, U, DX, DY, C, W, H, fps, dmax, status); break;
        case 2: k_flow_worlds<2><<<grid, 256, smem, st>>>(A, U, DX, DY, C, W, H, fps, dmax, status); break;
        case 3: k_flow_worlds<3><<<grid, 256, smem, st>>>(A, U, DX, DY, C, W, H, fps, dmax, status); break;
        case 4: k_flow_worlds<4><<<grid, 256, smem, st>>>(A, U, DX, DY, C, W, H, fps, dmax, status); break;
        default: k_flow_worlds<0><<<grid, 256, smem, st>>>(A, U, DX, DY, C, W, H, fps, dmax, status); break;
    }
}

void launch_gather_worlds(const float* DX, const float* DY, const float* A, float* An, int B, int C, int W, int H,
                          const FlowParams* fps, bool pow2, const int* dmax, cudaStream_t st) {
    dim3 grid((W + GT_W - 1) / GT_W, (H + gt_h(ADJ_GBY) - 1) / gt_h(ADJ_GBY), B * C);
    const size_t smem = gather_smem_bytes_inl(ADJ_GBY);
    if (pow2)
        k_gather_worlds<true><<<grid, 256, smem, st>>>(DX, DY, A, An, C, W, H, fps, dmax);
    else
        k_gather_worlds<false><<<grid, 256, smem, st>>>(DX, DY, A, An, C, W, H, fps, dmax);
}

// U_t = sum over kernels targeting t (kernel order) of w G(conv_k), with the
// growth epilogue's arithmetic (growth.rs:45-59).
__global__ void __launch_bounds__(256) k_growth_worlds(const float* __restrict__ conv, float* __restrict__ U,
                                                       const AdjKern* __restrict__ ak, int K, int C, int N) {
    const int p = blockIdx.y, w = p / C, c = p - w * C;
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= N) return;
    float u = 0.f;
    for (int k = 0; k < K; ++k) {
        const AdjKern d = ak[w * K + k];
        if (d.tgt != c) continue;
        const float v = conv[size_t(w * K + k) * N + i];
        const float diff = __fsub_rn(v, d.mu);
        const float e = expf(__fmul_rn(__fmul_rn(-diff, diff), d.inv2s2));
        const float g = __fsub_rn(__fmul_rn(2.0f, e), 1.0f);
        u = __fadd_rn(u, __fmul_rn(d.weight, g));
    }
    U[size_t(p) * N + i] = u;
}

void launch_growth_worlds(const float* conv, float* U, const AdjKern* ak, int B, int K, int C, int N,
                          cudaStream_t st) {
    dim3 grid((N + 255) / 256, B * C);
    k_growth_worlds<<<grid, 256, 0, st>>>(conv, U, ak, K, C, N);
}

// ------------------------------------------------------------- adjoints ----
__device__ __forceinline__ double block_sum_d(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < int(blockDim.x >> 5); ++i) t += red[i];
    return t;  // valid in thread 0
}

// Reintegration adjoint, one thread per source cell (reintegration.rs:60-167).
// Forward: A'(X) += m' * ow(X) * oh(Y) with m' = m / (2s)^2, ow = max(min(X+1,
// dx+s) - max(X, dx-s), 0).  Given G = dL/dA':
//   dL/dm  = sum_X G(X) ow oh / (2s)^2
//   dL/ddx = m' sum_X G(X) oh ([dx+s < X+1] - [dx-s > X])   (and y alike)
// and F^ = dt dest^.  Sources below the reference's 1e-10 threshold carry no
// mass and get zero gradients.
template <bool POW2>
__global__ void __launch_bounds__(256) k_adj_reint(const float* __restrict__ DX, const float* __restrict__ DY,
                                                   const float* __restrict__ A, const float* __restrict__ G,
                                                   float* __restrict__ MBAR, float* __restrict__ FXB,
                                                   float* __restrict__ FYB, int C, int W, int H,
                                                   const FlowParams* __restrict__ fps) {
    const int p = blockIdx.z, w = p / C;
    const int X = blockIdx.x * 32 + (threadIdx.x & 31), Y = blockIdx.y * 8 + (threadIdx.x >> 5);
    if (X >= W || Y >= H) return;
    const FlowParams fp = fps[w];
    const size_t N = size_t(W) * H;
    const size_t idx = size_t(p) * N + size_t(Y) * W + X;
    const float m = source_mass<POW2>(A[idx], fp);
    if (m == 0.f) {
        MBAR[idx] = 0.f;
        FXB[idx] = 0.f;
        FYB[idx] = 0.f;
        return;
    }
    const float dx = DX[idx], dy = DY[idx];
    const float* g = G + size_t(p) * N;
    if (fp.point_mode) {
        const int nx = wrap_coord(f2i_sat(roundf(dx)), W), ny = wrap_coord(f2i_sat(roundf(dy)), H);
        MBAR[idx] = g[size_t(ny) * W + nx];
        FXB[idx] = 0.f;
        FYB[idx] = 0.f;
        return;
    }
    const float s = fp.s;
    const float xmin = dx - s, xmax = dx + s, ymin = dy - s, ymax = dy + s;
    const int ix_lo = max(f2i_sat(floorf(xmin)), -W), ix_hi = min(f2i_sat(ceilf(xmax)), 2 * W);
    const int iy_lo = max(f2i_sat(floorf(ymin)), -H), iy_hi = min(f2i_sat(ceilf(ymax)), 2 * H);
    float mb = 0.f, gx = 0.f, gy = 0.f;
    for (int iy = iy_lo; iy <= iy_hi; ++iy) {
        const float fy = float(iy);
        const float oh = fmaxf(fminf(fy + 1.0f, ymax) - fmaxf(fy, ymin), 0.f);
        if (!(oh > 0.f)) continue;
        const float doh = (ymax < fy + 1.0f ? 1.f : 0.f) - (ymin > fy ? 1.f : 0.f);
        const float* row = g + size_t(wrap_near(iy, H)) * W;
        for (int ix = ix_lo; ix <= ix_hi; ++ix) {
            const float fx = float(ix);
            const float ow = fmaxf(fminf(fx + 1.0f, xmax) - fmaxf(fx, xmin), 0.f);
            if (!(ow > 0.f)) continue;
            const float dow = (xmax < fx + 1.0f ? 1.f : 0.f) - (xmin > fx ? 1.f : 0.f);
            const float gb = row[wrap_near(ix, W)];
            mb += ow * oh * gb;
            gx += gb * dow * oh;
            gy += gb * ow * doh;
        }
    }
    const float coef = POW2 ? fp.inv_area : 1.0f / fp.total_area;
    const float mprime = POW2 ? m : m * coef;  // mass / (2s)^2
    MBAR[idx] = mb * coef;
    FXB[idx] = fp.dt * mprime * gx;
    FYB[idx] = fp.dt * mprime * gy;
}

void launch_adj_reint(const float* DX, const float* DY, const float* A, const float* G, float* MBAR, float* FXB,
                      float* FYB, int B, int C, int W, int H, const FlowParams* fps, bool pow2, cudaStream_t st) {
    dim3 grid((W + 31) / 32, (H + 7) / 8, B * C);
    if (pow2) k_adj_reint<true><<<grid, 256, 0, st>>>(DX, DY, A, G, MBAR, FXB, FYB, C, W, H, fps);
    else k_adj_reint<false><<<grid, 256, 0, st>>>(DX, DY, A, G, MBAR, FXB, FYB, C, W, H, fps);
}

// Stage C planes of a field family over a 34x10 region (1-cell torus halo).
__device__ __forceinline__ void stage_halo(float* dst, const float* __restrict__ src, int nplanes, size_t plane_stride,
                                           const int* colx, const int* rowy, int W) {
    for (int i = threadIdx.x; i < nplanes * FL_RC; i += 256) {
        const int k = i / FL_RC, cell = i - k * FL_RC;
        const int ly = cell / FL_RW, lx = cell - ly * FL_RW;
        dst[i] = src[size_t(k) * plane_stride + size_t(rowy[ly]) * W + colx[lx]];
    }
}

__device__ __forceinline__ void sobel_at(const float* a, float& gx, float& gy) {
    sobel2(a[0], a[1], a[2], a[FL_RW], a[FL_RW + 2], a[2 * FL_RW], a[2 * FL_RW + 1], a[2 * FL_RW + 2], gx, gy);
}

// (S/beta)^(n-1) and (S/beta)^n for the alpha derivative (flow.rs:14-32).
__device__ __forceinline__ void alpha_powers(float ratio, float n, float& pn1, float& pn) {
    if (n == 1.0f) { pn1 = 1.0f; pn = ratio; }
    else if (n == 2.0f) { pn1 = ratio; pn = ratio * ratio; }
    else if (n == 3.0f) { pn1 = ratio * ratio; pn = pn1 * ratio; }
    else if (n == 4.0f) { pn1 = ratio * ratio * ratio; pn = pn1 * ratio; }
    else { pn1 = powf(ratio, n - 1.0f); pn = powf(ratio, n); }
}

// Flow adjoint, one thread per cell of one world (flow.rs:68-87 and 14-32):
// from F^_c (FXB, FYB): gU^_c = (1-a) F^_c, gS^ = -a sum_c F^_c,
// a^ = -sum_c F^_c . (gU_c + gS); S^_local = a^ da/dS; beta^ += a^ da/dbeta.
__global__ void __launch_bounds__(256) k_adj_flow(const float* __restrict__ A, const float* __restrict__ U,
                                                  const float* __restrict__ FXB, const float* __restrict__ FYB,
                                                  float* __restrict__ GUX, float* __restrict__ GUY,
                                                  float* __restrict__ GSX, float* __restrict__ GSY,
                                                  float* __restrict__ SBL, double* __restrict__ pgrad, int P, int C,
                                                  int W, int H, const FlowParams* __restrict__ fps) {
    extern __shared__ __align__(16) float sm[];
    __shared__ int colx[FL_RW], rowy[FL_RH];
    __shared__ double red[8];
    const int w = blockIdx.z;
    const int x0 = blockIdx.x * FL_W, y0 = blockIdx.y * FL_H;
    const size_t N = size_t(W) * H;
    const size_t off = size_t(w) * C * N;
    const FlowParams fp = fps[w];
    float* as = sm;                    // C A planes
    float* us = sm + C * FL_RC;        // C U planes
    float* asum = sm + 2 * C * FL_RC;  // channel sum
    const int tid = threadIdx.x;
    if (tid < FL_RW) colx[tid] = wrap_near(x0 - 1 + tid, W);
    else if (tid < FL_RW + FL_RH) rowy[tid - FL_RW] = wrap_near(y0 - 1 + (tid - FL_RW), H);
    __syncthreads();
    stage_halo(as, A + off, C, N, colx, rowy, W);
    stage_halo(us, U + off, C, N, colx, rowy, W);
    __syncthreads();
    for (int i = tid; i < FL_RC; i += 256) {
        float a = 0.f;
        for (int k = 0; k < C; ++k) a = __fadd_rn(a, as[k * FL_RC + i]);
        asum[i] = a;
    }
    __syncthreads();
    const int lx = tid & 31, ly = tid >> 5;
    const int X = x0 + lx, Y = y0 + ly;
    double bsum = 0.0;
    if (X < W && Y < H) {
        const int o = ly * FL_RW + lx;
        float gsx, gsy;
        sobel_at(asum + o, gsx, gsy);
        const float S = asum[o + FL_RW + 1];
        const float alpha = flow_alpha(S, fp.beta_a, fp.nexp);
        const float ratio = S / fp.beta_a;
        float pn1, pn;
        alpha_powers(ratio, fp.nexp, pn1, pn);
        const bool inside = pn > 0.f && pn < 1.f;
        const float dadS = inside ? fp.nexp * pn1 / fp.beta_a : 0.f;
        const float dadb = inside ? -fp.nexp * pn / fp.beta_a : 0.f;
        const size_t cell = size_t(Y) * W + X;
        float fsx = 0.f, fsy = 0.f, abar = 0.f;
        for (int c = 0; c < C; ++c) {
            float gux, guy;
            sobel_at(us + c * FL_RC + o, gux, guy);
            const size_t i = off + size_t(c) * N + cell;
            const float fx = FXB[i], fy = FYB[i];
            GUX[i] = (1.0f - alpha) * fx;
            GUY[i] = (1.0f - alpha) * fy;
            fsx += fx;
            fsy += fy;
            abar -= fx * (gux + gsx) + fy * (guy + gsy);
        }
        const size_t j = size_t(w) * N + cell;
        GSX[j] = -alpha * fsx;
        GSY[j] = -alpha * fsy;
        SBL[j] = abar * dadS;
        bsum = double(abar) * double(dadb);
    }
    const double t = block_sum_d(bsum, red);
    if (tid == 0 && t != 0.0) atomicAdd(pgrad + size_t(w) * P, t);
}

void launch_adj_flow(const float* A, const float* U, const float* FXB, const float* FYB, float* GUX, float* GUY,
                     float* GSX, float* GSY, float* SBL, double* pgrad, int P, int B, int C, int W, int H,
                     const FlowParams* fps, cudaStream_t st) {
    dim3 grid((W + FL_W - 1) / FL_W, (H + FL_H - 1) / FL_H, B);
    k_adj_flow<<<grid, 256, sizeof(float) * (2 * C + 1) * FL_RC, st>>>(A, U, FXB, FYB, GUX, GUY, GSX, GSY, SBL, pgrad,
                                                                         P, C, W, H, fps);
}

// Transpose of the 2D Sobel (gradient.rs:99-102) at the centre of a staged
// 3x3 window: f^(x,y) = 1/8 sum_{i,j} Kx(i,j) gx^(x-i,y-j) + Ky(i,j) gy^(x-i,y-j).
__device__ __forceinline__ float sobel_t_at(const float* gx, const float* gy) {
    // window element (dy+1, dx+1) holds the value at (x+dx, y+dy)
    auto X = [&](int dxo, int dyo) { return gx[(dyo + 1) * FL_RW + dxo + 1]; };
    auto Yv = [&](int dxo, int dyo) { return gy[(dyo + 1) * FL_RW + dxo + 1]; };
    float v = -X(1, 1) + X(-1, 1) - 2.0f * X(1, 0) + 2.0f * X(-1, 0) - X(1, -1) + X(-1, -1);
    v += -Yv(1, 1) - 2.0f * Yv(0, 1) - Yv(-1, 1) + Yv(1, -1) + 2.0f * Yv(0, -1) + Yv(-1, -1);
    return 0.125f * v;
}

// U^_c = SobelT(gU^_c); S^ = S^_local + SobelT(gS^); A^_c = m^_c + S^.
__global__ void __launch_bounds__(256) k_adj_sobel_t(const float* __restrict__ GUX, const float* __restrict__ GUY,
                                                     const float* __restrict__ GSX, const float* __restrict__ GSY,
                                                     const float* __restrict__ SBL, const float* __restrict__ MBAR,
                                                     float* __restrict__ UBAR, float* __restrict__ GOUT, int C, int W,
                                                     int H) {
    extern __shared__ __align__(16) float sm[];
    __shared__ int colx[FL_RW], rowy[FL_RH];
    const int w = blockIdx.z;
    const int x0 = blockIdx.x * FL_W, y0 = blockIdx.y * FL_H;
    const size_t N = size_t(W) * H;
    const size_t off = size_t(w) * C * N;
    float* ux = sm;
    float* uy = ux + C * FL_RC;
    float* sx = uy + C * FL_RC;
    float* sy = sx + FL_RC;
    const int tid = threadIdx.x;
    if (tid < FL_RW) colx[tid] = wrap_near(x0 - 1 + tid, W);
    else if (tid < FL_RW + FL_RH) rowy[tid - FL_RW] = wrap_near(y0 - 1 + (tid - FL_RW), H);
    __syncthreads();
    stage_halo(ux, GUX + off, C, N, colx, rowy, W);
    stage_halo(uy, GUY + off, C, N, colx, rowy, W);
    stage_halo(sx, GSX + size_t(w) * N, 1, N, colx, rowy, W);
    stage_halo(sy, GSY + size_t(w) * N, 1, N, colx, rowy, W);
    __syncthreads();
    const int lx = tid & 31, ly = tid >> 5;
    const int X = x0 + lx, Y = y0 + ly;
    if (X >= W || Y >= H) return;
    const int o = ly * FL_RW + lx;
    const size_t cell = size_t(Y) * W + X;
    const float sb = SBL[size_t(w) * N + cell] + sobel_t_at(sx + o, sy + o);
    for (int c = 0; c < C; ++c) {
        const size_t i = off + size_t(c) * N + cell;
        UBAR[i] = sobel_t_at(ux + c * FL_RC + o, uy + c * FL_RC + o);
        GOUT[i] = MBAR[i] + sb;
    }
}

void launch_adj_sobel_t(const float* GUX, const float* GUY, const float* GSX, const float* GSY, const float* SBL,
                        const float* MBAR, float* UBAR, float* GOUT, int B, int C, int W, int H, cudaStream_t st) {
    dim3 grid((W + FL_W - 1) / FL_W, (H + FL_H - 1) / FL_H, B);
    k_adj_sobel_t<<<grid, 256, sizeof(float) * (2 * C + 2) * FL_RC, st>>>(GUX, GUY, GSX, GSY, SBL, MBAR, UBAR, GOUT,
                                                                            C, W, H);
}

// Growth adjoint (growth.rs:11-15): G(u) = 2e - 1, e = exp(-(u-mu)^2 / (2 s^2)).
// conv^ = U^ w G'(u) = -U^ w 2e (u-mu)/s^2; mu^ += U^ w 2e (u-mu)/s^2;
// sigma^ += U^ w 2e (u-mu)^2/s^3; w^ += U^ G(u).
__global__ void __launch_bounds__(256) k_adj_growth(const float* __restrict__ conv, const float* __restrict__ UBAR,
                                                    float* __restrict__ CB, const AdjKern* __restrict__ ak,
                                                    double* __restrict__ pgrad, int P, int K, int C, int N) {
    __shared__ double red[8];
    const int q = blockIdx.y, w = q / K, k = q - w * K;
    const AdjKern d = ak[q];
    const float is2 = 1.0f / (d.sigma * d.sigma);
    double s_mu = 0.0, s_sig = 0.0, s_w = 0.0;
    const float* u = conv + size_t(q) * N;
    const float* ub = UBAR + size_t(w * C + d.tgt) * N;
    float* cb = CB + size_t(q) * N;
    for (int i = blockIdx.x * 256 + threadIdx.x; i < N; i += gridDim.x * 256) {
        const float diff = u[i] - d.mu;
        const float e2 = 2.0f * expf(-diff * diff * d.inv2s2);
        const float b = ub[i];
        const float t = b * d.weight * e2 * diff * is2;
        cb[i] = -t;
        s_mu += double(t);
        s_sig += double(t) * double(diff) / double(d.sigma);
        s_w += double(b) * double(e2 - 1.0f);
    }
    const double a = block_sum_d(s_w, red);
    if (threadIdx.x == 0) atomicAdd(pgrad + size_t(w) * P + 1 + 3 * k, a);
    const double bm = block_sum_d(s_mu, red);
    if (threadIdx.x == 0) atomicAdd(pgrad + size_t(w) * P + 2 + 3 * k, bm);
    const double bs = block_sum_d(s_sig, red);
    if (threadIdx.x == 0) atomicAdd(pgrad + size_t(w) * P + 3 + 3 * k, bs);
}

void launch_adj_growth(const float* conv, const float* UBAR, float* CB, const AdjKern* ak, double* pgrad, int P,
                       int B, int K, int C, int N, cudaStream_t st) {
    int bx = (N + 255) / 256;
    bx = bx > 32 ? 32 : bx;  // a few CTAs per field: fewer FP64 atomics
    dim3 grid(bx, B * K);
    k_adj_growth<<<grid, 256, 0, st>>>(conv, UBAR, CB, ak, pgrad, P, K, C, N);
}

// Spectral adjoint of the convolutions, per frequency bin of one world:
//   SB_s  = sum_{k: slot(k)=s} conj(K^_k) CB^_k          (source adjoint)
//   KS_k += conj(A^_slot(k)) CB^_k                         (kernel correlation)
__global__ void __launch_bounds__(256) k_adj_spectral(const float2* __restrict__ KH, const float2* __restrict__ CBH,
                                                      const float2* __restrict__ AH, float2* __restrict__ SB,
                                                      float2* __restrict__ KS, const AdjKern* __restrict__ ak, int K,
                                                      int nsrc, int nbins) {
    const int w = blockIdx.y;
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= nbins) return;
    float2 acc[ADJ_MAX_SRC];
#pragma unroll
    for (int s = 0; s < ADJ_MAX_SRC; ++s) acc[s] = make_float2(0.f, 0.f);
    for (int k = 0; k < K; ++k) {
        const AdjKern d = ak[w * K + k];
        const size_t qk = size_t(w * K + k) * nbins + i;
        const float2 cb = CBH[qk];
        const float2 kh = KH[qk];
        const float2 ah = AH[size_t(w * nsrc + d.slot) * nbins + i];
        const float2 a = make_float2(kh.x * cb.x + kh.y * cb.y, kh.x * cb.y - kh.y * cb.x);  // conj(kh) cb
#pragma unroll
        for (int s = 0; s < ADJ_MAX_SRC; ++s)
            if (s == d.slot) { acc[s].x += a.x; acc[s].y += a.y; }
        float2 ks = KS[qk];
        ks.x += ah.x * cb.x + ah.y * cb.y;
        ks.y += ah.x * cb.y - ah.y * cb.x;
        KS[qk] = ks;
    }
#pragma unroll
    for (int s = 0; s < ADJ_MAX_SRC; ++s)
        if (s < nsrc) SB[size_t(w * nsrc + s) * nbins + i] = acc[s];
}

void launch_adj_spectral(const float2* KH, const float2* CBH, const float2* AH, float2* SB, float2* KS,
                         const AdjKern* ak, int B, int K, int nsrc, int nbins, cudaStream_t st) {
    dim3 grid((nbins + 255) / 256, B);
    k_adj_spectral<<<grid, 256, 0, st>>>(KH, CBH, AH, SB, KS, ak, K, nsrc, nbins);
}

void adjoint_set_attributes() {
    auto set = [](const void* f, size_t bytes) {
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    };
    set((const void*)k_flow_worlds<0>, flow_smem_bytes(ADJ_MAX_CHANNELS));
    set((const void*)k_gather_worlds<true>, gather_smem_bytes_inl(ADJ_GBY));
    set((const void*)k_gather_worlds<false>, gather_smem_bytes_inl(ADJ_GBY));
    set((const void*)k_adj_flow, sizeof(float) * (2 * ADJ_MAX_CHANNELS + 1) * FL_RC);
    set((const void*)k_adj_sobel_t, sizeof(float) * (2 * ADJ_MAX_CHANNELS + 2) * FL_RC);
}

}  // namespace flp
