// FFT convolution path for 2D worlds (replaces the rustfft-based
// CachedConvolver, src/compute/fft.rs:218-393, and the growth accumulation,
// src/compute/growth.rs:45-59 / propagator.rs:270-279).
//
// Three kernels per step, all with Stockham autosort FFTs in shared memory:
//   fft_rows_r2c        real rows -> half spectra (W/2 complex FFT + split),
//                       written transposed as S[c][kx][y];
//   fft_cols_conv       per kernel k: column FFT of S[src_k], multiply by the
//                       precomputed K^_k (scaled by 1/(W*H)), inverse column
//                       FFT -> T[k][kx][y];
//   fft_rows_c2r_growth per target channel: for each kernel k targeting it
//                       (kernel order) inverse real row FFT of T[k], growth
//                       G(u; mu, sigma), weighted sum -> U[c][y][x].
// The half-spectrum (W/2+1 bins) is the real-to-complex saving over the
// reference, which transforms full complex grids.
#include "common.cuh"
#include "fft_items.cuh"
#include "fft_warp.cuh"
#include "kernels.h"

#include <math.h>

#include <stdexcept>

namespace flp {

// Transforms `nlines` lines of length p.L held in `a`; element (line, i) sits
// at line*ls + i*is.  Uses `b` as the ping-pong buffer and returns the buffer
// holding the result.  tw[t] = exp(-2 pi i t / L).  No scaling.
__device__ float2* smem_fft(float2* a, float2* b, const FftPlan& p, int nlines, int ls, int is, bool lines_fastest,
                            const float2* __restrict__ tw, bool inverse) {
    const int L = p.L;
    const int nt = blockDim.x * blockDim.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    int ns = 1;
    for (int s = 0; s < p.nst; ++s) {
        const int rad = p.rad[s];
        const int nb = L / rad;
        const int tstep = L / (ns * rad);
        const int total = nb * nlines;
        for (int idx = tid; idx < total; idx += nt) {
            int line, j;
            if (lines_fastest) { line = idx % nlines; j = idx / nlines; }
            else { j = idx % nb; line = idx / nb; }
            const int k = j % ns;
            const float2* src = a + line * ls;
            float2* dst = b + line * ls;
            const int out0 = (j / ns) * ns * rad + k;
            if (rad == 4) {
                float2 v0 = src[j * is], v1 = src[(j + nb) * is], v2 = src[(j + 2 * nb) * is], v3 = src[(j + 3 * nb) * is];
                if (k) {
                    float2 w1 = tw[k * tstep], w2 = tw[2 * k * tstep], w3 = tw[3 * k * tstep];
                    if (inverse) { w1 = cconj(w1); w2 = cconj(w2); w3 = cconj(w3); }
                    v1 = cmul(v1, w1); v2 = cmul(v2, w2); v3 = cmul(v3, w3);
                }
                float2 t0 = cadd(v0, v2), t1 = csub(v0, v2), t2 = cadd(v1, v3), t3 = csub(v1, v3);
                float2 t3r = inverse ? make_float2(-t3.y, t3.x) : make_float2(t3.y, -t3.x);
                dst[out0 * is] = cadd(t0, t2);
                dst[(out0 + ns) * is] = cadd(t1, t3r);
                dst[(out0 + 2 * ns) * is] = csub(t0, t2);
                dst[(out0 + 3 * ns) * is] = csub(t1, t3r);
            } else if (rad == 2) {
                float2 v0 = src[j * is], v1 = src[(j + nb) * is];
                if (k) {
                    float2 w1 = tw[k * tstep];
                    if (inverse) w1 = cconj(w1);
                    v1 = cmul(v1, w1);
                }
                dst[out0 * is] = cadd(v0, v1);
                dst[(out0 + ns) * is] = csub(v0, v1);
            } else if (rad == 3) {
                float2 v0 = src[j * is], v1 = src[(j + nb) * is], v2 = src[(j + 2 * nb) * is];
                if (k) {
                    float2 w1 = tw[k * tstep], w2 = tw[2 * k * tstep];
                    if (inverse) { w1 = cconj(w1); w2 = cconj(w2); }
                    v1 = cmul(v1, w1); v2 = cmul(v2, w2);
                }
                const float h = 0.866025403784438647f;  // sqrt(3)/2
                float2 t1 = cadd(v1, v2);
                float2 t2 = make_float2(v0.x - 0.5f * t1.x, v0.y - 0.5f * t1.y);
                float2 d = make_float2(h * (v1.x - v2.x), h * (v1.y - v2.y));
                float2 mid = inverse ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);  // +-i*d
                dst[out0 * is] = cadd(v0, t1);
                dst[(out0 + ns) * is] = cadd(t2, mid);
                dst[(out0 + 2 * ns) * is] = csub(t2, mid);
            } else {
                // generic radix (5 and other small primes): direct DFT
                float2 v[8];
                for (int q = 0; q < rad; ++q) {
                    float2 x = src[(j + q * nb) * is];
                    if (k && q) {
                        float2 w = tw[(k * q * tstep) % L];
                        if (inverse) w = cconj(w);
                        x = cmul(x, w);
                    }
                    v[q] = x;
                }
                const int wstep = L / rad;
                for (int r = 0; r < rad; ++r) {
                    float2 acc = v[0];
                    for (int q = 1; q < rad; ++q) {
                        float2 w = tw[((q * r) % rad) * wstep];
                        if (inverse) w = cconj(w);
                        acc = cadd(acc, cmul(v[q], w));
                    }
                    dst[(out0 + r * ns) * is] = acc;
                }
            }
        }
        __syncthreads();
        float2* t = a;
        a = b;
        b = t;
        ns *= rad;
    }
    return a;
}

__device__ void load_twiddles(float2* dst, const float2* __restrict__ src, int n) {
    const int nt = blockDim.x * blockDim.y;
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    for (int i = tid; i < n; i += nt) dst[i] = src[i];
}

// ------------------------------------------------------ real row -> spec ---
// grid (ceil(H/NR), n_src); block 256.  srcs[blockIdx.y] = channel index.
// smem: twM[M] | twW[M+1] | a[NR*(M+1)] | b[NR*(M+1)]
__global__ void __launch_bounds__(256) fft_rows_r2c(const float* __restrict__ A, float2* __restrict__ S,
                                                    const int* __restrict__ srcs, int W, int H, int NR, FftPlan pm,
                                                    const float2* __restrict__ twM_g, const float2* __restrict__ twW_g,
                                                    int* reset_slot, int nreset) {
    dep_enter();
    extern __shared__ float2 fsm[];
    const int M = W / 2, Wc = M + 1;
    float2* twM = fsm;
    float2* twW = twM + M;
    float2* a = twW + Wc;
    float2* b = a + NR * Wc;
    const int tid = threadIdx.x;
    if (reset_slot && blockIdx.x == 0 && blockIdx.y == 0 && tid == 0)
        for (int i = 0; i < nreset; ++i) reset_slot[i] = 0;
    const int y0 = blockIdx.x * NR;
    const int slot = blockIdx.y;
    const int c = srcs ? srcs[slot] : slot;
    const float* x = A + size_t(c) * W * H;
    load_twiddles(twM, twM_g, M);
    load_twiddles(twW, twW_g, Wc);
    // z[n] = x[2n] + i x[2n+1], interleaved [n][row]
    for (int i = tid; i < NR * M; i += 256) {
        int r = i % NR, n = i / NR;
        int y = y0 + r;
        float2 v = make_float2(0.f, 0.f);
        if (y < H) v = *reinterpret_cast<const float2*>(x + size_t(y) * W + 2 * n);
        a[n * NR + r] = v;
    }
    __syncthreads();
    float2* Z = smem_fft(a, b, pm, NR, 1, NR, true, twM, false);
    float2* X = (Z == a) ? b : a;
    for (int i = tid; i < NR * Wc; i += 256) {
        int r = i % NR, k = i / NR;
        float2 zk = Z[(k % M) * NR + r];
        float2 zm = cconj(Z[((M - k) % M) * NR + r]);
        float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
        float2 d = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y - zm.y));
        float2 o = make_float2(d.y, -d.x);  // d / i
        X[k * NR + r] = cadd(e, cmul(twW[k], o));
    }
    __syncthreads();
    float2* Sc = S + size_t(slot) * Wc * H;
    for (int i = tid; i < NR * Wc; i += 256) {
        int r = i % NR, k = i / NR;
        int y = y0 + r;
        if (y < H) Sc[size_t(k) * H + y] = X[k * NR + r];
    }
}

// ----------------------------------------------- column conv (fwd*K^ inv) ---
// grid (ceil(Wc/NC), K); block 256.  slot_of_kernel[k] = spectrum slot of src.
// mode 0: T[k] = IFFT_col(FFT_col(S[slot]) * KH[k]);  mode 1 (kernel-spectrum
// setup): T[k] = FFT_col(S[k]) * scale.
// smem: twH[H] | a[NC*H] | b[NC*H]
__global__ void __launch_bounds__(256) fft_cols_conv(const float2* __restrict__ S, const float2* __restrict__ KH,
                                                     float2* __restrict__ T, const int* __restrict__ slot_of_kernel,
                                                     int Wc, int H, int NC, FftPlan ph,
                                                     const float2* __restrict__ twH_g, int mode, float scale) {
    dep_enter();
    extern __shared__ float2 fsm[];
    float2* twH = fsm;
    float2* a = twH + H;
    float2* b = a + NC * H;
    const int tid = threadIdx.x;
    const int kx0 = blockIdx.x * NC;
    const int k = blockIdx.y;
    const int nl = min(NC, Wc - kx0);
    const int slot = mode == 0 ? slot_of_kernel[k] : k;
    load_twiddles(twH, twH_g, H);
    const float2* src = S + (size_t(slot) * Wc + kx0) * H;
    for (int i = tid; i < nl * H; i += 256) a[i] = src[i];
    __syncthreads();
    float2* F = smem_fft(a, b, ph, nl, H, 1, false, twH, false);
    float2* G = (F == a) ? b : a;
    float2* dst = T + (size_t(k) * Wc + kx0) * H;
    if (mode == 1) {
        for (int i = tid; i < nl * H; i += 256) dst[i] = make_float2(F[i].x * scale, F[i].y * scale);
        return;
    }
    const float2* kh = KH + (size_t(k) * Wc + kx0) * H;
    for (int i = tid; i < nl * H; i += 256) F[i] = cmul(F[i], kh[i]);
    __syncthreads();
    float2* R = smem_fft(F, G, ph, nl, H, 1, false, twH, true);
    for (int i = tid; i < nl * H; i += 256) dst[i] = R[i];
}

// --------------------------------------------- spec -> real rows + growth ---
// grid (ceil(H/NR), C); block 256.
// smem: twM[M] | twW[M+1] | a[NR*(M+1)] | b[NR*(M+1)] | u[NR*W] (floats)
__global__ void __launch_bounds__(256) fft_rows_c2r_growth(const float2* __restrict__ T, float* __restrict__ U,
                                                           const KDesc* __restrict__ kd, int K, int W, int H, int NR,
                                                           FftPlan pm, const float2* __restrict__ twM_g,
                                                           const float2* __restrict__ twW_g) {
    dep_enter();
    extern __shared__ float2 fsm[];
    const int M = W / 2, Wc = M + 1;
    float2* twM = fsm;
    float2* twW = twM + M;
    float2* a = twW + Wc;
    float2* b = a + NR * Wc;
    float* u = reinterpret_cast<float*>(b + NR * Wc);
    const int tid = threadIdx.x;
    const int y0 = blockIdx.x * NR;
    const int c = blockIdx.y;
    load_twiddles(twM, twM_g, M);
    load_twiddles(twW, twW_g, Wc);
    for (int i = tid; i < NR * W; i += 256) u[i] = 0.f;
    for (int k = 0; k < K; ++k) {
        const KDesc d = kd[k];
        if (d.tgt != c) continue;
        const float2* t = T + size_t(k) * Wc * H;
        __syncthreads();
        for (int i = tid; i < NR * Wc; i += 256) {
            int r = i % NR, kk = i / NR;
            int y = y0 + r;
            a[kk * NR + r] = y < H ? t[size_t(kk) * H + y] : make_float2(0.f, 0.f);
        }
        __syncthreads();
        // Z[k] = (X[k] + conj X[M-k]) + i (X[k] - conj X[M-k]) e^{+2 pi i k / W}
        for (int i = tid; i < NR * M; i += 256) {
            int r = i % NR, kk = i / NR;
            float2 xk = a[kk * NR + r];
            float2 xm = cconj(a[(M - kk) * NR + r]);
            float2 e = cadd(xk, xm);
            float2 o = cmul(csub(xk, xm), cconj(twW[kk]));
            b[kk * NR + r] = make_float2(e.x - o.y, e.y + o.x);
        }
        __syncthreads();
        float2* z = smem_fft(b, a, pm, NR, 1, NR, true, twM, true);
        // growth + weighted accumulation in kernel order (growth.rs:45-59)
        for (int i = tid; i < NR * W; i += 256) {
            int r = i / W, x = i - r * W;
            float2 v = z[(x >> 1) * NR + r];
            float conv = (x & 1) ? v.y : v.x;
            float diff = __fsub_rn(conv, d.mu);
            float e = expf(__fmul_rn(__fmul_rn(-diff, diff), d.inv2s2));
            float g = __fsub_rn(__fmul_rn(2.0f, e), 1.0f);
            u[i] = __fadd_rn(u[i], __fmul_rn(d.weight, g));
        }
    }
    __syncthreads();
    float* uc = U + size_t(c) * W * H;
    for (int i = tid; i < NR * W; i += 256) {
        int r = i / W, x = i - r * W;
        int y = y0 + r;
        if (y < H) uc[size_t(y) * W + x] = u[i];
    }
}

// ---- plain (single-world) kernels over the items
// Complex values per CTA of the single-world row passes (a CTA holds
// E / (W/2) rows).
constexpr int SW_R2C_ELEMS = 1024, SW_C2R_ELEMS = 1024;
template <int M>
__global__ void __launch_bounds__(256) k_r2c_t(const float* __restrict__ A, float2* __restrict__ S,
                                               const int* __restrict__ srcs, int H, const float2* __restrict__ twM,
                                               const float2* __restrict__ twW, int* reset_slot, int nreset) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    if (reset_slot && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
        for (int i = 0; i < nreset; ++i) reset_slot[i] = 0;
    const int slot = blockIdx.y;
    const int c = srcs ? srcs[slot] : slot;
    constexpr int W = 2 * M, Wc = M + 1;
    r2c_rows_item<M, SW_R2C_ELEMS>(fsm, A + size_t(c) * W * H, S + size_t(slot) * Wc * H, H,
                                   blockIdx.x * RowCfg<M, SW_R2C_ELEMS>::NR, twM, twW);
}

template <int H>
__global__ void __launch_bounds__(256) k_cols_t(const float2* __restrict__ S, const float2* __restrict__ KH,
                                                float2* __restrict__ T, const int* __restrict__ slot_of_kernel, int Wc,
                                                int mode, float scale, const float2* __restrict__ twH) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    constexpr int NC = ColCfg<H>::NC;
    const int kx0 = blockIdx.x * NC, k = blockIdx.y;
    const int nl = min(NC, Wc - kx0);
    const int slot = mode == 0 ? slot_of_kernel[k] : k;
    cols_conv_item<H>(fsm, S + (size_t(slot) * Wc + kx0) * H, mode == 0 ? KH + (size_t(k) * Wc + kx0) * H : nullptr,
                      T + (size_t(k) * Wc + kx0) * H, nl, mode, scale, twH);
}

template <int M>
__global__ void __launch_bounds__(256) k_c2r_t(const float2* __restrict__ T, float* __restrict__ U,
                                               const KDesc* __restrict__ kd, int K, int H,
                                               const float2* __restrict__ twM, const float2* __restrict__ twW) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    const int c = blockIdx.y;
    constexpr int W = 2 * M;
    c2r_growth_item<M, SW_C2R_ELEMS>(fsm, T, kd, K, c, U + size_t(c) * W * H, H, blockIdx.x * RowCfg<M, SW_C2R_ELEMS>::NR,
                                     twM, twW);
}

template <int M>
__global__ void __launch_bounds__(256) k_c2r_raw_t(const float2* __restrict__ T, float* __restrict__ out,
                                                   const int* __restrict__ planes, int H, float scale, int accumulate,
                                                   const float2* __restrict__ twM, const float2* __restrict__ twW) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    const int slot = blockIdx.y;
    const int plane = planes ? planes[slot] : slot;
    constexpr int W = 2 * M, Wc = M + 1;
    c2r_raw_item<M>(fsm, T + size_t(slot) * Wc * H, out + size_t(plane) * W * H, H, blockIdx.x * RowCfg<M>::NR,
                    scale, accumulate != 0, twM, twW);
}

// ---- warp-synchronous single-world kernels (fft_warp.cuh)
// COPY: the planes read (A may be mapped host memory) are also written to Acopy.
template <int M, int WPC, bool COPY = false>
__global__ void __launch_bounds__(32 * WPC, 16 / WPC) k_r2c_w(const float* __restrict__ A, float2* __restrict__ S,
                                                               const int* __restrict__ srcs, int H,
                                                               const float2* __restrict__ twM,
                                                               const float2* __restrict__ twW, int* reset_slot,
                                                               int nreset, float* __restrict__ Acopy) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    if (reset_slot && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
        for (int i = 0; i < nreset; ++i) reset_slot[i] = 0;
    const int slot = blockIdx.y;
    const int c = srcs ? srcs[slot] : slot;
    constexpr int W = 2 * M, Wc = M + 1;
    const size_t off = size_t(c) * W * H;
    r2c_rows_witem<M, WPC, COPY>(fsm, A + off, S + size_t(slot) * Wc * H, H, blockIdx.x * WRowCfg<M, WPC>::NRC, twM,
                                 twW, COPY ? Acopy + off : nullptr);
}

// blockIdx.y: a source slot (share) or a kernel (one transform per kernel).
template <int H, int WPC>
__global__ void __launch_bounds__(32 * WPC, 16 / WPC) k_cols_w(const float2* __restrict__ S,
                                                                const float2* __restrict__ KH, float2* __restrict__ T,
                                                                const int* __restrict__ slot_of_kernel, int Wc,
                                                                int slots_per_group, int kernels_per_group, int share,
                                                                const float2* __restrict__ twH) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    int slot, kb, ke;
    if (share) {
        slot = blockIdx.y;
        kb = (slot / slots_per_group) * kernels_per_group;
        ke = kb + kernels_per_group;
    } else {
        kb = blockIdx.y;
        ke = kb + 1;
        slot = slot_of_kernel[kb];
    }
    cols_witem<H, WPC>(fsm, S + size_t(slot) * Wc * H, KH, T, slot_of_kernel, kb, ke, slot, Wc,
                       blockIdx.x * WColCfg<H, WPC>::NCC, twH);
}

// blockIdx.y: slot (nlines lines of H each); INV: inverse, else forward times scale.
template <int H, int WPC, bool INV>
__global__ void __launch_bounds__(32 * WPC, 16 / WPC) k_lines_w(const float2* __restrict__ src, float2* __restrict__ dst,
                                                                int nlines, float scale,
                                                                const float2* __restrict__ twH) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    const size_t off = size_t(blockIdx.y) * nlines * H;
    cols_plain_witem<H, WPC, INV>(fsm, src + off, dst + off, nlines, blockIdx.x * WColCfg<H, WPC>::NCC, scale, twH);
}

template <int M, int WPC>
__global__ void __launch_bounds__(32 * WPC, 24 / WPC) k_c2r_w(const float2* __restrict__ T, float* __restrict__ U,
                                                               const KDesc* __restrict__ kd, int K, int H,
                                                               const float2* __restrict__ twM,
                                                               const float2* __restrict__ twW) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    const int c = blockIdx.y;
    constexpr int W = 2 * M;
    c2r_growth_witem<M, WPC>(fsm, T, kd, K, c, U + size_t(c) * W * H, H, blockIdx.x * WRowCfg<M, WPC>::NRC, twM,
                             twW);
}

template <int M, int WPC>
__global__ void __launch_bounds__(32 * WPC, 16 / WPC) k_c2r_raw_w(const float2* __restrict__ T, float* __restrict__ out,
                                                                   const int* __restrict__ planes, int H, float scale,
                                                                   int accumulate, const float2* __restrict__ twM,
                                                                   const float2* __restrict__ twW) {
    dep_enter();
    extern __shared__ __align__(16) float2 fsm[];
    const int slot = blockIdx.y;
    const int plane = planes ? planes[slot] : slot;
    constexpr int W = 2 * M, Wc = M + 1;
    c2r_raw_witem<M, WPC>(fsm, T + size_t(slot) * Wc * H, out + size_t(plane) * W * H, H,
                          blockIdx.x * WRowCfg<M, WPC>::NRC, scale, accumulate != 0, twM, twW);
}

bool fft_row_templated(int M) {
#define X(n) if (M == n) return true;
    FLP_ROW_SIZES(X)
#undef X
    return false;
}
bool fft_col_templated(int H) {
#define X(n) if (H == n) return true;
    FLP_COL_SIZES(X)
#undef X
    return false;
}

// ------------------------------------------------------------- launchers ---
size_t fft_rows_smem(int W, int NR, bool with_u) {
    int M = W / 2, Wc = M + 1;
    size_t bytes = sizeof(float2) * (size_t(M) + Wc + 2 * size_t(NR) * Wc);
    if (with_u) bytes += sizeof(float) * size_t(NR) * W;
    return bytes;
}
size_t fft_cols_smem(int H, int NC) { return sizeof(float2) * (size_t(H) + 2 * size_t(NC) * H); }

void fft2d_set_attributes(size_t max_bytes) {
    auto set = [&](const void* f) {
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, int(max_bytes));
        cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    };
    set((const void*)fft_rows_r2c);
    set((const void*)fft_cols_conv);
    set((const void*)fft_rows_c2r_growth);
#define X(n) set((const void*)k_r2c_t<n>); set((const void*)k_c2r_t<n>); set((const void*)k_c2r_raw_t<n>);     \
    set((const void*)k_r2c_w<n, 4>); set((const void*)k_r2c_w<n, 8>); set((const void*)k_c2r_w<n, 4>);            \
    set((const void*)k_r2c_w<n, 4, true>); set((const void*)k_r2c_w<n, 8, true>);                                  \
    set((const void*)k_c2r_w<n, 8>); set((const void*)k_c2r_raw_w<n, 8>); set((const void*)k_c2r_raw_w<n, 4>);
    FLP_ROW_SIZES(X)
#undef X
#define X(n) set((const void*)k_cols_t<n>); set((const void*)k_cols_w<n, 4>); set((const void*)k_cols_w<n, 8>);     \
    set((const void*)k_lines_w<n, 4, false>); set((const void*)k_lines_w<n, 4, true>);
    FLP_COL_SIZES(X)
#undef X
}

bool fft_rows_copy_width(int W) {
    const int M = W / 2;
#define X(n) if (W % 2 == 0 && M == n) return true;
    FLP_ROW_SIZES(X)
#undef X
    return false;
}

void launch_fft_r2c(const float* A, float2* S, const int* srcs, int nsrc, int W, int H, const FftGeom& g,
                    int* reset_slot, int nreset, cudaStream_t st, float* Acopy) {
    const int M = W / 2;
#define X(n)                                                                                                 \
    if (M == n) {                                                                                            \
        if (g.wpc_r2c == 4) {                                                                                \
            dim3 grid((H + WRowCfg<n, 4>::NRC - 1) / WRowCfg<n, 4>::NRC, nsrc);                              \
            if (Acopy)                                                                                       \
                launch_dep(k_r2c_w<n, 4, true>, grid, 128, WRowCfg<n, 4>::smem_r2c, st, A, S, srcs, H, g.twM,  \
                           g.twW, reset_slot, nreset, Acopy);                                                \
            else                                                                                             \
                launch_dep(k_r2c_w<n, 4>, grid, 128, WRowCfg<n, 4>::smem_r2c, st, A, S, srcs, H, g.twM, g.twW, \
                           reset_slot, nreset, Acopy);                                                       \
        } else {                                                                                             \
            dim3 grid((H + WRowCfg<n, 8>::NRC - 1) / WRowCfg<n, 8>::NRC, nsrc);                              \
            if (Acopy)                                                                                       \
                launch_dep(k_r2c_w<n, 8, true>, grid, 256, WRowCfg<n, 8>::smem_r2c, st, A, S, srcs, H, g.twM,  \
                           g.twW, reset_slot, nreset, Acopy);                                                \
            else                                                                                             \
                launch_dep(k_r2c_w<n, 8>, grid, 256, WRowCfg<n, 8>::smem_r2c, st, A, S, srcs, H, g.twM, g.twW, \
                           reset_slot, nreset, Acopy);                                                       \
        }                                                                                                    \
        return;                                                                                              \
    }
    FLP_ROW_SIZES(X)
#undef X
    if (Acopy) throw std::runtime_error("row transform with a plane copy: no warp-synchronous kernel for this width");
    launch_fft_r2c_legacy(A, S, srcs, nsrc, W, H, g, reset_slot, nreset, st);
}

void launch_fft_r2c_legacy(const float* A, float2* S, const int* srcs, int nsrc, int W, int H, const FftGeom& g,
                           int* reset_slot, int nreset, cudaStream_t st) {
    const int M = W / 2;
#define X(n)                                                                                        \
    if (M == n) {                                                                                   \
        dim3 grid((H + RowCfg<n, SW_R2C_ELEMS>::NR - 1) / RowCfg<n, SW_R2C_ELEMS>::NR, nsrc);       \
        launch_dep(k_r2c_t<n>, grid, 256, RowCfg<n, SW_R2C_ELEMS>::smem_r2c, st, A, S, srcs, H, g.twM, g.twW, reset_slot, \
                                                            nreset);                                \
        return;                                                                                     \
    }
    FLP_ROW_SIZES(X)
#undef X
    dim3 grid((H + g.NR - 1) / g.NR, nsrc);
    launch_dep(fft_rows_r2c, grid, 256, fft_rows_smem(W, g.NR, false), st, A, S, srcs, W, H, g.NR, g.pm, g.twM, g.twW,
                                                                    reset_slot, nreset);
}

void launch_fft_lines(const float2* S, const float2* KH, float2* T, const int* slot_of_kernel, int K, int nlines,
                      int H, const FftGeom& g, int mode, float scale, cudaStream_t st) {
    if (mode != 0) {
        // plain forward (mode 1, scaled) or inverse (mode 2) transforms of K slots
#define X(n)                                                                                                    \
        if (H == n) {                                                                                           \
            dim3 grid((nlines + WColCfg<n, 4>::NCC - 1) / WColCfg<n, 4>::NCC, K);                              \
            if (mode == 1)                                                                                      \
                launch_dep(k_lines_w<n, 4, false>, grid, 128, WColCfg<n, 4>::smem, st, S, T, nlines, scale, g.twH); \
            else                                                                                                \
                launch_dep(k_lines_w<n, 4, true>, grid, 128, WColCfg<n, 4>::smem, st, S, T, nlines, scale, g.twH);  \
            return;                                                                                             \
        }
        FLP_COL_SIZES(X)
#undef X
    }
#define X(n)                                                                                                   \
    if (H == n) {                                                                                              \
        dim3 grid((nlines + ColCfg<n>::NC - 1) / ColCfg<n>::NC, K);                                            \
        launch_dep(k_cols_t<n>, grid, 256, ColCfg<n>::smem, st, S, KH, T, slot_of_kernel, nlines, mode, scale, g.twH); \
        return;                                                                                                \
    }
    FLP_COL_SIZES(X)
#undef X
    dim3 grid((nlines + g.NC - 1) / g.NC, K);
    launch_dep(fft_cols_conv, grid, 256, fft_cols_smem(H, g.NC), st, S, KH, T, slot_of_kernel, nlines, H, g.NC, g.ph, g.twH,
                                                              mode, scale);
}

void launch_fft_cols(const float2* S, const float2* KH, float2* T, const int* slot_of_kernel, int K, int W, int H,
                     const FftGeom& g, int mode, float scale, cudaStream_t st) {
    launch_fft_lines(S, KH, T, slot_of_kernel, K, W / 2 + 1, H, g, mode, scale, st);
}

void launch_fft_cols_conv(const float2* S, const float2* KH, float2* T, const int* slot_of_kernel, int nslots, int K,
                          int groups, int W, int H, const FftGeom& g, cudaStream_t st) {
    const int Wc = W / 2 + 1;
    const int share = g.share_cols ? 1 : 0;
    const int spg = nslots / groups, kpg = K / groups;
#define X(n)                                                                                                   \
    if (H == n) {                                                                                              \
        if (g.wpc_cols == 4) {                                                                                 \
            dim3 grid((Wc + WColCfg<n, 4>::NCC - 1) / WColCfg<n, 4>::NCC, share ? nslots : K);                 \
            launch_dep(k_cols_w<n, 4>, grid, 128, WColCfg<n, 4>::smem, st, S, KH, T, slot_of_kernel, Wc, spg,   \
                       kpg, share, g.twH);                                                                     \
        } else {                                                                                               \
            dim3 grid((Wc + WColCfg<n, 8>::NCC - 1) / WColCfg<n, 8>::NCC, share ? nslots : K);                 \
            launch_dep(k_cols_w<n, 8>, grid, 256, WColCfg<n, 8>::smem, st, S, KH, T, slot_of_kernel, Wc, spg,   \
                       kpg, share, g.twH);                                                                     \
        }                                                                                                      \
        return;                                                                                                \
    }
    FLP_COL_SIZES(X)
#undef X
    launch_fft_lines(S, KH, T, slot_of_kernel, K, Wc, H, g, 0, 1.f, st);
}

void launch_fft_c2r_growth(const float2* T, float* U, const KDesc* kd, int K, int W, int H, int C, const FftGeom& g,
                           cudaStream_t st) {
    const int M = W / 2;
#define X(n)                                                                                                  \
    if (M == n) {                                                                                             \
        if (g.wpc_c2r == 4) {                                                                                 \
            dim3 grid((H + WRowCfg<n, 4>::NRC - 1) / WRowCfg<n, 4>::NRC, C);                                  \
            launch_dep(k_c2r_w<n, 4>, grid, 128, WRowCfg<n, 4>::smem_c2r, st, T, U, kd, K, H, g.twM, g.twW);    \
        } else {                                                                                              \
            dim3 grid((H + WRowCfg<n, 8>::NRC - 1) / WRowCfg<n, 8>::NRC, C);                                  \
            launch_dep(k_c2r_w<n, 8>, grid, 256, WRowCfg<n, 8>::smem_c2r, st, T, U, kd, K, H, g.twM, g.twW);    \
        }                                                                                                     \
        return;                                                                                               \
    }
    FLP_ROW_SIZES(X)
#undef X
    launch_fft_c2r_growth_legacy(T, U, kd, K, W, H, C, g, st);
}

void launch_fft_c2r_growth_legacy(const float2* T, float* U, const KDesc* kd, int K, int W, int H, int C,
                                  const FftGeom& g, cudaStream_t st) {
    const int M = W / 2;
#define X(n)                                                                                     \
    if (M == n) {                                                                                \
        dim3 grid((H + RowCfg<n, SW_C2R_ELEMS>::NR - 1) / RowCfg<n, SW_C2R_ELEMS>::NR, C);       \
        launch_dep(k_c2r_t<n>, grid, 256, RowCfg<n, SW_C2R_ELEMS>::smem_c2r, st, T, U, kd, K, H, g.twM, g.twW);       \
        return;                                                                                  \
    }
    FLP_ROW_SIZES(X)
#undef X
    dim3 grid((H + g.NR - 1) / g.NR, C);
    launch_dep(fft_rows_c2r_growth, grid, 256, fft_rows_smem(W, g.NR, true), st, T, U, kd, K, W, H, g.NR, g.pm, g.twM,
                                                                          g.twW);
}

void launch_fft_c2r_raw(const float2* T, float* out, const int* planes, int nslots, int W, int H, float scale,
                        bool accumulate, const FftGeom& g, cudaStream_t st) {
    const int M = W / 2;
#define X(n)                                                                                                  \
    if (M == n) {                                                                                             \
        if (g.wpc_c2r == 4) {                                                                                 \
            dim3 grid((H + WRowCfg<n, 4>::NRC - 1) / WRowCfg<n, 4>::NRC, nslots);                             \
            launch_dep(k_c2r_raw_w<n, 4>, grid, 128, WRowCfg<n, 4>::smem_r2c, st, T, out, planes, H, scale,     \
                       accumulate ? 1 : 0, g.twM, g.twW);                                                     \
        } else {                                                                                              \
            dim3 grid((H + WRowCfg<n, 8>::NRC - 1) / WRowCfg<n, 8>::NRC, nslots);                             \
            launch_dep(k_c2r_raw_w<n, 8>, grid, 256, WRowCfg<n, 8>::smem_r2c, st, T, out, planes, H, scale,     \
                       accumulate ? 1 : 0, g.twM, g.twW);                                                     \
        }                                                                                                     \
        return;                                                                                               \
    }
    FLP_ROW_SIZES(X)
#undef X
    throw std::runtime_error("inverse row pass without growth needs W/2 in {16..256}");
}

}  // namespace flp
