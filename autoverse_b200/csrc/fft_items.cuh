// Compile-time shared-memory FFT building blocks and the per-CTA work items
// of the three FFT passes (row R2C, column convolution, row C2R + growth).
// Shared by the single-world kernels (fft2d.cu) and the batched persistent
// kernels (batch.cu).
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace flp {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// 8-byte asynchronous copy global -> shared (both 8-byte aligned), and the
// commit / wait of the copies issued so far.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all_groups() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// ------------------------------------------------- compile-time FFTs -----
// For the line lengths of the benchmarked worlds every size, radix, stride and
// thread mapping is a compile-time constant.  Lines sit contiguously in shared
// memory with one float2 of padding per 8 (pad(i) = i + i/8) and an odd line
// stride, so the strided reads and writes of the Stockham stages spread over
// the banks.  Radix-8 stages run first (3 passes for 512 points), then 4, 2, 3.
template <int L>
struct CtPlan {
    __host__ __device__ static constexpr int pick(int m) {
        return m % 8 == 0 ? 8 : m % 4 == 0 ? 4 : m % 2 == 0 ? 2 : m % 3 == 0 ? 3 : m % 5 == 0 ? 5 : m;
    }
    __host__ __device__ static constexpr int nst() {
        int m = L, n = 0;
        while (m > 1) { m /= pick(m); ++n; }
        return n;
    }
    __host__ __device__ static constexpr int rad(int s) {
        int m = L;
        for (int i = 0; i < s; ++i) m /= pick(m);
        return pick(m);
    }
    __host__ __device__ static constexpr int ns(int s) {
        int p = 1;
        for (int i = 0; i < s; ++i) p *= rad(i);
        return p;
    }
    static constexpr int LS = L + L / 8 + ((L + L / 8) % 2 == 0 ? 1 : 0);  // odd line stride (float2)
};

__device__ __forceinline__ int pad8(int i) { return i + (i >> 3); }

template <bool INV>
__device__ __forceinline__ float2 tw_get(const float2* tw, int i) {
    float2 w = tw[i];
    return INV ? cconj(w) : w;
}

// Forward (INV=false) or inverse DFT of 4 points in place.
template <bool INV>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
    const float2 b0 = cadd(a0, a2), b1 = csub(a0, a2), b2 = cadd(a1, a3), d = csub(a1, a3);
    const float2 b3 = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);  // (+-i) * d
    a0 = cadd(b0, b2);
    a1 = cadd(b1, b3);
    a2 = csub(b0, b2);
    a3 = csub(b1, b3);
}

// One Stockham stage over NL padded lines of stride LS.
template <int L, int NL, bool INV, int S>
__device__ __forceinline__ void ct_stage(const float2* __restrict__ a, float2* __restrict__ b,
                                         const float2* __restrict__ tw) {
    constexpr int rad = CtPlan<L>::rad(S), ns = CtPlan<L>::ns(S), nb = L / rad, tstep = L / (ns * rad);
    constexpr int LS = CtPlan<L>::LS;
    constexpr int total = nb * NL;
#pragma unroll
    for (int base = 0; base < total; base += 256) {
        const int idx = base + int(threadIdx.x);
        if (total % 256 != 0 && idx >= total) break;
        const int line = idx / nb, j = idx - line * nb;
        const int k = j % ns;
        const float2* src = a + line * LS;
        float2* dst = b + line * LS;
        const int out0 = (j / ns) * ns * rad + k;
        if constexpr (rad == 8) {
            float2 v[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) v[q] = src[pad8(j + q * nb)];
            if (ns > 1) {
                const float2 w1 = tw_get<INV>(tw, k * tstep), w2 = tw_get<INV>(tw, 2 * k * tstep),
                             w4 = tw_get<INV>(tw, 4 * k * tstep);
                const float2 w3 = cmul(w1, w2);
                v[1] = cmul(v[1], w1); v[2] = cmul(v[2], w2); v[3] = cmul(v[3], w3); v[4] = cmul(v[4], w4);
                v[5] = cmul(v[5], cmul(w1, w4)); v[6] = cmul(v[6], cmul(w2, w4)); v[7] = cmul(v[7], cmul(w3, w4));
            }
            // X[2m] = DFT4(v_q + v_{q+4})[m], X[2m+1] = DFT4(W8^q (v_q - v_{q+4}))[m]
            float2 t0 = cadd(v[0], v[4]), t1 = cadd(v[1], v[5]), t2 = cadd(v[2], v[6]), t3 = cadd(v[3], v[7]);
            float2 u0 = csub(v[0], v[4]), u1 = csub(v[1], v[5]), u2 = csub(v[2], v[6]), u3 = csub(v[3], v[7]);
            const float h = 0.707106781186547524f;
            // W8 = (h, -h) forward, (h, h) inverse; W8^2 = -i / +i; W8^3 = (-h, -h) / (-h, h)
            u1 = INV ? make_float2(h * (u1.x - u1.y), h * (u1.x + u1.y)) : make_float2(h * (u1.x + u1.y), h * (u1.y - u1.x));
            u2 = INV ? make_float2(-u2.y, u2.x) : make_float2(u2.y, -u2.x);
            u3 = INV ? make_float2(-h * (u3.x + u3.y), h * (u3.x - u3.y)) : make_float2(h * (u3.y - u3.x), -h * (u3.x + u3.y));
            dft4<INV>(t0, t1, t2, t3);
            dft4<INV>(u0, u1, u2, u3);
            dst[pad8(out0)] = t0;
            dst[pad8(out0 + ns)] = u0;
            dst[pad8(out0 + 2 * ns)] = t1;
            dst[pad8(out0 + 3 * ns)] = u1;
            dst[pad8(out0 + 4 * ns)] = t2;
            dst[pad8(out0 + 5 * ns)] = u2;
            dst[pad8(out0 + 6 * ns)] = t3;
            dst[pad8(out0 + 7 * ns)] = u3;
        } else if constexpr (rad == 4) {
            float2 v0 = src[pad8(j)], v1 = src[pad8(j + nb)], v2 = src[pad8(j + 2 * nb)], v3 = src[pad8(j + 3 * nb)];
            if (ns > 1) {
                v1 = cmul(v1, tw_get<INV>(tw, k * tstep));
                v2 = cmul(v2, tw_get<INV>(tw, 2 * k * tstep));
                v3 = cmul(v3, tw_get<INV>(tw, 3 * k * tstep));
            }
            dft4<INV>(v0, v1, v2, v3);
            dst[pad8(out0)] = v0;
            dst[pad8(out0 + ns)] = v1;
            dst[pad8(out0 + 2 * ns)] = v2;
            dst[pad8(out0 + 3 * ns)] = v3;
        } else if constexpr (rad == 2) {
            float2 v0 = src[pad8(j)], v1 = src[pad8(j + nb)];
            if (ns > 1) v1 = cmul(v1, tw_get<INV>(tw, k * tstep));
            dst[pad8(out0)] = cadd(v0, v1);
            dst[pad8(out0 + ns)] = csub(v0, v1);
        } else if constexpr (rad == 3) {
            float2 v0 = src[pad8(j)], v1 = src[pad8(j + nb)], v2 = src[pad8(j + 2 * nb)];
            if (ns > 1) {
                v1 = cmul(v1, tw_get<INV>(tw, k * tstep));
                v2 = cmul(v2, tw_get<INV>(tw, 2 * k * tstep));
            }
            const float hh = 0.866025403784438647f;
            float2 t1 = cadd(v1, v2);
            float2 t2 = make_float2(v0.x - 0.5f * t1.x, v0.y - 0.5f * t1.y);
            float2 d = make_float2(hh * (v1.x - v2.x), hh * (v1.y - v2.y));
            float2 mid = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
            dst[pad8(out0)] = cadd(v0, t1);
            dst[pad8(out0 + ns)] = cadd(t2, mid);
            dst[pad8(out0 + 2 * ns)] = csub(t2, mid);
        } else {
            float2 v[rad];
#pragma unroll
            for (int q = 0; q < rad; ++q) {
                float2 x = src[pad8(j + q * nb)];
                if (q && k) x = cmul(x, tw_get<INV>(tw, (k * q * tstep) % L));
                v[q] = x;
            }
#pragma unroll
            for (int r = 0; r < rad; ++r) {
                float2 acc = v[0];
#pragma unroll
                for (int q = 1; q < rad; ++q) acc = cadd(acc, cmul(v[q], tw_get<INV>(tw, ((q * r) % rad) * (L / rad))));
                dst[pad8(out0 + r * ns)] = acc;
            }
        }
    }
}

template <int L, int NL, bool INV, int S = 0>
__device__ __forceinline__ float2* ct_fft(float2* a, float2* b, const float2* __restrict__ tw) {
    if constexpr (S == CtPlan<L>::nst()) {
        return a;
    } else {
        ct_stage<L, NL, INV, S>(a, b, tw);
        __syncthreads();
        return ct_fft<L, NL, INV, S + 1>(b, a, tw);
    }
}

// Rows per CTA for a row pass of half-length M (E complex values per CTA: 1024
// for the single-world kernels, which run under one wave and want many CTAs;
// 2048 for the batched ones, which are throughput-bound and keep all threads
// of a CTA busy in the radix-8 stages), columns per CTA for a column pass of
// length H: about 2048 complex values per CTA.
template <int M, int E = 1024>
struct RowCfg {
    static constexpr int NR = (E / M) < 1 ? 1 : (E / M);  // E complex values per CTA
    static constexpr int LS = CtPlan<M>::LS;
    static constexpr size_t buf = size_t(NR) * LS;  // float2 per buffer (LS > M+1)
    static constexpr size_t smem_r2c = sizeof(float2) * (M + M + 1 + 2 * buf);
    // plus the U rows and a prefetch buffer for the next kernel's rows
    static constexpr size_t smem_c2r = smem_r2c + sizeof(float) * NR * 2 * M + sizeof(float2) * buf;
};
template <int H>
struct ColCfg {
    static constexpr int NC = H >= 512 ? 4 : (2048 / H);
    static constexpr int LS = CtPlan<H>::LS;
    static constexpr size_t buf = size_t(NC) * LS;
    static constexpr size_t smem = sizeof(float2) * (H + 2 * buf);
    // with the kernel spectrum prefetched during the forward FFT (batched engine)
    static constexpr size_t smem_prefetch = smem + sizeof(float2) * size_t(NC) * H;
};

// ---- items: one CTA's share of a pass, shared by the plain and batched launches

// NR rows of one real plane -> transposed half spectra S[kx][y0..y0+NR).
template <int M, int E = 1024>
__device__ void r2c_rows_item(float2* sm, const float* __restrict__ x, float2* __restrict__ Sc, int H, int y0,
                              const float2* __restrict__ twM_g, const float2* __restrict__ twW_g) {
    constexpr int NR = RowCfg<M, E>::NR, LS = RowCfg<M, E>::LS, Wc = M + 1, W = 2 * M;
    float2* twM = sm;
    float2* twW = twM + M;
    float2* a = twW + Wc;
    float2* b = a + RowCfg<M, E>::buf;
    const int tid = threadIdx.x;
    for (int i = tid; i < M; i += 256) twM[i] = twM_g[i];
    for (int i = tid; i < Wc; i += 256) twW[i] = twW_g[i];
#pragma unroll 4
    for (int i = tid; i < NR * M; i += 256) {
        const int r = i / M, n = i - r * M;  // n fastest: coalesced row reads
        const int y = y0 + r;
        float2 v = make_float2(0.f, 0.f);
        if (y < H) v = *reinterpret_cast<const float2*>(x + size_t(y) * W + 2 * n);
        a[r * LS + pad8(n)] = v;
    }
    __syncthreads();
    float2* Z = ct_fft<M, NR, false>(a, b, twM);
    float2* X = (Z == a) ? b : a;
#pragma unroll 4
    for (int i = tid; i < NR * Wc; i += 256) {
        const int r = i % NR, k = i / NR;
        const float2 zk = Z[r * LS + pad8(k == M ? 0 : k)];
        const float2 zm = cconj(Z[r * LS + pad8(k == 0 ? 0 : M - k)]);
        const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y + zm.y));
        const float2 d = make_float2(0.5f * (zk.x - zm.x), 0.5f * (zk.y - zm.y));
        const float2 o = make_float2(d.y, -d.x);  // d / i
        X[r * LS + k] = cadd(e, cmul(twW[k], o));
    }
    __syncthreads();
#pragma unroll 4
    for (int i = tid; i < NR * Wc; i += 256) {
        const int r = i % NR, k = i / NR;  // r fastest: NR consecutive y per kx
        const int y = y0 + r;
        if (y < H) Sc[size_t(k) * H + y] = X[r * LS + k];
    }
}

// nl (<= NC) contiguous columns of length H: forward FFT, then either scale
// (mode 1) or multiply by the kernel spectrum and inverse FFT (mode 0); mode 2
// is the inverse FFT alone.
// PREFETCH copies the kernel spectrum in with cp.async while the forward FFT
// runs: a gain when many CTAs share the SMs (batched engine), a loss for a
// single world under one wave, where the copies delay the column loads.
template <int H, bool PREFETCH = false>
__device__ void cols_conv_item(float2* sm, const float2* __restrict__ src, const float2* __restrict__ kh,
                               float2* __restrict__ dst, int nl, int mode, float scale,
                               const float2* __restrict__ twH_g) {
    constexpr int NC = ColCfg<H>::NC, LS = ColCfg<H>::LS;
    float2* twH = sm;
    float2* a = twH + H;
    float2* b = a + ColCfg<H>::buf;
    float2* khs = b + ColCfg<H>::buf;  // PREFETCH, mode 0: the kernel spectrum
    const int tid = threadIdx.x;
    for (int i = tid; i < H; i += 256) twH[i] = twH_g[i];
    if (PREFETCH && mode == 0) {
        for (int i = tid; i < nl * H; i += 256) cp_async8(khs + i, kh + i);
        cp_async_commit();
    }
#pragma unroll 4
    for (int i = tid; i < NC * H; i += 256) {
        const int l = i / H, y = i - l * H;
        a[l * LS + pad8(y)] = l < nl ? src[i] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    if (mode == 2) {
        float2* R2 = ct_fft<H, NC, true>(a, b, twH);
#pragma unroll 4
        for (int i = tid; i < nl * H; i += 256) {
            const int l = i / H, y = i - l * H;
            dst[i] = R2[l * LS + pad8(y)];
        }
        __syncthreads();
        return;
    }
    float2* F = ct_fft<H, NC, false>(a, b, twH);
    float2* G = (F == a) ? b : a;
    if (mode == 1) {
        for (int i = tid; i < nl * H; i += 256) {
            const int l = i / H, y = i - l * H;
            const float2 f = F[l * LS + pad8(y)];
            dst[i] = make_float2(f.x * scale, f.y * scale);
        }
        __syncthreads();
        return;
    }
    if (PREFETCH) cp_async_wait_all_groups();  // each thread multiplies the values it copied
#pragma unroll 4
    for (int i = tid; i < NC * H; i += 256) {
        const int l = i / H, y = i - l * H;
        float2& f = F[l * LS + pad8(y)];
        f = l < nl ? cmul(f, PREFETCH ? khs[i] : kh[i]) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* R = ct_fft<H, NC, true>(F, G, twH);
#pragma unroll 4
    for (int i = tid; i < nl * H; i += 256) {
        const int l = i / H, y = i - l * H;
        dst[i] = R[l * LS + pad8(y)];
    }
    __syncthreads();
}

// Lines along z of a [z][y] block (element (z, y) at z*H + y): NZ adjacent
// y's starting at y0 (ny of them valid), each a line of D points.  mode 0:
// forward FFT, multiply by the kernel spectrum (same layout), inverse FFT;
// mode 1: forward FFT scaled.  Loads and stores move NZ contiguous complex
// values per z.
template <int D>
struct ZCfg {
    static constexpr int NZ = D >= 512 ? 4 : (2048 / D);
    static constexpr int LS = CtPlan<D>::LS;
    static constexpr size_t buf = size_t(NZ) * LS;
    static constexpr size_t smem = sizeof(float2) * (D + 2 * buf);
};

template <int D>
__device__ void zconv_item(float2* sm, const float2* __restrict__ src, const float2* __restrict__ kh,
                           float2* __restrict__ dst, int H, int y0, int ny, int mode, float scale,
                           const float2* __restrict__ twD_g) {
    constexpr int NZ = ZCfg<D>::NZ, LS = ZCfg<D>::LS;
    float2* twD = sm;
    float2* a = twD + D;
    float2* b = a + ZCfg<D>::buf;
    const int tid = threadIdx.x;
    for (int i = tid; i < D; i += 256) twD[i] = twD_g[i];
#pragma unroll 4
    for (int i = tid; i < NZ * D; i += 256) {
        const int z = i / NZ, l = i - z * NZ;
        a[l * LS + pad8(z)] = l < ny ? src[size_t(z) * H + y0 + l] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* F = ct_fft<D, NZ, false>(a, b, twD);
    float2* G = (F == a) ? b : a;
    if (mode == 1) {
        for (int i = tid; i < NZ * D; i += 256) {
            const int z = i / NZ, l = i - z * NZ;
            if (l < ny) {
                const float2 f = F[l * LS + pad8(z)];
                dst[size_t(z) * H + y0 + l] = make_float2(f.x * scale, f.y * scale);
            }
        }
        __syncthreads();
        return;
    }
#pragma unroll 4
    for (int i = tid; i < NZ * D; i += 256) {
        const int z = i / NZ, l = i - z * NZ;
        float2& f = F[l * LS + pad8(z)];
        f = l < ny ? cmul(f, kh[size_t(z) * H + y0 + l]) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* R = ct_fft<D, NZ, true>(F, G, twD);
#pragma unroll 4
    for (int i = tid; i < NZ * D; i += 256) {
        const int z = i / NZ, l = i - z * NZ;
        if (l < ny) dst[size_t(z) * H + y0 + l] = R[l * LS + pad8(z)];
    }
    __syncthreads();
}

// NR rows of one target channel: inverse real FFT of each kernel spectrum
// targeting it (kernel order), growth, weighted sum -> U rows.
template <int M, int E = 1024>
__device__ void c2r_growth_item(float2* sm, const float2* __restrict__ T, const KDesc* __restrict__ kd, int K, int c,
                                float* __restrict__ Uc, int H, int y0, const float2* __restrict__ twM_g,
                                const float2* __restrict__ twW_g) {
    constexpr int NR = RowCfg<M, E>::NR, LS = RowCfg<M, E>::LS, Wc = M + 1, W = 2 * M;
    float2* twM = sm;
    float2* twW = twM + M;
    float2* a = twW + Wc;
    float2* b = a + RowCfg<M, E>::buf;
    float* u = reinterpret_cast<float*>(b + RowCfg<M, E>::buf);
    float2* pre = reinterpret_cast<float2*>(u + NR * W);  // rows of the next kernel, loaded during this one
    const int tid = threadIdx.x;
    for (int i = tid; i < M; i += 256) twM[i] = twM_g[i];
    for (int i = tid; i < Wc; i += 256) twW[i] = twW_g[i];
    for (int i = tid; i < NR * W; i += 256) u[i] = 0.f;
    auto next = [&](int k) {
        for (++k; k < K; ++k)
            if (kd[k].tgt == c) break;
        return k;
    };
    auto prefetch = [&](int k) {
        const float2* t = T + size_t(k) * Wc * H;
#pragma unroll 4
        for (int i = tid; i < NR * Wc; i += 256) {
            const int r = i % NR, kk = i / NR;
            const int y = y0 + r;
            if (y < H) cp_async8(pre + r * LS + kk, t + size_t(kk) * H + y);
            else pre[r * LS + kk] = make_float2(0.f, 0.f);
        }
        cp_async_commit();
    };
    int kn = next(-1);
    if (kn < K) prefetch(kn);
    while (kn < K) {
        const KDesc d = kd[kn];
        cp_async_wait_all_groups();
        __syncthreads();
        // Z[k] = (X[k] + conj X[M-k]) + i (X[k] - conj X[M-k]) e^{+2 pi i k / W}
#pragma unroll 4
        for (int i = tid; i < NR * M; i += 256) {
            const int r = i / M, kk = i - r * M;
            const float2 xk = pre[r * LS + kk];
            const float2 xm = cconj(pre[r * LS + M - kk]);
            const float2 e = cadd(xk, xm);
            const float2 o = cmul(csub(xk, xm), cconj(twW[kk]));
            b[r * LS + pad8(kk)] = make_float2(e.x - o.y, e.y + o.x);
        }
        __syncthreads();
        kn = next(kn);
        if (kn < K) prefetch(kn);  // overlaps the transform below
        const float2* z = ct_fft<M, NR, true>(b, a, twM);
#pragma unroll 4
        for (int i = tid; i < NR * W; i += 256) {
            const int r = i / W, x = i - r * W;
            const float2 v = z[r * LS + pad8(x >> 1)];
            const float conv = (x & 1) ? v.y : v.x;
            const float diff = __fsub_rn(conv, d.mu);
            const float e = expf(__fmul_rn(__fmul_rn(-diff, diff), d.inv2s2));
            const float g = __fsub_rn(__fmul_rn(2.0f, e), 1.0f);
            u[i] = __fadd_rn(u[i], __fmul_rn(d.weight, g));
        }
    }
    __syncthreads();
#pragma unroll 4
    for (int i = tid; i < NR * W; i += 256) {
        const int r = i / W, x = i - r * W;
        const int y = y0 + r;
        if (y < H) Uc[size_t(y) * W + x] = u[i];
    }
    __syncthreads();
}

// NR rows of one spectrum slot: inverse real FFT, times `scale`, written to
// (or, with accumulate, added to) the rows of `out`.  Same arithmetic as the
// growth epilogue's inverse, without the growth.
template <int M, int E = 1024>
__device__ void c2r_raw_item(float2* sm, const float2* __restrict__ t, float* __restrict__ out, int H, int y0,
                             float scale, bool accumulate, const float2* __restrict__ twM_g,
                             const float2* __restrict__ twW_g) {
    constexpr int NR = RowCfg<M, E>::NR, LS = RowCfg<M, E>::LS, Wc = M + 1, W = 2 * M;
    float2* twM = sm;
    float2* twW = twM + M;
    float2* a = twW + Wc;
    float2* b = a + RowCfg<M, E>::buf;
    const int tid = threadIdx.x;
    for (int i = tid; i < M; i += 256) twM[i] = twM_g[i];
    for (int i = tid; i < Wc; i += 256) twW[i] = twW_g[i];
#pragma unroll 4
    for (int i = tid; i < NR * Wc; i += 256) {
        const int r = i % NR, kk = i / NR;
        const int y = y0 + r;
        a[r * LS + kk] = y < H ? t[size_t(kk) * H + y] : make_float2(0.f, 0.f);
    }
    __syncthreads();
#pragma unroll 4
    for (int i = tid; i < NR * M; i += 256) {
        const int r = i / M, kk = i - r * M;
        const float2 xk = a[r * LS + kk];
        const float2 xm = cconj(a[r * LS + M - kk]);
        const float2 e = cadd(xk, xm);
        const float2 o = cmul(csub(xk, xm), cconj(twW[kk]));
        b[r * LS + pad8(kk)] = make_float2(e.x - o.y, e.y + o.x);
    }
    __syncthreads();
    const float2* z = ct_fft<M, NR, true>(b, a, twM);
#pragma unroll 4
    for (int i = tid; i < NR * W; i += 256) {
        const int r = i / W, x = i - r * W;
        const int y = y0 + r;
        if (y >= H) continue;
        const float2 v = z[r * LS + pad8(x >> 1)];
        const float val = __fmul_rn((x & 1) ? v.y : v.x, scale);
        float* o = out + size_t(y) * W + x;
        *o = accumulate ? __fadd_rn(*o, val) : val;
    }
    __syncthreads();
}

#define FLP_ROW_SIZES(X) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256)
#define FLP_COL_SIZES(X) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512)


}  // namespace flp
