// Warp-synchronous line FFTs and the work items of the three FFT passes of a
// step (row R2C, column convolution, row C2R + growth) built on them.
//
// A warp owns whole lines: NLW lines of L points, transformed in its own two
// shared-memory buffers with __syncwarp between the stages and no block-wide
// barrier, so the warps of an SM progress independently and hide each
// other's latencies.  The first stage of a transform reads its inputs through
// a functor (global memory, a spectrum product, the unpacking of a half
// spectrum) and the last stage hands its outputs to a functor (registers,
// global memory, the growth epilogue): of the stages of a transform only the
// ones in between touch shared memory.
//
// Plans are symmetric (the same radix R0 first and last) so that the register
// layout in which the last stage of a forward transform leaves its outputs is
// the layout in which the first stage of an inverse transform wants its
// inputs: the column pass keeps each source column's forward transform in
// registers and runs the inverse transform of every kernel that reads that
// source from them, one forward transform per source instead of per kernel.
//
// The algorithms are the textbook Stockham autosort FFT (mixed radix 8, 4, 2,
// 3; twiddles from the tables of the old items) and the packing of a real row
// of 2M points into an M-point complex transform.
#pragma once

#include "common.cuh"
#include "fft_items.cuh"
#include "kernels.h"

namespace flp {

// Complex arithmetic with every rounding spelled out (no contraction left to
// the compiler), so that the same transform compiled into different kernels
// -- the single-world passes and the batched persistent kernels -- gives the
// same bits.
__device__ __forceinline__ float2 xmul(float2 a, float2 b) {
    return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)), __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}
__device__ __forceinline__ float2 xadd(float2 a, float2 b) { return make_float2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y)); }
__device__ __forceinline__ float2 xsub(float2 a, float2 b) { return make_float2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y)); }
__device__ __forceinline__ float2 xscale(float s, float2 a) { return make_float2(__fmul_rn(s, a.x), __fmul_rn(s, a.y)); }

// Forward (INV=false) or inverse DFT of 4 points in place.
template <bool INV>
__device__ __forceinline__ void xdft4(float2& a0, float2& a1, float2& a2, float2& a3) {
    const float2 b0 = xadd(a0, a2), b1 = xsub(a0, a2), b2 = xadd(a1, a3), d = xsub(a1, a3);
    const float2 b3 = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);  // (+-i) * d, exact
    a0 = xadd(b0, b2);
    a1 = xadd(b1, b3);
    a2 = xsub(b0, b2);
    a3 = xsub(b1, b3);
}

template <int L>
struct WPlan {
    // first and last radix: 8 when 64 | L, 4 when 16 | L, else 2 (L = 2^a 3^b, a >= 2)
    static constexpr int R0 = (L % 64 == 0) ? 8 : (L % 16 == 0) ? 4 : 2;
    __host__ __device__ static constexpr int pickm(int m) {
        return m % 8 == 0 ? 8 : m % 4 == 0 ? 4 : m % 2 == 0 ? 2 : m % 3 == 0 ? 3 : m;
    }
    __host__ __device__ static constexpr int nst() {
        int m = L / (R0 * R0), n = 2;
        while (m > 1) {
            m /= pickm(m);
            ++n;
        }
        return n;
    }
    __host__ __device__ static constexpr int rad(int s) {
        if (s == 0 || s == nst() - 1) return R0;
        int m = L / (R0 * R0);
        for (int i = 1; i < s; ++i) m /= pickm(m);
        return pickm(m);
    }
    __host__ __device__ static constexpr int ns(int s) {
        int p = 1;
        for (int i = 0; i < s; ++i) p *= rad(i);
        return p;
    }
    __host__ __device__ static constexpr bool fits(int n) {
        for (int s = 0; s < nst(); ++s)
            if ((n * (L / rad(s))) % 32 != 0) return false;
        return true;
    }
    // Lines per warp: the fewest that give every stage a multiple of 32
    // butterflies, unless that holds more than 512 points; then the fewest
    // that give the first stage at least 32 (some lanes idle in some stages).
    __host__ __device__ static constexpr int nlw() {
        int n = 1;
        while (!fits(n)) ++n;
        if (n * L <= 512) return n;
        n = 1;
        while (n * (L / R0) < 32) ++n;
        return n;
    }
    static constexpr int NLW = nlw();
    static constexpr int LS = CtPlan<L>::LS;                   // padded line stride (float2)
    static constexpr int WBUF = NLW * LS;                      // one warp buffer (float2)
    static constexpr int NB0 = (NLW * (L / R0) + 31) / 32;     // radix-R0 butterflies per lane, first and last stage
    static constexpr int NREG = NB0 * R0;                      // values per lane between two transforms
};

// Radix-RAD butterfly in place: inputs v[q] (element j + q*nb of the stage),
// twiddled by w^(k*q*tstep) unless ns == 1, outputs v[r] (element out0 + r*ns).
template <int RAD, bool INV>
__device__ __forceinline__ void wbutterfly(float2 (&v)[RAD], int k, int tstep, int ns,
                                           const float2* __restrict__ tw) {
    if constexpr (RAD == 8) {
        if (ns > 1) {
            const float2 w1 = tw_get<INV>(tw, k * tstep), w2 = tw_get<INV>(tw, 2 * k * tstep),
                         w4 = tw_get<INV>(tw, 4 * k * tstep);
            const float2 w3 = xmul(w1, w2);
            v[1] = xmul(v[1], w1); v[2] = xmul(v[2], w2); v[3] = xmul(v[3], w3); v[4] = xmul(v[4], w4);
            v[5] = xmul(v[5], xmul(w1, w4)); v[6] = xmul(v[6], xmul(w2, w4)); v[7] = xmul(v[7], xmul(w3, w4));
        }
        float2 t0 = xadd(v[0], v[4]), t1 = xadd(v[1], v[5]), t2 = xadd(v[2], v[6]), t3 = xadd(v[3], v[7]);
        float2 u0 = xsub(v[0], v[4]), u1 = xsub(v[1], v[5]), u2 = xsub(v[2], v[6]), u3 = xsub(v[3], v[7]);
        const float h = 0.707106781186547524f;
        u1 = INV ? make_float2(__fmul_rn(h, __fsub_rn(u1.x, u1.y)), __fmul_rn(h, __fadd_rn(u1.x, u1.y)))
                 : make_float2(__fmul_rn(h, __fadd_rn(u1.x, u1.y)), __fmul_rn(h, __fsub_rn(u1.y, u1.x)));
        u2 = INV ? make_float2(-u2.y, u2.x) : make_float2(u2.y, -u2.x);
        u3 = INV ? make_float2(__fmul_rn(-h, __fadd_rn(u3.x, u3.y)), __fmul_rn(h, __fsub_rn(u3.x, u3.y)))
                 : make_float2(__fmul_rn(h, __fsub_rn(u3.y, u3.x)), __fmul_rn(-h, __fadd_rn(u3.x, u3.y)));
        xdft4<INV>(t0, t1, t2, t3);
        xdft4<INV>(u0, u1, u2, u3);
        v[0] = t0; v[1] = u0; v[2] = t1; v[3] = u1; v[4] = t2; v[5] = u2; v[6] = t3; v[7] = u3;
    } else if constexpr (RAD == 4) {
        if (ns > 1) {
            v[1] = xmul(v[1], tw_get<INV>(tw, k * tstep));
            v[2] = xmul(v[2], tw_get<INV>(tw, 2 * k * tstep));
            v[3] = xmul(v[3], tw_get<INV>(tw, 3 * k * tstep));
        }
        xdft4<INV>(v[0], v[1], v[2], v[3]);
    } else if constexpr (RAD == 2) {
        if (ns > 1) v[1] = xmul(v[1], tw_get<INV>(tw, k * tstep));
        const float2 a = v[0], b = v[1];
        v[0] = xadd(a, b);
        v[1] = xsub(a, b);
    } else {
        static_assert(RAD == 3, "radix 8, 4, 2 or 3");
        if (ns > 1) {
            v[1] = xmul(v[1], tw_get<INV>(tw, k * tstep));
            v[2] = xmul(v[2], tw_get<INV>(tw, 2 * k * tstep));
        }
        const float hh = 0.866025403784438647f;
        const float2 t1 = xadd(v[1], v[2]);
        const float2 t2 = xsub(v[0], xscale(0.5f, t1));
        const float2 d = xscale(hh, xsub(v[1], v[2]));
        const float2 mid = INV ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
        v[0] = xadd(v[0], t1);
        v[1] = xadd(t2, mid);
        v[2] = xsub(t2, mid);
    }
}

// Stage S over the warp's NLW lines: butterfly b = lane + 32 t (b < NLW nb)
// is line b / nb, index j = b % nb.  ld(t, q, line, i) returns input element i,
// st(t, r, line, i, value) takes output element i.
template <int L, bool INV, int S, class Ld, class St>
__device__ __forceinline__ void wstage(Ld& ld, St& st, const float2* __restrict__ tw) {
    using P = WPlan<L>;
    constexpr int rad = P::rad(S), ns = P::ns(S), nb = L / rad, tstep = L / (ns * rad);
    constexpr int NBT = P::NLW * nb, NT = (NBT + 31) / 32;
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
        const int b = lane + 32 * t;
        if (NBT % 32 != 0 && b >= NBT) break;  // lanes without a butterfly in this round
        const int line = b / nb, j = b - line * nb;
        const int k = j % ns;
        const int out0 = (j / ns) * ns * rad + k;
        float2 v[rad];
#pragma unroll
        for (int q = 0; q < rad; ++q) v[q] = ld(t, q, line, j + q * nb);
        wbutterfly<rad, INV>(v, k, tstep, ns, tw);
#pragma unroll
        for (int r = 0; r < rad; ++r) st(t, r, line, out0 + r * ns, v[r]);
    }
}

// Line and element that a lane's (t, r) output of the last stage (and input
// of the first stage, q = r) refers to.
template <int L>
__device__ __forceinline__ void wlast_pos(int t, int r, int& line, int& i) {
    using P = WPlan<L>;
    constexpr int nb = L / P::R0;
    const int b = (threadIdx.x & 31) + 32 * t;
    line = b / nb;
    i = (b - line * nb) + r * nb;
}

// Transform of the warp's NLW lines.  Stage 0 reads through ld0, the last
// stage writes through stl, the stages between ping-pong in the warp's
// buffers a and b (lines of stride LS, elements at pad8(i)).  Ends with a
// __syncwarp, so the buffers may be reused at once.
template <int L, bool INV, int S = 0, class Ld, class St>
__device__ __forceinline__ void wfft(float2* a, float2* b, Ld& ld0, St& stl, const float2* __restrict__ tw) {
    using P = WPlan<L>;
    constexpr int n = P::nst();
    auto rd = [a](int, int, int line, int i) { return a[line * P::LS + pad8(i)]; };
    auto wr = [b](int, int, int line, int i, float2 v) { b[line * P::LS + pad8(i)] = v; };
    if constexpr (S == 0) {
        auto wa = [a](int, int, int line, int i, float2 v) { a[line * P::LS + pad8(i)] = v; };
        wstage<L, INV, 0>(ld0, wa, tw);
        __syncwarp();
        wfft<L, INV, 1>(a, b, ld0, stl, tw);
    } else if constexpr (S == n - 1) {
        wstage<L, INV, S>(rd, stl, tw);
        __syncwarp();
    } else {
        wstage<L, INV, S>(rd, wr, tw);
        __syncwarp();
        wfft<L, INV, S + 1>(b, a, ld0, stl, tw);
    }
}

// ---- CTA shapes ------------------------------------------------------------
// WPC warps per CTA.  Row passes: NRC = WPC * NLW rows per CTA.  Column pass:
// WPC * NLW columns per CTA.
template <int M, int WPC>
struct WRowCfg {
    using P = WPlan<M>;
    static constexpr int NRC = WPC * P::NLW;
    // Transposed row buffers ([kx][row]) with an odd row-group stride, so that
    // a warp reading one row across consecutive kx touches distinct banks.
    static constexpr int XS = NRC + 1;
    static constexpr size_t warp_bytes = sizeof(float2) * size_t(WPC) * 2 * P::WBUF;
    static constexpr size_t smem_r2c = warp_bytes + sizeof(float2) * size_t(M + 1) * XS;
    static constexpr size_t smem_c2r = warp_bytes + 2 * sizeof(float2) * size_t(M + 1) * XS;
};
template <int H, int WPC>
struct WColCfg {
    using P = WPlan<H>;
    static constexpr int NCC = WPC * P::NLW;
    static constexpr size_t smem = sizeof(float2) * size_t(WPC) * 2 * P::WBUF;
};

// ---- items -------------------------------------------------------------------

// NRC rows of one real plane x (width 2M) -> half spectra written transposed,
// Sc[kx][y] for kx <= M.  z[n] = x[2n] + i x[2n+1]; X[k] = (Z[k] + conj
// Z[M-k]) / 2 + e^{-2 pi i k / 2M} (Z[k] - conj Z[M-k]) / 2i.
// With COPY, every row value read is also written to xcopy at the same
// offset (the first stage reads each value of a row exactly once): a plane
// read from mapped host memory leaves its device copy behind.
template <int M, int WPC, bool COPY = false>
__device__ void r2c_rows_witem(float2* sm, const float* __restrict__ x, float2* __restrict__ Sc, int H, int y0,
                               const float2* __restrict__ twM, const float2* __restrict__ twW,
                               float* __restrict__ xcopy = nullptr) {
    using P = WPlan<M>;
    constexpr int NLW = P::NLW, LS = P::LS, Wc = M + 1, W = 2 * M, NRC = WRowCfg<M, WPC>::NRC;
    constexpr int XS = WRowCfg<M, WPC>::XS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float2* a = sm + warp * 2 * P::WBUF;
    float2* b = a + P::WBUF;
    float2* xs = sm + WPC * 2 * P::WBUF;  // [k][row of the CTA]
    const int row0 = warp * NLW;
    auto ld0 = [&](int, int, int line, int n) -> float2 {
        const int y = y0 + row0 + line;
        if (y >= H) return make_float2(0.f, 0.f);
        const size_t o = size_t(y) * W + 2 * n;
        const float2 v = *reinterpret_cast<const float2*>(x + o);
        if constexpr (COPY) *reinterpret_cast<float2*>(xcopy + o) = v;
        return v;
    };
    float2* z = ((P::nst() - 1) % 2 == 0) ? a : b;  // the buffer the last stage writes
    auto stz = [z](int, int, int line, int n, float2 v) { z[line * LS + pad8(n)] = v; };
    wfft<M, false>(a, b, ld0, stz, twM);
#pragma unroll 2
    for (int i = lane; i < NLW * Wc; i += 32) {
        const int line = i / Wc, k = i - line * Wc;
        const float2 zk = z[line * LS + pad8(k == M ? 0 : k)];
        const float2 zm = cconj(z[line * LS + pad8(k == 0 ? 0 : M - k)]);
        const float2 e = xscale(0.5f, xadd(zk, zm));
        const float2 d = xscale(0.5f, xsub(zk, zm));
        const float2 o = make_float2(d.y, -d.x);  // d / i
        xs[k * XS + row0 + line] = xadd(e, xmul(__ldg(twW + k), o));
    }
    __syncthreads();
    for (int i = threadIdx.x; i < Wc * NRC; i += 32 * WPC) {
        const int k = i / NRC, r = i - k * NRC;  // r fastest: NRC consecutive y per kx
        const int y = y0 + r;
        if (y < H) Sc[size_t(k) * H + y] = xs[k * XS + r];
    }
    __syncthreads();
}

// Column convolution of source slot `slot`: each warp takes NLW consecutive
// columns c0.. of the slot's spectrum (kx-major, columns of H contiguous),
// transforms them forward once (kept in registers), then for every kernel k
// in [k_begin, k_end) reading this slot (kernel order) multiplies by the
// kernel spectrum (scaled by 1/(W H)), transforms back and writes T[k].  (The
// kernel spectrum is read by the inverse transform's first stage straight
// from global memory: staging it in shared memory with cp.async during the
// forward transform was measured slower, 12.4 -> 14.3 us at 512x512.)
template <int H, int WPC>
__device__ void cols_witem(float2* sm, const float2* __restrict__ Sslot, const float2* __restrict__ KH,
                           float2* __restrict__ T, const int* __restrict__ slot_of_kernel, int k_begin, int k_end,
                           int slot, int Wc, int kx0, const float2* __restrict__ twH) {
    using P = WPlan<H>;
    const int warp = threadIdx.x >> 5;
    float2* a = sm + warp * 2 * P::WBUF;
    float2* b = a + P::WBUF;
    const int c0 = kx0 + warp * P::NLW;
    if (c0 >= Wc) return;  // no block-wide barrier in this item
    const int nl = min(P::NLW, Wc - c0);
    float2 F[P::NREG];
    auto ld0 = [&](int, int, int line, int i) -> float2 {
        return line < nl ? Sslot[size_t(c0 + line) * H + i] : make_float2(0.f, 0.f);
    };
    auto stF = [&F](int t, int r, int, int, float2 v) { F[t * P::R0 + r] = v; };
    wfft<H, false>(a, b, ld0, stF, twH);
    for (int k = k_begin; k < k_end; ++k) {
        if (slot_of_kernel[k] != slot) continue;
        const float2* kh = KH + size_t(k) * Wc * H;
        float2* out = T + size_t(k) * Wc * H;
        auto ldk = [&](int t, int q, int line, int i) -> float2 {
            return line < nl ? xmul(F[t * P::R0 + q], __ldg(kh + size_t(c0 + line) * H + i)) : make_float2(0.f, 0.f);
        };
        auto stT = [&](int, int, int line, int i, float2 v) {
            if (line < nl) out[size_t(c0 + line) * H + i] = v;
        };
        wfft<H, true>(a, b, ldk, stT, twH);
    }
}

// Plain column transforms of one slot's lines (columns of H, contiguous):
// forward and times `scale` (INV = false) or inverse (INV = true), from src to
// dst (which may be src: a warp reads all its lines before it writes them).
template <int H, int WPC, bool INV>
__device__ void cols_plain_witem(float2* sm, const float2* __restrict__ src, float2* __restrict__ dst, int nlines,
                                 int kx0, float scale, const float2* __restrict__ twH) {
    using P = WPlan<H>;
    const int warp = threadIdx.x >> 5;
    float2* a = sm + warp * 2 * P::WBUF;
    float2* b = a + P::WBUF;
    const int c0 = kx0 + warp * P::NLW;
    if (c0 >= nlines) return;
    const int nl = min(P::NLW, nlines - c0);
    auto ld0 = [&](int, int, int line, int i) -> float2 {
        return line < nl ? src[size_t(c0 + line) * H + i] : make_float2(0.f, 0.f);
    };
    auto st = [&](int, int, int line, int i, float2 v) {
        if (line < nl) dst[size_t(c0 + line) * H + i] = INV ? v : xscale(scale, v);
    };
    wfft<H, INV>(a, b, ld0, st, twH);
}

// NRC rows of target channel c: for each kernel targeting it (kernel order),
// the inverse real FFT of its spectrum rows T[k][kx][y] (prefetched into
// shared memory with cp.async during the previous kernel's transform), the
// growth G(u; mu, sigma) and the weighted sum, kept in registers; then the U
// rows.  Z[n] = (X[n] + conj X[M-n]) + i (X[n] - conj X[M-n]) e^{+2 pi i n / 2M}.
template <int M, int WPC>
__device__ void c2r_growth_witem(float2* sm, const float2* __restrict__ T, const KDesc* __restrict__ kd, int K, int c,
                                 float* __restrict__ Uc, int H, int y0, const float2* __restrict__ twM,
                                 const float2* __restrict__ twW) {
    using P = WPlan<M>;
    constexpr int NLW = P::NLW, Wc = M + 1, W = 2 * M, NRC = WRowCfg<M, WPC>::NRC, NT = 32 * WPC;
    constexpr int XS = WRowCfg<M, WPC>::XS;
    const int tid = threadIdx.x, warp = tid >> 5;
    float2* a = sm + warp * 2 * P::WBUF;
    float2* b = a + P::WBUF;
    float2* pre0 = sm + WPC * 2 * P::WBUF;  // [kx][row], two buffers
    float2* pre1 = pre0 + Wc * XS;
    const int row0 = warp * NLW;
    auto next = [&](int k) {
        for (++k; k < K; ++k)
            if (kd[k].tgt == c) break;
        return k;
    };
    auto prefetch = [&](int k, float2* dst) {
        const float2* t = T + size_t(k) * Wc * H;
        for (int i = tid; i < Wc * NRC; i += NT) {
            const int kk = i / NRC, r = i - kk * NRC;
            const int y = y0 + r;
            if (y < H) cp_async8(dst + kk * XS + r, t + size_t(kk) * H + y);
            else dst[kk * XS + r] = make_float2(0.f, 0.f);
        }
        cp_async_commit();
    };
    float u[2 * P::NREG];
#pragma unroll
    for (int i = 0; i < 2 * P::NREG; ++i) u[i] = 0.f;
    int kn = next(-1);
    if (kn < K) prefetch(kn, pre0);
    bool second = false;
    while (kn < K) {
        const KDesc d = kd[kn];
        cp_async_wait_all_groups();
        __syncthreads();  // this kernel's rows are in; every warp is done with the other buffer
        const float2* cur = second ? pre1 : pre0;
        const int knext = next(kn);
        if (knext < K) prefetch(knext, second ? pre0 : pre1);
        auto ld0 = [&](int, int, int line, int n) -> float2 {
            const int r = row0 + line;
            const float2 xk = cur[n * XS + r];
            const float2 xm = cconj(cur[(M - n) * XS + r]);
            const float2 e = xadd(xk, xm);
            const float2 o = xmul(xsub(xk, xm), cconj(__ldg(twW + n)));
            return make_float2(__fsub_rn(e.x, o.y), __fadd_rn(e.y, o.x));
        };
        auto grow = [&](int t, int r, int, int, float2 v) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const float conv = h ? v.y : v.x;
                const float diff = __fsub_rn(conv, d.mu);
                const float e = expf(__fmul_rn(__fmul_rn(-diff, diff), d.inv2s2));
                const float g = __fsub_rn(__fmul_rn(2.0f, e), 1.0f);
                float& acc = u[2 * (t * P::R0 + r) + h];
                acc = __fadd_rn(acc, __fmul_rn(d.weight, g));
            }
        };
        wfft<M, true>(a, b, ld0, grow, twM);
        kn = knext;
        second = !second;
    }
#pragma unroll
    for (int t = 0; t < P::NB0; ++t)
#pragma unroll
        for (int r = 0; r < P::R0; ++r) {
            int line, n;
            wlast_pos<M>(t, r, line, n);
            const int y = y0 + row0 + line;
            if (line < NLW && y < H)
                *reinterpret_cast<float2*>(Uc + size_t(y) * W + 2 * n) =
                    make_float2(u[2 * (t * P::R0 + r)], u[2 * (t * P::R0 + r) + 1]);
        }
    __syncthreads();  // the prefetch buffers are free for the CTA's next item
}

// NRC rows of one spectrum slot t ([kx][y]): inverse real FFT, times scale,
// written to (or, with accumulate, added to) the rows of `out`.  The same
// transform as the growth item's, without the growth.
template <int M, int WPC>
__device__ void c2r_raw_witem(float2* sm, const float2* __restrict__ t, float* __restrict__ out, int H, int y0,
                              float scale, bool accumulate, const float2* __restrict__ twM,
                              const float2* __restrict__ twW) {
    using P = WPlan<M>;
    constexpr int NLW = P::NLW, Wc = M + 1, W = 2 * M, NRC = WRowCfg<M, WPC>::NRC, NT = 32 * WPC;
    constexpr int XS = WRowCfg<M, WPC>::XS;
    const int tid = threadIdx.x, warp = tid >> 5;
    float2* a = sm + warp * 2 * P::WBUF;
    float2* b = a + P::WBUF;
    float2* cur = sm + WPC * 2 * P::WBUF;
    const int row0 = warp * NLW;
    for (int i = tid; i < Wc * NRC; i += NT) {
        const int kk = i / NRC, r = i - kk * NRC;
        const int y = y0 + r;
        cur[kk * XS + r] = y < H ? t[size_t(kk) * H + y] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    auto ld0 = [&](int, int, int line, int n) -> float2 {
        const int r = row0 + line;
        const float2 xk = cur[n * XS + r];
        const float2 xm = cconj(cur[(M - n) * XS + r]);
        const float2 e = xadd(xk, xm);
        const float2 o = xmul(xsub(xk, xm), cconj(__ldg(twW + n)));
        return make_float2(__fsub_rn(e.x, o.y), __fadd_rn(e.y, o.x));
    };
    auto st = [&](int, int, int line, int n, float2 v) {
        const int y = y0 + row0 + line;
        if (y >= H) return;
        float2* o = reinterpret_cast<float2*>(out + size_t(y) * W + 2 * n);
        float2 val = make_float2(__fmul_rn(v.x, scale), __fmul_rn(v.y, scale));
        if (accumulate) {
            const float2 old = *o;
            val = make_float2(__fadd_rn(old.x, val.x), __fadd_rn(old.y, val.y));
        }
        *o = val;
    };
    wfft<M, true>(a, b, ld0, st, twM);
    __syncthreads();
}

}  // namespace flp
